"""susy_b200_DSq_noalloc against the regular DSq entry point (GPU).

The no-allocation entry point serves callers that own every device buffer
themselves and cannot let a library call cudaMalloc (an application with its
own device memory pool, or code that must not risk the synchronisation an
allocation can cause).  This test owns all device memory through torch,
hands plain device pointers to the entry point and checks two calls in a row
(the second reusing the library's fixed scratch array after the first left
its contents there) against the handle-based susy_b200_DSq, to the FP64
operator tolerance used throughout the tests (1e-13 relative, max-norm).
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import Lattice, synth
from susy_b200.lattice import load_library

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-13


def device_layout(field):
    """[K, V, N, N] complex (lexicographic) -> [K][N][N][S] complex128, S padded."""
    K, V, N, _ = field.shape
    S = (V + 31) // 32 * 32
    out = np.zeros((K, N, N, S), dtype=np.complex128)
    out[..., :V] = np.transpose(field, (0, 2, 3, 1))
    return out


def from_device_layout(arr, V):
    """[K][N][N][S] complex128 -> [K, V, N, N]."""
    return np.ascontiguousarray(np.transpose(arr[..., :V], (0, 3, 1, 2)))


def to_gpu(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).cuda()


def noalloc_fn():
    lib = load_library()
    f = lib.susy_b200_DSq_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int] * 6 + [C.c_double, C.c_double] + [C.c_void_p] * 6
    return f


@pytest.mark.parametrize("dims,N,G,fmass", [((4, 4, 4, 8), 2, 0.05, 0.0),
                                            ((4, 4, 2, 4), 3, 0.05, 0.3),
                                            ((8, 8, 8, 8), 4, 0.0, 0.0)])
def test_noalloc_matches_regular_dsq_on_two_calls(dims, N, G, fmass):
    import torch
    f = noalloc_fn()
    U = synth.links(dims, N, 0.2, 5)
    lat = Lattice(dims, N, pbc=-1, G=G, fmass=fmass)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, -1)
    der = O.compute_derived(geo, O.Params(G=G, N=N), U)
    V = geo.V
    d_links = to_gpu(device_layout(U))
    d_uinv = to_gpu(device_layout(der.Uinv))
    pd = der.plaqdet.reshape(25, 1, 1, V)
    d_pd = to_gpu(device_layout(np.moveaxis(pd, 3, 1)))
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (11, 12):
        src = synth.tf_source(dims, N, seed)
        want = np.zeros(lat.tf_doubles)
        lat.DSq(synth.to_ref(dims, src), want)
        d_src = to_gpu(device_layout(src))
        d_dst = torch.full_like(d_src, float("nan"))
        rc = f(*dims, N, -1, G, fmass, d_links.data_ptr(), d_uinv.data_ptr(), d_pd.data_ptr(),
               d_src.data_ptr(), d_dst.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = d_dst.cpu().numpy().view(np.complex128).reshape(16, N, N, -1)
        got = synth.to_ref(dims, from_device_layout(got, V))
        assert np.abs(got - want).max() / np.abs(want).max() < FP64_TOL


def test_noalloc_rejects_lattices_beyond_its_scratch():
    f = noalloc_fn()
    lib = load_library()
    # 16 x 9 x 8^3 x 16 complex doubles > 2^20: refused before any pointer is used
    rc = f(8, 8, 8, 16, 3, -1, 0.0, 0.0, None, None, None, None, None, None)
    assert rc == -6
    assert b"scratch" in lib.susy_b200_error_string(rc)
    assert f(8, 8, 8, 8, 5, -1, 0.0, 0.0, None, None, None, None, None, None) == -1
