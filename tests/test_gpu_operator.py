"""GPU parity of the fermion operator, DSq and derived fields.

The CUDA path (through the C ABI) is compared with the numpy restatement of
the reference (oracle/susy_np.py) on identical seeded inputs.  Tolerances:
FP64 results within 1e-13 relative (max-norm) of the oracle; FP32 operator
within 1e-5 relative.
"""
import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import Lattice, SusyError
from susy_b200 import synth

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-13
FP32_TOL = 1e-5


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def setup(dims, N, pbc=-1, G=0.05, noise=0.2, seed=3):
    U = synth.links(dims, N, noise, seed)
    lat = Lattice(dims, N, pbc=pbc, lam=1.0, bmass=0.2, G=G)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, pbc)
    prm = O.Params(lam=1.0, bmass=0.2, G=G, N=N)
    der = O.compute_derived(geo, prm, U)
    return lat, geo, prm, U, der


CASES = [((4, 4, 4, 4), 2, -1, 0.05), ((4, 4, 4, 4), 3, -1, 0.05),
         ((2, 2, 2, 2), 2, -1, 0.05), ((4, 2, 4, 6), 3, 1, 0.05),
         ((6, 4, 4, 8), 2, -1, 0.0), ((4, 4, 4, 4), 4, -1, 0.1)]


@pytest.mark.parametrize("dims,N,pbc,G", CASES)
def test_derived_fields(dims, N, pbc, G):
    lat, geo, prm, U, der = setup(dims, N, pbc, G)
    pd, D, F, Ui = lat.derived()
    V = geo.V
    pd = pd.reshape(V, 5, 5, 2)
    pd = pd[..., 0] + 1j * pd[..., 1]
    pd = np.moveaxis(pd[geo.node_index()], 0, -1)
    mask = ~np.eye(5, dtype=bool)
    assert rel(pd[mask], der.plaqdet[mask]) < FP64_TOL
    assert rel(synth.from_ref(dims, D, 1, N)[0], der.DmuUmu) < FP64_TOL
    assert rel(synth.from_ref(dims, F, 10, N), der.Fmunu) < FP64_TOL
    assert rel(synth.from_ref(dims, Ui, 5, N), der.Uinv) < FP64_TOL


@pytest.mark.parametrize("dims,N,pbc,G", CASES)
@pytest.mark.parametrize("sign", [1, -1])
def test_fermion_op_fp64(dims, N, pbc, G, sign):
    lat, geo, prm, U, der = setup(dims, N, pbc, G)
    src = synth.tf_source(dims, N, seed=17)
    want = O.fermion_op(geo, prm, U, der, src, sign)
    out = np.zeros(lat.tf_doubles)
    lat.fermion_op(synth.to_ref(dims, src), out, sign)
    assert rel(synth.from_ref(dims, out, 16, N), want) < FP64_TOL


@pytest.mark.parametrize("dims,N,pbc,G", CASES[:4])
def test_dsq_fp64(dims, N, pbc, G):
    lat, geo, prm, U, der = setup(dims, N, pbc, G)
    src = synth.tf_source(dims, N, seed=5)
    want = O.DSq(geo, prm, U, der, src)
    out = np.zeros(lat.tf_doubles)
    lat.DSq(synth.to_ref(dims, src), out)
    assert rel(synth.from_ref(dims, out, 16, N), want) < FP64_TOL


def test_dsq_fmass():
    dims, N = (4, 4, 4, 4), 2
    U = synth.links(dims, N, 0.2, 1)
    lat = Lattice(dims, N, pbc=-1, fmass=0.3, G=0.05)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, -1)
    prm = O.Params(fmass=0.3, G=0.05, N=N)
    der = O.compute_derived(geo, prm, U)
    src = synth.tf_source(dims, N, seed=2)
    out = np.zeros(lat.tf_doubles)
    lat.DSq(synth.to_ref(dims, src), out)
    assert rel(synth.from_ref(dims, out, 16, N), O.DSq(geo, prm, U, der, src)) < FP64_TOL


@pytest.mark.parametrize("N", [2, 3])
def test_dsq_fp32_vs_fp64(N):
    dims = (4, 4, 4, 8)
    lat, geo, prm, U, der = setup(dims, N)
    src = synth.tf_source(dims, N, seed=9)
    a64, b64 = lat.tf(64), lat.tf(64)
    a32, b32 = lat.tf(32), lat.tf(32)
    a64.upload(synth.to_ref(dims, src))
    lat.dev_convert(a64, a32)
    lat.dev_DSq(a64, b64)
    lat.dev_DSq(a32, b32)
    r64 = b64.download()
    r32 = b32.download()
    want = O.DSq(geo, prm, U, der, src)
    assert rel(synth.from_ref(dims, r64, 16, N), want) < FP64_TOL
    assert rel(synth.from_ref(dims, r32, 16, N), want) < FP32_TOL


def test_bad_sign_raises():
    dims, N = (4, 4, 4, 4), 2
    lat = Lattice(dims, N)
    src = np.zeros(lat.tf_doubles)
    with pytest.raises(ValueError):
        lat.fermion_op(src, src.copy(), 0)
    # the C ABI itself rejects it too, with an error code instead of exiting
    rc = lat.lib.susy_b200_fermion_op(lat.h, src.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double)),
        src.ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)), 2)
    assert rc == -1


@pytest.mark.parametrize("dims,N,pbc", [((2, 2, 2, 6), 3, -1), ((4, 2, 2, 6), 2, -1),
                                        ((4, 2, 4, 6), 3, 1)])
def test_every_variant_where_warps_straddle_time_slices(dims, N, pbc):
    """With 8 or 16 sites per time slice a 32-site tile spans several time
    slices, boundary slices included, so the temporal BC sign of a product
    differs between the lanes of one warp.  Every kernel variant, D and
    D^dag, FP64 to 1e-13 and FP32 to 1e-5 against the oracle."""
    from susy_b200.lattice import FOP_NVARIANTS
    lat, geo, prm, U, der = setup(dims, N, pbc, 0.05)
    src = synth.tf_source(dims, N, seed=23)
    a, b = lat.tf(64), lat.tf(64)
    a32, b32 = lat.tf(32), lat.tf(32)
    a.upload(synth.to_ref(dims, src))
    lat.dev_convert(a, a32)
    for sign in (1, -1):
        want = O.fermion_op(geo, prm, U, der, src, sign)
        for v in range(FOP_NVARIANTS):
            lat.fop_variant(64, v)
            lat.fop_variant(32, v)
            lat.dev_fermion_op(a, b, sign)
            assert rel(synth.from_ref(dims, b.download(), 16, N), want) < FP64_TOL, (v, sign)
            lat.dev_fermion_op(a32, b32, sign)
            lat.dev_convert(b32, b)
            assert rel(synth.from_ref(dims, b.download(), 16, N), want) < FP32_TOL, (v, sign)


@pytest.mark.parametrize("N", [2, 3])
def test_links_and_momenta_in_place_with_a_site_stride(N):
    """The reference keeps link[5] and mom[5] inside its per-site struct
    (susy/lattice.h:29-59) and would hand &lattice[0].link[0] with stride
    sizeof(site).  Emulate that with a padded record per site (links and
    momenta at odd offsets inside a record much larger than them, bytes in
    between filled with a marker): set_links / set_mom read the strided
    fields, the operator matches the contiguous upload, and get_links /
    get_mom write back into the records without touching the bytes between
    them."""
    import ctypes as C
    dims = (4, 4, 2, 6)
    lat, geo, prm, U, der = setup(dims, N, -1, 0.05)
    V = lat.V
    m5 = 5 * N * N * 2                              # doubles in link[5]
    rec = 8 * (3 * m5 + 37)                         # bytes per site record
    off_link, off_mom = 8 * 11, 8 * (11 + m5 + 17)
    links = synth.to_ref(dims, U)
    mom = synth.to_ref(dims, synth.links(dims, N, 0.4, 12) - np.eye(N))
    buf = np.full(V * rec // 8, -7.25)
    view = buf.reshape(V, rec // 8)
    view[:, off_link // 8: off_link // 8 + m5] = links.reshape(V, m5)
    view[:, off_mom // 8: off_mom // 8 + m5] = mom.reshape(V, m5)
    dp = C.POINTER(C.c_double)
    base = buf.ctypes.data
    lib = lat.lib
    assert lib.susy_b200_set_links(lat.h, C.cast(base + off_link, dp), rec) == 0
    assert lib.susy_b200_set_mom(lat.h, C.cast(base + off_mom, dp), rec) == 0
    src = synth.tf_source(dims, N, seed=41)
    out = np.zeros(lat.tf_doubles)
    lat.fermion_op(synth.to_ref(dims, src), out, 1)
    want = O.fermion_op(geo, prm, U, der, src, 1)
    assert rel(synth.from_ref(dims, out, 16, N), want) < FP64_TOL
    assert np.array_equal(lat.get_mom(), mom)
    # write back into fresh records: the fields land in place, the rest stays
    back = np.full_like(buf, -7.25)
    assert lib.susy_b200_get_links(lat.h, C.cast(back.ctypes.data + off_link, dp), rec) == 0
    assert lib.susy_b200_get_mom(lat.h, C.cast(back.ctypes.data + off_mom, dp), rec) == 0
    assert np.array_equal(back, buf)


@pytest.mark.parametrize("N", [2, 3])
def test_rescaled_operator(N):
    """The reference's RESCALE option (eta doubled in and out of fermion_op,
    utilities.c:795,841): D, D^dag and DSq against the oracle with the same
    option, FP64 to 1e-13 and the FP32 operator to 1e-5, for every variant
    the option admits; clearing it restores the plain operator."""
    from susy_b200.lattice import FOP_NVARIANTS
    dims = (4, 2, 4, 6)
    lat, geo, prm, U, der = setup(dims, N, -1, 0.05)
    prm_r = O.Params(lam=1.0, bmass=0.2, G=0.05, N=N, rescale=True)
    src = synth.tf_source(dims, N, seed=29)
    assert lat.set_rescale(1) == 0
    out = np.zeros(lat.tf_doubles)
    a, b = lat.tf(64), lat.tf(64)
    a32, b32 = lat.tf(32), lat.tf(32)
    a.upload(synth.to_ref(dims, src))
    lat.dev_convert(a, a32)
    for v in range(3, FOP_NVARIANTS):
        lat.fop_variant(64, v)
        lat.fop_variant(32, v)
        for sign in (1, -1):
            want = O.fermion_op(geo, prm_r, U, der, src, sign)
            lat.fermion_op(synth.to_ref(dims, src), out, sign)
            assert rel(synth.from_ref(dims, out, 16, N), want) < FP64_TOL, (v, sign)
            lat.dev_fermion_op(a32, b32, sign)
            lat.dev_convert(b32, b)
            assert rel(synth.from_ref(dims, b.download(), 16, N), want) < FP32_TOL, (v, sign)
        lat.DSq(synth.to_ref(dims, src), out)
        assert rel(synth.from_ref(dims, out, 16, N), O.DSq(geo, prm_r, U, der, src)) < FP64_TOL
    assert lat.set_rescale(0) == 1
    lat.fermion_op(synth.to_ref(dims, src), out, 1)
    assert rel(synth.from_ref(dims, out, 16, N), O.fermion_op(geo, prm, U, der, src, 1)) < FP64_TOL
