"""The C-ABI library loads and exports every entry point include/*.h declares.

CPU only: no compute call is made (there is no GPU here); creating a lattice
without a GPU must fail cleanly with NULL, never crash.
"""
import ctypes as C
import glob
import os
import re

import pytest

from susy_b200 import lattice as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(susy_b200_[A-Za-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("susy_b200_fermion_op", "susy_b200_DSq", "susy_b200_congrad_multi",
                 "susy_b200_fermion_force", "susy_b200_gauge_force", "susy_b200_det_force",
                 "susy_b200_update_u", "susy_b200_update", "susy_b200_action",
                 "susy_b200_compute_plaqdet", "susy_b200_compute_Uinv",
                 "susy_b200_compute_DmuUmu", "susy_b200_compute_Fmunu",
                 "susy_b200_ranmom", "susy_b200_grsource"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = L.load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_error_strings_and_null_handles():
    lib = L.load_library()
    assert lib.susy_b200_error_string(0) == b"ok"
    assert lib.susy_b200_error_string(-1) == b"invalid argument"
    assert lib.susy_b200_last_error(None) == -1
    assert lib.susy_b200_fermion_op(None, None, None, 1) == -1
    assert lib.susy_b200_get_stream(None) is None
    # solver settings refuse a missing handle before touching the device
    for name, arg in (("susy_b200_pf_streams", 1), ("susy_b200_mixed_correction", 1),
                      ("susy_b200_use_graphs", 1), ("susy_b200_cg_blocked", 1),
                      ("susy_b200_mixed_reliable_interval", 50)):
        f = getattr(lib, name)
        f.restype = C.c_int
        assert f(None, arg) == -1, name


def test_create_rejects_bad_geometry_without_gpu_work():
    lib = L.load_library()
    p = L.Params(5, 4, 4, 4, 2, -1, 0.5, 0, 0, 0, 0, 41, 0)   # odd nx
    assert not lib.susy_b200_create(C.byref(p))
    p = L.Params(4, 4, 4, 4, 7, -1, 0.5, 0, 0, 0, 0, 41, 0)   # NCOL 7
    assert not lib.susy_b200_create(C.byref(p))
    p = L.Params(4, 4, 4, 4, 2, 0, 0.5, 0, 0, 0, 0, 41, 0)    # PBC 0
    assert not lib.susy_b200_create(C.byref(p))


def test_lattice_without_gpu_raises_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(L.SusyError):
        L.Lattice((4, 4, 4, 4), 2)


def test_create_rejects_extents_whose_volume_overflows_int():
    """Extents whose product wraps a 32-bit int are refused before anything
    is sized from them (the wrapped value could look small)."""
    lib = L.load_library()
    for dims in ((2, 2, 2048, 524290), (65536, 65536, 2, 2), (1 << 30, 2, 2, 2)):
        p = L.Params(*dims, 2, -1, 0.5, 0, 0, 0, 0, 41, 0)
        assert not lib.susy_b200_create(C.byref(p)), dims


def test_noalloc_refuses_overflowing_extents_before_any_device_work():
    lib = L.load_library()
    f = lib.susy_b200_DSq_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int] * 6 + [C.c_double, C.c_double] + [C.c_void_p] * 6
    # 2 x 2 x 2048 x 524290 wraps to 16384 sites in int arithmetic
    for dims in ((2, 2, 2048, 524290), (65536, 65536, 2, 2), (46342, 46342, 2, 2)):
        assert f(*dims, 2, -1, 0.0, 0.0, None, None, None, None, None, None) == -6, dims
    # malformed extents stay invalid arguments
    assert f(2, 2, 2047, 4, 2, -1, 0.0, 0.0, None, None, None, None, None, None) == -1
    assert f(-2, 2, 2, 4, 2, -1, 0.0, 0.0, None, None, None, None, None, None) == -1


def test_batch_dsq_refuses_bad_arguments_before_any_device_work():
    """susy_b200_DSq_batch checks its arguments before touching a handle or
    the device: NULL arrays or entries, n outside 1..SUSY_B200_BATCH_MAX and
    a precision other than 64 / 32 return SUSY_B200_EINVAL (-1)."""
    lib = L.load_library()
    f = lib.susy_b200_DSq_batch
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_void_p)] * 3 + [C.c_int, C.c_int, C.c_void_p]
    hdr = open(os.path.join(ROOT, "include", "susy_b200.h")).read()
    nmax = int(re.search(r"#define SUSY_B200_BATCH_MAX (\d+)", hdr).group(1))
    null3 = (C.c_void_p * 3)()
    assert f(None, None, None, 1, 64, None) == -1
    assert f(null3, null3, null3, 1, 64, None) == -1      # NULL handle
    assert f(null3, null3, null3, 0, 64, None) == -1
    big = (C.c_void_p * (nmax + 1))()
    assert f(big, big, big, nmax + 1, 64, None) == -1
    assert f(null3, null3, null3, 1, 16, None) == -1


def test_batch_solve_refuses_bad_arguments_before_any_device_work():
    """susy_b200_dev_congrad_multi_batch checks its arguments before it
    touches a handle or the device: NULL arrays or handles and n outside
    1..SUSY_B200_BATCH_MAX return SUSY_B200_EINVAL (-1)."""
    lib = L.load_library()
    f = lib.susy_b200_dev_congrad_multi_batch
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                  C.POINTER(C.POINTER(C.c_void_p)), C.POINTER(C.c_int),
                  C.POINTER(C.POINTER(C.c_double)), C.c_int, C.c_int, C.c_double,
                  C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p]
    null = (C.c_void_p * 2)()
    rows = (C.POINTER(C.c_void_p) * 2)()
    norder = (C.c_int * 2)(1, 1)
    shifts = (C.POINTER(C.c_double) * 2)()
    assert f(None, None, None, None, None, 1, 10, 1e-16, None, None, None) == -1
    assert f(null, null, rows, norder, shifts, 1, 10, 1e-16, None, None, None) == -1
    assert f(null, null, rows, norder, shifts, 0, 10, 1e-16, None, None, None) == -1
    assert f(null, null, rows, norder, shifts, 65, 10, 1e-16, None, None, None) == -1
