"""Python mirror of the reference's hot-path interface over the C ABI.

The method names, argument meaning and error behaviour follow the reference
C functions (4d_Q16/susy/susy_includes.h:23-105): ``fermion_op(src, dest,
sign)``, ``DSq(src, dest)``, ``congrad_multi(src, psim, MaxCG, errormin)``,
``fermion_force``, ``gauge_force``, ``update_u``, ``update`` ...  Host arrays
are float64 in the reference's own memory layout (Twist_Fermion /
link-matrix arrays over sites in node_index order, see include/susy_b200.h).
Every call goes through ``libsusy_b200.so``; there is no CPU fallback: if
the library or a GPU is missing, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsusy_b200.so")

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


class SusyError(RuntimeError):
    """Raised when the CUDA library reports an error."""


class RHMCParams(C.Structure):
    """susy_b200_rhmc: rational approximation and integrator settings."""
    _fields_ = [("Nroot", C.c_int), ("Norder", C.c_int), ("amp4", _dp), ("shift4", _dp),
                ("amp8", _dp), ("shift8", _dp), ("ampdeg4", C.c_double),
                ("ampdeg8", C.c_double), ("nsteps", C.c_int * 2), ("traj_length", C.c_double),
                ("niter", C.c_int), ("rsqmin", C.c_double), ("solver", C.c_int),
                ("no_metropolis", C.c_int), ("algorithm", C.c_int), ("friction", C.c_double)]


class TrajResult(C.Structure):
    _fields_ = [("delta_S", C.c_double), ("start_S", C.c_double), ("end_S", C.c_double),
                ("xrandom", C.c_double), ("start_parts", C.c_double * 5),
                ("end_parts", C.c_double * 5), ("accept", C.c_int), ("iters", C.c_int),
                ("gnorm", C.c_double), ("max_gf", C.c_double), ("fnorm", C.c_double * 4),
                ("max_ff", C.c_double * 4)]


SOLVER_FP64 = 0
SOLVER_MIXED = 1
HMC = 0
SMD = 1
FOP_NVARIANTS = 15


class Meas(C.Structure):
    """susy_b200_meas: the measurements of control.c:85-138."""
    _fields_ = [("linktr", C.c_double * 5), ("linktr_ave", C.c_double),
                ("linktr_width", C.c_double), ("link_det", C.c_double * 5),
                ("det_ave", C.c_double), ("det_width", C.c_double),
                ("ploop_re", C.c_double), ("ploop_im", C.c_double), ("ploop_mod", C.c_double),
                ("ss_plaq", C.c_double), ("st_plaq", C.c_double),
                ("gauge_action", C.c_double),
                ("lines_re", C.c_double * 5), ("lines_im", C.c_double * 5),
                ("lines_polar_re", C.c_double * 5), ("lines_polar_im", C.c_double * 5),
                ("det_tot_re", C.c_double), ("det_tot_im", C.c_double),
                ("det_sq_re", C.c_double), ("det_sq_im", C.c_double), ("det_wsq", C.c_double),
                ("width_plaq", C.c_double), ("width_det_re", C.c_double),
                ("width_det_im", C.c_double),
                ("uubar_ave", C.c_double * 4), ("uubar_width", C.c_double * 4),
                ("uubar_min", C.c_double * 4), ("uubar_max", C.c_double * 4),
                ("polar_ave", C.c_double * 4), ("polar_width", C.c_double * 4),
                ("polar_min", C.c_double * 4), ("polar_max", C.c_double * 4)]


class RHMC:
    """Owns the coefficient arrays behind a RHMCParams structure."""

    def __init__(self, Norder=15, Nroot=1, nstep=5, nstep_gauge=4, traj_length=1.0,
                 niter=5000, error_per_site=1e-5, solver=SOLVER_FP64, tables=None,
                 no_metropolis=False, algorithm=HMC, friction=0.0):
        if tables is None:
            from .rhmc_tables import rhmc
            tables = rhmc(Norder, Nroot)
        self.t = {k: (np.ascontiguousarray(v, dtype=np.float64) if isinstance(v, list) else v)
                  for k, v in tables.items()}
        self.p = RHMCParams()
        self.p.Nroot = Nroot
        self.p.Norder = Norder
        for k in ("amp4", "shift4", "amp8", "shift8"):
            setattr(self.p, k, self.t[k].ctypes.data_as(_dp))
        self.p.ampdeg4 = self.t["ampdeg4"]
        self.p.ampdeg8 = self.t["ampdeg8"]
        self.p.nsteps[0] = nstep
        self.p.nsteps[1] = nstep_gauge
        self.p.traj_length = traj_length
        self.p.niter = niter
        self.p.rsqmin = error_per_site * error_per_site   # setup.c:356-359
        self.p.solver = solver
        self.p.no_metropolis = int(no_metropolis)
        self.p.algorithm = int(algorithm)
        self.p.friction = float(friction)


class Params(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nt", C.c_int),
                ("ncol", C.c_int), ("pbc", C.c_int), ("kappa", C.c_double),
                ("bmass", C.c_double), ("fmass", C.c_double), ("kappa_u1", C.c_double),
                ("G", C.c_double), ("iseed", C.c_int), ("device", C.c_int)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libsusy_b200.so and declare its C signatures (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SusyError("libsusy_b200.so not built: run `python -m susy_b200.build`")
    L = C.CDLL(path)
    L.susy_b200_create.restype = _vp
    L.susy_b200_create.argtypes = [C.POINTER(Params)]
    L.susy_b200_destroy.argtypes = [_vp]
    L.susy_b200_last_error.argtypes = [_vp]
    L.susy_b200_error_string.restype = C.c_char_p
    L.susy_b200_error_string.argtypes = [C.c_int]
    L.susy_b200_set_stream.argtypes = [_vp, _vp]
    L.susy_b200_get_stream.restype = _vp
    L.susy_b200_get_stream.argtypes = [_vp]
    L.susy_b200_sync.argtypes = [_vp]
    L.susy_b200_volume.argtypes = [_vp]
    L.susy_b200_launch_count.restype = C.c_longlong
    L.susy_b200_launch_count.argtypes = []
    for name in ("set_links", "get_links", "set_mom", "get_mom"):
        getattr(L, "susy_b200_" + name).argtypes = [_vp, _dp, C.c_size_t]
    for name in ("compute_plaqdet", "compute_Uinv", "compute_DmuUmu", "compute_Fmunu"):
        getattr(L, "susy_b200_" + name).argtypes = [_vp]
    L.susy_b200_get_derived.argtypes = [_vp, _dp, _dp, _dp, _dp]
    L.susy_b200_fermion_op.argtypes = [_vp, _dp, _dp, C.c_int]
    L.susy_b200_DSq.argtypes = [_vp, _dp, _dp]
    L.susy_b200_congrad_multi.argtypes = [_vp, _dp, C.POINTER(_dp), C.c_int, _dp, C.c_int,
                                          C.c_double, _dp]
    L.susy_b200_tf_alloc.restype = _vp
    L.susy_b200_tf_alloc.argtypes = [_vp, C.c_int]
    L.susy_b200_tf_free.argtypes = [_vp, _vp]
    L.susy_b200_tf_bytes.restype = C.c_size_t
    L.susy_b200_tf_bytes.argtypes = [_vp, C.c_int]
    L.susy_b200_tf_upload.argtypes = [_vp, _vp, C.c_int, _dp]
    L.susy_b200_tf_download.argtypes = [_vp, _vp, C.c_int, _dp]
    L.susy_b200_tf_convert.argtypes = [_vp, _vp, C.c_int, _vp, C.c_int]
    L.susy_b200_dev_fermion_op.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int]
    L.susy_b200_dev_DSq.argtypes = [_vp, _vp, _vp, C.c_int]
    L.susy_b200_autotune.argtypes = [_vp]
    L.susy_b200_fop_variant.argtypes = [_vp, C.c_int, C.c_int, C.POINTER(C.c_float)]
    L.susy_b200_measure.restype = C.c_int
    L.susy_b200_measure.argtypes = [_vp, C.POINTER(Meas)]
    L.susy_b200_plaquette.restype = C.c_int
    L.susy_b200_plaquette.argtypes = [_vp, _dp, _dp]
    L.susy_b200_mixed_params.restype = C.c_int
    L.susy_b200_mixed_params.argtypes = [_vp, C.c_double, C.c_double]
    L.susy_b200_mixed_reliable_interval.restype = C.c_int
    L.susy_b200_mixed_reliable_interval.argtypes = [_vp, C.c_int]
    L.susy_b200_mixed_correction.restype = C.c_int
    L.susy_b200_mixed_correction.argtypes = [_vp, C.c_int]
    L.susy_b200_set_solver.restype = C.c_int
    L.susy_b200_set_solver.argtypes = [_vp, C.c_int]
    L.susy_b200_use_graphs.restype = C.c_int
    L.susy_b200_use_graphs.argtypes = [_vp, C.c_int]
    L.susy_b200_pf_streams.restype = C.c_int
    L.susy_b200_pf_streams.argtypes = [_vp, C.c_int]
    L.susy_b200_cg_blocked.restype = C.c_int
    L.susy_b200_cg_blocked.argtypes = [_vp, C.c_int]
    L.susy_b200_set_rescale.restype = C.c_int
    L.susy_b200_set_rescale.argtypes = [_vp, C.c_int]
    L.susy_b200_mixed_vectors.restype = C.c_int
    L.susy_b200_mixed_vectors.argtypes = [_vp, C.c_int]
    L.susy_b200_cg_freeze_iterations.restype = C.c_int
    L.susy_b200_cg_freeze_iterations.argtypes = [_vp, C.POINTER(C.c_int), C.c_int]
    L.susy_b200_dev_congrad_multi.argtypes = [_vp, _vp, C.POINTER(_vp), C.c_int, _dp, C.c_int,
                                              C.c_double, _dp, C.POINTER(C.c_int)]
    L.susy_b200_dev_congrad_multi_mixed.argtypes = [_vp, _vp, C.POINTER(_vp), C.c_int, _dp,
                                                    C.c_int, C.c_double, _dp,
                                                    C.POINTER(C.c_int)]
    L.susy_b200_update_u.argtypes = [_vp, C.c_double]
    L.susy_b200_gauge_force.argtypes = [_vp, C.c_double, _dp]
    L.susy_b200_det_force.argtypes = [_vp, C.c_double, _dp]
    L.susy_b200_fermion_force.argtypes = [_vp, C.c_double, _dp, C.POINTER(_dp), C.c_int, _dp,
                                          _dp]
    L.susy_b200_dev_fermion_force.argtypes = [_vp, C.c_double, C.POINTER(_vp), C.c_int, _dp,
                                              _dp]
    L.susy_b200_action.argtypes = [_vp, C.c_int, C.POINTER(_dp), C.POINTER(_dp), C.c_int, _dp,
                                   C.c_double, _dp]
    L.susy_b200_seed.argtypes = [_vp, C.c_int]
    L.susy_b200_ranmom.argtypes = [_vp]
    L.susy_b200_update_batch.restype = C.c_int
    L.susy_b200_update_batch.argtypes = [C.POINTER(_vp), C.POINTER(C.POINTER(RHMCParams)),
                                         C.POINTER(TrajResult), C.c_int, C.c_int]
    L.susy_b200_dev_congrad_multi_batch.restype = C.c_int
    L.susy_b200_dev_congrad_multi_batch.argtypes = [
        C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.POINTER(_vp)), C.POINTER(C.c_int),
        C.POINTER(_dp), C.c_int, C.c_int, C.c_double, _dp, C.POINTER(C.c_int), _vp]
    L.susy_b200_DSq_batch.restype = C.c_int
    L.susy_b200_DSq_batch.argtypes = [C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.c_int,
                                      C.c_int, _vp]
    L.susy_b200_smdmom.restype = C.c_int
    L.susy_b200_smdmom.argtypes = [_vp, C.c_double, C.c_double]
    L.susy_b200_gaussian_tf.argtypes = [_vp, _dp]
    L.susy_b200_grsource.argtypes = [_vp, C.POINTER(RHMCParams), _dp]
    L.susy_b200_update.argtypes = [_vp, C.POINTER(RHMCParams), C.POINTER(TrajResult)]
    L.susy_b200_update_replay.argtypes = [_vp, C.POINTER(RHMCParams), C.POINTER(TrajResult),
                                          _dp, C.POINTER(_dp)]
    _lib = L
    return L


def launch_count() -> int:
    """Kernels launched by libsusy_b200.so so far in this process."""
    return int(load_library().susy_b200_launch_count())


def _ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


class DeviceTF:
    """A Twist_Fermion field resident on the GPU (FP64 or FP32)."""

    def __init__(self, lat: "Lattice", prec: int = 64):
        self.lat = lat
        self.prec = prec
        self.ptr = lat.lib.susy_b200_tf_alloc(lat.h, prec)
        if not self.ptr:
            lat._check(-3)

    def upload(self, host: np.ndarray):
        self.lat._check(self.lat.lib.susy_b200_tf_upload(self.lat.h, self.ptr, self.prec,
                                                         _ptr(host)))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.lat.tf_doubles)
        self.lat._check(self.lat.lib.susy_b200_tf_download(self.lat.h, self.ptr, self.prec,
                                                           _ptr(out)))
        return out

    def free(self):
        if self.ptr:
            self.lat.lib.susy_b200_tf_free(self.lat.h, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Lattice:
    """One lattice on one GPU, mirroring the reference's global-state API."""

    def __init__(self, dims, ncol, pbc=-1, lam=1.0, bmass=0.0, fmass=0.0, kappa_u1=0.0,
                 G=0.0, iseed=41, device=0):
        self.lib = load_library()
        nx, ny, nz, nt = dims
        self.dims = tuple(dims)
        self.N = ncol
        self.prm = Params(nx, ny, nz, nt, ncol, pbc, ncol * 0.25 / lam, bmass, fmass,
                          kappa_u1, G, iseed, device)
        self.lam = lam
        h = self.lib.susy_b200_create(C.byref(self.prm))
        if not h:
            raise SusyError("susy_b200_create failed (no GPU, bad parameters or out of memory)")
        self.h = h
        self.V = self.lib.susy_b200_volume(h)
        self.mat_doubles = 2 * ncol * ncol
        self.tf_doubles = self.V * 16 * self.mat_doubles
        self.link_doubles = self.V * 5 * self.mat_doubles

    def close(self):
        if getattr(self, "h", None):
            self.lib.susy_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc is not None and rc < 0:
            msg = self.lib.susy_b200_error_string(int(rc)).decode()
            raise SusyError("susy_b200 error %d: %s" % (rc, msg))
        return rc

    def set_stream(self, stream_ptr: int | None):
        self._check(self.lib.susy_b200_set_stream(self.h, stream_ptr))

    @property
    def stream(self) -> int:
        """The cudaStream_t (as an integer) the lattice launches on."""
        return int(self.lib.susy_b200_get_stream(self.h) or 0)

    def sync(self):
        self._check(self.lib.susy_b200_sync(self.h))

    # ---- fields ------------------------------------------------------------
    def set_links(self, links: np.ndarray):
        self._check(self.lib.susy_b200_set_links(self.h, _ptr(links), 0))

    def get_links(self) -> np.ndarray:
        out = np.zeros(self.link_doubles)
        self._check(self.lib.susy_b200_get_links(self.h, _ptr(out), 0))
        return out

    def set_mom(self, mom: np.ndarray):
        self._check(self.lib.susy_b200_set_mom(self.h, _ptr(mom), 0))

    def get_mom(self) -> np.ndarray:
        out = np.zeros(self.link_doubles)
        self._check(self.lib.susy_b200_get_mom(self.h, _ptr(out), 0))
        return out

    def compute_plaqdet(self):
        self._check(self.lib.susy_b200_compute_plaqdet(self.h))

    def compute_Uinv(self):
        self._check(self.lib.susy_b200_compute_Uinv(self.h))

    def compute_DmuUmu(self):
        self._check(self.lib.susy_b200_compute_DmuUmu(self.h))

    def compute_Fmunu(self):
        self._check(self.lib.susy_b200_compute_Fmunu(self.h))

    def derived(self):
        """(plaqdet [V*25*2], DmuUmu, Fmunu, Uinv) in reference order."""
        pd = np.zeros(self.V * 50)
        D = np.zeros(self.V * self.mat_doubles)
        F = np.zeros(self.V * 10 * self.mat_doubles)
        Ui = np.zeros(self.link_doubles)
        self._check(self.lib.susy_b200_get_derived(self.h, _ptr(pd), _ptr(D), _ptr(F), _ptr(Ui)))
        return pd, D, F, Ui

    # ---- operators ---------------------------------------------------------
    def fermion_op(self, src: np.ndarray, dest: np.ndarray, sign: int):
        """fermion_op(src, dest, sign), utilities.c:765; sign must be +-1."""
        if sign not in (1, -1):
            raise ValueError("Error: incorrect sign in fermion_op: %r" % (sign,))
        self._check(self.lib.susy_b200_fermion_op(self.h, _ptr(src), _ptr(dest), int(sign)))

    def DSq(self, src: np.ndarray, dest: np.ndarray):
        """DSq(src, dest) = (D^dag D + fmass^2) src, utilities.c:874."""
        self._check(self.lib.susy_b200_DSq(self.h, _ptr(src), _ptr(dest)))

    def congrad_multi(self, src: np.ndarray, psim, shift, MaxCG: int, errormin: float):
        """congrad_multi(src, psim, MaxCG, errormin, &size_r), congrad_multi.c:26.

        psim: list of Norder output arrays.  Returns (iterations, size_r).
        """
        shift = np.ascontiguousarray(shift, dtype=np.float64)
        n = len(shift)
        arr = (_dp * n)(*[_ptr(p) for p in psim])
        sr = C.c_double(0.0)
        it = self.lib.susy_b200_congrad_multi(self.h, _ptr(src), arr, n, _ptr(shift),
                                              int(MaxCG), float(errormin), C.byref(sr))
        self._check(it)
        return it, sr.value

    # ---- forces, link update, actions (update_h.c, update_o.c, action.c) ---
    def gauge_force(self, eps: float) -> float:
        n = C.c_double(0.0)
        self._check(self.lib.susy_b200_gauge_force(self.h, float(eps), C.byref(n)))
        return n.value

    def det_force(self, eps: float) -> float:
        n = C.c_double(0.0)
        self._check(self.lib.susy_b200_det_force(self.h, float(eps), C.byref(n)))
        return n.value

    def fermion_force(self, eps: float, src, sol, amp4) -> float:
        amp4 = np.ascontiguousarray(amp4, dtype=np.float64)
        arr = (_dp * len(sol))(*[_ptr(x) for x in sol])
        n = C.c_double(0.0)
        self._check(self.lib.susy_b200_fermion_force(self.h, float(eps),
                                                     None if src is None else _ptr(src), arr,
                                                     len(sol), _ptr(amp4), C.byref(n)))
        return n.value

    def update_u(self, eps: float):
        self._check(self.lib.susy_b200_update_u(self.h, float(eps)))

    def action(self, srcs=(), sols=(), amp4=None, ampdeg4=0.0):
        """(gauge, bmass, det, fermion, mom) as action.c:293 sums them."""
        parts = np.zeros(5)
        nroot = len(srcs)
        norder = len(sols[0]) if nroot else 0
        a = np.ascontiguousarray(amp4 if amp4 is not None else [0.0], dtype=np.float64)
        sarr = (_dp * max(nroot, 1))(*[_ptr(x) for x in srcs])
        flat = [x for row in sols for x in row]
        parr = (_dp * max(len(flat), 1))(*[_ptr(x) for x in flat])
        self._check(self.lib.susy_b200_action(self.h, nroot, sarr, parr, norder, _ptr(a),
                                              float(ampdeg4), _ptr(parts)))
        return parts

    # ---- random fields and the trajectory ---------------------------------
    def seed(self, iseed: int):
        self._check(self.lib.susy_b200_seed(self.h, int(iseed)))

    def ranmom(self):
        self._check(self.lib.susy_b200_ranmom(self.h))

    def smdmom(self, eps: float, friction: float):
        """smdmom(eps) (grsource.c:13): mom <- c1 mom + c2 gaussian"""
        self._check(self.lib.susy_b200_smdmom(self.h, float(eps), float(friction)))

    def gaussian_tf(self) -> np.ndarray:
        out = np.zeros(self.tf_doubles)
        self._check(self.lib.susy_b200_gaussian_tf(self.h, _ptr(out)))
        return out

    def grsource(self, rhmc: RHMC):
        out = np.zeros(self.tf_doubles)
        it = self._check(self.lib.susy_b200_grsource(self.h, C.byref(rhmc.p), _ptr(out)))
        return out, it

    @staticmethod
    def _traj(res: TrajResult) -> dict:
        return dict(delta_S=res.delta_S, start=res.start_S, end=res.end_S,
                    xrandom=res.xrandom, accept=bool(res.accept), iters=res.iters,
                    start_parts=list(res.start_parts), end_parts=list(res.end_parts),
                    gnorm=res.gnorm, max_gf=res.max_gf, fnorm=list(res.fnorm),
                    max_ff=list(res.max_ff))

    def update(self, rhmc: RHMC) -> dict:
        """One HMC trajectory, update_o.c:127."""
        res = TrajResult()
        self._check(self.lib.susy_b200_update(self.h, C.byref(rhmc.p), C.byref(res)))
        return self._traj(res)

    def update_replay(self, rhmc: RHMC, mom: np.ndarray | None, srcs) -> dict:
        res = TrajResult()
        arr = None
        if srcs is not None:
            arr = (_dp * len(srcs))(*[_ptr(x) for x in srcs])
        self._check(self.lib.susy_b200_update_replay(self.h, C.byref(rhmc.p), C.byref(res),
                                                     None if mom is None else _ptr(mom), arr))
        return self._traj(res)

    # ---- operator kernel selection -----------------------------------------
    def autotune(self):
        self._check(self.lib.susy_b200_autotune(self.h))

    def mixed_params(self, fp32_below: float = 3e-4, reliable_factor: float = 1e-2):
        """Mixed solver: FP32 operator once |r| < fp32_below |src|; FP64
        residual replacement whenever |r| fell by reliable_factor."""
        self._check(self.lib.susy_b200_mixed_params(self.h, float(fp32_below),
                                                    float(reliable_factor)))

    def mixed_reliable_interval(self, iters: int = 0):
        """Mixed solver: FP64 residual replacement every iters iterations
        (rounded up to a block boundary) instead of the reliable_factor
        trigger; 0 restores the trigger."""
        self._check(self.lib.susy_b200_mixed_reliable_interval(self.h, int(iters)))

    def mixed_correction(self, fp32: bool = True):
        """Mixed solver: per-shift correction solves with the FP32 operator
        (iterative refinement against the FP64 true residual) or in FP64."""
        self._check(self.lib.susy_b200_mixed_correction(self.h, 1 if fp32 else 0))

    def set_rescale(self, on: int = -1) -> int:
        """The reference's RESCALE option (the site component of the
        operator's input and output doubled); returns the previous setting."""
        return self._check(self.lib.susy_b200_set_rescale(self.h, int(on)))

    def mixed_vectors(self, fp32: int = -1) -> int:
        """Mixed solver: FP32 (1) or FP64 (0) ring and search vectors in its
        FP32-operator phase; returns the previous setting."""
        return self._check(self.lib.susy_b200_mixed_vectors(self.h, int(fp32)))

    def measure(self) -> dict:
        """Measurements of control.c:85-138 on the current links, keyed as
        the oracle's measurements()."""
        m = Meas()
        self._check(self.lib.susy_b200_measure(self.h, C.byref(m)))
        n = self.N
        a = lambda x, k=5: np.array(list(x)[:k])
        return {"linktr": a(m.linktr), "linktr_ave": m.linktr_ave,
                "linktr_width": m.linktr_width, "link_det": a(m.link_det),
                "det_ave": m.det_ave, "det_width": m.det_width,
                "ploop_re": m.ploop_re, "ploop_im": m.ploop_im, "ploop_mod": m.ploop_mod,
                "ss_plaq": m.ss_plaq, "st_plaq": m.st_plaq, "gauge_action": m.gauge_action,
                "lines": a(m.lines_re) + 1j * a(m.lines_im),
                "lines_polar": a(m.lines_polar_re) + 1j * a(m.lines_polar_im),
                "det": np.array([m.det_tot_re, m.det_tot_im, m.det_sq_re, m.det_sq_im,
                                 m.det_wsq]),
                "widths": np.array([m.width_plaq, m.width_det_re, m.width_det_im]),
                "uubar": (a(m.uubar_ave, n), a(m.uubar_width, n), a(m.uubar_min, n),
                          a(m.uubar_max, n)),
                "polar": (a(m.polar_ave, n), a(m.polar_width, n), a(m.polar_min, n),
                          a(m.polar_max, n))}

    def plaquette(self):
        """(ss_plaq, st_plaq), plaq.c:7"""
        ss, st = C.c_double(), C.c_double()
        self._check(self.lib.susy_b200_plaquette(self.h, C.byref(ss), C.byref(st)))
        return ss.value, st.value

    def set_solver(self, solver: int) -> int:
        """Solver behind congrad_multi (SOLVER_FP64 or SOLVER_MIXED)."""
        return self._check(self.lib.susy_b200_set_solver(self.h, int(solver)))

    def use_graphs(self, on: int = -1) -> int:
        """CUDA-graph replay (1) or plain launches (0) of the solver's
        iteration chunks; returns the previous setting."""
        return self._check(self.lib.susy_b200_use_graphs(self.h, int(on)))

    def pf_streams(self, on: int = -1) -> int:
        """Overlap the pseudofermion solves of a trajectory on two streams
        (1) or solve them in turn (0); returns the previous setting."""
        return self._check(self.lib.susy_b200_pf_streams(self.h, int(on)))

    def cg_blocked(self, on: int = -1) -> int:
        """Blocked (1) or per-iteration (0) vector update of the FP64
        multi-shift CG; returns the previous setting (on < 0 only queries)."""
        return self._check(self.lib.susy_b200_cg_blocked(self.h, int(on)))

    def cg_freeze_iterations(self, norder: int) -> list:
        """Iteration at which each shift of the last multi-shift solve froze
        (the solve's iteration count for the base shift)."""
        out = (C.c_int * norder)()
        self._check(self.lib.susy_b200_cg_freeze_iterations(self.h, out, int(norder)))
        return list(out)

    def fop_variant(self, prec: int = 64, set_to: int = -1):
        """(current variant, autotuner ms per variant) for one precision."""
        ms = (C.c_float * FOP_NVARIANTS)()
        v = self._check(self.lib.susy_b200_fop_variant(self.h, prec, set_to, ms))
        return v, [ms[i] for i in range(FOP_NVARIANTS)]

    # ---- device-resident variants -----------------------------------------
    def tf(self, prec: int = 64) -> DeviceTF:
        return DeviceTF(self, prec)

    def dev_fermion_op(self, src: DeviceTF, dst: DeviceTF, sign: int):
        self._check(self.lib.susy_b200_dev_fermion_op(self.h, src.ptr, dst.ptr, int(sign),
                                                      src.prec))

    def dev_DSq(self, src: DeviceTF, dst: DeviceTF):
        self._check(self.lib.susy_b200_dev_DSq(self.h, src.ptr, dst.ptr, src.prec))

    def dev_convert(self, src: DeviceTF, dst: DeviceTF):
        self._check(self.lib.susy_b200_tf_convert(self.h, src.ptr, src.prec, dst.ptr, dst.prec))

    def dev_congrad_multi(self, src: DeviceTF, psim, shift, MaxCG: int, errormin: float,
                          mixed: bool = False):
        """Solve on device fields; mixed=True uses the mixed-precision solver."""
        shift = np.ascontiguousarray(shift, dtype=np.float64)
        n = len(shift)
        arr = (_vp * n)(*[p.ptr for p in psim])
        sr = C.c_double(0.0)
        it = C.c_int(0)
        fn = (self.lib.susy_b200_dev_congrad_multi_mixed if mixed
              else self.lib.susy_b200_dev_congrad_multi)
        self._check(fn(self.h, src.ptr, arr, n, _ptr(shift), int(MaxCG), float(errormin),
                       C.byref(sr), C.byref(it)))
        return it.value, sr.value


def update_batch(lattices, rhmcs, threads: int = 8):
    """One trajectory on each lattice, concurrently (susy_b200_update_batch):
    a list of the dicts Lattice.update returns."""
    n = len(lattices)
    assert len(rhmcs) == n and n > 0
    lib = lattices[0].lib
    hs = (_vp * n)(*[lat.h for lat in lattices])
    rs = (C.POINTER(RHMCParams) * n)(*[C.pointer(r.p) for r in rhmcs])
    res = (TrajResult * n)()
    rc = lib.susy_b200_update_batch(hs, rs, res, n, int(threads))
    if rc < 0:
        lattices[0]._check(rc)
    return [lat._traj(res[i]) for i, lat in enumerate(lattices)]


def dsq_batch(srcs, dsts, stream_ptr: int | None = None):
    """dst[i] = (D^dag D + fmass^2) src[i] on each DeviceTF's lattice, all
    lattices in two launches (susy_b200_DSq_batch); one NCOL and precision."""
    n = len(srcs)
    assert len(dsts) == n and n > 0
    lats = [s.lat for s in srcs]
    assert all(d.lat is l for d, l in zip(dsts, lats))
    prec = srcs[0].prec
    assert all(x.prec == prec for x in list(srcs) + list(dsts))
    lib = lats[0].lib
    hs = (_vp * n)(*[lat.h for lat in lats])
    sp = (_vp * n)(*[x.ptr for x in srcs])
    dp = (_vp * n)(*[x.ptr for x in dsts])
    lats[0]._check(lib.susy_b200_DSq_batch(hs, sp, dp, n, int(prec), stream_ptr))


def congrad_multi_batch(srcs, psims, shifts, MaxCG: int, errormin: float,
                        stream_ptr: int | None = None):
    """congrad_multi on several lattices at once (FP64 device fields,
    susy_b200_dev_congrad_multi_batch): srcs[i] is lattice i's source,
    psims[i] its solutions (one DeviceTF per shift), shifts[i] its shifts.
    Returns the per-lattice iteration counts and final |r|^2."""
    n = len(srcs)
    assert len(psims) == n and len(shifts) == n and n > 0
    lats = [x.lat for x in srcs]
    lib = lats[0].lib
    hs = (_vp * n)(*[lat.h for lat in lats])
    sp = (_vp * n)(*[x.ptr for x in srcs])
    rows = [(_vp * len(p))(*[x.ptr for x in p]) for p in psims]
    pp = (C.POINTER(_vp) * n)(*[C.cast(r, C.POINTER(_vp)) for r in rows])
    norder = (C.c_int * n)(*[len(p) for p in psims])
    sh = [np.ascontiguousarray(x, dtype=np.float64) for x in shifts]
    shp = (_dp * n)(*[_ptr(a) for a in sh])
    size_r = (C.c_double * n)()
    iters = (C.c_int * n)()
    lats[0]._check(lib.susy_b200_dev_congrad_multi_batch(
        hs, sp, pp, norder, shp, n, int(MaxCG), float(errormin), size_r, iters, stream_ptr))
    return list(iters), list(size_r)
