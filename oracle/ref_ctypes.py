"""ctypes access to the reference CPU code built under oracle/_ref/.

TEST INFRASTRUCTURE ONLY (see oracle/ref_harness.c).  The reference keeps
one lattice per process in globals, so each ``RefLattice`` must live in its
own process: use :func:`run_in_fresh_process`.
"""
from __future__ import annotations

import ctypes as C
import multiprocessing as mp
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)


def lib_path(ncol: int, smd: bool = False) -> str:
    return os.path.join(REF_DIR, "libsusyref_n%d%s.so" % (ncol, "_smd" if smd else ""))


def available(ncol: int, smd: bool = False) -> bool:
    return os.path.exists(lib_path(ncol, smd))


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def input_text(dims, pbc=-1, iseed=41, Nroot=1, Norder=15, traj_length=1.0,
               nstep=5, nstep_gauge=4, lam=1.0, kappa_u1=0.0, bmass=0.0,
               fmass=0.0, G=0.0, max_cg=5000, error_per_site=1e-5, friction=None):
    """Key/value input in the order setup.c:43-54,320-420 reads it
    (friction, setup.c:160-162, only for the SMD build)."""
    nx, ny, nz, nt = dims
    return "\n".join([
        "prompt 0", "nx %d" % nx, "ny %d" % ny, "nz %d" % nz, "nt %d" % nt,
        "PBC %d" % pbc, "iseed %d" % iseed, "Nroot %d" % Nroot,
        "Norder %d" % Norder, "warms 0", "trajecs 1",
        "traj_length %.17g" % traj_length] +
        (["friction %.17g" % friction] if friction is not None else []) + [
        "nstep %d" % nstep,
        "nstep_gauge %d" % nstep_gauge, "traj_between_meas 1",
        "lambda %.17g" % lam, "kappa_u1 %.17g" % kappa_u1,
        "bmass %.17g" % bmass, "fmass %.17g" % fmass, "G %.17g" % G,
        "max_cg_iterations %d" % max_cg,
        "error_per_site %.17g" % error_per_site, "fresh", "forget", ""])


class RefLattice:
    """One reference lattice in this process."""

    def __init__(self, ncol: int, quiet=True, smd=False, **params):
        self.ncol = ncol
        self.lib = C.CDLL(lib_path(ncol, smd))
        L = self.lib
        for name in ("ref_gauge_force", "ref_det_force", "ref_fermion_force",
                     "ref_update_gauge_step"):
            getattr(L, name).restype = C.c_double
        L.ref_gauge_force.argtypes = [C.c_double]
        L.ref_det_force.argtypes = [C.c_double]
        L.ref_update_u.argtypes = [C.c_double]
        L.ref_update_gauge_step.argtypes = [C.c_double]
        L.ref_fermion_force.argtypes = [C.c_double, _dp, _dp]
        self.quiet = quiet
        fd, path = tempfile.mkstemp(suffix=".in")
        with os.fdopen(fd, "w") as f:
            f.write(input_text(**params))
        self._logfd, self.log_path = tempfile.mkstemp(suffix=".log")
        os.close(self._logfd)
        if quiet:
            L.ref_redirect_stdout(self.log_path.encode())
        V = L.ref_init(path.encode())
        os.unlink(path)
        if V <= 0:
            raise RuntimeError("reference set-up failed: %d" % V)
        self.V = V
        self.tfd = L.ref_tf_doubles()
        self.md = 2 * ncol * ncol
        co = np.zeros(4 * V, dtype=np.int32)
        L.ref_site_coords(co.ctypes.data_as(C.POINTER(C.c_int)))
        self.coords = co.reshape(V, 4)
        prm = np.zeros(16)
        L.ref_params(_ptr(prm))
        self.params = prm

    def log(self) -> str:
        self.lib.ref_redirect_stdout(b"")
        with open(self.log_path) as f:
            txt = f.read()
        if self.quiet:
            self.lib.ref_redirect_stdout(self.log_path.encode())
        return txt

    # fields ---------------------------------------------------------------
    def links(self):
        out = np.zeros(self.V * 5 * self.md)
        self.lib.ref_get_links(_ptr(out))
        return out

    def set_links(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.float64)
        self.lib.ref_set_links(_ptr(flat))

    def mom(self):
        out = np.zeros(self.V * 5 * self.md)
        self.lib.ref_get_mom(_ptr(out))
        return out

    def set_mom(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.float64)
        self.lib.ref_set_mom(_ptr(flat))

    def compute_all(self):
        self.lib.ref_compute_all()

    def plaqdet(self):
        out = np.zeros(self.V * 25 * 2)
        self.lib.ref_get_plaqdet(_ptr(out))
        return out

    def DmuUmu(self):
        out = np.zeros(self.V * self.md)
        self.lib.ref_get_DmuUmu(_ptr(out))
        return out

    def Fmunu(self):
        out = np.zeros(self.V * 10 * self.md)
        self.lib.ref_get_Fmunu(_ptr(out))
        return out

    def Uinv(self):
        out = np.zeros(self.V * 5 * self.md)
        self.lib.ref_get_Uinv(_ptr(out))
        return out

    def site_prn(self):
        out = np.zeros(self.V * 10, dtype=np.uint64)
        self.lib.ref_site_prn(out.ctypes.data_as(C.POINTER(C.c_ulong)))
        return out.reshape(self.V, 10)

    def node_prn(self):
        out = np.zeros(10, dtype=np.uint64)
        self.lib.ref_node_prn(out.ctypes.data_as(C.POINTER(C.c_ulong)))
        return out

    def rhmc(self):
        n = 32
        a4, s4, a8, s8 = (np.zeros(n) for _ in range(4))
        degs = np.zeros(2)
        k = self.lib.ref_rhmc(_ptr(a4), _ptr(s4), _ptr(a8), _ptr(s8), _ptr(degs))
        return dict(amp4=a4[:k].copy(), shift4=s4[:k].copy(), amp8=a8[:k].copy(),
                    shift8=s8[:k].copy(), ampdeg4=degs[0], ampdeg8=degs[1])

    # operators --------------------------------------------------------------
    def fermion_op(self, src, sign):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.zeros_like(src)
        self.lib.ref_fermion_op(_ptr(src), _ptr(out), int(sign))
        return out

    def DSq(self, src):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.zeros_like(src)
        self.lib.ref_DSq(_ptr(src), _ptr(out))
        return out

    def congrad_multi(self, src, shifts, MaxCG, errormin):
        src = np.ascontiguousarray(src, dtype=np.float64)
        shifts = np.ascontiguousarray(shifts, dtype=np.float64)
        psim = np.zeros(len(shifts) * src.size)
        sr = C.c_double(0.0)
        tot = C.c_int(0)
        self.lib.ref_congrad_multi.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_double,
                                               C.POINTER(C.c_double),
                                               C.POINTER(C.c_int)]
        it = self.lib.ref_congrad_multi(_ptr(src), _ptr(psim), _ptr(shifts), len(shifts),
                                        int(MaxCG), float(errormin),
                                        C.byref(sr), C.byref(tot))
        if it < 0:
            raise ValueError("congrad_multi: %d shifts, the setup has fewer" % len(shifts))
        return psim.reshape(len(shifts), -1), it, sr.value

    def fermion_force(self, eps, src, sol):
        src = np.ascontiguousarray(src, dtype=np.float64)
        sol = np.ascontiguousarray(sol, dtype=np.float64).reshape(-1)
        return self.lib.ref_fermion_force(float(eps), _ptr(src), _ptr(sol))

    def gauge_force(self, eps):
        return self.lib.ref_gauge_force(float(eps))

    def det_force(self, eps):
        return self.lib.ref_det_force(float(eps))

    def update_u(self, eps):
        self.lib.ref_update_u(float(eps))

    def action_parts(self, src=None, sol=None):
        out = np.zeros(5)
        if src is None:
            self.lib.ref_action_parts(None, None, _ptr(out))
        else:
            src = np.ascontiguousarray(src, dtype=np.float64)
            sol = np.ascontiguousarray(sol, dtype=np.float64).reshape(-1)
            self.lib.ref_action_parts(_ptr(src), _ptr(sol), _ptr(out))
        return out

    def ranmom(self):
        self.lib.ref_ranmom()

    def grsource(self):
        out = np.zeros(self.V * self.tfd)
        it = self.lib.ref_grsource(_ptr(out))
        return out, it

    # per-trajectory measurements (control.c:85-138) ------------------------
    def ploop(self, d: int, project: int):
        out = np.zeros(3)
        self.lib.ref_ploop(int(d), int(project), _ptr(out))
        return complex(out[0], out[1]), out[2]

    def link_trace(self):
        L = self.lib
        L.ref_link_trace.restype = C.c_double
        lt, ld = np.zeros(5), np.zeros(5)
        w, da, dw = C.c_double(), C.c_double(), C.c_double()
        ave = L.ref_link_trace(_ptr(lt), C.byref(w), _ptr(ld), C.byref(da), C.byref(dw))
        return {"linktr": lt, "linktr_ave": ave, "linktr_width": w.value, "link_det": ld,
                "det_ave": da.value, "det_width": dw.value}

    def scalar_eig(self, project: int):
        n = self.ncol
        a, w, mn, mx = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.ref_scalar_eig(int(project), _ptr(a), _ptr(w), _ptr(mn), _ptr(mx))
        return a, w, mn, mx

    def gauge_action(self, do_det: int = 0):
        self.lib.ref_gauge_action.restype = C.c_double
        return self.lib.ref_gauge_action(int(do_det))

    def _printed(self, fn, tag):
        self.log()
        start = len(self.log())
        fn()
        for line in self.log()[start:].splitlines():
            if line.startswith(tag + " "):
                return np.array([float(x) for x in line.split()[1:]])
        raise RuntimeError("no %s line" % tag)

    def measure_det(self):
        """DET line of measure_det (determinant.c:92-120): 5 numbers"""
        return self._printed(self.lib.ref_measure_det, "DET")

    def widths(self):
        """WIDTHS line of widths (widths.c:8-71): 3 numbers"""
        return self._printed(self.lib.ref_widths, "WIDTHS")

    def plaquette(self):
        ss, st = C.c_double(), C.c_double()
        self.lib.ref_plaquette(C.byref(ss), C.byref(st))
        return ss.value, st.value

    def update(self):
        return self.lib.ref_update()


def _worker(fn, args, kwargs, q):
    try:
        q.put(("ok", fn(*args, **kwargs)))
    except BaseException as e:  # report any failure to the parent
        import traceback
        q.put(("err", "%s\n%s" % (e, traceback.format_exc())))


def run_in_fresh_process(fn, *args, **kwargs):
    """Run fn(*args) in a spawned process (one reference lattice each)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_worker, args=(fn, args, kwargs, q))
    p.start()
    status, val = q.get()
    p.join()
    if status != "ok":
        raise RuntimeError("reference worker failed: " + val)
    return val
