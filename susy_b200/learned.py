"""Learned preconditioner: host side (susy_b200_net_* in include/susy_b200.h).

The network (gauge-covariant, parallel-transported nearest-neighbour
convolutions, 16 -> 32 -> 32 -> 16 channels, bfloat16 weights, FP32
arithmetic) runs on the device: forward for the preconditioner, forward and
backward for training.  This module owns the FP32 master weights and the
Adam optimiser, generates training pairs (r, (D^dag D + sigma)^-1 r) with the
library's own FP64 solver, and runs the preconditioned solve.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .lattice import Lattice, DeviceTF, _vp, _dp, _ptr

NTAP = 11
CHANNELS = (16, 32, 32, 16)


def weight_shapes():
    return [(NTAP, co, ci) for ci, co in zip(CHANNELS[:-1], CHANNELS[1:])]


def init_weights(seed: int = 0, scale: float = 1e-2):
    """Near the identity: the site tap passes channel c to c, small noise on
    every weight (the same initialisation the CPU definition uses)."""
    rng = np.random.default_rng(seed)
    Ws = []
    for (k, co, ci) in weight_shapes():
        W = scale * (rng.standard_normal((k, co, ci))
                     + 1j * rng.standard_normal((k, co, ci))) / np.sqrt(k * ci)
        for c in range(min(ci, co)):
            W[0, c, c] += 1.0
        Ws.append(W)
    return Ws


def _setup(L):
    if getattr(L, "_net_ready", False):
        return
    L.susy_b200_net_nweights.restype = C.c_int
    L.susy_b200_net_create.restype = _vp
    L.susy_b200_net_create.argtypes = [_vp]
    L.susy_b200_net_destroy.argtypes = [_vp]
    L.susy_b200_net_set_weights.restype = C.c_int
    L.susy_b200_net_set_weights.argtypes = [_vp, _dp]
    L.susy_b200_net_tensor_cores.restype = C.c_int
    L.susy_b200_net_tensor_cores.argtypes = [_vp, C.c_int]
    L.susy_b200_net_apply.restype = C.c_int
    L.susy_b200_net_apply.argtypes = [_vp, _vp, _vp]
    L.susy_b200_net_loss_grad.restype = C.c_int
    L.susy_b200_net_loss_grad.argtypes = [_vp, _vp, _vp, _dp, _dp]
    L.susy_b200_net_loss_grad2.restype = C.c_int
    L.susy_b200_net_loss_grad2.argtypes = [_vp, _vp, _vp, C.c_double, _dp, _dp]
    L.susy_b200_dev_congrad_multi_learned.restype = C.c_int
    L.susy_b200_dev_congrad_multi_learned.argtypes = [
        _vp, _vp, _vp, C.POINTER(_vp), C.c_int, _dp, C.c_int, C.c_double, C.c_int, C.c_double,
        _dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L._net_ready = True


def flatten(Ws) -> np.ndarray:
    return np.concatenate([np.stack([W.real, W.imag], -1).reshape(-1) for W in Ws])


def unflatten(v: np.ndarray):
    out, off = [], 0
    for shp in weight_shapes():
        n = int(np.prod(shp))
        z = v[off:off + 2 * n].reshape(shp + (2,))
        out.append(z[..., 0] + 1j * z[..., 1])
        off += 2 * n
    return out


class Net:
    """The device network bound to one lattice (reads its current links)."""

    def __init__(self, lat: Lattice, weights=None):
        self.lat = lat
        self.lib = lat.lib
        _setup(self.lib)
        self.h = self.lib.susy_b200_net_create(lat.h)
        if not self.h:
            raise MemoryError("susy_b200_net_create failed")
        self.nw = self.lib.susy_b200_net_nweights()
        self.set_weights(init_weights() if weights is None else weights)

    def close(self):
        if self.h:
            self.lib.susy_b200_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_weights(self, Ws):
        self.Ws = [np.array(W, dtype=np.complex128) for W in Ws]
        v = np.ascontiguousarray(flatten(self.Ws))
        assert v.size == 2 * self.nw
        self.lat._check(self.lib.susy_b200_net_set_weights(self.h, _ptr(v)))

    def tensor_cores(self, on: int = -1) -> int:
        """Inference mixes on the tensor cores (1, BF16 transports) or in
        FP32 (0); returns the previous setting."""
        return self.lat._check(self.lat.lib.susy_b200_net_tensor_cores(self.h, int(on)))

    def apply(self, src: DeviceTF, dst: DeviceTF):
        self.lat._check(self.lib.susy_b200_net_apply(self.h, src.ptr, dst.ptr))

    def loss_grad(self, r: DeviceTF, e: DeviceTF, sigma: float = -1.0):
        """(loss, dL/dW* per layer): |N(r) - e|^2 / |e|^2 for sigma < 0, the
        A-norm error (d, A d) / (e, A e) with A = D^dag D + sigma otherwise"""
        loss = C.c_double()
        g = np.zeros(2 * self.nw)
        self.lat._check(self.lib.susy_b200_net_loss_grad2(self.h, r.ptr, e.ptr, float(sigma),
                                                          C.byref(loss), _ptr(g)))
        return loss.value, unflatten(g)

    def train(self, pairs, steps=200, lr=2e-3, batch=8, seed=0, log=None, sigma=-1.0):
        """Adam on the complex weights (FP32 master copy here, bfloat16 on
        the device) over (r, e) device pairs; returns the loss history.
        A pair (r, e, links) also carries its configuration (host links in
        the reference layout): the lattice is switched to it before the
        pair's loss is evaluated (a batch is taken config by config)."""
        rng = np.random.default_rng(seed)
        Ws = [W.copy() for W in self.Ws]
        m = [np.zeros_like(W) for W in Ws]
        v = [np.zeros(W.shape) for W in Ws]
        b1, b2, eps = 0.9, 0.999, 1e-8
        hist = []
        for t in range(1, steps + 1):
            idx = rng.choice(len(pairs), size=min(batch, len(pairs)), replace=False)
            idx = sorted(idx, key=lambda i: id(pairs[i][2]) if len(pairs[i]) > 2 else 0)
            tot = 0.0
            gs = [np.zeros_like(W) for W in Ws]
            for i in idx:
                if len(pairs[i]) > 2 and getattr(self, "_links_id", None) != id(pairs[i][2]):
                    self.lat.set_links(pairs[i][2])
                    self._links_id = id(pairs[i][2])
                loss, g = self.loss_grad(pairs[i][0], pairs[i][1], sigma=sigma)
                tot += loss
                for a, b in zip(gs, g):
                    a += b
            hist.append(tot / len(idx))
            for k in range(len(Ws)):
                gk = gs[k] / len(idx)
                m[k] = b1 * m[k] + (1 - b1) * gk
                v[k] = b2 * v[k] + (1 - b2) * np.abs(gk) ** 2
                mh = m[k] / (1 - b1 ** t)
                vh = v[k] / (1 - b2 ** t)
                Ws[k] = (Ws[k] - lr * mh / (np.sqrt(vh) + eps)).astype(np.complex64).astype(
                    np.complex128)
            self.set_weights(Ws)
            if log and (t % log == 0 or t == 1):
                print("step %d loss %.6f" % (t, hist[-1]), flush=True)
        return hist


def make_pairs(lat: Lattice, sigma: float, nsrc: int, seed: int, errormin=1e-20):
    """(r, e) with r complex Gaussian (unit variance per entry) and
    e = (D^dag D + fmass^2 + sigma)^-1 r from the FP64 solver, both
    normalised by |r|."""
    from . import synth
    pairs = []
    for k in range(nsrc):
        r_host = synth.to_ref(lat.dims, synth.tf_source(lat.dims, lat.N, seed + k))
        r_host /= np.sqrt(np.dot(r_host, r_host))
        r = lat.tf(64)
        r.upload(r_host)
        e = lat.tf(64)
        lat.dev_congrad_multi(r, [e], np.array([sigma]), 20000, errormin)
        pairs.append((r, e))
    return pairs


def congrad_multi_learned(lat: Lattice, net, src: DeviceTF, psim, shift, MaxCG: int,
                          errormin: float, nrefine: int = 4, loose: float = 1e-12):
    """susy_b200_dev_congrad_multi_learned: (iterations, refinement
    iterations, worst true |r|^2); net None = unpreconditioned refinement."""
    _setup(lat.lib)
    n = len(psim)
    arr = (_vp * n)(*[p.ptr for p in psim])
    shift = np.ascontiguousarray(shift, dtype=np.float64)
    sr = C.c_double()
    it = C.c_int()
    rit = C.c_int()
    lat._check(lat.lib.susy_b200_dev_congrad_multi_learned(
        lat.h, net.h if net is not None else None, src.ptr, arr, n, _ptr(shift), int(MaxCG),
        float(errormin), int(nrefine), float(loose), C.byref(sr), C.byref(it), C.byref(rit)))
    return it.value, rit.value, sr.value
