"""CPU restatement (numpy, complex128) of the learned preconditioner.

TEST INFRASTRUCTURE ONLY: the checker of the device network in
susy_b200/csrc/learned.cu (forward, backward, loss); the shipped library
never imports it.  The network has no counterpart in the reference
("parity unpinned" for the network itself): this module is its definition,
and its gradients are checked here against finite differences.

The network maps a Twist_Fermion residual r to an approximation of
(D^dag D + sigma)^-1 r, gauge covariantly:

* embed: each component becomes a site-type matrix (x -> x) by closing its
  path with inverse links: S_0 = eta, S_{1+a} = psi_a U_a(x)^-1,
  S_{6+p(a,b)} = chi_ab U_b(x+a)^-1 U_a(x)^-1 (psi_a runs x -> x+a,
  chi_ab x -> x+a+b, as the operator's terms D+ psi, U psi(x+a) show);
* three layers of parallel-transported nearest-neighbour convolutions,
  16 -> 32 -> 32 -> 16 channels, linear:
  out_c(x) = sum_{k, c'} W[k, c, c'] T_k(in_c')(x) with the 11 transports
  T_0 X = X, T_{1+mu} X = U_mu(x) X(x+mu) U_mu(x)^-1,
  T_{6+mu} X = U_mu(x-mu)^-1 X(x-mu) U_mu(x-mu), complex weights;
* unembed: the inverse of embed (psi_a = S U_a(x), chi_ab = S U_a(x)
  U_b(x+a)).

Loss over samples: L = sum_s |N(r_s) - e_s|^2 / |e_s|^2.  Gradients are
dL/dW* in the Wirtinger sense: for L real and W = u + i v, the returned
G satisfies dL/du = 2 Re G, dL/dv = 2 Im G.
"""
from __future__ import annotations

import numpy as np

from . import susy_np as O

NTAP = 11
CHANNELS = (16, 32, 32, 16)


def adj(m):
    return np.conj(np.swapaxes(m, -1, -2))


def embed(geo, U, Uinv, tf):
    """[16, V, N, N] Twist_Fermion -> [16, V, N, N] site-type channels"""
    S = np.empty_like(tf)
    S[0] = tf[0]
    for a in range(5):
        S[1 + a] = tf[1 + a] @ Uinv[a]
    for (a, b) in O.PLAQ_PAIRS:
        p = O.PLAQ_INDEX[a, b]
        S[6 + p] = tf[6 + p] @ geo.shift(Uinv[b], a) @ Uinv[a]
    return S


def unembed(geo, U, S):
    tf = np.empty_like(S)
    tf[0] = S[0]
    for a in range(5):
        tf[1 + a] = S[1 + a] @ U[a]
    for (a, b) in O.PLAQ_PAIRS:
        p = O.PLAQ_INDEX[a, b]
        tf[6 + p] = S[6 + p] @ U[a] @ geo.shift(U[b], a)
    return tf


def unembed_adjoint(geo, U, G):
    """Adjoint of unembed w.r.t. sum Re Tr(A^dag B)"""
    out = np.empty_like(G)
    out[0] = G[0]
    for a in range(5):
        out[1 + a] = G[1 + a] @ adj(U[a])
    for (a, b) in O.PLAQ_PAIRS:
        p = O.PLAQ_INDEX[a, b]
        out[6 + p] = G[6 + p] @ adj(U[a] @ geo.shift(U[b], a))
    return out


def transports(geo, U, Uinv, X):
    """[C, V, N, N] -> [11, C, V, N, N]"""
    out = [X]
    for mu in range(5):
        out.append(U[mu] @ geo.shift(X, mu) @ Uinv[mu])
    for mu in range(5):
        out.append(geo.shift(Uinv[mu] @ X @ U[mu], mu, sign=-1))
    return np.stack(out)


def transports_adjoint(geo, U, Uinv, G):
    """Adjoint of transports: [11, C, V, N, N] -> [C, V, N, N]"""
    out = G[0].copy()
    for mu in range(5):
        # T_f X = U X(x+mu) U^-1: adjoint at y is U(y-mu)^dag G(y-mu) U(y-mu)^-dag
        out += geo.shift(adj(U[mu]) @ G[1 + mu] @ adj(Uinv[mu]), mu, sign=-1)
    for mu in range(5):
        # T_b X = U(x-mu)^-1 X(x-mu) U(x-mu): adjoint at y is U(y)^-dag G(y+mu) U(y)^dag
        out += adj(Uinv[mu]) @ geo.shift(G[6 + mu], mu) @ adj(U[mu])
    return out


def layer(T, W):
    """out[c] = sum_{k,c'} W[k,c,c'] T[k,c']"""
    return np.einsum("kdc,kcvij->dvij", W, T)


def bf16(w):
    """Round real and imaginary parts to bfloat16 (round to nearest even),
    the precision the device stores the weights in."""
    def r(x):
        b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
        b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
        return b.astype(np.uint32).view(np.float32).astype(np.float64)
    return r(w.real) + 1j * r(w.imag)


def init_weights(seed=0, scale=1e-2):
    """Near the identity: the T_0 tap passes channel c to c; small noise
    everywhere else."""
    rng = np.random.default_rng(seed)
    Ws = []
    for cin, cout in zip(CHANNELS[:-1], CHANNELS[1:]):
        W = scale * (rng.standard_normal((NTAP, cout, cin))
                     + 1j * rng.standard_normal((NTAP, cout, cin))) / np.sqrt(NTAP * cin)
        for c in range(min(cin, cout)):
            W[0, c, c] += 1.0
        Ws.append(W)
    return Ws


def forward(geo, U, Uinv, Ws, tf, keep=False, bf16_act=False):
    """bf16_act: the transports are rounded to bfloat16 (real and imaginary
    parts, nearest even) before each channel mix, as the device's
    tensor-core inference path feeds them to its BF16 matrix multiplies
    (FP32 accumulation)."""
    X = embed(geo, U, Uinv, tf)
    acts = []
    for W in Ws:
        T = transports(geo, U, Uinv, X)
        if bf16_act:
            T = bf16(T.astype(np.complex64))
        acts.append(T)
        X = layer(T, W)
    out = unembed(geo, U, X)
    return (out, acts) if keep else out


def loss_and_grad(geo, U, Uinv, Ws, rs, es):
    """L = sum_s |N(r_s) - e_s|^2 / |e_s|^2 and dL/dW* per layer"""
    L = 0.0
    grads = [np.zeros_like(W) for W in Ws]
    for r, e in zip(rs, es):
        z, acts = forward(geo, U, Uinv, Ws, r, keep=True)
        en = float(np.sum(np.abs(e) ** 2))
        d = z - e
        L += float(np.sum(np.abs(d) ** 2)) / en
        g = unembed_adjoint(geo, U, d / en)          # dL/dS* at the last layer
        for li in range(len(Ws) - 1, -1, -1):
            T = acts[li]
            grads[li] += np.einsum("kcvij,dvij->kdc", np.conj(T), g)
            if li > 0:
                gT = np.einsum("kdc,dvij->kcvij", np.conj(Ws[li]), g)
                g = transports_adjoint(geo, U, Uinv, gT)
    return L, grads
