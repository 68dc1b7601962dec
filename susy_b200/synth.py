"""Seeded synthetic inputs in the reference's host layout.

Links "identity + s * complex Gaussian": U_a(x)_ij = delta_ij + s (g1 + i g2)
with g1, g2 ~ N(0, 1/2) (unit variance per complex entry).  Twist_Fermion
sources: every complex entry (g1 + i g2), g1, g2 ~ N(0, 1) unless stated.
Generator: numpy PCG64 seeded with the given integer; arrays are produced
in lexicographic site order and permuted to the reference's node_index order
(even sites first, 4d_Q16/generic/layout_hyper_prime.c:157-170).
"""
from __future__ import annotations

import numpy as np


def node_index(dims) -> np.ndarray:
    """node_index for every lexicographic site index."""
    nx, ny, nz, nt = dims
    V = nx * ny * nz * nt
    i = np.arange(V)
    x = i % nx
    y = (i // nx) % ny
    z = (i // (nx * ny)) % nz
    t = i // (nx * ny * nz)
    even = ((x + y + z + t) % 2) == 0
    return np.where(even, i // 2, (i + V) // 2)


def to_ref(dims, field: np.ndarray) -> np.ndarray:
    """[K, V, N, N] complex (lexicographic) -> flat reference doubles."""
    K, V, N, _ = field.shape
    out = np.zeros((V, K, N, N, 2))
    a = np.moveaxis(field, 0, 1)
    ni = node_index(dims)
    out[ni, ..., 0] = a.real
    out[ni, ..., 1] = a.imag
    return out.reshape(-1)


def from_ref(dims, flat: np.ndarray, K: int, N: int) -> np.ndarray:
    """Flat reference doubles -> [K, V, N, N] complex (lexicographic)."""
    V = int(np.prod(dims))
    a = flat.reshape(V, K, N, N, 2)
    a = a[..., 0] + 1j * a[..., 1]
    return np.ascontiguousarray(np.moveaxis(a[node_index(dims)], 0, 1))


def links(dims, N: int, noise: float, seed: int) -> np.ndarray:
    """[5, V, N, N] complex near-identity links (lexicographic)."""
    V = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((5, V, N, N, 2)) * np.sqrt(0.5)
    return np.eye(N)[None, None] + noise * (g[..., 0] + 1j * g[..., 1])


def tf_source(dims, N: int, seed: int, scale: float = 1.0) -> np.ndarray:
    """[16, V, N, N] complex Gaussian Twist_Fermion (lexicographic)."""
    V = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((16, V, N, N, 2)) * scale
    return g[..., 0] + 1j * g[..., 1]


def geometric_shifts(n: int = 15, lo: float = 1e-5, hi: float = 1e3) -> np.ndarray:
    """sigma_j = lo * (hi/lo)^(j/(n-1)), j = 0..n-1."""
    return lo * (hi / lo) ** (np.arange(n) / (n - 1.0))
