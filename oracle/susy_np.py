"""CPU restatement (numpy) of the 4d_Q16 RHMC fermion path of SUSY LATTICE.

TEST INFRASTRUCTURE ONLY.  This module is the oracle: tests, ``smoke()`` and
the CPU leg of ``bench.py`` may import it, as the checker; the shipped
library ``susy_b200`` never does.  It restates, in vectorised numpy over all
sites at once, the algorithm of the reference C code (paths relative to the
reference project, ``4d_Q16/``):

* site layout, neighbours and temporal boundary signs
  (generic/layout_hyper_prime.c:157, susy/setup_offset.c:67-201),
* U(N) generators, epsilon tensor and term tables
  (susy/setup_lambda.c:10-64,123-297),
* plaquette determinants, inverses, DmuUmu, Fmunu
  (susy/utilities.c:17-127, susy/action.c:15-98),
* the twisted fermion operator and its square
  (susy/utilities.c:141-885),
* the multi-shift CG (susy/congrad_multi.c:26-221),
* the fermion, gauge and determinant forces
  (susy/update_h.c:15-978, susy/det_force.c:6-78),
* actions, link update, site RNG, momenta, pseudofermions and the Omelyan
  HMC trajectory (susy/action.c:106-328, susy/update_o.c:20-282,
  susy/grsource.c:44-304, generic/ranstuff.c:22-63,
  libraries/gaussrand.c:12-32),
* the per-trajectory measurements of susy/control.c:85-138 (plaq.c,
  ploop.c, link_trace.c, determinant.c:92-120, widths.c, scalar_eig.c,
  unit.c:52-98).

Pinned against the reference itself: ``tests/test_oracle_golden.py`` checks
this module against vectors produced by the unmodified reference code
(``tests/golden/``, made by ``tests/golden/make_golden.py`` through
``oracle/_ref``), and the reference's regression goldens
(testsuite/scalar/hmc.U2.ref) are reproduced by ``oracle/_ref`` itself.

Layout here: sites in lexicographic order ``x + nx*(y + ny*(z + nz*t))``;
a matrix field is complex128 ``[..., V, N, N]``; a Twist_Fermion field is
``[16, V, N, N]`` with component 0 = site (eta), 1..5 = links (psi_a),
6..15 = plaquettes chi_ab for a < b in plaq_index order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from itertools import permutations

import numpy as np

NUMLINK = 5
NPLAQ = 10
C2 = 1.0
IMAG_TOL = 1.0e-8
LAMBDA = 0.193        # Omelyan parameters, susy/defines.h:16-18
TWO_LAMBDA = 0.386
LAMBDA_MID = 0.614

# Link offsets: four axes plus DIR_5 = (-1,-1,-1,-1)  (setup_offset.c:155-162)
OFFSETS = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1],
                    [-1, -1, -1, -1]], dtype=np.int64)


# ---------------------------------------------------------------------------
# Constant tables
def plaq_index_table() -> np.ndarray:
    """(a, b) -> linear plaquette index, setup_lambda.c:142-152."""
    pi = -np.ones((NUMLINK, NUMLINK), dtype=np.int64)
    for mu in range(NUMLINK):
        for nu in range(mu + 1, NUMLINK):
            idx = mu * (NUMLINK - 1) - mu * (mu + 1) // 2 + nu - 1
            pi[mu, nu] = pi[nu, mu] = idx
    return pi


PLAQ_INDEX = plaq_index_table()
PLAQ_PAIRS = [(a, b) for a in range(NUMLINK) for b in range(a + 1, NUMLINK)]


def _perm_sign(seq) -> float:
    s = list(seq)
    sign = 1.0
    for i in range(len(s)):
        for j in range(len(s) - 1 - i):
            if s[j] > s[j + 1]:
                s[j], s[j + 1] = s[j + 1], s[j]
                sign = -sign
    return sign


def epsilon_table() -> np.ndarray:
    """Totally antisymmetric epsilon_{abcde}, setup_lambda.c:123-193."""
    eps = np.zeros((NUMLINK,) * 5)
    for p in permutations(range(NUMLINK)):
        eps[p] = _perm_sign(p)
    return eps


PERM = epsilon_table()


def term_tables():
    """Term lists {a,b,c,d,e} of setup_lambda.c:202-297 (same order)."""
    dbp, dbm, fq = [], [], []
    for a in range(5):
        for b in range(a + 1, 5):
            for c in range(5):
                if c in (a, b):
                    continue
                for d in range(5):
                    if d in (c, a, b):
                        continue
                    for e in range(d + 1, 5):
                        if e in (c, a, b):
                            continue
                        dbp.append((a, b, c, d, e))
    for d in range(5):
        for e in range(d + 1, 5):
            for c in range(5):
                if c in (d, e):
                    continue
                for a in range(5):
                    if a in (c, d, e):
                        continue
                    for b in range(a + 1, 5):
                        if b in (c, d, e):
                            continue
                        dbm.append((a, b, c, d, e))
    for c in range(5):
        for d in range(5):
            if d == c:
                continue
            for e in range(d + 1, 5):
                if e == c:
                    continue
                for a in range(5):
                    if a in (d, e, c):
                        continue
                    for b in range(a + 1, 5):
                        if b in (d, e, c):
                            continue
                        fq.append((a, b, c, d, e))
    return dbp, dbm, fq


DBPLUS_TERMS, DBMINUS_TERMS, FQ_TERMS = term_tables()


def lambda_generators(N: int) -> np.ndarray:
    """U(N) generators with Tr(T_a T_b) = -delta_ab, setup_lambda.c:10-64."""
    dimf = N * N
    L = np.zeros((dimf, N, N), dtype=np.complex128)
    count = 0
    s2 = 1.0 / math.sqrt(2.0)
    for i in range(N):
        for j in range(i + 1, N):
            L[count, i, j] += 1j * s2
            L[count + 1, i, j] += s2
            L[count, j, i] += 1j * s2
            L[count + 1, j, i] -= s2
            count += 2
    for i in range(N - 1):
        j = N * (N - 1) + i
        k = i + 1
        v = 1j / math.sqrt(k * (k + 1.0))
        for l in range(k + 1):
            L[j, l, l] = v
        L[j, k, k] = v * (-1.0 * k)
    L[dimf - 1] = 0.0
    for i in range(N):
        L[dimf - 1, i, i] = 1j * math.sqrt(1.0 / N)
    return L


# ---------------------------------------------------------------------------
# Matrix helpers
def adj(m):
    return np.conj(np.swapaxes(m, -1, -2))


def tr(m):
    return np.trace(m, axis1=-2, axis2=-1)


def realtrace(a, b):
    """Re Tr(a^dag b) summed, libraries/realtr.c:19-29."""
    return float(np.sum(a.real * b.real + a.imag * b.imag))


# ---------------------------------------------------------------------------
# Lattice geometry
@dataclass
class Geometry:
    """Site indexing, neighbour tables and temporal boundary signs."""
    dims: tuple
    pbc: int

    def __post_init__(self):
        nx, ny, nz, nt = self.dims
        self.V = nx * ny * nz * nt
        idx = np.arange(self.V)
        self.x = idx % nx
        self.y = (idx // nx) % ny
        self.z = (idx // (nx * ny)) % nz
        self.t = idx // (nx * ny * nz)
        self.coords = np.stack([self.x, self.y, self.z, self.t], axis=1)
        self._nbr = {}
        self._bc = {}

    def index(self, c):
        nx, ny, nz, nt = self.dims
        return c[..., 0] + nx * (c[..., 1] + ny * (c[..., 2] + nz * c[..., 3]))

    def nbr(self, disp) -> np.ndarray:
        """Index of x + disp for every x (cubic_neighbor, setup_offset.c:17)."""
        key = tuple(int(v) for v in disp)
        if key not in self._nbr:
            c = (self.coords + np.array(key)) % np.array(self.dims)
            self._nbr[key] = self.index(c)
        return self._nbr[key]

    def disp(self, *links, sign=1):
        d = np.zeros(4, dtype=np.int64)
        for a in links:
            d += OFFSETS[a]
        return sign * d

    def shift(self, f, *links, sign=1):
        """Field value at x + sign*sum(e_links), for every x."""
        return np.take(f, self.nbr(self.disp(*links, sign=sign)), axis=-3)

    def shift_c(self, f, *links, sign=1):
        """Same as shift for a complex scalar field [..., V]."""
        return np.take(f, self.nbr(self.disp(*links, sign=sign)), axis=-1)

    def bc(self, *links, sign=1) -> np.ndarray:
        """Temporal BC factor for a path of net displacement sign*sum(e_a).

        PBC where t + dt leaves [0, nt-1], else 1 (setup_offset.c:67-145):
        bc[a] = bc(a), bc[OPP(a)] = bc(a, sign=-1), bc2[a][b] = bc(a, b),
        bc2[OPP a][OPP b] = bc(a, b, sign=-1), likewise bc3.
        """
        dt = int(self.disp(*links, sign=sign)[3])
        if dt not in self._bc:
            tt = self.t + dt
            nt = self.dims[3]
            self._bc[dt] = np.where((tt < 0) | (tt > nt - 1), float(self.pbc), 1.0)
        return self._bc[dt]

    # Reference site order (even sites first, layout_hyper_prime.c:157-170)
    def node_index(self) -> np.ndarray:
        """node_index(x,y,z,t) for every lexicographic site."""
        V = self.V
        i = np.arange(V)
        even = ((self.x + self.y + self.z + self.t) % 2) == 0
        return np.where(even, i // 2, (i + V) // 2)


def bcol(b):
    """Broadcast a per-site real factor over matrix axes."""
    return b[:, None, None]


# ---------------------------------------------------------------------------
# Parameters and state
@dataclass
class Params:
    """Action and algorithm parameters (lattice.h:72-130, setup.c:307-557)."""
    lam: float = 1.0
    bmass: float = 0.0
    fmass: float = 0.0
    kappa_u1: float = 0.0
    G: float = 0.0
    N: int = 2
    # the reference's compile-time RESCALE (defines.h:30; set for its
    # susy_cheb and susy_mode programs): fermion_op doubles the site
    # component of its input and of its output (utilities.c:795,841)
    rescale: bool = False

    @property
    def kappa(self):
        return self.N * 0.25 / self.lam          # setup.c:459

    @property
    def doG(self):
        return self.G > IMAG_TOL                 # setup.c:450


@dataclass
class Derived:
    """Fields recomputed after every link update (update_o.c:31-34)."""
    det: np.ndarray = None        # [5, V]
    plaqdet: np.ndarray = None    # [5, 5, V]
    ZW: np.ndarray = None         # [5, 5, V]
    Uinv: np.ndarray = None       # [5, V, N, N]
    DmuUmu: np.ndarray = None     # [V, N, N]
    Fmunu: np.ndarray = None      # [10, V, N, N]


def compute_derived(geo: Geometry, prm: Params, U: np.ndarray) -> Derived:
    """compute_plaqdet/Uinv (utilities.c:17-127), DmuUmu/Fmunu (action.c:15-98)."""
    d = Derived()
    N = U.shape[-1]
    det = np.linalg.det(U)                         # [5, V]
    d.det = det
    pd = np.zeros((NUMLINK, NUMLINK, geo.V), dtype=np.complex128)
    for a in range(NUMLINK):
        for b in range(NUMLINK):
            if a == b:
                continue
            # conj(det U_a(x)) det U_b(x) conj(det U_b(x+a)) det U_a(x+b)
            pd[a, b] = (np.conj(det[a]) * det[b]
                        * np.conj(geo.shift_c(det[b], a)) * geo.shift_c(det[a], b))
    d.plaqdet = pd
    d.ZW = pd * np.conj(pd - 1.0)
    d.Uinv = np.linalg.inv(U)
    D = np.zeros((geo.V, N, N), dtype=np.complex128)
    for mu in range(NUMLINK):
        D += U[mu] @ adj(U[mu]) - geo.shift(adj(U[mu]) @ U[mu], mu, sign=-1)
    if prm.doG:
        s = np.zeros(geo.V, dtype=np.complex128)
        for mu in range(NUMLINK):
            for nu in range(NUMLINK):
                if mu != nu:
                    s += prm.G * (pd[mu, nu] - 1.0)
        D += s[:, None, None] * np.eye(N)
    d.DmuUmu = D
    F = np.zeros((NPLAQ, geo.V, N, N), dtype=np.complex128)
    for (mu, nu) in PLAQ_PAIRS:
        F[PLAQ_INDEX[mu, nu]] = (U[mu] @ geo.shift(U[nu], mu)
                                 - U[nu] @ geo.shift(U[mu], nu))
    d.Fmunu = F
    return d


def _anti(field16, a, b, base):
    """chi_ab from a plaquette set with chi_ba = -chi_ab (utilities.c:288)."""
    m = field16[base + PLAQ_INDEX[a, b]]
    return m if a < b else -m


# ---------------------------------------------------------------------------
# Fermion operator
def fermion_op(geo: Geometry, prm: Params, U, der: Derived, src, sign: int):
    """D (sign=+1) or D^dag (sign=-1) on a Twist_Fermion, utilities.c:765-865."""
    if sign not in (1, -1):
        raise ValueError("incorrect sign in fermion_op: %d" % sign)
    N = U.shape[-1]
    s = src if sign == 1 else adj(src)
    if prm.rescale:                              # utilities.c:795-797
        s = s.copy()
        s[0] = 2.0 * s[0]
    eta = s[0]
    psi = s[1:6]
    V = geo.V
    dest = np.zeros_like(s)
    tr_eta = tr(eta)
    bcl = [geo.bc(a) for a in range(NUMLINK)]
    bcm = [geo.bc(a, sign=-1) for a in range(NUMLINK)]

    # Dplus: link -> plaq (utilities.c:137-221), overwrites plaq_dest
    for (a, b) in PLAQ_PAIRS:
        p = 6 + PLAQ_INDEX[a, b]
        dest[p] = (bcol(bcl[a]) * (U[a] @ geo.shift(psi[b], a))
                   - psi[b] @ geo.shift(U[a], b)
                   - bcol(bcl[b]) * (U[b] @ geo.shift(psi[a], b))
                   + psi[a] @ geo.shift(U[b], a))
    # Dminus: plaq -> link (utilities.c:228-321), overwrites link_dest
    for b in range(NUMLINK):
        acc = np.zeros((V, N, N), dtype=np.complex128)
        for a in range(NUMLINK):
            if a == b:
                continue
            chi = _anti(s, a, b, 6)
            acc += geo.shift(U[a], b) @ chi
            acc -= bcol(bcm[a]) * geo.shift(chi @ U[a], a, sign=-1)
        dest[1 + b] = acc
    # DbplusStoL: site -> link, 1/2 (utilities.c:517-545)
    for a in range(NUMLINK):
        dest[1 + a] += 0.5 * (bcol(bcl[a]) * (geo.shift(eta, a) @ adj(U[a]))
                              - adj(U[a]) @ eta)
    # detStoL (utilities.c:551-628)
    if prm.doG:
        localG = -0.5 * C2 * prm.G
        td = tr_eta[None, None, :] * der.plaqdet
        for a in range(NUMLINK):
            acc = np.zeros(V, dtype=np.complex128)
            for b in range(NUMLINK):
                if b == a:
                    continue
                acc += td[b, a] + bcm[b] * geo.shift_c(td[a, b], b, sign=-1)
            dest[1 + a] += (localG * acc)[:, None, None] * der.Uinv[a]
    # DbminusLtoS: link -> site, 1/2 (utilities.c:634-682), overwrites
    acc = np.zeros((V, N, N), dtype=np.complex128)
    for a in range(NUMLINK):
        acc += psi[a] @ adj(U[a])
        acc -= bcol(bcm[a]) * geo.shift(adj(U[a]) @ psi[a], a, sign=-1)
    dest[0] = 0.5 * acc
    # detLtoS (utilities.c:688-756)
    if prm.doG:
        localG = 0.5 * C2 * prm.G * math.sqrt(N)
        T = tr(der.Uinv @ psi)                       # [5, V]
        acc = np.zeros(V, dtype=np.complex128)
        for a in range(NUMLINK):
            for b in range(NUMLINK):
                if a == b:
                    continue
                acc += 1j * localG * der.plaqdet[a, b] * (
                    T[b] + bcl[b] * geo.shift_c(T[a], b))
        dest[0] -= (1j * math.sqrt(1.0 / N) * acc)[:, None, None] * np.eye(N)
    # DbminusPtoP (utilities.c:420-510), adds
    for (a, b, c, d, e) in DBMINUS_TERMS:
        trf = 0.5 * PERM[a, b, c, d, e]
        chi = s[6 + PLAQ_INDEX[a, b]]
        dest[6 + PLAQ_INDEX[d, e]] += trf * (
            bcol(geo.bc(a, b, sign=-1))
            * (geo.shift(chi, a, b, sign=-1) @ adj(geo.shift(U[c], a, b, c, sign=-1)))
            - bcol(geo.bc(a, b, c, sign=-1))
            * (adj(geo.shift(U[c], c, sign=-1)) @ geo.shift(chi, a, b, c, sign=-1)))
    # DbplusPtoP (utilities.c:327-414), adds
    for (a, b, c, d, e) in DBPLUS_TERMS:
        trf = 0.5 * PERM[a, b, c, d, e]
        chi = s[6 + PLAQ_INDEX[d, e]]
        dest[6 + PLAQ_INDEX[a, b]] += trf * (
            bcol(geo.bc(a, b, c)) * (geo.shift(chi, a, b, c) @ adj(geo.shift(U[c], a, b)))
            - bcol(geo.bc(a, b))
            * (adj(geo.shift(U[c], c, sign=-1)) @ geo.shift(chi, a, b)))
    if prm.rescale:                              # utilities.c:841-844
        dest[0] = 2.0 * dest[0]
    if sign == 1:
        return dest
    return -adj(dest)


def DSq(geo, prm, U, der, src):
    """(D^dag D + fmass^2) src, utilities.c:874-885."""
    out = fermion_op(geo, prm, U, der, fermion_op(geo, prm, U, der, src, 1), -1)
    if prm.fmass > IMAG_TOL:
        out = out + prm.fmass * prm.fmass * src
    return out


def magsq(f):
    return float(np.sum(f.real * f.real + f.imag * f.imag))


def rdot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


# ---------------------------------------------------------------------------
# Multi-shift CG
def congrad_multi(geo, prm, U, der, src, shifts, MaxCG, errormin):
    """Jegerlehner multi-mass CG, congrad_multi.c:26-221.

    Returns (psim [Norder, 16, V, N, N], iterations, final rsq).
    """
    shifts = np.asarray(shifts, dtype=np.float64)
    n = len(shifts)
    rm = src.copy()
    pm0 = src.copy()
    psim = np.zeros((n,) + src.shape, dtype=src.dtype)
    pm = [None] + [src.copy() for _ in range(1, n)]
    converged = [False] * n
    source_norm = magsq(src)
    rsq = source_norm
    rsqstop = errormin * source_norm
    zeta_im1 = np.ones(n)
    zeta_i = np.ones(n)
    zeta_ip1 = np.ones(n)
    alpha = np.zeros(n)
    beta_im1 = np.ones(n)
    beta_i = np.zeros(n)
    iteration = 0
    N_iter = 0
    while N_iter < MaxCG and rsq > rsqstop:
        mpm = DSq(geo, prm, U, der, pm0) + shifts[0] * pm0
        iteration += 1
        cd = rdot(pm0, mpm)
        beta_i[0] = -rsq / cd
        zeta_ip1[0] = 1.0
        for j in range(1, n):
            if not converged[j]:
                zeta_ip1[j] = zeta_i[j] * zeta_im1[j] * beta_im1[0]
                c1 = beta_i[0] * alpha[0] * (zeta_im1[j] - zeta_i[j])
                c2 = zeta_im1[j] * beta_im1[0] * (1 - (shifts[j] - shifts[0]) * beta_i[0])
                zeta_ip1[j] /= c1 + c2
                beta_i[j] = beta_i[0] * zeta_ip1[j] / zeta_i[j]
        psim[0] -= beta_i[0] * pm0
        for j in range(1, n):
            if not converged[j]:
                psim[j] -= beta_i[j] * pm[j]
        rm += beta_i[0] * mpm
        rsqnew = magsq(rm)
        alpha[0] = rsqnew / rsq
        for j in range(1, n):
            if not converged[j]:
                alpha[j] = alpha[0] * zeta_ip1[j] * beta_i[j] / (zeta_i[j] * beta_i[0])
        pm0 = zeta_ip1[0] * rm + alpha[0] * pm0
        for j in range(1, n):
            if not converged[j]:
                pm[j] = zeta_ip1[j] * rm + alpha[j] * pm[j]
        rsq = rsqnew
        for j in range(1, n):
            if not converged[j]:
                if rsq * zeta_ip1[j] * zeta_ip1[j] <= rsqstop:
                    converged[j] = True
        for j in range(n):
            if not converged[j]:
                beta_im1[j] = beta_i[j]
                zeta_im1[j] = zeta_i[j]
                zeta_i[j] = zeta_ip1[j]
        N_iter += 1
    return psim, iteration, rsq


# ---------------------------------------------------------------------------
# Forces
def _detF(geo, prm, U, der, eta, psi, sign, fU):
    """Plaquette-determinant fermion force, update_h.c:469-651."""
    localG = 0.5 * C2 * prm.G * (-1.0 if sign == 1 else 1.0)
    tr_eta = tr(eta)
    T = tr(der.Uinv @ psi)                            # [5, V]
    D = tr_eta[None, None, :] * der.plaqdet
    Udag_inv = adj(der.Uinv)
    for a in range(NUMLINK):
        plaq_term = np.zeros(geo.V, dtype=np.complex128)
        adj_term = np.zeros(geo.V, dtype=np.complex128)
        inv_term = np.zeros(geo.V, dtype=np.complex128)
        for b in range(NUMLINK):
            if a == b:
                continue
            bca = geo.bc(a)
            bcb = geo.bc(b)
            bcmb = geo.bc(b, sign=-1)
            Dab_mb = geo.shift_c(D[a, b], b, sign=-1)
            Dba_mb = geo.shift_c(D[b, a], b, sign=-1)
            plaq_term += D[b, a] * (T[a] + bca * geo.shift_c(T[b], a))
            plaq_term += Dab_mb * (geo.shift_c(T[b], b, sign=-1) + bcmb * T[a])
            adj_term += D[a, b] * (T[b] + bcb * geo.shift_c(T[a], b))
            step = bca * geo.shift_c(T[b], a)
            adj_term += Dba_mb * (geo.shift_c(T[a], b, sign=-1)
                                  + geo.shift_c(step, b, sign=-1))
            inv_term += D[b, a] + bcmb * Dab_mb
        upsiu = der.Uinv[a] @ psi[a] @ der.Uinv[a]
        fU[a] += (localG * plaq_term)[:, None, None] * der.Uinv[a]
        fU[a] += adj((localG * adj_term)[:, None, None] * Udag_inv[a])
        fU[a] -= (localG * inv_term)[:, None, None] * upsiu


def assemble_fermion_force(geo, prm, U, der, sol, psol):
    """f_U from one pole, update_h.c:666-916."""
    V = geo.V
    N = U.shape[-1]
    site_src = sol[0]
    link_src = sol[1:6]
    site_dest = adj(psol[0])
    link_dest = adj(psol[1:6])
    plaq_dest = adj(psol[6:16])
    fU = np.zeros((NUMLINK, V, N, N), dtype=np.complex128)
    bcl = [geo.bc(a) for a in range(NUMLINK)]
    # S/L terms (update_h.c:705-746)
    for mu in range(NUMLINK):
        up = link_src[mu] @ (bcol(bcl[mu]) * geo.shift(site_dest, mu)) \
            - site_dest @ link_src[mu]
        up -= link_dest[mu] @ (bcol(bcl[mu]) * geo.shift(site_src, mu))
        up += site_src @ link_dest[mu]
        fU[mu] = 0.5 * adj(up)
    # VP terms (update_h.c:753-894)
    pd_full = np.concatenate([np.zeros((6, V, N, N), dtype=np.complex128), plaq_dest])
    for mu in range(NUMLINK):
        for nu in range(NUMLINK):
            if mu == nu:
                continue
            P = _anti(pd_full, mu, nu, 6)
            fU[mu] += -bcol(bcl[mu]) * (geo.shift(link_src[nu], mu) @ P)
            fU[mu] += geo.shift(P @ link_src[nu], nu, sign=-1)
    for mu in range(NUMLINK):
        for nu in range(NUMLINK):
            if mu == nu:
                continue
            C = _anti(sol, mu, nu, 6)
            fU[mu] += geo.shift(link_dest[nu], mu) @ (bcol(bcl[mu]) * C)
            fU[mu] -= geo.shift(C @ link_dest[nu], nu, sign=-1)
    if prm.doG:
        _detF(geo, prm, U, der, site_dest, link_src, 1, fU)
        _detF(geo, prm, U, der, site_src, link_dest, -1, fU)
    # Q-closed pieces F1Q, F2Q (update_h.c:272-462)
    for (a, b, c, d, e) in FQ_TERMS:
        sol_ab = sol[6 + PLAQ_INDEX[a, b]]
        psol_de = plaq_dest[PLAQ_INDEX[d, e]]
        permm = PERM[d, e, c, a, b]
        f1 = permm * geo.bc(a, b, c) * bcl[c]
        f2 = -permm * geo.bc(a, b, sign=-1) * bcl[c]
        tm = geo.shift(psol_de, a, b, c) @ (bcol(f1) * geo.shift(sol_ab, c))
        tm += (bcol(f2) * geo.shift(sol_ab, a, b, sign=-1)) @ geo.shift(psol_de, c)
        fU[c] += -0.5 * adj(tm)
    for (a, b, c, d, e) in FQ_TERMS:
        psol_ab = plaq_dest[PLAQ_INDEX[a, b]]
        sol_de = sol[6 + PLAQ_INDEX[d, e]]
        permm = PERM[a, b, c, d, e]
        f1 = permm * geo.bc(a, b, sign=-1) * bcl[c]
        f2 = -permm * geo.bc(a, b, c) * bcl[c]
        tm = geo.shift(psol_ab, a, b, sign=-1) @ (bcol(f1) * geo.shift(sol_de, c))
        tm += (bcol(f2) * geo.shift(sol_de, a, b, c)) @ geo.shift(psol_ab, c)
        fU[c] += -0.5 * adj(tm)
    return fU


def fermion_force(geo, prm, U, der, mom, eps, sol, amp4):
    """Sum of pole forces into mom, update_h.c:928-978.  Returns the norm."""
    full = np.zeros_like(mom)
    for n in range(len(amp4)):
        psol = amp4[n] * fermion_op(geo, prm, U, der, sol[n], 1)
        full += adj(assemble_fermion_force(geo, prm, U, der, sol[n], psol))
    mom -= eps * full
    ret = magsq(full)
    return eps * math.sqrt(ret) / geo.V


def det_force(geo, prm, U, der, mom, eps):
    """kappa_u1 determinant force, det_force.c:6-78.  Returns sum |f_U|^2."""
    fU = np.zeros_like(U)
    for a in range(NUMLINK):
        td = np.zeros(geo.V, dtype=np.complex128)
        for b in range(NUMLINK):
            if a == b:
                continue
            td += der.ZW[b, a] + geo.shift_c(der.ZW[a, b], b, sign=-1)
        td = prm.kappa_u1 * td
        fU[a] = td[:, None, None] * der.Uinv[a]
        mom[a] -= eps * adj(fU[a])
    return magsq(fU)


def gauge_force(geo, prm, U, der, mom, eps):
    """Bosonic force into mom, update_h.c:15-261.  Returns the norm."""
    N = U.shape[-1]
    V = geo.V
    D = der.DmuUmu
    fU = np.zeros_like(U)
    for mu in range(NUMLINK):
        fU[mu] = adj(U[mu]) @ D - geo.shift(D, mu) @ adj(U[mu])
    if prm.doG:
        tcD = tr(D)
        Dd = tcD[None, None, :] * der.plaqdet
        for mu in range(NUMLINK):
            acc = np.zeros(V, dtype=np.complex128)
            for nu in range(NUMLINK):
                if nu == mu:
                    continue
                acc += Dd[nu, mu] + geo.shift_c(Dd[mu, nu], nu, sign=-1)
            fU[mu] += (prm.G * acc)[:, None, None] * der.Uinv[mu]
    Fm = np.concatenate([np.zeros((6, V, N, N), dtype=np.complex128), der.Fmunu])
    for mu in range(NUMLINK):
        for nu in range(NUMLINK):
            if mu == nu:
                continue
            F = _anti(Fm, mu, nu, 6)
            fU[mu] += 2.0 * (geo.shift(U[nu], mu) @ adj(F)
                             - geo.shift(adj(F) @ U[nu], nu, sign=-1))
    if prm.bmass > IMAG_TOL:
        dmu = 2.0 * prm.bmass * prm.bmass / N
        for mu in range(NUMLINK):
            trv = np.sum(np.abs(U[mu]) ** 2, axis=(-1, -2)) / N - 1.0
            fU[mu] += (dmu * trv)[:, None, None] * adj(U[mu])
    kap = prm.kappa
    mom -= kap * eps * adj(fU)
    ret = magsq(fU) * kap * kap
    if prm.kappa_u1 > IMAG_TOL:
        ret += det_force(geo, prm, U, der, mom, eps)
    return eps * math.sqrt(ret) / V


# ---------------------------------------------------------------------------
# Actions
def action_parts(geo, prm, U, der, mom, srcs, sols, amp4, ampdeg4):
    """gauge, bmass, det, fermion[n], mom (action.c:106-328)."""
    N = U.shape[-1]
    D = der.DmuUmu
    t = 0.5 * C2 * (D @ D)
    t = t + 2.0 * np.sum(adj(der.Fmunu) @ der.Fmunu, axis=0)
    g_act = prm.kappa * float(np.sum(tr(t).real))
    b_act = 0.0
    if prm.bmass > IMAG_TOL:
        trv = np.sum(np.abs(U) ** 2, axis=(-1, -2)) / N - 1.0
        b_act = prm.kappa * prm.bmass ** 2 * float(np.sum(trv * trv))
    d_act = 0.0
    if prm.kappa_u1 > IMAG_TOL:
        s = 0.0
        for (a, b) in PLAQ_PAIRS:
            p = der.plaqdet[a, b]
            s += float(np.sum((p.real - 1.0) ** 2 + p.imag ** 2))
        d_act = prm.kappa_u1 * s
    f_acts = []
    for src, sol in zip(srcs, sols):
        f = ampdeg4 * magsq(src)
        for j in range(len(amp4)):
            f += amp4[j] * rdot(src, sol[j])
        f_acts.append(f)
    p_act = magsq(mom)
    return g_act, b_act, d_act, f_acts, p_act


# ---------------------------------------------------------------------------
# Site random numbers (generic/ranstuff.c, libraries/gaussrand.c)
def _i32(v):
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def initialize_prn(seed: int, index):
    """Per-site generator state, ranstuff.c:22-42, vectorised over index.

    Returns uint64 array [..., 10]: r0..r6, multiplier, addend, ic_state
    (ic_state kept modulo 2^32, the only bits myrand ever uses).
    """
    index = np.asarray(index, dtype=np.int64)
    mult = (69607 + 8 * index).astype(np.uint64)
    st = np.zeros(index.shape + (10,), dtype=np.uint64)
    sd = np.full(index.shape, seed & 0xFFFFFFFF, dtype=np.uint64)
    m32 = np.uint64(0xFFFFFFFF)
    for k in range(7):
        sd = (mult * sd + np.uint64(12345)) & m32
        st[..., k] = (sd >> np.uint64(8)) & np.uint64(0xFFFFFF)
    sd = (mult * sd + np.uint64(12345)) & m32
    st[..., 7] = (100005 + 8 * index).astype(np.uint64)
    st[..., 8] = 12345
    st[..., 9] = sd
    return st


def myrand(st, mask=None):
    """Uniform [0,1) from each state row (ranstuff.c:48-63); advances st."""
    if mask is None:
        mask = np.ones(st.shape[:-1], dtype=bool)
    s = st[mask]
    r4, r5, r6 = s[:, 4], s[:, 5], s[:, 6]
    t = (((r5 >> np.uint64(7)) | (r6 << np.uint64(17)))
         ^ ((r4 >> np.uint64(1)) | (r5 << np.uint64(23)))) & np.uint64(0xFFFFFF)
    s[:, 6] = s[:, 5]
    s[:, 5] = s[:, 4]
    s[:, 4] = s[:, 3]
    s[:, 3] = s[:, 2]
    s[:, 2] = s[:, 1]
    s[:, 1] = s[:, 0]
    s[:, 0] = t
    ic = (s[:, 9] * s[:, 7] + s[:, 8]) & np.uint64(0xFFFFFFFF)
    s[:, 9] = ic
    st[mask] = s
    out = (t ^ ((ic >> np.uint64(8)) & np.uint64(0xFFFFFF))).astype(np.float64)
    return out / float(1 << 24)


def gaussian_pair(st):
    """One call pair of gaussian_rand_no per site (gaussrand.c:12-32).

    Density exp(-x^2); returns (first, second) as the reference hands them
    out: v2*fac then v1*fac.  Every site draws an even count in ranmom and
    grsource, so the static pairing of the reference stays site-local.
    """
    n = st.shape[0]
    v1 = np.zeros(n)
    v2 = np.zeros(n)
    r = np.zeros(n)
    todo = np.ones(n, dtype=bool)
    while todo.any():
        a = 2.0 * myrand(st, todo) - 1.0
        b = 2.0 * myrand(st, todo) - 1.0
        rr = a * a + b * b
        v1[todo] = a
        v2[todo] = b
        r[todo] = rr
        ok = rr < 1.0
        idx = np.nonzero(todo)[0]
        todo[idx[ok]] = False
    # libm log per element, as the reference calls it (numpy's vector log
    # may differ from libm in the last bit)
    logr = np.array([math.log(v) for v in r])
    fac = np.sqrt(-logr / r)
    return v2 * fac, v1 * fac


def ranmom(st, N):
    """Gaussian momenta sum_j (g + i g') Lambda_j, grsource.c:44-64."""
    L = lambda_generators(N)
    V = st.shape[0]
    mom = np.zeros((NUMLINK, V, N, N), dtype=np.complex128)
    for mu in range(NUMLINK):
        for j in range(N * N):
            gr, gi = gaussian_pair(st)
            mom[mu] += (gr + 1j * gi)[:, None, None] * L[j]
    return mom


def gaussian_tf(st, N):
    """Gaussian Twist_Fermion in grsource's draw order, grsource.c:213-245."""
    L = lambda_generators(N)
    V = st.shape[0]
    R = np.zeros((16, V, N, N), dtype=np.complex128)
    for j in range(N * N):
        for comp in range(16):
            gr, gi = gaussian_pair(st)
            R[comp] += (gr + 1j * gi)[:, None, None] * L[j]
    return R


# ---------------------------------------------------------------------------
# HMC trajectory (update_o.c)
@dataclass
class RHMC:
    """Rational approximation (setup_rhmc.c) for Norder poles."""
    amp4: np.ndarray
    shift4: np.ndarray
    amp8: np.ndarray
    shift8: np.ndarray
    ampdeg4: float
    ampdeg8: float


@dataclass
class HMCState:
    geo: Geometry
    prm: Params
    U: np.ndarray
    mom: np.ndarray
    site_prn: np.ndarray            # [V, 10] in lexicographic order
    node_prn: np.ndarray            # [10]
    rhmc: RHMC
    Nroot: int = 1
    nsteps: tuple = (1, 1)
    traj_length: float = 1.0
    niter: int = 5000
    rsqmin: float = 1e-20
    total_iters: int = 0
    der: Derived = None
    log: list = field(default_factory=list)

    def refresh(self):
        self.der = compute_derived(self.geo, self.prm, self.U)


def update_u(h: HMCState, eps):
    """link += eps * mom, then recompute (update_o.c:20-35)."""
    h.U = h.U + eps * h.mom
    h.refresh()


def update_gauge_step(h: HMCState, eps):
    """Omelyan gauge sub-steps, update_o.c:42-61."""
    n = h.nsteps[1]
    norm = gauge_force(h.geo, h.prm, h.U, h.der, h.mom, eps * LAMBDA)
    for i in range(1, n + 1):
        update_u(h, 0.5 * eps)
        norm += gauge_force(h.geo, h.prm, h.U, h.der, h.mom, eps * LAMBDA_MID)
        update_u(h, 0.5 * eps)
        if i < n:
            norm += gauge_force(h.geo, h.prm, h.U, h.der, h.mom, eps * TWO_LAMBDA)
        else:
            norm += gauge_force(h.geo, h.prm, h.U, h.der, h.mom, eps * LAMBDA)
    return norm / n


def _cg(h, src, shifts):
    psim, it, _ = congrad_multi(h.geo, h.prm, h.U, h.der, src, shifts,
                                h.niter, h.rsqmin)
    h.total_iters += it
    return psim, it


def update_step(h: HMCState, srcs, psims):
    """Two-level Omelyan integrator, update_o.c:67-121."""
    iters = 0
    f_eps = h.traj_length / h.nsteps[0]
    g_eps = f_eps / (2.0 * h.nsteps[1])
    amp4 = h.rhmc.amp4
    for n in range(h.Nroot):
        fermion_force(h.geo, h.prm, h.U, h.der, h.mom, f_eps * LAMBDA, psims[n], amp4)
    for i in range(1, h.nsteps[0] + 1):
        update_gauge_step(h, g_eps)
        for n in range(h.Nroot):
            psims[n], it = _cg(h, srcs[n], h.rhmc.shift4)
            iters += it
            fermion_force(h.geo, h.prm, h.U, h.der, h.mom, f_eps * LAMBDA_MID,
                          psims[n], amp4)
        update_gauge_step(h, g_eps)
        for n in range(h.Nroot):
            psims[n], it = _cg(h, srcs[n], h.rhmc.shift4)
            iters += it
            e = f_eps * (TWO_LAMBDA if i < h.nsteps[0] else LAMBDA)
            fermion_force(h.geo, h.prm, h.U, h.der, h.mom, e, psims[n], amp4)
    return iters


def action(h: HMCState, srcs, psims):
    g, b, d, f, p = action_parts(h.geo, h.prm, h.U, h.der, h.mom, srcs, psims,
                                 h.rhmc.amp4, h.rhmc.ampdeg4)
    h.log.append(("action", g, b, d, list(f), p))
    return g + b + d + sum(f) + p


def grsource(h: HMCState):
    """src = (D^dag D)^(1/8Nroot) R, grsource.c:200-304."""
    N = h.U.shape[-1]
    R = gaussian_tf(h.site_prn, N)
    psim, it = _cg(h, R, h.rhmc.shift8)
    src = h.rhmc.ampdeg8 * R
    for j in range(len(h.rhmc.amp8)):
        src = src + h.rhmc.amp8[j] * psim[j]
    return src, it


def update(h: HMCState, srcs_in=None, mom_in=None):
    """One HMC trajectory with Metropolis, update_o.c:127-282.

    srcs_in / mom_in optionally replace the refreshed pseudofermion sources
    and momenta (to replay a trajectory from given fields).
    Returns dict with delta_S, start/end action, accept, iters.
    """
    N = h.U.shape[-1]
    iters = 0
    h.mom = ranmom(h.site_prn, N)
    if mom_in is not None:
        h.mom = mom_in.copy()
    srcs = []
    for n in range(h.Nroot):
        s, it = grsource(h)
        iters += it
        srcs.append(s)
    if srcs_in is not None:
        srcs = [s.copy() for s in srcs_in]
    psims = []
    for n in range(h.Nroot):
        p, it = _cg(h, srcs[n], h.rhmc.shift4)
        iters += it
        psims.append(p)
    start = action(h, srcs, psims)
    old_U = h.U.copy()
    old_mom = h.mom.copy()
    iters += update_step(h, srcs, psims)
    end = action(h, srcs, psims)
    change = end - start
    if abs(change) > 1e20:
        change = 1.0e20
    xr = float(myrand(h.node_prn[None, :])[0])
    accept = not (math.exp(-change) < xr)
    if not accept:
        h.U = old_U
        h.mom = -old_mom
        h.refresh()
    return dict(delta_S=change, start=start, end=end, accept=accept,
                iters=iters, xrandom=xr)


# ---------------------------------------------------------------------------
# Layout conversion between the reference's AoS (node_index order) and here
# ---------------------------------------------------------------------------
# Per-trajectory measurements printed by control.c:85-138
def link_trace(U):
    """Tr[U Ubar]/N per direction, its average and width, and the real
    determinant of the traceless part of U Ubar (link_trace.c:9-56)."""
    N, V = U.shape[-1], U.shape[1]
    M = U @ adj(U)
    trs = np.real(tr(M))                                   # [5, V]
    linktr = trs.sum(axis=1) / N / V
    ave = float(linktr.mean())
    sq = float((trs ** 2).sum()) / (N * N * V * NUMLINK)
    T = M - (trs / N)[..., None, None] * np.eye(N)
    dets = np.real(np.linalg.det(T))
    link_det = dets.sum(axis=1) / V
    det_ave = float(link_det.mean())
    dsq = float((dets ** 2).sum()) / (V * NUMLINK)
    return {"linktr": linktr, "linktr_ave": ave, "linktr_width": math.sqrt(sq - ave * ave),
            "link_det": link_det, "det_ave": det_ave,
            "det_width": math.sqrt(dsq - det_ave * det_ave)}


def polar(U):
    """U = P u with P = sqrt(U U^dag) Hermitian positive, u unitary
    (unit.c:52-98); returns (u, P)."""
    w, v = np.linalg.eigh(U @ adj(U))
    P = (v * np.sqrt(w)[..., None, :]) @ adj(v)
    Pinv = (v / np.sqrt(w)[..., None, :]) @ adj(v)
    return Pinv @ U, P


def ploop(geo: Geometry, U, d: int, project: int):
    """Average trace of the product of links along direction d through the
    whole lattice, from the sites with coordinate 0 along it (t for DIR_5),
    and the average modulus (ploop.c:8-126).  project: polar-projected links."""
    L = polar(U[d])[0] if project else U[d]
    axis = d if d < 4 else 3
    length = geo.dims[axis]
    starts = np.nonzero(geo.coords[:, axis] == 0)[0]
    cur = starts
    prod = L[cur]
    step = geo.nbr(OFFSETS[d])
    for _ in range(1, length):
        cur = step[cur]
        prod = prod @ L[cur]
    t = tr(prod)
    norm = 1.0 / len(starts)
    return complex(t.sum() * norm), float(np.abs(t).sum() * norm)


def plaquette(geo: Geometry, U):
    """Space-space and space-time plaquette averages (plaq.c:7-53):
    Re Tr[U_a(x+b)^dag U_b(x)^dag U_a(x) U_b(x+a)] over b < a, the pairs with
    the temporal link (a or b = 3) in st."""
    ss = st = 0.0
    for a in range(1, NUMLINK):
        for b in range(a):
            v = realtrace(geo.shift(U[a], b), adj(U[b]) @ U[a] @ geo.shift(U[b], a))
            if a == 3 or b == 3:
                st += v
            else:
                ss += v
    return ss / (6.0 * geo.V), st / (4.0 * geo.V)


def measure_det(geo: Geometry, der: Derived):
    """DET line of measure_det (determinant.c:92-120)."""
    tot = 0j
    sq_re = sq_im = wsq = 0.0
    for a in range(1, NUMLINK):
        for b in range(a):
            p = der.plaqdet[a, b]
            tot += p.sum()
            sq_re += float((p.real ** 2).sum())
            sq_im += float((p.imag ** 2).sum())
            wsq += float((np.abs(p - 1.0) ** 2).sum())
    norm = 1.0 / (geo.V * NPLAQ)
    return np.array([tot.real * norm, tot.imag * norm, sq_re * norm, sq_im * norm, wsq * norm])


def widths(geo: Geometry, U):
    """WIDTHS line (widths.c:8-71): widths of Re Tr P_ab and of the real and
    imaginary parts of det P_ab, P_ab = U_b(x) U_a(x+b) [U_a(x) U_b(x+a)]^dag."""
    acc = np.zeros(6)
    for a in range(NUMLINK):
        for b in range(a + 1, NUMLINK):
            P = U[b] @ geo.shift(U[a], b) @ adj(U[a] @ geo.shift(U[b], a))
            t = np.real(tr(P))
            d = np.linalg.det(P)
            acc += [t.sum(), (t ** 2).sum(), d.real.sum(), (d.real ** 2).sum(),
                    d.imag.sum(), (d.imag ** 2).sum()]
    acc *= 0.1 / geo.V
    return np.array([math.sqrt(acc[1] - acc[0] ** 2), math.sqrt(acc[3] - acc[2] ** 2),
                     math.sqrt(acc[5] - acc[4] ** 2)])


def scalar_eig(U, project: int):
    """Average, width, minimum and maximum of each (ascending) eigenvalue
    over sites and links (scalar_eig.c:15-115): of the traceless part of
    U Ubar, or (project) of log P from the polar decomposition, whose
    eigenvalues are log(w)/2 for the eigenvalues w of U Ubar."""
    N = U.shape[-1]
    M = U @ adj(U)
    if project:
        e = 0.5 * np.log(np.linalg.eigvalsh(M))
    else:
        t = np.real(tr(M)) / N
        e = np.linalg.eigvalsh(M - t[..., None, None] * np.eye(N))
    e = e.reshape(-1, N)
    ave = e.mean(axis=0)
    width = np.sqrt((e ** 2).mean(axis=0) - ave ** 2)
    return ave, width, e.min(axis=0), e.max(axis=0)


def gauge_action(prm: Params, der: Derived):
    """gauge_action(NODET) (action.c:106-142): kappa sum Re Tr[C2/2 D^2 +
    2 sum F^dag F], C2 = 1."""
    D, F = der.DmuUmu, der.Fmunu
    t = 0.5 * np.real(tr(D @ D)).sum() + 2.0 * np.real(tr(adj(F) @ F)).sum()
    return prm.kappa * float(t)


def measurements(geo: Geometry, prm: Params, U, der: Derived):
    """Every quantity control.c:85-138 prints after a trajectory."""
    m = link_trace(U)
    p, pm = ploop(geo, U, 3, 0)
    m.update({"ploop_re": p.real, "ploop_im": p.imag, "ploop_mod": pm})
    m["ss_plaq"], m["st_plaq"] = plaquette(geo, U)
    m["gauge_action"] = gauge_action(prm, der)
    lines = [ploop(geo, U, d, 0)[0] for d in range(NUMLINK)]
    polar_lines = [ploop(geo, U, d, 1)[0] for d in range(NUMLINK)]
    m["lines"] = np.array(lines)
    m["lines_polar"] = np.array(polar_lines)
    m["det"] = measure_det(geo, der)
    m["widths"] = widths(geo, U)
    m["uubar"] = scalar_eig(U, 0)
    m["polar"] = scalar_eig(U, 1)
    return m


def tf_from_ref(geo: Geometry, flat: np.ndarray, N: int) -> np.ndarray:
    """Reference Twist_Fermion array (flat doubles) -> [16, V, N, N]."""
    a = flat.reshape(geo.V, 16, N, N, 2)
    a = a[..., 0] + 1j * a[..., 1]
    return np.ascontiguousarray(np.moveaxis(a[geo.node_index()], 0, 1))


def tf_to_ref(geo: Geometry, tf: np.ndarray) -> np.ndarray:
    N = tf.shape[-1]
    out = np.zeros((geo.V, 16, N, N, 2))
    a = np.moveaxis(tf, 0, 1)
    out[geo.node_index(), ..., 0] = a.real
    out[geo.node_index(), ..., 1] = a.imag
    return out.reshape(-1)


def links_from_ref(geo: Geometry, flat: np.ndarray, N: int, nmat=NUMLINK):
    a = flat.reshape(geo.V, nmat, N, N, 2)
    a = a[..., 0] + 1j * a[..., 1]
    return np.ascontiguousarray(np.moveaxis(a[geo.node_index()], 0, 1))


def links_to_ref(geo: Geometry, U: np.ndarray) -> np.ndarray:
    nmat, V, N, _ = U.shape
    out = np.zeros((V, nmat, N, N, 2))
    a = np.moveaxis(U, 0, 1)
    out[geo.node_index(), ..., 0] = a.real
    out[geo.node_index(), ..., 1] = a.imag
    return out.reshape(-1)


def site_prn_lex(geo: Geometry, iseed: int) -> np.ndarray:
    """Site generators seeded by lexicographic index (make_lattice.c:48)."""
    return initialize_prn(iseed, np.arange(geo.V))


def node_prn(geo: Geometry, iseed: int) -> np.ndarray:
    """Node generator, initialize_prn(&node_prn, iseed, volume) (setup.c:246)."""
    return initialize_prn(iseed, np.array([geo.V]))[0]
