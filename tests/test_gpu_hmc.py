"""GPU parity of forces, actions, random fields and the HMC trajectory.

Reference functions: gauge_force / det_force (update_h.c:15, det_force.c:6),
fermion_force (update_h.c:928), update_u (update_o.c:20), action pieces
(action.c:106-286), ranmom / grsource draws (grsource.c:44,200), update()
(update_o.c:127).  The oracle is oracle/susy_np.py on identical inputs.
Tolerances: FP64 fields 1e-12 relative (max-norm); force norms and actions
1e-12 relative; Gaussian fields 1e-12 (device log() may round differently
from libm in the last bit); the trajectory's delta S to 1e-7 absolute with
the same accept decision and iteration count within +-2 per solve.
"""
import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import Lattice, RHMC, SOLVER_FP64, SOLVER_MIXED, SusyError
from susy_b200 import synth
from susy_b200.rhmc_tables import rhmc as rhmc_table

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def make(dims, N, seed=3, noise=0.2, **kw):
    U = synth.links(dims, N, noise, seed)
    lat = Lattice(dims, N, pbc=-1, **kw)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, -1)
    prm = O.Params(lam=kw.get("lam", 1.0), bmass=kw.get("bmass", 0.0),
                   fmass=kw.get("fmass", 0.0), kappa_u1=kw.get("kappa_u1", 0.0),
                   G=kw.get("G", 0.0), N=N)
    return lat, geo, prm, U


@pytest.mark.parametrize("N", [2, 3])
def test_gauge_force(N):
    dims = (4, 4, 4, 4)
    lat, geo, prm, U = make(dims, N, lam=1.5, bmass=0.3, G=0.05, kappa_u1=0.4)
    der = O.compute_derived(geo, prm, U)
    mom0 = synth.links(dims, N, 0.5, 9) - np.eye(N)
    lat.set_mom(synth.to_ref(dims, mom0))
    mom = mom0.copy()
    want = O.gauge_force(geo, prm, U, der, mom, 0.07)
    got = lat.gauge_force(0.07)
    assert abs(got - want) <= 1e-12 * abs(want)
    assert rel(synth.from_ref(dims, lat.get_mom(), 5, N), mom) < 1e-12


def test_det_force():
    dims, N = (4, 4, 4, 4), 2
    lat, geo, prm, U = make(dims, N, kappa_u1=0.7, G=0.05)
    der = O.compute_derived(geo, prm, U)
    mom = np.zeros_like(U)
    lat.set_mom(synth.to_ref(dims, mom))
    want = O.det_force(geo, prm, U, der, mom, 0.05)
    got = lat.det_force(0.05)
    assert abs(got - want) <= 1e-12 * abs(want)
    assert rel(synth.from_ref(dims, lat.get_mom(), 5, N), mom) < 1e-12


@pytest.mark.parametrize("N,G", [(2, 0.05), (3, 0.05), (2, 0.0)])
def test_fermion_force(N, G):
    dims = (4, 4, 4, 4)
    lat, geo, prm, U = make(dims, N, G=G, bmass=0.2)
    der = O.compute_derived(geo, prm, U)
    sols = [synth.tf_source(dims, N, 40 + k) for k in range(3)]
    amp = np.array([0.3, 1.7, 0.02])
    mom = np.zeros_like(U)
    lat.set_mom(synth.to_ref(dims, mom))
    want = O.fermion_force(geo, prm, U, der, mom, 0.11, sols, amp)
    got = lat.fermion_force(0.11, None, [synth.to_ref(dims, s) for s in sols], amp)
    assert abs(got - want) <= 1e-12 * abs(want)
    assert rel(synth.from_ref(dims, lat.get_mom(), 5, N), mom) < 1e-12


def test_update_u_and_derived():
    dims, N = (4, 4, 4, 4), 3
    lat, geo, prm, U = make(dims, N, G=0.05)
    mom = synth.links(dims, N, 0.3, 12) - np.eye(N)
    lat.set_mom(synth.to_ref(dims, mom))
    lat.update_u(0.13)
    U2 = U + 0.13 * mom
    assert rel(synth.from_ref(dims, lat.get_links(), 5, N), U2) < 1e-14
    der = O.compute_derived(geo, prm, U2)
    pd, D, F, Ui = lat.derived()
    assert rel(synth.from_ref(dims, D, 1, N)[0], der.DmuUmu) < 1e-12


@pytest.mark.parametrize("N", [2, 3])
def test_action_parts(N):
    dims = (4, 4, 4, 4)
    lat, geo, prm, U = make(dims, N, lam=0.8, bmass=0.4, G=0.05, kappa_u1=0.3)
    der = O.compute_derived(geo, prm, U)
    mom = synth.links(dims, N, 0.3, 12) - np.eye(N)
    lat.set_mom(synth.to_ref(dims, mom))
    src = synth.tf_source(dims, N, 1)
    sols = [synth.tf_source(dims, N, 2 + k) for k in range(4)]
    amp = np.array([0.1, 0.2, 0.3, 0.4])
    g, b, d, f, p = O.action_parts(geo, prm, U, der, mom, [src], [sols], amp, 0.37)
    parts = lat.action([synth.to_ref(dims, src)], [[synth.to_ref(dims, s) for s in sols]],
                       amp, 0.37)
    for got, want in zip(parts, [g, b, d, f[0], p]):
        assert abs(got - want) <= 1e-12 * abs(want)


@pytest.mark.parametrize("N", [2, 3])
def test_ranmom_and_gaussian_source(N):
    dims = (4, 4, 2, 4)
    lat = Lattice(dims, N, iseed=41)
    geo = O.Geometry(dims, -1)
    st = O.site_prn_lex(geo, 41)
    lat.ranmom()
    want = O.ranmom(st, N)
    assert rel(synth.from_ref(dims, lat.get_mom(), 5, N), want) < 1e-12
    R = lat.gaussian_tf()
    assert rel(synth.from_ref(dims, R, 16, N), O.gaussian_tf(st, N)) < 1e-12


def test_trajectory_matches_oracle():
    dims, N = (4, 4, 4, 4), 2
    kw = dict(lam=1.0, bmass=0.2, G=0.05, kappa_u1=0.0)
    lat, geo, prm, U = make(dims, N, noise=0.1, seed=5, iseed=41, **kw)
    tab = rhmc_table(15, 1)
    r = RHMC(15, 1, nstep=2, nstep_gauge=2, traj_length=0.5, error_per_site=1e-6,
             solver=SOLVER_FP64)
    got = lat.update(r)
    h = O.HMCState(geo=geo, prm=prm, U=U.copy(), mom=np.zeros_like(U),
                   site_prn=O.site_prn_lex(geo, 41), node_prn=O.node_prn(geo, 41),
                   rhmc=O.RHMC(**tab), Nroot=1, nsteps=(2, 2), traj_length=0.5,
                   niter=5000, rsqmin=1e-12)
    h.refresh()
    want = O.update(h)
    assert got["accept"] == want["accept"]
    assert abs(got["start"] - want["start"]) < 1e-8 * abs(want["start"])
    assert abs(got["delta_S"] - want["delta_S"]) < 1e-7
    assert abs(got["iters"] - want["iters"]) <= 2 * 12
    assert rel(synth.from_ref(dims, lat.get_links(), 5, N), h.U) < 1e-9


def test_reversibility():
    """Integrate, flip the momenta, integrate back: the links must return."""
    dims, N = (4, 4, 4, 4), 2
    lat, geo, prm, U = make(dims, N, noise=0.1, seed=6, lam=1.0, bmass=0.2, G=0.05)
    r = RHMC(15, 1, nstep=3, nstep_gauge=2, traj_length=0.6, error_per_site=1e-10,
             solver=SOLVER_FP64, no_metropolis=True)
    U0 = lat.get_links()
    mom0 = synth.to_ref(dims, synth.links(dims, N, 0.5, 21) - np.eye(N))
    src = [synth.to_ref(dims, synth.tf_source(dims, N, 22, 0.3))]
    a = lat.update_replay(r, mom0, src)
    P1 = lat.get_mom()
    b = lat.update_replay(r, -P1, src)
    U2 = lat.get_links()
    P2 = lat.get_mom()
    assert np.abs(U2 - U0).max() < 1e-8
    assert np.abs(P2 + mom0).max() < 1e-8
    assert abs(a["delta_S"] + b["delta_S"]) < 1e-6


def test_reversibility_mixed_solver():
    """The reversibility test with the mixed-precision solver at the FP64
    true residual 1e-10 per site: links and momenta return to 1e-8, and
    the forward and backward delta S cancel."""
    dims, N = (4, 4, 4, 4), 3
    lat, geo, prm, U = make(dims, N, noise=0.1, seed=6, lam=1.0, bmass=0.2, G=0.05)
    r = RHMC(15, 1, nstep=3, nstep_gauge=2, traj_length=0.6, error_per_site=1e-10,
             solver=SOLVER_MIXED, no_metropolis=True)
    U0 = lat.get_links()
    mom0 = synth.to_ref(dims, synth.links(dims, N, 0.5, 21) - np.eye(N))
    src = [synth.to_ref(dims, synth.tf_source(dims, N, 22, 0.3))]
    a = lat.update_replay(r, mom0, src)
    P1 = lat.get_mom()
    b = lat.update_replay(r, -P1, src)
    assert np.abs(lat.get_links() - U0).max() < 1e-8
    assert np.abs(lat.get_mom() + mom0).max() < 1e-8
    assert abs(a["delta_S"] + b["delta_S"]) < 1e-6


@pytest.mark.parametrize("N", [2, 3])
def test_mixed_and_fp64_integrate_the_same_trajectory(N):
    """Same start links, momenta and pseudofermion sources, error_per_site
    1e-10: the trajectory with the mixed-precision solver ends where the
    FP64 one does (links to 1e-9, delta S to 1e-7 absolute)."""
    dims = (4, 4, 4, 8)
    lat, geo, prm, U = make(dims, N, noise=0.15, seed=8, lam=1.0, bmass=0.2, G=0.05)
    U0 = lat.get_links()
    mom0 = synth.to_ref(dims, synth.links(dims, N, 0.5, 23) - np.eye(N))
    src = [synth.to_ref(dims, synth.tf_source(dims, N, 24, 0.3)) for _ in range(2)]
    out = {}
    for name, solver in (("fp64", SOLVER_FP64), ("mixed", SOLVER_MIXED)):
        lat.set_links(U0)
        r = RHMC(15, 2, nstep=4, nstep_gauge=2, traj_length=1.0, error_per_site=1e-10,
                 solver=solver, no_metropolis=True)
        res = lat.update_replay(r, mom0, src)
        out[name] = (res, lat.get_links())
    assert np.abs(out["mixed"][1] - out["fp64"][1]).max() < 1e-9
    assert abs(out["mixed"][0]["delta_S"] - out["fp64"][0]["delta_S"]) < 1e-7


@pytest.mark.parametrize("vec32", [1, 0])
@pytest.mark.parametrize("N", [2, 3])
def test_mixed_solver_reaches_fp64_residual(N, vec32):
    """Every shift's FP64 true residual within the bound, with FP32 (vec32 =
    1, the default) or FP64 ring and search vectors in the FP32 phase."""
    dims = (4, 4, 4, 8)
    lat, geo, prm, U = make(dims, N, G=0.05)
    lat.mixed_vectors(vec32)
    der = O.compute_derived(geo, prm, U)
    src = synth.tf_source(dims, N, 31)
    shifts = np.array(rhmc_table(15, 1)["shift4"])
    errormin = 1e-20
    s64 = lat.tf(64)
    s64.upload(synth.to_ref(dims, src))
    psim = [lat.tf(64) for _ in shifts]
    it, worst = lat.dev_congrad_multi(s64, psim, shifts, 20000, errormin, mixed=True)
    b2 = O.magsq(src)
    assert worst <= errormin * b2
    for j, s in enumerate(shifts):
        x = synth.from_ref(dims, psim[j].download(), 16, N)
        res = O.DSq(geo, prm, U, der, x) + s * x - src
        assert O.magsq(res) <= 1.5 * errormin * b2


@pytest.mark.parametrize("N", [2, 3, 4])
def test_operator_variants_agree(N):
    """Every operator kernel variant against the oracle: D^dag D in FP64 to
    1e-13 and in FP32 to 2e-6 (relative, max-norm), and one short FP64
    multi-shift solve through each variant (the operator's fused
    axpy + dot epilogue) to the same iteration count and stopping bound."""
    from susy_b200.lattice import FOP_NVARIANTS
    dims = (4, 4, 4, 8)
    lat, geo, prm, U = make(dims, N, G=0.05)
    der = O.compute_derived(geo, prm, U)
    src = synth.tf_source(dims, N, 77)
    want = O.DSq(geo, prm, U, der, src)
    a, b = lat.tf(64), lat.tf(64)
    a.upload(synth.to_ref(dims, src))
    a32, b32 = lat.tf(32), lat.tf(32)
    lat.dev_convert(a, a32)
    shifts = np.array([1e-3, 0.1, 2.0])
    psim = [lat.tf(64) for _ in shifts]
    solves = []
    for v in range(FOP_NVARIANTS):
        lat.fop_variant(64, v)
        lat.fop_variant(32, v)
        lat.dev_DSq(a, b)
        assert rel(synth.from_ref(dims, b.download(), 16, N), want) < 1e-13, v
        lat.dev_DSq(a32, b32)
        lat.dev_convert(b32, b)
        assert rel(synth.from_ref(dims, b.download(), 16, N), want) < 2e-6, v
        it, rsq = lat.dev_congrad_multi(a, psim, shifts, 500, 1e-16)
        solves.append((it, rsq))
    # variants sum the products in different orders: rounding may move the
    # stopping iteration by one
    assert all(abs(x[0] - solves[0][0]) <= 1 for x in solves), solves
    b2 = O.magsq(src)
    assert all(x[1] <= 1e-16 * b2 for x in solves), solves


def test_smdmom_partial_refresh():
    """smdmom (grsource.c:13-40): mom <- c1 mom + c2 G with G the momenta
    ranmom would draw from the same generator state, c1 = exp(-eps friction),
    c1^2 + c2^2 = 1; friction < 0 gives c1 = 0."""
    import math
    dims, N = (4, 4, 2, 4), 3
    a, _, _, U = make(dims, N)
    b, _, _, _ = make(dims, N)
    mom0 = synth.to_ref(dims, synth.links(dims, N, 0.5, 9) - np.eye(N))
    b.ranmom()
    G = b.get_mom()
    for eps, fr in ((0.7, 0.5), (1.0, -1.0)):
        a.seed(41)
        b.seed(41)
        b.ranmom()
        G = b.get_mom()
        a.set_mom(mom0)
        a.smdmom(eps, fr)
        c1 = 0.0 if fr < 0 else math.exp(-eps * fr)
        c2 = math.sqrt(1 - c1 * c1)
        want = c1 * mom0 + c2 * G
        assert np.abs(a.get_mom() - want).max() <= 1e-14 * np.abs(want).max()


def test_smd_friction_zero_carries_the_momenta():
    """friction 0: c1 = 1, c2 = 0, so the momenta enter the next trajectory
    as the last one left them (negated after a rejection), and the integer
    c1 of smdgrsource (grsource.c:79) keeps the pseudofermion source."""
    from susy_b200 import SMD
    dims, N = (4, 4, 4, 4), 2
    lat, _, _, _ = make(dims, N, G=0.05, noise=0.05)
    r0 = RHMC(15, 1, nstep=4, nstep_gauge=2, traj_length=0.5, error_per_site=1e-6,
              algorithm=SMD, friction=0.0)
    t1 = lat.update(r0)
    m1 = lat.get_mom()
    t2 = lat.update(r0)
    # the start action's momentum term is that of the carried-over momenta
    assert abs(t2["start_parts"][4] - float(np.dot(m1, m1))) <= 1e-9 * t2["start_parts"][4]


def test_update_batch_equals_one_by_one():
    """susy_b200_update_batch: independent lattices of different volume and
    NCOL run concurrently and each gets exactly the trajectory it gets alone."""
    from susy_b200 import update_batch
    specs = [((4, 4, 4, 4), 2, 0.1), ((4, 4, 2, 8), 2, 0.2), ((2, 4, 2, 4), 3, 0.15),
             ((6, 6, 6, 6), 2, 0.3)]
    def build():
        out = []
        for i, (dims, N, noise) in enumerate(specs):
            lat = Lattice(dims, N, pbc=-1, lam=1.0 + i, bmass=0.2, G=0.05, iseed=7 + i)
            lat.set_links(synth.to_ref(dims, synth.links(dims, N, noise, 30 + i)))
            # a fixed kernel variant: the autotuner's pick depends on timing,
            # which concurrency changes
            lat.fop_variant(64, 3)
            lat.fop_variant(32, 3)
            out.append(lat)
        return out
    rh = [RHMC(15, 1, nstep=3, nstep_gauge=2, traj_length=0.5, error_per_site=1e-6)
          for _ in specs]
    got = update_batch(build(), rh, threads=4)
    want = [lat.update(r) for lat, r in zip(build(), rh)]
    for g, w in zip(got, want):
        assert g["accept"] == w["accept"] and g["iters"] == w["iters"]
        assert g["delta_S"] == w["delta_S"] and g["start"] == w["start"]


def test_update_batch_with_more_threads_than_sixteen():
    """48 lattices on 48 host threads, each on its own stream (one per
    lattice; the pool once had a 16-thread cap): every lattice's trajectory
    is exactly its solo one."""
    from susy_b200 import update_batch
    vols = [(4, 4, 4, 4), (2, 2, 2, 4), (4, 4, 2, 4), (2, 4, 2, 4)]

    def build():
        out = []
        for i in range(48):
            dims = vols[i % len(vols)]
            lat = Lattice(dims, 2, pbc=-1, lam=[0.5, 1.0, 2.0, 4.0][i % 4], bmass=0.2, G=0.05,
                          iseed=100 + i)
            lat.set_links(synth.to_ref(dims, synth.links(dims, 2, 0.1 + 0.01 * i, 60 + i)))
            lat.fop_variant(64, 3)
            lat.fop_variant(32, 3)
            out.append(lat)
        return out
    rh = [RHMC(15, 1, nstep=2, nstep_gauge=2, traj_length=0.5, error_per_site=1e-6)
          for _ in range(48)]
    lats = build()
    assert len({lat.stream for lat in lats}) == len(lats)
    got = update_batch(lats, rh, threads=48)
    want = [lat.update(r) for lat, r in zip(build(), rh)]
    for g, w in zip(got, want):
        assert g["accept"] == w["accept"] and g["iters"] == w["iters"]
        assert g["delta_S"] == w["delta_S"] and g["start"] == w["start"]


def test_update_batch_refuses_lattices_sharing_a_stream():
    """Two handles on one stream (a worker's graph capture would take in the
    other worker's launches): SUSY_B200_EINVAL before any work; on their own
    streams again, the same batch runs."""
    from susy_b200 import update_batch
    dims = (2, 2, 2, 4)
    lats = []
    for i in range(2):
        lat = Lattice(dims, 2, pbc=-1, lam=1.0, bmass=0.2, G=0.05, iseed=300 + i)
        lat.set_links(synth.to_ref(dims, synth.links(dims, 2, 0.1, 70 + i)))
        lats.append(lat)
    rh = [RHMC(15, 1, nstep=2, nstep_gauge=2, traj_length=0.5, error_per_site=1e-6)
          for _ in lats]
    own = lats[1].stream
    lats[1].set_stream(lats[0].stream)
    with pytest.raises(SusyError):
        update_batch(lats, rh, threads=2)
    with pytest.raises(SusyError):
        update_batch([lats[0], lats[0]], rh, threads=2)
    lats[1].set_stream(None)
    assert lats[1].stream == own
    assert len(update_batch(lats, rh, threads=2)) == 2


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [0, 1])
def test_overlapped_pseudofermion_solves_give_the_same_trajectory(solver):
    """Nroot = 2: the two pseudofermions' solves overlapped on two streams
    (the default) give exactly the trajectory of solving them in turn, with
    the FP64 and with the mixed solver, over two trajectories in a row."""
    dims, N = (4, 4, 4, 8), 2
    def run(pf):
        lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05, iseed=21)
        lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 22)))
        lat.fop_variant(64, 8)
        lat.fop_variant(32, 9)
        assert lat.pf_streams(pf) == 1
        r = RHMC(15, 2, nstep=3, nstep_gauge=2, traj_length=0.5, error_per_site=1e-8,
                 solver=solver)
        res = [lat.update(r) for _ in range(2)]
        return res, lat.get_links()
    (a, la), (b, lb) = run(1), run(0)
    for x, y in zip(a, b):
        assert x["iters"] == y["iters"] and x["accept"] == y["accept"]
        assert x["delta_S"] == y["delta_S"] and x["start"] == y["start"]
    assert np.array_equal(la, lb)
