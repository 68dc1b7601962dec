"""GPU parity of the multi-shift CG (congrad_multi.c:26-221).

The FP64 device solver runs the reference's recurrences; on the same input
it must take the same number of iterations as the oracle (the FP64
reductions are summed in a different order, so +-1 is allowed) and its
solutions must agree to 1e-9 relative.  Every shift's true residual
|(D^dag D + sigma_j) psi_j - src|^2 must be below the stopping bound
errormin |src|^2 times a small safety factor (the reference stops on the
iterated residual).
"""
import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import Lattice
from susy_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,N,errormin", [((4, 4, 4, 4), 2, 1e-20),
                                             ((4, 4, 4, 4), 3, 1e-14),
                                             ((2, 2, 2, 4), 2, 1e-20)])
def test_congrad_multi_matches_oracle(dims, N, errormin):
    U = synth.links(dims, N, 0.2, 4)
    lat = Lattice(dims, N, pbc=-1, G=0.05)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, -1)
    prm = O.Params(G=0.05, N=N)
    der = O.compute_derived(geo, prm, U)
    src = synth.tf_source(dims, N, seed=8)
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    want, wit, wrsq = O.congrad_multi(geo, prm, U, der, src, shifts, 5000, errormin)
    psim = [np.zeros(lat.tf_doubles) for _ in shifts]
    it, rsq = lat.congrad_multi(synth.to_ref(dims, src), psim, shifts, 5000, errormin)
    assert abs(it - wit) <= 1
    src_n = O.magsq(src)
    for j, s in enumerate(shifts):
        got = synth.from_ref(dims, psim[j], 16, N)
        assert np.abs(got - want[j]).max() / np.abs(want[j]).max() < 1e-9
        res = O.DSq(geo, prm, U, der, got) + s * got - src
        assert O.magsq(res) <= 100 * errormin * src_n


def test_congrad_multi_maxcg_returns_iterations():
    dims, N = (4, 4, 4, 4), 2
    lat = Lattice(dims, N, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 4)))
    src = synth.to_ref(dims, synth.tf_source(dims, N, seed=8))
    shifts = synth.geometric_shifts(5, 1e-3, 1.0)
    psim = [np.zeros(lat.tf_doubles) for _ in shifts]
    it, rsq = lat.congrad_multi(src, psim, shifts, 7, 1e-20)
    assert it == 7 and rsq > 0


@pytest.mark.parametrize("maxcg,errormin", [(5000, 1e-20), (13, 1e-20), (7, 1e-20),
                                            (5000, 1e-8)])
def test_blocked_update_matches_per_iteration(maxcg, errormin):
    """The blocked vector update (one pass per 8 iterations) against the
    per-iteration update of congrad_multi.c:109-150: same iteration count,
    same iterated residual and solutions to 1e-11 relative, including solves
    that end inside a block (MaxCG 7 and 13) and shifts that freeze
    mid-block (the loose 1e-8 stop)."""
    dims, N = (4, 4, 4, 4), 3
    lat = Lattice(dims, N, pbc=-1, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 4)))
    src = synth.to_ref(dims, synth.tf_source(dims, N, seed=8))
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    out = {}
    for on in (0, 1):
        lat.cg_blocked(on)
        psim = [np.zeros(lat.tf_doubles) for _ in shifts]
        it, rsq = lat.congrad_multi(src, psim, shifts, maxcg, errormin)
        out[on] = (it, rsq, psim)
    assert out[0][0] == out[1][0]
    assert abs(out[0][1] - out[1][1]) <= 1e-9 * out[0][1]
    for a, b in zip(out[0][2], out[1][2]):
        assert np.abs(a - b).max() <= 1e-11 * np.abs(a).max()


@pytest.mark.parametrize("mixed", [False, True])
def test_graph_replay_matches_plain_launches(mixed):
    """The solver's iteration chunks replayed as CUDA graphs give the same
    solve, bit for bit, as launching the kernels one by one."""
    dims, N = (4, 4, 4, 8), 2
    lat = Lattice(dims, N, pbc=-1, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 4)))
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, N, seed=8)))
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    out = {}
    for on in (0, 1):
        lat.use_graphs(on)
        psim = [lat.tf(64) for _ in shifts]
        it, rsq = lat.dev_congrad_multi(src, psim, shifts, 5000, 1e-20, mixed=mixed)
        out[on] = (it, rsq, [p.download() for p in psim])
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    for a, b in zip(out[0][2], out[1][2]):
        assert np.array_equal(a, b)


def test_microbench_operator_precisions_and_solvers():
    """The operator and solver microbenchmark configuration (8^4 U(2),
    links identity + 0.2 noise, lambda 1, bmass 0.2, G 0.05): D^dag D in
    FP64 and FP32 against the FP64 oracle on complex-Gaussian sources, and
    the 15-shift solve (shifts 1e-5 ... 1e3, FP64 true residual 1e-10 per
    site) with the FP64 and the mixed solver: same bound for every shift,
    solutions agreeing to 1e-8."""
    dims, N = (8, 8, 8, 8), 2
    U = synth.links(dims, N, 0.2, 1)
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, -1)
    prm = O.Params(lam=1.0, bmass=0.2, G=0.05, N=N)
    der = O.compute_derived(geo, prm, U)
    for k in range(2):
        src = synth.tf_source(dims, N, 50 + k)
        want = O.DSq(geo, prm, U, der, src)
        a, b = lat.tf(64), lat.tf(64)
        a.upload(synth.to_ref(dims, src))
        lat.dev_DSq(a, b)
        got = synth.from_ref(dims, b.download(), 16, N)
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
        a32, b32 = lat.tf(32), lat.tf(32)
        lat.dev_convert(a, a32)
        lat.dev_DSq(a32, b32)
        lat.dev_convert(b32, b)
        got = synth.from_ref(dims, b.download(), 16, N)
        assert np.abs(got - want).max() <= 2e-6 * np.abs(want).max()
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, N, 60)))
    b2 = float(np.dot(src.download(), src.download()))
    sols = {}
    for mixed in (False, True):
        psim = [lat.tf(64) for _ in shifts]
        lat.dev_congrad_multi(src, psim, shifts, 20000, 1e-20, mixed=mixed)
        sols[mixed] = [p.download() for p in psim]
        t = lat.tf(64)
        for j, s in enumerate(shifts):
            lat.dev_DSq(psim[j], t)
            r = src.download() - t.download() - s * sols[mixed][j]
            assert float(np.dot(r, r)) <= 1.5e-20 * b2
    for x, y in zip(sols[False], sols[True]):
        assert np.abs(x - y).max() <= 1e-8 * np.abs(x).max()


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [True, False])
def test_mixed_corrections_meet_bound(fp32):
    """The mixed solver switched to the FP32 operator early (|r| < 1e-2
    |src|), so that most shifts need per-shift correction solves: with the
    FP32 corrections (iterative refinement against the FP64 true residual)
    and with FP64 ones, every shift ends at the FP64 true-residual bound and
    agrees with the FP64 solver's solution."""
    dims, N = (8, 8, 8, 8), 2
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 1)))
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, N, 61)))
    b2 = float(np.dot(src.download(), src.download()))
    ref = [lat.tf(64) for _ in shifts]
    lat.dev_congrad_multi(src, ref, shifts, 20000, 1e-20, mixed=False)
    lat.mixed_params(1e-2, 1e-2)
    lat.mixed_correction(fp32)
    psim = [lat.tf(64) for _ in shifts]
    lat.dev_congrad_multi(src, psim, shifts, 20000, 1e-20, mixed=True)
    t = lat.tf(64)
    for j, s in enumerate(shifts):
        lat.dev_DSq(psim[j], t)
        x = psim[j].download()
        r = src.download() - t.download() - s * x
        assert float(np.dot(r, r)) <= 1.5e-20 * b2
        y = ref[j].download()
        assert np.abs(x - y).max() <= 1e-8 * np.abs(y).max()
    assert lat.lib.susy_b200_mixed_correction(lat.h, 2) < 0


@pytest.mark.parametrize("interval", [50, 0])
def test_mixed_fp32_from_start_with_fixed_reliable_updates(interval):
    """The microbenchmark's literal schedule: the FP32 operator from the
    first iteration (fp32_below = 1) with the FP64 true residual replacing
    the iterated one every 50 iterations (rounded up to a block boundary)
    or on the residual trigger: every shift still ends at the FP64 true
    residual bound and agrees with the FP64 solver's solution."""
    dims, N = (8, 8, 8, 8), 2
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 1)))
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, N, 62)))
    b2 = float(np.dot(src.download(), src.download()))
    ref = [lat.tf(64) for _ in shifts]
    it64, _ = lat.dev_congrad_multi(src, ref, shifts, 20000, 1e-20, mixed=False)
    lat.mixed_params(1.0, 1e-2)
    lat.mixed_reliable_interval(interval)
    psim = [lat.tf(64) for _ in shifts]
    it, _ = lat.dev_congrad_multi(src, psim, shifts, 20000, 1e-20, mixed=True)
    assert it < 3 * it64
    t = lat.tf(64)
    for j, s in enumerate(shifts):
        lat.dev_DSq(psim[j], t)
        x = psim[j].download()
        r = src.download() - t.download() - s * x
        assert float(np.dot(r, r)) <= 1.5e-20 * b2
        y = ref[j].download()
        assert np.abs(x - y).max() <= 1e-8 * np.abs(y).max()
    assert lat.lib.susy_b200_mixed_reliable_interval(lat.h, -1) < 0


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [0, 1])
def test_host_congrad_multi_early_copies(solver):
    """susy_b200_congrad_multi into page-locked host buffers hands each
    frozen shift's solution back while the solve continues: the solutions
    are the ones pageable buffers get (copied after the solve), with the
    FP64 and the mixed solver."""
    import torch
    dims, N = (8, 8, 8, 8), 2
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 1)))
    lat.set_solver(solver)
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    src = synth.to_ref(dims, synth.tf_source(dims, N, 62))
    pinned = [torch.empty(lat.tf_doubles, dtype=torch.float64, pin_memory=True).numpy()
              for _ in shifts]
    pageable = [np.empty(lat.tf_doubles) for _ in shifts]
    for outs in (pinned, pageable):
        for o in outs:
            o[:] = np.nan
        lat.congrad_multi(src, outs, shifts, 20000, 1e-20)
    for a, b in zip(pinned, pageable):
        assert np.array_equal(a, b)
