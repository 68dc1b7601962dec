"""The CUDA path against vectors and regression output of the reference itself.

ops_U{2,3}.npz hold the UNMODIFIED reference's outputs on seeded inputs
(tests/golden/make_golden.py); hmc_U{2,3}.json are the reference's own
regression goldens testsuite/scalar/hmc.U{2,3}.ref (3 trajectories each,
printed to 8-12 significant digits), run here from the same starting
configuration and parameters through the C ABI.
"""
import json
import os

import numpy as np
import pytest

from measlines import mismatches, printed

from susy_b200 import Lattice, RHMC, SOLVER_FP64, SOLVER_MIXED
from susy_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def lattice_from_ops(d):
    dims = tuple(int(x) for x in d["dims"])
    N = int(d["N"])
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.3, G=0.05, kappa_u1=0.4, iseed=41)
    lat.set_links(np.ascontiguousarray(d["links"]))
    return lat, dims, N


def test_u3_operator_matches_reference_on_8x8x8x16():
    """fermion_op(+1), fermion_op(-1) and DSq on an 8^3 x 16 U(3) lattice
    against the reference operator (tests/golden/ops_U3_8x8x8x16.npz, made
    by tests/golden/make_golden_u3_large.py from seeded inputs regenerated
    here): every FP64 kernel variant, 256 sampled sites (both temporal
    boundaries included) to 1e-13 relative, whole-lattice |out|^2 and four
    weighted projections to 1e-12 relative."""
    import importlib.util
    from susy_b200.lattice import FOP_NVARIANTS
    spec = importlib.util.spec_from_file_location(
        "mg", os.path.join(GOLD, "make_golden_u3_large.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    f = np.load(os.path.join(GOLD, "ops_U3_8x8x8x16.npz"))
    dims, N = tuple(int(x) for x in f["dims"]), int(f["N"])
    lat = Lattice(dims, N, pbc=-1, lam=2.0, bmass=0.3, G=0.05)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, mg.LINK_SEED)))
    src = synth.to_ref(dims, synth.tf_source(dims, N, mg.SRC_SEED))
    out = np.zeros(lat.tf_doubles)

    def check(name):
        at, n2, pj = mg.summarise(out, f["sites"])
        want = f[name]
        assert rel(at, want) < 1e-13, name
        assert abs(n2 - float(f["norm2_" + name])) < 1e-12 * float(f["norm2_" + name]), name
        assert np.abs(pj - f["proj_" + name]).max() < 1e-12 * np.abs(f["proj_" + name]).max()

    for v in range(FOP_NVARIANTS):
        lat.fop_variant(64, v)
        lat.fermion_op(src, out, 1)
        check("fop_plus")
        lat.fermion_op(src, out, -1)
        check("fop_minus")
    lat.autotune()
    lat.DSq(src, out)
    check("DSq")


@pytest.mark.parametrize("N", [2, 3])
def test_cuda_matches_reference_vectors(N):
    d = dict(np.load(os.path.join(GOLD, "ops_U%d.npz" % N)))
    lat, dims, N = lattice_from_ops(d)
    pd, D, F, Ui = lat.derived()
    V = lat.V
    m = np.tile(~np.eye(5, dtype=bool).reshape(-1), V)
    pdr = d["plaqdet"].reshape(-1, 2)[m]
    assert rel(pd.reshape(-1, 2)[m], pdr) < 1e-13
    assert rel(D, d["DmuUmu"]) < 1e-13
    assert rel(F, d["Fmunu"]) < 1e-13
    assert rel(Ui, d["Uinv"]) < 1e-13
    out = np.zeros(lat.tf_doubles)
    lat.fermion_op(d["src"], out, 1)
    assert rel(out, d["fop_plus"]) < 1e-13
    lat.fermion_op(d["src"], out, -1)
    assert rel(out, d["fop_minus"]) < 1e-13
    lat.DSq(d["src"], out)
    assert rel(out, d["DSq"]) < 1e-13
    shifts = d["cg_shifts"]
    psim = [np.zeros(lat.tf_doubles) for _ in shifts]
    it, rsq = lat.congrad_multi(d["src"], psim, shifts, 5000, 1e-20)
    assert abs(it - int(d["cg_iters"])) <= 1
    for k, j in enumerate(d["cg_keep"]):
        assert rel(psim[j], d["cg_psim"][k]) < 1e-9
    lat.set_mom(np.zeros(lat.link_doubles))
    fn = lat.fermion_force(0.11, None, [np.ascontiguousarray(s) for s in d["ff_sol"]],
                           d["ff_amp"])
    assert abs(fn - float(d["ff_norm"])) <= 1e-12 * abs(fn)
    assert rel(lat.get_mom(), d["ff_mom"]) < 1e-12
    lat.set_mom(np.ascontiguousarray(d["gf_mom0"]))
    gn = lat.gauge_force(0.07)
    assert abs(gn - float(d["gf_norm"])) <= 1e-12 * abs(gn)
    assert rel(lat.get_mom(), d["gf_mom"]) < 1e-12
    lat.set_mom(np.ascontiguousarray(d["gf_mom0"]))
    full = [np.zeros(lat.tf_doubles) for _ in d["action_amp4"]]
    lat.congrad_multi(d["src"], full, shifts, 5000, 1e-20)
    parts = lat.action([d["src"]], [full], d["action_amp4"], float(d["action_ampdeg4"]))
    for got, want in zip(parts, d["action_parts"]):
        assert abs(got - want) <= 1e-9 * abs(want)
    lat.ranmom()
    assert rel(lat.get_mom(), d["ranmom"]) < 1e-13


def run_hmc_ref(N, solver, **kw):
    gold = json.load(open(os.path.join(GOLD, "hmc_U%d.json" % N)))
    cfg = np.load(os.path.join(GOLD, "config_U%d_4444.npz" % N))
    inp = gold["input"]
    dims = tuple(int(x) for x in cfg["dims"])
    lat = Lattice(dims, N, pbc=int(inp["PBC"]), lam=float(inp["lambda"]),
                  bmass=float(inp["bmass"]), fmass=float(inp["fmass"]),
                  kappa_u1=float(inp["kappa_u1"]), G=float(inp["G"]), iseed=int(inp["iseed"]))
    lat.set_links(synth.to_ref(dims, cfg["links"].astype(np.complex128)))
    r = RHMC(int(inp["Norder"]), int(inp["Nroot"]), nstep=int(inp["nstep"]),
             nstep_gauge=int(inp["nstep_gauge"]), traj_length=float(inp["traj_length"]),
             niter=int(inp["max_cg_iterations"]), error_per_site=float(inp["error_per_site"]),
             solver=solver, **kw)
    out = []
    for _ in gold["trajectories"]:
        t = lat.update(r)
        t["meas"] = lat.measure()
        t["V"] = lat.V
        out.append(t)
    return gold, out


@pytest.mark.parametrize("N", [2, 3])
def test_cuda_reproduces_hmc_regression_output(N):
    gold, got = run_hmc_ref(N, SOLVER_FP64)
    for g, t in zip(got, gold["trajectories"]):
        for a, b in zip(g["start_parts"], t["start_action"][:5]):
            assert abs(a - b) <= 5e-8 * abs(b)
        for a, b in zip(g["end_parts"], t["end_action"][:5]):
            assert abs(a - b) <= 5e-8 * abs(b)
        assert g["accept"] == t["accept"]
        assert abs(g["start"] - t["start_S"]) < 1e-6
        assert abs(g["end"] - t["end_S"]) < 1e-6
        assert abs(g["delta_S"] - t["delta_S"]) <= 1e-3 * max(abs(t["delta_S"]), 1e-3)
        assert abs(g["iters"] - t["it_per_traj"]) <= 12
        assert g["gnorm"] == pytest.approx(t["monitor"][0], rel=2e-3)
        assert g["max_gf"] == pytest.approx(t["monitor"][1], rel=2e-3)
        assert g["fnorm"][0] == pytest.approx(t["monitor"][2], rel=2e-3)
        assert g["max_ff"][0] == pytest.approx(t["monitor"][3], rel=2e-3)
        # the measurement lines printed after the trajectory (control.c:85-138)
        want = dict(t["meas"])
        want["GMES"] = [x for k, x in enumerate(want["GMES"]) if k != 2]
        got_lines = printed(g["meas"], g["V"])
        got_lines["GMES"] = [x for k, x in enumerate(got_lines["GMES"]) if k != 2]
        assert not mismatches(got_lines, want)


@pytest.mark.parametrize("N", [2, 3])
def test_mixed_solver_keeps_the_accept_decisions(N):
    """The mixed-precision solver reaches the same FP64 true-residual bound,
    so the trajectories, accept/reject decisions and delta S are those of
    the golden to the tolerances the FP64 solver meets."""
    gold, got = run_hmc_ref(N, SOLVER_MIXED)
    for g, t in zip(got, gold["trajectories"]):
        assert g["accept"] == t["accept"]
        assert abs(g["start"] - t["start_S"]) < 1e-6
        assert abs(g["end"] - t["end_S"]) < 1e-6
        assert abs(g["delta_S"] - t["delta_S"]) <= 1e-3 * max(abs(t["delta_S"]), 1e-3)


def test_smd_with_full_refresh_is_the_hmc_regression_run():
    """SMD (grsource.c:13-197, update_o.c SMD_ALGORITHM branches) with a
    friction so large that c1 = exp(-traj_length friction) = 0 refreshes the
    momenta completely (c2 = 1, the same gaussian draws as ranmom) and draws
    fresh pseudofermion sources, which is the HMC trajectory: the three
    trajectories of hmc.U2.ref come out again."""
    from susy_b200 import SMD
    gold, got = run_hmc_ref(2, SOLVER_FP64, algorithm=SMD, friction=1e300)
    for g, t in zip(got, gold["trajectories"]):
        assert g["accept"] == t["accept"]
        assert abs(g["start"] - t["start_S"]) < 1e-6
        assert abs(g["end"] - t["end_S"]) < 1e-6


def test_config0_trajectories_match_the_reference():
    """The 4^4 U(2) configuration of the benchmark's first config (identity
    + 0.05 noise links, lambda 1, bmass 0.2, G 0.05, B = kappa_u1 = 0,
    Nroot 1, 10 x 2 steps, error_per_site 1e-10, seed 41) run by the
    reference itself through the harness (tests/golden/config0_U2.json):
    two trajectories on the GPU reproduce its action pieces, delta S,
    accept and force monitors."""
    gold = json.load(open(os.path.join(GOLD, "config0_U2.json")))
    p = gold["params"]
    dims = tuple(p["dims"])
    lat = Lattice(dims, 2, pbc=p["pbc"], lam=p["lam"], bmass=p["bmass"], fmass=p["fmass"],
                  kappa_u1=p["kappa_u1"], G=p["G"], iseed=p["iseed"])
    U = synth.links(dims, 2, gold["links"]["noise"], gold["links"]["seed"])
    lat.set_links(synth.to_ref(dims, U))
    r = RHMC(p["Norder"], p["Nroot"], nstep=p["nstep"], nstep_gauge=p["nstep_gauge"],
             traj_length=p["traj_length"], niter=p["max_cg"],
             error_per_site=p["error_per_site"])
    for t in gold["trajectories"]:
        g = lat.update(r)
        for a, b in zip(g["start_parts"], t["start_action"][:5]):
            assert abs(a - b) <= 5e-8 * max(abs(b), 1e-3)
        for a, b in zip(g["end_parts"], t["end_action"][:5]):
            assert abs(a - b) <= 5e-8 * max(abs(b), 1e-3)
        assert g["accept"] == t["accept"]
        assert abs(g["delta_S"] - t["delta_S"]) <= 1e-3 * max(abs(t["delta_S"]), 1e-3)
        assert abs(g["iters"] - t["it_per_traj"]) <= 12
        assert g["gnorm"] == pytest.approx(t["monitor"][0], rel=2e-3)
        assert g["fnorm"][0] == pytest.approx(t["monitor"][2], rel=2e-3)
