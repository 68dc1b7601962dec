"""Pin the numpy oracle (oracle/susy_np.py) to the reference itself.

Fixtures in tests/golden/ come from the UNMODIFIED reference code
(tests/golden/make_golden.py through oracle/_ref) and from the reference's
own regression output testsuite/scalar/hmc.U2.ref.  CPU only.
"""
import json
import os

import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import synth

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_ops(N):
    return dict(np.load(os.path.join(GOLD, "ops_U%d.npz" % N)))


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def setup(d):
    dims = tuple(int(x) for x in d["dims"])
    N = int(d["N"])
    geo = O.Geometry(dims, -1)
    prm = O.Params(lam=1.0, bmass=0.3, G=0.05, kappa_u1=0.4, fmass=0.0, N=N)
    U = synth.from_ref(dims, d["links"], 5, N)
    return dims, N, geo, prm, U, O.compute_derived(geo, prm, U)


@pytest.mark.parametrize("N", [2, 3])
def test_derived_fields(N):
    d = load_ops(N)
    dims, N, geo, prm, U, der = setup(d)
    V = geo.V
    pd = d["plaqdet"].reshape(V, 5, 5, 2)
    pd = np.moveaxis((pd[..., 0] + 1j * pd[..., 1])[geo.node_index()], 0, -1)
    m = ~np.eye(5, dtype=bool)
    assert rel(der.plaqdet[m], pd[m]) < 1e-13
    assert rel(der.DmuUmu, synth.from_ref(dims, d["DmuUmu"], 1, N)[0]) < 1e-13
    assert rel(der.Fmunu, synth.from_ref(dims, d["Fmunu"], 10, N)) < 1e-13
    assert rel(der.Uinv, synth.from_ref(dims, d["Uinv"], 5, N)) < 1e-13


@pytest.mark.parametrize("N", [2, 3])
def test_fermion_op_and_dsq(N):
    d = load_ops(N)
    dims, N, geo, prm, U, der = setup(d)
    src = synth.from_ref(dims, d["src"], 16, N)
    for sign, key in ((1, "fop_plus"), (-1, "fop_minus")):
        got = O.fermion_op(geo, prm, U, der, src, sign)
        assert rel(got, synth.from_ref(dims, d[key], 16, N)) < 1e-13
    assert rel(O.DSq(geo, prm, U, der, src), synth.from_ref(dims, d["DSq"], 16, N)) < 1e-13


@pytest.mark.parametrize("N", [2, 3])
def test_congrad_multi(N):
    d = load_ops(N)
    dims, N, geo, prm, U, der = setup(d)
    src = synth.from_ref(dims, d["src"], 16, N)
    psim, it, rsq = O.congrad_multi(geo, prm, U, der, src, d["cg_shifts"], 5000, 1e-20)
    assert abs(it - int(d["cg_iters"])) <= 1
    for k, j in enumerate(d["cg_keep"]):
        assert rel(psim[j], synth.from_ref(dims, d["cg_psim"][k], 16, N)) < 1e-9


@pytest.mark.parametrize("N", [2, 3])
def test_forces(N):
    d = load_ops(N)
    dims, N, geo, prm, U, der = setup(d)
    sols = [synth.from_ref(dims, s, 16, N) for s in d["ff_sol"]]
    mom = np.zeros_like(U)
    fn = O.fermion_force(geo, prm, U, der, mom, 0.11, sols, d["ff_amp"])
    assert abs(fn - float(d["ff_norm"])) <= 1e-12 * abs(fn)
    assert rel(mom, synth.from_ref(dims, d["ff_mom"], 5, N)) < 1e-12
    mom = synth.from_ref(dims, d["gf_mom0"], 5, N)
    gn = O.gauge_force(geo, prm, U, der, mom, 0.07)
    assert abs(gn - float(d["gf_norm"])) <= 1e-12 * abs(gn)
    assert rel(mom, synth.from_ref(dims, d["gf_mom"], 5, N)) < 1e-12


@pytest.mark.parametrize("N", [2, 3])
def test_action_and_ranmom(N):
    d = load_ops(N)
    dims, N, geo, prm, U, der = setup(d)
    src = synth.from_ref(dims, d["src"], 16, N)
    psim, _, _ = O.congrad_multi(geo, prm, U, der, src, d["cg_shifts"], 5000, 1e-20)
    mom = synth.from_ref(dims, d["gf_mom0"], 5, N)
    g, b, dt, f, p = O.action_parts(geo, prm, U, der, mom, [src], [psim], d["action_amp4"],
                                    float(d["action_ampdeg4"]))
    want = d["action_parts"]
    for got, w in zip([g, b, dt, f[0], p], want):
        assert abs(got - w) <= 1e-10 * abs(w)
    st = O.site_prn_lex(geo, 41)
    assert rel(O.ranmom(st, N), synth.from_ref(dims, d["ranmom"], 5, N)) == 0.0


def test_oracle_reproduces_hmc_U2_ref():
    """First trajectory of testsuite/scalar/hmc.U2.ref from config.U2.4444."""
    gold = json.load(open(os.path.join(GOLD, "hmc_U2.json")))
    cfg = np.load(os.path.join(GOLD, "config_U2_4444.npz"))
    inp = gold["input"]
    dims = tuple(int(x) for x in cfg["dims"])
    N = 2
    U = cfg["links"].astype(np.complex128)
    geo = O.Geometry(dims, int(inp["PBC"]))
    prm = O.Params(lam=float(inp["lambda"]), bmass=float(inp["bmass"]),
                   fmass=float(inp["fmass"]), kappa_u1=float(inp["kappa_u1"]),
                   G=float(inp["G"]), N=N)
    from susy_b200.rhmc_tables import rhmc
    eps = float(inp["error_per_site"])
    h = O.HMCState(geo=geo, prm=prm, U=U, mom=np.zeros_like(U),
                   site_prn=O.site_prn_lex(geo, int(inp["iseed"])),
                   node_prn=O.node_prn(geo, int(inp["iseed"])),
                   rhmc=O.RHMC(**rhmc(int(inp["Norder"]), int(inp["Nroot"]))),
                   Nroot=int(inp["Nroot"]), nsteps=(int(inp["nstep"]), int(inp["nstep_gauge"])),
                   traj_length=float(inp["traj_length"]), niter=int(inp["max_cg_iterations"]),
                   rsqmin=eps * eps)
    h.refresh()
    r = O.update(h)
    t0 = gold["trajectories"][0]
    act = h.log[0]
    start_parts = [act[1], act[2], act[3], act[4][0], act[5]]
    for got, want in zip(start_parts, t0["start_action"][:5]):
        assert abs(got - want) <= 5e-8 * abs(want)
    assert r["accept"] == t0["accept"]
    assert abs(r["start"] - t0["start_S"]) < 1e-6
    assert abs(r["end"] - t0["end_S"]) < 1e-6
    assert abs(r["delta_S"] - t0["delta_S"]) < 1e-3 * max(abs(t0["delta_S"]), 1e-3)
    assert abs(r["iters"] - t0["it_per_traj"]) <= 12


@pytest.mark.parametrize("N", [2, 3])
def test_measurements(N):
    """control.c:85-138 measurements of the oracle against the reference's
    own functions on the same links (ops fixtures): link_trace, ploop in all
    directions with and without polar projection, plaquette, scalar_eig and
    gauge_action to 1e-12; measure_det and widths, which the reference only
    prints (%.6g), to printed precision."""
    d = load_ops(N)
    dims, N, geo, prm, U, der = setup(d)
    m = O.measurements(geo, prm, U, der)
    assert rel(m["linktr"], d["meas_linktr"]) < 1e-12
    assert rel(m["link_det"], d["meas_link_det"]) < 1e-12
    assert rel(np.array([m["linktr_ave"], m["linktr_width"], m["det_ave"], m["det_width"]]),
               d["meas_lt_scalars"]) < 1e-12
    assert rel(np.concatenate([m["lines"], m["lines_polar"]]), d["meas_lines"]) < 1e-12
    assert abs(m["ploop_mod"] - float(d["meas_ploop_mod"])) < 1e-12 * abs(m["ploop_mod"])
    assert rel(np.array([m["ss_plaq"], m["st_plaq"]]), d["meas_plaq"]) < 1e-12
    assert rel(np.array(m["uubar"]), d["meas_uubar"]) < 1e-12
    assert rel(np.array(m["polar"]), d["meas_polar"]) < 1e-12
    assert abs(m["gauge_action"] - float(d["meas_gauge_action"])) < 1e-12 * m["gauge_action"]
    assert rel(m["det"], d["meas_det"]) < 3e-5
    assert rel(m["widths"], d["meas_widths"]) < 3e-5


@pytest.mark.parametrize("N", [2, 3])
def test_measurements_on_the_regression_start_config(N):
    """FLINK and FLINK_DET of the regression run's starting configuration
    (testsuite/scalar/hmc.U{2,3}.ref, printed before the first trajectory)."""
    from measlines import mismatches, printed
    gold = json.load(open(os.path.join(GOLD, "hmc_U%d.json" % N)))
    cfg = np.load(os.path.join(GOLD, "config_U%d_4444.npz" % N))
    dims = tuple(int(x) for x in cfg["dims"])
    geo = O.Geometry(dims, -1)
    prm = O.Params(lam=float(gold["input"]["lambda"]), G=float(gold["input"]["G"]), N=N)
    U = cfg["links"].astype(np.complex128)
    m = O.measurements(geo, prm, U, O.compute_derived(geo, prm, U))
    assert not mismatches(printed(m, geo.V), gold["start_meas"])


def test_oracle_operator_matches_reference_on_8x8x8x16_u3():
    """The numpy restatement against the reference operator on the 8^3 x 16
    U(3) fixture (sampled sites to 1e-13 relative, whole-lattice norms and
    weighted projections to 1e-12)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mg", os.path.join(GOLD, "make_golden_u3_large.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    f = np.load(os.path.join(GOLD, "ops_U3_8x8x8x16.npz"))
    dims, N = tuple(int(x) for x in f["dims"]), int(f["N"])
    geo = O.Geometry(dims, -1)
    prm = O.Params(lam=2.0, bmass=0.3, G=0.05, N=N)
    U = synth.links(dims, N, 0.2, mg.LINK_SEED)
    der = O.compute_derived(geo, prm, U)
    src = synth.tf_source(dims, N, mg.SRC_SEED)
    for name, val in (("fop_plus", O.fermion_op(geo, prm, U, der, src, 1)),
                      ("fop_minus", O.fermion_op(geo, prm, U, der, src, -1))):
        at, n2, pj = mg.summarise(synth.to_ref(dims, val), f["sites"])
        want = f[name]
        assert np.abs(at - want).max() / np.abs(want).max() < 1e-13, name
        assert abs(n2 - float(f["norm2_" + name])) < 1e-12 * float(f["norm2_" + name]), name
        wp = f["proj_" + name]
        assert np.abs(pj - wp).max() < 1e-12 * np.abs(wp).max(), name
