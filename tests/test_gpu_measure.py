"""GPU parity of the per-trajectory measurements (control.c:85-138):
link_trace, ploop (every direction, with and without polar projection),
plaquette, gauge_action, measure_det, widths and scalar_eig, computed by
susy_b200_measure on the device.

Against the oracle on seeded links for NCOL = 2, 3, 4 to 1e-11 (the
eigenvalues come from a Jacobi solver on the device and LAPACK in the
oracle); against the reference's own outputs on the fixture links; against
the lines hmc.U{2,3}.ref prints for the regression start configuration (to
printed precision); and after each regression trajectory in
test_gpu_golden.py.
"""
import json
import os

import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import Lattice, synth

from measlines import mismatches, printed

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def flat(m):
    keys = ["linktr", "link_det", "linktr_ave", "linktr_width", "det_ave", "det_width",
            "ploop_re", "ploop_im", "ploop_mod", "ss_plaq", "st_plaq", "gauge_action"]
    parts = [np.atleast_1d(np.asarray(m[k], dtype=float)) for k in keys]
    parts += [np.asarray(m["lines"]).real, np.asarray(m["lines"]).imag,
              np.asarray(m["lines_polar"]).real, np.asarray(m["lines_polar"]).imag,
              np.asarray(m["det"]), np.asarray(m["widths"]),
              np.asarray(m["uubar"]).ravel(), np.asarray(m["polar"]).ravel()]
    return np.concatenate(parts)


@pytest.mark.parametrize("dims,N", [((4, 4, 2, 4), 2), ((2, 4, 2, 4), 3), ((2, 2, 2, 4), 4),
                                    ((4, 2, 4, 6), 3)])
def test_measure_matches_oracle(dims, N):
    U = synth.links(dims, N, 0.3, 17)
    prm = O.Params(lam=1.5, G=0.05, N=N)
    lat = Lattice(dims, N, pbc=-1, lam=1.5, G=0.05)
    lat.set_links(synth.to_ref(dims, U))
    geo = O.Geometry(dims, -1)
    want = flat(O.measurements(geo, prm, U, O.compute_derived(geo, prm, U)))
    got = flat(lat.measure())
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-3)
    assert err.max() < 1e-11, (int(err.argmax()), got[err.argmax()], want[err.argmax()])
    ss, st = lat.plaquette()
    assert ss == pytest.approx(lat.measure()["ss_plaq"], rel=1e-15)


@pytest.mark.parametrize("N", [2, 3])
def test_measure_matches_reference_outputs(N):
    d = dict(np.load(os.path.join(GOLD, "ops_U%d.npz" % N)))
    dims = tuple(int(x) for x in d["dims"])
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.3, G=0.05, kappa_u1=0.4)
    lat.set_links(d["links"])
    m = lat.measure()
    r = lambda a, b: float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(b).max())
    assert r(m["linktr"], d["meas_linktr"]) < 1e-12
    assert r(m["link_det"], d["meas_link_det"]) < 1e-12
    assert r(np.concatenate([m["lines"], m["lines_polar"]]), d["meas_lines"]) < 1e-12
    assert r([m["ss_plaq"], m["st_plaq"]], d["meas_plaq"]) < 1e-13
    assert r(np.array(m["uubar"]), d["meas_uubar"]) < 1e-11
    assert r(np.array(m["polar"]), d["meas_polar"]) < 1e-11
    assert abs(m["gauge_action"] - float(d["meas_gauge_action"])) < 1e-12 * m["gauge_action"]
    assert r(m["det"], d["meas_det"]) < 3e-5
    assert r(m["widths"], d["meas_widths"]) < 3e-5


@pytest.mark.parametrize("N", [2, 3])
def test_measure_regression_start_config(N):
    gold = json.load(open(os.path.join(GOLD, "hmc_U%d.json" % N)))
    cfg = np.load(os.path.join(GOLD, "config_U%d_4444.npz" % N))
    dims = tuple(int(x) for x in cfg["dims"])
    lat = Lattice(dims, N, pbc=-1, lam=float(gold["input"]["lambda"]), G=float(gold["input"]["G"]))
    lat.set_links(synth.to_ref(dims, cfg["links"].astype(np.complex128)))
    assert not mismatches(printed(lat.measure(), lat.V), gold["start_meas"])
