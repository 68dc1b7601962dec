"""The reference's own program, with its hot path taken from libsusy_b200.

oracle/build_ref.sh <N> shim<N> links the reference's susy_hmc (its setup,
update() driver with the Metropolis step, grsource, ranmom, actions and
every measurement of control.c, all unmodified) with
susy_b200/shim/b200_shim.c in place of fermion_op, DSq, congrad_multi,
fermion_force, gauge_force and update_u, which go to the GPU through the C
ABI with links and momenta handed over in place from lattice[] (stride
sizeof(site)).  Run on the reference's regression input (the parameters of
testsuite/in.U<N>.hmc and its starting configuration config.U<N>.4444, both
regenerated here from tests/golden), its stdout must reproduce the
regression output testsuite/scalar/hmc.U<N>.ref (tests/golden/hmc_U<N>.json)
to the tolerances the FP64 path meets through the Python binding: action
pieces 5e-8 relative, start/end S 1e-6, delta S 1e-3 relative, accept,
CG iterations per trajectory +-12, force monitors 2e-3 relative, and every
measurement line to its printed digits (the reference's run_tests:32
compares the text with only its timing lines ignored).
"""
import importlib.util
import json
import os
import subprocess

import numpy as np
import pytest

from measlines import mismatches

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")


def parser():
    spec = importlib.util.spec_from_file_location("mg", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.parse_hmc_text


@pytest.mark.parametrize("N", [2, 3])
def test_reference_program_with_the_shim_reproduces_its_regression_output(N, tmp_path):
    from susy_b200 import io_lat
    exe = os.path.join(ROOT, "oracle", "_ref", "n%d" % N, "susy_hmc_b200")
    if not os.path.exists(exe):
        pytest.skip("shimmed reference program not built (oracle/build_ref.sh %d shim%d "
                    "needs the reference sources)" % (N, N))
    gold = json.load(open(os.path.join(GOLD, "hmc_U%d.json" % N)))
    cfg = np.load(os.path.join(GOLD, "config_U%d_4444.npz" % N))
    dims = tuple(int(x) for x in cfg["dims"])
    inp = gold["input"]
    io_lat.write_gauge(str(tmp_path / inp["reload_serial"]), dims,
                       cfg["links"].astype(np.complex128))
    text = "\n".join("%s %s" % kv for kv in inp.items()) + "\nforget\n"
    run = subprocess.run([exe], input=text, cwd=str(tmp_path), capture_output=True, text=True,
                         timeout=900)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    assert "susy_b200: hot path on the GPU" in run.stdout
    got = parser()(run.stdout)
    assert len(got["trajectories"]) == len(gold["trajectories"])
    for g, t in zip(got["trajectories"], gold["trajectories"]):
        for a, b in zip(g["start_action"], t["start_action"]):
            assert abs(a - b) <= 5e-8 * abs(b)
        for a, b in zip(g["end_action"], t["end_action"]):
            assert abs(a - b) <= 5e-8 * abs(b)
        assert g["accept"] == t["accept"]
        assert abs(g["start_S"] - t["start_S"]) < 1e-6
        assert abs(g["end_S"] - t["end_S"]) < 1e-6
        assert abs(g["delta_S"] - t["delta_S"]) <= 1e-3 * max(abs(t["delta_S"]), 1e-3)
        assert abs(g["it_per_traj"] - t["it_per_traj"]) <= 12
        for a, b in zip(g["monitor"], t["monitor"]):
            assert a == pytest.approx(b, rel=2e-3)
        want = dict(t["meas"])
        have = dict(g["meas"])
        # GMES carries the CG iteration count of the last solve
        want["GMES"] = [x for k, x in enumerate(want["GMES"]) if k != 2]
        have["GMES"] = [x for k, x in enumerate(have["GMES"]) if k != 2]
        assert not mismatches(have, want)
    for tag, vals in gold["start_meas"].items():
        assert not mismatches({tag: got["start_meas"][tag]}, {tag: vals})


def run_app(prog, N, tmp_path):
    """Run the reference's susy_<prog> linked with the shim on its regression
    input; returns the parsed output and the golden."""
    from susy_b200 import io_lat
    exe = os.path.join(ROOT, "oracle", "_ref", "n%d%s" % (N, prog), "susy_%s_b200" % prog)
    if not os.path.exists(exe):
        pytest.skip("shimmed susy_%s not built (oracle/build_ref.sh %s%d needs the "
                    "reference sources)" % (prog, prog, N))
    gold = json.load(open(os.path.join(GOLD, "%s_U%d.json" % (prog, N))))
    cfg = np.load(os.path.join(GOLD, "config_U%d_4444.npz" % N))
    dims = tuple(int(x) for x in cfg["dims"])
    conf = dict(gold["input"])["reload_serial"]
    io_lat.write_gauge(str(tmp_path / conf), dims, cfg["links"].astype(np.complex128))
    text = "\n".join("%s %s" % (k, v) for k, v in gold["input"]) + "\nforget\n"
    run = subprocess.run([exe], input=text, cwd=str(tmp_path), capture_output=True, text=True,
                         timeout=900)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    assert "susy_b200: hot path on the GPU" in run.stdout
    spec = importlib.util.spec_from_file_location("ma", os.path.join(GOLD, "make_golden_apps.py"))
    ma = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ma)
    return ma.parse_output(run.stdout), gold


@pytest.mark.parametrize("N", [2, 3])
def test_reference_chebyshev_program_with_the_shim(N, tmp_path):
    """susy_cheb (chebyshev.c:45,60 apply DSq to stochastic sources) with
    DSq from the library reproduces cheb.U<N>.ref: every Chebyshev
    coefficient to its printed 8 digits, its error to its 4 digits."""
    got, gold = run_app("cheb", N, tmp_path)
    assert len(got["chebyshev"]) == len(gold["chebyshev"]) > 0
    for g, w in zip(got["chebyshev"], gold["chebyshev"]):
        assert g[0] == w[0]
        assert abs(g[1] - w[1]) <= 3e-7 * abs(w[1]) + 1e-12, (g, w)
        assert abs(g[2] - w[2]) <= 3e-3 * abs(w[2]) + 1e-12, (g, w)


@pytest.mark.parametrize("N", [2, 3])
def test_reference_mode_number_program_with_the_shim(N, tmp_path):
    """susy_mode (modenumber.c:26,63,66 call congrad_multi on stochastic
    sources, error_per_site 1e-5) with congrad_multi from the library
    reproduces mode.U<N>.ref: the step-function line exactly, every mode
    number to 1e-5 relative (the solves stop at a residual of 1e-5 per
    site, and the solver's summation order may move the stop by an
    iteration), its error to its printed 4 digits."""
    got, gold = run_app("mode", N, tmp_path)
    assert got["step"] == gold["step"]
    assert len(got["mode"]) == len(gold["mode"]) > 0
    for g, w in zip(got["mode"], gold["mode"]):
        assert g[0] == w[0]
        assert abs(g[1] - w[1]) <= 1e-5 * abs(w[1]), (g, w)
        assert abs(g[2] - w[2]) <= 3e-3 * abs(w[2]) + 1e-12, (g, w)
