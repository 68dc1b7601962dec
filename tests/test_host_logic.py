"""Host-side logic: layouts, gauge-file I/O, RHMC tables, replica plumbing."""
import os

import numpy as np
import pytest

from susy_b200 import synth
from susy_b200.io_lat import read_gauge, write_gauge
from susy_b200.rhmc_tables import TABLES, rhmc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (2, 2, 2, 2), (12, 12, 12, 24), (4, 2, 6, 8)])
def test_node_index_is_a_bijection_even_sites_first(dims):
    ni = synth.node_index(dims)
    V = int(np.prod(dims))
    assert sorted(ni.tolist()) == list(range(V))
    i = np.arange(V)
    x, y = i % dims[0], (i // dims[0]) % dims[1]
    z, t = (i // (dims[0] * dims[1])) % dims[2], i // (dims[0] * dims[1] * dims[2])
    even = (x + y + z + t) % 2 == 0
    assert ni[even].max() < V // 2 <= ni[~even].min()


def test_ref_layout_roundtrip():
    dims, N = (4, 2, 2, 4), 3
    f = synth.tf_source(dims, N, 5)
    assert np.array_equal(synth.from_ref(dims, synth.to_ref(dims, f), 16, N), f)


def test_gauge_file_roundtrip(tmp_path):
    dims, N = (4, 4, 2, 2), 3
    U = synth.links(dims, N, 0.3, 7).astype(np.complex64).astype(np.complex128)
    p = str(tmp_path / "cfg")
    s29, s31 = write_gauge(p, dims, U, stamp="test")
    d2, n2, U2, info = read_gauge(p)
    assert d2 == dims and n2 == N and info["checksum_ok"]
    assert (info["sum29"], info["sum31"]) == (s29, s31)
    assert np.array_equal(U2, U)


def test_reference_config_checksums_from_fixture():
    cfg = np.load(os.path.join(GOLD, "config_U2_4444.npz"))
    from susy_b200.io_lat import checksums
    U = cfg["links"]
    a = np.moveaxis(U, 0, 1)
    words = np.stack([a.real, a.imag], -1).astype("<f4").reshape(-1).view("<u4")
    # checksums of the reference's own config.U2.4444 (its .info file)
    assert checksums(words) == (0x632f69a0, 0x0bb8becc)
    assert (int(cfg["sum29"]), int(cfg["sum31"])) == (0x632f69a0, 0x0bb8becc)


def test_rhmc_degree15_tables():
    t1 = rhmc(15, 1)
    assert len(t1["amp4"]) == 15 and t1["ampdeg4"] == pytest.approx(9.5797060554725838e-02)
    assert t1["shift4"][0] == pytest.approx(3.1085594175442315e-08)
    t2 = rhmc(15, 2)
    assert all(np.diff(t2["shift4"]) > 0)
    assert (15, 1) in TABLES and (15, 2) in TABLES


def test_geometric_shifts():
    s = synth.geometric_shifts(15, 1e-5, 1e3)
    assert s[0] == pytest.approx(1e-5) and s[-1] == pytest.approx(1e3)


def test_reference_arm_assembles_a_solve_from_one_step_of_samples():
    """bench.py's CPU reference arm: one timed step samples 1, 8 and 15 live
    shifts; the per-iteration time a + b k is fitted from them and summed
    over the recorded FP64 schedule, divided by the replicas."""
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    arm = bench.CpuArm.__new__(bench.CpuArm)
    arm.P, arm.kind = 16, "reference"
    a, b = 2.5, 0.1
    arm.samples = [(k, a + b * k) for k in bench.REF_SAMPLE_SHIFTS]
    iters, live_sum, _ = bench.solve_profile()
    v, desc = arm.value()
    assert v == pytest.approx((iters * a + b * live_sum) / 16, rel=1e-9)
    assert "16 single-core replicas" in desc
    assert len(set(bench.REF_SAMPLE_SHIFTS)) >= 2


def _bench_module():
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def test_operator_variant_count_agrees_across_header_binding_and_kernels():
    """ms_per_variant arrays are sized by SUSY_B200_FOP_NVARIANTS: the C
    header, the ctypes binding and the kernels' variant enum must agree."""
    import re
    from susy_b200.lattice import FOP_NVARIANTS
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    hdr = open(os.path.join(root, "include", "susy_b200.h")).read()
    kern = open(os.path.join(root, "susy_b200", "csrc", "kernels.h")).read()
    n_hdr = int(re.search(r"#define SUSY_B200_FOP_NVARIANTS (\d+)", hdr).group(1))
    n_enum = int(re.search(r"FOP_NVARIANTS = (\d+)", kern).group(1))
    assert n_hdr == n_enum == FOP_NVARIANTS


def test_bench_quotes_ncu_traffic_only_for_captured_variants():
    """roofline.traffic comes from the committed single-kernel capture of
    the variant the autotuner picked, and is None for one never captured."""
    bench = _bench_module()
    t64, t32 = bench.committed_traffic(14, 14)
    alg64 = bench.algorithmic_bytes_fop(12 * 12 * 12 * 24, 3, 16)
    alg32 = bench.algorithmic_bytes_fop(12 * 12 * 12 * 24, 3, 8)
    assert alg64 == 264093696 and alg32 == 132046848
    # DRAM traffic of a real capture: near the algorithmic bytes, not far below
    assert 0.9 * alg64 < t64 < 2.0 * alg64 and 0.9 * alg32 < t32 < 2.0 * alg32
    assert bench.committed_traffic(0, 1) == (None, None)
