"""Benchmark of the RHMC fermion path on B200.

Workload (the metric's configuration): 12^3 x 24 lattice, U(3) (NCOL = 3),
lambda = 2, bmass = 0.3, G = 0.05, antiperiodic temporal BC, on the links
of configs/thermalised_12x12x12x24_u3.lat (identity + 0.1 noise, seed 11,
thermalised by 20 RHMC trajectories of this integrator: configs/
thermalise.py; the file's checksums are verified and reported).  One
"step" is one multi-shift CG solve of the degree-15 RHMC system with
Nroot = 2 (the 15 shift4 poles of setup_rhmc.c) on a complex-Gaussian
Twist_Fermion source, to an FP64 true residual |r|^2 <= 1e-20 |src|^2
(error_per_site 1e-10).  Inputs are resident in HBM when the timed region
starts; the working set (~3 GB) is larger than L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--solver mixed|fp64] [--no-traj]

The timed solver is the mixed one by default (FP64 operator until
|r| < 3e-4 |src|, FP32 operator after, FP64 residual replacement and
per-shift FP64 check: the same FP64 true-residual bound as the FP64 solver,
reported as true_residual_rel_max); the FP64 solver of the reference's
recurrences is timed right after it in the same run (fp64_s_per_solve).
On one GPU the line also carries one full RHMC trajectory per solver (15 x
3 steps, the same start links and random numbers for both): s_per_traj,
delta S, acceptance and CG iterations.

N > 1 runs one independent replica per GPU (torchrun, NCCL only for the
barrier and the max-over-ranks time): "value" is the whole-job seconds per
solve, max rank time / (K * N).  The reference arm times the reference's own
CPU congrad_multi (oracle/_ref) on bounded samples of the same solve,
weighted by the solve's recorded schedule of live shifts
(configs/solve_profile_12x12x12x24_u3.json).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (12, 12, 12, 24)
NCOL = 3
LAM, BMASS, G = 2.0, 0.3, 0.05
LINK_NOISE, LINK_SEED, SRC_SEED = 0.1, 11, 12
TRAJ_SEED = 13
NORDER, NROOT = 15, 2
ERRORMIN = 1e-20          # error_per_site 1e-10 squared (setup.c:356-359)
MAXCG = 20000
REF_SAMPLE_ITERS = 2
# live-shift counts the reference arm samples (cycled over its steps); its
# per-iteration cost is fitted as a + b * (live shifts)
REF_SAMPLE_SHIFTS = (1, 8, 15)
REF_SAMPLE_TIMEOUT = 600   # seconds one sample (set-up of the replicas included) may take
METRIC = "s/RHMC traj & CG solve time, 12^3x24 U(3): FP32+learned vs FP64 @1e-10 resid"
WORKLOAD = ("12^3x24 U(3) multi-shift CG solve, Norder 15 / Nroot 2 shift4 poles, "
            "FP64 true residual 1e-10 per site, thermalised links")
LINKS_FILE = os.path.join(ROOT, "configs", "thermalised_12x12x12x24_u3.lat")
PROFILE_FILE = os.path.join(ROOT, "configs", "solve_profile_12x12x12x24_u3.json")


def workload_links():
    """The benchmark links in the reference host layout and the file's
    header facts; raises if the file is absent or its checksums fail."""
    from susy_b200 import io_lat, synth
    dims, ncol, links, info = io_lat.read_gauge(LINKS_FILE)
    if tuple(dims) != DIMS or ncol != NCOL:
        raise RuntimeError("%s holds a %s U(%d) lattice" % (LINKS_FILE, dims, ncol))
    if not info["checksum_ok"]:
        raise RuntimeError("checksum mismatch in " + LINKS_FILE)
    info["checksums"] = "%x %x" % (info["sum29"], info["sum31"])
    return synth.to_ref(DIMS, links), info


def bench_config(extra=None):
    """config keys shared by both arms."""
    c = {"workload": WORKLOAD, "lattice": "12x12x12x24", "ncol": NCOL, "lambda": LAM,
         "bmass": BMASS, "G": G, "norder": NORDER, "nroot": NROOT,
         "links": "configs/thermalised_12x12x12x24_u3.lat"}
    c.update(extra or {})
    return c


def algorithmic_bytes_fop(V, N, w, doG=True):
    """Bytes one fermion_op moves with perfect neighbour reuse:
    V [(16 + 16 + 5) N^2 w + g (5 N^2 w + 20 w)], w = bytes per complex."""
    return V * ((16 + 16 + 5) * N * N * w + (5 * N * N * w + 20 * w if doG else 0))


def flops_fop(V, N):
    """220 NCOL x NCOL complex products per site: 1760 N^3 flop per site."""
    return 1760 * N ** 3 * V


def committed_traffic(v64, v32):
    """DRAM bytes per operator launch (ncu dram__bytes_read.sum +
    dram__bytes_write.sum) of the FP64 and FP32 kernel variants the
    autotuner picked, from the committed single-kernel capture summary
    profiles/fermion_op_12x12x12x24_u3.json; None for a variant that was
    never captured (the figure is only quoted for the kernel it measured)."""
    try:
        with open(os.path.join(ROOT, "profiles", "fermion_op_12x12x12x24_u3.json")) as f:
            d = json.load(f)["variants"]
    except Exception:
        return None, None
    t64 = d.get(str(v64), {}).get("fp64_dram_bytes_per_launch")
    t32 = d.get(str(v32), {}).get("fp32_dram_bytes_per_launch")
    return t64, t32


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
_REF = {}


def _ref_init(kind):
    """Pool worker set-up: one reference lattice (or the numpy port's
    fields) on the workload links, kept for all of this worker's samples."""
    from susy_b200 import synth
    from susy_b200.rhmc_tables import rhmc
    links, _ = workload_links()
    src = synth.to_ref(DIMS, synth.tf_source(DIMS, NCOL, SRC_SEED))
    _REF["shifts"] = np.array(rhmc(NORDER, NROOT)["shift4"])
    _REF["kind"] = kind
    if kind == "reference":
        from oracle.ref_ctypes import RefLattice
        ref = RefLattice(NCOL, dims=DIMS, pbc=-1, lam=LAM, bmass=BMASS, G=G, Nroot=NROOT,
                         Norder=NORDER)
        ref.set_links(links)
        ref.compute_all()
        _REF["ref"], _REF["src"] = ref, src
    else:
        from oracle import susy_np as O
        geo = O.Geometry(DIMS, -1)
        prm = O.Params(lam=LAM, bmass=BMASS, G=G, N=NCOL)
        U = synth.from_ref(DIMS, links, 5, NCOL)
        _REF["port"] = (geo, prm, U, O.compute_derived(geo, prm, U))
        _REF["src"] = synth.from_ref(DIMS, src, 16, NCOL)


def _ref_sample(nshift, iters):
    """Seconds per iteration of the CPU congrad_multi with nshift live
    shifts (the first nshift poles), over `iters` iterations from the zero
    initial guess (no shift freezes that early)."""
    sh = _REF["shifts"][:nshift]
    t0 = time.perf_counter()
    if _REF["kind"] == "reference":
        _, it, _ = _REF["ref"].congrad_multi(_REF["src"], sh, iters, ERRORMIN)
    else:
        from oracle import susy_np as O
        geo, prm, U, der = _REF["port"]
        _, it, _ = O.congrad_multi(geo, prm, U, der, _REF["src"], sh, iters, ERRORMIN)
    return (time.perf_counter() - t0) / max(it, 1)


def host_workers():
    """Reference replicas the host can run at once: every core, as far as
    memory allows (a 12^3x24 U(3) reference solve holds ~4 GB)."""
    n = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            kv = {l.split(":")[0]: l.split()[1] for l in f}
        n = min(n, max(1, int(int(kv["MemAvailable"]) / (5 * 1024 * 1024))))
    except Exception:
        pass
    return max(1, min(n, 128))


def solve_profile():
    """(iterations, live shifts summed over the iterations) of the FP64
    solve of this workload, from configs/solve_profile_12x12x12x24_u3.json
    (configs/solve_profile.py)."""
    with open(PROFILE_FILE) as f:
        p = json.load(f)
    return int(p["iterations"]), int(sum(p["live_shifts_per_iteration"])), p


class CpuArm:
    """The reference's CPU solve, sampled: the reference is single threaded
    (its parallel path is MPI, which this image lacks), so every host core
    runs an independent single-core replica and all of them time the same
    bounded sample at once.  A sample is REF_SAMPLE_ITERS iterations of
    congrad_multi with k live shifts; its per-iteration time is fitted as
    t(k) = a + b k over the samples, and one solve costs
    iterations * a + b * (live shifts summed over its iterations), the
    schedule of the FP64 solve of this workload.  Seconds per solve of the
    host = that / replicas."""

    def __init__(self, workers=None):
        import multiprocessing as mp
        from oracle.ref_ctypes import available
        self.kind = "reference" if available(NCOL) else "port"
        self.P = workers or host_workers()
        self.pool = mp.get_context("spawn").Pool(self.P, initializer=_ref_init,
                                                 initargs=(self.kind,))
        self.samples = []     # (k, seconds per iteration, averaged over replicas)

    def sample(self, k):
        t0 = time.perf_counter()
        # bounded wait: a worker that died would otherwise leave the map
        # waiting for good
        per = self.pool.starmap_async(_ref_sample, [(k, REF_SAMPLE_ITERS)] * self.P,
                                      chunksize=1).get(timeout=REF_SAMPLE_TIMEOUT)
        self.samples.append((k, statistics.mean(per)))
        return time.perf_counter() - t0

    def close(self):
        self.pool.terminate()

    def value(self):
        iters, live_sum, _ = solve_profile()
        ks = np.array([k for k, _ in self.samples], dtype=float)
        ts = np.array([t for _, t in self.samples])
        if len(set(ks)) > 1:
            b, a = np.polyfit(ks, ts, 1)
        else:
            b, a = ts.mean() / ks.mean(), 0.0
        per_replica = iters * a + b * live_sum
        desc = ("%d samples of %d iterations of the reference's congrad_multi with 1, 8 or "
                "15 live shifts, on each of %d single-core replicas running at once on "
                "the host; per-iteration time fitted as %.3f s + %.4f s per live shift and "
                "summed over the FP64 solve's recorded schedule (%d iterations, %d "
                "shift-iterations; configs/solve_profile_12x12x12x24_u3.json), divided "
                "by the replica count"
                % (len(self.samples), REF_SAMPLE_ITERS, self.P, a, b, iters, live_sum))
        return per_replica / self.P, desc


def cpu_baseline(nsamples=3):
    arm = CpuArm()
    try:
        for i in range(nsamples):
            arm.sample(REF_SAMPLE_SHIFTS[i % len(REF_SAMPLE_SHIFTS)])
        v, desc = arm.value()
    finally:
        arm.close()
    return {"value": v, "unit": "s/solve", "cores": arm.P, "kind": arm.kind, "sample": desc}


# ---------------------------------------------------------------------------
def run_reference_arm(args, rank, world):
    if rank != 0:
        return None
    arm = CpuArm()
    walls = []
    try:
        # a warm-up step is one sample; a timed step samples every live-shift
        # count of REF_SAMPLE_SHIFTS, so that any number of timed steps (one
        # included) fits both terms of t(k) = a + b k
        for i in range(args.warmup):
            arm.sample(REF_SAMPLE_SHIFTS[i % len(REF_SAMPLE_SHIFTS)])
        arm.samples = []
        for _ in range(max(1, args.steps)):
            walls.append(sum(arm.sample(k) for k in REF_SAMPLE_SHIFTS))
        v, desc = arm.value()
    finally:
        arm.close()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s/solve",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(walls) * 1e3,
            "ms_per_step_note": "wall time of one bounded sample per live-shift count (all "
                                "replicas); value is the full solve assembled from the samples",
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": bench_config({"solver": "reference congrad_multi (FP64, CPU)",
                                    "parallelism": "replicas"}),
            "cpu_baseline": {"value": v, "unit": "s/solve", "cores": arm.P, "kind": arm.kind,
                             "sample": desc},
            "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return line


def trajectories(lat, st, links, solvers):
    """One RHMC trajectory per solver from the given links with the site and
    node generators reseeded (TRAJ_SEED), timed with CUDA events on the
    lattice's stream (the trajectory's host work included): 15 fermion x 3
    gauge steps, trajectory length 1, Nroot 2, degree 15, error_per_site
    1e-10, Metropolis.  The handle's links are left as they were."""
    import torch
    from susy_b200 import RHMC
    runs = []
    for name in solvers:
        lat.set_links(links)
        lat.seed(TRAJ_SEED)
        r = RHMC(NORDER, NROOT, nstep=15, nstep_gauge=3, traj_length=1.0, niter=MAXCG,
                 error_per_site=1e-10, solver=1 if name == "mixed" else 0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        res = lat.update(r)
        e1.record(st)
        e1.synchronize()
        runs.append({"solver": name, "s_per_traj": e0.elapsed_time(e1) / 1e3,
                     "delta_S": res["delta_S"], "accept": bool(res["accept"]),
                     "cg_iterations": res["iters"]})
    lat.set_links(links)
    by = {r["solver"]: r for r in runs}
    out = {"nstep": 15, "nstep_gauge": 3, "traj_length": 1.0, "runs": runs}
    if "mixed" in by and "fp64" in by:
        out["delta_S_mixed_minus_fp64"] = by["mixed"]["delta_S"] - by["fp64"]["delta_S"]
    return out


def run_ours(args, rank, world, device):
    import torch
    import torch.distributed as dist
    from susy_b200 import Lattice, synth
    from susy_b200.lattice import launch_count
    from susy_b200.replicas import max_over_ranks, rank_seed, seconds_per_solve
    from susy_b200.rhmc_tables import rhmc

    torch.cuda.set_device(device)
    lat = Lattice(DIMS, NCOL, pbc=-1, lam=LAM, bmass=BMASS, G=G, device=device)
    st = torch.cuda.Stream(device=device)
    lat.set_stream(st.cuda_stream)
    links, links_info = workload_links()
    lat.set_links(links)
    # every replica solves its own source on the workload links
    src_host = synth.to_ref(DIMS, synth.tf_source(DIMS, NCOL, rank_seed(SRC_SEED, rank)))
    shifts = np.array(rhmc(NORDER, NROOT)["shift4"])
    src = lat.tf(64)
    src.upload(src_host)
    psim = [lat.tf(64) for _ in shifts]
    if args.fop_variant >= 0:
        # pinned kernel (e.g. for an ncu launch list, under which the
        # autotuner's timings are distorted)
        lat.fop_variant(64, args.fop_variant)
        lat.fop_variant(32, args.fop_variant)
    else:
        lat.autotune()
    mixed = args.solver == "mixed"

    def solve(m=None):
        return lat.dev_congrad_multi(src, psim, shifts, MAXCG, ERRORMIN,
                                     mixed=mixed if m is None else m)

    def barrier():
        if world > 1:
            dist.barrier()

    iters = []
    for _ in range(args.warmup):
        iters.append(solve()[0])
    lat.sync()
    barrier()
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    n0 = launch_count()
    with ClockSampler(device) as clk:
        e0.record(st)
        for _ in range(args.steps):
            it, rsq = solve()
            iters.append(it)
        e1.record(st)
        e1.synchronize()
    launches = launch_count() - n0
    barrier()
    torch.cuda.synchronize(device)
    ms_max = max_over_ranks(e0.elapsed_time(e1))
    # the other solver on the same input, timed the same way (after one
    # warm-up solve), for the FP32-vs-FP64 comparison of the metric
    other = not mixed
    solve(other)
    lat.sync()
    barrier()
    torch.cuda.synchronize(device)
    o0 = torch.cuda.Event(enable_timing=True)
    o1 = torch.cuda.Event(enable_timing=True)
    o0.record(st)
    other_iters = 0
    for _ in range(args.steps):
        other_iters = solve(other)[0]
    o1.record(st)
    o1.synchronize()
    other_ms = max_over_ranks(o0.elapsed_time(o1))
    solve()                     # leave the timed solver's solutions in psim
    # FP64 true residual of every shift of the last solve, relative to |src|^2
    # (the stopping bound is 1e-20): checked on the host from the downloaded
    # solutions and their D^dag D
    b2 = float(np.dot(src_host, src_host))
    t = lat.tf(64)
    true_rel = []
    for j, sg in enumerate(shifts):
        lat.dev_DSq(psim[j], t)
        x = psim[j].download()
        r = src_host - t.download() - sg * x
        true_rel.append(float(np.dot(r, r)) / b2)

    # Dominant kernel: the fermion operator inside DSq, timed live on the
    # launching stream after the timed region.
    a = lat.tf(64)
    b = lat.tf(64)
    a.upload(src_host)
    lat.dev_DSq(a, b)
    reps = 10
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(st)
    for _ in range(reps):
        lat.dev_DSq(a, b)
    f1.record(st)
    f1.synchronize()
    fop_ms = f0.elapsed_time(f1) / (2 * reps)
    a32, b32 = lat.tf(32), lat.tf(32)
    lat.dev_convert(a, a32)
    lat.dev_DSq(a32, b32)
    f0.record(st)
    for _ in range(reps):
        lat.dev_DSq(a32, b32)
    f1.record(st)
    f1.synchronize()
    fop32_ms = f0.elapsed_time(f1) / (2 * reps)
    V = lat.V
    algo = algorithmic_bytes_fop(V, NCOL, 16)
    achieved = algo / (fop_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic, traffic32 = committed_traffic(lat.fop_variant(64)[0], lat.fop_variant(32)[0])

    # End to end through the public host API: source H2D, every solution D2H
    e2e_ms = None
    h2d = d2h = 0
    if not args.no_e2e:
        import torch as _t
        lat.set_solver(1 if mixed else 0)
        host_src = _t.empty(lat.tf_doubles, dtype=_t.float64, pin_memory=True).numpy()
        host_src[:] = src_host
        outs = [_t.empty(lat.tf_doubles, dtype=_t.float64, pin_memory=True).numpy()
                for _ in shifts]
        lat.congrad_multi(host_src, outs, shifts, MAXCG, ERRORMIN)
        barrier()
        g0 = _t.cuda.Event(enable_timing=True)
        g1 = _t.cuda.Event(enable_timing=True)
        g0.record(st)
        for _ in range(args.steps):
            lat.congrad_multi(host_src, outs, shifts, MAXCG, ERRORMIN)
        g1.record(st)
        g1.synchronize()
        e2e_ms = max_over_ranks(g0.elapsed_time(g1))
        h2d = host_src.nbytes
        d2h = sum(o.nbytes for o in outs)

    # One full RHMC trajectory per solver (one GPU only: ~2 x 1-3 minutes),
    # both from the workload links and the same random numbers, so both
    # integrate the same trajectory and only the solves differ
    traj = None
    if world == 1 and not args.no_traj:
        traj = trajectories(lat, st, links, ["mixed", "fp64"] if mixed else ["fp64", "mixed"])

    if rank != 0:
        return None
    value = seconds_per_solve(ms_max, args.steps, world)
    line = {"metric": METRIC, "value": value, "unit": "s/solve", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if not mixed else "f32+f64",
            "data": "synthetic",
            "config": bench_config({
                       "links_checksums": links_info["checksums"],
                       "solver": args.solver,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set ~3 GB > 126 MB L2; no flush",
                       "iterations_per_solve": iters[-1],
                       "true_residual_rel_max": max(true_rel),
                       ("fp64" if mixed else "mixed") + "_s_per_solve":
                           seconds_per_solve(other_ms, args.steps, world),
                       ("fp64" if mixed else "mixed") + "_iterations": other_iters,
                       "speedup_vs_fp64": (other_ms / ms_max) if mixed else 1.0,
                       "fop_variant": lat.fop_variant(64)[0]}),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "kernel": "fermion_op (FP64, in DSq)",
                         "algorithmic_bytes_per_launch": algo, "launch_ms": fop_ms,
                         "fp64_tflops": flops_fop(V, NCOL) / (fop_ms * 1e-3) / 1e12,
                         "fp32_launch_ms": fop32_ms,
                         "fp32_achieved": algorithmic_bytes_fop(V, NCOL, 8) / (fop32_ms * 1e-3) / 1e9,
                         "fp32_frac": algorithmic_bytes_fop(V, NCOL, 8) / (fop32_ms * 1e-3) / 1e9 / peak,
                         "fp32_variant": lat.fop_variant(32)[0],
                         "fp32_traffic": traffic32},
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "e2e": {"value": seconds_per_solve(e2e_ms, args.steps, world) if e2e_ms else None,
                    "unit": "s/solve", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}}
    if traj:
        line["trajectory"] = traj
        t = {r["solver"]: r for r in traj["runs"]}
        if "mixed" in t and "fp64" in t:
            line["trajectory"]["speedup_vs_fp64"] = t["fp64"]["s_per_traj"] / t["mixed"]["s_per_traj"]
    if world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline()
        except Exception as e:  # the checker is optional: report why it is absent
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)[:200]}
    print(json.dumps(line), flush=True)
    return line


def run_dsq_case(args):
    """Operator microbenchmark on the bench lattice (or --dims / --ncol):
    D^dag D per kernel variant and precision (CUDA events on the launching
    stream, 20 applications after 3 warm-up ones; the working set per
    application must exceed the 126 MB L2 for an HBM figure: 0.26 GB at
    12^3x24 U(3) FP64).  --variant V restricts it to one variant (the small
    case an ncu capture of one kernel runs)."""
    import torch
    from susy_b200 import Lattice, synth
    from susy_b200.lattice import FOP_NVARIANTS
    dims = tuple(int(x) for x in args.dims.split(",")) if args.dims else DIMS
    ncol = args.ncol or NCOL
    lat = Lattice(dims, ncol, pbc=-1, lam=LAM, bmass=BMASS, G=G)
    st = torch.cuda.Stream()
    lat.set_stream(st.cuda_stream)
    if dims == DIMS and ncol == NCOL:
        lat.set_links(workload_links()[0])
    else:
        lat.set_links(synth.to_ref(dims, synth.links(dims, ncol, LINK_NOISE, LINK_SEED)))
    src = synth.to_ref(dims, synth.tf_source(dims, ncol, SRC_SEED))
    peak, peak_kind = measured_peaks()
    variants = [args.variant] if args.variant >= 0 else list(range(FOP_NVARIANTS))
    reps = 3 if args.variant >= 0 else 20
    for prec, w in ((64, 16), (32, 8)):
        a, b = lat.tf(prec), lat.tf(prec)
        if prec == 64:
            a.upload(src)
        else:
            a64 = lat.tf(64)
            a64.upload(src)
            lat.dev_convert(a64, a)
        for v in variants:
            lat.fop_variant(prec, v)
            for _ in range(3):
                lat.dev_DSq(a, b)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                lat.dev_DSq(a, b)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / (2 * reps)
            algo = algorithmic_bytes_fop(lat.V, ncol, w)
            gbs = algo / (ms * 1e-3) / 1e9
            print(json.dumps({"case": "fermion_op", "lattice": "x".join(map(str, dims)),
                              "ncol": ncol, "prec": prec, "variant": v, "ms_per_launch": ms,
                              "algorithmic_gbs": gbs, "frac": gbs / peak,
                              "peak_kind": peak_kind,
                              "tflops": flops_fop(lat.V, ncol) / (ms * 1e-3) / 1e12}),
                  flush=True)


# Operator and solver microbenchmark: 8^4 U(2), links identity + 0.2
# noise, lambda 1, bmass 0.2, G 0.05, antiperiodic in time; 32
# complex-Gaussian sources; 15 shifts geometrically spaced 1e-5 ... 1e3.
MB_DIMS, MB_NCOL, MB_SOURCES, MB_DSQ = (8, 8, 8, 8), 2, 32, 1000


def run_microbench_case(args):
    """D^dag D applied 1000 times in FP64 and in FP32, cycling over the 32
    sources (CUDA events on the launching stream; sources and results,
    2 x 32 x 4.2 MB in FP64, exceed the 126 MB L2, the 1.3 MB of links stay
    in it): ms per application, algorithmic GB/s and the FP32 result's
    error against the FP64 one (the FP64 operator itself is pinned to the
    oracle at 1e-13 on this configuration by the GPU tests).  Then every
    source solved with the 15 shifts to the FP64 true residual 1e-10 per
    site by the FP64 solver, the mixed solver at its defaults, and the
    mixed solver with the FP32 operator from the first iteration and FP64
    reliable updates every 50 iterations (rounded up to the 8-iteration
    block): iterations, ms per solve, and per shift the worst FP64 true
    residual |b - (D^dag D + sigma) x| / |b| and the worst solution error
    against the FP64 solver's, max |x - x64| / max |x64|."""
    import torch
    from susy_b200 import Lattice, synth
    dims, N = MB_DIMS, MB_NCOL
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    st = torch.cuda.Stream()
    lat.set_stream(st.cuda_stream)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, 1)))
    peak, peak_kind = measured_peaks()
    srcs = [synth.to_ref(dims, synth.tf_source(dims, N, 100 + k)) for k in range(MB_SOURCES)]
    a64 = [lat.tf(64) for _ in srcs]
    b64 = [lat.tf(64) for _ in srcs]
    for a, x in zip(a64, srcs):
        a.upload(x)
    a32 = [lat.tf(32) for _ in srcs]
    b32 = [lat.tf(32) for _ in srcs]
    for a, c in zip(a64, a32):
        lat.dev_convert(a, c)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    report = {"case": "operator_solver_microbench", "lattice": "x".join(map(str, dims)), "ncol": N,
              "sources": len(srcs), "dsq_applications": MB_DSQ, "peak_gbs": peak,
              "peak_kind": peak_kind}
    for prec, w, A, B in ((64, 16, a64, b64), (32, 8, a32, b32)):
        for k in range(3):
            lat.dev_DSq(A[k], B[k])
        e0, e1 = ev(), ev()
        e0.record(st)
        for k in range(MB_DSQ):
            lat.dev_DSq(A[k % len(A)], B[k % len(B)])
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / MB_DSQ
        gbs = 2 * algorithmic_bytes_fop(lat.V, N, w) / (ms * 1e-3) / 1e9
        report["dsq_fp%d" % prec] = {"ms_per_dsq": ms, "algorithmic_gbs": gbs,
                                     "frac": gbs / peak}
    t64 = lat.tf(64)
    err = 0.0
    for k in range(len(srcs)):
        lat.dev_DSq(a64[k], b64[k])
        lat.dev_convert(b32[k], t64)
        want, got = b64[k].download(), t64.download()
        err = max(err, float(np.abs(got - want).max() / np.abs(want).max()))
    report["dsq_fp32_max_rel_err_vs_fp64"] = err

    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    psim = [lat.tf(64) for _ in shifts]
    solvers = (("fp64", False, None), ("mixed", True, (3e-4, 1e-2, 0)),
               ("fp32_reliable50", True, (1.0, 1e-2, 50)))
    stats = {name: {"iters": [], "ms": [], "true_res": np.zeros(len(shifts)),
                    "sol_err": np.zeros(len(shifts))} for name, _, _ in solvers}
    for k in range(len(srcs)):
        b = srcs[k]
        bn = float(np.sqrt(np.dot(b, b)))
        x64 = None
        for name, mixed, prm in solvers:
            if prm:
                lat.mixed_params(prm[0], prm[1])
                lat.mixed_reliable_interval(prm[2])
            e0, e1 = ev(), ev()
            e0.record(st)
            it, _ = lat.dev_congrad_multi(a64[k], psim, shifts, MAXCG, ERRORMIN, mixed=mixed)
            e1.record(st)
            e1.synchronize()
            S = stats[name]
            S["iters"].append(it)
            S["ms"].append(e0.elapsed_time(e1))
            xs = [p.download() for p in psim]
            for j, sg in enumerate(shifts):
                lat.dev_DSq(psim[j], t64)
                r = b - t64.download() - sg * xs[j]
                S["true_res"][j] = max(S["true_res"][j], float(np.sqrt(np.dot(r, r))) / bn)
                if x64 is not None:
                    S["sol_err"][j] = max(S["sol_err"][j], float(
                        np.abs(xs[j] - x64[j]).max() / np.abs(x64[j]).max()))
            if not mixed:
                x64 = xs
    lat.mixed_params()
    lat.mixed_reliable_interval(0)
    for name, S in stats.items():
        report[name] = {"iters_mean": float(np.mean(S["iters"])),
                        "iters_min": int(min(S["iters"])), "iters_max": int(max(S["iters"])),
                        "ms_per_solve_mean": float(np.mean(S["ms"])),
                        "max_true_residual_per_shift": [float(x) for x in S["true_res"]],
                        "max_sol_err_vs_fp64_per_shift": [float(x) for x in S["sol_err"]]}
    report["shifts"] = [float(x) for x in shifts]
    print(json.dumps(report), flush=True)


# Batched parameter scan of independent U(2) lattices: volumes from
# {4^4, 6^4, 8^4, 4^3x8, 6^3x12, 8^3x16}, lambda from {0.5, 1, 2, 4}, link
# noise 0.1-0.3, all seed-derived; bmass 0.2, G 0.05; degree-15 Nroot 1
# rational approximation, 5 fermion steps x 4 gauge steps, error_per_site
# 1e-5.
BATCH_VOLS = [(4, 4, 4, 4), (6, 6, 6, 6), (8, 8, 8, 8), (4, 4, 4, 8), (6, 6, 6, 12),
              (8, 8, 8, 16)]
BATCH_LAMS = [0.5, 1.0, 2.0, 4.0]


def run_batch_dsq_case(args):
    """D^dag D on --lattices independent U(2) lattices (the batched scan's
    volumes, lambdas and link noise), FP64 and FP32: all lattices in one
    pair of persistent launches over a work table (susy_b200_DSq_batch)
    against each lattice's own D^dag D in turn on one stream (two launches
    per lattice, the autotuned variant).  Device time with CUDA events, 3
    warm-up and 20 timed repetitions; site-applications/s = sum of volumes /
    time per repetition, and the largest relative difference between the
    batched and the per-lattice results.  Every lattice launches on one
    stream here, so both ways are timed by the same events."""
    import torch
    from susy_b200 import Lattice, dsq_batch, synth
    rng = np.random.default_rng(2024)
    lats = []
    for i in range(args.lattices):
        dims = BATCH_VOLS[int(rng.integers(len(BATCH_VOLS)))]
        lam = float(rng.choice(BATCH_LAMS))
        noise = float(rng.uniform(0.1, 0.3))
        lat = Lattice(dims, 2, pbc=-1, lam=lam, bmass=0.2, G=0.05, iseed=1000 + i)
        lat.set_links(synth.to_ref(dims, synth.links(dims, 2, noise, 500 + i)))
        lat.autotune()
        lats.append(lat)
    sites = sum(lat.V for lat in lats)
    # both ways on one stream, so the events on it see every launch
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    for lat in lats:
        lat.set_stream(st.cuda_stream)
    for prec in (64, 32):
        srcs, outs, refs = [], [], []
        for i, lat in enumerate(lats):
            s64 = lat.tf(64)
            s64.upload(synth.to_ref(lat.dims, synth.tf_source(lat.dims, 2, 700 + i)))
            if prec == 64:
                s = s64
            else:
                s = lat.tf(32)
                lat.dev_convert(s64, s)
            srcs.append(s)
            outs.append(lat.tf(prec))
            refs.append(lat.tf(prec))
        torch.cuda.synchronize()

        def one_by_one():
            for lat, s, r in zip(lats, srcs, refs):
                lat.dev_DSq(s, r)

        def batched():
            dsq_batch(srcs, outs, st.cuda_stream)

        res = {}
        for name, fn in (("batched", batched), ("one_by_one", one_by_one)):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(20):
                fn()
            e1.record(st)
            torch.cuda.synchronize()
            res[name] = e0.elapsed_time(e1) / 20
        err = max(float(np.abs(o.download() - r.download()).max() /
                        np.abs(r.download()).max()) for o, r in zip(outs, refs))
        print(json.dumps({"case": "dsq_batch", "lattices": len(lats), "sites": sites,
                          "prec": prec, "ms_batched": res["batched"],
                          "ms_one_by_one": res["one_by_one"],
                          "site_applications_per_s_batched": sites / (res["batched"] * 1e-3),
                          "site_applications_per_s_one_by_one":
                              sites / (res["one_by_one"] * 1e-3),
                          "speedup": res["one_by_one"] / res["batched"],
                          "max_rel_diff": err}), flush=True)


def run_batch_cg_case(args):
    """The multi-shift solve (15 shift4 poles of the Nroot 1 degree-15
    approximation, FP64 residual 1e-10 per site) on --lattices independent
    U(2) lattices of the batched scan: all lattices in one batched solve
    (susy_b200_dev_congrad_multi_batch: six launches per iteration for all
    of them) against each lattice's own solve in turn (its default FP64
    solver: blocked vector update, graph-replayed iteration chunks), every
    lattice on one stream.  Device time with CUDA events; also the largest
    iteration difference and the largest relative solution difference."""
    import torch
    from susy_b200 import Lattice, congrad_multi_batch, synth
    from susy_b200.rhmc_tables import rhmc
    rng = np.random.default_rng(2024)
    shifts = np.array(rhmc(15, 1)["shift4"])
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    lats, srcs = [], []
    for i in range(args.lattices):
        dims = BATCH_VOLS[int(rng.integers(len(BATCH_VOLS)))]
        lam = float(rng.choice(BATCH_LAMS))
        noise = float(rng.uniform(0.1, 0.3))
        lat = Lattice(dims, 2, pbc=-1, lam=lam, bmass=0.2, G=0.05, iseed=1000 + i)
        lat.set_links(synth.to_ref(dims, synth.links(dims, 2, noise, 500 + i)))
        lat.autotune()
        lat.set_stream(st.cuda_stream)
        src = lat.tf(64)
        src.upload(synth.to_ref(dims, synth.tf_source(dims, 2, 700 + i)))
        lats.append(lat)
        srcs.append(src)
    sites = sum(lat.V for lat in lats)
    solo = [[lat.tf(64) for _ in shifts] for lat in lats]
    batch = [[lat.tf(64) for _ in shifts] for lat in lats]

    def one_by_one():
        return [lat.dev_congrad_multi(s, p, shifts, MAXCG, ERRORMIN)[0]
                for lat, s, p in zip(lats, srcs, solo)]

    def batched():
        return congrad_multi_batch(srcs, batch, [shifts] * len(lats), MAXCG, ERRORMIN,
                                   st.cuda_stream)[0]

    res = {}
    for name, fn in (("batched", batched), ("one_by_one", one_by_one)):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        its = fn()
        e1.record(st)
        torch.cuda.synchronize()
        res[name] = (e0.elapsed_time(e1), its)
    err = max(float(np.abs(b.download() - a.download()).max() / np.abs(a.download()).max())
              for pa, pb in zip(solo, batch) for a, b in zip(pa, pb))
    itb, ito = res["batched"][1], res["one_by_one"][1]
    print(json.dumps({"case": "congrad_multi_batch", "lattices": len(lats), "sites": sites,
                      "shifts": len(shifts), "errormin": ERRORMIN,
                      "ms_batched": res["batched"][0], "ms_one_by_one": res["one_by_one"][0],
                      "speedup": res["one_by_one"][0] / res["batched"][0],
                      "iterations_batched_max": max(itb), "iterations_solo_max": max(ito),
                      "max_iteration_difference": max(abs(a - b) for a, b in zip(itb, ito)),
                      "site_iterations_per_s_batched":
                          sum(lat.V * it for lat, it in zip(lats, itb)) / (res["batched"][0] * 1e-3),
                      "max_rel_solution_diff": err}), flush=True)


def run_batch_case(args):
    """One RHMC trajectory on each of --lattices independent lattices,
    concurrently (susy_b200_update_batch) and one after another, from the
    same starting state: aggregate site-updates/s both ways (device time:
    CUDA events on every lattice's stream, first start to last end) and the
    largest |delta S| difference between a lattice batched and alone."""
    import torch
    from susy_b200 import Lattice, RHMC, synth, update_batch
    rng = np.random.default_rng(2024)
    lats, rhs, starts, streams = [], [], [], []
    for i in range(args.lattices):
        dims = BATCH_VOLS[int(rng.integers(len(BATCH_VOLS)))]
        lam = float(rng.choice(BATCH_LAMS))
        noise = float(rng.uniform(0.1, 0.3))
        lat = Lattice(dims, 2, pbc=-1, lam=lam, bmass=0.2, G=0.05, iseed=1000 + i)
        # every lattice keeps its own stream (torch.cuda.Stream() hands out
        # a pool of 32 per device, so lattices 32 apart would share one);
        # the events are recorded on it through an ExternalStream
        st = torch.cuda.ExternalStream(lat.stream)
        links = synth.to_ref(dims, synth.links(dims, 2, noise, 500 + i))
        lats.append(lat)
        streams.append(st)
        starts.append(links)
        rhs.append(RHMC(15, 1, nstep=5, nstep_gauge=4, traj_length=1.0, error_per_site=1e-5))

    def reset():
        for lat, links, i in zip(lats, starts, range(len(lats))):
            lat.set_links(links)
            lat.set_mom(np.zeros_like(links))
            lat.seed(1000 + i)
        torch.cuda.synchronize()

    def timed(fn):
        e0 = [torch.cuda.Event(enable_timing=True) for _ in lats]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in lats]
        for e, st in zip(e0, streams):
            e.record(st)
        out = fn()
        for e, st in zip(e1, streams):
            e.record(st)
        torch.cuda.synchronize()
        return out, max(e0[0].elapsed_time(e) for e in e1)

    update_batch(lats, rhs, args.threads)            # warm-up: allocation, autotune
    reset()
    batched, t_b = timed(lambda: update_batch(lats, rhs, args.threads))
    reset()
    alone, t_a = timed(lambda: [lat.update(r) for lat, r in zip(lats, rhs)])
    sites = sum(lat.V for lat in lats)
    dS = max(abs(b["delta_S"] - a["delta_S"]) for b, a in zip(batched, alone))
    print(json.dumps({"case": "batched_lattices", "lattices": len(lats), "ncol": 2,
                      "threads": args.threads, "total_sites": sites,
                      "site_updates_per_s": sites / (t_b * 1e-3),
                      "sequential_site_updates_per_s": sites / (t_a * 1e-3),
                      "batched_ms": t_b, "sequential_ms": t_a, "speedup": t_a / t_b,
                      "max_abs_delta_S_diff_vs_alone": dS,
                      "accepted": sum(int(b["accept"]) for b in batched),
                      "cg_iterations": sum(b["iters"] for b in batched)}), flush=True)


def run_traj_case(args):
    """Full RHMC trajectories of the bench lattice with the trajectory
    parameters of the metric's configuration (12^3x24 U(3), lambda 2,
    bmass 0.3, G 0.05, degree-15 rational approximation, Nroot 2, 15
    fermion steps x 3 gauge steps, error_per_site 1e-10, traj_length 1),
    from the thermalised workload links.  Each solver runs --steps
    trajectories from those links and the same random-number state (so
    every solver integrates the same trajectory and only the solves differ),
    timed with CUDA events on the lattice's stream (each trajectory's host
    work included).  Solvers: mixed (FP32 per-shift corrections), mixed
    with FP64 corrections, FP64."""
    import torch
    from susy_b200 import Lattice, RHMC
    lat = Lattice(DIMS, NCOL, pbc=-1, lam=LAM, bmass=BMASS, G=G)
    st = torch.cuda.Stream()
    lat.set_stream(st.cuda_stream)
    start = workload_links()[0]
    mk = lambda solver: RHMC(NORDER, NROOT, nstep=15, nstep_gauge=3, traj_length=1.0,
                             niter=MAXCG, error_per_site=1e-10, solver=solver)
    out = []
    for name, solver, c32 in (("mixed", 1, True), ("mixed_fp64_corrections", 1, False),
                              ("fp64", 0, True)):
        if args.traj_solvers and name not in args.traj_solvers.split(","):
            continue
        lat.set_links(start)
        lat.seed(TRAJ_SEED)
        lat.mixed_correction(c32)
        r = mk(solver)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        res = [lat.update(r) for _ in range(args.steps)]
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out.append({"solver": name, "s_per_traj": ms / 1e3,
                    "cg_iterations": [t["iters"] for t in res],
                    "delta_S": [t["delta_S"] for t in res],
                    "accept": [t["accept"] for t in res]})
        print(json.dumps(out[-1]), flush=True)
    lat.mixed_correction(True)
    print(json.dumps({"case": "rhmc_trajectory", "lattice": "12x12x12x24", "ncol": NCOL,
                      "nstep": 15, "nstep_gauge": 3, "nroot": NROOT, "norder": NORDER,
                      "runs": out}), flush=True)


def run_net_case(args):
    """The learned network's inference alone (the small case an ncu capture
    of its kernels runs): 8^4 U(3) (or --dims / --ncol), random weights,
    three applications to a complex-Gaussian Twist_Fermion, the time of the
    last two with CUDA events on the lattice's stream."""
    import torch
    from susy_b200 import Lattice, synth
    from susy_b200.learned import Net, init_weights
    dims = tuple(int(x) for x in args.dims.split(",")) if args.dims else (8, 8, 8, 8)
    ncol = args.ncol or 3
    lat = Lattice(dims, ncol, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    st = torch.cuda.ExternalStream(lat.stream)
    lat.set_links(synth.to_ref(dims, synth.links(dims, ncol, 0.2, 3)))
    net = Net(lat, init_weights(5, scale=0.4))
    a, b = lat.tf(64), lat.tf(64)
    a.upload(synth.to_ref(dims, synth.tf_source(dims, ncol, 1)))
    net.apply(a, b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(2):
        net.apply(a, b)
    e1.record(st)
    e1.synchronize()
    print(json.dumps({"case": "net_apply", "lattice": "x".join(map(str, dims)), "ncol": ncol,
                      "tensor_cores": bool(net.tensor_cores()),
                      "ms_per_apply": e0.elapsed_time(e1) / 2,
                      "out_max": float(np.abs(b.download()).max())}), flush=True)


def run_learned_case(args):
    """The learned-preconditioner protocol on one lattice (default 8^4 U(2);
    --dims / --ncol), lambda 1, bmass 0.2, G 0.05:
      chain   near-identity links (noise 0.2, seed 31), 200 RHMC
              trajectories (Nroot 1, degree 15, 10 x 2 steps, length 1,
              error_per_site 1e-5), every 5th saved: 40 configurations;
      pairs   --learned-pairs (100) per configuration, r complex Gaussian,
              e = (D^dag D + sigma_0)^-1 r by the FP64 solver (sigma_0 the
              smallest shift4 pole of Nroot 2), 30 configurations train, 10
              are held out;
      train   Adam on the A-norm error (the quantity CG minimises),
              --learned-steps steps of --learned-batch pairs;
      eval    on each held-out configuration one Gaussian source, the 15
              shift4 poles to the FP64 true residual 1e-10 per site: the
              FP64 multi-shift, the mixed solver, and a multi-shift pass to
              1e-6 followed by flexible CG on the 4 smallest shifts with
              and without the network (tensor-core inference); every
              solve capped at --learned-maxcg (50000) iterations.
    Prints one JSON line per held-out configuration and a summary."""
    import torch
    from susy_b200 import Lattice, RHMC, synth
    from susy_b200.learned import Net, congrad_multi_learned, make_pairs
    from susy_b200.rhmc_tables import rhmc
    dims = tuple(int(x) for x in args.dims.split(",")) if args.dims else (8, 8, 8, 8)
    ncol = args.ncol or 2
    lat = Lattice(dims, ncol, pbc=-1, lam=1.0, bmass=0.2, G=0.05, iseed=31)
    st = torch.cuda.Stream()
    lat.set_stream(st.cuda_stream)
    lat.set_links(synth.to_ref(dims, synth.links(dims, ncol, 0.2, 31)))
    chain = RHMC(15, 1, nstep=10, nstep_gauge=2, traj_length=1.0, error_per_site=1e-5)
    t0 = time.time()
    configs, acc = [], 0
    for i in range(1, 201):
        acc += int(lat.update(chain)["accept"])
        if i % 5 == 0:
            configs.append(lat.get_links())
    t_chain = time.time() - t0
    shifts = np.array(rhmc(15, 2)["shift4"])
    sigma0 = float(shifts[0])
    t0 = time.time()
    pairs = []
    for c, links in enumerate(configs[:30]):
        lat.set_links(links)
        for r, e in make_pairs(lat, sigma0, args.learned_pairs, seed=10000 + 1000 * c):
            pairs.append((r, e, links))
    t_pairs = time.time() - t0
    lat.set_links(configs[0])
    net = Net(lat)
    t0 = time.time()
    hist = net.train(pairs, steps=args.learned_steps, lr=2e-3, batch=args.learned_batch,
                     sigma=sigma0, log=max(1, args.learned_steps // 10))
    t_train = time.time() - t0
    del pairs
    print(json.dumps({"case": "learned_train", "lattice": "x".join(map(str, dims)), "ncol": ncol,
                      "trajectories": 200, "accepted": acc, "configs": len(configs),
                      "train_pairs": 30 * args.learned_pairs, "sigma0": sigma0,
                      "loss_first": hist[0], "loss_last10": float(np.mean(hist[-10:])),
                      "chain_s": t_chain, "pairs_s": t_pairs, "train_s": t_train}), flush=True)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        out = fn()
        e1.record(st)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    rows = []
    for c, links in enumerate(configs[30:]):
        lat.set_links(links)
        src = lat.tf(64)
        src.upload(synth.to_ref(dims, synth.tf_source(dims, ncol, 50000 + c)))
        b2 = float(np.dot(src.download(), src.download()))
        psim = [lat.tf(64) for _ in shifts]
        row = {"case": "learned_heldout", "config": 30 + c}
        cap = args.learned_maxcg
        lat.dev_congrad_multi(src, psim, shifts, cap, 1e-20)     # warm-up
        (it, _), ms = timed(lambda: lat.dev_congrad_multi(src, psim, shifts, cap, 1e-20))
        row["fp64"] = {"iterations": it, "ms": ms}
        (it, _), ms = timed(lambda: lat.dev_congrad_multi(src, psim, shifts, cap, 1e-20,
                                                          mixed=True))
        row["mixed"] = {"iterations": it, "ms": ms}
        for name, nn in (("refine_plain", None), ("refine_learned", net)):
            res, ms = timed(lambda: congrad_multi_learned(lat, nn, src, psim, shifts, cap,
                                                           1e-20, nrefine=4, loose=1e-12))
            it, rit, worst = res
            row[name] = {"iterations": it, "refine_iterations": rit, "ms": ms,
                         "true_residual_rel_max": worst / b2}
        rows.append(row)
        print(json.dumps(row), flush=True)
    summ = {k: {"iterations": float(np.mean([r[k]["iterations"] for r in rows])),
                "ms": float(np.mean([r[k]["ms"] for r in rows]))}
            for k in ("fp64", "mixed", "refine_plain", "refine_learned")}
    for k in ("refine_plain", "refine_learned"):
        summ[k]["refine_iterations"] = float(np.mean([r[k]["refine_iterations"] for r in rows]))
    print(json.dumps({"case": "learned_summary", "lattice": "x".join(map(str, dims)),
                      "ncol": ncol, "heldout": len(rows), "mean": summ,
                      "learned_vs_fp64": summ["fp64"]["ms"] / summ["refine_learned"]["ms"],
                      "learned_vs_plain_refinement":
                          summ["refine_plain"]["ms"] / summ["refine_learned"]["ms"]}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solver", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-traj", action="store_true",
                    help="skip the per-solver trajectory timing of the one-GPU line")
    ap.add_argument("--dsq-case", action="store_true",
                    help="operator microbenchmark per kernel variant instead of the solve")
    ap.add_argument("--variant", type=int, default=-1)
    ap.add_argument("--fop-variant", type=int, default=-1,
                    help="pin the operator kernel variant of the solve in both precisions "
                         "instead of autotuning it")
    ap.add_argument("--dims", default="", help="--dsq-case lattice, e.g. 24,24,24,24")
    ap.add_argument("--ncol", type=int, default=0, help="--dsq-case NCOL")
    ap.add_argument("--microbench-case", action="store_true",
                    help="8^4 U(2) operator and solver microbenchmark, 32 sources")
    ap.add_argument("--batch-case", action="store_true",
                    help="independent U(2) lattices of uneven volume, batched vs one by one")
    ap.add_argument("--batch-dsq-case", action="store_true",
                    help="D^dag D on the independent lattices in one launch vs one by one")
    ap.add_argument("--batch-cg-case", action="store_true",
                    help="the multi-shift solve on the independent lattices, batched vs one by one")
    ap.add_argument("--traj-solvers", default="",
                    help="with --traj-case: comma list of mixed, mixed_fp64_corrections, fp64")
    ap.add_argument("--traj-case", action="store_true",
                    help="full RHMC trajectories of the bench lattice, mixed and FP64 solver")
    ap.add_argument("--learned-case", action="store_true",
                    help="the learned-preconditioner protocol: chain, pairs, training, "
                         "held-out solves")
    ap.add_argument("--net-case", action="store_true",
                    help="the learned network's inference alone, 8^4 U(3)")
    ap.add_argument("--learned-pairs", type=int, default=100)
    ap.add_argument("--learned-steps", type=int, default=300)
    ap.add_argument("--learned-batch", type=int, default=8)
    ap.add_argument("--learned-maxcg", type=int, default=50000)
    ap.add_argument("--lattices", type=int, default=48)
    ap.add_argument("--threads", type=int, default=48)
    args = ap.parse_args()
    if args.dsq_case:
        run_dsq_case(args)
        return
    if args.microbench_case:
        run_microbench_case(args)
        return
    if args.batch_case:
        run_batch_case(args)
        return
    if args.batch_dsq_case:
        run_batch_dsq_case(args)
        return
    if args.batch_cg_case:
        run_batch_cg_case(args)
        return
    if args.traj_case:
        run_traj_case(args)
        return
    if args.learned_case:
        run_learned_case(args)
        return
    if args.net_case:
        run_net_case(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
