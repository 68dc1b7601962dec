"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources and oracle/_ref (oracle/build_ref.sh) exist:

    python tests/golden/make_golden.py

Writes
  ops_U2.npz, ops_U3.npz   seeded inputs and the UNMODIFIED reference's outputs
                           (oracle/_ref, reference layout, node_index order) for
                           compute_plaqdet/Uinv/DmuUmu/Fmunu, fermion_op(+-1),
                           DSq, congrad_multi, fermion_force, gauge_force
                           (with det_force), action pieces and ranmom;
  hmc_U2.json, hmc_U3.json the reference's regression outputs
                           testsuite/scalar/hmc.U{2,3}.ref (per-trajectory
                           action pieces, delta S, accept, IT_PER_TRAJ) with
                           the run parameters of testsuite/in.U{2,3}.hmc;
  config_U2_4444.npz, config_U3_4444.npz
                           the starting links of those runs (testsuite/
                           config.U{2,3}.4444, read with susy_b200.io_lat);
  config0_U2.json          the reference run through the harness on the
                           4^4 U(2) configuration the benchmark's first
                           config names (identity + 0.05 noise links from
                           synth.links seed 0, lambda 1, bmass 0.2, G 0.05,
                           Nroot 1, Norder 15, 10 x 2 steps, error_per_site
                           1e-10): two trajectories' action lines, delta S,
                           accept, IT_PER_TRAJ and force monitors.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get("SUSY_REFERENCE", "/root/reference") + "/4d_Q16"

OPS = {2: dict(dims=(4, 4, 2, 4), seed=101), 3: dict(dims=(2, 4, 2, 4), seed=202)}
PARAMS = dict(lam=1.0, bmass=0.3, G=0.05, kappa_u1=0.4, fmass=0.0, pbc=-1, iseed=41)
SHIFTS = [1e-5 * 1e8 ** (j / 14.0) for j in range(15)]
KEEP = [0, 7, 14]


def ops_job(N, dims, seed):
    from oracle.ref_ctypes import RefLattice
    from susy_b200 import synth
    ref = RefLattice(N, dims=dims, pbc=PARAMS["pbc"], iseed=PARAMS["iseed"], lam=PARAMS["lam"],
                     bmass=PARAMS["bmass"], G=PARAMS["G"], kappa_u1=PARAMS["kappa_u1"],
                     fmass=PARAMS["fmass"])
    U = synth.links(dims, N, 0.2, seed)
    links = synth.to_ref(dims, U)
    ref.set_links(links)
    ref.compute_all()
    out = dict(dims=np.array(dims), N=N, seed=seed, links=links)
    out["plaqdet"] = ref.plaqdet()
    out["DmuUmu"] = ref.DmuUmu()
    out["Fmunu"] = ref.Fmunu()
    out["Uinv"] = ref.Uinv()
    src = synth.to_ref(dims, synth.tf_source(dims, N, seed + 1))
    out["src"] = src
    out["fop_plus"] = ref.fermion_op(src, 1)
    out["fop_minus"] = ref.fermion_op(src, -1)
    out["DSq"] = ref.DSq(src)
    psim, it, rsq = ref.congrad_multi(src, np.array(SHIFTS), 5000, 1e-20)
    out["cg_shifts"] = np.array(SHIFTS)
    out["cg_iters"] = it
    out["cg_rsq"] = rsq
    out["cg_keep"] = np.array(KEEP)
    out["cg_psim"] = psim[KEEP]
    amp = np.array([0.3, 1.7, 0.02])
    sols = np.stack([synth.to_ref(dims, synth.tf_source(dims, N, seed + 10 + k))
                     for k in range(3)])
    out["ff_sol"] = sols
    out["ff_amp"] = amp
    ref.set_mom(np.zeros_like(links))
    # fermion_force reads amp4/Norder globals: give it Norder = 3 poles via the
    # harness by solving the identity that amp4 are the first Norder entries
    out["ff_norm"] = _fermion_force_with_amps(ref, 0.11, src, sols, amp)
    out["ff_mom"] = ref.mom()
    mom0 = synth.to_ref(dims, synth.links(dims, N, 0.5, seed + 20) - np.eye(N))
    out["gf_mom0"] = mom0
    ref.set_mom(mom0)
    out["gf_norm"] = ref.gauge_force(0.07)
    out["gf_mom"] = ref.mom()
    ref.set_mom(mom0)
    out["action_parts"] = ref.action_parts(src, psim)
    out["action_amp4"] = ref.rhmc()["amp4"]
    out["action_ampdeg4"] = ref.rhmc()["ampdeg4"]
    ref.ranmom()
    out["ranmom"] = ref.mom()
    # per-trajectory measurements of control.c:85-138 on these links
    ref.set_links(links)
    ref.compute_all()
    lt = ref.link_trace()
    for k in ("linktr", "link_det"):
        out["meas_" + k] = lt[k]
    out["meas_lt_scalars"] = np.array([lt["linktr_ave"], lt["linktr_width"], lt["det_ave"],
                                       lt["det_width"]])
    pl = [ref.ploop(d, p) for p in (0, 1) for d in range(5)]
    out["meas_lines"] = np.array([c for c, _ in pl])
    out["meas_ploop_mod"] = pl[3][1]
    out["meas_plaq"] = np.array(ref.plaquette())
    out["meas_det"] = ref.measure_det()
    out["meas_widths"] = ref.widths()
    out["meas_uubar"] = np.array(ref.scalar_eig(0))
    out["meas_polar"] = np.array(ref.scalar_eig(1))
    out["meas_gauge_action"] = ref.gauge_action(0)
    return out


def _fermion_force_with_amps(ref, eps, src, sols, amp):
    """fermion_force over len(amp) poles with the given amplitudes.

    The reference takes Norder and amp4 from globals set by setup_rhmc; the
    harness exposes amp4 through ref_rhmc only, so the amplitudes are
    written into the reference's amp4 array through ctypes."""
    import ctypes as C
    lib = ref.lib
    amp4 = C.POINTER(C.c_double).in_dll(lib, "amp4")
    norder = C.c_int.in_dll(lib, "Norder")
    saved = [amp4[j] for j in range(norder.value)]
    saved_n = norder.value
    for j, a in enumerate(amp):
        amp4[j] = a
    norder.value = len(amp)
    try:
        return ref.fermion_force(eps, src, sols)
    finally:
        for j, a in enumerate(saved):
            amp4[j] = a
        norder.value = saved_n


def parse_hmc_ref(path):
    return parse_hmc_text(open(path).read())


def parse_hmc_text(txt):
    trajs = []
    acts = re.findall(r"action: gauge (\S+) bmass (\S+) det (\S+) fermion0 (\S+) mom (\S+) sum (\S+)",
                      txt)
    acc = re.findall(r"(ACCEPT|REJECT): delta S = (\S+) start S = (\S+) end S = (\S+)", txt)
    its = re.findall(r"IT_PER_TRAJ (\d+)", txt)
    mon = re.findall(r"MONITOR_FORCE_GAUGE\s+(\S+) (\S+)\nMONITOR_FORCE_FERMION0 (\S+) (\S+)", txt)
    for k in range(len(acc)):
        trajs.append(dict(start_action=[float(x) for x in acts[2 * k]],
                          end_action=[float(x) for x in acts[2 * k + 1]],
                          accept=acc[k][0] == "ACCEPT", delta_S=float(acc[k][1]),
                          start_S=float(acc[k][2]), end_S=float(acc[k][3]),
                          it_per_traj=int(its[k]),
                          monitor=[float(x) for x in mon[k]]))
    start = re.search(r"START (\S+) (\S+) (\S+) (\S+)", txt)
    start = start.groups() if start else ()
    # measurement lines (control.c:52-68 at start, :85-138 per trajectory)
    nums = lambda line: [float(x) for x in line.split()[1:]]
    lines = txt.splitlines()
    meas, cur = [], None
    start_meas = {}
    for ln in lines:
        tag = ln.split()[0] if ln.split() else ""
        if tag in ("FLINK", "FLINK_DET") and not trajs_started(lines, ln):
            start_meas[tag] = nums(ln)
        if tag == "FLINK" and trajs_started(lines, ln):
            cur = {}
            meas.append(cur)
        if cur is not None and tag in ("FLINK", "GMES", "BACTION", "LINES", "LINES_POLAR", "DET",
                                       "WIDTHS"):
            cur[tag] = nums(ln)
        if cur is not None and tag in ("UUBAR_EIG", "POLAR_EIG"):
            cur.setdefault(tag, []).append(nums(ln)[1:])
    for k, m in enumerate(meas):
        trajs[k]["meas"] = m
    stop = re.search(r"STOP (\S+) (\S+) (\S+) (\S+)", txt)
    return dict(trajectories=trajs, start_line=[float(x) for x in start], start_meas=start_meas,
                stop_line=[float(x) for x in stop.groups()] if stop else None)


def trajs_started(lines, line):
    """True once the first trajectory's output precedes this line"""
    i = lines.index(line)
    return any(l.startswith("IT_PER_TRAJ") for l in lines[:i])


CONFIG0 = dict(dims=(4, 4, 4, 4), pbc=-1, iseed=41, Nroot=1, Norder=15, traj_length=1.0,
               nstep=10, nstep_gauge=2, lam=1.0, kappa_u1=0.0, bmass=0.2, fmass=0.0, G=0.05,
               max_cg=5000, error_per_site=1e-10)
CONFIG0_LINKS = dict(noise=0.05, seed=0)


def config0_job(ntraj=2):
    from oracle.ref_ctypes import RefLattice
    from susy_b200 import synth
    ref = RefLattice(2, **CONFIG0)
    U = synth.links(CONFIG0["dims"], 2, CONFIG0_LINKS["noise"], CONFIG0_LINKS["seed"])
    ref.set_links(synth.to_ref(CONFIG0["dims"], U))
    ref.set_mom(np.zeros_like(synth.to_ref(CONFIG0["dims"], U)))
    ref.compute_all()
    out = []
    for _ in range(ntraj):
        start = len(ref.log())
        ref.update()
        out.append(parse_hmc_text(ref.log()[start:])["trajectories"][0])
    return out


def parse_input(path):
    kv = {}
    for line in open(path):
        p = line.split()
        if len(p) == 2:
            kv[p[0]] = p[1]
    return kv


def main():
    from oracle.ref_ctypes import run_in_fresh_process
    from susy_b200.io_lat import read_gauge
    for N, cfg in OPS.items():
        res = run_in_fresh_process(ops_job, N, cfg["dims"], cfg["seed"])
        np.savez(os.path.join(HERE, "ops_U%d.npz" % N), **res)
        print("ops_U%d.npz: cg iters %d" % (N, res["cg_iters"]))
    for N in (2, 3):
        d = parse_hmc_ref(os.path.join(REF, "testsuite/scalar/hmc.U%d.ref" % N))
        d["input"] = parse_input(os.path.join(REF, "testsuite/in.U%d.hmc" % N))
        with open(os.path.join(HERE, "hmc_U%d.json" % N), "w") as f:
            json.dump(d, f, indent=1)
        dims, ncol, links, info = read_gauge(os.path.join(REF, "testsuite/config.U%d.4444" % N))
        assert info["checksum_ok"]
        np.savez(os.path.join(HERE, "config_U%d_4444.npz" % N), dims=np.array(dims),
                 links=links.astype(np.complex64), sum29=info["sum29"], sum31=info["sum31"])
        print("hmc_U%d.json: %d trajectories" % (N, len(d["trajectories"])))
    c0 = run_in_fresh_process(config0_job)
    with open(os.path.join(HERE, "config0_U2.json"), "w") as f:
        json.dump({"params": {k: list(v) if isinstance(v, tuple) else v
                              for k, v in CONFIG0.items()},
                   "links": CONFIG0_LINKS, "trajectories": c0}, f, indent=1)
    print("config0_U2.json: %d trajectories" % len(c0))


if __name__ == "__main__":
    main()
