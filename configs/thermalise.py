"""Thermalise the 12^3 x 24 U(3) benchmark lattice and save it.

The benchmark configuration (lambda 2, bmass 0.3, G 0.05, antiperiodic
temporal fermion BC) starts from links near the identity (noise 0.1, seed
11: susy_b200.synth.links) and is thermalised by 20 RHMC trajectories of
the benchmark's own integrator: degree-15 rational approximation with
Nroot 2, 15 fermion steps x 3 gauge steps, trajectory length 1,
error_per_site 1e-10, Metropolis with the node generator (site and node
generators seeded with 13), run on the GPU by this library.  The final
links are written in the reference's serial gauge format (io_lat.c:377,
float32 links with checksums, plus the .info file) as
configs/thermalised_12x12x12x24_u3.lat, and every trajectory's delta S,
acceptance, CG iterations and plaquette go to
configs/thermalised_12x12x12x24_u3.json.  bench.py reads the file and
checks its checksums.

  python configs/thermalise.py [--trajectories 20] [--solver mixed|fp64] [--out PATH]
                               [--resume PATH.state.npz]

The state is saved after every trajectory, so a run that is stopped can be
continued with --resume (the generators are then reseeded with 13 plus the
number of trajectories done).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

DIMS = (12, 12, 12, 24)
NCOL = 3
LAM, BMASS, G = 2.0, 0.3, 0.05
LINK_NOISE, LINK_SEED, SEED = 0.1, 11, 13
OUT = os.path.join(HERE, "thermalised_12x12x12x24_u3.lat")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--trajectories", type=int, default=20)
    ap.add_argument("--solver", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--out", default=OUT)
    ap.add_argument("--resume", default="",
                    help="continue from the .state.npz a previous run left")
    a = ap.parse_args()
    out = a.out
    from susy_b200 import Lattice, RHMC, io_lat, synth
    from susy_b200.lattice import SOLVER_FP64, SOLVER_MIXED
    import numpy as np
    lat = Lattice(DIMS, NCOL, pbc=-1, lam=LAM, bmass=BMASS, G=G, iseed=SEED)
    lat.set_links(synth.to_ref(DIMS, synth.links(DIMS, NCOL, LINK_NOISE, LINK_SEED)))
    r = RHMC(15, 2, nstep=15, nstep_gauge=3, traj_length=1.0, niter=50000,
             error_per_site=1e-10, solver=SOLVER_MIXED if a.solver == "mixed" else SOLVER_FP64)
    log = []

    def save():
        # the state after every trajectory: FP64 links (.npz, to continue
        # from) and the gauge file with the log
        links = synth.from_ref(DIMS, lat.get_links(), 5, NCOL)
        np.savez(os.path.splitext(out)[0] + ".state.npz", links=links, log=json.dumps(log))
        s29, s31 = io_lat.write_gauge(out, DIMS, links,
                                      stamp="thermalised %d RHMC trajectories" % len(log))
        with open(os.path.splitext(out)[0] + ".json", "w") as f:
            json.dump({"lattice": "x".join(map(str, DIMS)), "ncol": NCOL, "lambda": LAM,
                       "bmass": BMASS, "G": G, "start": "identity + %g noise, seed %d"
                       % (LINK_NOISE, LINK_SEED), "seed": SEED, "nroot": 2, "norder": 15,
                       "nstep": 15, "nstep_gauge": 3, "traj_length": 1.0,
                       "error_per_site": 1e-10, "solver": a.solver,
                       "checksums": "%x %x" % (s29, s31), "trajectories": log}, f, indent=1)
        return s29, s31

    if a.resume:
        st = np.load(a.resume)
        log = json.loads(str(st["log"]))
        lat.set_links(synth.to_ref(DIMS, st["links"]))
        # the generators continue as a fresh seed plus the trajectories done
        lat.seed(SEED + len(log))
    for i in range(len(log), a.trajectories):
        t0 = time.time()
        res = lat.update(r)
        ss, st = lat.plaquette()
        rec = {"trajectory": i + 1, "delta_S": res["delta_S"], "accept": int(res["accept"]),
               "cg_iterations": res["iters"], "ss_plaq": ss, "st_plaq": st,
               "seconds": time.time() - t0}
        log.append(rec)
        print(json.dumps(rec), flush=True)
        s29, s31 = save()
    print("wrote %s (checksums %x %x)" % (out, s29, s31))


if __name__ == "__main__":
    main()
