"""Record the FP64 multi-shift solve of the benchmark workload.

On the thermalised 12^3 x 24 U(3) configuration
(configs/thermalised_12x12x12x24_u3.lat), the benchmark's source
(synth.tf_source seed 12) and the 15 shift4 poles of the Nroot = 2 degree-15
rational approximation, the FP64 multi-shift CG (the reference's
recurrences and freeze rule, congrad_multi.c:76-181) to the true residual
1e-10 per site: its iteration count and the iteration at which each shift
froze.  The reference's CPU solve takes the same iterations (the
recurrences are the same; tests pin the count to +-1), so bench.py's
reference arm weights its per-iteration samples by this schedule of live
shifts.  Writes configs/solve_profile_12x12x12x24_u3.json.

  python configs/solve_profile.py [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
OUT = os.path.join(HERE, "solve_profile_12x12x12x24_u3.json")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    import numpy as np
    import bench
    from susy_b200 import Lattice, synth
    from susy_b200.rhmc_tables import rhmc
    links, info = bench.workload_links()
    lat = Lattice(bench.DIMS, bench.NCOL, pbc=-1, lam=bench.LAM, bmass=bench.BMASS, G=bench.G)
    lat.set_links(links)
    shifts = np.array(rhmc(bench.NORDER, bench.NROOT)["shift4"])
    src = lat.tf(64)
    src.upload(synth.to_ref(bench.DIMS, synth.tf_source(bench.DIMS, bench.NCOL, bench.SRC_SEED)))
    psim = [lat.tf(64) for _ in shifts]
    it, rsq = lat.dev_congrad_multi(src, psim, shifts, bench.MAXCG, bench.ERRORMIN)
    frozen = lat.cg_freeze_iterations(len(shifts))
    live = [sum(1 for f in frozen if f >= i) for i in range(1, it + 1)]
    out = {"workload": bench.WORKLOAD, "links_checksums": info["checksums"],
           "solver": "fp64 multi-shift", "iterations": it, "final_rsq": rsq,
           "shifts": list(shifts), "freeze_iteration": frozen,
           "live_shifts_per_iteration": live}
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print("iterations %d, live shifts summed over iterations %d -> %s" % (it, sum(live), a.out))


if __name__ == "__main__":
    main()
