"""Generate tests/golden/ops_U3_8x8x8x16.npz from the reference itself.

The unmodified reference operator (oracle/_ref/libsusyref_n3.so, built by
oracle/build_ref.sh) applied to seeded inputs on an 8^3 x 16 U(3) lattice:
links synth.links(dims, 3, 0.2, seed 303), source synth.tf_source(dims, 3,
seed 304), lambda 2, bmass 0.3, G 0.05, antiperiodic temporal BC.  Both
inputs are regenerated from the seeds where the fixture is used, so the
file keeps only what pins the outputs without holding whole fields
(a full U(3) Twist_Fermion at this size is 18.9 MB):

  sites         256 site indices (node_index order): random sites plus
                sites on both temporal boundaries
  fop_plus, fop_minus, DSq
                the reference's outputs at those sites, [256, 16, 3, 3, 2]
  norm2_*       |output|^2 over the whole lattice
  proj_*        Re and Im of sum_x w(x) . output(x) for 4 complex Gaussian
                weight fields w (numpy PCG64 seeds 305..308)

Run where the reference sources and oracle/_ref exist:

    python tests/golden/make_golden_u3_large.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DIMS = (8, 8, 8, 16)
N = 3
LINK_SEED, SRC_SEED, SITE_SEED = 303, 304, 309
PROJ_SEEDS = (305, 306, 307, 308)
PARAMS = dict(lam=2.0, bmass=0.3, G=0.05, pbc=-1)


def weights(seed, n):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def pick_sites():
    """256 node_index sites: 192 at random, 64 on the t = 0 and t = nt-1 slices."""
    from susy_b200 import synth
    V = int(np.prod(DIMS))
    rng = np.random.default_rng(SITE_SEED)
    lex = rng.choice(V, 192, replace=False)
    per_t = V // DIMS[3]
    lex = np.concatenate([lex, rng.choice(per_t, 32, replace=False),
                          V - per_t + rng.choice(per_t, 32, replace=False)])
    return np.unique(synth.node_index(DIMS)[lex])


def summarise(flat, sites):
    V = int(np.prod(DIMS))
    a = flat.reshape(V, 16, N, N, 2)
    z = (a[..., 0] + 1j * a[..., 1]).reshape(-1)
    proj = [complex(np.sum(weights(sd, z.size) * z)) for sd in PROJ_SEEDS]
    return a[sites], float(np.vdot(z, z).real), np.array([[p.real, p.imag] for p in proj])


def job():
    from oracle.ref_ctypes import RefLattice
    from susy_b200 import synth
    ref = RefLattice(N, dims=DIMS, pbc=PARAMS["pbc"], lam=PARAMS["lam"],
                     bmass=PARAMS["bmass"], G=PARAMS["G"])
    ref.set_links(synth.to_ref(DIMS, synth.links(DIMS, N, 0.2, LINK_SEED)))
    ref.compute_all()
    src = synth.to_ref(DIMS, synth.tf_source(DIMS, N, SRC_SEED))
    sites = pick_sites()
    out = dict(dims=np.array(DIMS), N=N, sites=sites)
    for name, val in (("fop_plus", ref.fermion_op(src, 1)), ("fop_minus", ref.fermion_op(src, -1)),
                      ("DSq", ref.DSq(src))):
        at, n2, pj = summarise(val, sites)
        out[name] = at
        out["norm2_" + name] = n2
        out["proj_" + name] = pj
    return out


def main():
    from oracle.ref_ctypes import run_in_fresh_process
    out = run_in_fresh_process(job)
    path = os.path.join(HERE, "ops_U3_8x8x8x16.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
