"""congrad_multi on many lattices at once (susy_b200_dev_congrad_multi_batch).

Every lattice of the batch must follow its own solve: the same FP64
recurrences as the per-iteration solver run alone (susy_b200_cg_blocked(h,
0)), so its iteration count within 1 of the solo one and every shift's
solution within 1e-8 relative (max-norm) of the solo solution at an FP64
residual of 1e-10 per site (the two differ only in the summation order of
the inner products).  The lattices differ in extents, couplings, fermion
mass, boundary condition, RESCALE and their shifts, so they stop at
different iterations while the others go on.
"""
import numpy as np
import pytest

from susy_b200 import Lattice, SusyError, congrad_multi_batch, synth

pytestmark = pytest.mark.gpu

FRONT = 12   # FOP_SITE_MAJOR_FRONT: the batched operator's products and order

CASES = [  # dims, lambda, G, fmass, pbc, rescale, shifts
    ((4, 4, 4, 4), 1.0, 0.05, 0.0, -1, 0, synth.geometric_shifts(6, 1e-3, 1.0)),
    ((6, 4, 4, 8), 2.0, 0.0, 0.1, -1, 0, synth.geometric_shifts(15, 1e-5, 1e3)),
    ((2, 2, 2, 2), 0.5, 0.1, 0.0, 1, 0, synth.geometric_shifts(3, 1e-2, 1.0)),
    ((8, 8, 8, 8), 4.0, 0.05, 0.0, -1, 0, synth.geometric_shifts(10, 1e-4, 1e2)),
    ((4, 4, 4, 8), 1.0, 0.05, 0.2, -1, 1, np.array([1e-2])),
]


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def setup(k, dims, lam, G, fm, pbc, rs):
    lat = Lattice(dims, 2, pbc=pbc, lam=lam, bmass=0.2, G=G, fmass=fm)
    lat.set_links(synth.to_ref(dims, synth.links(dims, 2, 0.2, 30 + k)))
    if rs:
        lat.set_rescale(1)
    lat.fop_variant(64, FRONT)
    lat.cg_blocked(0)
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, 2, 80 + k)))
    return lat, src


def test_batch_solve_follows_each_lattice_alone():
    maxcg, errormin = 5000, 1e-20
    lats, srcs, solo, solo_it, psims = [], [], [], [], []
    for k, (dims, lam, G, fm, pbc, rs, shifts) in enumerate(CASES):
        lat, src = setup(k, dims, lam, G, fm, pbc, rs)
        ref = [lat.tf(64) for _ in shifts]
        it, _ = lat.dev_congrad_multi(src, ref, shifts, maxcg, errormin)
        solo.append([p.download() for p in ref])
        solo_it.append(it)
        lats.append(lat)
        srcs.append(src)
        psims.append([lat.tf(64) for _ in shifts])
    iters, rsq = congrad_multi_batch(srcs, psims, [c[6] for c in CASES], maxcg, errormin)
    assert len(set(iters)) > 1          # the lattices stop at different iterations
    for k in range(len(CASES)):
        assert abs(iters[k] - solo_it[k]) <= 1, (k, iters[k], solo_it[k])
        assert np.isfinite(rsq[k])
        for x, want in zip(psims[k], solo[k]):
            assert rel(x.download(), want) <= 1e-8, k


def test_batch_solve_refuses_a_handle_twice_and_bad_counts():
    lat, src = setup(0, *CASES[0][:6])
    shifts = CASES[0][6]
    ps = [lat.tf(64) for _ in shifts]
    with pytest.raises(SusyError):
        congrad_multi_batch([src, src], [ps, ps], [shifts, shifts], 100, 1e-16)
    with pytest.raises(SusyError):
        congrad_multi_batch([src], [[lat.tf(64) for _ in range(33)]],
                            [synth.geometric_shifts(33, 1e-3, 1.0)], 100, 1e-16)
