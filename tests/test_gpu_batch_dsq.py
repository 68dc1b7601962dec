"""Many lattices in one operator launch (susy_b200_DSq_batch).

The batched D^dag D walks one work table of (lattice, 128-site tile, output
component) items for all lattices in a single persistent launch per sign.
Each lattice must get what its own site-major table-driven kernel gives it
(variant FOP_SITE_MAJOR_FRONT, the same products in the same order): FP64
within 1e-13 and FP32 within 1e-6 relative (max-norm), and the FP64 result
of one lattice is also checked against the numpy oracle at 1e-13.
Lattices differ in extents, couplings (G = 0 switches the determinant
terms off), fermion mass, boundary condition and the RESCALE setting.
"""
import numpy as np
import pytest

from oracle import susy_np as O
from susy_b200 import Lattice, SusyError, dsq_batch, synth

pytestmark = pytest.mark.gpu

FRONT = 12   # FOP_SITE_MAJOR_FRONT

MIXED = [  # dims, lambda, G, fmass, pbc, rescale
    ((4, 4, 4, 4), 1.0, 0.05, 0.0, -1, 0),
    ((6, 4, 4, 8), 2.0, 0.0, 0.1, -1, 0),
    ((2, 2, 2, 2), 0.5, 0.1, 0.0, 1, 0),
    ((8, 8, 8, 8), 4.0, 0.05, 0.0, -1, 0),
    ((4, 4, 4, 8), 1.0, 0.05, 0.2, -1, 1),
]


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def make(dims, N, lam, G, fmass, pbc, rescale, seed):
    lat = Lattice(dims, N, pbc=pbc, lam=lam, bmass=0.2, G=G, fmass=fmass)
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.2, seed)))
    if rescale:
        lat.set_rescale(1)
    return lat


def run(cases, N, prec):
    lats, srcs, refs, outs, host = [], [], [], [], []
    for k, (dims, lam, G, fm, pbc, rs) in enumerate(cases):
        lat = make(dims, N, lam, G, fm, pbc, rs, 10 + k)
        lat.fop_variant(prec, FRONT)
        h = synth.to_ref(dims, synth.tf_source(dims, N, 50 + k))
        s64 = lat.tf(64)
        s64.upload(h)
        if prec == 64:
            s = s64
        else:
            s = lat.tf(32)
            lat.dev_convert(s64, s)
        r, o = lat.tf(prec), lat.tf(prec)
        lat.dev_DSq(s, r)
        lats.append(lat)
        srcs.append(s)
        refs.append(r)
        outs.append(o)
        host.append(h)
    dsq_batch(srcs, outs)
    return lats, host, [r.download() for r in refs], [o.download() for o in outs]


@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-6)])
def test_batch_equals_each_lattice_alone(prec, tol):
    _, _, refs, outs = run(MIXED, 2, prec)
    for r, o in zip(refs, outs):
        assert rel(o, r) <= tol


def test_batch_matches_the_oracle():
    lats, host, _, outs = run(MIXED[:2], 3, 64)
    dims, lam, G, fm, pbc, _ = MIXED[1]
    U = synth.links(dims, 3, 0.2, 11)
    geo = O.Geometry(dims, pbc)
    prm = O.Params(lam=lam, bmass=0.2, G=G, N=3, fmass=fm)
    der = O.compute_derived(geo, prm, U)
    want = O.DSq(geo, prm, U, der, synth.from_ref(dims, host[1], 16, 3))
    assert rel(synth.from_ref(dims, outs[1], 16, 3), want) <= 1e-13


def test_batch_of_config4_volumes():
    """48 U(2) lattices drawn from the batched scan's volumes and couplings
    in one pair of launches, each equal to its own launch."""
    vols = [(4, 4, 4, 4), (6, 6, 6, 6), (8, 8, 8, 8), (4, 4, 4, 8), (6, 6, 6, 12), (8, 8, 8, 16)]
    lams = [0.5, 1.0, 2.0, 4.0]
    cases = [(vols[k % 6], lams[k % 4], 0.05, 0.0, -1, 0) for k in range(48)]
    for prec, tol in ((64, 1e-13), (32, 1e-6)):
        _, _, refs, outs = run(cases, 2, prec)
        assert max(rel(o, r) for r, o in zip(refs, outs)) <= tol


def test_batch_refuses_bad_input_before_any_launch():
    a = make((4, 4, 4, 4), 2, 1.0, 0.05, 0.0, -1, 0, 1)
    b = make((4, 4, 4, 4), 3, 1.0, 0.05, 0.0, -1, 0, 2)
    sa, da, sb, db = a.tf(64), a.tf(64), b.tf(64), b.tf(64)
    with pytest.raises(SusyError):
        dsq_batch([sa, sb], [da, db])           # NCOL 2 and 3
    with pytest.raises(SusyError):
        dsq_batch([sa] * 65, [da] * 65)         # above SUSY_B200_BATCH_MAX
