"""CPU checks of the learned preconditioner's definition (oracle/learned_np.py):
analytic weight gradients against central finite differences, and gauge
covariance of the network under a random GL(N) gauge transformation (the
network has no reference counterpart; these pin its definition)."""
import numpy as np
import pytest

from oracle import susy_np as O
from oracle import learned_np as Lr
from susy_b200 import synth


def setup(dims=(2, 2, 2, 4), N=2):
    geo = O.Geometry(dims, -1)
    U = synth.links(dims, N, 0.3, 3)
    return geo, U, np.linalg.inv(U)


def test_gradient_matches_finite_differences():
    geo, U, Ui = setup()
    Ws = Lr.init_weights(1, scale=0.3)
    rs = [synth.tf_source(geo.dims, 2, 10 + i) for i in range(2)]
    es = [synth.tf_source(geo.dims, 2, 20 + i) for i in range(2)]
    _, G = Lr.loss_and_grad(geo, U, Ui, Ws, rs, es)
    rng = np.random.default_rng(0)
    h = 1e-6
    for li in range(3):
        for _ in range(3):
            k, d, c = [int(rng.integers(s)) for s in Ws[li].shape]
            for unit in (1.0, 1j):
                Wp = [w.copy() for w in Ws]
                Wm = [w.copy() for w in Ws]
                Wp[li][k, d, c] += h * unit
                Wm[li][k, d, c] -= h * unit
                num = (Lr.loss_and_grad(geo, U, Ui, Wp, rs, es)[0]
                       - Lr.loss_and_grad(geo, U, Ui, Wm, rs, es)[0]) / (2 * h)
                an = 2 * (G[li][k, d, c].real if unit == 1.0 else G[li][k, d, c].imag)
                assert abs(num - an) <= 1e-6 * max(abs(an), 1e-3)


def test_network_is_gauge_covariant():
    geo, U, Ui = setup()
    N = 2
    rng = np.random.default_rng(4)
    g = np.eye(N) + 0.3 * (rng.standard_normal((geo.V, N, N)) + 1j * rng.standard_normal((geo.V, N, N)))
    gi = np.linalg.inv(g)
    Ug = np.stack([g @ U[m] @ geo.shift(gi, m) for m in range(5)])

    def transform(tf):
        o = np.empty_like(tf)
        o[0] = g @ tf[0] @ gi
        for a in range(5):
            o[1 + a] = g @ tf[1 + a] @ geo.shift(gi, a)
        for (a, b) in O.PLAQ_PAIRS:
            p = O.PLAQ_INDEX[a, b]
            o[6 + p] = g @ tf[6 + p] @ geo.shift(gi, a, b)
        return o

    Ws = Lr.init_weights(2, scale=0.5)
    r = synth.tf_source(geo.dims, N, 5)
    z = Lr.forward(geo, U, Ui, Ws, r)
    zg = Lr.forward(geo, Ug, np.linalg.inv(Ug), Ws, transform(r))
    assert np.abs(zg - transform(z)).max() <= 1e-12 * np.abs(zg).max()


def test_transport_adjoint():
    geo, U, Ui = setup((2, 4, 2, 4), 3)
    rng = np.random.default_rng(1)
    X = rng.standard_normal((2, geo.V, 3, 3)) + 1j * rng.standard_normal((2, geo.V, 3, 3))
    G = rng.standard_normal((11, 2, geo.V, 3, 3)) + 1j * rng.standard_normal((11, 2, geo.V, 3, 3))
    lhs = np.vdot(Lr.transports(geo, U, Ui, X), G)
    rhs = np.vdot(X, Lr.transports_adjoint(geo, U, Ui, G))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
