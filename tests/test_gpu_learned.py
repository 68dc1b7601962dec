"""GPU checks of the learned preconditioner (susy_b200/csrc/learned.cu)
against its CPU definition (oracle/learned_np.py, itself checked by
tests/test_learned_oracle.py): the forward pass and the loss gradient with
the same bfloat16 weights, to FP32 accuracy (1e-5 forward, 1e-4 gradient);
the learned solve's FP64 true residual; and what training gains.
"""
import numpy as np
import pytest

from oracle import susy_np as O
from oracle import learned_np as Lr
from susy_b200 import Lattice, synth
from susy_b200.learned import Net, congrad_multi_learned, init_weights, make_pairs

pytestmark = pytest.mark.gpu


def setup(dims, N, seed=3):
    U = synth.links(dims, N, 0.25, seed)
    lat = Lattice(dims, N, pbc=-1, lam=1.0, bmass=0.2, G=0.05)
    lat.set_links(synth.to_ref(dims, U))
    return lat, O.Geometry(dims, -1), U


@pytest.mark.parametrize("dims,N", [((4, 4, 2, 4), 2), ((2, 2, 2, 4), 3), ((2, 2, 2, 4), 4)])
def test_forward_and_gradient_match_the_definition(dims, N):
    lat, geo, U = setup(dims, N)
    Ws = [Lr.bf16(W) for W in init_weights(5, scale=0.4)]
    net = Net(lat, Ws)
    r = synth.tf_source(dims, N, 11)
    e = synth.tf_source(dims, N, 12)
    dr, de, dz = lat.tf(64), lat.tf(64), lat.tf(64)
    dr.upload(synth.to_ref(dims, r))
    de.upload(synth.to_ref(dims, e))
    Ui = np.linalg.inv(U)
    want = Lr.forward(geo, U, Ui, Ws, r)
    # FP32 channel mixes: the definition to FP32 accuracy
    assert net.tensor_cores(0) == 1
    net.apply(dr, dz)
    got = synth.from_ref(dims, dz.download(), 16, N)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    # tensor-core mixes (BF16 transports, FP32 accumulation): bfloat16
    # accuracy (8 significant bits) through three layers against the FP32
    # definition, and closer to the definition with its transports rounded
    # to bfloat16 than to the FP32 one.  The device's FP32 transports and
    # the definition's FP64 ones differ in the last FP32 bits, so a few of
    # them round to neighbouring bf16 values, and those differences grow
    # over the layers: the bf16 definition is no bit-level emulation
    # (measured: 1.6-2.6e-3 against it, 3.3-4.6e-3 against FP32)
    net.tensor_cores(1)
    net.apply(dr, dz)
    got = synth.from_ref(dims, dz.download(), 16, N)
    want16 = Lr.forward(geo, U, Ui, Ws, r, bf16_act=True)
    e16 = np.abs(got - want16).max() / np.abs(want16).max()
    e32 = np.abs(got - want).max() / np.abs(want).max()
    print("tensor-core forward: rel. error %.2e vs bf16 definition, %.2e vs FP32" % (e16, e32))
    assert e32 <= 1e-2 and e16 < e32
    loss, g = net.loss_grad(dr, de)
    wl, wg = Lr.loss_and_grad(geo, U, Ui, Ws, [r], [e])
    assert abs(loss - wl) <= 1e-5 * wl
    for a, b in zip(g, wg):
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()


def test_learned_solve_reaches_the_fp64_bound():
    dims, N = (4, 4, 4, 4), 2
    lat, geo, U = setup(dims, N)
    net = Net(lat)
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, N, 7)))
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    psim = [lat.tf(64) for _ in shifts]
    it, rit, worst = congrad_multi_learned(lat, net, src, psim, shifts, 20000, 1e-20)
    b2 = float(np.dot(src.download(), src.download()))
    assert worst <= 1e-20 * b2 and rit > 0
    for j, s in enumerate(shifts):
        x = psim[j].download()
        t = lat.tf(64)
        lat.dev_DSq(psim[j], t)
        r = src.download() - t.download() - s * x
        assert float(np.dot(r, r)) <= 1e-20 * b2


@pytest.mark.parametrize("sigma_loss", [False, True])
def test_training_lowers_the_loss_and_reports_the_gain(sigma_loss):
    """Train on pairs from one configuration (plain relative error, or the
    A-norm error CG minimises), evaluate the refinement iterations of the 4
    smallest shifts on a held-out configuration with and without the
    trained network.  Both solves must meet the FP64 bound; the iteration
    counts are printed (the gain is measured, not assumed)."""
    dims, N = (4, 4, 4, 4), 2
    shifts = synth.geometric_shifts(15, 1e-5, 1e3)
    lat, geo, U = setup(dims, N, seed=3)
    net = Net(lat)
    pairs = make_pairs(lat, shifts[0], 16, seed=100)
    hist = net.train(pairs, steps=60, lr=3e-3, batch=8,
                     sigma=shifts[0] if sigma_loss else -1.0)
    assert np.mean(hist[-5:]) < 0.9 * hist[0]
    lat.set_links(synth.to_ref(dims, synth.links(dims, N, 0.25, 4)))   # held out
    src = lat.tf(64)
    src.upload(synth.to_ref(dims, synth.tf_source(dims, N, 999)))
    res = {}
    for name, nn in (("plain", None), ("learned", net)):
        psim = [lat.tf(64) for _ in shifts]
        res[name] = congrad_multi_learned(lat, nn, src, psim, shifts, 20000, 1e-20)
    print("refinement iterations plain %d learned %d (loss %.4f -> %.4f)"
          % (res["plain"][1], res["learned"][1], hist[0], hist[-1]))
    b2 = float(np.dot(src.download(), src.download()))
    assert res["plain"][2] <= 1e-20 * b2 and res["learned"][2] <= 1e-20 * b2
