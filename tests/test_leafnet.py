"""The turn-leaf value network: the tcgen05 matrix product, forward pass,
gradients and training against the CPU restatement in oracle/leafnet.py.

Tolerances: the products take bf16 inputs and accumulate in f32 on the
tensor cores, the oracle accumulates the same bf16 values in f64 -- a
product must agree within 1e-5 of sum |a||b| per entry.  Through the net a
hidden activation whose f32 value sits on a bf16 rounding boundary may round
the other way (one bf16 step, 2^-8 relative); outputs and gradients are held
to 1e-2 of their largest magnitude, the loss to 1e-4 relative."""
import numpy as np
import pytest

from oracle import leafnet as O

RNG = np.random.default_rng(7)


def _params(net):
    return [net.params(l) for l in range(net.nhidden + 1)]


def test_oracle_gradients_match_finite_differences():
    """The oracle's backward formulas (f64, no rounding) against central
    differences of its loss."""
    rng = np.random.default_rng(3)
    shapes = [(7, 5), (7, 7), (4, 7)]
    params = [(rng.normal(0, 0.5, s), rng.normal(0, 0.1, s[0])) for s in shapes]
    x = rng.normal(0, 1, (6, 5))
    t = rng.normal(0, 1, (6, 4))
    m = (rng.random((6, 4)) > 0.3).astype(np.float64)
    _, grads = O.gradients_f64(params, x, t, m)
    eps = 1e-6
    for l, (w, b) in enumerate(params):
        for arr, g in ((w, grads[l][0]), (b, grads[l][1])):
            it = np.nditer(arr, flags=["multi_index"])
            for _ in it:
                i = it.multi_index
                old = arr[i]
                arr[i] = old + eps
                lp, _ = O.gradients_f64(params, x, t, m)
                arr[i] = old - eps
                lm, _ = O.gradients_f64(params, x, t, m)
                arr[i] = old
                assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-6 * max(1.0, abs(g[i])), (l, i)


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-30], np.float32)
    r = O.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert np.array_equal(O.from_bf16_bits(O.bf16_bits(x)), r)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 384, 576), (384, 256, 2816), (1024, 1024, 1024)])
def test_gemm_matches_f64(m, n, k):
    import gtopen_b200 as g

    a = O.bf16_round(RNG.normal(0, 1, (m, k)).astype(np.float32))
    b = O.bf16_round(RNG.normal(0, 1, (n, k)).astype(np.float32))
    c = g.gemm_bf16(O.bf16_bits(a), O.bf16_bits(b))
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    bound = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    assert np.all(np.abs(c - ref) <= 1e-5 * bound + 1e-6)


@pytest.mark.gpu
def test_gemm_refuses_unpadded_shapes():
    import gtopen_b200 as g

    with pytest.raises(g.GtobError):
        g.gemm_bf16(np.zeros((100, 64), np.uint16), np.zeros((128, 64), np.uint16))


def _small_net(seed=5):
    import gtopen_b200 as g

    return g.LeafNet(200, 256, 3, 150, seed=seed)


@pytest.mark.gpu
def test_forward_matches_oracle():
    net = _small_net()
    x = RNG.normal(0, 1, (300, 200)).astype(np.float32)
    y = net.forward(x)
    ref = O.forward(_params(net), x)
    assert y.shape == ref.shape
    assert np.max(np.abs(y - ref)) <= 1e-2 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_gradients_match_oracle():
    net = _small_net(9)
    x = RNG.normal(0, 1, (260, 200)).astype(np.float32)
    t = RNG.normal(0, 1, (260, 150)).astype(np.float32)
    m = (RNG.random((260, 150)) > 0.25).astype(np.float32)
    loss = net.gradients(x, t, m)
    ref_loss, ref = O.gradients(_params(net), x, t, m)
    assert abs(loss - ref_loss) <= 1e-4 * ref_loss
    for l in range(net.nhidden + 1):
        gw, gb = net.grads(l)
        rw, rb = ref[l]
        assert np.max(np.abs(gw - rw)) <= 1e-2 * np.max(np.abs(rw)), l
        assert np.max(np.abs(gb - rb)) <= 1e-2 * np.max(np.abs(rb)), l


@pytest.mark.gpu
def test_training_fits_a_teacher():
    """Adam on the device: a 3-layer student learns a random teacher's map."""
    import gtopen_b200 as g

    teacher = g.LeafNet(64, 128, 2, 32, seed=11)
    x = RNG.normal(0, 1, (4096, 64)).astype(np.float32)
    t = teacher.forward(x) * 10.0
    m = np.ones_like(t)
    student = g.LeafNet(64, 128, 3, 32, seed=12)
    losses = student.train(x, t, m, epochs=40, batch=512, lr=2e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.25 * losses[0], losses
    assert np.all(np.diff(losses[5:]) < 0), losses  # still descending at the end
