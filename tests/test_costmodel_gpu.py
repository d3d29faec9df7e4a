"""The learned cost model's network on the GPU (bohrium_b200/csrc/ve_cuda/mlp.cu) against the
float64 CPU restatement in oracle/costmodel.py: forward values, gradients, training."""
import numpy as np
import pytest

from oracle import costmodel as O

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, O.F)).astype(np.float32)
    w = rng.standard_normal(O.F)
    t = (np.tanh(X @ w / 4.0) + 0.1 * np.sin(3 * X[:, 0])).astype(np.float32)
    return X, t


def test_forward_matches_oracle():
    from bohrium_b200.costmodel import Network
    net = Network(seed=3)
    X, _ = _data(777, 1)
    y = net.predict(X)
    want = O.forward(net.params, X)
    np.testing.assert_allclose(y, want, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("rows", [1, 127, 128, 300, 1000])
def test_gradient_matches_oracle(rows):
    """Hand-written backward kernel vs the float64 gradient (fp32 accumulation: 1e-5 of the norm)."""
    from bohrium_b200.costmodel import Network
    net = Network(seed=5)
    X, t = _data(rows, 2)
    loss, g = net.gradient(X, t)
    want_loss, want = O.loss_and_grad(net.params, X, t)
    assert abs(loss - want_loss) <= 1e-5 * max(want_loss, 1e-3)
    err = np.linalg.norm(g - want) / max(np.linalg.norm(want), 1e-12)
    assert err < 1e-5, err
    # every parameter block carries gradient
    for lo, hi in [(O.OFF_W1, O.OFF_B1), (O.OFF_W2, O.OFF_B2), (O.OFF_W3, O.OFF_B3)]:
        assert np.abs(want[lo:hi]).max() > 0


def test_training_fits_and_is_deterministic():
    from bohrium_b200.costmodel import Network
    X, t = _data(4000, 3)
    a, b = Network(seed=9), Network(seed=9)
    l0, _ = a.gradient(X, t)
    la = a.train(X, t, epochs=40, batch=256, lr=2e-3, seed=1)
    lb = b.train(X, t, epochs=40, batch=256, lr=2e-3, seed=1)
    assert la < 0.1 * l0, (l0, la)
    assert la == lb
    assert np.array_equal(a.params, b.params)
    # the reported loss is the oracle's loss of the trained parameters
    want, _ = O.loss_and_grad(a.params, X, t)
    assert abs(la - want) <= 1e-4 * max(want, 1e-3)


def test_model_file_round_trip(tmp_path):
    from bohrium_b200.costmodel import CostModel
    rng = np.random.default_rng(4)
    F = rng.random((500, O.F)) * 10
    times = np.exp(F[:, 0] * 0.3 + F[:, 2] * 0.1) + 1.0
    m = CostModel(seed=2)
    m.fit(F, times, epochs=30)
    path = str(tmp_path / "cm.bin")
    m.save(path)
    m2 = CostModel.load(path)
    np.testing.assert_array_equal(m.predict_us(F[:50]), m2.predict_us(F[:50]))
    # predictions track the targets (log-space correlation)
    p = m.predict_us(F)
    assert np.corrcoef(np.log(p), np.log(times))[0, 1] > 0.9
