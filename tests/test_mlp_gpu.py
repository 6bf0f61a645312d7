"""GPU MLP kernels against the double-precision oracle: forward outputs,
gradients (the hand-written backward pass), deterministic training, loss
decrease, and the by-value single-sample predictor."""
import numpy as np
import pytest

from bespokeolap_artifacts_b200.learned import Mlp
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("F,O,n", [(8, 1, 64), (8, 2, 130), (32, 4, 1000), (3, 1, 1)])
def test_forward_and_gradients_match_oracle(engine, torch_cuda, F, O, n):
    torch = torch_cuda
    rng = np.random.default_rng(F * 100 + n)
    m = Mlp(engine.ctx, F, O, seed=3)
    p = m.get_params()
    x = rng.normal(0, 1, (n, F)).astype(np.float32)
    t = rng.normal(0, 1, (n, O)).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = torch.empty((n, O), dtype=torch.float32, device="cuda")
    m.infer_device(xd, n, y)
    g = torch.empty(m.P, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    m.gradients(xd, td, n, g, loss)
    engine.synchronize()
    y_ref, _ = mlp_ref.forward(p, x, F, O)
    l_ref, g_ref = mlp_ref.loss_and_grad(p, x, t, F, O)
    # FP32 kernels vs a float64 restatement of the same math
    np.testing.assert_allclose(y.cpu().numpy(), y_ref, rtol=1e-4, atol=1e-5)
    assert abs(loss.item() - l_ref) <= 1e-5 * max(1.0, abs(l_ref))
    gg = g.cpu().numpy().astype(np.float64)
    scale = np.abs(g_ref).max()
    assert np.max(np.abs(gg - g_ref)) <= 1e-4 * scale + 1e-7


def test_training_is_deterministic_and_reduces_loss(engine):
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (500, 6)).astype(np.float32)
    t = (np.sin(x[:, :1]) + 0.5 * x[:, 1:2] ** 2).astype(np.float32)
    runs = []
    for _ in range(2):
        m = Mlp(engine.ctx, 6, 1, seed=11)
        l0 = m.train(x, t, epochs=1, lr=1e-3)
        l1 = m.train(x, t, epochs=400, lr=3e-3)
        runs.append(m.get_params())
        assert l1 < 0.25 * l0
    assert np.array_equal(runs[0], runs[1])  # fixed-order reductions: bitwise reproducible


def test_predict_counts_by_value(engine, torch_cuda):
    torch = torch_cuda
    m = Mlp(engine.ctx, 8, 2, seed=2)
    p = m.get_params()
    f = np.linspace(-1, 1, 8).astype(np.float32)
    c = torch.empty(2, dtype=torch.float32, device="cuda")
    lg = torch.empty(2, dtype=torch.float32, device="cuda")
    m.predict_counts_device(f, c, lg)
    engine.synchronize()
    y_ref, _ = mlp_ref.forward(p, f[None, :], 8, 2)
    np.testing.assert_allclose(lg.cpu().numpy(), y_ref[0], rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(c.cpu().numpy(), np.maximum(np.expm1(y_ref[0]), 0), rtol=1e-3, atol=1e-4)
