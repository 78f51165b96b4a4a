"""The warm-start MLP: forward and gradients of the tensor-core kernels against the CPU
restatement (oracle/mlp_ref.py), and a training run that fits a synthetic target."""
import numpy as np
import pytest

import rfdem
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _data(torch, rows, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((rows, 64)).astype(np.float32)
    X[:, 59:] = 0.0
    X[:, 58] = 1.0
    Xb = torch.from_numpy(X).to(torch.bfloat16).cuda()
    T = (0.5 * np.tanh(X[:, :6] + 0.3 * X[:, 6:12]) + 0.1 * X[:, 12:18]).astype(np.float32)
    return Xb, torch.from_numpy(T).cuda(), Xb.float().cpu().numpy().astype(np.float64), T


@pytest.mark.parametrize("rows", [300, 4096])
def test_mlp_forward_and_gradients_vs_oracle(cuda, rows):
    torch = cuda
    m = rfdem.MLP(seed=7)
    ws = m.weights()
    rp = (rows + 127) // 128 * 128
    Xb, Td, X, T = _data(torch, rows, rows)
    Y = torch.zeros(rp, 16, device="cuda")
    m.forward(Xb, rows, Y)
    torch.cuda.synchronize()
    y_ref, _ = mlp_ref.forward(ws, X)
    y = Y[:rows].cpu().numpy()
    scale = np.abs(y_ref[:, :6]).max() + 1e-6
    assert np.max(np.abs(y[:, :6] - y_ref[:, :6])) <= 2e-2 * scale
    loss = m.train_step(Xb, Td, rows, 0.0)           # gradients only
    loss_ref, g_ref = mlp_ref.backward(ws, X, T)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    g = m.grads()
    for l in range(4):
        for a, b in zip(g[l], g_ref[l]):
            n = np.linalg.norm(b)
            if n == 0:
                assert np.linalg.norm(a) == 0
                continue
            rel = np.linalg.norm(a - b) / n
            assert rel < 2e-2, (l, rel)
    m.close()


def test_mlp_training_reduces_loss(cuda):
    torch = cuda
    m = rfdem.MLP(seed=3)
    rows = 20000
    Xb, Td, _, _ = _data(torch, rows, 1)
    first = m.train_step(Xb, Td, rows, 3e-3)
    for _ in range(300):
        last = m.train_step(Xb, Td, rows, 3e-3)
    print("loss %.4e -> %.4e" % (first, last))
    assert last < 0.1 * first
    m.close()
