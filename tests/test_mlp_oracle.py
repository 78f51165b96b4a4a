"""The MLP restatement itself (CPU): BF16 rounding and the backward pass against
finite differences of the loss (roundings off)."""
import numpy as np

from oracle import mlp_ref


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.0078125, 1.001953125, 1.005859375, -3.3, 0.0], np.float32)
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125      # ties to even
    assert r[3] == 1.0 and r[4] == 1.0078125
    assert abs(r[5] + 3.3) < 0.02 and r[6] == 0.0


def test_backward_matches_finite_differences():
    mlp_ref.ROUND = False
    try:
        rng = np.random.default_rng(0)
        ws = []
        for din, dout in zip((64, 128, 128, 128), (128, 128, 128, 16)):
            W = (rng.standard_normal((dout, din)) * np.sqrt(2.0 / din)).astype(np.float64)
            if dout == 16:
                W[6:] = 0
            ws.append((W, rng.standard_normal(dout) * 0.1))
        X = rng.standard_normal((40, 64))
        T = rng.standard_normal((40, 6))
        loss, g = mlp_ref.backward(ws, X, T)
        eps = 1e-6
        for l, (i, o) in [(0, (3, 5)), (1, (7, 2)), (2, (11, 100)), (3, (17, 4))]:
            W, b = ws[l]
            W2 = W.copy()
            W2[o, i] += eps
            ws2 = list(ws)
            ws2[l] = (W2, b)
            l2, _ = mlp_ref.backward(ws2, X, T)
            fd = (l2 - loss) / eps
            assert abs(fd - g[l][0][i, o]) <= 1e-4 * max(1.0, abs(fd)), (l, fd, g[l][0][i, o])
            b2 = b.copy()
            b2[o] += eps
            ws2[l] = (W, b2)
            l3, _ = mlp_ref.backward(ws2, X, T)
            fdb = (l3 - loss) / eps
            assert abs(fdb - g[l][1][o]) <= 1e-4 * max(1.0, abs(fdb))
    finally:
        mlp_ref.ROUND = True
