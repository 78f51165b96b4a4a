"""Quasi-static FIRE load increments of the extended model on the GPU: against the
oracle's restatement of the same relaxation (float forces, and the FP64 oracle), and
the warm-start path with an exact predictor."""
import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem

pytestmark = pytest.mark.gpu


def test_fire_increments_vs_oracle(cuda):
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, min_stress=1e3)
    e = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    p = e.relax_params(max_iter=40000, strain_inc=1e-4)
    n = 5
    res = [e.load_increment(p) for _ in range(n)]
    Re = e.positions_f64()
    e.close()
    assert all(r.error == 0 for r in res)
    assert res[-1].converged == 1 and res[-1].residual <= p.tol
    of = oracle.qs_ext(mc.clone(t), x, R, rad, p, n)
    od = oracle.qs_ext(mc.clone(t), x, R, rad, p, n, fp64=True)
    assert of["converged"][-1] == 1 and od["converged"][-1] == 1
    ext = float(np.ptp(R))
    # the same relaxation in the same arithmetic up to the order of the FP64 sums
    assert np.max(np.abs(Re - of["R"])) < 1e-6 * ext
    # against the FP64 oracle: relaxed positions and the platen stress of the loaded specimen
    assert np.max(np.abs(Re - od["R"])) < 1e-5 * ext
    s_e, s_d = res[-1].stress, od["stress"][-1]
    print("stress engine %.6e  FP64 oracle %.6e  rel %.2e" % (s_e, s_d, abs(s_e - s_d) / s_d))
    assert s_d > 1e-6 and abs(s_e - s_d) <= 5e-3 * s_d, (s_e, s_d)
    it_e = np.array([r.iterations for r in res], float)
    it_o = of["iters"].astype(float)
    assert abs(it_e.sum() - it_o.sum()) <= 0.3 * it_o.sum()


def test_fire_exact_warm_start_cuts_iterations(cuda):
    """Warm start with the relaxed answer of the same increment (two engines in lockstep)."""
    import torch
    N, r0 = 4000, 0.25
    R0, rad, D, H, mo = rfdem.pack_cylinder(N, r0, aspect=2.0, phi=0.58, seed=0xB2000000 + 77)
    x = extspec.stiff_params()
    t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, r0, min_stress=1e3)
    A = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    B = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    p = A.relax_params(max_iter=60000)
    loaded = 0
    for k in range(30):                      # until the platen carries load
        a, b = A.load_increment(p), B.load_increment(p)
        assert a.iterations == b.iterations and a.stress == b.stress
        if a.stress > 1e-7 and a.converged:
            loaded += 1
        if loaded >= 2:
            break
    assert loaded >= 2
    a = A.load_increment(p)
    _, dx, rot = A.increment_fields()
    warm = torch.from_numpy(np.concatenate([dx, rot], 1).astype(np.float32)).cuda()
    b = B.load_increment(p, warm)
    print("plain %d iterations, exact warm start %d" % (a.iterations, b.iterations))
    assert a.converged == 1 and b.converged == 1
    assert b.iterations * 2 < a.iterations
    assert abs(b.stress - a.stress) <= 1e-3 * a.stress
    A.close(); B.close()


def test_mlp_warm_start_behind_its_gate(cuda):
    """The MLP warm start on a loaded specimen (three engines in lockstep until the
    evaluation): trained on plain-FIRE pairs of its own history, the gated MLP start relaxes
    every evaluated increment to the plain run's stress, in fewer iterations than plain
    FIRE; the gate lets the MLP predict an increment only after its error on the previous
    one was below the gate times the last-increment motion's error. The last-increment
    start is run beside it for reference."""
    from rfdem.warm import WarmStart
    N, r0 = 4000, 0.25
    R0, rad, D, H, mo = rfdem.pack_cylinder(N, r0, aspect=2.0, phi=0.58, seed=0xB2000000 + 78)
    x = extspec.stiff_params()
    t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, r0, min_stress=1e3)
    A, B, Cn = (rfdem.Engine(mc.clone(t), R, ext=x, radius=rad) for _ in range(3))
    p = A.relax_params(max_iter=60000)
    ws = WarmStart(N, p.strain_inc, seed=0xB2000000 + 79)
    loaded = 0
    for k in range(30):                      # until the platen carries load
        rs = [E.load_increment(p) for E in (A, B, Cn)]
        if rs[0].stress > 1e-7 and rs[0].converged:
            loaded += 1
        if loaded >= 2:
            break
    assert loaded >= 2
    for k in range(4):                       # training pairs from the plain engine
        ws.features(A)
        for E in (A, B, Cn):
            E.load_increment(p)
        ws.collect(A)
    losses = ws.train(steps=300)
    assert losses[-1] < losses[0]
    it = {"plain": 0, "mlp": 0, "last": 0}
    for k in range(5):
        a = A.load_increment(p)
        b = B.load_increment_pred(p, ws.predict(B), 16)
        ratio = ws.observe(B)
        c = Cn.load_increment_pred(p, ws.predict(Cn, use_mlp=False), 16)
        print("increment %d: iterations plain %d, MLP %d (used %d, error / last-increment error %.3f), "
              "last increment %d" % (k, a.iterations, b.iterations, ws.log[-1][1], ratio, c.iterations))
        assert a.converged == 1 and b.converged == 1 and c.converged == 1
        assert abs(b.stress - a.stress) <= 1e-3 * abs(a.stress)
        assert abs(c.stress - a.stress) <= 1e-3 * abs(a.stress)
        it["plain"] += a.iterations
        it["mlp"] += b.iterations
        it["last"] += c.iterations
    print("iterations over 5 increments:", it)
    assert it["mlp"] < it["plain"]
    for (r_prev, _), (_, used) in zip(ws.log[:-1], ws.log[1:]):
        assert used == (r_prev < ws.gate)
    ws.close()
    A.close(); B.close(); Cn.close()
