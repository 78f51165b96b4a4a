"""The reference's FIRE pieces: md_CalculateIncrementsFIRE, md_CalculateDecrementsHalfStepFIRE
and md_FdotVEntire against the oracle (GPU), and the host decision md_SetFIREData /
md_FireDecide against the reference loop's rules (CPU)."""
import ctypes as C

import numpy as np
import pytest

import mdcall as mc
import oracle
import rfdem


def _fields(N, seed):
    rng = np.random.default_rng(seed)
    F = (rng.standard_normal(3 * N) * 1e-3).astype(np.float32)
    V = (rng.standard_normal(3 * N) * 1e-4).astype(np.float32)
    R = (10.0 + rng.random(3 * N) * 20.0).astype(np.float32)
    F[: 3 * 7: 3] = 0.0          # a few particles with F = 0 take the |F|^2 <= 1e-12 branch
    F[N: N + 7] = 0.0
    F[2 * N: 2 * N + 7] = 0.0
    return F, V, R


@pytest.mark.gpu
@pytest.mark.parametrize("N", [1, 1000, 70001])
def test_fire_kernels_bitexact(cuda, N):
    torch = cuda
    F, V, R = _fields(N, 0xB2000000 + N)
    dtm, dt, a = np.float32(0.0123), np.float32(0.0371), np.float32(0.25)
    dF, dV, dR = mc.dev(torch, F), mc.dev(torch, V), mc.dev(torch, R)
    rfdem.check(rfdem.lib.md_CalculateDecrementsHalfStepFIRE(dV.data_ptr(), dR.data_ptr(), N, np.float32(0.5) * dt,
                                                             None), "half")
    rfdem.check(rfdem.lib.md_CalculateIncrementsFIRE(dF.data_ptr(), dV.data_ptr(), dR.data_ptr(), N, dtm, dt, a, None),
                "inc")
    torch.cuda.synchronize()
    Ro, Vo = R.copy(), V.copy()
    L = oracle.load()
    L.rfo_fire_half_f(Vo.ctypes.data, Ro.ctypes.data, N, np.float32(0.5) * dt)
    L.rfo_fire_increments_f(F.ctypes.data, Vo.ctypes.data, Ro.ctypes.data, N, dtm, dt, a)
    assert np.array_equal(mc.host(dV, np.float32), Vo)
    assert np.array_equal(mc.host(dR, np.float32), Ro)
    nb = N // 1024 + 1
    part = torch.zeros(nb, dtype=torch.float64, device="cuda")
    rfdem.check(rfdem.lib.md_FdotVEntire(dV.data_ptr(), dF.data_ptr(), part.data_ptr(), nb, N, None), "fdotv")
    torch.cuda.synchronize()
    p_gpu = float(part.sum().item())
    p_ref = L.rfo_fdotv_f(Vo.ctypes.data, F.ctypes.data, N)
    scale = float(np.sum(np.abs(F.astype(np.float64) * Vo.astype(np.float64))))
    assert abs(p_gpu - p_ref) <= 1e-12 * max(scale, 1e-300)


def test_fire_decision_rules(rfdem):
    po = rfdem.granite_potential()
    t = rfdem.Task()
    t.Po = po
    ss = (C.c_double * 3)(0.02, 0.02, 0.03)
    ls = (C.c_double * 3)(0.01, 0.01, 0.02)
    t.N = 100
    t.K = 32
    rfdem.check(rfdem.lib.rf_task_prepare(C.byref(t), ss, ls, 2.0 * po.a_farcut, -2e-4, 0.015, 0.1), "prep")
    f = rfdem.Fire()
    rfdem.check(rfdem.lib.md_SetFIREData(C.byref(f), 5000, C.byref(t.Po)), "set")
    dt0 = np.float32(t.Po.dt)
    assert f.dt0 == dt0 and f.dt == dt0 and f.Ndelay == 20 and f.NPnegativeMax == 30000
    assert f.bloks4 == 5000 // 1024 + 1
    assert f.dtmax == np.float32(100.0 * float(dt0)) and f.dtmin == np.float32(0.001 * float(dt0))
    hs, stop = C.c_int(0), C.c_int(0)
    # Ndelay positive steps leave dt alone; the next ones grow it by 1.1 up to dtmax, alpha shrinks
    for s in range(20):
        rfdem.lib.md_FireDecide(C.byref(f), 1.0, s, C.byref(hs), C.byref(stop))
        assert hs.value == 0 and f.dt == dt0
    rfdem.lib.md_FireDecide(C.byref(f), 1.0, 20, C.byref(hs), C.byref(stop))
    assert f.dt == np.float32(dt0 * np.float32(1.1)) and f.alpha == np.float32(np.float32(0.25) * np.float32(0.99))
    # an uphill step after the delay: half step back, dt halves, alpha resets
    d = f.dt
    rfdem.lib.md_FireDecide(C.byref(f), -1.0, 21, C.byref(hs), C.byref(stop))
    assert hs.value == 1 and stop.value == 0 and f.dt == np.float32(d * np.float32(0.5)) and f.alpha == np.float32(0.25)
    assert f.NPpositive == 0 and f.NPnegative == 1
    # uphill within the first Ndelay steps: half step, dt unchanged
    f2 = rfdem.Fire()
    rfdem.lib.md_SetFIREData(C.byref(f2), 5000, C.byref(t.Po))
    rfdem.lib.md_FireDecide(C.byref(f2), 0.0, 3, C.byref(hs), C.byref(stop))
    assert hs.value == 1 and f2.dt == dt0
    # dt never drops below dtmin; NPnegativeMax uphill steps in a row stop the loop
    f2.NPnegativeMax = 50
    for s in range(100, 149):          # with the one above: 50 uphill steps in a row
        rfdem.lib.md_FireDecide(C.byref(f2), -1.0, s, C.byref(hs), C.byref(stop))
    assert f2.dt >= f2.dtmin and stop.value == 0
    rfdem.lib.md_FireDecide(C.byref(f2), -1.0, 150, C.byref(hs), C.byref(stop))
    assert stop.value == 1
