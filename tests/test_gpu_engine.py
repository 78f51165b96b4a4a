"""The fused engine against the oracle: whole explicit runs, bit for bit.

The engine keeps its own layout (slot-major rows, Verlet candidate lists, one fused
kernel per step); after export its state must equal the oracle's reference-layout
state exactly, step count for step count."""
import os

import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem

pytestmark = pytest.mark.gpu

KEYS = ["R", "V", "W", "IL", "ILtype", "iL", "Rij", "Oijt", "Mijn", "Mijt"]


def assert_state_equal(e, o, keys=KEYS):
    for k in keys:
        a, b = e[k], o[k]
        if k == "IL":
            b = b.astype(a.dtype)
        same = np.array_equal(a.view(np.uint8), np.ascontiguousarray(b).view(np.uint8))
        if not same:
            bad = np.nonzero(a != b)[0]
            raise AssertionError("%s differs at %d places, first %s: %s vs %s" % (k, bad.size, bad[:5], a[bad[:5]],
                                                                                 b[bad[:5]]))


# (kind, diameter, height, steps, platen speed factor, window must show damage). The two
# damage windows break bonds, load contacts and change rows (asserted); the uniaxial one
# drives its platen at 5x the reference's speed so that damage starts within 3000 steps.
# The 10k-particle case checks the multi-CTA paths at a larger size over a short window.
CASES = [(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, 3000, 5.0, True), (rfdem.RF_TEST_BRAZIL, 16.0, 6.0, 3000, 1.0, True),
         (rfdem.RF_TEST_UNIAXIAL, 20.0, 30.0, 60, 1.0, False)]


@pytest.mark.parametrize("kind,d,h,steps,vf,damage", CASES, ids=["uniaxial", "brazil", "uniaxial-10k"])
def test_engine_run_bitexact_vs_oracle(cuda, kind, d, h, steps, vf, damage):
    v = (-10.0 if kind == rfdem.RF_TEST_UNIAXIAL else -100.0) * 0.02 / 1e3 * vf
    t, R = rfdem.make_test(kind, d, h, seed=0xB2000000 + 21, v_load=v, max_strain=1.0)
    to = mc.clone(t)
    n, ost, curve_o, status = oracle.run_f(to, R, steps)
    assert status == 0
    e = rfdem.Engine(t, R)
    e.step(steps)
    te, res = e.sync()
    assert res.error == 0
    assert res.steps == n
    assert_state_equal(e.export(), ost)
    # scalar test state: FP64 sums in a different order -> last-bit differences only
    assert te.Compress.Loading == to.Compress.Loading and te.Compress.Fracture == to.Compress.Fracture
    np.testing.assert_allclose(te.Compress.Stress, to.Compress.Stress, rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(te.Compress.FractureStress, to.Compress.FractureStress, rtol=1e-9, atol=1e-15)
    assert te.Compress.Strain == to.Compress.Strain
    ce = e.curve()
    np.testing.assert_allclose(ce, curve_o, rtol=1e-9, atol=1e-12)
    c = e.counters()
    assert c["bonds"] > 2 * t.N and c["steps"] == n
    e.close()
    if damage:
        N, K = int(t.N), int(t.K)
        _, st0, _, _ = oracle.run_f(mc.clone(t), R, 0)
        _, contacts = extspec.pair_counts(ost["R"], N, K, ost["IL"], ost["ILtype"], np.full(N, t.Po.p_r))
        broken, changed = int(ost["broke"].sum()), int((ost["IL"] != st0["IL"]).sum())
        print("%d steps: bonds broken %d, overlapping contact slots %d, row slots changed %d" %
              (steps, broken, contacts, changed))
        assert res.broken_bonds == broken > 0 and contacts > 0 and changed > 0


def test_graph_and_stream_paths_agree(cuda):
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=5)
    a = rfdem.Engine(mc.clone(t), R)
    os.environ["RF_ENGINE_NO_GRAPH"] = "1"
    try:
        b = rfdem.Engine(mc.clone(t), R)
    finally:
        del os.environ["RF_ENGINE_NO_GRAPH"]
    for chunk in (1, 7, 50, 142):
        a.step(chunk)
        b.step(chunk)
    assert_state_equal(a.export(), b.export())
    assert a.counters()["steps"] == b.counters()["steps"] == 200
    a.close(); b.close()


def test_resume_from_export_is_bitexact(cuda):
    t, R = rfdem.make_test(rfdem.RF_TEST_BRAZIL, 14.0, 6.0, seed=8)
    a = rfdem.Engine(mc.clone(t), R)
    a.step(300)
    ref = a.export()
    b = rfdem.Engine(mc.clone(t), R)
    b.step(150)
    mid_task, _ = b.sync()
    snap = b.export()
    c = rfdem.Engine(mid_task, R)          # fresh engine carrying the mid-run scalar state
    c.load(snap)
    c.step(150)
    assert_state_equal(c.export(), ref)
    a.close(); b.close(); c.close()


def test_driver_api_matches_oracle(cuda):
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=12)
    to = mc.clone(t)
    n, ost, curve_o, _ = oracle.run_f(to, R, 250)
    res, curve, Rout = rfdem.run_test(t, R, max_steps=250, curve_cap=250, want_positions=True)
    assert res.steps == n == 250
    assert np.array_equal(Rout, ost["R"])
    np.testing.assert_allclose(curve, curve_o, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(t.Compress.FractureStress, to.Compress.FractureStress, rtol=1e-9)


def test_host_buffer_step_roundtrip(cuda):
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=13)
    a = rfdem.Engine(mc.clone(t), R)
    b = rfdem.Engine(mc.clone(t), R)
    out = np.zeros_like(R)
    cur = R.copy()
    for _ in range(4):
        b.step_host(cur, 25, out)      # re-upload the state it just returned: a no-op for the physics
        cur = out.copy()
    a.step(100)
    assert_state_equal(a.export(), b.export())
    a.close(); b.close()


def test_fracture_stops_on_device(cuda):
    """A weak specimen breaks; the device loop stops at the reference's fracture test and
    further step requests do nothing."""
    po = rfdem.granite_potential()
    po.m_Ec *= 0.05
    po.m_Gc *= 0.05
    t, R = rfdem.make_test(rfdem.RF_TEST_BRAZIL, 12.0, 4.0, seed=3, potential=po, min_stress=2e-5)
    e = rfdem.Engine(t, R)
    e.step(60000)
    te, res = e.sync()
    if not res.Fracture:
        pytest.skip("specimen did not fracture within the step budget")
    s0 = res.steps
    e.step(100)
    _, res2 = e.sync()
    assert res2.steps == s0
    assert res.broken_bonds > 0
    e.close()


def test_checkpoint_file_resume_is_bitexact(cuda, tmp_path):
    """rf_engine_checkpoint mid-run, rf_engine_restore in a fresh engine: the restored run
    continues the uninterrupted one bit for bit; the file's payload is the reference's
    SaveAllData layout, which rf_load_all_data reads back."""
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=21)
    a = rfdem.Engine(mc.clone(t), R)
    a.step(260)
    ref = a.export()
    b = rfdem.Engine(mc.clone(t), R)
    b.step(130)
    path = tmp_path / "mid.ckpt"
    b.checkpoint(str(path))
    mid = b.export()
    c = rfdem.Engine.restore(str(path))
    assert_state_equal(c.export(), mid)
    c.step(130)
    assert_state_equal(c.export(), ref)
    a.close(); b.close(); c.close()
