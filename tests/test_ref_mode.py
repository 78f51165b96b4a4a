"""The extended model in its reference-constants mode (rf_ext_params.ref_mode = 1)
against the reference model, on the oracle (CPU).

This is the link between the engine's headline kernel (k_step_ext: FP64 positions,
float forces, per-bond constants) and the model that the reference's own kernels pin
(k_step, tests/test_gpu_reference.py). With every radius p_r, bonds where the centre
distance is below b_d, bond radius b_r, stiffness per area E/L0 and G/L0 of each bond,
strengths m_Ec and m_Gc, the reference's extra dt*E/(4 L0) factor on the summed bending
moment (md_calculateforcesdem3.cu:131-152) and platen coordinates rounded to float as the
reference's drivers pass them, the extended model is the reference model:

* in FP64 the two formulations follow one trajectory (they differ only in where an
  expression is rounded: 1e-9 mm after thousands of steps);
* with the engine's arithmetic (float forces, FP64 positions) the extended model stays
  far closer to that FP64 trajectory than the reference's own FP32 path does.

The GPU side (k_step_ext in this mode bit for bit against this oracle, and against the
reference's kernels) is tests/test_gpu_ref_mode.py."""
import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem

# (kind, diameter, height, seed, steps). The uniaxial window runs into damage (about 100
# bonds broken, contacts formed, rows changed). The Brazilian disc's platens carry
# friction that switches on the tangential speed of a particle (|v|^2 > 1e-9,
# md_braziltest_simple2.cu:49-60): two runs that differ by 1e-12 mm switch it on
# different steps and part within ~800 steps, so its window stops before that.
CASES = [(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, 55, 6000), (rfdem.RF_TEST_BRAZIL, 16.0, 6.0, 52, 600)]
IDS = ["uniaxial-585", "brazil-885"]


def _windows(kind, d, h, seed, steps):
    t, Rf, R64, rad, x = extspec.ref_mode_case(kind, d, h, 0xB2000000 + seed, max_strain=1.0)
    td = mc.clone(t)
    nd, Rd, curve_d, tyd, sd = oracle.run_d(td, Rf, steps)
    te = mc.clone(t)
    o64 = oracle.run_ext(te, x, R64, rad, steps, fp64=True)
    tf = mc.clone(t)
    o = oracle.run_ext(tf, x, R64, rad, steps)
    tr = mc.clone(t)
    nr, st, curve_r, sr = oracle.run_f(tr, Rf, steps)
    return dict(t=t, rad=rad, R64=R64, d=(td, Rd, curve_d, tyd, nd), e64=(te, o64), e=(tf, o),
                r=(tr, st, curve_r, nr))


@pytest.mark.parametrize("kind,d,h,seed,steps", CASES, ids=IDS)
def test_fp64_formulations_follow_one_trajectory(oracle, kind, d, h, seed, steps):
    """The FP64 extended model with the reference constants against the reference
    model's FP64 oracle over a window of loading: positions within 1e-6 mm, the same bond
    flags, and the load curve
    within 1e-5 relative (a platen particle's reaction is its bonds' stiffness, ~17 in
    model units, times a position difference of ~1e-12 mm, against reactions of ~1e-4)."""
    w = _windows(kind, d, h, seed, steps)
    t = w["t"]
    N, K = int(t.N), int(t.K)
    td, Rd, curve_d, tyd, nd = w["d"]
    te, o64 = w["e64"]
    assert nd == o64["steps"] == steps
    err = np.abs(o64["R"] - Rd).max()
    print("max |R_ext64 - R_ref64| = %.3e mm after %d steps; stress %.6e vs %.6e" %
          (err, steps, te.Compress.Stress, td.Compress.Stress))
    assert err < 1e-6
    np.testing.assert_allclose(o64["curve"], curve_d, rtol=1e-5, atol=1e-9 * np.abs(curve_d).max())
    assert np.array_equal(o64["ILtype"], tyd)
    # the window exercised contacts and list changes, not only intact bonds
    start = oracle.run_ext(mc.clone(t), extspec.ref_params(), w["R64"], w["rad"], 0, fp64=True)
    changed = int((start["IL"] != o64["IL"]).sum())
    bonds, contacts = extspec.pair_counts(o64["R"], N, K, o64["IL"], o64["ILtype"], w["rad"])
    print("bond slots %d, overlapping contact slots %d, row slots changed %d, bonds broken %d" %
          (bonds, contacts, changed, o64["broken"]))
    assert changed > 0 and td.Compress.Stress > 0.0
    if kind == rfdem.RF_TEST_UNIAXIAL:
        assert contacts > 0 and o64["broken"] > 0


@pytest.mark.parametrize("kind,d,h,seed,steps", CASES, ids=IDS)
def test_float_forces_track_fp64_closer_than_reference_fp32(oracle, kind, d, h, seed, steps):
    """The engine's arithmetic in this mode (float forces, FP64 positions) against the
    FP64 trajectory, beside the reference's own FP32 path (positions in float: increments
    of ~1e-5 mm on coordinates of ~20 mm lose most of their bits) against the same one."""
    w = _windows(kind, d, h, seed, steps)
    td, Rd, curve_d, tyd, nd = w["d"]
    tf, o = w["e"]
    tr, st, curve_r, nr = w["r"]
    assert o["steps"] == nr == nd == steps
    e_ext = np.abs(o["R"] - Rd)
    e_ref = np.abs(st["R"].astype(np.float64) - Rd)
    print("|R - R_ref64| mm: extended (float forces, FP64 positions) max %.3e p99 %.3e; "
          "reference FP32 max %.3e p99 %.3e" % (e_ext.max(), np.percentile(e_ext, 99), e_ref.max(),
                                                np.percentile(e_ref, 99)))
    assert e_ext.max() <= 0.1 * e_ref.max()
    assert np.percentile(e_ext, 99) <= 0.1 * np.percentile(e_ref, 99)
    s_d = td.Compress.Stress
    print("stress: FP64 %.6e, extended %.6e (rel %.2e), reference FP32 %.6e (rel %.2e)" %
          (s_d, tf.Compress.Stress, tf.Compress.Stress / s_d - 1, tr.Compress.Stress, tr.Compress.Stress / s_d - 1))
    assert abs(tf.Compress.Stress / s_d - 1) <= 1e-4


def test_reference_mode_needs_monosized_radii(rfdem):
    t, Rf, R64, rad, x = extspec.ref_mode_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 8.0, 0xB2000000 + 3)
    rad = rad.copy()
    rad[3] *= 1.01
    import ctypes as C
    h = rfdem.P()
    st = rfdem.lib.rf_engine_create_ext(C.byref(mc.clone(t)), C.byref(x), R64.ctypes.data, rad.ctypes.data, C.byref(h))
    assert st == rfdem.RF_ERR_INVALID
    assert b"ref_mode" in rfdem.lib.rf_last_error_string()
