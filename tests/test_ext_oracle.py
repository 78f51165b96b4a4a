"""The extended model's oracle on the CPU: the float-force instance (the engine's
arithmetic) against the FP64 instance, bond formation and the strength draws."""
import ctypes as C

import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem


@pytest.mark.parametrize("kind,d,h", [(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0), (rfdem.RF_TEST_BRAZIL, 10.0, 4.0)],
                         ids=["uniaxial", "brazil"])
def test_ext_float_vs_fp64(kind, d, h):
    t, R, rad, x = extspec.ext_case(kind, d, h, min_stress=1e3)    # no fracture stop in this window
    N, K = int(t.N), int(t.K)
    steps = 150
    f = oracle.run_ext(mc.clone(t), x, R, rad, steps)
    g = oracle.run_ext(mc.clone(t), x, R, rad, steps, fp64=True)
    assert f["steps"] == steps and g["steps"] == steps
    assert f["status"] == 0 and g["status"] == 0
    bonds = int(np.count_nonzero(f["ILtype"]))
    assert bonds > 3 * N, "lattice neighbours within 0.05 r_min should bond (%d bonds, %d particles)" % (bonds, N)
    # FP32 forces with FP64 positions track the FP64 oracle closely over a short run
    ext = float(np.max(R) - np.min(R))
    err = np.max(np.abs(f["R"] - g["R"]))
    assert err < 1e-6 * ext, err
    # both instances keep the same lists and bond states here (no threshold bonds)
    assert np.array_equal(f["IL"], g["IL"])
    assert np.array_equal(f["ILtype"], g["ILtype"])


def test_ext_bond_rule_and_rest_length():
    """Step 0 bonds exactly the listed pairs whose gap is below gap_frac * min radius."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 5.0, 6.0)
    N, K = int(t.N), int(t.K)
    f = oracle.run_ext(mc.clone(t), x, R, rad, 0)
    IL = f["IL"].reshape(N, K)
    ty = f["ILtype"].reshape(N, K)
    P = R.reshape(3, N).T
    E = np.iinfo(np.uint64).max
    for i in range(N):
        for k in range(K):
            j = IL[i, k]
            if j == E:
                assert ty[i, k] == 0
                continue
            L = np.sqrt(np.sum((P[j] - P[i]) ** 2))
            want = (L - rad[i] - rad[j]) < x.gap_frac * min(rad[i], rad[j])
            assert bool(ty[i, k]) == want, (i, k, j)


def test_ext_directed_bonds_pair_up():
    """Both directions of a pair are bonded together (the rule is symmetric)."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_BRAZIL, 8.0, 3.0)
    N, K = int(t.N), int(t.K)
    f = oracle.run_ext(mc.clone(t), x, R, rad, 0)
    IL = f["IL"].reshape(N, K)
    ty = f["ILtype"].reshape(N, K)
    pairs = {(i, int(IL[i, k])) for i in range(N) for k in range(K) if ty[i, k]}
    assert pairs and all((j, i) in pairs for (i, j) in pairs)


def _qs_total(on):
    L = oracle.load()
    L.rfo_set_qs_total.argtypes = [C.c_int]
    L.rfo_set_qs_total(on)


def test_exact_warm_start_lands_on_the_relaxed_state():
    """Warm-starting a FIRE increment with its own relaxed answer (displacements and
    rotations), FP64 oracle. With the bond state computed from the increment's start
    state and the motion since then (the engine's FIRE mode) the jump lands on the relaxed
    state: the first pass's residual is within a few times the tolerance and the warm run
    converges in a small fraction of the iterations, to the same stress. With the state
    integrated iteration by iteration instead (the explicit steps' rule) the shear forces
    and moments depend on the relaxation's path: the jump starts far above the tolerance
    and saves only part of the iterations."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, min_stress=1e3)
    p = rfdem.RelaxParams()
    rfdem.lib.rf_relax_default_params(C.byref(p), C.byref(t))
    p.max_iter, p.strain_inc = 40000, 1e-4
    try:
        out = {}
        for total in (1, 0):
            _qs_total(total)
            one = oracle.warm_probe(mc.clone(t), x, R, rad, p, 4, 1)
            full = oracle.warm_probe(mc.clone(t), x, R, rad, p, 4, 40000)
            out[total] = (one, full)
    finally:
        _qs_total(1)
    one, full = out[1]
    assert one["res_plain"] <= p.tol
    assert one["res_warm"] < 20 * p.tol
    assert full["stress_plain"] > 1e-5                              # the platen carries load
    assert full["conv_warm"] == 1 and full["it_warm"] * 10 < full["it_plain"]
    assert abs(full["stress_warm"] - full["stress_plain"]) <= 1e-5 * abs(full["stress_plain"])
    one0, full0 = out[0]
    assert one0["res_warm"] > 50 * one["res_warm"]
    assert 0 < one0["dMijt"] < 1e-3 * one0["maxMijt"]
    assert full0["conv_warm"] == 1 and full0["it_warm"] > 3 * full["it_warm"]


def test_post_peak_drop_stop_rule():
    """post_peak_drop = d stops a run at the first step, once loading has begun, whose
    stress is below (1 - d) times the peak so far; up to there the run is the plain one."""
    po = rfdem.granite_potential()
    R0, rad = extspec.lattice_ext(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, seed=0xB2000000 + 100)
    t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, 0.5, v_load=-2e-4, min_stress=4e-4)
    x = extspec.stiff_params(sigma_c=po.m_Ec * 0.1, tau_c=po.m_Gc * 0.1)
    x.post_peak_drop = 0.5
    o = oracle.run_ext(mc.clone(t), x, R, rad, 10 ** 5)
    S = o["steps"]
    assert o["status"] == 0 and 100 < S < 5000
    c = o["curve"]
    s = 0.5 * (np.abs(c[:, 1]) + np.abs(c[:, 2]))
    assert s.shape[0] == S
    loading = np.flatnonzero(s > t.Compress.MinStress)
    assert loading.size and loading[0] < S - 1
    peak = np.maximum.accumulate(s)
    assert s[-1] < 0.5 * peak[-1]
    assert np.all(s[loading[0]:S - 1] >= 0.5 * peak[loading[0]:S - 1])
    x.post_peak_drop = 0.0
    p = oracle.run_ext(mc.clone(t), x, R, rad, S)
    assert p["steps"] == S and np.array_equal(p["R"], o["R"])
    q = oracle.run_ext(mc.clone(t), x, R, rad, S + 50)
    assert q["steps"] == S + 50                        # without the rule the run goes on


@pytest.mark.parametrize("gap", [0.1, 0.25])
def test_list_gap_rows_hold_exactly_the_pairs_within_their_cutoff(gap):
    """With a list gap g the initial rows hold exactly the pairs within
    min(a_farcut, r_i + r_j + g) (FP64 distances); the rows are shorter than under the
    reference's uniform a_farcut, the bonds are the same, and the float-force oracle still
    tracks the FP64 one."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 5.0, 6.0, min_stress=1e3)
    N, K = int(t.N), int(t.K)
    u = oracle.run_ext(mc.clone(t), x, R, rad, 0)
    x.list_gap = gap * 0.5
    f = oracle.run_ext(mc.clone(t), x, R, rad, 0)
    assert f["status"] == 0
    E = np.iinfo(np.uint64).max
    IL = f["IL"].reshape(N, K)
    P = R.reshape(3, N).T
    a_far = float(t.Po.a_farcut)
    for i in range(N):
        d = np.sqrt(((P - P[i]) ** 2).sum(axis=1))
        cut = np.minimum(a_far, rad[i] + rad + x.list_gap)
        want = set(np.flatnonzero((d ** 2 < cut ** 2) & (np.arange(N) != i)).tolist())
        got = set(int(j) for j in IL[i] if j != E)
        assert got == want, i
    assert (f["IL"] != E).sum() < (u["IL"] != E).sum()
    assert int(np.count_nonzero(f["ILtype"])) == int(np.count_nonzero(u["ILtype"]))
    steps = 150
    a = oracle.run_ext(mc.clone(t), x, R, rad, steps)
    b = oracle.run_ext(mc.clone(t), x, R, rad, steps, fp64=True)
    assert a["status"] == 0 and b["status"] == 0
    assert np.max(np.abs(a["R"] - b["R"])) < 1e-6 * float(np.max(R) - np.min(R))


def test_position_precision_fp64_vs_hilo_vs_fp32():
    """Float forces with positions as FP64, as hi/lo float pairs, or as plain floats,
    each against the FP64 oracle: FP64 and hi/lo positions both track it to the float
    forces' own error, while float positions lose the small increments (the platen
    stress then drifts by tens of percent)."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, min_stress=1e3)
    steps = 1000
    g = oracle.run_ext(mc.clone(t), x, R, rad, steps, fp64=True)
    err, stress = {}, {}
    for mode in ("f64", "hilo", "f32"):
        f = oracle.run_ext(mc.clone(t), x, R, rad, steps, positions=mode)
        assert f["steps"] == steps and f["status"] == 0
        err[mode] = float(np.max(np.abs(f["R"] - g["R"])))
        stress[mode] = abs(f["curve"][-1, 1] / g["curve"][-1, 1] - 1.0)
    ext = float(np.max(R) - np.min(R))
    assert err["f64"] < 1e-8 * ext and err["hilo"] < 1e-8 * ext
    assert stress["f64"] < 1e-5 and stress["hilo"] < 1e-5
    assert err["f32"] > 1e4 * max(err["f64"], err["hilo"])
    assert stress["f32"] > 0.05


def test_inexact_warm_starts_reach_the_plain_relaxed_state():
    """Float forces (the engine's arithmetic): a warm start with the exact answer lands in a
    few passes; one off by 20 % (over- or under-predicted, or with 20 % per-particle
    noise) still converges, to the plain run's platen stress -- particles the platens held
    stay on them, so the prediction cannot lift the specimen off a platen."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, min_stress=1e3)
    p = rfdem.RelaxParams()
    rfdem.lib.rf_relax_default_params(C.byref(p), C.byref(t))
    p.max_iter, p.strain_inc = 40000, 1e-4
    exact = oracle.warm_probe(mc.clone(t), x, R, rad, p, 4, 40000, fp64=False)
    assert exact["conv_warm"] == 1 and exact["it_warm"] * 20 < exact["it_plain"]
    for scale, noise in ((1.2, 0.0), (0.8, 0.0), (1.0, 0.2)):
        o = oracle.warm_probe(mc.clone(t), x, R, rad, p, 4, 40000, fp64=False, scale=scale, noise=noise)
        assert o["conv_warm"] == 1 and o["it_warm"] < o["it_plain"], (scale, noise)
        assert abs(o["stress_warm"] / o["stress_plain"] - 1.0) < 1e-4, (scale, noise)


def test_brazil_fire_increments_and_exact_warm_start():
    """The quasi-static path on a Brazilian disc (platens along y): float-force FIRE
    converges every increment with the stress rising, and an exact warm start lands in a
    few passes on the same stress."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_BRAZIL, 8.0, 3.0, min_stress=1e3)
    p = rfdem.RelaxParams()
    rfdem.lib.rf_relax_default_params(C.byref(p), C.byref(t))
    p.max_iter, p.strain_inc = 20000, 1e-4
    o = oracle.qs_ext(mc.clone(t), x, R, rad, p, 5)
    assert o["status"] == 0 and np.all(o["converged"] == 1)
    assert np.all(np.diff(o["stress"]) > 0) and o["stress"][0] > 0
    w = oracle.warm_probe(mc.clone(t), x, R, rad, p, 3, 20000, fp64=False)
    assert w["conv_warm"] == 1 and w["it_warm"] * 10 < w["it_plain"]
    assert abs(w["stress_warm"] / w["stress_plain"] - 1.0) < 1e-5


def test_intact_bonds_outlive_the_list_cutoff(oracle):
    """With a list gap (pairs listed within r_i + r_j + g) a bond stretched past that
    cutoff but not past 1.45 times its rest length stays until its strength breaks it:
    after a 20 % lateral pre-strain every bond lost in the window is a strength break."""
    r0 = 0.25
    R0, rad = extspec.lattice_ext(0, 24 * r0, 40 * r0, r0=r0, seed=0xB2000000 + 77, rlo=0.9, jitter=0.02)
    t, R = rfdem.make_test_ext(0, R0, rad, r0, dt=0.01, v_load=-0.1 * 40 * r0 * 1e-6, max_strain=1.0,
                               min_stress=1e30)     # a fixed window: the fracture stop out of reach
    x = rfdem.ext_params_si()
    x.list_gap = 0.25 * r0
    N, K = int(t.N), int(t.K)
    b0, _ = extspec.pair_counts(R, N, K, oracle.run_ext(mc.clone(t), x, R, rad, 0)["IL"],
                                oracle.run_ext(mc.clone(t), x, R, rad, 0)["ILtype"], rad)
    o = oracle.run_ext(mc.clone(t), x, R, rad, 200, strain=(0.2, 0.2, -0.03))
    b1, contacts = extspec.pair_counts(o["R"], N, K, o["IL"], o["ILtype"], rad)
    print("bond slots %d -> %d, broken by strength %d, overlapping contacts %d" % (b0, b1, o["broken"], contacts))
    assert o["broken"] > 0 and contacts > 0
    assert b0 - b1 == o["broken"]
