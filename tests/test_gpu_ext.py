"""Extended model on the GPU: the packer, and the engine's extended-model step
against the oracle's float-force restatement (bit for bit) and the FP64 oracle."""
import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem

pytestmark = pytest.mark.gpu


def run_engine_ext(t, x, R, rad, steps, no_graph=False, monkeypatch=None):
    if no_graph:
        monkeypatch.setenv("RF_ENGINE_NO_GRAPH", "1")
    e = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    assert e.uses_graph() == (not no_graph)
    e.step(steps)
    _, res = e.sync()
    st = e.export()
    st["R64"] = e.positions_f64()
    e.close()
    return res, st


def assert_damage(t, x, R, rad, o, res):
    """The window broke bonds, loaded contacts and changed rows (so the break, contact
    and list paths were compared, not only intact bonds)."""
    N, K = int(t.N), int(t.K)
    start = oracle.run_ext(mc.clone(t), x, R, rad, 0)
    _, contacts = extspec.pair_counts(o["R"], N, K, o["IL"], o["ILtype"], rad)
    changed = int((start["IL"] != o["IL"]).sum())
    print("bonds broken %d, overlapping contact slots %d, row slots changed %d" % (o["broken"], contacts, changed))
    assert res.broken_bonds == o["broken"] > 0 and contacts > 0 and changed > 0


# The uniaxial window drives its platen at 5x the reference's speed so that damage starts
# within 2000 steps.
@pytest.mark.parametrize("kind,d,h,steps,vf", [(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, 2000, 5.0),
                                               (rfdem.RF_TEST_BRAZIL, 10.0, 4.0, 2000, 1.0)], ids=["uniaxial", "brazil"])
def test_ext_engine_bitexact_vs_oracle(cuda, kind, d, h, steps, vf):
    v = (-10.0 if kind == rfdem.RF_TEST_UNIAXIAL else -100.0) * 0.02 / 1e3 * vf
    t, R, rad, x = extspec.ext_case(kind, d, h, min_stress=1e3, v_load=v, max_strain=1.0)
    o = oracle.run_ext(mc.clone(t), x, R, rad, steps)
    res, st = run_engine_ext(t, x, R, rad, steps)
    assert res.steps == o["steps"] == steps
    assert res.error == 0 and o["status"] == 0
    assert np.array_equal(st["R64"], o["R"]), np.max(np.abs(st["R64"] - o["R"]))
    assert np.array_equal(st["V"], o["V"])
    assert np.array_equal(st["IL"].astype(np.uint64), o["IL"])
    assert np.array_equal(st["ILtype"], o["ILtype"])
    assert res.broken_bonds == o["broken"]
    assert_damage(t, x, R, rad, o, res)


def test_ext_engine_stream_equals_graph(cuda, monkeypatch):
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 8.0, min_stress=1e3)
    _, a = run_engine_ext(t, x, R, rad, 120)
    _, b = run_engine_ext(t, x, R, rad, 120, no_graph=True, monkeypatch=monkeypatch)
    assert np.array_equal(a["R64"], b["R64"])
    assert np.array_equal(a["IL"], b["IL"]) and np.array_equal(a["ILtype"], b["ILtype"])


def test_pack_cylinder_overlap_container_determinism(cuda):
    N, r0 = 3000, 0.25
    R, rad, D, H, mo = rfdem.pack_cylinder(N, r0, aspect=2.0, phi=0.55, seed=0xB2000000 + 11)
    assert mo < 2e-4
    assert np.all(rad >= 0.8 * r0 - 1e-12) and np.all(rad <= 1.2 * r0 + 1e-12)
    P = R.reshape(3, N)
    rho = np.sqrt(P[0] ** 2 + P[1] ** 2)
    # the wall is a soft contact too: allow the same relative overlap
    assert np.all(rho + rad <= 0.5 * D + 2e-4 * rad + 1e-9)
    assert np.all(np.abs(P[2]) + rad <= 0.5 * H + 2e-4 * rad + 1e-9)
    assert abs(H / D - 2.0) < 1e-12
    # pairwise overlap check (brute force over a cell-free O(N^2) in blocks)
    X = P.T
    worst = 0.0
    for s in range(0, N, 500):
        dd = np.sqrt(((X[s:s + 500, None, :] - X[None, :, :]) ** 2).sum(-1))
        rr = rad[s:s + 500, None] + rad[None, :]
        np.fill_diagonal(dd[:, s:s + 500], np.inf)
        ov = (rr - dd) / np.minimum(rad[s:s + 500, None], rad[None, :])
        worst = max(worst, float(ov.max()))
    assert worst < 2e-4 + 1e-9
    R2, rad2, _, _, _ = rfdem.pack_cylinder(N, r0, aspect=2.0, phi=0.55, seed=0xB2000000 + 11)
    assert np.array_equal(R, R2) and np.array_equal(rad, rad2)


def test_ext_packed_specimen_vs_oracle_and_fp64(cuda):
    """A packed polydisperse cylinder: engine == float oracle bit for bit; the FP64
    oracle stays within a small position error over the window."""
    N, r0 = 2500, 0.25
    R0, rad, D, H, mo = rfdem.pack_cylinder(N, r0, aspect=2.0, phi=0.55, seed=0xB2000000 + 2001)
    t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, r0, min_stress=1e3)
    x = rfdem.ext_params_si()
    steps = 400
    o = oracle.run_ext(mc.clone(t), x, R, rad, steps)
    res, st = run_engine_ext(t, x, R, rad, steps)
    assert res.steps == steps and res.error == 0
    assert np.array_equal(st["R64"], o["R"])
    assert np.array_equal(st["ILtype"], o["ILtype"])
    g = oracle.run_ext(mc.clone(t), x, R, rad, steps, fp64=True)
    err = float(np.max(np.abs(o["R"] - g["R"])))
    print("packed N=%d bonds=%d max |R_f32force - R_fp64| = %.3e mm" % (N, int(o["ILtype"].sum()), err))
    assert err < 1e-6 * (H + D)


def test_autotune_leaves_results_unchanged(cuda):
    """The autotuner's trial steps are undone: an autotuned engine steps exactly like an
    untuned one, whichever variant it picked."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_UNIAXIAL, 6.0, 10.0, min_stress=1e3)
    a = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    b = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    pick, ms = b.autotune(50)
    assert pick in (5, 6, 8) and all(m > 0 for m in ms)
    a.step(150)
    b.step(150)
    assert np.array_equal(a.positions_f64(), b.positions_f64())
    sa, sb = a.export(), b.export()
    assert np.array_equal(sa["IL"], sb["IL"]) and np.array_equal(sa["V"], sb["V"])
    assert a.counters()["steps"] == b.counters()["steps"] == 150
    a.close(); b.close()


@pytest.mark.parametrize("gap", [0.0, 0.5], ids=["uniform-cutoff", "list-gap"])
def test_ext_log_uniform_radius_ratio_3_vs_oracle(cuda, gap):
    """Radii log-uniform in [0.5, 1.5] r0 (radius ratio 3): the packer keeps the range and
    the overlap bound, the list cutoff widens to just past 2 r_max, and the engine's step
    equals the float oracle's bit for bit, with the uniform cutoff and with a list gap
    of 0.5 r0 (pair cutoff min(a_farcut, r_i + r_j + g))."""
    N, r0 = 3000, 0.25
    R0, rad, D, H, mo = rfdem.pack_cylinder(N, r0, rmin=0.5, rmax=1.5, aspect=2.0, phi=0.55,
                                            seed=0xB2000000 + 5001, dist="log-uniform")
    assert mo < 2e-4
    assert np.all(rad >= 0.5 * r0 - 1e-12) and np.all(rad <= 1.5 * r0 + 1e-12)
    # log-uniform: log(r) is uniform, so its mean sits at the middle of the log range
    lr = np.log(rad / r0)
    assert abs(lr.mean() - 0.5 * (np.log(0.5) + np.log(1.5))) < 0.03
    t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, r0, min_stress=1e3)
    assert abs(t.Po.a_farcut - 2.02 * rad.max()) < 1e-12
    x = rfdem.ext_params_si()
    x.list_gap = gap * r0
    steps = 300
    o = oracle.run_ext(mc.clone(t), x, R, rad, steps)
    res, st = run_engine_ext(t, x, R, rad, steps)
    assert res.steps == steps and res.error == 0 and o["status"] == 0
    assert np.array_equal(st["R64"], o["R"])
    assert np.array_equal(st["IL"].astype(np.uint64), o["IL"])
    assert np.array_equal(st["ILtype"], o["ILtype"])
    rows = (st["IL"].reshape(N, -1) != rfdem.EMPTY).sum(axis=1)
    print("radius ratio 3, list gap %g r0: slots per row mean %.1f max %d of %d" % (gap, rows.mean(), rows.max(),
                                                                                  int(t.K)))


def test_ext_list_gap_lattice_vs_oracle(cuda):
    """A list gap on the lattice specimen (both test kinds' code paths share it): engine ==
    float oracle bit for bit over steps that break bonds and form contacts."""
    t, R, rad, x = extspec.ext_case(rfdem.RF_TEST_BRAZIL, 10.0, 4.0, min_stress=1e3, max_strain=1.0)
    x.list_gap = 0.1
    steps = 2000
    o = oracle.run_ext(mc.clone(t), x, R, rad, steps)
    res, st = run_engine_ext(t, x, R, rad, steps)
    assert res.steps == o["steps"] == steps and res.error == 0 and o["status"] == 0
    assert np.array_equal(st["R64"], o["R"])
    assert np.array_equal(st["IL"].astype(np.uint64), o["IL"])
    assert np.array_equal(st["ILtype"], o["ILtype"])
    assert_damage(t, x, R, rad, o, res)


def test_prestrained_window_bitexact_vs_oracle(cuda):
    """rf_engine_affine_strain (20 % lateral, -3 % axial) on a polydisperse specimen with
    the benchmark's bond constants and list gap, then explicit steps: engine == float
    oracle bit for bit through the burst of strength breaks and the loaded contacts that
    follow."""
    r0 = 0.25
    R0, rad = extspec.lattice_ext(0, 24 * r0, 40 * r0, r0=r0, seed=0xB2000000 + 77, rlo=0.9, jitter=0.02)
    t, R = rfdem.make_test_ext(0, R0, rad, r0, dt=0.01, v_load=-0.1 * 40 * r0 * 1e-6, max_strain=1.0,
                               min_stress=1e30)     # a fixed window: the fracture stop out of reach
    x = rfdem.ext_params_si()
    x.list_gap = 0.25 * r0
    steps, strain = 1500, (0.2, 0.2, -0.03)
    o = oracle.run_ext(mc.clone(t), x, R, rad, steps, strain=strain)
    e = rfdem.Engine(mc.clone(t), R, ext=x, radius=rad)
    e.affine_strain(*strain)
    e.step(steps)
    _, res = e.sync()
    st = e.export()
    st["R64"] = e.positions_f64()
    e.close()
    assert res.error == 0 and o["status"] == 0 and res.steps == o["steps"] == steps
    assert np.array_equal(st["R64"], o["R"]), np.abs(st["R64"] - o["R"]).max()
    assert np.array_equal(st["V"], o["V"])
    assert np.array_equal(st["IL"].astype(np.uint64), o["IL"])
    assert np.array_equal(st["ILtype"], o["ILtype"])
    assert_damage(t, x, R, rad, o, res)
