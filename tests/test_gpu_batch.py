"""Several extended-model specimens in one engine: each specimen of the batch must
evolve exactly as the oracle's run of that specimen alone (on the batch's cell grid,
shifted as the batch places it), and a specimen that finishes early is frozen while
the others go on."""
import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem

pytestmark = pytest.mark.gpu


def _specimens(short=None):
    """Three lattice specimens; specimen `short` is pulled (platen moving outwards) so that
    its strain reaches MaxStrain within a few tens of steps (under compression the
    reference's Strain < MaxStrain test never ends a run)."""
    out = []
    for q, (d, h) in enumerate([(6.0, 10.0), (6.0, 8.0), (7.0, 10.0)]):
        R0, rad = extspec.lattice_ext(rfdem.RF_TEST_UNIAXIAL, d, h, seed=0xB2000000 + 100 + q)
        kw = dict(v_load=2e-4, max_strain=2e-4) if q == short else {}
        t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, 0.5, min_stress=1e3, **kw)
        x = extspec.stiff_params(seed=0xB2000000 + 200 + q, weibull_m=3.0 + 3.0 * q)
        out.append((t, R, rad, x))
    return out


def _check_against_oracle(e, specs, steps_each):
    Rall = e.positions_f64()
    st = e.export()
    Ntot = e.N
    E = np.iinfo(np.uint64).max
    for q, (t, R, rad, x) in enumerate(specs):
        first, n, off, tq = e.spec_info(q)
        assert n == int(t.N)
        Rq = R.reshape(3, n).copy()
        Rq[0] += off
        o = oracle.run_ext(tq, x, Rq.reshape(-1), rad, steps_each[q])
        assert o["steps"] == steps_each[q] and o["status"] == 0
        Re = Rall.reshape(3, Ntot)[:, first:first + n].reshape(-1)
        assert np.array_equal(Re, o["R"]), (q, np.abs(Re - o["R"]).max())
        K = int(t.K)
        IL = st["IL"].reshape(Ntot, K)[first:first + n].astype(np.uint64)
        IL = np.where(IL == np.uint64(rfdem.EMPTY), E, IL - np.uint64(first))
        assert np.array_equal(IL.reshape(-1), o["IL"]), q
        assert np.array_equal(st["ILtype"].reshape(Ntot, K)[first:first + n].reshape(-1), o["ILtype"]), q
        _, r = e.sync_spec(q)
        assert r.steps == steps_each[q]


def test_batch_matches_single_runs(cuda):
    specs = _specimens()
    e = rfdem.BatchEngine([s[0] for s in specs], [s[3] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    assert rfdem.lib.rf_engine_batch_size(e.h) == 3
    steps = 250
    e.step(steps)
    _check_against_oracle(e, specs, [steps] * 3)
    e.close()


def test_batch_specimen_finishing_early_is_frozen(cuda):
    specs = _specimens(short=1)
    # the specimen's own stop step, from the oracle
    t1, R1, rad1, x1 = specs[1]
    e = rfdem.BatchEngine([s[0] for s in specs], [s[3] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    _, _, off, tq = e.spec_info(1)
    Rq = R1.reshape(3, -1).copy()
    Rq[0] += off
    o = oracle.run_ext(tq, x1, Rq.reshape(-1), rad1, 10 ** 6)
    stop = o["steps"]
    assert 0 < stop < 200
    e.step(200)
    _check_against_oracle(e, specs, [200, stop, 200])
    c1 = e.curve_spec(1)
    assert c1.shape[0] == stop
    e.close()


def _drop_specimens():
    """Three weak lattice specimens (strengths a tenth of the granite's) under slow
    compression that reach a peak and lose half of it within a few thousand steps."""
    po = rfdem.granite_potential()
    out = []
    for q, (d, h) in enumerate([(6.0, 10.0), (6.0, 8.0), (7.0, 10.0)]):
        R0, rad = extspec.lattice_ext(rfdem.RF_TEST_UNIAXIAL, d, h, seed=0xB2000000 + 100 + q)
        t, R = rfdem.make_test_ext(rfdem.RF_TEST_UNIAXIAL, R0, rad, 0.5, v_load=-2e-4, min_stress=4e-4)
        x = extspec.stiff_params(seed=0xB2000000 + 200 + q, weibull_m=3.0 + 3.0 * q, sigma_c=po.m_Ec * 0.1,
                                 tau_c=po.m_Gc * 0.1)
        x.post_peak_drop = 0.5
        out.append((t, R, rad, x))
    return out


def test_batch_post_peak_drop_stop(cuda):
    """Each specimen runs to a post-peak load drop of 50 % and stops at the step the
    oracle stops at, with the oracle's positions and rows."""
    specs = _drop_specimens()
    e = rfdem.BatchEngine([s[0] for s in specs], [s[3] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    stops = []
    for q, (t, R, rad, x) in enumerate(specs):
        _, _, off, tq = e.spec_info(q)
        Rq = R.reshape(3, -1).copy()
        Rq[0] += off
        o = oracle.run_ext(tq, x, Rq.reshape(-1), rad, 10 ** 5)
        assert o["status"] == 0
        stops.append(o["steps"])
    assert len(set(stops)) == 3 and max(stops) < 5000
    e.step(10 ** 5)                                   # ends when every specimen has stopped
    _check_against_oracle(e, specs, stops)
    for q in range(3):
        tq, r = e.sync_spec(q)
        assert r.Fracture == 1
        c = e.curve_spec(q)
        s = 0.5 * (np.abs(c[:, 1]) + np.abs(c[:, 2]))
        assert s[-1] < 0.5 * s.max()
    e.close()


def test_sharded_run_matches_the_batch(cuda):
    """rfdem.shard on one rank: the rank's share (all specimens) runs in one batched
    engine, and the gathered table equals the batch's own per-specimen results."""
    from rfdem.shard import RESULT_FIELDS, run_sharded
    specs = _specimens(short=1)
    tasks, params, Rs, rads = [s[0] for s in specs], [s[3] for s in specs], [s[1] for s in specs], [s[2] for s in specs]
    table = run_sharded(tasks, params, Rs, rads, steps=200)
    e = rfdem.BatchEngine(tasks, params, Rs, rads)
    e.step(200)
    for q in range(3):
        _, r = e.sync_spec(q)
        assert [float(getattr(r, f)) for f in RESULT_FIELDS] == table[q].tolist()
    e.close()
    assert table[1][0] < 200 and table[0][0] == table[2][0] == 200


def test_fire_batch_matches_single_specimens(cuda):
    """Quasi-static load increments of a batch (rf_engine_load_increment_batch): every
    specimen relaxes on its own FIRE scalars and ends each increment where its run alone
    ends (a one-specimen engine on the same placed specimen), up to the order of the FP64
    sums: a batch groups a specimen's particles into CTAs differently."""
    specs = _specimens()
    e = rfdem.BatchEngine([s[0] for s in specs], [s[3] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    p = e.relax_params(max_iter=40000, strain_inc=1e-4)
    n = 4
    res = [e.load_increment(p) for _ in range(n)]
    Rall = e.positions_f64()
    iters = [[r.iterations for r in rk] for rk in res]
    print("batch iterations per increment and specimen:", iters)
    assert len({tuple(row) for row in zip(*iters)}) > 1 or n == 1   # the specimens stop at their own counts
    for q, (t, R, rad, x) in enumerate(specs):
        first, m, off, tq = e.spec_info(q)
        Rq = R.reshape(3, m).copy()
        Rq[0] += off
        Rq = Rq.reshape(-1)
        a = rfdem.Engine(mc.clone(tq), Rq, ext=x, radius=rad)
        ra = [a.load_increment(p) for _ in range(n)]
        Ra = a.positions_f64()
        a.close()
        Re = Rall.reshape(3, e.N)[:, first:first + m].reshape(-1)
        ext = float(np.ptp(Rq.reshape(3, m)[2]))
        for k in range(n):
            rb = res[k][q]
            print("specimen %d increment %d: iterations batch %d alone %d, stress batch %.9e alone %.9e" %
                  (q, k, rb.iterations, ra[k].iterations, rb.stress, ra[k].stress))
            assert rb.error == 0 and rb.converged == 1 and ra[k].converged == 1
            assert abs(rb.stress - ra[k].stress) <= 1e-6 * abs(ra[k].stress) + 1e-15
            assert abs(rb.iterations - ra[k].iterations) <= 0.1 * ra[k].iterations + 5
        assert ra[-1].stress > 0
        assert np.max(np.abs(Re - Ra)) < 1e-7 * ext, (q, np.abs(Re - Ra).max())
    e.close()
