"""The oracle against golden fixtures made by the reference's OWN kernels
(tests/golden/make_golden.py ran them on a B200 on these seeded inputs): cells, rows and
bond flags bit for bit; one force evaluation within the bound set by the reference
build's FMA contractions and library norm; a 200-step whole run within tolerance.
Runs on the CPU: the inputs are regenerated with the same seeded generator."""
import os

import numpy as np
import pytest

import mdcall as mc
import oracle
import rfdem

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"uniaxial": (rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0), "brazil": (rfdem.RF_TEST_BRAZIL, 16.0, 6.0)}
SEED = 0xB2000000 + 31
FORCE_STEPS, RUN_STEPS = 40, 200


def to64(a):
    out = a.astype(np.uint64)
    out[a == np.uint32(0xFFFFFFFF)] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return out


@pytest.fixture(scope="module", params=list(CASES))
def gold(request):
    kind, d, h = CASES[request.param]
    t, R = rfdem.make_test(kind, d, h, seed=SEED)
    return t, R, dict(np.load(os.path.join(HERE, "ref_%s.npz" % request.param)))


def test_cells_rows_bonds_bitexact(gold):
    t, R, g = gold
    N, K = R.size // 3, int(t.K)
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    assert np.array_equal(CI, to64(g["CI"]))
    assert np.array_equal(CIs, to64(g["CIs"]))
    assert np.array_equal(pnC, to64(g["pnC"]))
    _, IL = mc.oracle_list_construct(t, R, CIs, pnC)
    assert np.array_equal(IL, to64(g["IL"]))
    ty, iL = np.zeros(N * K, np.uint8), np.zeros(N * K, np.float32)
    _, tyo, iLo, _ = mc.oracle_bonds_delete(t, R, IL, ty, iL, mc.zeros_state(N, K), np.float32(t.Po.b_dd),
                                            np.float32(t.Po.aa_farcut), True, False)
    assert np.array_equal(tyo, g["bond_ty"])
    assert np.array_equal(iLo.view(np.uint32), g["bond_iL"].view(np.uint32))


def test_forces_within_bound(gold):
    t, R, g = gold
    N, K = R.size // 3, int(t.K)
    _, st = mc.oracle_state_after(t, R, FORCE_STEPS)
    rng = np.random.default_rng(4)
    V = st["V"] + rng.normal(scale=2e-4, size=3 * N).astype(np.float32)
    W = st["W"] + rng.normal(scale=2e-3, size=3 * N).astype(np.float32)
    S = {k: st[k].copy() for k in ["Rij", "Oijt", "Mijn", "Mijt"]}
    o = mc.oracle_forces(t, st["R"], V, W, st["IL"], st["ILtype"], st["iL"], S)
    flips = np.nonzero(g["force_ty"] != o["ty"])[0]
    assert flips.size <= 2, flips
    # one ulp of |r| (library norm3df vs sqrt of the float sum) moves the bond normal
    # force by E*A*(1/L0)*ulp(|r|); 4 such ulps per particle
    P = t.Po
    ulp_r = np.spacing(np.float32(1.0 / st["iL"][st["iL"] > 0].min()))
    dF = 4 * P.m_E * np.pi * P.b_r ** 2 * st["iL"].max() * ulp_r
    assert np.abs(g["force_F"].astype(np.float64) - o["F"]).max() <= dF
    assert np.abs(g["force_M"].astype(np.float64) - o["M"]).max() <= dF * 2 * P.p_r
    sc = np.abs(o["Oijt"]).max() + 1e-30
    np.testing.assert_allclose(g["force_Oijt"], o["Oijt"], rtol=0, atol=1e-4 * sc)


def test_whole_run(gold):
    t, R, g = gold
    N, K = R.size // 3, int(t.K)
    n, st, curve, status = oracle.run_f(mc.clone(t), R, RUN_STEPS)
    assert n == RUN_STEPS and status == 0
    ext = np.ptp(R)
    np.testing.assert_allclose(st["R"], g["run_R"], rtol=0, atol=1e-5 * ext)

    def pairs(IL, ty):
        rows, tys = IL.reshape(N, K), ty.reshape(N, K)
        return {(i, int(rows[i, k])): int(tys[i, k]) for i in range(N) for k in range(K) if rows[i, k] < N}
    pr = pairs(to64(g["run_IL"]), g["run_ty"])
    po = pairs(st["IL"], st["ILtype"])
    Rr = g["run_R"].reshape(3, N)
    acut = float(np.sqrt(np.float32(t.aacut)))
    near = lambda p: abs(float(np.linalg.norm(Rr[:, p[1]] - Rr[:, p[0]])) - acut) < 1e-4
    assert not [p for p in set(pr) ^ set(po) if not near(p)]
    assert len([p for p in set(pr) & set(po) if pr[p] != po[p]]) <= 2
    m = min(len(curve), RUN_STEPS)
    gc = g["run_curve"].reshape(-1, 3)[:m]
    # platen stresses: sums of bond forces whose stretches are ~1e-6 mm, so the
    # reference build's contracted arithmetic moves them by a few % of the peak
    sc = np.abs(gc[:, 1:]).max() + 1e-30
    np.testing.assert_allclose(curve[:m, 1:], gc[:, 1:], rtol=0, atol=5e-2 * sc)
    np.testing.assert_allclose(curve[:m, 0], gc[:, 0], rtol=0, atol=1e-12)
