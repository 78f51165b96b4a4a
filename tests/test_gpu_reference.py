"""The oracle and the engine against the reference's OWN kernels (compiled unmodified
from its sources for sm_100a into oracle/_ref), on identical seeded inputs.

Integer outputs (cells, rows, bond flags) must match bit for bit. Float outputs are
compared within tolerance: the reference build lets nvcc contract a*b+c into FMAs
and uses the library norm3df, while the oracle and engine evaluate each operation
separately and use sqrt(x*x+y*y+z*z)."""
import numpy as np
import pytest

import mdcall as mc
import oracle
import rfdem

pytestmark = pytest.mark.gpu

REF = oracle.ref_gpu()
needs_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref/libmdref_gpu.so not built")


def ref_cells(t, R):
    N, CN = R.size // 3, int(t.C.N)
    CI, CIs, pnC = np.zeros(N, np.uint32), np.zeros(2 * N, np.uint32), np.zeros(2 * CN, np.uint32)
    assert REF.ref_cell_distribution(R.ctypes.data, N, CI.ctypes.data, CIs.ctypes.data, pnC.ctypes.data, CN, t.C.a,
                                     t.C._1d_a, t.C.Nr) == 0
    return CI, CIs, pnC


def to64(a):
    out = a.astype(np.uint64)
    out[a == np.uint32(0xFFFFFFFF)] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return out


def to32(a):
    out = a.astype(np.uint32)
    out[a == np.uint64(0xFFFFFFFFFFFFFFFF)] = np.uint32(0xFFFFFFFF)
    return out


@pytest.fixture(scope="module", params=[(0, 9.0, 14.0), (1, 16.0, 6.0), (0, 24.0, 40.0)],
                ids=["uniaxial-1k", "brazil-1k", "uniaxial-18k"])
def case(request):
    kind, d, h = request.param
    return rfdem.make_test(kind, d, h, seed=0xB2000000 + 31)


@needs_ref
def test_cells_and_rows_bitexact_vs_reference(cuda, case):
    t, R = case
    N, K = R.size // 3, int(t.K)
    CI, CIs, pnC = ref_cells(t, R)
    _, CIo, CIso, pnCo = mc.oracle_cells(t, R)
    assert np.array_equal(to64(CI), CIo)
    assert np.array_equal(to64(CIs), CIso)
    assert np.array_equal(to64(pnC), pnCo)
    IL = np.zeros(N * K, np.uint32)
    assert REF.ref_list_construct(R.ctypes.data, N, K, int(t.C.N), t.C.a, t.C._1d_a, t.aacut, t.C.Nr,
                                  IL.ctypes.data) == 0
    _, ILo = mc.oracle_list_construct(t, R, CIso, pnCo)
    assert np.array_equal(to64(IL), ILo)
    # engine md_* path too
    _, ILg = mc.gpu_list_construct(cuda, t, R, CIso, pnCo)
    assert np.array_equal(ILg, ILo)


@needs_ref
def test_reconstruct_bitexact_vs_reference(cuda, case):
    t, R = case
    N, K = R.size // 3, int(t.K)
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    _, IL = mc.oracle_list_construct(t, R, CIs, pnC)
    rng = np.random.default_rng(17)
    holes = IL.copy()
    live = np.nonzero(holes != rfdem.EMPTY)[0]
    holes[rng.choice(live, size=len(live) // 4, replace=False)] = rfdem.EMPTY
    ty = rng.integers(0, 2, size=N * K).astype(np.uint8)
    IL32, ty_r = to32(holes), ty.copy()
    assert REF.ref_reconstruct_bpm(R.ctypes.data, N, K, int(t.C.N), t.C.a, t.C._1d_a, t.aacut, t.C.Nr,
                                   IL32.ctypes.data, ty_r.ctypes.data) == 0
    _, ILo, tyo = mc.oracle_reconstruct(t, R, CIs, pnC, holes, ty)
    assert np.array_equal(to64(IL32), ILo)
    assert np.array_equal(ty_r, tyo)


@needs_ref
def test_bond_construction_vs_reference(cuda, case):
    """Bond flags and 1/L0 (the FMA-contracted |r|^2 and the correctly rounded rsqrt)."""
    t, R = case
    N, K = R.size // 3, int(t.K)
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    _, IL = mc.oracle_list_construct(t, R, CIs, pnC)
    ty, iL = np.zeros(N * K, np.uint8), np.zeros(N * K, np.float32)
    ty_r, iL_r = ty.copy(), iL.copy()
    IL32 = to32(IL)                        # kept alive across the call
    assert REF.ref_construct_bonds(R.ctypes.data, N, K, IL32.ctypes.data, ty_r.ctypes.data, iL_r.ctypes.data,
                                   np.float32(t.Po.b_dd), np.float32(t.Po.b_r)) == 0
    ILo, tyo, iLo, _ = mc.oracle_bonds_delete(t, R, IL, ty, iL, mc.zeros_state(N, K), np.float32(t.Po.b_dd),
                                              np.float32(t.Po.aa_farcut), True, False)
    assert np.array_equal(ty_r, tyo)
    assert np.array_equal(iL_r.view(np.uint32), iLo.view(np.uint32))


def oracle_criteria(t, st, V, W, S):
    """The oracle's break criteria (Sc, Mc) of every bond slot on a state, [N*K, 2]."""
    L = oracle.load()
    N, K = st["R"].size // 3, int(t.K)
    S = {k: v.copy() for k, v in S.items()}
    ty = st["ILtype"].copy()
    F, M = np.zeros(3 * N, np.float32), np.zeros(3 * N, np.float32)
    crit = np.zeros(2 * N * K, np.float32)
    big = [float(np.float32(3e38))] * 2           # strengths nothing reaches: every criterion is evaluated
    L.rfo_forces_22_crit_f(st["R"].ctypes.data, V.ctypes.data, W.ctypes.data, st["IL"].ctypes.data, ty.ctypes.data,
                           st["iL"].ctypes.data, S["Rij"].ctypes.data, S["Oijt"].ctypes.data, S["Mijn"].ctypes.data,
                           S["Mijt"].ctypes.data, F.ctypes.data, M.ctypes.data, N, K, *mc.bond_params(t)[:4], *big,
                           None, crit.ctypes.data)
    return crit.reshape(-1, 2)


def threshold_eps(t, il):
    """Stated epsilon of the tensile break test for a bond of 1/L0 = il: the criterion's
    stress E*(|r| - L0)/L0 moves by E*il*ulp(|r|) for one ulp of |r| (the reference's
    norm3df and FMA-contracted sums against the correctly rounded sqrt here), so four such
    ulps; near_threshold adds 1e-5 of the criterion for its moment terms."""
    P = t.Po
    L0 = np.float32(1.0) / np.float32(il)
    return 4.0 * P.m_E * float(il) * float(np.spacing(L0))


def near_threshold(t, st, crit, k, sig_c, tau_c):
    """Slot k's tensile criterion within threshold_eps + 1e-5 of itself + 4 ulp of sig_c of
    sig_c, or its shear criterion within 1e-5 of itself + 4 ulp of tau_c of tau_c."""
    Sc, Mc = float(crit[k, 0]), float(crit[k, 1])
    eS = threshold_eps(t, st["iL"][k]) + 1e-5 * abs(Sc) + 4 * float(np.spacing(np.float32(sig_c)))
    eM = 1e-5 * abs(Mc) + 4 * float(np.spacing(np.float32(tau_c)))
    return abs(Sc - sig_c) <= eS or abs(Mc - tau_c) <= eM


@needs_ref
def test_break_decisions_vs_reference_near_threshold_only(cuda):
    """Break decisions of d_CalculateForcesDEM_22 on a loaded state (a 585-particle
    cylinder after 20,000 steps), with the strengths set to the median tensile and the
    90th-percentile shear criterion of its bonds, so that one step decides hundreds of
    breaks and several bonds sit near a threshold. The reference's own kernel, the oracle
    and the engine's md_ kernel decide; the engine equals the oracle bit for bit, and every
    decision where the reference differs is a bond listed as near the threshold (its
    criterion within the stated epsilon of the strength)."""
    t, R = rfdem.make_test(0, 9.0, 14.0, seed=0xB2000000 + 55, max_strain=1.0)
    N, K = R.size // 3, int(t.K)
    _, st = mc.oracle_state_after(t, R, 20000)
    S = {k: st[k].copy() for k in ["Rij", "Oijt", "Mijn", "Mijt"]}
    crit = oracle_criteria(t, st, st["V"], st["W"], S)
    bond = np.nonzero(st["ILtype"] == 1)[0]
    sig_c = float(np.float32(np.quantile(crit[bond, 0], 0.5)))
    tau_c = float(np.float32(np.quantile(crit[bond, 1], 0.9)))
    tq = mc.clone(t)
    tq.Po.m_Ec, tq.Po.m_Gc = sig_c, tau_c
    o = mc.oracle_forces(tq, st["R"], st["V"], st["W"], st["IL"], st["ILtype"], st["iL"], S)
    g = mc.gpu_forces(cuda, tq, st["R"], st["V"], st["W"], st["IL"], st["ILtype"], st["iL"], S)
    assert np.array_equal(g["ty"], o["ty"])
    assert np.array_equal(g["F"].view(np.uint32), o["F"].view(np.uint32))
    ref = {k: v.copy() for k, v in S.items()}
    ty_r = st["ILtype"].copy()
    F, M = np.zeros(3 * N, np.float32), np.zeros(3 * N, np.float32)
    p22 = np.array(mc.bond_params(tq), np.float32)
    p21 = np.array(mc.contact_params(tq), np.float32)
    IL32 = to32(st["IL"])
    assert REF.ref_forces(st["R"].ctypes.data, st["V"].ctypes.data, st["W"].ctypes.data, N, K, IL32.ctypes.data,
                          ty_r.ctypes.data, st["iL"].ctypes.data, ref["Rij"].ctypes.data, ref["Oijt"].ctypes.data,
                          ref["Mijn"].ctypes.data, ref["Mijt"].ctypes.data, F.ctypes.data, M.ctypes.data,
                          p22.ctypes.data, p21.ctypes.data, 1) == 0
    broke_o = bond[o["ty"][bond] == 0]
    broke_r = bond[ty_r[bond] == 0]
    listed = [int(k) for k in bond if near_threshold(tq, st, crit, k, sig_c, tau_c)]
    flips = np.nonzero(ty_r != o["ty"])[0]
    print("bond slots %d; breaks: oracle/engine %d, reference %d; near-threshold bonds listed separately %d; "
          "decisions that differ %d" % (bond.size, broke_o.size, broke_r.size, len(listed), flips.size))
    print("near-threshold list (slot, Sc - sig_c, Mc - tau_c):",
          [(k, float(crit[k, 0]) - sig_c, float(crit[k, 1]) - tau_c) for k in listed[:20]])
    assert broke_o.size > 100 and len(listed) > 0
    off_list = [int(k) for k in flips if k not in set(listed)]
    assert not off_list, [(k, float(crit[k, 0]) - sig_c, float(crit[k, 1]) - tau_c) for k in off_list[:10]]


def _force_scale(F):
    n = F.size // 3
    return np.sqrt(F[:n] ** 2 + F[n:2 * n] ** 2 + F[2 * n:] ** 2).max()


@needs_ref
def test_forces_vs_reference_within_tolerance(cuda, case):
    t, R = case
    steps = 40 if R.size // 3 < 5000 else 10
    t2, st = mc.oracle_state_after(t, R, steps)
    N, K = R.size // 3, int(t.K)
    S = {k: st[k].copy() for k in ["Rij", "Oijt", "Mijn", "Mijt"]}
    rng = np.random.default_rng(4)
    V = st["V"] + rng.normal(scale=2e-4, size=3 * N).astype(np.float32)
    W = st["W"] + rng.normal(scale=2e-3, size=3 * N).astype(np.float32)
    o = mc.oracle_forces(t, st["R"], V, W, st["IL"], st["ILtype"], st["iL"], S)
    ref = {k: v.copy() for k, v in S.items()}
    ty_r = st["ILtype"].copy()
    F, M = np.zeros(3 * N, np.float32), np.zeros(3 * N, np.float32)
    p22 = np.array(mc.bond_params(t), np.float32)
    p21 = np.array(mc.contact_params(t), np.float32)
    IL32 = to32(st["IL"])                  # kept alive across the call
    assert REF.ref_forces(st["R"].ctypes.data, V.ctypes.data, W.ctypes.data, N, K, IL32.ctypes.data,
                          ty_r.ctypes.data, st["iL"].ctypes.data, ref["Rij"].ctypes.data, ref["Oijt"].ctypes.data,
                          ref["Mijn"].ctypes.data, ref["Mijt"].ctypes.data, F.ctypes.data, M.ctypes.data,
                          p22.ctypes.data, p21.ctypes.data, 3) == 0
    # break decisions: identical except for bonds whose criterion sits within the stated
    # epsilon of the strength (near_threshold; none of these bonds is close to breaking)
    flips = np.nonzero(ty_r != o["ty"])[0]
    crit = oracle_criteria(t, st, V, W, S)
    assert flips.size == 0 or all(near_threshold(t, st, crit, k, *mc.bond_params(t)[4:6]) for k in flips), flips
    # The bond normal force E*A*(|r| - L0)/L0 cancels |r| against L0 ~ 1 mm, so one ulp of
    # |r| (library norm3df in the reference, sqrt of the float sum here) moves it by
    # E*A*(1/L0)*ulp(|r|). Tolerance: 4 such ulps per particle; moments 4 ulps of the
    # same force times the bond length.
    P = t.Po
    ulp_r = np.spacing(np.float32(1.0 / st["iL"][st["iL"] > 0].min()))
    dF = 4 * P.m_E * np.pi * P.b_r ** 2 * st["iL"].max() * ulp_r
    dM = dF * 2 * P.p_r
    err_F = np.abs(F.astype(np.float64) - o["F"])
    err_M = np.abs(M.astype(np.float64) - o["M"])
    print("max |dF| %.3e (bound %.3e, force scale %.3e); max |dM| %.3e (bound %.3e)" %
          (err_F.max(), dF, _force_scale(o["F"]), err_M.max(), dM))
    assert err_F.max() <= dF
    assert err_M.max() <= dM
    for k in ["Rij", "Oijt", "Mijn", "Mijt"]:
        sc = np.abs(o[k]).max() + 1e-30
        np.testing.assert_allclose(ref[k], o[k], rtol=0, atol=1e-4 * sc, err_msg=k)


@needs_ref
@pytest.mark.parametrize("kind,d,h,steps", [(0, 9.0, 14.0, 300), (1, 16.0, 6.0, 300)], ids=["uniaxial", "brazil"])
def test_whole_run_vs_reference(cuda, kind, d, h, steps):
    """A short whole test through the reference's own driver sequence: rows and bond flags
    equal, positions and load curve within tolerance, error against the FP64 oracle reported."""
    t, R = rfdem.make_test(kind, d, h, seed=0xB2000000 + 41)
    N, K = R.size // 3, int(t.K)
    tr = mc.clone(t)
    out = dict(R=np.zeros(3 * N, np.float32), V=np.zeros(3 * N, np.float32), W=np.zeros(3 * N, np.float32),
               IL=np.zeros(N * K, np.uint32), ty=np.zeros(N * K, np.uint8), iL=np.zeros(N * K, np.float32),
               Rij=np.zeros(3 * N * K, np.float32), Oijt=np.zeros(3 * N * K, np.float32),
               Mijn=np.zeros(3 * N * K, np.float32), Mijt=np.zeros(3 * N * K, np.float32))
    curve_r = np.zeros(3 * steps, np.float64)
    import ctypes as C
    ns = C.c_uint64(0)
    n = REF.ref_run(C.byref(tr), R.ctypes.data, steps, *[out[k].ctypes.data for k in
                                                        ["R", "V", "W", "IL", "ty", "iL", "Rij", "Oijt", "Mijn", "Mijt"]],
                    curve_r.ctypes.data, steps, C.byref(ns))
    assert n == steps
    e = rfdem.Engine(mc.clone(t), R)
    e.step(steps)
    eg = e.export()
    e.close()
    # Links and bond flags as pair sets. The reference build's FMA contractions and
    # library norm shift positions by a few ulps per step, so a pair whose distance sits
    # at the a_farcut threshold (add / delete) may enter or leave on a different step:
    # such pairs are listed separately (|r - a_farcut| < 1e-4 mm), everything else must match.
    def pairs(IL, ty):
        rows = IL.reshape(N, K)
        tys = ty.reshape(N, K)
        d = {}
        for i in range(N):
            for k in range(K):
                j = int(rows[i, k])
                if j < N:
                    d[(i, j)] = int(tys[i, k])
        return d
    pr = pairs(to64(out["IL"]).astype(np.uint64), out["ty"])
    pe = pairs(eg["IL"].astype(np.uint64), eg["ILtype"])
    Rr = out["R"].reshape(3, N)
    acut = float(np.sqrt(np.float32(t.aacut)))
    near = lambda p: abs(float(np.linalg.norm(Rr[:, p[1]] - Rr[:, p[0]])) - acut) < 1e-4
    only = [p for p in set(pr) ^ set(pe) if not near(p)]
    flips = [p for p in set(pr) & set(pe) if pr[p] != pe[p]]
    print("pairs: reference %d engine %d, threshold pairs listed separately %d, other differences %d, "
          "bond-flag flips %d" % (len(pr), len(pe), len(set(pr) ^ set(pe)) - len(only), len(only), len(flips)))
    assert not only, only[:10]
    # no bond of this window comes near its strength: every bond flag must match
    assert not flips, flips
    ext = np.ptp(R)
    np.testing.assert_allclose(out["R"], eg["R"], rtol=0, atol=1e-5 * ext)
    to = mc.clone(t)
    nd, Rd, curve_d, _, _ = oracle.run_d(to, R, steps)
    # Error against the FP64 oracle, reported. FP32 positions of ~20 mm drop increments
    # below half an ulp (~1e-6 mm) and thresholds (break, clamp, row change) are crossed
    # on other steps, so every FP32 run, the reference's own included, sits O(1e-2 mm)
    # from the FP64 trajectory; the engine must be no less accurate than the reference.
    e_eng = np.abs(eg["R"].astype(np.float64) - Rd)
    e_ref = np.abs(out["R"].astype(np.float64) - Rd)
    p_eng, p_ref = np.percentile(e_eng, 99), np.percentile(e_ref, 99)
    print("|R - R_fp64| mm: engine max %.3e p99 %.3e, reference max %.3e p99 %.3e" %
          (e_eng.max(), p_eng, e_ref.max(), p_ref))
    assert p_eng < 0.05 and p_ref < 0.05
    assert p_eng <= 2.0 * p_ref + 1e-6
