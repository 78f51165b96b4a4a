"""md_* drop-in kernels against the oracle, bit for bit, on seeded specimens."""
import numpy as np
import pytest

import extspec
import mdcall as mc
import oracle
import rfdem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(0, 9.0, 14.0), (1, 16.0, 6.0), (0, 24.0, 40.0)],
                ids=["uniaxial-1k", "brazil-1k", "uniaxial-18k"])
def case(request):
    kind, d, h = request.param
    t, R = rfdem.make_test(kind, d, h, seed=0xB2000000 + 11)
    return t, R


def test_cell_distribution_bitexact(cuda, case):
    t, R = case
    st, CI, CIs, pnC = mc.gpu_cells(cuda, t, R)
    so, CIo, CIso, pnCo = mc.oracle_cells(t, R)
    assert st == so == 0
    assert np.array_equal(CI, CIo)
    assert np.array_equal(CIs, CIso)
    assert np.array_equal(pnC, pnCo)


def test_cell_last_run_quirk(cuda):
    """The reference's run scan reads past N: the last cell's count grows by one when the
    first sorted id equals the last cell index (md_calculate_cell.cu:72)."""
    t, R = rfdem.make_test(0, 9.0, 14.0)
    N = R.size // 3
    _, CI, CIs, _ = mc.oracle_cells(t, R)
    last = int(CIs[N - 1])
    first_id = int(CIs[N])
    # move the particle whose id equals `last` into the lowest occupied cell so it sorts first
    if last < N:
        lo = int(np.argmin(CI))
        R2 = R.copy()
        for c in range(3):
            R2[last + c * N] = R[lo + c * N]
        st, CI2, CIs2, pnC2 = mc.gpu_cells(cuda, t, R2)
        _, CIo, CIso, pnCo = mc.oracle_cells(t, R2)
        assert np.array_equal(pnC2, pnCo) and np.array_equal(CIs2, CIso)
    else:
        pytest.skip("specimen too small for the quirk layout (first id %d)" % first_id)


def test_list_construct_bitexact(cuda, case):
    t, R = case
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    st, IL = mc.gpu_list_construct(cuda, t, R, CIs, pnC)
    so, ILo = mc.oracle_list_construct(t, R, CIs, pnC)
    assert st == so == 0
    assert np.array_equal(IL, ILo)


def test_list_matches_bruteforce(cuda, case):
    """h_CheckInteractions (md_check_test.cu:26-95): every pair within a_farcut is in the
    row and nothing beyond it is, by an all-pairs scan."""
    t, R = case
    N, K = R.size // 3, int(t.K)
    if N > 5000:
        pytest.skip("all-pairs scan kept to small specimens")
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    _, IL = mc.gpu_list_construct(cuda, t, R, CIs, pnC)
    X = R.reshape(3, N).T.astype(np.float32)
    rows = IL.reshape(N, K)
    for i in range(N):
        d = X - X[i]
        rr = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        want = set(np.nonzero((rr < np.float32(t.aacut)) & (np.arange(N) != i))[0].tolist())
        got = set(int(j) for j in rows[i] if j != rfdem.EMPTY)
        assert got == want, i


def test_reconstruct_bitexact_with_holes_and_quirks(cuda, case):
    t, R = case
    N, K = R.size // 3, int(t.K)
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    _, IL = mc.oracle_list_construct(t, R, CIs, pnC)
    rng = np.random.default_rng(5)
    holes = IL.copy()
    live = np.nonzero(holes != rfdem.EMPTY)[0]
    holes[rng.choice(live, size=len(live) // 3, replace=False)] = rfdem.EMPTY
    holes[0] = rfdem.EMPTY          # particle 0, slot 0: the kdxfree == 0 quirk
    ty = rng.integers(0, 2, size=N * K).astype(np.uint8)
    st, ILg, tyg = mc.gpu_reconstruct(cuda, t, R, CIs, pnC, holes, ty)
    so, ILo, tyo = mc.oracle_reconstruct(t, R, CIs, pnC, holes, ty)
    assert st == so == 0
    assert np.array_equal(ILg, ILo)
    assert np.array_equal(tyg, tyo)
    # every hole refilled: same link sets per row as the full build
    assert np.array_equal(np.sort(ILg.reshape(N, K), 1), np.sort(IL.reshape(N, K), 1))


def test_reconstruct_row_overflow_reports(cuda):
    t, R = rfdem.make_test(0, 9.0, 14.0)
    t.K = 4
    N, K = R.size // 3, 4
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    IL = np.full(N * K, rfdem.EMPTY, dtype=rfdem.ID_NP)
    ty = np.zeros(N * K, np.uint8)
    st, ILg, _ = mc.gpu_reconstruct(cuda, t, R, CIs, pnC, IL, ty)
    so, ILo, _ = mc.oracle_reconstruct(t, R, CIs, pnC, IL, ty)
    assert st == rfdem.RF_ERR_ROW_OVERFLOW and so == rfdem.RF_ERR_ROW_OVERFLOW
    assert np.array_equal(ILg, ILo)


def test_bonds_and_delete_bitexact(cuda, case):
    t, R = case
    N, K = R.size // 3, int(t.K)
    _, CI, CIs, pnC = mc.oracle_cells(t, R)
    _, IL = mc.oracle_list_construct(t, R, CIs, pnC)
    ty, iL, S = np.zeros(N * K, np.uint8), np.zeros(N * K, np.float32), mc.zeros_state(N, K)
    aa_create, aa_far = np.float32(t.Po.b_dd), np.float32(t.Po.aa_farcut)
    g = mc.gpu_bonds_delete(cuda, t, R, IL, ty, iL, S, aa_create, aa_far, True, False)
    o = mc.oracle_bonds_delete(t, R, IL, ty, iL, S, aa_create, aa_far, True, False)
    for a, b in zip(g[:3], o[:3]):
        assert np.array_equal(a, b)
    assert (g[1] == 1).sum() > 3 * N
    # move some particles so links cross a_farcut, then delete
    rng = np.random.default_rng(9)
    R2 = R + rng.normal(scale=0.12, size=R.size).astype(np.float32)
    g2 = mc.gpu_bonds_delete(cuda, t, R2, g[0], g[1], g[2], g[3], aa_create, aa_far, False, True)
    o2 = mc.oracle_bonds_delete(t, R2, o[0], o[1], o[2], o[3], aa_create, aa_far, False, True)
    for a, b in zip(g2[:3], o2[:3]):
        assert np.array_equal(a, b)
    for k in ["Rij", "Oijt", "Mijn", "Mijt"]:
        assert np.array_equal(g2[3][k], o2[3][k])
    assert (g2[0] == rfdem.EMPTY).sum() > (g[0] == rfdem.EMPTY).sum()


def test_forces_bitexact_on_evolved_state(cuda, case):
    """_22 then _21 from a state evolved by the oracle (rotations, shear history, broken
    bonds, contacts): forces, moments, slot state and break flags bit for bit."""
    t, R = case
    steps = 40 if R.size // 3 < 5000 else 10
    t2, st = mc.oracle_state_after(t, R, steps)
    S = {k: st[k] for k in ["Rij", "Oijt", "Mijn", "Mijt"]}
    rng = np.random.default_rng(3)
    V = st["V"] + rng.normal(scale=2e-4, size=st["V"].size).astype(np.float32)
    W = st["W"] + rng.normal(scale=2e-3, size=st["W"].size).astype(np.float32)
    g = mc.gpu_forces(cuda, t, st["R"], V, W, st["IL"], st["ILtype"], st["iL"], S)
    o = mc.oracle_forces(t, st["R"], V, W, st["IL"], st["ILtype"], st["iL"], S)
    for k in ["F", "M", "ty", "Rij", "Oijt", "Mijn", "Mijt"]:
        assert np.array_equal(g[k].view(np.uint8), o[k].view(np.uint8)), k
    assert np.abs(o["F"]).max() > 0


def test_forces_bitexact_on_damaged_state(cuda):
    """_22 then _21 on a state with broken bonds and loaded contacts (a 585-particle
    cylinder after 3000 steps at 5x the reference's platen speed): forces, moments, slot
    state and break flags bit for bit, and the state holds what the claim needs."""
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=0xB2000000 + 21, max_strain=1.0,
                           v_load=-10.0 * 0.02 / 1e3 * 5.0)
    N, K = R.size // 3, int(t.K)
    _, st = mc.oracle_state_after(t, R, 3000)
    S = {k: st[k] for k in ["Rij", "Oijt", "Mijn", "Mijt"]}
    g = mc.gpu_forces(cuda, t, st["R"], st["V"], st["W"], st["IL"], st["ILtype"], st["iL"], S)
    o = mc.oracle_forces(t, st["R"], st["V"], st["W"], st["IL"], st["ILtype"], st["iL"], S)
    for k in ["F", "M", "ty", "Rij", "Oijt", "Mijn", "Mijt"]:
        assert np.array_equal(g[k].view(np.uint8), o[k].view(np.uint8)), k
    _, contacts = extspec.pair_counts(st["R"], N, K, st["IL"], st["ILtype"], np.full(N, t.Po.p_r))
    oz = np.abs(o["Oijt"].reshape(-1, 3)).sum(1) > 0
    loaded = int((oz & (st["ILtype"] == 0) & (st["IL"] != rfdem.EMPTY)).sum())
    print("broken bonds %d, overlapping contacts %d, contact slots with tangential overlap %d" %
          (int(st["broke"].sum()), contacts, loaded))
    assert int(st["broke"].sum()) > 0 and contacts > 0 and loaded > 0
