"""md_CellDistributionNoAlloc: cell binning for callers that cannot allocate device
memory where they bin (a framework that owns every device byte through its own
allocator, or a plugin that is handed only its input and output buffers).

It must give exactly what md_CellDistribution gives with caller scratch, on two calls
in a row (the fixed scratch array keeps the previous call's contents), also when some
particles lie outside the cell grid (both report RF_ERR_CELL_RANGE), leave the device's
free memory unchanged, and reject a grid larger than its fixed array. This file is
collected last on purpose."""
import numpy as np
import pytest

import rfdem

pytestmark = pytest.mark.gpu


def _with_scratch(torch, t, R, expect=rfdem.RF_OK):
    N, CN = R.size // 3, int(t.C.N)
    dR = torch.from_numpy(R).cuda()
    CI = torch.zeros(N, dtype=torch.int64, device="cuda")
    CIs = torch.zeros(2 * N, dtype=torch.int64, device="cuda")
    pnC = torch.zeros(2 * CN, dtype=torch.int64, device="cuda")
    sb = rfdem.lib.md_CellDistributionScratchBytes(N, CN)
    scratch = torch.zeros(sb, dtype=torch.uint8, device="cuda")
    st = rfdem.lib.md_CellDistribution(dR.data_ptr(), N, CI.data_ptr(), CIs.data_ptr(), pnC.data_ptr(), CN,
                                       t.C._1d_a, t.C.Nr, scratch.data_ptr(), sb, None)
    assert st == expect, rfdem.lib.rf_last_error_string()
    torch.cuda.synchronize()
    return CI.cpu().numpy(), CIs.cpu().numpy(), pnC.cpu().numpy()


def _no_alloc(torch, t, R, expect=rfdem.RF_OK, free_out=None):
    N, CN = R.size // 3, int(t.C.N)
    dR = torch.from_numpy(R).cuda()
    # output buffers filled with garbage: every element must be written by the call
    CI = torch.full((N,), -7, dtype=torch.int64, device="cuda")
    CIs = torch.full((2 * N,), -7, dtype=torch.int64, device="cuda")
    pnC = torch.full((2 * CN,), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = rfdem.lib.md_CellDistributionNoAlloc(dR.data_ptr(), N, CI.data_ptr(), CIs.data_ptr(), pnC.data_ptr(),
                                              CN, t.C._1d_a, t.C.Nr, None)
    torch.cuda.synchronize()
    if free_out is not None:
        free_out.append((free0, torch.cuda.mem_get_info()[0]))
    assert st == expect, rfdem.lib.rf_last_error_string()
    return CI.cpu().numpy(), CIs.cpu().numpy(), pnC.cpu().numpy()


def test_no_alloc_binning_matches_scratch_version_twice(cuda):
    # two different specimens, one after the other: the second call must not see the
    # first one's counters in the shared fixed array
    first = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 24.0, 40.0, seed=101)
    second = rfdem.make_test(rfdem.RF_TEST_BRAZIL, 30.0, 8.0, seed=102)
    for t, R in (first, second):
        want = _with_scratch(cuda, t, R)
        got = _no_alloc(cuda, t, R)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
        # the counts cover every particle once (one more when the reference's last-run
        # overrun applies)
        assert int(got[2][int(t.C.N):].sum()) in (R.size // 3, R.size // 3 + 1)


def test_no_alloc_rejects_grids_beyond_its_array(cuda):
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=103)
    N = R.size // 3
    big = rfdem.u3(128, 128, 64)            # 1,048,576 cells > 524,287
    CN = 128 * 128 * 64
    dR = cuda.from_numpy(R).cuda()
    CI = cuda.zeros(N, dtype=cuda.int64, device="cuda")
    CIs = cuda.zeros(2 * N, dtype=cuda.int64, device="cuda")
    pnC = cuda.zeros(2 * CN, dtype=cuda.int64, device="cuda")
    st = rfdem.lib.md_CellDistributionNoAlloc(dR.data_ptr(), N, CI.data_ptr(), CIs.data_ptr(), pnC.data_ptr(), CN,
                                              t.C._1d_a, big, None)
    assert st == rfdem.RF_ERR_INVALID
    assert b"fixed scratch limit" in rfdem.lib.rf_last_error_string()


def test_no_alloc_particles_outside_the_grid(cuda):
    """Particles outside the cell grid: one whose linear key lies past the grid (tail
    bin, sorted after every in-grid particle) and two whose x or y cell is past the
    grid while the key wraps into another row of it (binned under that key, as the
    reference's sort orders keys). Both entry points report RF_ERR_CELL_RANGE and write
    the oracle's keys, sorted ids and cell pointers."""
    import ctypes as C
    import oracle
    L = oracle.load()
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 12.0, 18.0, seed=104)
    N, CN = R.size // 3, int(t.C.N)
    R = R.copy()
    a = float(t.C.a)
    R[2 * N + (N - 3)] = a * (int(t.C.Nr.z) + 3)          # z past the grid: key >= CN
    R[0 * N + 5] = a * (int(t.C.Nr.x) + 1) + 0.25 * a     # x past the grid, key wraps
    R[1 * N + N // 2] = a * (int(t.C.Nr.y) + 1) + 0.25 * a
    CI, CIs, pnC = np.zeros(N, np.uint64), np.zeros(2 * N, np.uint64), np.zeros(2 * CN, np.uint64)
    st = L.rfo_cell_distribution_f(R.ctypes.data, N, CI.ctypes.data, CIs.ctypes.data, pnC.ctypes.data, CN,
                                   t.C._1d_a, t.C.Nr)
    assert st == rfdem.RF_ERR_CELL_RANGE
    want = (CI, CIs, pnC)
    assert int(CI[N - 3]) >= CN and int(CI[5]) < CN and int(CI[N // 2]) < CN
    for got in (_with_scratch(cuda, t, R, expect=rfdem.RF_ERR_CELL_RANGE),
                _no_alloc(cuda, t, R, expect=rfdem.RF_ERR_CELL_RANGE)):
        for g, w in zip(got, want):
            assert np.array_equal(g.view(np.uint64), w)
        assert int(got[1][2 * N - 1]) == N - 3              # the tail-bin particle sorts last
    # a clean specimen afterwards: the call clears the status the stray particles raised
    t2, R2 = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=105)
    for g, w in zip(_no_alloc(cuda, t2, R2), _with_scratch(cuda, t2, R2)):
        assert np.array_equal(g, w)


def test_no_alloc_leaves_free_device_memory_unchanged(cuda):
    t, R = rfdem.make_test(rfdem.RF_TEST_BRAZIL, 20.0, 6.0, seed=106)
    _no_alloc(cuda, t, R)                       # first call on this device: address look-up
    seen = []
    _no_alloc(cuda, t, R, free_out=seen)
    _no_alloc(cuda, t, R, free_out=seen)
    for before, after in seen:
        assert before == after
