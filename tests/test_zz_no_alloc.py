"""md_CellDistributionNoAlloc: cell binning for callers that cannot allocate device
memory where they bin (a framework that owns every device byte through its own
allocator, or a step loop that cannot afford cudaMalloc's implicit synchronisation).

It must give exactly what md_CellDistribution gives with caller scratch, on two calls
in a row (the fixed scratch array keeps the previous call's contents), and reject a
grid larger than its fixed array. This file is collected last on purpose."""
import numpy as np
import pytest

import rfdem

pytestmark = pytest.mark.gpu


def _with_scratch(torch, t, R):
    N, CN = R.size // 3, int(t.C.N)
    dR = torch.from_numpy(R).cuda()
    CI = torch.zeros(N, dtype=torch.int64, device="cuda")
    CIs = torch.zeros(2 * N, dtype=torch.int64, device="cuda")
    pnC = torch.zeros(2 * CN, dtype=torch.int64, device="cuda")
    sb = rfdem.lib.md_CellDistributionScratchBytes(N, CN)
    scratch = torch.zeros(sb, dtype=torch.uint8, device="cuda")
    rfdem.check(rfdem.lib.md_CellDistribution(dR.data_ptr(), N, CI.data_ptr(), CIs.data_ptr(), pnC.data_ptr(), CN,
                                              t.C._1d_a, t.C.Nr, scratch.data_ptr(), sb, None), "md_CellDistribution")
    torch.cuda.synchronize()
    return CI.cpu().numpy(), CIs.cpu().numpy(), pnC.cpu().numpy()


def _no_alloc(torch, t, R):
    N, CN = R.size // 3, int(t.C.N)
    dR = torch.from_numpy(R).cuda()
    # output buffers filled with garbage: every element must be written by the call
    CI = torch.full((N,), -7, dtype=torch.int64, device="cuda")
    CIs = torch.full((2 * N,), -7, dtype=torch.int64, device="cuda")
    pnC = torch.full((2 * CN,), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rfdem.check(rfdem.lib.md_CellDistributionNoAlloc(dR.data_ptr(), N, CI.data_ptr(), CIs.data_ptr(), pnC.data_ptr(),
                                                     CN, t.C._1d_a, t.C.Nr, None), "md_CellDistributionNoAlloc")
    torch.cuda.synchronize()
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
