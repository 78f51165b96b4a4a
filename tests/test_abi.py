"""CPU checks of the C ABI: the library loads, exports what the header declares,
and its host-side reference arithmetic (parameter derivation, platen bookkeeping,
specimen generator) matches the oracle bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rockfit_b200.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:md|rf)_[A-Za-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(rfdem):
    names = header_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(rfdem.lib, n)]
    assert not missing, missing
    # every header function has a ctypes prototype in the Python mirror
    assert set(names) <= set(rfdem.ABI_SYMBOLS) | {"rf_stream"}, set(names) - set(rfdem.ABI_SYMBOLS)


def test_id_width_is_uint_fast32(rfdem):
    assert rfdem.lib.rf_id_bytes() == C.sizeof(C.c_size_t)   # glibc: uint_fast32_t is 8 bytes


def _fields(s, prefix=""):
    out = {}
    for name, typ in s._fields_:
        v = getattr(s, name)
        if isinstance(v, C.Structure):
            out.update(_fields(v, prefix + name + "."))
        else:
            out[prefix + name] = v
    return out


def _prepared(rfdem, oracle, kind, via_oracle):
    t = rfdem.Task()
    t.kind = kind
    t.K = 32
    t.N = 12345
    t.Po = rfdem.granite_potential()
    # the reference's own sample sizes (mp_determineconjgradient.cu:130-142), as float3 values
    f = np.float32
    if kind == rfdem.RF_TEST_UNIAXIAL:
        ls = [float(f(0.5 * 0.025)), float(f(0.5 * 0.025)), float(f(0.5 * 0.05))]
        ss = [float(f(0.04)), float(f(0.04)), float(f(0.06))]
        vl, ms = -10.0 * 0.02 / 1e3, 15e6 / 1e9
    else:
        ls = [float(f(0.5 * 0.05)), float(f(0.5 * 0.05)), float(f(0.5 * 0.02))]
        ss = [float(f(0.065)), float(f(0.065)), float(f(0.03))]
        vl, ms = -100.0 * 0.02 / 1e3, 2.1e6 / 1e9
    cell_a = float(np.float32(2.0 * t.Po.a_farcut))
    a_ss = (C.c_double * 3)(*ss)
    a_ls = (C.c_double * 3)(*ls)
    if via_oracle:
        assert oracle.load().rfo_task_prepare(C.byref(t), a_ss, a_ls, cell_a, vl, ms, 0.1) == 0
    else:
        rfdem.check(rfdem.lib.rf_task_prepare(C.byref(t), a_ss, a_ls, cell_a, vl, ms, 0.1))
    return t


@pytest.mark.parametrize("kind", [0, 1])
def test_task_prepare_matches_oracle(rfdem, oracle, kind):
    a = _fields(_prepared(rfdem, oracle, kind, False))
    b = _fields(_prepared(rfdem, oracle, kind, True))
    diff = {k: (a[k], b[k]) for k in a if not (a[k] == b[k] or (a[k] != a[k] and b[k] != b[k]))}
    assert not diff, diff


def test_task_prepare_reference_values(rfdem, oracle):
    t = _prepared(rfdem, oracle, rfdem.RF_TEST_UNIAXIAL, False)
    # hand-checked: dt = 0.1 * Rayleigh time for the granite parameters
    assert abs(t.Po.dt - 0.0312812265) < 1e-9
    assert (t.C.Nr.x, t.C.Nr.y, t.C.Nr.z) == (15, 15, 24)   # floor(42.929/2.9)+1, floor(62.929/2.9)+3
    assert abs(t.aacut - 2.1025) < 1e-6
    assert t.Compress.Size0 > 0 and t.Compress.Top > t.Compress.Bottom


@pytest.mark.parametrize("kind", [0, 1])
def test_compress_and_sum_forces_match_oracle(rfdem, oracle, kind):
    L = oracle.load()
    ta = _prepared(rfdem, oracle, kind, False)
    tb = _prepared(rfdem, oracle, kind, False)
    rng = np.random.default_rng(7)
    sz0 = float(ta.Compress.size.z)
    fl = np.zeros(8, np.float32)
    for step in range(300):
        s0, s1 = rng.normal(scale=1e-2, size=2) * (1 if step > 20 else 0)
        fl[:] = 0
        fl[0], fl[4] = np.float32(-abs(s0)), np.float32(abs(s1))
        rfdem.check(rfdem.lib.md_SumForcesULoading(C.byref(ta), fl.ctypes.data, 4, step, 1, sz0, None, None))
        L.rfo_sum_forces(C.byref(tb), float(fl[0]), float(fl[4]), sz0)
        (rfdem.lib.md_CompressB if kind else rfdem.lib.md_CompressU)(C.byref(ta), ta.Compress.Stress)
        L.rfo_compress(C.byref(tb), tb.Compress.Stress)
    assert _fields(ta) == _fields(tb)


def test_specimen_seeded_and_deterministic(rfdem):
    a = rfdem.specimen_positions(0, 1, 0.5, 10.0, 20.0, (20.0, 20.0, 20.0))
    b = rfdem.specimen_positions(0, 1, 0.5, 10.0, 20.0, (20.0, 20.0, 20.0))
    c = rfdem.specimen_positions(0, 2, 0.5, 10.0, 20.0, (20.0, 20.0, 20.0))
    assert a.size == b.size == c.size and a.size % 3 == 0
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    n = a.size // 3
    x, y, z = a[:n] - 20.0, a[n:2 * n] - 20.0, a[2 * n:] - 20.0
    assert np.all(np.hypot(x, y) <= 5.0) and np.all(np.abs(z) <= 10.0)


def test_engine_needs_device_and_fails_loudly(rfdem):
    """Without a GPU the engine refuses to run rather than falling back to the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 6.0, 8.0)
    with pytest.raises(rfdem.RFError) as ei:
        rfdem.Engine(t, R)
    assert ei.value.code in (rfdem.RF_ERR_CUDA, 7)
