"""State files against the reference's own writers (compiled from its sources into the
oracle's reference build): the LAMMPS data text of SaveLammpsDATASimple and the binary
state dump of SaveAllData, byte for byte; and the dump's read-back."""
import ctypes as C
import os

import numpy as np
import pytest

import mdcall as mc
import oracle
import rfdem

REF_IO = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libmdref_io.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_IO), reason="reference build absent (oracle/build.py)")


def _state():
    t, R = rfdem.make_test(rfdem.RF_TEST_BRAZIL, 8.0, 3.0, seed=0xB2000000 + 31)
    N, K = int(t.N), int(t.K)
    steps, st, _, status = oracle.run_f(mc.clone(t), R, 3)
    rng = np.random.default_rng(5)
    st["V"] = rng.normal(size=3 * N).astype(np.float32) * 1e-3
    st["W"] = rng.normal(size=3 * N).astype(np.float32) * 1e-2
    return t, N, K, st


def _ids32(IL):
    return np.where(IL == np.iinfo(IL.dtype).max, np.uint32(0xFFFFFFFF), IL).astype(np.uint32)


@needs_ref
@pytest.mark.parametrize("flagv", [1, 0])
def test_lammps_text_matches_reference(tmp_path, flagv):
    t, N, K, st = _state()
    ours, ref = tmp_path / "ours.data", tmp_path / "ref.data"
    rfdem.save_lammps_data(str(ours), t, st, with_energy=bool(flagv))
    L = C.CDLL(REF_IO)
    P = C.c_void_p
    L.ref_save_lammps.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, P, P, P, P, P, P, P, C.c_double, C.c_double,
                                  C.c_double, C.c_int]
    A = np.array([t.S.A.x, t.S.A.y, t.S.A.z], np.float32)
    B = np.array([t.S.B.x, t.S.B.y, t.S.B.z], np.float32)
    IL32 = _ids32(st["IL"])
    arrs = [st["R"], st["V"], st["W"], IL32, st["ILtype"], A, B]
    assert L.ref_save_lammps(os.fsencode(str(ref)), N, K, *[a.ctypes.data for a in arrs], t.Po.dt, t.Po.p_m,
                             t.Po.p_I, flagv) == 0
    a, b = ours.read_bytes(), ref.read_bytes()
    assert a == b
    assert b"bonds" in a and int(np.count_nonzero((IL32 != 0xFFFFFFFF) & (st["ILtype"] == 1))) > 0


@needs_ref
def test_all_data_matches_reference_and_reads_back(tmp_path):
    import torch
    t, N, K, st = _state()
    rng = np.random.default_rng(9)
    NK = N * K
    extra = {k: rng.normal(size=3 * N).astype(np.float32) for k in ("F", "M")}
    extra["Q"] = rng.normal(size=4 * N).astype(np.float32)
    for k in ("Fijn", "Fijt", "Mijadd"):
        extra[k] = rng.normal(size=3 * NK).astype(np.float32)
    full = dict(st, **extra)
    pn = 12345
    ours = tmp_path / "ours.dat"
    rfdem.save_all_data(str(ours), t.S, full, N, K, t.acut, pn=pn, id_bytes=4)
    if not torch.cuda.is_available():
        # the reference's writer (its device copies fail without a GPU; the host arrays are written)
        d = tmp_path / "ref"
        (d / "result").mkdir(parents=True)
        L = C.CDLL(REF_IO)
        P = C.c_void_p
        L.ref_save_all.argtypes = [C.c_char_p, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float] + [P] * 10
        S = t.S
        sample = np.array([S.L.x, S.L.y, S.L.z, S.A.x, S.A.y, S.A.z, S.B.x, S.B.y, S.B.z, S.axis.x, S.axis.y,
                           S.axis.z, S.center.x, S.center.y, S.center.z, S.size.x, S.size.y, S.size.z, S.R0, S.H0,
                           S.Vgenmax], np.float32)
        slots = np.concatenate([full[k] for k in ("Rij", "Oijt", "Fijn", "Fijt", "Mijn", "Mijt", "Mijadd")])
        arrs = [full["F"], full["V"], full["R"], full["M"], full["W"], full["Q"], _ids32(full["IL"]), full["ILtype"],
                full["iL"], slots]
        assert L.ref_save_all(os.fsencode(str(d)), sample.ctypes.data, pn, N, K, t.acut,
                              *[np.ascontiguousarray(a).ctypes.data for a in arrs]) == 0
        assert ours.read_bytes() == (d / "result" / "DATA.dat").read_bytes()
    for id_bytes in (4, 8):
        path = tmp_path / ("rt%d.dat" % id_bytes)
        rfdem.save_all_data(str(path), t.S, full, N, K, t.acut, pn=pn, id_bytes=id_bytes)
        S2, pn2, ac2, n2, k2, back = rfdem.load_all_data(str(path), id_bytes=id_bytes)
        assert (n2, k2, ac2) == (N, K, t.acut)
        assert pn2 == (pn if id_bytes == 4 else 0)
        for key in back:
            assert np.array_equal(back[key], np.asarray(full[key]).astype(back[key].dtype)), key
        assert (S2.R0, S2.H0, S2.Vgenmax) == (t.S.R0, t.S.H0, t.S.Vgenmax)
        P3 = full["R"].reshape(3, N)
        assert S2.A_real.x == float(P3[0].min()) and S2.B_real.z == float(P3[2].max())


def test_state_file_error_paths(tmp_path):
    """Bad id widths, truncated dumps and files that are not checkpoints are refused with
    an error status (no GPU involved: restore reads and checks the header first)."""
    t, N, K, st = _state()
    with pytest.raises(rfdem.RFError):
        rfdem.save_all_data(str(tmp_path / "x.dat"), t.S, st, N, K, t.acut, id_bytes=5)
    good = tmp_path / "good.dat"
    rfdem.save_all_data(str(good), t.S, st, N, K, t.acut, id_bytes=4)
    data = good.read_bytes()
    cut = tmp_path / "cut.dat"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(rfdem.RFError):
        rfdem.load_all_data(str(cut), id_bytes=4)
    with pytest.raises(rfdem.RFError):
        rfdem.load_all_data(str(good), id_bytes=8)             # wrong width: counts do not match
    with pytest.raises(rfdem.RFError):
        rfdem.Engine.restore(str(good))                        # a dump, not a checkpoint
    with pytest.raises(rfdem.RFError):
        rfdem.Engine.restore(str(tmp_path / "missing.ckpt"))


def test_position_text_matches_the_reference_format(rfdem, tmp_path):
    """rf_save_positions_txt writes SaveParticleDATAtxt's text (md_createcylindersample.cu:104-114):
    the count, then x y z in metres -- float mm times the length unit 1e-3 as doubles in the
    stream's default format, which is C's %g at 6 significant digits -- and
    rf_load_positions_txt reads it back as LoadParticleDATAtxt does (x / 1e-3 to float)."""
    t, R = rfdem.make_test(rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0, seed=0xB2000000 + 61)
    n = R.size // 3
    path = tmp_path / "Sample_0.txt"
    rfdem.save_positions_txt(str(path), R)
    lines = [str(n)] + ["%g %g %g" % tuple(float(v) * 1e-3 for v in (R[i], R[i + n], R[i + 2 * n]))
                        for i in range(n)]
    assert path.read_text() == "\n".join(lines) + "\n"
    back = rfdem.load_positions_txt(str(path))
    want = np.array([float(w) for line in lines[1:] for w in line.split()], np.float64).reshape(n, 3).T
    assert np.array_equal(back, (want * (1.0 / 1e-3)).astype(np.float32).reshape(-1))
    # six digits: the round trip moves a coordinate by at most half a unit of the sixth digit
    assert np.max(np.abs(back - R) / np.maximum(np.abs(R), 1e-3)) < 5.1e-6
