"""Generate the golden fixtures of tests/test_golden.py by running the reference's OWN
kernels (oracle/_ref/libmdref_gpu.so: the reference's .cu sources compiled unmodified
for sm_100a, plus a thin harness) on seeded inputs. Needs a CUDA device and the built
reference library:

    python tests/golden/make_golden.py --out tests/golden

The inputs are not stored: tests/test_golden.py regenerates them with the same seeded
generator (rfdem.make_test) and checks the oracle against these outputs on the CPU.
"""
import argparse
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "rockfit-dem_b200"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np

import mdcall as mc
import oracle
import rfdem

CASES = {"uniaxial": (rfdem.RF_TEST_UNIAXIAL, 9.0, 14.0), "brazil": (rfdem.RF_TEST_BRAZIL, 16.0, 6.0)}
SEED = 0xB2000000 + 31
FORCE_STEPS, RUN_STEPS = 40, 200


def to32(a):
    out = a.astype(np.uint32)
    out[a == np.uint64(0xFFFFFFFFFFFFFFFF)] = np.uint32(0xFFFFFFFF)
    return out


def make(name, out_dir):
    REF = oracle.ref_gpu()
    assert REF is not None, "oracle/_ref/libmdref_gpu.so not built"
    kind, d, h = CASES[name]
    t, R = rfdem.make_test(kind, d, h, seed=SEED)
    N, K, CN = R.size // 3, int(t.K), int(t.C.N)
    g = {}
    CI, CIs, pnC = np.zeros(N, np.uint32), np.zeros(2 * N, np.uint32), np.zeros(2 * CN, np.uint32)
    assert REF.ref_cell_distribution(R.ctypes.data, N, CI.ctypes.data, CIs.ctypes.data, pnC.ctypes.data, CN, t.C.a,
                                     t.C._1d_a, t.C.Nr) == 0
    g.update(CI=CI, CIs=CIs, pnC=pnC)
    IL = np.zeros(N * K, np.uint32)
    assert REF.ref_list_construct(R.ctypes.data, N, K, CN, t.C.a, t.C._1d_a, t.aacut, t.C.Nr, IL.ctypes.data) == 0
    g["IL"] = IL.copy()
    ty, iL = np.zeros(N * K, np.uint8), np.zeros(N * K, np.float32)
    assert REF.ref_construct_bonds(R.ctypes.data, N, K, IL.ctypes.data, ty.ctypes.data, iL.ctypes.data,
                                   np.float32(t.Po.b_dd), np.float32(t.Po.b_r)) == 0
    g.update(bond_ty=ty, bond_iL=iL)
    # forces of one evaluation on the oracle's state after FORCE_STEPS steps, perturbed V, W
    _, st = mc.oracle_state_after(t, R, FORCE_STEPS)
    rng = np.random.default_rng(4)
    V = st["V"] + rng.normal(scale=2e-4, size=3 * N).astype(np.float32)
    W = st["W"] + rng.normal(scale=2e-3, size=3 * N).astype(np.float32)
    S = {k: st[k].copy() for k in ["Rij", "Oijt", "Mijn", "Mijt"]}
    ty_f = st["ILtype"].copy()
    F, M = np.zeros(3 * N, np.float32), np.zeros(3 * N, np.float32)
    p22 = np.array(mc.bond_params(t), np.float32)
    p21 = np.array(mc.contact_params(t), np.float32)
    IL32 = to32(st["IL"])                  # kept alive across the call
    assert REF.ref_forces(st["R"].ctypes.data, V.ctypes.data, W.ctypes.data, N, K, IL32.ctypes.data,
                          ty_f.ctypes.data, st["iL"].ctypes.data, S["Rij"].ctypes.data, S["Oijt"].ctypes.data,
                          S["Mijn"].ctypes.data, S["Mijt"].ctypes.data, F.ctypes.data, M.ctypes.data,
                          p22.ctypes.data, p21.ctypes.data, 3) == 0
    g.update(force_F=F, force_M=M, force_ty=ty_f, force_Oijt=S["Oijt"])
    # a whole run through the reference's driver sequence
    tr = mc.clone(t)
    o = dict(R=np.zeros(3 * N, np.float32), V=np.zeros(3 * N, np.float32), W=np.zeros(3 * N, np.float32),
             IL=np.zeros(N * K, np.uint32), ty=np.zeros(N * K, np.uint8), iL=np.zeros(N * K, np.float32),
             Rij=np.zeros(3 * N * K, np.float32), Oijt=np.zeros(3 * N * K, np.float32),
             Mijn=np.zeros(3 * N * K, np.float32), Mijt=np.zeros(3 * N * K, np.float32))
    curve = np.zeros(3 * RUN_STEPS, np.float64)
    ns = C.c_uint64(0)
    n = REF.ref_run(C.byref(tr), R.ctypes.data, RUN_STEPS, *[o[k].ctypes.data for k in
                                                            ["R", "V", "W", "IL", "ty", "iL", "Rij", "Oijt", "Mijn",
                                                             "Mijt"]], curve.ctypes.data, RUN_STEPS, C.byref(ns))
    assert n == RUN_STEPS
    g.update(run_R=o["R"], run_IL=o["IL"], run_ty=o["ty"], run_curve=curve)
    path = os.path.join(out_dir, "ref_%s.npz" % name)
    np.savez_compressed(path, **g)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for name in CASES:
        make(name, a.out)
