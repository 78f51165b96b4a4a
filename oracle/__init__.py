"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes bindings of the CPU restatement (oracle/rf_oracle.cpp -> oracle/_build/liboracle.so)
and of the reference builds in oracle/_ref. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import this package; the engine never does.

Slot arrays use the reference layout: ids uint64 (uint_fast32_t on Linux), rows of K
slots per particle, per-slot vectors as float3 AoS.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libmdref_gpu.so")
REF_CPU_LIB = os.path.join(HERE, "_ref", "libmdref_cpu.so")
EMPTY64 = np.uint64(0xFFFFFFFFFFFFFFFF)
EMPTY32 = np.uint32(0xFFFFFFFF)

_lib = None


def load():
    """Load (building first if needed) the oracle library."""
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            from . import build
            build.build_oracle()
        _lib = C.CDLL(ORACLE_LIB)
        _declare(_lib)
    return _lib


def _declare(L):
    P, u64, f32, f64, i32 = C.c_void_p, C.c_uint64, C.c_float, C.c_double, C.c_int
    import rfdem
    u3, f3 = rfdem.u3, rfdem.f3
    T = C.POINTER(rfdem.Task)
    proto = {
        "rfo_cell_distribution_f": (i32, [P, u64, P, P, P, u64, f32, u3]),
        "rfo_construct_list_f": (i32, [P, u64, P, P, P, u64, f32, f32, f32, u3, u64]),
        "rfo_reconstruct_bpm_f": (i32, [P, u64, P, P, P, P, u64, f32, f32, f32, u3, u64]),
        "rfo_delete_far_links_f": (None, [P, u64, P, P, P, P, P, P, u64, f32]),
        "rfo_construct_bonds_f": (None, [P, u64, P, P, P, P, P, P, P, u64, f32]),
        "rfo_forces_22_f": (None, [P, P, P, P, P, P, P, P, P, P, P, P, u64, u64, f32, f32, f32, f32, f32, f32, P]),
        "rfo_forces_22_crit_f": (None, [P, P, P, P, P, P, P, P, P, P, P, P, u64, u64, f32, f32, f32, f32, f32, f32,
                                        P, P]),
        "rfo_forces_21_f": (None, [P, P, P, P, P, P, P, P, u64, u64, f32, f32, f32, f32, f32, f32, f32, f32]),
        "rfo_increments_f": (None, [P, P, P, P, P, u64, f32, f32, f32]),
        "rfo_brazil_platen_f": (None, [P, P, P, u64, f3, f32, f32, f32, f32, f32, f32, f32, P]),
        "rfo_uniaxial_platen_f": (None, [P, P, P, u64, f3, f32, f32, f32, f32, f32, f32, f32, P]),
        "rfo_cut_restriction_f": (None, [P, P, P, u64, f3, f3, f3]),
        "rfo_rsqrt_rn_array_f": (None, [P, P, u64]),
        "rfo_task_prepare": (i32, [T, P, P, f64, f64, f64, f64]),
        "rfo_compress": (None, [T, f64]),
        "rfo_sum_forces": (None, [T, f64, f64, f64]),
        "rfo_run_f": (u64, [T, P, u64, P, P, P, P, P, P, P, P, P, P, P, u64, P, P]),
        "rfo_run_d": (u64, [T, P, u64, P, P, u64, P, P, P]),
        "rfo_fire_increments_f": (None, [P, P, P, u64, f32, f32, f32]),
        "rfo_fire_half_f": (None, [P, P, u64, f32]),
        "rfo_fdotv_f": (f64, [P, P, u64]),
        "rfo_qs_ext_f": (i32, [T, C.POINTER(rfdem.ExtParams), P, P, C.POINTER(rfdem.RelaxParams), u64, P, P, P, P, P, u64]),
        "rfo_qs_ext_d": (i32, [T, C.POINTER(rfdem.ExtParams), P, P, C.POINTER(rfdem.RelaxParams), u64, P, P, P, P, P, u64]),
        "rfo_warm_probe_ext_d": (None, [T, C.POINTER(rfdem.ExtParams), P, P, C.POINTER(rfdem.RelaxParams), u64, u64, P]),
        "rfo_warm_probe_ext_f": (None, [T, C.POINTER(rfdem.ExtParams), P, P, C.POINTER(rfdem.RelaxParams), u64, u64, P,
                                        f64, f64]),
        "rfo_run_ext_f": (u64, [T, C.POINTER(rfdem.ExtParams), P, P, u64, P, P, P, P, u64, P, P, P]),
        "rfo_run_ext_pos_f": (u64, [T, C.POINTER(rfdem.ExtParams), P, P, u64, P, P, P, P, u64, P, P, P, i32]),
        "rfo_run_ext_d": (u64, [T, C.POINTER(rfdem.ExtParams), P, P, u64, P, P, P, P, u64, P, P, P]),
        "rfo_time_ext_f": (f64, [T, C.POINTER(rfdem.ExtParams), P, P, P, u64, i32, P]),
        "rfo_run_ext_strained_f": (u64, [T, C.POINTER(rfdem.ExtParams), P, P, P, u64, P, P, P, P, u64, P, P, P]),
    }
    for n, (r, a) in proto.items():
        f = getattr(L, n)
        f.restype = r
        f.argtypes = a


def p(a):
    return None if a is None else a.ctypes.data


def run_f(task, R0, max_steps):
    """Full FP32 run from positions R0 (planar); returns (steps, state dict, curve, status)."""
    L = load()
    N, K = int(task.N), int(task.K)
    st = dict(R=np.array(R0, np.float32, copy=True), V=np.zeros(3 * N, np.float32), W=np.zeros(3 * N, np.float32),
              IL=np.zeros(N * K, np.uint64), ILtype=np.zeros(N * K, np.uint8), iL=np.zeros(N * K, np.float32),
              Rij=np.zeros(3 * N * K, np.float32), Oijt=np.zeros(3 * N * K, np.float32),
              Mijn=np.zeros(3 * N * K, np.float32), Mijt=np.zeros(3 * N * K, np.float32),
              broke=np.zeros(N * K, np.uint8))
    cap = max(int(max_steps), 1) + 1
    curve = np.zeros(3 * cap, np.float64)
    ns = C.c_uint64(0)
    status = C.c_int(0)
    steps = L.rfo_run_f(C.byref(task), p(st["R"]), max_steps, p(st["V"]), p(st["W"]), p(st["IL"]), p(st["ILtype"]),
                        p(st["iL"]), p(st["Rij"]), p(st["Oijt"]), p(st["Mijn"]), p(st["Mijt"]), p(st["broke"]),
                        p(curve), cap, C.byref(ns), C.byref(status))
    return int(steps), st, curve[:3 * min(ns.value, cap)].reshape(-1, 3), status.value


def run_d(task, R0, max_steps):
    """Full FP64 run (the FP64 oracle); returns (steps, R double planar, curve, ILtype, status)."""
    L = load()
    N, K = int(task.N), int(task.K)
    R = np.zeros(3 * N, np.float64)
    ty = np.zeros(N * K, np.uint8)
    cap = max(int(max_steps), 1) + 1
    curve = np.zeros(3 * cap, np.float64)
    ns = C.c_uint64(0)
    status = C.c_int(0)
    steps = L.rfo_run_d(C.byref(task), p(np.ascontiguousarray(R0, np.float32)), max_steps, p(R), p(curve), cap,
                        C.byref(ns), p(ty), C.byref(status))
    return int(steps), R, curve[:3 * min(ns.value, cap)].reshape(-1, 3), ty, status.value


def run_ext(task, x, R0, radius, max_steps, fp64=False, positions="f64", strain=None):
    """Extended model run (float forces as the engine computes them, or the FP64 oracle;
    positions "hilo" / "f32": float forces with positions kept as hi/lo float pairs / floats;
    strain (float forces only): rf_engine_affine_strain applied to the built specimen first).
    Returns dict(steps, R (double planar, after the pending delete pass), V, IL, ILtype,
    curve, status, broken)."""
    L = load()
    N, K = int(task.N), int(task.K)
    R = np.array(R0, np.float64, copy=True)
    rad = np.ascontiguousarray(radius, np.float64)
    V = np.zeros(3 * N, np.float64 if fp64 else np.float32)
    IL = np.zeros(N * K, np.uint64)
    ty = np.zeros(N * K, np.uint8)
    cap = max(int(max_steps), 1) + 1
    curve = np.zeros(3 * cap, np.float64)
    ns, status, broken = C.c_uint64(0), C.c_int(0), C.c_uint64(0)
    args = [C.byref(task), C.byref(x), p(R), p(rad), max_steps, p(V), p(IL), p(ty), p(curve), cap, C.byref(ns),
            C.byref(status), C.byref(broken)]
    if strain is not None:
        sv = (C.c_double * 3)(*strain)
        steps = L.rfo_run_ext_strained_f(*(args[:4] + [sv] + args[4:]))
    elif positions != "f64" and not fp64:
        steps = L.rfo_run_ext_pos_f(*args, {"hilo": 1, "f32": 2}[positions])
    else:
        steps = (L.rfo_run_ext_d if fp64 else L.rfo_run_ext_f)(*args)
    return dict(steps=int(steps), R=R, V=V, IL=IL, ILtype=ty, curve=curve[:3 * min(ns.value, cap)].reshape(-1, 3),
                status=status.value, broken=int(broken.value))


def time_ext(task, x, R0, radius, steps, threads, strain=None):
    """Seconds of `steps` explicit steps of the extended model on `threads` host threads
    (bond construction and the pre-strain untimed); returns (seconds, steps done)."""
    L = load()
    R = np.ascontiguousarray(R0, np.float64)
    rad = np.ascontiguousarray(radius, np.float64)
    sv = None if strain is None else (C.c_double * 3)(*strain)
    done = C.c_uint64(0)
    secs = L.rfo_time_ext_f(C.byref(task), C.byref(x), p(R), p(rad), sv, steps, threads, C.byref(done))
    return secs, int(done.value)


def qs_ext(task, x, R0, radius, params, n_inc, fp64=False, trace_cap=0):
    """Quasi-static FIRE load increments of the extended model; returns dict(R, iters,
    converged, residual, stress, trace, status)."""
    L = load()
    R = np.array(R0, np.float64, copy=True)
    rad = np.ascontiguousarray(radius, np.float64)
    it = np.zeros(n_inc, np.uint64)
    cv = np.zeros(n_inc, np.int32)
    rs = np.zeros(n_inc, np.float64)
    st = np.zeros(n_inc, np.float64)
    tr = np.zeros(max(trace_cap, 1), np.float64)
    fn = L.rfo_qs_ext_d if fp64 else L.rfo_qs_ext_f
    status = fn(C.byref(task), C.byref(x), p(R), p(rad), C.byref(params), n_inc, p(it), p(cv), p(rs), p(st),
                p(tr) if trace_cap else None, trace_cap)
    return dict(R=R, iters=it, converged=cv, residual=rs, stress=st, trace=tr[:trace_cap], status=status)


def warm_probe(task, x, R0, radius, params, n_pre, warm_iters, fp64=True, scale=1.0, noise=0.0):
    """FP64 extended oracle: after n_pre plain FIRE increments, relax the next increment
    plainly and, from the same state, warm-started with that plain answer (displacements
    and rotations; fp64=False: float forces, the warm start scaled by scale + noise * U[-1, 1)
    per particle) for at most warm_iters iterations. Returns a dict of iterations,
    residuals, platen stresses and the largest bond-state differences between the two."""
    L = load()
    out = np.zeros(15, np.float64)
    args = [C.byref(task), C.byref(x), p(np.ascontiguousarray(R0, np.float64)),
            p(np.ascontiguousarray(radius, np.float64)), C.byref(params), n_pre, warm_iters, p(out)]
    if fp64:
        assert scale == 1.0 and noise == 0.0, "the FP64 probe warm-starts with the exact answer"
        L.rfo_warm_probe_ext_d(*args)
    else:
        L.rfo_warm_probe_ext_f(*args, scale, noise)
    keys = ["it_plain", "res_plain", "res_warm", "stress_plain", "stress_warm", "dOijt", "maxOijt", "dMijn", "maxMijn",
            "dMijt", "maxMijt", "dRij", "dx", "it_warm", "conv_warm"]
    return dict(zip(keys, out.tolist()))


def ref_gpu():
    """The reference's own kernels (oracle/_ref/libmdref_gpu.so), or None when not built."""
    if not os.path.exists(REF_GPU_LIB):
        return None
    L = C.CDLL(REF_GPU_LIB)
    P, u32, u64, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float
    import rfdem
    u3 = rfdem.u3
    L.ref_cell_distribution.argtypes = [P, u32, P, P, P, u32, f32, f32, u3]
    L.ref_list_construct.argtypes = [P, u32, u32, u32, f32, f32, f32, u3, P]
    L.ref_reconstruct_bpm.argtypes = [P, u32, u32, u32, f32, f32, f32, u3, P, P]
    L.ref_construct_bonds.argtypes = [P, u32, u32, P, P, P, f32, f32]
    L.ref_forces.argtypes = [P, P, P, u32, u32, P, P, P, P, P, P, P, P, P, P, P, C.c_int]
    L.ref_run.argtypes = [C.POINTER(rfdem.Task), P, u32, P, P, P, P, P, P, P, P, P, P, P, u64, P]
    L.ref_run.restype = C.c_longlong
    return L


def ref_cpu():
    """The reference's own CPU bond-force function (oracle/_ref/libmdref_cpu.so), or None."""
    if not os.path.exists(REF_CPU_LIB):
        return None
    L = C.CDLL(REF_CPU_LIB)
    P, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    L.ref_cpu_bond_forces.argtypes = [P, P, P, P, P, P, u32, u32, f32, f32, f32, f32, f32, f32, C.c_int, C.c_int, P]
    L.ref_cpu_bond_forces.restype = C.c_double
    L.ref_cpu_bond_forces_rb.argtypes = [P, P, P, P, P, P, u32, u32, f32, f32, f32, P, f32, f32, C.c_int, C.c_int,
                                         P]
    L.ref_cpu_bond_forces_rb.restype = C.c_double
    return L
