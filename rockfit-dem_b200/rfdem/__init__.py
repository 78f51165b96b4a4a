"""Python host mirror of the rockfit-b200 C ABI (include/rockfit_b200.h).

The engine is the CUDA library ``rockfit-dem_b200/lib/librfdem.so``; this module
only binds it with ctypes. There is no CPU fallback: importing the module raises
if the library is missing, and every call raises ``RFError`` on a non-zero status.

Units are the reference's (md_phys_constants.h): mm, mg, us; stress in 1e9 Pa.
"""
import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RFDEM_LIBRARY") or os.path.join(os.path.dirname(_HERE), "lib", "librfdem.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("rockfit-b200 engine library not built: %s (run rockfit-dem_b200/build.py)" % LIB_PATH)
lib = C.CDLL(LIB_PATH)

STATUS = {0: "RF_OK", 1: "RF_ERR_INVALID", 2: "RF_ERR_CUDA", 3: "RF_ERR_ROW_OVERFLOW", 4: "RF_ERR_CELL_RANGE",
          5: "RF_ERR_NOT_CONVERGED", 6: "RF_ERR_CAPACITY", 7: "RF_ERR_NO_DEVICE", 8: "RF_ERR_STATE"}
RF_OK, RF_ERR_INVALID, RF_ERR_CUDA, RF_ERR_ROW_OVERFLOW, RF_ERR_CELL_RANGE = 0, 1, 2, 3, 4
RF_TEST_UNIAXIAL, RF_TEST_BRAZIL = 0, 1


class RFError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__("%s: %s (%s)" % (what, STATUS.get(code, code), lib.rf_last_error_string().decode()))


def check(code, what=""):
    if code != 0:
        raise RFError(code, what)
    return code


# --- structs (field for field with include/rockfit_b200.h) ------------------
class f3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class u3(C.Structure):
    _fields_ = [("x", C.c_uint), ("y", C.c_uint), ("z", C.c_uint)]


class d3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


_POT_IN = ["m_E", "m_nu", "m_Ec", "m_Gc", "m_ro", "b_r", "b_d", "p_r", "p_e", "p_mu", "p_mur", "a_farcut"]
_POT_OUT = ["m_G", "b_S", "p_V", "p_m", "b_dd", "p_1d_m", "p_I", "hm_E", "hm_G", "p_A", "aa_farcut", "Trayleigh",
            "Tsim", "dt", "D", "a", "_1d_a", "aa", "dt_d_m", "dt_d_I"]


class Potential(C.Structure):
    _fields_ = [(n, C.c_double) for n in _POT_IN + _POT_OUT]


class Sample(C.Structure):
    _fields_ = [("A_real", d3), ("B_real", d3), ("size_real", d3), ("center_real", d3), ("Vext", C.c_double)] + \
               [(n, f3) for n in ["L", "A", "B", "axis", "center", "size", "sized2", "hidenpoint", "spacesize",
                                  "spacesized2"]] + \
               [("R0", C.c_float), ("H0", C.c_float), ("Vgenmax", C.c_float)]


class Cells(C.Structure):
    _fields_ = [("Nr", u3), ("N", C.c_uint64), ("a", C.c_float), ("_1d_a", C.c_float), ("_1d_Nr", f3)]


class Compression(C.Structure):
    _fields_ = [("Loading", C.c_int32), ("Fracture", C.c_int32), ("center", f3), ("size", f3), ("sized2", f3),
                ("size_d", d3), ("center_d", d3)] + \
               [(n, C.c_float) for n in ["R", "RR", "Hd2", "C", "mu", "Area", "_1d_Area"]] + \
               [(n, C.c_double) for n in ["V", "VLoad", "Top", "Bottom", "TopR", "BottomR", "FractureStress",
                                          "FractureStrain", "MinStress", "ZeroStress", "Stress", "Strain",
                                          "MaxStrain", "Size0"]]


class Task(C.Structure):
    _fields_ = [("kind", C.c_int), ("N", C.c_uint64), ("K", C.c_uint32), ("acut", C.c_float), ("aacut", C.c_float),
                ("Po", Potential), ("S", Sample), ("C", Cells), ("Compress", Compression), ("bloks", C.c_uint64),
                ("sz0", C.c_double)]


class RunResult(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("FractureStress", C.c_double), ("FractureStrain", C.c_double),
                ("Stress", C.c_double), ("Strain", C.c_double), ("Fracture", C.c_int32),
                ("broken_bonds", C.c_uint64), ("bonds_initial", C.c_uint64), ("error", C.c_int)]


RF_EPI_RELU_BF16, RF_EPI_LINEAR_F32, RF_EPI_MASK_BF16, RF_EPI_ATOMIC_F32 = 0, 1, 2, 3


class Fire(C.Structure):
    """rf_fire: firerelax_data without its buffers."""
    _fields_ = [(n, C.c_uint64) for n in ("bloks4", "NPpositiveMax", "NPnegativeMax", "NPpositive", "NPnegative",
                                          "Ndelay", "MaxStepsRelaxation")] + \
               [(n, C.c_float) for n in ("dtmax", "dtmin", "dt0", "dt", "alpha0", "alpha", "dtgrow", "dtshrink",
                                         "alphashrink")] + [("FdotV", C.c_double)]


class ExtParams(C.Structure):
    """rf_ext_params: bond constants and strength distribution of the extended model."""
    _fields_ = [("kn", C.c_double), ("ks", C.c_double), ("bond_lambda", C.c_double), ("gap_frac", C.c_double),
                ("weibull_m", C.c_double), ("sigma_c", C.c_double), ("tau_c", C.c_double), ("seed", C.c_uint64),
                ("post_peak_drop", C.c_double), ("list_gap", C.c_double), ("ref_mode", C.c_int32),
                ("reserved", C.c_int32)]


class RelaxParams(C.Structure):
    _fields_ = [("strain_inc", C.c_double), ("tol", C.c_double), ("dt0", C.c_double), ("dt_max", C.c_double),
                ("dt_min", C.c_double), ("alpha0", C.c_double), ("f_inc", C.c_double), ("f_dec", C.c_double),
                ("f_alpha", C.c_double), ("n_delay", C.c_uint32), ("max_iter", C.c_uint64)]


class RelaxResult(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("converged", C.c_int32), ("residual", C.c_double),
                ("mean_force", C.c_double), ("stress", C.c_double), ("strain", C.c_double),
                ("broken_bonds", C.c_uint64), ("error", C.c_int)]


# --- prototypes ---------------------------------------------------------------
P = C.c_void_p
ID = C.c_uint64 if lib.rf_id_bytes() == 8 else C.c_uint32     # uint_fast32_t
ID_NP = np.uint64 if lib.rf_id_bytes() == 8 else np.uint32
EMPTY = np.iinfo(ID_NP).max
u64, f32, f64, i32 = C.c_uint64, C.c_float, C.c_double, C.c_int
_proto = {
    "rf_last_error_string": (C.c_char_p, []),
    "rf_version": (i32, []), "rf_id_bytes": (i32, []),
    "rf_task_prepare": (i32, [C.POINTER(Task), P, P, f64, f64, f64, f64]),
    "md_CompressU": (i32, [C.POINTER(Task), f64]), "md_CompressB": (i32, [C.POINTER(Task), f64]),
    "md_SumForcesULoading": (i32, [C.POINTER(Task), P, u64, u64, u64, f64, P, P]),
    "md_CalculateCellIndex": (i32, [P, ID, P, f32, u3, P]),
    "md_CellDistributionScratchBytes": (C.c_size_t, [ID, ID]),
    "md_CellDistribution": (i32, [P, ID, P, P, P, ID, f32, u3, P, C.c_size_t, P]),
    "md_CellDistributionNoAlloc": (i32, [P, ID, P, P, P, ID, f32, u3, P]),
    "md_InteractionListConstruct": (i32, [P, ID, P, P, P, ID, f32, f32, f32, u3, ID, P]),
    "md_InteractionListReConstructBPM": (i32, [P, ID, P, P, P, P, ID, f32, f32, f32, u3, ID, P]),
    "md_DeleteFarLinks": (i32, [P, ID, P, P, P, P, P, P, P, P, P, P, ID, f32, P]),
    "md_ConstructBoundInteractions": (i32, [P, P, P, P, P, P, P, P, P, P, P, P, P, ID, ID, f32, f32, P]),
    "md_CalculateForcesDEM_22": (i32, [P, P, P, P, P, P, P, P, P, P, P, P, ID, ID, f32, f32, f32, f32, f32, f32, P]),
    "md_CalculateForcesDEM_21": (i32, [P, P, P, P, P, P, P, P, P, P, ID, ID, f32, f32, f32, f32, f32, f32, f32, f32, P]),
    "md_CalculateIncrementsDEM": (i32, [P, P, P, P, P, ID, f32, f32, f32, P]),
    "md_braziltest_simple2": (i32, [P, P, P, P, ID, f3, f32, f32, f32, f32, f32, f32, f32, u64, P]),
    "md_UniaxialCompression3_simple": (i32, [P, P, P, P, ID, f3, f32, f32, f32, f32, f32, f32, f32, u64, P]),
    "md_ParallelepipedCutRestriction": (i32, [P, P, P, ID, f3, f3, f3, P]),
    "md_CalculateIncrementsFIRE": (i32, [P, P, P, ID, f32, f32, f32, P]),
    "md_CalculateDecrementsHalfStepFIRE": (i32, [P, P, ID, f32, P]),
    "md_FdotVEntire": (i32, [P, P, P, u64, ID, P]),
    "md_SetFIREData": (i32, [C.POINTER(Fire), ID, C.POINTER(Potential)]),
    "md_FireDecide": (i32, [C.POINTER(Fire), f64, u64, C.POINTER(i32), C.POINTER(i32)]),
    "md_CalculationBrazilTest": (i32, [C.POINTER(Task), P, u64, P, u64, P, C.POINTER(RunResult)]),
    "md_CalculationUniaxialCompression": (i32, [C.POINTER(Task), P, u64, P, u64, P, C.POINTER(RunResult)]),
    "rf_engine_create": (i32, [C.POINTER(Task), P, C.POINTER(P)]),
    "rf_engine_destroy": (i32, [P]),
    "rf_engine_step": (i32, [P, u64]),
    "rf_engine_affine_strain": (i32, [P, C.POINTER(C.c_double)]),
    "rf_save_positions_txt": (i32, [C.c_char_p, P, u64]),
    "rf_load_positions_txt": (i32, [C.c_char_p, P, u64, C.POINTER(u64)]),
    "rf_engine_step_host": (i32, [P, P, u64, P]),
    "rf_engine_sync": (i32, [P, C.POINTER(Task), C.POINTER(RunResult)]),
    "rf_engine_export": (i32, [P] + [P] * 10),
    "rf_save_all_data": (i32, [C.c_char_p, i32, C.POINTER(Sample), u64, u64, C.c_uint32, f32] + [P] * 16),
    "rf_load_all_data": (i32, [C.c_char_p, i32, C.POINTER(Sample), P, P, P, P] + [P] * 16),
    "rf_save_lammps_data": (i32, [C.c_char_p, C.POINTER(Task), u64, C.c_uint32, P, P, P, P, P, i32]),
    "rf_engine_checkpoint": (i32, [P, C.c_char_p]),
    "rf_engine_restore": (i32, [C.c_char_p, P]),
    "rf_engine_import": (i32, [P] + [P] * 10),
    "rf_engine_curve": (i32, [P, P, u64, P]),
    "rf_engine_counters": (i32, [P, P, i32]),
    "rf_engine_launches_per_step": (i32, []),
    "rf_engine_stream": (P, [P]),
    "rf_engine_uses_graph": (i32, [P]),
    "rf_engine_create_ext": (i32, [C.POINTER(Task), C.POINTER(ExtParams), P, P, C.POINTER(P)]),
    "rf_engine_positions_f64": (i32, [P, P]),
    "rf_engine_autotune": (i32, [P, i32, C.POINTER(i32), P]),
    "rf_engine_create_batch": (i32, [C.POINTER(Task), C.POINTER(ExtParams), P, P, i32, C.POINTER(P)]),
    "rf_engine_batch_size": (i32, [P]),
    "rf_engine_spec_info": (i32, [P, i32, P, P, P, C.POINTER(Task)]),
    "rf_engine_sync_spec": (i32, [P, i32, C.POINTER(Task), C.POINTER(RunResult)]),
    "rf_engine_curve_spec": (i32, [P, i32, P, u64, P]),
    "rf_relax_default_params": (i32, [C.POINTER(RelaxParams), C.POINTER(Task)]),
    "rf_engine_load_increment": (i32, [P, C.POINTER(RelaxParams), P, C.POINTER(RelaxResult)]),
    "rf_engine_increment_fields": (i32, [P, P, P, P]),
    "rf_pack_cylinder": (i32, [u64, u64, f64, f64, f64, f64, f64, P, P, P, P, P, P]),
    "rf_pack_cylinder_dist": (i32, [u64, u64, f64, f64, f64, i32, f64, f64, P, P, P, P, P, P]),
    "rf_gemm_bf16": (i32, [P, i32, P, i32, i32, i32, i32, i32, P, P, i32, P, i32, P, i32, P, i32, i32, f32, i32, P]),
    "rf_gemm_status": (i32, [P]),
    "rf_mlp_create": (i32, [u64, C.POINTER(P)]),
    "rf_mlp_destroy": (i32, [P]),
    "rf_mlp_stream": (P, [P]),
    "rf_mlp_forward": (i32, [P, P, i32, P, i32, i32]),
    "rf_mlp_train_step": (i32, [P, P, P, i32, f32, C.POINTER(C.c_double)]),
    "rf_mlp_get": (i32, [P, i32, P, P]),
    "rf_mlp_set_residual": (i32, [P, i32]),
    "rf_mlp_set": (i32, [P, i32, P, P]),
    "rf_mlp_grad": (i32, [P, i32, P, P]),
    "rf_engine_warm_features": (i32, [P, f64, P]),
    "rf_engine_warm_targets": (i32, [P, f64, P]),
    "rf_engine_load_increment_pred": (i32, [P, C.POINTER(RelaxParams), P, i32, C.POINTER(RelaxResult)]),
    "rf_engine_load_increment_batch": (i32, [P, C.POINTER(RelaxParams), P, i32, i32, C.POINTER(RelaxResult)]),
    "rf_specimen_lattice_cylinder": (i32, [u64, f64, f64, f64, f64, f64, P, P, u64, P]),
    "rf_specimen_lattice_disc": (i32, [u64, f64, f64, f64, f64, f64, P, P, u64, P]),
}
for _n, (_r, _a) in _proto.items():
    _f = getattr(lib, _n)
    _f.restype = _r
    _f.argtypes = _a

ABI_SYMBOLS = sorted(_proto)


def ptr(a):
    """Address of a numpy array, a torch tensor, or None."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


# --- reference parameter presets ----------------------------------------------
LENGTH = 1e-3          # md_phys_constants.h: length_const
STRESS = 1e9           # force_const / length_const^2 with force_const = 1e3


def granite_potential():
    """The reference's granite start point (mp_determineconjgradient.cu:15-38, :123-127), mm-mg-us units."""
    po = Potential()
    po.m_nu = 0.247
    po.m_E = 1.95255e+11 / STRESS
    po.m_Ec = 5.1447e+08 / STRESS
    po.m_Gc = 3.7131e+08 / STRESS
    po.m_ro = 2610 / 1e3
    po.b_r = 0.5 * 0.000330015 / LENGTH
    po.p_r = 0.5 * 0.001 / LENGTH
    po.b_d = 2.0 * po.p_r + 5.93169e-05 / LENGTH
    po.p_e = 0.6
    po.p_mu = 0.45
    po.p_mur = 0.05
    po.a_farcut = 2.9 * po.p_r
    return po


def specimen_positions(kind, seed, p_r, diameter, height, center, gap_frac=0.02, jitter=0.02):
    """Seeded jittered-lattice specimen (cylinder, or Brazilian disc with axis z), planar float32[3N]."""
    fn = lib.rf_specimen_lattice_disc if kind == RF_TEST_BRAZIL else lib.rf_specimen_lattice_cylinder
    c = (C.c_double * 3)(*center)
    n = C.c_uint64(0)
    check(fn(seed, p_r, gap_frac, jitter, diameter, height, c, None, 0, C.byref(n)), "specimen")
    R = np.zeros(3 * n.value, np.float32)
    check(fn(seed, p_r, gap_frac, jitter, diameter, height, c, R.ctypes.data, n.value, C.byref(n)), "specimen")
    return R


def lattice_extent(p_r, gap_frac, size):
    """Particle-centre half extent the lattice generator realises for a specimen dimension."""
    sp = 2.0 * p_r * (1.0 + gap_frac)
    return math.floor((0.5 * size - p_r) / sp) * sp


def make_test(kind, diameter, height, seed=0xB2000000, potential=None, K=32, gap_frac=0.02, jitter=0.02,
              margin=None, v_load=None, min_stress=None, max_strain=0.1):
    """A prepared task plus its seeded specimen: returns (Task, R planar float32).

    kind: RF_TEST_UNIAXIAL (cylinder along z, platens on z) or RF_TEST_BRAZIL (disc of
    thickness `height` along z, platens on y). Sizes in mm. Defaults follow the
    reference's CG driver (mp_determineconjgradient.cu:79-80, :97-98).
    """
    po = potential or granite_potential()
    p_r = po.p_r
    ext_r = lattice_extent(p_r, gap_frac, diameter)
    ext_z = lattice_extent(p_r, gap_frac, height)
    # SetLSi takes the specimen size + 2 p_r and stores particle-centre extents L
    # the platens start at the outermost particle centre (lattice extent + jitter)
    L = [2 * ext_r + 2 * jitter * p_r, 2 * ext_r + 2 * jitter * p_r, 2 * ext_z + 2 * jitter * p_r]
    if margin is None:
        margin = 4.0 * p_r + 0.25 * max(L)
    space = [L[0] + 2 * p_r + 2 * margin, L[1] + 2 * p_r + 2 * margin, L[2] + 2 * p_r + 2 * margin]
    t = Task()
    t.kind = kind
    t.K = K
    t.Po = po
    if v_load is None:
        v_load = (-10.0 if kind == RF_TEST_UNIAXIAL else -100.0) * 0.02 / 1e3
    if min_stress is None:
        min_stress = (15e6 if kind == RF_TEST_UNIAXIAL else 2.1e6) / STRESS
    ss = (C.c_double * 3)(*[s * LENGTH for s in space])
    ls = (C.c_double * 3)(*[(x + 2 * p_r) * LENGTH for x in L])
    t.N = 1
    check(lib.rf_task_prepare(C.byref(t), ss, ls, 2.0 * po.a_farcut, v_load, min_stress, max_strain), "rf_task_prepare")
    ctr = (t.S.center.x, t.S.center.y, t.S.center.z)
    R = specimen_positions(kind, seed, p_r, diameter, height, ctr, gap_frac, jitter)
    t.N = R.size // 3
    t.bloks = t.N // 1024 + 1
    return t, R


# --- extended model: packed polydisperse specimens ------------------------------
RF_RADII_UNIFORM, RF_RADII_LOG_UNIFORM = 0, 1


def pack_cylinder(N, r0, rmin=0.8, rmax=1.2, aspect=2.0, phi=0.6, seed=0xB2000000, center=(0.0, 0.0, 0.0),
                  dist="uniform"):
    """Seeded FIRE packing on the GPU (rf_pack_cylinder_dist); radii r0 * U[rmin, rmax]
    (dist "uniform") or log-uniform on [rmin, rmax] * r0 ("log-uniform"). Returns
    (R float64[3N] planar, radius float64[N], diameter, height, max relative overlap);
    sizes in mm."""
    kinds = {"uniform": RF_RADII_UNIFORM, "log-uniform": RF_RADII_LOG_UNIFORM}
    R = np.zeros(3 * N, np.float64)
    rad = np.zeros(N, np.float64)
    D, H, mo = C.c_double(0), C.c_double(0), C.c_double(0)
    c = (C.c_double * 3)(*center)
    check(lib.rf_pack_cylinder_dist(seed, N, r0, rmin, rmax, kinds[dist], aspect, phi, c, R.ctypes.data,
                                    rad.ctypes.data, C.byref(D), C.byref(H), C.byref(mo)), "rf_pack_cylinder_dist")
    return R, rad, D.value, H.value, mo.value


def ext_params_si(kn=1e11, ks=None, bond_lambda=0.330015, gap_frac=0.05, weibull_m=5.0, sigma_c=10e6, tau_c=30e6,
                  seed=0xB2000000):
    """rf_ext_params from SI values: kn, ks in N/m^3 (ks defaults to kn/2.5), strengths in Pa.
    bond_lambda defaults to the reference's b_r / p_r."""
    x = ExtParams()
    x.kn = kn / (STRESS / LENGTH)
    x.ks = (ks if ks is not None else kn / 2.5) / (STRESS / LENGTH)
    x.bond_lambda = bond_lambda
    x.gap_frac = gap_frac
    x.weibull_m = weibull_m
    x.sigma_c = sigma_c / STRESS
    x.tau_c = tau_c / STRESS
    x.seed = seed
    return x


def make_test_ext(kind, R0, radius, r0, K=32, potential=None, margin=None, v_load=None, min_stress=None,
                  max_strain=0.1, dt=None):
    """A prepared task for a packed specimen (kind as make_test: uniaxial along z, or
    Brazilian disc of axis z loaded along y). The particle-centre box is centred on the
    task's centre, so the platens start on the outermost particles. Returns (Task, R).
    dt (microseconds) overrides the derived step."""
    po = potential or granite_potential()
    po.p_r = r0
    po.b_r = 0.330015 * r0
    po.b_d = 2.0 * r0 + 0.0593169 * r0 * 2.0
    # the reference's list and delete cutoff, widened just past the largest contact
    # distance 2 r_max where that reaches it (radius ratios above 2.4)
    po.a_farcut = max(2.9 * r0, 2.02 * float(np.max(radius)))
    N = radius.size
    P3 = R0.reshape(3, N).copy()
    # the platens act on the particle surfaces (centre +- (radius - r0)): box the specimen
    # by those coordinates, centred on the task's centre, so the platens start touching it
    off = np.asarray(radius, np.float64) - r0
    hi = (P3 + off[None, :]).max(axis=1)
    lo = (P3 - off[None, :]).min(axis=1)
    P3 -= (0.5 * (hi + lo))[:, None]
    L = [float(hi[a] - lo[a]) for a in range(3)]
    if margin is None:
        margin = 4.0 * r0 + 0.25 * max(L)
    space = [x + 2 * r0 + 2 * margin for x in L]
    t = Task()
    t.kind = kind
    t.K = K
    t.Po = po
    if v_load is None:
        v_load = (-10.0 if kind == RF_TEST_UNIAXIAL else -100.0) * 0.02 / 1e3
    if min_stress is None:
        min_stress = (15e6 if kind == RF_TEST_UNIAXIAL else 2.1e6) / STRESS
    ss = (C.c_double * 3)(*[x * LENGTH for x in space])
    ls = (C.c_double * 3)(*[(x + 2 * r0) * LENGTH for x in L])
    t.N = N
    check(lib.rf_task_prepare(C.byref(t), ss, ls, 2.0 * po.a_farcut, v_load, min_stress, max_strain), "rf_task_prepare")
    if dt is not None:
        t.Po.dt = dt
    ctr = np.array([t.S.center.x, t.S.center.y, t.S.center.z], np.float64)
    R = (P3 + ctr[:, None]).reshape(-1).copy()
    t.bloks = N // 1024 + 1
    return t, R


class Engine:
    """The fused engine on the current CUDA device."""

    @classmethod
    def restore(cls, path):
        """An engine from a checkpoint file (rf_engine_restore) continuing the saved run."""
        h = P()
        check(lib.rf_engine_restore(os.fsencode(path), C.byref(h)), "rf_engine_restore")
        e = cls.__new__(cls)
        e.h = h
        e.ext = False
        t, _ = e.sync()
        e.task, e.N, e.K = t, int(t.N), int(t.K)
        return e

    def checkpoint(self, path):
        """Write a checkpoint file (rf_engine_checkpoint)."""
        check(lib.rf_engine_checkpoint(self.h, os.fsencode(path)), "rf_engine_checkpoint")

    def __init__(self, task, R, ext=None, radius=None):
        self.task = task
        self.N = int(task.N)
        self.K = int(task.K)
        self.ext = ext is not None
        h = P()
        if self.ext:
            R = np.ascontiguousarray(R, np.float64)
            rad = np.ascontiguousarray(radius, np.float64)
            assert R.size == 3 * self.N and rad.size == self.N
            check(lib.rf_engine_create_ext(C.byref(task), C.byref(ext), R.ctypes.data, rad.ctypes.data, C.byref(h)),
                  "rf_engine_create_ext")
        else:
            R = np.ascontiguousarray(R, np.float32)
            assert R.size == 3 * self.N
            check(lib.rf_engine_create(C.byref(task), R.ctypes.data, C.byref(h)), "rf_engine_create")
        self.h = h

    def relax_params(self, **kw):
        p = RelaxParams()
        check(lib.rf_relax_default_params(C.byref(p), C.byref(self.task)), "rf_relax_default_params")
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    def load_increment(self, params, warm=None):
        """One quasi-static load increment; warm: device tensor float32 [N, 6] or None."""
        r = RelaxResult()
        check(lib.rf_engine_load_increment(self.h, C.byref(params), ptr(warm), C.byref(r)), "rf_engine_load_increment")
        return r

    def increment_fields(self):
        x0, dx, rot = (np.zeros((self.N, 3), np.float64) for _ in range(3))
        check(lib.rf_engine_increment_fields(self.h, x0.ctypes.data, dx.ctypes.data, rot.ctypes.data),
              "rf_engine_increment_fields")
        return x0, dx, rot

    def warm_features(self, strain_inc, out):
        """Features for the next increment into a device bf16 tensor [rows, 64]."""
        check(lib.rf_engine_warm_features(self.h, strain_inc, ptr(out)), "rf_engine_warm_features")

    def warm_targets(self, strain_inc, out):
        check(lib.rf_engine_warm_targets(self.h, strain_inc, ptr(out)), "rf_engine_warm_targets")

    def load_increment_pred(self, params, pred, ldp=16):
        r = RelaxResult()
        check(lib.rf_engine_load_increment_pred(self.h, C.byref(params), ptr(pred), ldp, C.byref(r)),
              "rf_engine_load_increment_pred")
        return r

    def autotune(self, steps=200):
        """Pick the fastest compiled step-kernel variant (state restored afterwards);
        returns (CTAs per SM of the pick, [ms for 8, 6, 5])."""
        ch = C.c_int(0)
        ms = np.zeros(3, np.float32)
        check(lib.rf_engine_autotune(self.h, steps, C.byref(ch), ms.ctypes.data), "rf_engine_autotune")
        return ch.value, ms.tolist()

    def positions_f64(self):
        R = np.zeros(3 * self.N, np.float64)
        check(lib.rf_engine_positions_f64(self.h, R.ctypes.data), "rf_engine_positions_f64")
        return R

    def close(self):
        if self.h:
            lib.rf_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n):
        check(lib.rf_engine_step(self.h, n), "rf_engine_step")

    def affine_strain(self, ex, ey, ez):
        """Homogeneous strain of the specimen about the platen box's centre (platens move with it)."""
        a = (C.c_double * 3)(ex, ey, ez)
        check(lib.rf_engine_affine_strain(self.h, a), "rf_engine_affine_strain")

    def step_host(self, R_in, n, R_out):
        check(lib.rf_engine_step_host(self.h, ptr(R_in), n, ptr(R_out)), "rf_engine_step_host")

    def sync(self):
        t = Task()
        r = RunResult()
        check(lib.rf_engine_sync(self.h, C.byref(t), C.byref(r)), "rf_engine_sync")
        return t, r

    def export(self):
        N, K = self.N, self.K
        out = dict(R=np.zeros(3 * N, np.float32), V=np.zeros(3 * N, np.float32), W=np.zeros(3 * N, np.float32),
                   IL=np.zeros(N * K, ID_NP), ILtype=np.zeros(N * K, np.uint8), iL=np.zeros(N * K, np.float32),
                   Rij=np.zeros(3 * N * K, np.float32), Oijt=np.zeros(3 * N * K, np.float32),
                   Mijn=np.zeros(3 * N * K, np.float32), Mijt=np.zeros(3 * N * K, np.float32))
        check(lib.rf_engine_export(self.h, *[ptr(out[k]) for k in
                                             ["R", "V", "W", "IL", "ILtype", "iL", "Rij", "Oijt", "Mijn", "Mijt"]]),
              "rf_engine_export")
        return out

    def load(self, st):
        check(lib.rf_engine_import(self.h, *[ptr(np.ascontiguousarray(st[k])) for k in
                                             ["R", "V", "W", "IL", "ILtype", "iL", "Rij", "Oijt", "Mijn", "Mijt"]]),
              "rf_engine_import")

    def curve(self):
        n = C.c_uint64(0)
        check(lib.rf_engine_curve(self.h, None, 0, C.byref(n)), "rf_engine_curve")
        m = min(n.value, 1 << 20)
        buf = np.zeros(3 * max(m, 1), np.float64)
        check(lib.rf_engine_curve(self.h, buf.ctypes.data, m, C.byref(n)), "rf_engine_curve")
        return buf[:3 * m].reshape(m, 3)

    def stream(self):
        return lib.rf_engine_stream(self.h)

    def uses_graph(self):
        return bool(lib.rf_engine_uses_graph(self.h))

    def counters(self):
        out = np.zeros(5, np.uint64)
        check(lib.rf_engine_counters(self.h, out.ctypes.data, 5), "rf_engine_counters")
        return dict(steps=int(out[0]), rebuilds=int(out[1]), bonds=int(out[2]), contacts=int(out[3]),
                    occupied=int(out[4]))


def run_test(task, R, max_steps=0, curve_cap=0, want_positions=False):
    """md_CalculationBrazilTest / md_CalculationUniaxialCompression from host buffers."""
    R = np.ascontiguousarray(R, np.float32)
    curve = np.zeros(3 * max(curve_cap, 1), np.float64)
    Rout = np.zeros_like(R) if want_positions else None
    res = RunResult()
    fn = lib.md_CalculationBrazilTest if task.kind == RF_TEST_BRAZIL else lib.md_CalculationUniaxialCompression
    check(fn(C.byref(task), R.ctypes.data, max_steps, curve.ctypes.data if curve_cap else None, curve_cap,
             ptr(Rout), C.byref(res)), "md_Calculation")
    return res, curve[:3 * curve_cap].reshape(-1, 3), Rout


MLP_DIN = (64, 128, 128, 128)
MLP_DOUT = (128, 128, 128, 16)


class MLP:
    """The warm-start MLP (rf_mlp_*) on the current CUDA device."""

    def __init__(self, seed=0xB2000000):
        h = P()
        check(lib.rf_mlp_create(seed, C.byref(h)), "rf_mlp_create")
        self.h = h

    def close(self):
        if self.h:
            lib.rf_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_residual(self, on=True):
        check(lib.rf_mlp_set_residual(self.h, 1 if on else 0), "rf_mlp_set_residual")

    def forward(self, X, rows, Y, ldy=16, ncols=16):
        check(lib.rf_mlp_forward(self.h, ptr(X), rows, ptr(Y), ldy, ncols), "rf_mlp_forward")

    def train_step(self, X, T, rows, lr):
        loss = C.c_double(0)
        check(lib.rf_mlp_train_step(self.h, ptr(X), ptr(T), rows, lr, C.byref(loss)), "rf_mlp_train_step")
        return loss.value

    def weights(self):
        out = []
        for l in range(4):
            W = np.zeros((MLP_DOUT[l], MLP_DIN[l]), np.float32)
            b = np.zeros(MLP_DOUT[l], np.float32)
            check(lib.rf_mlp_get(self.h, l, W.ctypes.data, b.ctypes.data), "rf_mlp_get")
            out.append((W, b))
        return out

    def set_weights(self, ws):
        for l, (W, b) in enumerate(ws):
            W = np.ascontiguousarray(W, np.float32)
            b = np.ascontiguousarray(b, np.float32)
            check(lib.rf_mlp_set(self.h, l, W.ctypes.data, b.ctypes.data), "rf_mlp_set")

    def grads(self):
        out = []
        for l in range(4):
            gT = np.zeros((MLP_DIN[l], MLP_DOUT[l]), np.float32)
            gb = np.zeros(MLP_DOUT[l], np.float32)
            check(lib.rf_mlp_grad(self.h, l, gT.ctypes.data, gb.ctypes.data), "rf_mlp_grad")
            out.append((gT, gb))
        return out


class BatchEngine(Engine):
    """Several extended-model specimens advanced by one step kernel (rf_engine_create_batch)."""

    def __init__(self, tasks, params, Rs, radii):
        n = len(tasks)
        self.tasks = (Task * n)(*tasks)
        self.params = (ExtParams * n)(*params)
        self._R = [np.ascontiguousarray(R, np.float64) for R in Rs]
        self._rad = [np.ascontiguousarray(r, np.float64) for r in radii]
        pR = (C.c_void_p * n)(*[R.ctypes.data for R in self._R])
        pr = (C.c_void_p * n)(*[r.ctypes.data for r in self._rad])
        h = P()
        check(lib.rf_engine_create_batch(self.tasks, self.params, pR, pr, n, C.byref(h)), "rf_engine_create_batch")
        self.h = h
        self.ext = True
        self.nspec = n
        self.N = int(sum(t.N for t in tasks))
        self.K = int(tasks[0].K)
        self.task = tasks[0]

    def load_increment(self, params, warm=None, ldw=6, scaled=False):
        """One quasi-static load increment of every specimen (rf_engine_load_increment_batch);
        warm: device tensor float32 [N, ldw] or None. Returns one RelaxResult per specimen."""
        rs = (RelaxResult * self.nspec)()
        check(lib.rf_engine_load_increment_batch(self.h, C.byref(params), ptr(warm), ldw, 1 if scaled else 0, rs),
              "rf_engine_load_increment_batch")
        return list(rs)

    def load_increment_pred(self, params, pred, ldp=16):
        """A load increment of every specimen from a WarmStart prediction [rows, ldp]."""
        return self.load_increment(params, pred, ldp, scaled=True)

    def spec_info(self, s):
        first, count, off = C.c_uint64(0), C.c_uint64(0), C.c_double(0)
        t = Task()
        check(lib.rf_engine_spec_info(self.h, s, C.byref(first), C.byref(count), C.byref(off), C.byref(t)),
              "rf_engine_spec_info")
        return int(first.value), int(count.value), off.value, t

    def sync_spec(self, s):
        t, r = Task(), RunResult()
        check(lib.rf_engine_sync_spec(self.h, s, C.byref(t), C.byref(r)), "rf_engine_sync_spec")
        return t, r

    def curve_spec(self, s):
        n = C.c_uint64(0)
        check(lib.rf_engine_curve_spec(self.h, s, None, 0, C.byref(n)), "rf_engine_curve_spec")
        m = min(n.value, 1 << 20)
        buf = np.zeros(3 * max(m, 1), np.float64)
        check(lib.rf_engine_curve_spec(self.h, s, buf.ctypes.data, m, C.byref(n)), "rf_engine_curve_spec")
        return buf[:3 * m].reshape(m, 3)


# --- state files ---------------------------------------------------------------
_ALL_PARTICLE = ["F", "V", "R", "M", "W"]
_ALL_SLOTS = ["Rij", "Oijt", "Fijn", "Fijt", "Mijn", "Mijt", "Mijadd"]


def save_all_data(path, sample, st, N, K, acut, pn=0, id_bytes=4):
    """The reference's SaveAllData file (rf_save_all_data) from a state dict in the
    reference layout (keys R, V, W, IL, ILtype, iL, Rij, Oijt, Mijn, Mijt as Engine.export
    returns them; optional F, M, Q, Fijn, Fijt, Mijadd; missing arrays are written as zeros)."""
    def a(k, dt):
        return None if st.get(k) is None else np.ascontiguousarray(st[k], dt)
    arrs = [a(k, np.float32) for k in _ALL_PARTICLE] + [a("Q", np.float32), a("IL", ID_NP), a("ILtype", np.uint8),
                                                         a("iL", np.float32)] + [a(k, np.float32) for k in _ALL_SLOTS]
    check(lib.rf_save_all_data(os.fsencode(path), id_bytes, C.byref(sample), pn, N, K, acut,
                               *[ptr(x) for x in arrs]), "rf_save_all_data")


def load_all_data(path, id_bytes=4):
    """Read a SaveAllData file: returns (Sample, pn, acut, N, K, state dict)."""
    S, pn, N, K, ac = Sample(), C.c_uint64(0), C.c_uint64(0), C.c_uint32(0), C.c_float(0)
    nul = [None] * 16
    check(lib.rf_load_all_data(os.fsencode(path), id_bytes, C.byref(S), C.byref(pn), C.byref(N), C.byref(K),
                               C.byref(ac), *nul), "rf_load_all_data")
    n, k = int(N.value), int(K.value)
    st = {key: np.zeros(3 * n, np.float32) for key in _ALL_PARTICLE}
    st["Q"] = np.zeros(4 * n, np.float32)
    st["IL"] = np.zeros(n * k, ID_NP)
    st["ILtype"] = np.zeros(n * k, np.uint8)
    st["iL"] = np.zeros(n * k, np.float32)
    for key in _ALL_SLOTS:
        st[key] = np.zeros(3 * n * k, np.float32)
    order = _ALL_PARTICLE + ["Q", "IL", "ILtype", "iL"] + _ALL_SLOTS
    check(lib.rf_load_all_data(os.fsencode(path), id_bytes, C.byref(S), C.byref(pn), C.byref(N), C.byref(K),
                               C.byref(ac), *[ptr(st[key]) for key in order]), "rf_load_all_data")
    return S, int(pn.value), ac.value, n, k, st


def save_lammps_data(path, task, st, with_energy=True):
    """LAMMPS data text of SaveLammpsDATASimple (rf_save_lammps_data) from a state dict."""
    N, K = int(task.N), int(task.K)
    arr = [np.ascontiguousarray(st[k], np.float32) for k in ("R", "V", "W")]
    check(lib.rf_save_lammps_data(os.fsencode(path), C.byref(task), N, K, *[ptr(x) for x in arr],
                                  ptr(np.ascontiguousarray(st["IL"], ID_NP)),
                                  ptr(np.ascontiguousarray(st["ILtype"], np.uint8)), 1 if with_energy else 0),
          "rf_save_lammps_data")


def save_positions_txt(path, R):
    """The reference's position text file (SaveParticleDATAtxt) of planar float32 R (mm)."""
    R = np.ascontiguousarray(R, np.float32)
    check(lib.rf_save_positions_txt(os.fsencode(path), R.ctypes.data, R.size // 3), "rf_save_positions_txt")


def load_positions_txt(path):
    """Positions of a reference position text file (LoadParticleDATAtxt), planar float32 (mm)."""
    n = C.c_uint64(0)
    check(lib.rf_load_positions_txt(os.fsencode(path), None, 0, C.byref(n)), "rf_load_positions_txt")
    R = np.zeros(3 * n.value, np.float32)
    check(lib.rf_load_positions_txt(os.fsencode(path), R.ctypes.data, n.value, C.byref(n)), "rf_load_positions_txt")
    return R
