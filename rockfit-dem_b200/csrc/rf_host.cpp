// Host side of the engine: error text, the reference's parameter derivation and
// platen bookkeeping (md_data_types.h, md_results.cu), the whole-test drivers
// (h_CalculationBrazilTest / h_CalculationUniaxialCompression) on top of the
// fused engine, and the seeded synthetic specimen generator.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/rockfit_b200.h"

namespace rf {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

rf_status cuda_status(cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return RF_ERR_CUDA;
}

static const double MC_pi = 3.1415926535897932384626433832795;   // md_math_constants.h:44
static const double MC_1d3 = 1.0 / 3.0;                           // md_math_constants.h:15
static const double length_const = 1e-3;                          // md_phys_constants.h:5

}  // namespace rf

using namespace rf;

extern "C" {

const char* rf_last_error_string(void) { return g_err; }
int rf_version(void) { return 100; }
int rf_id_bytes(void) { return (int)sizeof(uint_fast32_t); }

rf_status rf_task_prepare(rf_task* t, const double ss[3], const double ls[3], double cell_a, double vload,
                          double minstress, double maxstrain) {
    if (!t || !ss || !ls || !(cell_a > 0)) { set_error("rf_task_prepare: bad arguments"); return RF_ERR_INVALID; }
    rf_potential& P = t->Po;
    // potential_data::CalculateParameters (md_data_types.h:153-185)
    P.m_G = 0.5 * P.m_E / (1.0 + P.m_nu);
    P.b_S = MC_pi * P.b_r * P.b_r;
    P.p_V = 4.0 * MC_1d3 * MC_pi * P.p_r * P.p_r * P.p_r;
    P.p_m = P.m_ro * P.p_V;
    P.b_dd = P.b_d * P.b_d;
    P.p_1d_m = 1.0 / P.p_m;
    P.p_I = 0.4 * P.p_m * P.p_r * P.p_r;
    P.hm_E = 0.5 * P.m_E / (1.0 - P.m_nu * P.m_nu);
    P.hm_G = 0.5 * P.m_G / (2.0 - P.m_nu);
    const double le = std::log(P.p_e);
    P.p_A = le / std::sqrt(MC_pi * MC_pi + le * le);
    P.aa_farcut = P.a_farcut * P.a_farcut;
    P.Trayleigh = MC_pi * P.p_r * std::sqrt(2.0 * P.m_ro * (1.0 + P.m_nu)) /
                  (std::sqrt(P.m_E) * (0.163 * P.m_nu + 0.8766));
    const double k0 = P.m_E * P.b_S / (2.0 * P.p_r), k1 = P.m_G * P.b_S / (2.0 * P.p_r);
    P.Tsim = (k0 > k1) ? 2.0 * std::sqrt(P.p_m / k0) : 2.0 * std::sqrt(P.p_m / k1);
    P.dt = (P.Trayleigh < P.Tsim) ? 0.1 * P.Trayleigh : 0.1 * P.Tsim;
    P.D = 1e-15 * P.m_E * P.b_S / (2.0 * P.p_r);
    P.a = 2.0 * P.p_r;
    P._1d_a = 1.0 / P.a;
    P.aa = P.a * P.a;
    P.dt_d_m = P.p_1d_m * P.dt;
    P.dt_d_I = P.dt / P.p_I;

    rf_sample& S = t->S;
    rf_cells& C = t->C;
    C.a = (float)cell_a;
    // sample_data::SetSpaceSizeSi / SetLSi / SetAxis / CalculateParameters (md_data_types.h:86-121)
    S.spacesize.x = (float)(ss[0] / length_const);
    S.spacesize.y = (float)(ss[1] / length_const);
    S.spacesize.z = (float)(ss[2] / length_const);
    S.spacesized2.x = (float)(0.5 * S.spacesize.x);
    S.spacesized2.y = (float)(0.5 * S.spacesize.y);
    S.spacesized2.z = (float)(0.5 * S.spacesize.z);
    S.L.x = (float)(ls[0] / length_const - 2.0 * P.p_r);
    S.L.y = (float)(ls[1] / length_const - 2.0 * P.p_r);
    S.L.z = (float)(ls[2] / length_const - 2.0 * P.p_r);
    S.axis.x = 0.f; S.axis.y = 0.f; S.axis.z = 1.f;
    const double Ca = (double)C.a, pr = P.p_r;
    S.A.x = (float)(1.01 * Ca); S.A.y = (float)(1.01 * Ca); S.A.z = (float)(1.01 * Ca);
    S.B.x = S.A.x + S.spacesize.x; S.B.y = S.A.y + S.spacesize.y; S.B.z = S.A.z + S.spacesize.z;
    S.center.x = (float)(0.5 * (S.A.x + S.B.x));
    S.center.y = (float)(0.5 * (S.A.y + S.B.y));
    S.center.z = (float)(0.5 * (S.A.z + S.B.z));
    S.size = S.L;
    S.sized2.x = (float)(0.5 * S.L.x); S.sized2.y = (float)(0.5 * S.L.y); S.sized2.z = (float)(0.5 * S.L.z);
    S.R0 = (float)(0.5 * S.L.x);
    S.H0 = (float)(0.5 * S.L.z);
    S.Vext = MC_pi * (0.5 * S.L.x + pr) * (0.5 * S.L.x + pr) * (S.L.z + 2.0 * pr);
    S.hidenpoint.x = (float)(S.A.x + 0.5 * S.spacesize.x);
    S.hidenpoint.y = (float)(S.A.y + 0.5 * S.spacesize.y);
    {
        const float fl = std::floor((float)((double)S.B.z / Ca));   // floorf(B.z / C_a), argument narrowed
        const float f3v = fl + 3.0f;
        S.hidenpoint.z = (float)(((double)f3v - 0.5) * Ca);
    }
    const float ax = S.center.x - S.sized2.x, ay = S.center.y - S.sized2.y, az = S.center.z - S.sized2.z;
    const float bx = S.center.x + S.sized2.x, by = S.center.y + S.sized2.y, bz = S.center.z + S.sized2.z;
    S.A_real.x = ax; S.A_real.y = ay; S.A_real.z = az;
    S.B_real.x = bx; S.B_real.y = by; S.B_real.z = bz;
    S.size_real.x = S.B_real.x - S.A_real.x; S.size_real.y = S.B_real.y - S.A_real.y;
    S.size_real.z = S.B_real.z - S.A_real.z;
    S.center_real.x = 0.5 * (S.B_real.x + S.A_real.x);
    S.center_real.y = 0.5 * (S.B_real.y + S.A_real.y);
    S.center_real.z = 0.5 * (S.B_real.z + S.A_real.z);
    S.Vgenmax = 0.f;
    // interaction_list_data::CalculateParameters (md_data_types.h:137-143)
    t->acut = (float)P.a_farcut;
    t->aacut = t->acut * t->acut;
    // cell_data::CalculateParameters (md_data_types.h:42-55) with S.B (md_calculationbraziltest.cu:118)
    C._1d_a = (float)(1.0 / (double)C.a);
    C.Nr.x = (unsigned)(std::floor((float)((double)S.B.x * (double)C._1d_a)) + 1.0f);
    C.Nr.y = (unsigned)(std::floor((float)((double)S.B.y * (double)C._1d_a)) + 1.0f);
    C.Nr.z = (unsigned)(std::floor((float)((double)S.B.z * (double)C._1d_a)) + 3.0f);
    C.N = (uint64_t)C.Nr.x * C.Nr.y * C.Nr.z;
    C._1d_Nr.x = (float)(1.0 / (double)C.Nr.x);
    C._1d_Nr.y = (float)(1.0 / (double)C.Nr.y);
    C._1d_Nr.z = (float)(1.0 / (double)C.Nr.z);
    t->bloks = t->N / 1024 + 1;
    // compression_data::CalculateUParameters / CalculateBParameters (md_data_types.h:196-271)
    rf_compression& K = t->Compress;
    std::memset(&K, 0, sizeof(K));
    K.VLoad = vload;
    K.size_d = S.size_real;
    K.size.x = (float)K.size_d.x; K.size.y = (float)K.size_d.y; K.size.z = (float)K.size_d.z;
    K.sized2.x = (float)(0.5 * K.size_d.x); K.sized2.y = (float)(0.5 * K.size_d.y); K.sized2.z = (float)(0.5 * K.size_d.z);
    K.center_d = S.center_real;
    K.center.x = (float)K.center_d.x; K.center.y = (float)K.center_d.y; K.center.z = (float)K.center_d.z;
    K.Hd2 = K.sized2.z;
    K.C = (float)(P.m_E * P.b_S / (4.0 * P.p_r));
    K.mu = (float)P.p_mu;
    K.MinStress = minstress;
    K.MaxStrain = maxstrain;
    if (t->kind == RF_TEST_UNIAXIAL) {
        K.Size0 = K.size_d.z;
        K.Bottom = K.center_d.z - 0.5 * K.size_d.z;
        K.BottomR = K.Bottom + P.p_r;
        K.Top = K.center_d.z + 0.5 * K.size_d.z;
        K.TopR = K.Top - P.p_r;
        K.R = (float)(1.5 * K.sized2.x);
        K.Area = (float)(MC_pi * (K.sized2.x + P.p_r) * (K.sized2.x + P.p_r));
        K.ZeroStress = 0.33 * K.MinStress;
    } else {
        K.Size0 = K.size_d.y;
        K.Bottom = K.center_d.y - 0.5 * K.size_d.y;
        K.BottomR = K.Bottom + P.p_r;
        K.Top = K.center_d.y + 0.5 * K.size_d.y;
        K.TopR = K.Top - P.p_r;
        K.R = (K.sized2.x > K.sized2.z) ? K.sized2.x : (float)(1.05 * K.sized2.z);
        K.Area = (float)(0.5 * 2 * MC_pi * (K.sized2.x + P.p_r) * (K.size.z + 2.0 * P.p_r));
        K.ZeroStress = 0.5 * K.MinStress;
    }
    K.RR = K.R * K.R;
    K._1d_Area = (float)(1.0 / (double)K.Area);
    // The reference reads V and Strain before its first CompressU/B call sets them;
    // they start at zero here.
    K.V = 0.0;
    K.Strain = 0.0;
    t->sz0 = (double)K.size.z;
    return RF_OK;
}

static void compress_axis(rf_task* t, double pressure, int ax) {
    rf_compression& K = t->Compress;
    const double dt = t->Po.dt, pr = t->Po.p_r;
    K.V = (pressure < 1e-9) ? 10.0 * K.VLoad : K.VLoad;
    double* sd = ax == 1 ? &K.size_d.y : &K.size_d.z;
    double* cd = ax == 1 ? &K.center_d.y : &K.center_d.z;
    float* sz = ax == 1 ? &K.size.y : &K.size.z;
    float* s2 = ax == 1 ? &K.sized2.y : &K.sized2.z;
    float* cf = ax == 1 ? &K.center.y : &K.center.z;
    *sd += K.V * dt;
    K.Top += K.V * dt;
    K.TopR = K.Top - 2.0 * pr;
    *sz = (float)*sd;
    *s2 = (float)(0.5 * *sd);
    *cd += K.V * dt;
    *cf = (float)*cd;
    K.Hd2 = *s2;
    K.Strain = (*sd - K.Size0) / K.Size0;
}

rf_status md_CompressU(rf_task* t, double pressure) {
    if (!t) { set_error("md_CompressU: null task"); return RF_ERR_INVALID; }
    compress_axis(t, pressure, 2);
    return RF_OK;
}
rf_status md_CompressB(rf_task* t, double pressure) {
    if (!t) { set_error("md_CompressB: null task"); return RF_ERR_INVALID; }
    compress_axis(t, pressure, 1);
    return RF_OK;
}

rf_status md_SumForcesULoading(rf_task* t, const float* h_FL, uint64_t nblocks, uint64_t step, uint64_t dNsave,
                               double sz0, double* curve, uint64_t* nsaved) {
    if (!t || !h_FL || nblocks == 0) { set_error("md_SumForcesULoading: bad arguments"); return RF_ERR_INVALID; }
    rf_compression& K = t->Compress;
    double s0 = 0.0, s1 = 0.0;
    for (uint64_t b = 0; b < nblocks; ++b) s0 += h_FL[b];
    for (uint64_t b = nblocks; b < 2 * nblocks; ++b) s1 += h_FL[b];
    if (curve && nsaved && dNsave && step % dNsave == 0) {
        double* r = curve + 3 * *nsaved;
        r[0] = (K.size_d.z - sz0) / sz0;
        r[1] = s0 * (double)K._1d_Area;
        r[2] = s1 * (double)K._1d_Area;
        ++*nsaved;
    }
    K.Stress = 0.5 * (std::fabs(s0) + std::fabs(s1)) * (double)K._1d_Area;
    if (!K.Loading && K.Stress > K.MinStress) K.Loading = 1;
    if (K.FractureStress < K.Stress) {
        K.FractureStress = K.Stress;
        K.FractureStrain = (sz0 - K.size_d.z) / sz0;
    }
    if (K.Loading && K.Stress < K.ZeroStress) K.Fracture = 1;
    return RF_OK;
}

rf_status md_SetFIREData(rf_fire* f, uint_fast32_t N, const rf_potential* Po) {
    if (!f || !Po) { set_error("md_SetFIREData: bad arguments"); return RF_ERR_INVALID; }
    std::memset(f, 0, sizeof(*f));
    f->bloks4 = N / (4 * 256) + 1;          // SMEMDIM = 256
    f->dt0 = (float)Po->dt;
    f->dtmax = (float)(100.0 * (double)f->dt0);
    f->dtmin = (float)(0.001 * (double)f->dt0);
    f->dtgrow = 1.1f;
    f->dtshrink = 0.5f;
    f->alpha0 = 0.25f;
    f->alphashrink = 0.99f;
    f->NPnegativeMax = 30000;
    f->Ndelay = 20;
    f->NPpositive = 0;
    f->NPnegative = 0;
    f->dt = f->dt0;
    f->alpha = f->alpha0;
    return RF_OK;
}

rf_status md_FireDecide(rf_fire* f, double FdotV, uint64_t step, int* half_step, int* stop) {
    if (!f || !half_step || !stop) { set_error("md_FireDecide: bad arguments"); return RF_ERR_INVALID; }
    f->FdotV = FdotV;
    *half_step = 0;
    *stop = 0;
    if (FdotV > 0) {
        ++f->NPpositive;
        f->NPnegative = 0;
        if (f->NPpositive > f->Ndelay) {
            f->dt = (f->dt * f->dtgrow < f->dtmax) ? f->dt * f->dtgrow : f->dtmax;
            f->alpha *= f->alphashrink;
        }
    } else {
        f->NPpositive = 0;
        ++f->NPnegative;
        if (f->NPnegative > f->NPnegativeMax) { *stop = 1; return RF_OK; }
        if (step > f->Ndelay) {
            f->dt = (f->dt * f->dtshrink > f->dtmin) ? f->dt * f->dtshrink : f->dtmin;
            f->alpha = f->alpha0;
        }
        *half_step = 1;
    }
    return RF_OK;
}

static rf_status run_test(rf_task* t, const float* h_R, uint64_t max_steps, double* curve, uint64_t curve_cap,
                          float* h_R_out, rf_run_result* result) {
    if (!t || !h_R) { set_error("md_Calculation*: bad arguments"); return RF_ERR_INVALID; }
    rf_engine* e = nullptr;
    rf_status st = rf_engine_create(t, h_R, &e);
    if (st) return st;
    const uint64_t chunk = max_steps ? max_steps : (1ull << 22);
    rf_run_result r;
    std::memset(&r, 0, sizeof(r));
    for (;;) {
        if ((st = rf_engine_step(e, chunk))) break;
        if ((st = rf_engine_sync(e, t, &r))) break;
        const bool running = t->Compress.Strain < t->Compress.MaxStrain && !t->Compress.Fracture;
        if (max_steps || !running) break;
    }
    if (!st && curve && curve_cap) st = rf_engine_curve(e, curve, curve_cap, nullptr);
    if (!st && h_R_out) st = rf_engine_export(e, h_R_out, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                              nullptr, nullptr, nullptr);
    if (result) *result = r;
    rf_engine_destroy(e);
    return st;
}

rf_status md_CalculationBrazilTest(rf_task* t, const float* h_R, uint64_t max_steps, double* curve,
                                   uint64_t curve_cap, float* h_R_out, rf_run_result* result) {
    if (!t || t->kind != RF_TEST_BRAZIL) { set_error("md_CalculationBrazilTest: task kind must be RF_TEST_BRAZIL"); return RF_ERR_INVALID; }
    return run_test(t, h_R, max_steps, curve, curve_cap, h_R_out, result);
}

rf_status md_CalculationUniaxialCompression(rf_task* t, const float* h_R, uint64_t max_steps, double* curve,
                                            uint64_t curve_cap, float* h_R_out, rf_run_result* result) {
    if (!t || t->kind != RF_TEST_UNIAXIAL) {
        set_error("md_CalculationUniaxialCompression: task kind must be RF_TEST_UNIAXIAL");
        return RF_ERR_INVALID;
    }
    return run_test(t, h_R, max_steps, curve, curve_cap, h_R_out, result);
}

// ---------------------------------------------------------------------------
// Seeded specimens: splitmix64 counter stream -> uniforms in [0, 1).
// ---------------------------------------------------------------------------
static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
static inline double unif(uint64_t seed, uint64_t ctr) {
    return (double)(splitmix64(seed * 0x2545F4914F6CDD1Dull + ctr) >> 11) * (1.0 / 9007199254740992.0);
}

static rf_status lattice(uint64_t seed, double p_r, double gap_frac, double jitter, double d, double h,
                         const double c[3], float* R, uint64_t cap, uint64_t* n, bool disc) {
    if (!n || !c || !(p_r > 0) || !(d > 0) || !(h > 0)) { set_error("rf_specimen: bad arguments"); return RF_ERR_INVALID; }
    (void)disc;
    const double sp = 2.0 * p_r * (1.0 + gap_frac);
    const double rad = 0.5 * d - p_r;                     // particle centres inside the specimen
    const double hz = 0.5 * h - p_r;
    const long nx = (long)std::floor(rad / sp), nz = (long)std::floor(hz / sp);
    std::vector<double> pts;
    uint64_t ctr = 0;
    for (long iz = -nz; iz <= nz; ++iz)
        for (long iy = -nx; iy <= nx; ++iy)
            for (long ix = -nx; ix <= nx; ++ix) {
                const double x = ix * sp, y = iy * sp, z = iz * sp;
                const uint64_t id = ctr++;
                if (x * x + y * y > rad * rad) continue;
                const double jx = (2.0 * unif(seed, 3 * id) - 1.0) * jitter * p_r;
                const double jy = (2.0 * unif(seed, 3 * id + 1) - 1.0) * jitter * p_r;
                const double jz = (2.0 * unif(seed, 3 * id + 2) - 1.0) * jitter * p_r;
                pts.push_back(c[0] + x + jx);
                pts.push_back(c[1] + y + jy);
                pts.push_back(c[2] + z + jz);
            }
    const uint64_t m = pts.size() / 3;
    *n = m;
    if (!R) return RF_OK;
    if (m > cap) { set_error("rf_specimen: capacity %llu < %llu particles", (unsigned long long)cap, (unsigned long long)m); return RF_ERR_CAPACITY; }
    for (uint64_t i = 0; i < m; ++i) {
        R[i] = (float)pts[3 * i];
        R[i + m] = (float)pts[3 * i + 1];
        R[i + 2 * m] = (float)pts[3 * i + 2];
    }
    return RF_OK;
}

rf_status rf_specimen_lattice_cylinder(uint64_t seed, double p_r, double gap_frac, double jitter, double d, double h,
                                       const double center[3], float* R, uint64_t cap, uint64_t* n) {
    return lattice(seed, p_r, gap_frac, jitter, d, h, center, R, cap, n, false);
}
rf_status rf_specimen_lattice_disc(uint64_t seed, double p_r, double gap_frac, double jitter, double d, double h,
                                   const double center[3], float* R, uint64_t cap, uint64_t* n) {
    return lattice(seed, p_r, gap_frac, jitter, d, h, center, R, cap, n, true);
}

}  // extern "C"
