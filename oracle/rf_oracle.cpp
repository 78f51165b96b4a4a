// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the RockFit-DEM hot path (one thread per particle, serial,
// in the reference's own order of operations). It is the checker for the CUDA
// engine: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// may load it. Nothing in the product links or calls it.
//
// Built with -O2 -ffp-contract=off (no FMA contraction, SSE arithmetic), so every
// float operation below is one IEEE-754 round-to-nearest operation in source order.
// Each function is instantiated for T = float (the reference's precision; the
// engine's reference mode must match it bit for bit) and T = double (the FP64
// oracle used to report error). Reference citations are file:line in
// MSMS-LAB/RockFit-DEM.
//
// CUDA intrinsics the reference calls are restated as:
//   __fmul_rn(a,b)  -> a*b                      (IEEE product)
//   __frcp_rn(x)    -> 1/x                      (IEEE quotient)
//   __fsqrt_rn(x)   -> sqrt(x)                  (IEEE square root)
//   __frsqrt_rn(x)  -> correctly rounded 1/sqrt(x), computed in double and
//                      rounded once (exhaustively checked against the device)
//   norm3df(x,y,z)  -> sqrt(x*x + y*y + z*z)    (the engine uses the same formula;
//                      the reference's library norm may differ in the last bit)
// Quirks of the reference that are reproduced are marked "QUIRK".
// Where the reference reads or writes out of bounds, the oracle stops at the
// bound and reports a status instead (marked "BOUND").

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <limits>
#include <chrono>

#include "../include/rockfit_b200.h"

namespace rfo {

typedef uint64_t id_t;                        // uint_fast32_t on Linux glibc
static const id_t EMPTY = std::numeric_limits<id_t>::max();

enum { ST_OK = 0, ST_ROW_OVERFLOW = 3, ST_CELL_RANGE = 4 };

template <class T> struct V3 { T x, y, z; };

// float -> unsigned conversion as the device does it (saturating, NaN -> 0).
static inline uint32_t f2u_sat(double v) {
    if (!(v > 0.0)) return 0u;
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

template <class T> static inline T rsqrt_rn(T x);
template <> inline float rsqrt_rn<float>(float x) { return (float)(1.0 / std::sqrt((double)x)); }
template <> inline double rsqrt_rn<double>(double x) { return 1.0 / std::sqrt(x); }

template <class T> static inline T floor_t(T x);
template <> inline float floor_t<float>(float x) { return std::floor(x); }
template <> inline double floor_t<double>(double x) { return std::floor(x); }

// ---------------------------------------------------------------------------
// Cells: d_CalculateCellIndex (md_calculate_cell.cu:28-53)
// ---------------------------------------------------------------------------
template <class T>
static inline uint64_t cell_of(const T* R, uint64_t N, uint64_t i, T inv_a, const rf_uint3& cN,
                               uint32_t* ix, uint32_t* iy, uint32_t* iz) {
    uint32_t x = f2u_sat((double)floor_t<T>(R[i] * inv_a));
    uint32_t y = f2u_sat((double)floor_t<T>(R[i + N] * inv_a));
    uint32_t z = f2u_sat((double)floor_t<T>(R[i + 2 * N] * inv_a));
    if (ix) { *ix = x; *iy = y; *iz = z; }
    // iindx = indx.x + indx.y*cN.x + indx.z*cN.y*cN.x, in unsigned int then widened
    // to uint_fast32_t (md_calculate_cell.cu:47).
    uint32_t c = x + y * cN.x + z * cN.y * cN.x;
    return (uint64_t)c;
}

template <class T>
int cell_index(const T* R, uint64_t N, id_t* CI, T inv_a, rf_uint3 cN) {
    int st = ST_OK;
    for (uint64_t i = 0; i < N; ++i) {
        uint32_t x, y, z;
        CI[i] = cell_of(R, N, i, inv_a, cN, &x, &y, &z);
        if (x > cN.x - 1 || y > cN.y - 1 || z > cN.z - 1) st = ST_CELL_RANGE;  // pre_debugtest check :42-46
    }
    return st;
}

// CellDistribution (md_cell_distribution.cu:52-101): stable sort of (CI, 0..N-1)
// (cub radix sort is stable; values are the identity filled by d_FillIndex), then
// d_DetermineCellPointer (md_calculate_cell.cu:55-80) after a zero fill of pnC.
template <class T>
int cell_distribution(const T* R, uint64_t N, id_t* CI, id_t* CIs, id_t* pnC, uint64_t CN,
                      T inv_a, rf_uint3 cN) {
    int st = cell_index(R, N, CI, inv_a, cN);
    std::vector<id_t> ids(N);
    for (uint64_t i = 0; i < N; ++i) ids[i] = i;
    std::stable_sort(ids.begin(), ids.end(), [&](id_t a, id_t b) { return CI[a] < CI[b]; });
    for (uint64_t i = 0; i < N; ++i) { CIs[i] = CI[ids[i]]; CIs[N + i] = ids[i]; }
    std::memset(pnC, 0, sizeof(id_t) * 2 * CN);
    for (uint64_t i = 0; i < N; ++i) {
        id_t c = CIs[i];
        if (i == 0 || CIs[i - 1] != c) {
            if (c >= CN) { st = ST_CELL_RANGE; continue; }          // BOUND
            pnC[c] = i;
            uint64_t n = 1;
            // QUIRK (md_calculate_cell.cu:72): the run scan does not stop at N and
            // continues into the id half of CIs; ids are distinct, so at most one
            // extra match (CIs[N] == c) can extend the last run.
            while (i + n < 2 * N && CIs[i + n] == c) ++n;
            pnC[c + CN] = n;
        }
    }
    return st;
}

// The 8 octant cells in the order the reference visits them
// (md_interaction_list_construct.cu:59-85, md_interaction_list_reconstructbpm.cu:107-134).
template <class T>
static inline void octant_cells(const T* R, uint64_t N, uint64_t i, T a, T inv_a, const rf_uint3& cN,
                                int64_t cells[8]) {
    uint32_t ix, iy, iz;
    uint64_t c = cell_of(R, N, i, inv_a, cN, &ix, &iy, &iz);
    // indxx = copysignf(1, R - __fmul_rn(indx + 0.5f, a)); indx + 0.5f is float math
    T hx = (T)((T)ix + (T)0.5f), hy = (T)((T)iy + (T)0.5f), hz = (T)((T)iz + (T)0.5f);
    int sx = std::signbit(R[i] - hx * a) ? -1 : 1;
    int sy = std::signbit(R[i + N] - hy * a) ? -1 : 1;
    int sz = std::signbit(R[i + 2 * N] - hz * a) ? -1 : 1;
    int64_t ox = sx, oy = (int64_t)sy * cN.x, oz = (int64_t)sz * cN.y * cN.x;
    int64_t b = (int64_t)c;
    cells[0] = b;
    cells[1] = b + ox;
    cells[2] = b + oy;
    cells[3] = b + oz;
    cells[4] = b + ox + oy;
    cells[5] = b + ox + oz;
    cells[6] = b + oy + oz;
    cells[7] = b + ox + oy + oz;
}

template <class T>
static inline T dist2_rn(const T* R, uint64_t N, uint64_t i, uint64_t j) {
    // rr = __fmul_rn(dx,dx) + __fmul_rn(dy,dy) + __fmul_rn(dz,dz)
    T dx = R[j] - R[i], dy = R[j + N] - R[i + N], dz = R[j + 2 * N] - R[i + 2 * N];
    return dx * dx + dy * dy + dz * dz;
}

// InteractionListConstruct: memset IL to 0xFF, then d_ConstructInteractionList
// (md_interaction_list_construction.cu:163-168, md_interaction_list_construct.cu:13-98).
template <class T>
int construct_list(const T* R, uint64_t N, const id_t* CIs, const id_t* pnC, id_t* IL, uint64_t K,
                   T a, T inv_a, T aacut, rf_uint3 cN, uint64_t CN) {
    int st = ST_OK;
    for (uint64_t k = 0; k < N * K; ++k) IL[k] = EMPTY;
    for (uint64_t i = 0; i < N; ++i) {
        int64_t cells[8];
        octant_cells(R, N, i, a, inv_a, cN, cells);
        uint64_t n = 0;
        for (int c = 0; c < 8; ++c) {
            if (cells[c] < 0 || (uint64_t)cells[c] >= CN) { st = ST_CELL_RANGE; continue; }  // BOUND
            uint64_t start = pnC[cells[c]], cnt = pnC[cells[c] + CN];
            for (uint64_t m = 0; m < cnt; ++m) {
                if (start + m >= N) break;                                          // BOUND
                id_t j = CIs[start + m + N];
                if (j >= N) continue;                                               // BOUND
                T rr = dist2_rn(R, N, i, j);
                if (rr < aacut && j != i) {                                         // :26
                    if (n < K) IL[i * K + n] = j; else st = ST_ROW_OVERFLOW;        // BOUND (:89-92)
                    ++n;
                }
            }
        }
    }
    return st;
}

// d_ReConstructInteractionListbpm + addnewlinkbpm (md_interaction_list_reconstructbpm.cu:13-46,80-139)
template <class T>
int reconstruct_bpm(const T* R, uint64_t N, const id_t* CIs, const id_t* pnC, id_t* IL, uint8_t* ILtype,
                    uint64_t K, T a, T inv_a, T aacut, rf_uint3 cN, uint64_t CN) {
    int st = ST_OK;
    for (uint64_t i = 0; i < N; ++i) {
        int64_t cells[8];
        octant_cells(R, N, i, a, inv_a, cN, cells);
        for (int c = 0; c < 8; ++c) {
            if (cells[c] < 0 || (uint64_t)cells[c] >= CN) { st = ST_CELL_RANGE; continue; }  // BOUND
            uint64_t start = pnC[cells[c]], cnt = pnC[cells[c] + CN];
            for (uint64_t m = 0; m < cnt; ++m) {
                if (start + m >= N) break;                                          // BOUND
                id_t j = CIs[start + m + N];
                if (j >= N) continue;                                               // BOUND
                T rr = dist2_rn(R, N, i, j);
                if (rr < aacut && rr > 1e-10) {                                     // :28
                    // QUIRK (:30-36): kdxfree == 0 doubles as "no free slot found", so for
                    // particle 0 a free slot 0 is passed over while a later free slot exists.
                    uint64_t kdxfree = 0;
                    uint64_t s;
                    for (s = 0; s < K; ++s) {
                        id_t kj = IL[i * K + s];
                        if (kdxfree == 0 && kj == EMPTY) kdxfree = i * K + s;
                        if (kj == j) break;
                    }
                    if (s == K) {
                        // BOUND: with no free slot the reference writes IL[0]; here the row
                        // is left unchanged and overflow is reported.
                        bool has_free = false;
                        for (uint64_t q = 0; q < K; ++q) if (IL[i * K + q] == EMPTY) has_free = true;
                        if (!has_free) { st = ST_ROW_OVERFLOW; continue; }
                        IL[kdxfree] = j;
                        ILtype[kdxfree] = 0;
                    }
                }
            }
        }
    }
    return st;
}

// d_DeleteFarLinks (md_interaction_list_reconstructbpm.cu:141-186).
// QUIRK: the reference's "_1d_iL = 0;" clears its own pointer, not the element, so
// 1/L0 of a deleted slot is left as it was.
template <class T>
void delete_far_links(const T* R, uint64_t N, id_t* IL, uint8_t* ILtype, V3<T>* Rij, V3<T>* Oijt,
                      V3<T>* Mijn, V3<T>* Mijt, uint64_t K, T aacut) {
    for (uint64_t i = 0; i < N; ++i)
        for (uint64_t s = 0; s < K; ++s) {
            uint64_t k = i * K + s;
            id_t j = IL[k];
            if (j == EMPTY) continue;
            if (j >= N) continue;                                                   // BOUND
            T rr = dist2_rn(R, N, i, j);
            if (rr > aacut || rr < 1e-10) {
                IL[k] = EMPTY;
                ILtype[k] = 0;
                Rij[k] = {0, 0, 0};
                Oijt[k] = {0, 0, 0};
                Mijn[k] = {0, 0, 0};
                Mijt[k] = {0, 0, 0};
                // Fijn, Fijt, Mijadd are zeroed too; the live path never makes them non-zero.
            }
        }
}

// d_ConstructBoundInteractions (md_boundinteractions_construct.cu:35-106).
// rm2 = r.x*r.x + r.y*r.y + r.z*r.z is restated with the FMA contraction nvcc applies
// to that expression in the reference build: fma(z, z, fma(x, x, y*y)).
template <class T>
static inline T rm2_bond(T x, T y, T z) { return std::fma(z, z, std::fma(x, x, y * y)); }

template <class T>
void construct_bonds(const T* R, uint64_t N, const id_t* IL, uint8_t* ILtype, T* iL, V3<T>* Rij,
                     V3<T>* Oijt, V3<T>* Mijn, V3<T>* Mijt, uint64_t K, T aa_create) {
    for (uint64_t i = 0; i < N; ++i)
        for (uint64_t s = 0; s < K; ++s) {
            uint64_t k = i * K + s;
            id_t j = IL[k];
            if (j == EMPTY) continue;
            if (j >= N) continue;                                                   // BOUND
            T rx = R[j] - R[i], ry = R[j + N] - R[i + N], rz = R[j + 2 * N] - R[i + 2 * N];
            T rm2 = rm2_bond(rx, ry, rz);
            if (rm2 < aa_create && rm2 > 1e-18) {
                iL[k] = rsqrt_rn(rm2);
                ILtype[k] = 1;
            } else {
                ILtype[k] = 0;
            }
            Rij[k] = {0, 0, 0};   // QUIRK Q2: the unit bond direction is overwritten with 0*r (:69-80)
            Oijt[k] = {0, 0, 0};
            Mijn[k] = {0, 0, 0};
            Mijt[k] = {0, 0, 0};
        }
}

// ---------------------------------------------------------------------------
// Forces (md_calculateforcesdem3.cu)
// ---------------------------------------------------------------------------
template <class T> struct FP {
    // kernel scalar arguments as the drivers pass them (floats for T = float)
    T dt, m_E, m_G, b_r, m_Gcritn, m_Gcritt;          // _22
    T hm_E, hm_G, p_A, m_mu, m_muroll, mP, rP;        // _21
};

template <class T> static inline T pi_t() { return (T)3.14159265358979f; }   // MCf_pi
template <class T> static inline T two_thirds_t() { return (T)0.6666666667f; }  // MCf_2d3

template <class T>
static inline T norm3(T x, T y, T z) { return std::sqrt(x * x + y * y + z * z); }

// d_CalculateForcesDEM_22 (:424-483) with dd_Calculate_rijm_nij_2 (:38-52),
// dd_Calculate_fijn_bpm_2 (:91-103), dd_Calculate_M123_bpm_2 (:54-89),
// dd_Calculate_mijn_bpm_2 (:105-129), dd_Calculate_mijt_bpm_2 (:131-152),
// dd_Calculate_fijt_mijunsym_bpm_2 (:154-197), dd_CheckBreakConditionDEM_2 (:20-36).
// F and M are accumulated (+=), as the kernel does after the driver's memset.
template <class T>
void forces_22(const T* R, const T* V, const T* W, const id_t* IL, uint8_t* ILtype, const T* iL,
               V3<T>* Rij, V3<T>* Oijt, V3<T>* Mijn, V3<T>* Mijt, T* F, T* M, uint64_t N, uint64_t K,
               const FP<T>& p, uint8_t* broke /* may be null: 1 where a bond broke */,
               T* crit = nullptr /* may be null: the break criteria (Sc, Mc) of each bond slot */) {
    const T PI = pi_t<T>();
    for (uint64_t i = 0; i < N; ++i) {
        T fsx = 0, fsy = 0, fsz = 0, msx = 0, msy = 0, msz = 0;
        T Sc = 0, Mc = 0;
        for (uint64_t s = 0; s < K; ++s) {
            uint64_t k = i * K + s;
            id_t j = IL[k];
            if (!(j != EMPTY && ILtype[k] == 1)) continue;
            // rijm, nij
            T rx = R[j] - R[i], ry = R[j + N] - R[i + N], rz = R[j + 2 * N] - R[i + 2 * N];
            T rijm = norm3(rx, ry, rz);
            T inv_rm = (T)1 / rijm;
            T nx = rx * inv_rm, ny = ry * inv_rm, nz = rz * inv_rm;
            // normal force
            T il = iL[k];
            T cef = p.m_E * (rijm - (T)1 / il) * il;
            Sc = cef;
            cef *= p.b_r * p.b_r * PI;
            fsx += nx * cef; fsy += ny * cef; fsz += nz * cef;
            // rotation-increment matrix
            V3<T> rp = Rij[k];
            T tx = rp.y * nz - rp.z * ny;
            T ty = rp.z * nx - rp.x * nz;
            T tz = rp.x * ny - rp.y * nx;
            T wsx = W[j] + W[i], wsy = W[j + N] + W[i + N], wsz = W[j + 2 * N] + W[i + 2 * N];
            T cphi = (wsx * nx + wsy * ny + wsz * nz) * p.dt * (T)0.5f;
            T phx = nx * cphi, phy = ny * cphi, phz = nz * cphi;
            Rij[k] = {nx, ny, nz};
            T M1x = (T)1.0f + tz * phz + ty * phy;
            T M1y = phz - tz - ty * phx;
            T M1z = -phy - tz * phx + ty;
            T M2x = tz - phz - tx * phy;
            T M2y = tz * phz + (T)1.0f + tx * phx;
            T M2z = -tz * phy + phx - tx;
            T M3x = -ty - tx * phz + phy;
            T M3y = -ty * phz + tx - phx;
            T M3z = ty * phy + tx * phx + (T)1.0f;
            T dwx = W[j] - W[i], dwy = W[j + N] - W[i + N], dwz = W[j + 2 * N] - W[i + 2 * N];
            // torsion moment
            {
                T c1 = nx * dwx + ny * dwy + nz * dwz;
                c1 *= p.dt * (T)0.5f * p.m_G * il;
                V3<T> o = Mijn[k];
                T mx = M1x * o.x + M1y * o.y + M1z * o.z + nx * c1;
                T my = M2x * o.x + M2y * o.y + M2z * o.z + ny * c1;
                T mz = M3x * o.x + M3y * o.y + M3z * o.z + nz * c1;
                Mijn[k] = {mx, my, mz};
                c1 = PI * p.b_r * p.b_r * p.b_r * p.b_r;
                msx += mx * c1; msy += my * c1; msz += mz * c1;
            }
            // bending moment (QUIRK Q1: the summed moment carries dt*E/(4 L0) twice)
            {
                T c1 = nx * dwx + ny * dwy + nz * dwz;
                T c2 = p.dt * (T)0.25f * p.m_E * il;
                V3<T> o = Mijt[k];
                T mx = M1x * o.x + M1y * o.y + M1z * o.z + (dwx - nx * c1) * c2;
                T my = M2x * o.x + M2y * o.y + M2z * o.z + (dwy - ny * c1) * c2;
                T mz = M3x * o.x + M3y * o.y + M3z * o.z + (dwz - nz * c1) * c2;
                Mijt[k] = {mx, my, mz};
                c2 *= PI * p.b_r * p.b_r * p.b_r * p.b_r;
                msx += mx * c2; msy += my * c2; msz += mz * c2;
            }
            // shear force and asymmetric moment
            {
                T hx = (T)0.5f * wsx, hy = (T)0.5f * wsy, hz = (T)0.5f * wsz;
                T vx = V[j] - V[i] - hy * rz + hz * ry;
                T vy = V[j + N] - V[i + N] - hz * rx + hx * rz;
                T vz = V[j + 2 * N] - V[i + 2 * N] - hx * ry + hy * rx;
                T c = nx * vx + ny * vy + nz * vz;
                V3<T> o = Oijt[k];
                T ox = (M1x * o.x + M1y * o.y + M1z * o.z) + (vx - nx * c) * p.dt;
                T oy = (M2x * o.x + M2y * o.y + M2z * o.z) + (vy - ny * c) * p.dt;
                T oz = (M3x * o.x + M3y * o.y + M3z * o.z) + (vz - nz * c) * p.dt;
                c = p.m_G * il;
                Mc = c;
                c *= p.b_r * p.b_r * PI;
                fsx += ox * c; fsy += oy * c; fsz += oz * c;
                Oijt[k] = {ox, oy, oz};
                msx += (T)0.5f * (ry * oz - rz * oy) * c;
                msy += (T)0.5f * (rz * ox - rx * oz) * c;
                msz += (T)0.5f * (rx * oy - ry * ox) * c;
            }
            // break check
            {
                V3<T> o = Oijt[k], mt = Mijt[k], mn = Mijn[k];
                Mc *= norm3(o.x, o.y, o.z);
                Sc += norm3(mt.x, mt.y, mt.z) * (T)4.0f * p.b_r;
                Mc += norm3(mn.x, mn.y, mn.z) * (T)2.0f * p.b_r;
                if (crit) { crit[2 * k] = Sc; crit[2 * k + 1] = Mc; }
                if ((Sc > p.m_Gcritn) || (Mc > p.m_Gcritt)) {
                    ILtype[k] = 0;
                    Oijt[k] = {0, 0, 0};
                    Mijn[k] = {0, 0, 0};
                    Mijt[k] = {0, 0, 0};
                    if (broke) broke[k] = 1;
                }
            }
        }
        F[i] += fsx; F[i + N] += fsy; F[i + 2 * N] += fsz;
        M[i] += msx; M[i + N] += msy; M[i + 2 * N] += msz;
    }
}

// d_CalculateForcesDEM_21 (:338-422) with dd_Calculate_fijn_ppHM_2 (:199-253),
// dd_Calculate_fijtmijt_ppHM_2 (:255-314), dd_Calculate_mijroll_ppHM_2 (:316-336).
template <class T>
void forces_21(const T* R, const T* V, const T* W, const id_t* IL, const uint8_t* ILtype,
               V3<T>* Oijt, T* F, T* M, uint64_t N, uint64_t K, const FP<T>& p) {
    const T m_E = p.hm_E, m_G = p.hm_G, rP = p.rP, mP = p.mP;
    for (uint64_t i = 0; i < N; ++i) {
        T fsx = 0, fsy = 0, fsz = 0, msx = 0, msy = 0, msz = 0;
        for (uint64_t s = 0; s < K; ++s) {
            uint64_t k = i * K + s;
            id_t j = IL[k];
            if (j != EMPTY && ILtype[k] == 0) {
                T rx = R[j] - R[i], ry = R[j + N] - R[i + N], rz = R[j + 2 * N] - R[i + 2 * N];
                T rijm = norm3(rx, ry, rz);
                T inv_rm = (T)1 / rijm;
                T nx = rx * inv_rm, ny = ry * inv_rm, nz = rz * inv_rm;
                if (rijm < (T)2.0f * rP) {
                    // normal force with damping
                    T c1 = std::sqrt(rP * std::fabs(rP - (T)0.5f * rijm));
                    T Kn = (T)2.0f * m_E * c1;
                    T Kt = (T)8.0f * m_G * c1;
                    T wsx = W[j] + W[i], wsy = W[j + N] + W[i + N], wsz = W[j + 2 * N] + W[i + 2 * N];
                    T vx = V[j] - V[i] + rP * (ny * wsz - nz * wsy);
                    T vy = V[j + N] - V[i + N] + rP * (nz * wsx - nx * wsz);
                    T vz = V[j + 2 * N] - V[i + 2 * N] + rP * (nx * wsy - ny * wsx);
                    T vn = nx * vx + ny * vy + nz * vz;
                    T fn = (rijm - (T)2.0f * rP) * Kn * two_thirds_t<T>();
                    c1 = (T)-1.8257f * p.p_A * vn * std::sqrt(Kn * (T)0.5f * mP);
                    fsx += nx * (fn + c1); fsy += ny * (fn + c1); fsz += nz * (fn + c1);
                    T vtx = vx - nx * vn, vty = vy - ny * vn, vtz = vz - nz * vn;
                    // tangential spring, Coulomb cap, damping
                    V3<T> o = Oijt[k];
                    T c = nx * o.x + ny * o.y + nz * o.z;
                    T ox = o.x - nx * c, oy = o.y - ny * c, oz = o.z - nz * c;
                    c = ox * ox + oy * oy + oz * oz;
                    if (c > 1e-18) {
                        c = (T)1 / c;
                        c *= o.x * o.x + o.y * o.y + o.z * o.z;
                        c = std::sqrt(c);
                        ox *= c; oy *= c; oz *= c;
                    }
                    ox += vtx * p.dt; oy += vty * p.dt; oz += vtz * p.dt;
                    T ftx = ox * Kt, fty = oy * Kt, ftz = oz * Kt;
                    T ftm = ftx * ftx + fty * fty + ftz * ftz;
                    if (ftm > p.m_mu * p.m_mu * fn * fn) {
                        c = p.m_mu * std::fabs(fn) * rsqrt_rn(ftm);
                        ftx *= c; fty *= c; ftz *= c;
                        c = (T)1 / Kt;
                        ox = ftx * c; oy = fty * c; oz = ftz * c;
                    } else {
                        c = (T)-1.8257f * p.p_A * std::sqrt(Kt * (T)0.5f * mP);
                        ftx += vtx * c; fty += vty * c; ftz += vtz * c;
                    }
                    Oijt[k] = {ox, oy, oz};
                    fsx += ftx; fsy += fty; fsz += ftz;
                    msx += (ny * ftz - nz * fty) * rP;
                    msy += (nz * ftx - nx * ftz) * rP;
                    msz += (nx * fty - ny * ftx) * rP;
                    // rolling friction; QUIRK: a (near-)zero spin clears the whole moment sum
                    T wx = W[i], wy = W[i + N], wz = W[i + 2 * N];
                    T wim = wx * wx + wy * wy + wz * wz;
                    if (wim > 1e-18) {
                        T cr = -p.m_muroll * std::fabs(fn) * rsqrt_rn(wim);
                        msx += wx * cr; msy += wy * cr; msz += wz * cr;
                    } else {
                        msx = 0; msy = 0; msz = 0;
                    }
                } else {
                    Oijt[k] = {0, 0, 0};
                }
            } else if (j == EMPTY) {
                Oijt[k] = {0, 0, 0};
            }
        }
        F[i] += fsx; F[i + N] += fsy; F[i + 2 * N] += fsz;
        M[i] += msx; M[i + N] += msy; M[i + 2 * N] += msz;
    }
}

// d_CalculateIncrementsDEM (md_calculateincrementsdem.cu:19-49)
template <class T>
void increments(const T* F, T* V, T* R, const T* M, T* W, uint64_t N, T dt_d_m, T dt, T dt_d_I) {
    for (uint64_t i = 0; i < N; ++i)
        for (int c = 0; c < 3; ++c) {
            uint64_t q = i + c * N;
            V[q] += F[q] * dt_d_m;
            R[q] += V[q] * dt;
            W[q] += M[q] * dt_d_I;
        }
}

// d_braziltest_simple2 (md_braziltest_simple2.cu:19-151). The reaction sums are
// returned in double in particle order (the reference sums per-thread floats in a
// block tree, then block partials in double on the host).
template <class T>
void brazil_platen(T* R, T* V, T* F, uint64_t N, V3<T> c, T RR, T Yt, T Yb, T Ytr, T Ybr, T vt, T Zcut,
                   double* sfb_out, double* sft_out) {
    double sfb = 0, sft = 0;
    for (uint64_t i = 0; i < N; ++i) {
        T rx = R[i] - c.x, ry = R[i + N], rz = R[i + 2 * N] - c.z;
        if (rx * rx + rz * rz < RR && rz < Zcut) {
            if (ry - Ytr > -1e-9) {
                T fy = F[i + N];
                if (fy > 0) {
                    sft += (double)fy;
                    T iv = V[i] * V[i] + V[i + 2 * N] * V[i + 2 * N];
                    if (iv > 1e-9) {
                        iv = rsqrt_rn(iv);
                        F[i] -= (T)0.45f * fy * V[i] * iv;
                        F[i + 2 * N] -= (T)0.45f * fy * V[i + 2 * N] * iv;
                    }
                }
                if (ry - Yt > -1e-9) { R[i + N] = Yt; V[i + N] = vt; F[i + N] = 0; }
            }
            if (ry - Ybr < 1e-9) {
                T fy = F[i + N];
                if (fy < 0) {
                    sfb += (double)fy;
                    T iv = V[i] * V[i] + V[i + 2 * N] * V[i + 2 * N];
                    if (iv > 1e-9) {
                        iv = rsqrt_rn(iv);
                        F[i] += (T)0.45f * fy * V[i] * iv;
                        F[i + 2 * N] += (T)0.45f * fy * V[i + 2 * N] * iv;
                    }
                }
                if (ry - Yb < 1e-9) { R[i + N] = Yb; V[i + N] = 0; F[i + N] = 0; }
            }
        }
    }
    *sfb_out = sfb; *sft_out = sft;
}

// d_UniaxialCompression3_simple (md_uniaxialcompression3_simple.cu:19-136)
template <class T>
void uniaxial_platen(T* R, T* V, T* F, uint64_t N, V3<T> c, T RR, T Zt, T Zb, T Ztr, T Zbr, T vt, T Zcut,
                     double* sfb_out, double* sft_out) {
    double sfb = 0, sft = 0;
    for (uint64_t i = 0; i < N; ++i) {
        T rx = R[i] - c.x, ry = R[i + N] - c.y, rz = R[i + 2 * N];
        if (rx * rx + ry * ry < RR && rz < Zcut) {
            if (rz - Ztr > -1e-9) {
                T fz = F[i + 2 * N];
                if (fz > 0) sft += (double)fz;
                if (rz - Zt > -1e-9) { R[i + 2 * N] = Zt; V[i + 2 * N] = vt; F[i + 2 * N] = 0; }
            }
            if (rz - Zbr < 1e-9) {
                T fz = F[i + 2 * N];
                if (fz < 0) sfb += (double)fz;
                if (rz - Zb < 1e-9) { R[i + 2 * N] = Zb; V[i + 2 * N] = 0; F[i + 2 * N] = 0; }
            }
        }
    }
    *sfb_out = sfb; *sft_out = sft;
}

// d_ParallelepipedCutRestriction (md_parallelepipedrestriction.cu:73-159)
template <class T>
void cut_restriction(T* R, T* V, T* F, uint64_t N, V3<T> center, V3<T> sized2, V3<T> hp) {
    for (uint64_t i = 0; i < N; ++i) {
        T dx = R[i] - center.x, dy = R[i + N] - center.y, dz = R[i + 2 * N] - center.z;
        bool out = (dx - sized2.x > 0) || (dx + sized2.x < 0) || (dy - sized2.y > 0) ||
                   (dy + sized2.y < 0) || (dz - sized2.z > 0) || (dz + sized2.z < 0);
        if (out) {
            R[i] = hp.x; R[i + N] = hp.y; R[i + 2 * N] = hp.z;
            V[i] = 0; V[i + N] = 0; V[i + 2 * N] = 0;
            F[i] = 0; F[i + N] = 0; F[i + 2 * N] = 0;
        }
    }
}

}  // namespace rfo

// ===========================================================================
// Host scalar logic, restated from md_data_types.h and md_results.cu.
// ===========================================================================
namespace rfo {
static const double MC_pi = 3.1415926535897932384626433832795;   // md_math_constants.h:44
static const double MC_1d3 = 1.0 / 3.0;                           // md_math_constants.h:15
static const double length_const = 1e-3;                          // md_phys_constants.h:5

// potential_data::CalculateParameters (md_data_types.h:153-185)
static void potential_params(rf_potential& P) {
    P.m_G = 0.5 * P.m_E / (1.0 + P.m_nu);
    P.b_S = MC_pi * P.b_r * P.b_r;
    P.p_V = 4.0 * MC_1d3 * MC_pi * P.p_r * P.p_r * P.p_r;
    P.p_m = P.m_ro * P.p_V;
    P.b_dd = P.b_d * P.b_d;
    P.p_1d_m = 1.0 / P.p_m;
    P.p_I = 0.4 * P.p_m * P.p_r * P.p_r;
    P.hm_E = 0.5 * P.m_E / (1.0 - P.m_nu * P.m_nu);
    P.hm_G = 0.5 * P.m_G / (2.0 - P.m_nu);
    P.p_A = std::log(P.p_e) / std::sqrt(MC_pi * MC_pi + std::log(P.p_e) * std::log(P.p_e));
    P.aa_farcut = P.a_farcut * P.a_farcut;
    P.Trayleigh = MC_pi * P.p_r * std::sqrt(2.0 * P.m_ro * (1.0 + P.m_nu)) /
                  (std::sqrt(P.m_E) * (0.163 * P.m_nu + 0.8766));
    double t0 = P.m_E * P.b_S / (2.0 * P.p_r), t1 = P.m_G * P.b_S / (2.0 * P.p_r);
    P.Tsim = (t0 > t1) ? 2.0 * std::sqrt(P.p_m / t0) : 2.0 * std::sqrt(P.p_m / t1);
    P.dt = (P.Trayleigh < P.Tsim) ? 0.1 * P.Trayleigh : 0.1 * P.Tsim;
    P.D = 1e-15 * P.m_E * P.b_S / (2.0 * P.p_r);
    P.a = (2.0 + 0 * 1e-6) * P.p_r;
    P._1d_a = 1.0 / P.a;
    P.aa = P.a * P.a;
    P.dt_d_m = P.p_1d_m * P.dt;
    P.dt_d_I = P.dt / P.p_I;
}

static int prepare(rf_task* t, const double ss[3], const double ls[3], double cell_a, double vload,
                   double minstress, double maxstrain) {
    rf_potential& P = t->Po;
    potential_params(P);
    rf_sample& S = t->S;
    rf_cells& C = t->C;
    C.a = (float)cell_a;
    // sample_data::SetSpaceSizeSi (:86-93), SetLSi (:94-100), CalculateParameters (:105-121)
    S.spacesize = {(float)(ss[0] / length_const), (float)(ss[1] / length_const), (float)(ss[2] / length_const)};
    S.spacesized2 = {(float)(0.5 * S.spacesize.x), (float)(0.5 * S.spacesize.y), (float)(0.5 * S.spacesize.z)};
    S.L = {(float)(ls[0] / length_const - 2.0 * P.p_r), (float)(ls[1] / length_const - 2.0 * P.p_r),
           (float)(ls[2] / length_const - 2.0 * P.p_r)};
    S.axis = {0.f, 0.f, 1.f};
    double C_a = (double)C.a, p_r = P.p_r;
    S.A = {(float)(1.01 * C_a), (float)(1.01 * C_a), (float)(1.01 * C_a)};
    S.B = {S.A.x + S.spacesize.x, S.A.y + S.spacesize.y, S.A.z + S.spacesize.z};
    S.center = {(float)(0.5 * (S.A.x + S.B.x)), (float)(0.5 * (S.A.y + S.B.y)), (float)(0.5 * (S.A.z + S.B.z))};
    S.size = S.L;
    S.sized2 = {(float)(0.5 * S.L.x), (float)(0.5 * S.L.y), (float)(0.5 * S.L.z)};
    S.R0 = (float)(0.5 * S.L.x);
    S.H0 = (float)(0.5 * S.L.z);
    S.Vext = MC_pi * (0.5 * S.L.x + p_r) * (0.5 * S.L.x + p_r) * (S.L.z + 2.0 * p_r);
    S.hidenpoint.x = (float)(S.A.x + 0.5 * S.spacesize.x);
    S.hidenpoint.y = (float)(S.A.y + 0.5 * S.spacesize.y);
    {
        float fl = std::floor((float)((double)S.B.z / C_a));
        float f3 = fl + 3.0f;
        S.hidenpoint.z = (float)(((double)f3 - 0.5) * C_a);
    }
    S.A_real = {(double)(float)(S.center.x - S.sized2.x), (double)(float)(S.center.y - S.sized2.y),
                (double)(float)(S.center.z - S.sized2.z)};
    S.B_real = {(double)(float)(S.center.x + S.sized2.x), (double)(float)(S.center.y + S.sized2.y),
                (double)(float)(S.center.z + S.sized2.z)};
    S.size_real = {S.B_real.x - S.A_real.x, S.B_real.y - S.A_real.y, S.B_real.z - S.A_real.z};
    S.center_real = {0.5 * (S.B_real.x + S.A_real.x), 0.5 * (S.B_real.y + S.A_real.y),
                     0.5 * (S.B_real.z + S.A_real.z)};
    S.Vgenmax = 0.f;
    // interaction_list_data::CalculateParameters (:137-143)
    t->acut = (float)P.a_farcut;
    t->aacut = t->acut * t->acut;
    // cell_data::CalculateParameters (:42-55), called with S.B (md_calculationbraziltest.cu:118)
    C._1d_a = (float)(1.0 / (double)C.a);
    C.Nr.x = (unsigned)(std::floor((float)((double)S.B.x * (double)C._1d_a)) + 1.0f);
    C.Nr.y = (unsigned)(std::floor((float)((double)S.B.y * (double)C._1d_a)) + 1.0f);
    C.Nr.z = (unsigned)(std::floor((float)((double)S.B.z * (double)C._1d_a)) + 3.0f);
    C.N = (uint64_t)C.Nr.x * C.Nr.y * C.Nr.z;
    C._1d_Nr = {(float)(1.0 / (double)C.Nr.x), (float)(1.0 / (double)C.Nr.y), (float)(1.0 / (double)C.Nr.z)};
    t->bloks = t->N / 1024 + 1;
    // compression_data::CalculateUParameters / CalculateBParameters (:196-271)
    rf_compression& K = t->Compress;
    std::memset(&K, 0, sizeof(K));
    K.VLoad = vload;
    K.size_d = S.size_real;
    K.size = {(float)K.size_d.x, (float)K.size_d.y, (float)K.size_d.z};
    K.sized2 = {(float)(0.5 * K.size_d.x), (float)(0.5 * K.size_d.y), (float)(0.5 * K.size_d.z)};
    K.center_d = S.center_real;
    K.center = {(float)K.center_d.x, (float)K.center_d.y, (float)K.center_d.z};
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
    // V and Strain are read before the driver first sets them; they start at 0 here.
    K.V = 0.0;
    K.Strain = 0.0;
    t->sz0 = (double)K.size.z;
    return 0;
}

// compression_data::CompressU / CompressB (md_data_types.h:223-293)
static void compress(rf_task* t, double pressure) {
    rf_compression& K = t->Compress;
    const rf_potential& P = t->Po;
    K.V = (pressure < 1e-9) ? 10.0 * K.VLoad : K.VLoad;
    if (t->kind == RF_TEST_UNIAXIAL) {
        K.size_d.z += K.V * P.dt;
        K.Top += K.V * P.dt;
        K.TopR = K.Top - 2.0 * P.p_r;
        K.size.z = (float)K.size_d.z;
        K.sized2.z = (float)(0.5 * K.size_d.z);
        K.center_d.z += K.V * P.dt;
        K.center.z = (float)K.center_d.z;
        K.Hd2 = K.sized2.z;
        K.Strain = (K.size_d.z - K.Size0) / K.Size0;
    } else {
        K.size_d.y += K.V * P.dt;
        K.Top += K.V * P.dt;
        K.TopR = K.Top - 2.0 * P.p_r;
        K.size.y = (float)K.size_d.y;
        K.sized2.y = (float)(0.5 * K.size_d.y);
        K.center_d.y += K.V * P.dt;
        K.center.y = (float)K.center_d.y;
        K.Hd2 = K.sized2.y;
        K.Strain = (K.size_d.y - K.Size0) / K.Size0;
    }
}

// SumForcesULoading (md_results.cu:34-74) given the two reaction sums; sz0 = R.sz0.
static void sum_forces(rf_task* t, double sfb, double sft, double sz0, double* curve, uint64_t cap,
                       uint64_t* nsaved) {
    rf_compression& K = t->Compress;
    if (curve && *nsaved < cap) {
        curve[3 * *nsaved + 0] = (K.size_d.z - sz0) / sz0;
        curve[3 * *nsaved + 1] = sfb * (double)K._1d_Area;
        curve[3 * *nsaved + 2] = sft * (double)K._1d_Area;
    }
    if (curve) ++*nsaved;
    K.Stress = 0.5 * (std::fabs(sfb) + std::fabs(sft)) * (double)K._1d_Area;
    if (!K.Loading && K.Stress > K.MinStress) K.Loading = 1;
    if (K.FractureStress < K.Stress) {
        K.FractureStress = K.Stress;
        K.FractureStrain = (sz0 - K.size_d.z) / sz0;
    }
    if (K.Loading && K.Stress < K.ZeroStress) K.Fracture = 1;
}

// One whole test (h_CalculationBrazilTest md_calculationbraziltest.cu:113-214 /
// h_CalculationUniaxialCompression md_calculationuniaxialcompression.cu:113-216).
// State vectors are passed in and out so a run can be split and compared step by step.
template <class T>
struct Run {
    rf_task* t;
    uint64_t N, K, CN;
    std::vector<T> R, V, W, F, M, iL;
    std::vector<id_t> IL, CI, CIs, pnC;
    std::vector<uint8_t> type, broke;
    std::vector<V3<T>> Rij, Oijt, Mijn, Mijt;
    double sz0;
    int status;
    uint64_t steps, broken;

    void init(const float* R0) {
        N = t->N; K = t->K; CN = t->C.N;
        R.assign(3 * N, 0); V.assign(3 * N, 0); W.assign(3 * N, 0); F.assign(3 * N, 0); M.assign(3 * N, 0);
        for (uint64_t q = 0; q < 3 * N; ++q) R[q] = (T)R0[q];
        iL.assign(N * K, 0); IL.assign(N * K, EMPTY); type.assign(N * K, 0); broke.assign(N * K, 0);
        Rij.assign(N * K, {0, 0, 0}); Oijt = Rij; Mijn = Rij; Mijt = Rij;
        CI.assign(N, 0); CIs.assign(2 * N, 0); pnC.assign(2 * CN, 0);
        sz0 = t->sz0 != 0.0 ? t->sz0 : (double)t->Compress.size.z;   // R.sz0 (md_results.cu:21)
        status = 0; steps = 0; broken = 0;
        T inv_a = (T)t->C._1d_a, a = (T)t->C.a, aacut = (T)t->aacut;
        int s = cell_distribution<T>(R.data(), N, CI.data(), CIs.data(), pnC.data(), CN, inv_a, t->C.Nr);
        if (s) status = s;
        s = construct_list<T>(R.data(), N, CIs.data(), pnC.data(), IL.data(), K, a, inv_a, aacut, t->C.Nr, CN);
        if (s) status = s;
        construct_bonds<T>(R.data(), N, IL.data(), type.data(), iL.data(), Rij.data(), Oijt.data(), Mijn.data(),
                           Mijt.data(), K, (T)(float)t->Po.b_dd);
        delete_far_links<T>(R.data(), N, IL.data(), type.data(), Rij.data(), Oijt.data(), Mijn.data(), Mijt.data(),
                            K, (T)(float)t->Po.aa_farcut);
    }

    FP<T> fparams() const {
        FP<T> p;
        const rf_potential& P = t->Po;
        p.dt = (T)(float)P.dt; p.m_E = (T)(float)P.m_E; p.m_G = (T)(float)P.m_G; p.b_r = (T)(float)P.b_r;
        p.m_Gcritn = (T)(float)P.m_Ec; p.m_Gcritt = (T)(float)P.m_Gc;
        p.hm_E = (T)(float)P.hm_E; p.hm_G = (T)(float)P.hm_G; p.p_A = (T)(float)P.p_A;
        p.m_mu = (T)(float)P.p_mu; p.m_muroll = (T)(float)P.p_mur; p.mP = (T)(float)P.p_m; p.rP = (T)(float)P.p_r;
        return p;
    }

    bool running() const {
        return t->Compress.Strain < t->Compress.MaxStrain && !t->Compress.Fracture;
    }

    // One pass of the loop body (md_calculationbraziltest.cu:170-190).
    void step(double* curve, uint64_t cap, uint64_t* nsaved) {
        const rf_potential& P = t->Po;
        rf_compression& Kc = t->Compress;
        T inv_a = (T)t->C._1d_a, a = (T)t->C.a, aacut = (T)t->aacut;
        int s = cell_distribution<T>(R.data(), N, CI.data(), CIs.data(), pnC.data(), CN, inv_a, t->C.Nr);
        if (s && !status) status = s;
        s = reconstruct_bpm<T>(R.data(), N, CIs.data(), pnC.data(), IL.data(), type.data(), K, a, inv_a, aacut,
                               t->C.Nr, CN);
        if (s && !status) status = s;
        std::fill(F.begin(), F.end(), (T)0);
        std::fill(M.begin(), M.end(), (T)0);
        FP<T> p = fparams();
        forces_22<T>(R.data(), V.data(), W.data(), IL.data(), type.data(), iL.data(), Rij.data(), Oijt.data(),
                     Mijn.data(), Mijt.data(), F.data(), M.data(), N, K, p, broke.data());
        forces_21<T>(R.data(), V.data(), W.data(), IL.data(), type.data(), Oijt.data(), F.data(), M.data(), N, K, p);
        double sfb = 0, sft = 0;
        V3<T> c = {(T)Kc.center.x, (T)Kc.center.y, (T)Kc.center.z};
        if (t->kind == RF_TEST_BRAZIL) {
            T Zcut = (T)(float)((double)t->S.center.y + (double)t->S.spacesized2.y);
            brazil_platen<T>(R.data(), V.data(), F.data(), N, c, (T)Kc.RR, (T)(float)Kc.Top, (T)(float)Kc.Bottom,
                             (T)(float)Kc.TopR, (T)(float)Kc.BottomR, (T)(float)Kc.V, Zcut, &sfb, &sft);
        } else {
            T Zcut = (T)(float)((double)t->S.center.z + (double)t->S.spacesized2.z);
            uniaxial_platen<T>(R.data(), V.data(), F.data(), N, c, (T)Kc.RR, (T)(float)Kc.Top, (T)(float)Kc.Bottom,
                               (T)(float)Kc.TopR, (T)(float)Kc.BottomR, (T)(float)Kc.V, Zcut, &sfb, &sft);
        }
        sum_forces(t, sfb, sft, sz0, curve, cap, nsaved);
        increments<T>(F.data(), V.data(), R.data(), M.data(), W.data(), N, (T)(float)P.dt_d_m, (T)(float)P.dt,
                      (T)(float)P.dt_d_I);
        const rf_sample& S = t->S;
        cut_restriction<T>(R.data(), V.data(), F.data(), N, {(T)S.center.x, (T)S.center.y, (T)S.center.z},
                           {(T)S.spacesized2.x, (T)S.spacesized2.y, (T)S.spacesized2.z},
                           {(T)S.hidenpoint.x, (T)S.hidenpoint.y, (T)S.hidenpoint.z});
        delete_far_links<T>(R.data(), N, IL.data(), type.data(), Rij.data(), Oijt.data(), Mijn.data(), Mijt.data(),
                            K, (T)(float)P.aa_farcut);
        compress(t, Kc.Stress);
        ++steps;
    }
};
}  // namespace rfo

// ===========================================================================
// Extended model (polydisperse, FP64 positions, per-bond strengths). This model has
// no counterpart in the reference: it is the engine's own, and each formula is the
// reference's with the mono-sized constants replaced (E/L0 -> kn, G/L0 -> ks,
// b_r -> lambda*min(r_i, r_j), 2 r_P -> r_i + r_j, r_P(r_P - r/2) -> R* delta,
// m_P/2 -> m*, lever arm r_P -> r_i). The loop is the reference's
// (md_calculationbraziltest.cu:170-190) with DeleteFarLinks moved to the start of
// the next step (same positions) and all distance tests on the FP64 positions.
// TF = float restates the engine's arithmetic operation for operation (bit-exact
// target); TF = double is the FP64 oracle of the same model.
// ===========================================================================
namespace rfo {

template <class T> static inline T rcp(T x) { return (T)1 / x; }

struct ExtPar {
    double kn, ks, lambda, gap, wm, sig, tau;
    uint64_t seed;
    double drop;      // post-peak stop: fracture once the stress is below (1 - drop) x peak (0: off)
    double lgap;      // list gap: 0 lists pairs within a_farcut; g > 0 within min(a_farcut, r_i + r_j + g)
    int ref;          // reference constants (rf_ext_params.ref_mode): b_d bond rule, b_r, E/L0, G/L0,
                      // global strengths, the Q1 bending factor (md_calculateforcesdem3.cu:131-152)
};
static inline ExtPar ext_par(const rf_ext_params* xp) {
    return ExtPar{xp->kn, xp->ks, xp->bond_lambda, xp->gap_frac, xp->weibull_m, xp->sigma_c, xp->tau_c, xp->seed,
                  xp->post_peak_drop, xp->list_gap, xp->ref_mode};
}

static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Uniform in (0, 1) keyed on the unordered pair (a, b) and a stream number.
static inline double pair_uniform(uint64_t seed, uint64_t a, uint64_t b, uint32_t stream) {
    const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
    const uint64_t h = mix64(mix64(seed ^ (0x51ED270B27F3A4C1ull * (stream + 1))) + (hi << 32 | lo));
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// Bond state inside a quasi-static increment: carried from the increment's start state to
// the current configuration (1, bond_total: the engine's FIRE mode) or integrated iteration
// by iteration (0, the explicit steps' rule; kept for comparison).
static int g_qs_total = 1;

// Positions kept as hi/lo pairs of floats (x = hi + lo, |lo| at most half an ulp of hi)
// instead of doubles: a double is rounded to the nearest such pair, and an increment is
// added with float operations only (Knuth's two-sum of hi and the increment, the error
// folded into lo, Dekker's fast two-sum to renormalise). Every pair is a double exactly.
static inline double hilo_round(double x) {
    const float h = (float)x;
    const float l = (float)(x - (double)h);
    return (double)h + (double)l;
}
static inline double hilo_add(double x, float d) {
    const float h = (float)x;
    const float l = (float)(x - (double)h);
    const float s = h + d;
    const float bb = s - h;
    const float e = (h - (s - bb)) + (d - bb);
    const float t = l + e;
    const float hi = s + t;
    const float lo = t - (hi - s);
    return (double)hi + (double)lo;
}

template <class TF>
struct RunExt {
    int pos_mode = 0;           // positions as doubles (0), hi/lo float pairs (1, see hilo_add) or floats (2)
    // host threads of the per-particle loops (OpenMP). 1: serial, in particle order; more
    // threads reorder only the FP64 platen and force-magnitude sums, so they are for timing
    int nthreads = 1;
    rf_task* t;
    ExtPar x;
    uint64_t N, K, CN;
    std::vector<double> R, rad, L0, sig, tau;
    std::vector<TF> iL0;        // 1 / rest length per slot (reference constants: stiffness E/L0, G/L0)
    std::vector<float> Rf;
    std::vector<TF> V, W;
    std::vector<id_t> IL, CI, CIs, pnC;
    std::vector<uint8_t> type;
    std::vector<V3<TF>> Rij, Oijt, Mijn, Mijt;
    // tangential overlap of the contact an overlapping bonded pair carries in parallel with
    // its bond (the extended model; the reference constants have none); it becomes the
    // slot's contact state (Oijt) when the bond breaks
    std::vector<V3<TF>> Ocb;
    // bond state at the start of a quasi-static increment; during the increment's FIRE
    // iterations (qs_total) a bond's state is computed from it and the motion since then
    std::vector<V3<TF>> Rij0, Oijt0, Mijn0, Mijt0;
    bool qs_total = false;
    // inside a quasi-static increment's FIRE iterations a particle held by a platen does
    // not slide along it either (the platens hold what they touch; this removes the
    // specimen's rigid tilting and sliding, which would leave FIRE without a minimum)
    bool in_fire = false;
    double sz0, aa_farcut, aacut, a_farcut;
    int status;
    uint64_t steps, broken;
    TF dt, hm_E, hm_G, p_A, mu, mur, kn, ks, lambda, cmass;
    TF mE, mG, b_r;             // the task's moduli and bond radius (reference constants)

    void to_float() {
        for (uint64_t q = 0; q < 3 * N; ++q) Rf[q] = (float)R[q];
    }
    double rr(uint64_t i, uint64_t j) const {
        const double dx = R[j] - R[i], dy = R[j + N] - R[i + N], dz = R[j + 2 * N] - R[i + 2 * N];
        return dx * dx + dy * dy + dz * dz;
    }
    // squared list cutoffs of a pair (add and delete tests): the reference's float aacut
    // and double aa_farcut, or with a list gap min(a_farcut, r_i + r_j + g)^2 for both
    double cut2_add(uint64_t i, uint64_t j) const {
        if (x.lgap > 0.0) { const double q = std::fmin(a_farcut, (rad[i] + rad[j]) + x.lgap); return q * q; }
        return aacut;
    }
    double cut2_del(uint64_t i, uint64_t j) const {
        if (x.lgap > 0.0) { const double q = std::fmin(a_farcut, (rad[i] + rad[j]) + x.lgap); return q * q; }
        return aa_farcut;
    }
    void zero_slot(uint64_t k) {
        Rij[k] = {0, 0, 0}; Oijt[k] = {0, 0, 0}; Mijn[k] = {0, 0, 0}; Mijt[k] = {0, 0, 0}; Ocb[k] = {0, 0, 0};
    }

    void init(const double* R0, const double* r0) {
        N = t->N; K = t->K; CN = t->C.N;
        R.assign(R0, R0 + 3 * N); rad.assign(r0, r0 + N); Rf.assign(3 * N, 0.f);
        if (pos_mode == 1)
            for (double& v : R) v = hilo_round(v);
        if (pos_mode == 2)
            for (double& v : R) v = (double)(float)v;
        V.assign(3 * N, 0); W.assign(3 * N, 0);
        IL.assign(N * K, EMPTY); type.assign(N * K, 0); L0.assign(N * K, 1.0); sig.assign(N * K, 0.0);
        tau.assign(N * K, 0.0); iL0.assign(N * K, (TF)0);
        Rij.assign(N * K, {0, 0, 0}); Oijt = Rij; Mijn = Rij; Mijt = Rij; Ocb = Rij;
        CI.assign(N, 0); CIs.assign(2 * N, 0); pnC.assign(2 * CN, 0);
        sz0 = t->sz0 != 0.0 ? t->sz0 : (double)t->Compress.size.z;
        status = 0; steps = 0; broken = 0;
        const rf_potential& P = t->Po;
        dt = (TF)P.dt; hm_E = (TF)P.hm_E; hm_G = (TF)P.hm_G; p_A = (TF)P.p_A; mu = (TF)P.p_mu; mur = (TF)P.p_mur;
        kn = (TF)x.kn; ks = (TF)x.ks; lambda = (TF)x.lambda; cmass = (TF)(P.p_m / (P.p_r * P.p_r * P.p_r));
        mE = (TF)P.m_E; mG = (TF)P.m_G; b_r = (TF)P.b_r;
        aa_farcut = P.aa_farcut; aacut = (double)t->aacut; a_farcut = P.a_farcut;
        to_float();
        const float inv_a = t->C._1d_a, a = t->C.a;
        int s = cell_distribution<float>(Rf.data(), N, CI.data(), CIs.data(), pnC.data(), CN, inv_a, t->C.Nr);
        if (s) status = s;
        if (x.lgap > 0.0) s = construct_list_pairs();
        else s = construct_list<float>(Rf.data(), N, CIs.data(), pnC.data(), IL.data(), K, a, inv_a, t->aacut,
                                       t->C.Nr, CN);
        if (s) status = s;
        // bonds: gap below gap_frac * min radius; FP64 rest length; Weibull strengths per pair.
        // With the reference constants: centre distance below b_d (md_boundinteractions_construct.cu:62,
        // here on the FP64 distance), the global strengths m_Ec and m_Gc.
        for (uint64_t i = 0; i < N; ++i)
            for (uint64_t q = 0; q < K; ++q) {
                const uint64_t k = i * K + q;
                const id_t j = IL[k];
                if (j == EMPTY || j >= N) continue;
                const double dx = R[j] - R[i], dy = R[j + N] - R[i + N], dz = R[j + 2 * N] - R[i + 2 * N];
                const double L = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (x.ref) {
                    if (!(L < P.b_d) || !(L > 0)) continue;
                } else if (!(L - rad[i] - rad[j] < x.gap * std::fmin(rad[i], rad[j])) || !(L > 0)) {
                    continue;
                }
                type[k] = 1;
                L0[k] = L;
                iL0[k] = (TF)(1.0 / L);
                if (x.ref) {
                    sig[k] = P.m_Ec; tau[k] = P.m_Gc;
                } else {
                    const double us = pair_uniform(x.seed, i, j, 0), ut = pair_uniform(x.seed, i, j, 1);
                    sig[k] = x.sig * std::pow(-std::log(us), 1.0 / x.wm);
                    tau[k] = x.tau * std::pow(-std::log(ut), 1.0 / x.wm);
                }
                if (sizeof(TF) == 4) { sig[k] = (float)sig[k]; tau[k] = (float)tau[k]; }
            }
        // DeleteFarLinks on the float positions, as the initial build does (with a list gap
        // every listed pair is within its cutoff)
        if (!(x.lgap > 0.0)) {
            std::vector<V3<float>> z(N * K, {0, 0, 0});
            delete_far_links<float>(Rf.data(), N, IL.data(), type.data(), z.data(), z.data(), z.data(), z.data(), K,
                                    (float)P.aa_farcut);
        }
    }

    // construct_list's visiting order (the reference's initial construction) with the pair
    // cutoff min(a_farcut, r_i + r_j + g) tested on the FP64 positions
    int construct_list_pairs() {
        int st = ST_OK;
        std::fill(IL.begin(), IL.end(), EMPTY);
        const float inv_a = t->C._1d_a, a = t->C.a;
        for (uint64_t i = 0; i < N; ++i) {
            int64_t cells[8];
            octant_cells<float>(Rf.data(), N, i, a, inv_a, t->C.Nr, cells);
            uint64_t n = 0;
            for (int c = 0; c < 8; ++c) {
                if (cells[c] < 0 || (uint64_t)cells[c] >= CN) { st = ST_CELL_RANGE; continue; }
                const uint64_t start = pnC[cells[c]], cnt = pnC[cells[c] + CN];
                for (uint64_t m = 0; m < cnt; ++m) {
                    if (start + m >= N) break;
                    const id_t j = CIs[start + m + N];
                    if (j >= N) continue;
                    if (rr(i, j) < cut2_add(i, j) && j != i) {
                        if (n < K) IL[i * K + n] = j; else st = ST_ROW_OVERFLOW;
                        ++n;
                    }
                }
            }
        }
        return st;
    }

    void delete_far() {
#pragma omp parallel for schedule(static) if (nthreads > 1) num_threads(nthreads)
        for (uint64_t i = 0; i < N; ++i)
            for (uint64_t q = 0; q < K; ++q) {
                const uint64_t k = i * K + q;
                const id_t j = IL[k];
                if (j == EMPTY || j >= N) continue;
                const double d2 = rr(i, j);
                // an intact bond of the extended model is kept up to 1.45 L0 (the
                // reference's a_farcut / 2 p_r); the reference constants keep its rule
                double cut = cut2_del(i, j);
                if (type[k] == 1 && !x.ref) { const double q = 1.45 * L0[k]; cut = q * q; }
                if (d2 > cut || d2 < 1e-10) { IL[k] = EMPTY; type[k] = 0; zero_slot(k); }
            }
    }

    void add_links() {
        to_float();
        const float inv_a = t->C._1d_a, a = t->C.a;
        int s = cell_distribution<float>(Rf.data(), N, CI.data(), CIs.data(), pnC.data(), CN, inv_a, t->C.Nr);
        if (s && !status) status = s;
        int overflow = 0;
#pragma omp parallel for schedule(static) reduction(| : overflow) if (nthreads > 1) num_threads(nthreads)
        for (uint64_t i = 0; i < N; ++i) {
            int64_t cells[8];
            octant_cells<float>(Rf.data(), N, i, a, inv_a, t->C.Nr, cells);
            for (int c = 0; c < 8; ++c) {
                if (cells[c] < 0 || (uint64_t)cells[c] >= CN) continue;
                const uint64_t start = pnC[cells[c]], cnt = pnC[cells[c] + CN];
                for (uint64_t m = 0; m < cnt && start + m < N; ++m) {
                    const id_t j = CIs[start + m + N];
                    if (j >= N) continue;
                    const double d2 = rr(i, j);
                    if (!(d2 < cut2_add(i, j) && d2 > 1e-10)) continue;
                    bool have = false;
                    for (uint64_t q = 0; q < K; ++q) if (IL[i * K + q] == j) have = true;
                    if (have) continue;
                    int64_t kf = -1;
                    for (uint64_t q = 0; q < K; ++q)
                        if (IL[i * K + q] == EMPTY) {
                            // QUIRK (md_interaction_list_reconstructbpm.cu:30-36): particle 0 skips a
                            // free slot 0 while a later free slot exists
                            if (i == 0 && q == 0) {
                                bool later = false;
                                for (uint64_t u = 1; u < K; ++u) if (IL[u] == EMPTY) later = true;
                                if (later) continue;
                            }
                            kf = (int64_t)q;
                            break;
                        }
                    if (kf < 0) { overflow = 1; continue; }
                    IL[i * K + kf] = j;
                    type[i * K + kf] = 0;
                }
            }
        }
        if (overflow && !status) status = ST_ROW_OVERFLOW;
    }

    // The extended model's arithmetic is written with explicit fused multiply-adds, as the
    // engine's (rf_physics.cuh: fm, dot3, bond_core, contact_pair_ext); std::fma is the same
    // correctly rounded operation, so the float instance stays bit-exact with the engine.
    static TF fm(TF a, TF b, TF c) { return std::fma(a, b, c); }
    static TF dot3(TF ax, TF ay, TF az, TF bx, TF by, TF bz) { return fm(ax, bx, fm(ay, by, az * bz)); }
    static TF len_sq(double rr) { return std::sqrt((TF)rr); }
    static TF stretch_sq(double rr, double L0, TF rlen) { return (TF)std::fma(-L0, L0, rr) * rcp(rlen + (TF)L0); }

    // engine bond_core: the bond update shared by the explicit step (dts = dt, rates) and
    // the quasi-static total (dts = 1, displacements); Rp, Ot0, Mn0, Mt0 the state it
    // starts from, results into slot k. kt, kr, fnabs: the particle's float accumulators.
    bool bond_core(uint64_t k, TF kn, TF ks, TF br, const V3<TF>& r, TF rlen, TF stretch, TF dts, V3<TF> Rp,
                   V3<TF> ws, V3<TF> dw, V3<TF> du, V3<TF> Ot0, V3<TF> Mn0, V3<TF> Mt0, V3<TF>& fs, V3<TF>& ms,
                   TF& fnabs, TF& kt, TF& kr, bool q1) {
        const TF PI = pi_t<TF>();
        const TF inv_rm = rcp(rlen);
        const TF nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
        const TF A = br * br * PI;
        const TF J = A * (br * br);
        kt = fm(kn + ks, A, kt);
        kr = fm((TF)0.25f * ks * A, rlen * rlen, fm(fm((TF)0.25f, kn, (TF)0.5f * ks), J, kr));
        const TF Sn = kn * stretch;
        const TF cef = Sn * A;
        fnabs += std::fabs(cef);
        fs.x = fm(nx, cef, fs.x); fs.y = fm(ny, cef, fs.y); fs.z = fm(nz, cef, fs.z);
        const TF tx = fm(Rp.y, nz, -(Rp.z * ny)), ty = fm(Rp.z, nx, -(Rp.x * nz)), tz = fm(Rp.x, ny, -(Rp.y * nx));
        const TF cphi = dot3(ws.x, ws.y, ws.z, nx, ny, nz) * (dts * (TF)0.5f);
        const TF phx = nx * cphi, phy = ny * cphi, phz = nz * cphi;
        Rij[k] = {nx, ny, nz};
        const TF one = (TF)1.0f;
        const TF M1x = fm(tz, phz, fm(ty, phy, one)), M1y = fm(-ty, phx, phz - tz), M1z = fm(-tz, phx, ty - phy);
        const TF M2x = fm(-tx, phy, tz - phz), M2y = fm(tz, phz, fm(tx, phx, one)), M2z = fm(-tz, phy, phx - tx);
        const TF M3x = fm(-tx, phz, phy - ty), M3y = fm(-ty, phz, tx - phx), M3z = fm(ty, phy, fm(tx, phx, one));
        const TF c1 = dot3(nx, ny, nz, dw.x, dw.y, dw.z);
        {
            const TF ct = c1 * (dts * (TF)0.5f * ks);
            const TF mx = fm(M1x, Mn0.x, fm(M1y, Mn0.y, fm(M1z, Mn0.z, nx * ct)));
            const TF my = fm(M2x, Mn0.x, fm(M2y, Mn0.y, fm(M2z, Mn0.z, ny * ct)));
            const TF mz = fm(M3x, Mn0.x, fm(M3y, Mn0.y, fm(M3z, Mn0.z, nz * ct)));
            Mijn[k] = {mx, my, mz};
            ms.x = fm(mx, J, ms.x); ms.y = fm(my, J, ms.y); ms.z = fm(mz, J, ms.z);
        }
        {
            const TF c2 = dts * (TF)0.25f * kn;
            const TF mx = fm(M1x, Mt0.x, fm(M1y, Mt0.y, fm(M1z, Mt0.z, fm(-nx, c1, dw.x) * c2)));
            const TF my = fm(M2x, Mt0.x, fm(M2y, Mt0.y, fm(M2z, Mt0.z, fm(-ny, c1, dw.y) * c2)));
            const TF mz = fm(M3x, Mt0.x, fm(M3y, Mt0.y, fm(M3z, Mt0.z, fm(-nz, c1, dw.z) * c2)));
            Mijt[k] = {mx, my, mz};
            const TF q = q1 ? c2 * J : J;       // Q1 (md_calculateforcesdem3.cu:131-152) with the reference constants
            ms.x = fm(mx, q, ms.x); ms.y = fm(my, q, ms.y); ms.z = fm(mz, q, ms.z);
        }
        TF Mc;
        {
            const TF c = dot3(nx, ny, nz, du.x, du.y, du.z);
            const TF ox = fm(M1x, Ot0.x, fm(M1y, Ot0.y, fm(M1z, Ot0.z, fm(-nx, c, du.x) * dts)));
            const TF oy = fm(M2x, Ot0.x, fm(M2y, Ot0.y, fm(M2z, Ot0.z, fm(-ny, c, du.y) * dts)));
            const TF oz = fm(M3x, Ot0.x, fm(M3y, Ot0.y, fm(M3z, Ot0.z, fm(-nz, c, du.z) * dts)));
            Oijt[k] = {ox, oy, oz};
            const TF kk = ks * A;
            fs.x = fm(ox, kk, fs.x); fs.y = fm(oy, kk, fs.y); fs.z = fm(oz, kk, fs.z);
            const TF hk = (TF)0.5f * kk;
            ms.x = fm(fm(r.y, oz, -(r.z * oy)), hk, ms.x);
            ms.y = fm(fm(r.z, ox, -(r.x * oz)), hk, ms.y);
            ms.z = fm(fm(r.x, oy, -(r.y * ox)), hk, ms.z);
            Mc = ks * std::sqrt(dot3(ox, oy, oz, ox, oy, oz));
        }
        const V3<TF>& Mt = Mijt[k];
        const V3<TF>& Mn = Mijn[k];
        const TF Sc = fm(std::sqrt(dot3(Mt.x, Mt.y, Mt.z, Mt.x, Mt.y, Mt.z)), (TF)4.0f * br, Sn);
        Mc = fm(std::sqrt(dot3(Mn.x, Mn.y, Mn.z, Mn.x, Mn.y, Mn.z)), (TF)2.0f * br, Mc);
        if ((Sc > (TF)sig[k]) || (Mc > (TF)tau[k])) {
            Oijt[k] = {0, 0, 0}; Mijn[k] = {0, 0, 0}; Mijt[k] = {0, 0, 0};
            return true;
        }
        return false;
    }

    // One bond slot in an explicit step (engine bond_slot_ext). With the reference constants
    // the stiffness per area is E/L0 and G/L0 of the slot (the reference's E*_1d_iL,
    // G*_1d_iL) and the bending moment carries the extra dt*E/(4 L0) factor.
    bool bond(uint64_t k, const V3<TF>& r, double rr, const V3<TF>& vi, const V3<TF>& vj, const V3<TF>& wi,
              const V3<TF>& wj, TF br, V3<TF>& fs, V3<TF>& ms, TF& fnabs, TF& kt, TF& kr) {
        const TF kn_ = x.ref ? mE * iL0[k] : kn;
        const TF ks_ = x.ref ? mG * iL0[k] : ks;
        const TF rlen = len_sq(rr);
        const TF stretch = stretch_sq(rr, L0[k], rlen);
        const V3<TF> ws = {wj.x + wi.x, wj.y + wi.y, wj.z + wi.z};
        const V3<TF> dw = {wj.x - wi.x, wj.y - wi.y, wj.z - wi.z};
        const TF hx = (TF)0.5f * ws.x, hy = (TF)0.5f * ws.y, hz = (TF)0.5f * ws.z;
        const V3<TF> du = {fm(hz, r.y, fm(-hy, r.z, vj.x - vi.x)), fm(hx, r.z, fm(-hz, r.x, vj.y - vi.y)),
                           fm(hy, r.x, fm(-hx, r.y, vj.z - vi.z))};
        return bond_core(k, kn_, ks_, br, r, rlen, stretch, dt, Rij[k], ws, dw, du, Oijt[k], Mijn[k], Mijt[k], fs,
                         ms, fnabs, kt, kr, x.ref != 0);
    }

    // One bond slot inside a quasi-static increment (engine bond_slot_ext_total): the
    // increment's start state carried to the current configuration in one step -- start
    // normal Rij0 to the current normal, the particles' rotations ti, tj and the pair's
    // relative motion since the increment began less the mean rotation's part,
    // du = (r - r0) - ((ti + tj) / 2) x r, formed in double by the caller (in float its
    // terms cancel and the relaxation stalls on the rounding) -- so the state depends on
    // where the particles are, not on the path the relaxation took to get there.
    bool bond_total(uint64_t k, const V3<TF>& r, double rr, const V3<TF>& du, const V3<TF>& ti, const V3<TF>& tj,
                    TF br, V3<TF>& fs, V3<TF>& ms, TF& fnabs, TF& kt, TF& kr) {
        const TF rlen = len_sq(rr);
        const TF stretch = stretch_sq(rr, L0[k], rlen);
        const V3<TF> ws = {tj.x + ti.x, tj.y + ti.y, tj.z + ti.z};
        const V3<TF> dw = {tj.x - ti.x, tj.y - ti.y, tj.z - ti.z};
        return bond_core(k, kn, ks, br, r, rlen, stretch, (TF)1.0f, Rij0[k], ws, dw, du, Oijt0[k], Mijn0[k],
                         Mijt0[k], fs, ms, fnabs, kt, kr, false);
    }

    // One overlapping pair (engine contact_pair_ext): rr = |r|^2 and sr = r_i + r_j in
    // double with rr < sr^2; the overlap is (sr^2 - rr) / (sr + |r|). Returns true when the
    // zero-spin rule of the rolling resistance cleared the moment sum ms.
    bool contact(uint64_t k, const V3<TF>& r, double rr, double sr, TF ri, TF rj, TF mi, TF mj, const V3<TF>& vi,
                 const V3<TF>& vj, const V3<TF>& wi, const V3<TF>& wj, V3<TF>& fs, V3<TF>& ms, TF& fnabs, TF& kt,
                 TF& kr) {
        const TF rijm = len_sq(rr);
        const TF delta = (TF)std::fma(sr, sr, -rr) * rcp((TF)sr + rijm);
        const TF inv_rm = rcp(rijm);
        const TF nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
        const TF Rs = ri * rj * rcp(ri + rj);
        const TF ms_ = mi * mj * rcp(mi + mj);
        const TF c0 = std::sqrt(Rs * delta);
        const TF Kn = (TF)2.0f * hm_E * c0;
        const TF Kt = (TF)8.0f * hm_G * c0;
        kt += Kn + Kt;
        kr = fm(Kt, ri * ri, kr);
        const TF ax = fm(ri, wi.x, rj * wj.x), ay = fm(ri, wi.y, rj * wj.y), az = fm(ri, wi.z, rj * wj.z);
        const TF vx = fm(ny, az, fm(-nz, ay, vj.x - vi.x));
        const TF vy = fm(nz, ax, fm(-nx, az, vj.y - vi.y));
        const TF vz = fm(nx, ay, fm(-ny, ax, vj.z - vi.z));
        const TF vn = dot3(nx, ny, nz, vx, vy, vz);
        const TF fn = -delta * Kn * two_thirds_t<TF>();
        fnabs += std::fabs(fn);
        const TF fnd = fm((TF)-1.8257f * p_A * vn, std::sqrt(Kn * ms_), fn);
        fs.x = fm(nx, fnd, fs.x); fs.y = fm(ny, fnd, fs.y); fs.z = fm(nz, fnd, fs.z);
        const TF vtx = fm(-nx, vn, vx), vty = fm(-ny, vn, vy), vtz = fm(-nz, vn, vz);
        const V3<TF> o = Oijt[k];
        TF c = dot3(nx, ny, nz, o.x, o.y, o.z);
        TF ox = fm(-nx, c, o.x), oy = fm(-ny, c, o.y), oz = fm(-nz, c, o.z);
        c = dot3(ox, oy, oz, ox, oy, oz);
        if ((double)c > 1e-18) {
            c = std::sqrt(dot3(o.x, o.y, o.z, o.x, o.y, o.z) * rcp(c));
            ox *= c; oy *= c; oz *= c;
        }
        ox = fm(vtx, dt, ox); oy = fm(vty, dt, oy); oz = fm(vtz, dt, oz);
        TF ftx = ox * Kt, fty = oy * Kt, ftz = oz * Kt;
        const TF ftm = dot3(ftx, fty, ftz, ftx, fty, ftz);
        const TF fmax = mu * fn;
        if (ftm > fmax * fmax) {
            c = mu * std::fabs(fn) * rsqrt_rn<TF>(ftm);
            ftx *= c; fty *= c; ftz *= c;
            c = rcp(Kt);
            ox = ftx * c; oy = fty * c; oz = ftz * c;
        } else {
            c = (TF)-1.8257f * p_A * std::sqrt(Kt * ms_);
            ftx = fm(vtx, c, ftx); fty = fm(vty, c, fty); ftz = fm(vtz, c, ftz);
        }
        Oijt[k] = {ox, oy, oz};
        fs.x += ftx; fs.y += fty; fs.z += ftz;
        ms.x = fm(fm(ny, ftz, -(nz * fty)), ri, ms.x);
        ms.y = fm(fm(nz, ftx, -(nx * ftz)), ri, ms.y);
        ms.z = fm(fm(nx, fty, -(ny * ftx)), ri, ms.z);
        if (mur != (TF)0) {
            const TF wim = dot3(wi.x, wi.y, wi.z, wi.x, wi.y, wi.z);
            if ((double)wim > 1e-18) {
                const TF cr = -mur * std::fabs(fn) * rsqrt_rn<TF>(wim);
                ms.x = fm(wi.x, cr, ms.x); ms.y = fm(wi.y, cr, ms.y); ms.z = fm(wi.z, cr, ms.z);
            } else {
                ms = {0, 0, 0};    // QUIRK (md_calculateforcesdem3.cu:316-336): clears the contact sum
                return true;
            }
        }
        return false;
    }

    bool running() const { return t->Compress.Strain < t->Compress.MaxStrain && !t->Compress.Fracture; }

    // rf_engine_affine_strain: positions scaled by 1 + e per axis about the platen box's
    // centre, the load axis's platens with them, the platen zone by the larger lateral strain.
    void affine(double ex, double ey, double ez) {
        rf_compression& Kc = t->Compress;
        const double cx = Kc.center_d.x, cy = Kc.center_d.y, cz = Kc.center_d.z;
        for (uint64_t i = 0; i < N; ++i) {
            R[i] = cx + (1.0 + ex) * (R[i] - cx);
            R[i + N] = cy + (1.0 + ey) * (R[i + N] - cy);
            R[i + 2 * N] = cz + (1.0 + ez) * (R[i + 2 * N] - cz);
        }
        const bool brz = t->kind == RF_TEST_BRAZIL;
        const double e = brz ? ey : ez, el = brz ? std::fmax(ex, ez) : std::fmax(ex, ey);
        const double ca = brz ? Kc.center_d.y : Kc.center_d.z;
        const double dtr = Kc.TopR - Kc.Top, dbr = Kc.BottomR - Kc.Bottom;
        Kc.Top = ca + (1.0 + e) * (Kc.Top - ca);
        Kc.Bottom = ca + (1.0 + e) * (Kc.Bottom - ca);
        Kc.TopR = Kc.Top + dtr;
        Kc.BottomR = Kc.Bottom + dbr;
        double* sz = brz ? &Kc.size_d.y : &Kc.size_d.z;
        *sz *= 1.0 + e;
        if (brz) { Kc.size.y = (float)*sz; Kc.sized2.y = (float)(0.5 * *sz); Kc.Hd2 = Kc.sized2.y; }
        else { Kc.size.z = (float)*sz; Kc.sized2.z = (float)(0.5 * *sz); Kc.Hd2 = Kc.sized2.z; }
        Kc.Strain = (*sz - Kc.Size0) / Kc.Size0;
        Kc.RR = (float)((double)Kc.RR * (1.0 + el) * (1.0 + el));
    }

    // Forces and moments of every particle (the _22 then _21 slot orders), and the sums
    // of |normal pair force| and of the pair count over bonds and overlapping contacts.
    void pair_forces(std::vector<V3<TF>>& Fn, std::vector<V3<TF>>& Mn, double& fnsum, double& npair,
                     std::vector<double>* KT = nullptr, std::vector<double>* KR = nullptr) {
        fnsum = 0; npair = 0;
        double fs_ = 0, np_ = 0;
        uint64_t nb_ = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : fs_, np_, nb_) if (nthreads > 1) num_threads(nthreads)
        for (uint64_t i = 0; i < N; ++i) {
            double& fnsum = fs_;
            double& npair = np_;
            uint64_t& broken = nb_;
            // the particle's float sums of |normal pair force| and of its pair stiffnesses,
            // bonds and contacts apart, as the engine keeps them
            TF fnb = 0, ktb = 0, krb = 0, fnc = 0, ktc = 0, krc = 0;
            const V3<TF> vi = {V[i], V[i + N], V[i + 2 * N]}, wi = {W[i], W[i + N], W[i + 2 * N]};
            const TF ri = (TF)rad[i];
            const TF mi = cmass * ri * ri * ri;
            V3<TF> fsb = {0, 0, 0}, msb = {0, 0, 0}, fsc = {0, 0, 0}, msc = {0, 0, 0};
            uint32_t pc = 0;                                     // slots whose contact the bond pass took
            for (uint64_t q = 0; q < K; ++q) {                   // _22 order: bonds by slot
                const uint64_t k = i * K + q;
                const id_t j = IL[k];
                if (j == EMPTY || type[k] != 1) continue;
                const double dx = R[j] - R[i], dy = R[j + N] - R[i + N], dz = R[j + 2 * N] - R[i + 2 * N];
                const double d2 = dx * dx + dy * dy + dz * dz;
                const V3<TF> r = {(TF)dx, (TF)dy, (TF)dz};
                const V3<TF> vj = {V[j], V[j + N], V[j + 2 * N]}, wj = {W[j], W[j + N], W[j + 2 * N]};
                const TF br = x.ref ? b_r : lambda * std::min(ri, (TF)rad[j]);
                // the record's force, moment and float sums are formed from zero and then
                // added to the particle's, record by record (the engine hands each record
                // from the lane that evaluates it to the particle's lane)
                V3<TF> fr = {0, 0, 0}, mr = {0, 0, 0};
                TF fnr = 0, ktr = 0, krr = 0;
                bool broke, clear = false;
                if (qs_total) {
                    // the pair's relative displacement since the increment began, formed in
                    // double as (r - r0) so that it keeps its own precision (a difference of
                    // the two particles' float displacements loses it to their size)
                    const V3<TF> ti = {(TF)ROT[3 * i], (TF)ROT[3 * i + 1], (TF)ROT[3 * i + 2]};
                    const V3<TF> tj = {(TF)ROT[3 * j], (TF)ROT[3 * j + 1], (TF)ROT[3 * j + 2]};
                    const double hx = 0.5 * (ROT[3 * i] + ROT[3 * j]), hy = 0.5 * (ROT[3 * i + 1] + ROT[3 * j + 1]),
                                 hz = 0.5 * (ROT[3 * i + 2] + ROT[3 * j + 2]);
                    const V3<TF> du = {(TF)(dx - (X0[j] - X0[i]) - (hy * dz - hz * dy)),
                                       (TF)(dy - (X0[j + N] - X0[i + N]) - (hz * dx - hx * dz)),
                                       (TF)(dz - (X0[j + 2 * N] - X0[i + 2 * N]) - (hx * dy - hy * dx))};
                    broke = bond_total(k, r, d2, du, ti, tj, br, fr, mr, fnr, ktr, krr);
                } else {
                    broke = bond(k, r, d2, vi, vj, wi, wj, br, fr, mr, fnr, ktr, krr);
                }
                if (broke) { type[k] = 0; ++broken; }
                npair += 1;
                // the contact an overlapping bonded pair carries in parallel with the bond, its
                // overlap counted from min(r_i + r_j, L0) (explicit steps only: inside a FIRE
                // increment its state would depend on the path)
                const double sr = std::fmin(rad[i] + rad[j], L0[k]);
                if (!x.ref && !in_fire && d2 < sr * sr) {
                    const TF rj = (TF)rad[j];
                    std::swap(Oijt[k], Ocb[k]);
                    clear = contact(k, r, d2, sr, ri, rj, mi, cmass * rj * rj * rj, vi, vj, wi, wj, fr, mr, fnr, ktr,
                                    krr);
                    std::swap(Oijt[k], Ocb[k]);
                    npair += 1;
                    pc |= 1u << q;
                } else {
                    Ocb[k] = {0, 0, 0};
                }
                if (broke) Oijt[k] = Ocb[k];                     // the slot goes on as that contact
                fsb.x += fr.x; fsb.y += fr.y; fsb.z += fr.z;
                if (clear) msb = {0, 0, 0};                      // the zero-spin rule clears the moment sum
                else { msb.x += mr.x; msb.y += mr.y; msb.z += mr.z; }
                fnb += fnr; ktb += ktr; krb += krr;
            }
            for (uint64_t q = 0; q < K; ++q) {                   // _21 order: type-0 slots by slot
                const uint64_t k = i * K + q;
                const id_t j = IL[k];
                if (j == EMPTY || type[k] != 0 || ((pc >> q) & 1u)) continue;
                const double dx = R[j] - R[i], dy = R[j + N] - R[i + N], dz = R[j + 2 * N] - R[i + 2 * N];
                const double d2 = dx * dx + dy * dy + dz * dz;
                const TF rj = (TF)rad[j];
                const double sr = rad[i] + rad[j];
                if (!(d2 < sr * sr)) { Oijt[k] = {0, 0, 0}; continue; }
                const V3<TF> r = {(TF)dx, (TF)dy, (TF)dz};
                const V3<TF> vj = {V[j], V[j + N], V[j + 2 * N]}, wj = {W[j], W[j + N], W[j + 2 * N]};
                contact(k, r, d2, sr, ri, rj, mi, cmass * rj * rj * rj, vi, vj, wi, wj, fsc, msc, fnc, ktc, krc);
                npair += 1;
            }
            fnb += fnc; ktb += ktc; krb += krc;
            fnsum += (double)fnb;
            if (KT) { (*KT)[i] = (double)ktb; (*KR)[i] = (double)krb; }
            TF Fx = (TF)0 + fsb.x, Fy = (TF)0 + fsb.y, Fz = (TF)0 + fsb.z;
            Fx += fsc.x; Fy += fsc.y; Fz += fsc.z;
            TF Mx = (TF)0 + msb.x, My = (TF)0 + msb.y, Mz = (TF)0 + msb.z;
            Mx += msc.x; My += msc.y; Mz += msc.z;
            Fn[i] = {Fx, Fy, Fz}; Mn[i] = {Mx, My, Mz};
        }
        fnsum = fs_; npair = np_;
        broken += nb_;
    }

    // Platen of one particle (the extended model's d_braziltest_simple2 /
    // d_UniaxialCompression3_simple on FP64 coordinates).
    void platen(uint64_t i, TF& Fx, TF& Fy, TF& Fz, double& Rx, double& Ry, double& Rz, TF& Vx, TF& Vy, TF& Vz,
                TF vt, double& sfb, double& sft) const {
        const rf_compression& Kc = t->Compress;
        const float cx = Kc.center.x, cy = Kc.center.y, cz = Kc.center.z, RR = Kc.RR;
        // with the reference constants the platen coordinates are rounded to float, as the
        // reference's drivers pass them to d_UniaxialCompression3_simple / d_braziltest_simple2
        const double Top = x.ref ? (double)(float)Kc.Top : Kc.Top;
        const double Bottom = x.ref ? (double)(float)Kc.Bottom : Kc.Bottom;
        const double TopR = x.ref ? (double)(float)Kc.TopR : Kc.TopR;
        const double BottomR = x.ref ? (double)(float)Kc.BottomR : Kc.BottomR;
        const bool brz = t->kind == RF_TEST_BRAZIL;
        const double Zcut = brz ? (double)(float)((double)t->S.center.y + (double)t->S.spacesized2.y)
                                : (double)(float)((double)t->S.center.z + (double)t->S.spacesized2.z);
        const double off = rad[i] - t->Po.p_r;    // the platens act on the particle surfaces
        if (brz) {
            const TF rx = (TF)(float)(Rx - cx), rz = (TF)(float)(Rz - cz);
            if (rx * rx + rz * rz < (TF)RR && (double)rz < Zcut) {
                if (Ry + off - TopR > -1e-9) {
                    const TF fy = Fy;
                    if (fy > 0) {
                        sft += (double)fy;
                        TF iv = Vx * Vx + Vz * Vz;
                        if ((double)iv > 1e-9) {
                            iv = rsqrt_rn<TF>(iv);
                            Fx -= (TF)0.45f * fy * Vx * iv;
                            Fz -= (TF)0.45f * fy * Vz * iv;
                        }
                    }
                    if (Ry + off - Top > -1e-9) {
                        Ry = Top - off; Vy = vt; Fy = 0;
                        if (in_fire) { Fx = 0; Fz = 0; Vx = 0; Vz = 0; }
                    }
                }
                if (Ry - off - BottomR < 1e-9) {
                    const TF fy = Fy;
                    if (fy < 0) {
                        sfb += (double)fy;
                        TF iv = Vx * Vx + Vz * Vz;
                        if ((double)iv > 1e-9) {
                            iv = rsqrt_rn<TF>(iv);
                            Fx += (TF)0.45f * fy * Vx * iv;
                            Fz += (TF)0.45f * fy * Vz * iv;
                        }
                    }
                    if (Ry - off - Bottom < 1e-9) {
                        Ry = Bottom + off; Vy = 0; Fy = 0;
                        if (in_fire) { Fx = 0; Fz = 0; Vx = 0; Vz = 0; }
                    }
                }
            }
        } else {
            const TF rx = (TF)(float)(Rx - cx), ry = (TF)(float)(Ry - cy);
            if (rx * rx + ry * ry < (TF)RR && Rz < Zcut) {
                if (Rz + off - TopR > -1e-9) {
                    if (Fz > 0) sft += (double)Fz;
                    if (Rz + off - Top > -1e-9) {
                        Rz = Top - off; Vz = vt; Fz = 0;
                        if (in_fire) { Fx = 0; Fy = 0; Vx = 0; Vy = 0; }
                    }
                }
                if (Rz - off - BottomR < 1e-9) {
                    if (Fz < 0) sfb += (double)Fz;
                    if (Rz - off - Bottom < 1e-9) {
                        Rz = Bottom + off; Vz = 0; Fz = 0;
                        if (in_fire) { Fx = 0; Fy = 0; Vx = 0; Vy = 0; }
                    }
                }
            }
        }
    }

    void step(double* curve, uint64_t cap, uint64_t* nsaved) {
        rf_compression& Kc = t->Compress;
        delete_far();                       // the previous step's DeleteFarLinks
        add_links();
        std::vector<V3<TF>> Fn(N), Mn(N);
        double fnsum, npair;
        pair_forces(Fn, Mn, fnsum, npair);
        double sfb = 0, sft = 0;
        const TF vt = (TF)(float)Kc.V;
        const rf_sample& S = t->S;
#pragma omp parallel for schedule(static) reduction(+ : sfb, sft) if (nthreads > 1) num_threads(nthreads)
        for (uint64_t i = 0; i < N; ++i) {
            TF Fx = Fn[i].x, Fy = Fn[i].y, Fz = Fn[i].z;
            double Rx = R[i], Ry = R[i + N], Rz = R[i + 2 * N];
            TF Vx = V[i], Vy = V[i + N], Vz = V[i + 2 * N];
            platen(i, Fx, Fy, Fz, Rx, Ry, Rz, Vx, Vy, Vz, vt, sfb, sft);
            const TF ri = (TF)rad[i];
            const TF mi = cmass * ri * ri * ri;
            const TF dtm = dt / mi, dtI = dt / ((TF)0.4f * mi * ri * ri);
            Vx += Fx * dtm; Vy += Fy * dtm; Vz += Fz * dtm;
            if (pos_mode == 1) {
                Rx = hilo_add(Rx, (float)(Vx * dt)); Ry = hilo_add(Ry, (float)(Vy * dt));
                Rz = hilo_add(Rz, (float)(Vz * dt));
            } else if (pos_mode == 2) {
                Rx = (double)((float)Rx + (float)(Vx * dt)); Ry = (double)((float)Ry + (float)(Vy * dt));
                Rz = (double)((float)Rz + (float)(Vz * dt));
            } else {
                Rx += (double)(Vx * dt); Ry += (double)(Vy * dt); Rz += (double)(Vz * dt);
            }
            W[i] += Mn[i].x * dtI; W[i + N] += Mn[i].y * dtI; W[i + 2 * N] += Mn[i].z * dtI;
            const double dx = Rx - S.center.x, dy = Ry - S.center.y, dz = Rz - S.center.z;
            if ((dx - S.spacesized2.x > 0) || (dx + S.spacesized2.x < 0) || (dy - S.spacesized2.y > 0) ||
                (dy + S.spacesized2.y < 0) || (dz - S.spacesized2.z > 0) || (dz + S.spacesized2.z < 0)) {
                Rx = S.hidenpoint.x; Ry = S.hidenpoint.y; Rz = S.hidenpoint.z;
                Vx = 0; Vy = 0; Vz = 0;
            }
            R[i] = Rx; R[i + N] = Ry; R[i + 2 * N] = Rz;
            V[i] = Vx; V[i + N] = Vy; V[i + 2 * N] = Vz;
        }
        sum_forces(t, sfb, sft, sz0, curve, cap, nsaved);
        const double keep = x.drop > 0.0 ? 1.0 - x.drop : 0.0;
        if (Kc.Loading && Kc.Stress < keep * Kc.FractureStress) Kc.Fracture = 1;
        compress(t, Kc.Stress);
        ++steps;
    }

    // One quasi-static load increment relaxed by FIRE, as the engine runs it
    // (rf_engine_load_increment): platen advance, rest start, then iterations of
    // [delete, add, forces with the FIRE dt and without damping or rolling resistance,
    // platen clamp at rest, FIRE decision on FP64 sums, mixing and semi-implicit Euler].
    // trace (may be null) receives the residual of every iteration.
    std::vector<double> X0, ROT;      // start positions and accumulated rotation of the last increment
    std::vector<V3<TF>> Flast, Mlast; // net forces and moments of the last increment's last pass

    uint64_t fire_increment(const rf_relax_params& p, int* converged, double* residual, double* trace,
                            uint64_t trace_cap, const double* warm = nullptr) {
        rf_compression& Kc = t->Compress;
        X0 = R;
        ROT.assign(3 * N, 0.0);
        Rij0 = Rij; Oijt0 = Oijt; Mijn0 = Mijn; Mijt0 = Mijt;
        const int ax = t->kind == RF_TEST_BRAZIL ? 1 : 2;
        const double delta = p.strain_inc * Kc.Size0;
        double* sz = ax == 1 ? &Kc.size_d.y : &Kc.size_d.z;
        double* cd = ax == 1 ? &Kc.center_d.y : &Kc.center_d.z;
        *sz -= delta;
        Kc.Top -= delta;
        Kc.TopR = Kc.Top - 2.0 * t->Po.p_r;
        *cd -= delta;
        if (ax == 1) { Kc.size.y = (float)*sz; Kc.sized2.y = (float)(0.5 * *sz); Kc.center.y = (float)*cd; Kc.Hd2 = Kc.sized2.y; }
        else { Kc.size.z = (float)*sz; Kc.sized2.z = (float)(0.5 * *sz); Kc.center.z = (float)*cd; Kc.Hd2 = Kc.sized2.z; }
        Kc.Strain = (*sz - Kc.Size0) / Kc.Size0;
        std::fill(V.begin(), V.end(), (TF)0);
        std::fill(W.begin(), W.end(), (TF)0);
        // the platen pushes the particles it passed: clamp them now, so the first force
        // pass (and its convergence test) sees the loaded configuration; a warm start
        // (the engine's rf_engine_load_increment with a prediction) jumps the positions
        // and carries the motion into the first pass as velocities over dt0
        const TF idt0 = (TF)(float)(1.0 / p.dt0);
        for (uint64_t i = 0; i < N; ++i) {
            TF f0 = 0, f1 = 0, f2 = 0, v0 = 0, v1 = 0, v2 = 0;
            if (warm) {
                const double* q = warm + 6 * i;
                TF u[6];
                for (int a = 0; a < 6; ++a) u[a] = (TF)(float)q[a];
                // a particle the platens held at the end of the last increment stays on its
                // platen (the top one has moved by delta)
                const bool brz = t->kind == RF_TEST_BRAZIL;
                const double off = rad[i] - t->Po.p_r;
                const double Zcut = brz ? (double)(float)((double)t->S.center.y + (double)t->S.spacesized2.y)
                                        : (double)(float)((double)t->S.center.z + (double)t->S.spacesized2.z);
                const double a0 = brz ? R[i + N] : R[i + 2 * N];
                const float q0 = (float)(R[i] - Kc.center.x);
                const float q1 = brz ? (float)(R[i + 2 * N] - Kc.center.z) : (float)(R[i + N] - Kc.center.y);
                const bool zone = q0 * q0 + q1 * q1 < Kc.RR && (brz ? (double)(float)(R[i + 2 * N] - Kc.center.z) : a0) < Zcut;
                const bool at_top = zone && a0 + off - (Kc.Top + delta) > -1e-9;
                const bool at_bottom = zone && a0 - off - Kc.Bottom < 1e-9;
                R[i] += (double)u[0]; R[i + N] += (double)u[1]; R[i + 2 * N] += (double)u[2];
                double& ax = brz ? R[i + N] : R[i + 2 * N];
                if (at_top) ax = Kc.Top - off;
                else if (at_bottom) ax = Kc.Bottom + off;
                v0 = u[0] * idt0; v1 = u[1] * idt0; v2 = u[2] * idt0;
                W[i] = u[3] * idt0; W[i + N] = u[4] * idt0; W[i + 2 * N] = u[5] * idt0;
                ROT[3 * i] = u[3]; ROT[3 * i + 1] = u[4]; ROT[3 * i + 2] = u[5];
            }
            double sb = 0, st = 0;
            platen(i, f0, f1, f2, R[i], R[i + N], R[i + 2 * N], v0, v1, v2, (TF)0, sb, st);
            V[i] = v0; V[i + N] = v1; V[i + 2 * N] = v2;
        }
        const TF dt_keep = dt, pA_keep = p_A, mur_keep = mur;
        p_A = 0; mur = 0;
        qs_total = g_qs_total;
        in_fire = true;
        double fdt = p.dt0, alpha = p.alpha0, cv = 1, cf = 0, cm = 0;
        uint64_t npos = 0, it = 0;
        bool uphill = false;
        *converged = 0;
        std::vector<V3<TF>> Fn(N), Mn(N);
        std::vector<double> KT(N), KR(N);
        for (;;) {
            dt = (TF)(float)fdt;
            delete_far();
            add_links();
            double fnsum, npair;
            pair_forces(Fn, Mn, fnsum, npair, &KT, &KR);
            double P = 0, FF = 0, VV = 0, MM = 0, WW = 0, sfb = 0, sft = 0;
            for (uint64_t i = 0; i < N; ++i) {
                TF Fx = Fn[i].x, Fy = Fn[i].y, Fz = Fn[i].z;
                double Rx = R[i], Ry = R[i + N], Rz = R[i + 2 * N];
                TF Vx = V[i], Vy = V[i + N], Vz = V[i + 2 * N];
                platen(i, Fx, Fy, Fz, Rx, Ry, Rz, Vx, Vy, Vz, (TF)0, sfb, sft);
                R[i] = Rx; R[i + N] = Ry; R[i + 2 * N] = Rz;
                V[i] = Vx; V[i + N] = Vy; V[i + 2 * N] = Vz;
                Fn[i] = {Fx, Fy, Fz};
                const TF wx = W[i], wy = W[i + N], wz = W[i + 2 * N];
                const V3<TF> M = Mn[i];
                P += (double)Fx * Vx + (double)Fy * Vy + (double)Fz * Vz + (double)M.x * wx + (double)M.y * wy +
                     (double)M.z * wz;
                FF += (double)Fx * Fx + (double)Fy * Fy + (double)Fz * Fz;
                VV += (double)Vx * Vx + (double)Vy * Vy + (double)Vz * Vz;
                MM += (double)M.x * M.x + (double)M.y * M.y + (double)M.z * M.z;
                WW += (double)wx * wx + (double)wy * wy + (double)wz * wz;
            }
            const double mean = npair > 0 ? fnsum / npair : 0.0;
            const double res = mean > 0 ? std::sqrt(FF / (double)N) / mean : (FF > 0 ? 1e300 : 0.0);
            Kc.Stress = 0.5 * (std::fabs(sfb) + std::fabs(sft)) * (double)Kc._1d_Area;
            if (trace && it < trace_cap) trace[it] = res;
            ++it;
            *residual = res;
            if (res <= p.tol) { *converged = 1; break; }
            if (it >= p.max_iter) break;
            if (it == 1) {                  // first pass of the increment: start from rest
                npos = 0;
                uphill = true;
            } else if (P > 0) {
                cv = 1 - alpha;
                cf = FF > 0 ? alpha * std::sqrt(VV / FF) : 0;
                cm = MM > 0 ? alpha * std::sqrt(WW / MM) : 0;
                uphill = false;
                if (++npos > p.n_delay) { fdt = std::fmin(fdt * p.f_inc, p.dt_max); alpha *= p.f_alpha; }
            } else {
                npos = 0;
                fdt = std::fmax(fdt * p.f_dec, p.dt_min);
                alpha = p.alpha0;
                uphill = true;
            }
            const TF dtf = (TF)(float)fdt;
            for (uint64_t i = 0; i < N; ++i) {
                TF v[3] = {V[i], V[i + N], V[i + 2 * N]}, w[3] = {W[i], W[i + N], W[i + 2 * N]};
                const TF F[3] = {Fn[i].x, Fn[i].y, Fn[i].z}, M[3] = {Mn[i].x, Mn[i].y, Mn[i].z};
                // stiffness-scaled (Jacobi) masses: every particle's own frequency is 1
                const TF mt = (TF)std::max(KT[i], 1e-30), mr = (TF)std::max(KR[i], 1e-30);
                const TF dtm = dtf / mt, dtI = dtf / mr;
                for (int a = 0; a < 3; ++a) {
                    if (uphill) { v[a] = 0; w[a] = 0; }
                    else { v[a] = (TF)(float)cv * v[a] + (TF)(float)cf * F[a]; w[a] = (TF)(float)cv * w[a] + (TF)(float)cm * M[a]; }
                    v[a] += F[a] * dtm;
                    w[a] += M[a] * dtI;
                    R[i + a * N] += (double)v[a] * (double)dtf;
                    ROT[3 * i + a] += (double)w[a] * (double)dtf;
                    V[i + a * N] = v[a];
                    W[i + a * N] = w[a];
                }
            }
        }
        dt = dt_keep; p_A = pA_keep; mur = mur_keep;
        qs_total = false;
        in_fire = false;
        Flast = Fn; Mlast = Mn;
        return it;
    }
};

template <class TF>
static uint64_t run_ext(rf_task* t, const rf_ext_params* xp, double* R_io, const double* rad, uint64_t max_steps,
                        TF* V_out, uint64_t* IL_out, uint8_t* type_out, double* curve, uint64_t cap,
                        uint64_t* nsaved, int* status, uint64_t* broken, int pos_mode = 0,
                        const double* strain = nullptr) {
    RunExt<TF> r;
    r.pos_mode = pos_mode;
    r.t = t;
    r.x = ext_par(xp);
    r.init(R_io, rad);
    if (strain) r.affine(strain[0], strain[1], strain[2]);
    uint64_t ns = 0;
    while (r.running() && r.steps < max_steps) r.step(curve, cap, &ns);   // max_steps 0: bonds only
    r.delete_far();                         // the pending DeleteFarLinks of the last step
    if (nsaved) *nsaved = ns;
    std::memcpy(R_io, r.R.data(), sizeof(double) * 3 * r.N);
    if (V_out) std::memcpy(V_out, r.V.data(), sizeof(TF) * 3 * r.N);
    if (IL_out) std::memcpy(IL_out, r.IL.data(), sizeof(uint64_t) * r.N * r.K);
    if (type_out) std::memcpy(type_out, r.type.data(), r.N * r.K);
    if (status) *status = r.status;
    if (broken) *broken = r.broken;
    return r.steps;
}

}  // namespace rfo

namespace rfo {
// Quasi-static run: n_inc increments; per increment its iteration count, convergence,
// residual and platen stress. trace: residual per iteration of the last increment.
template <class TF>
static int qs_ext(rf_task* t, const rf_ext_params* xp, double* R_io, const double* rad, const rf_relax_params* p,
                  uint64_t n_inc, uint64_t* iters, int* conv, double* res, double* stress, double* trace,
                  uint64_t trace_cap) {
    RunExt<TF> r;
    r.t = t;
    r.x = ext_par(xp);
    r.init(R_io, rad);
    for (uint64_t k = 0; k < n_inc; ++k) {
        int c = 0;
        double rr = 0;
        const bool last = k + 1 == n_inc;
        iters[k] = r.fire_increment(*p, &c, &rr, last ? trace : nullptr, trace_cap);
        conv[k] = c; res[k] = rr; stress[k] = t->Compress.Stress;
    }
    std::memcpy(R_io, r.R.data(), sizeof(double) * 3 * r.N);
    return r.status;
}
}  // namespace rfo

namespace rfo {
// Exact warm start on the CPU: n_pre plain increments, then the next increment once plain
// (reference) and once from the same state warm-started with the plain answer; returns
// the warm start's residual after `warm_iters` iterations the largest differences of the
// bond state from the plain relaxed state, and the warm run's iterations and convergence flag.
// scale != 1 or noise != 0 make the warm start inexact: each particle's displacement and
// rotation times (scale + noise * u), u uniform in [-1, 1) from a fixed sequence.
template <class TF>
static void warm_probe(rf_task* t, const rf_ext_params* xp, const double* R0, const double* rad,
                       const rf_relax_params* p, uint64_t n_pre, uint64_t warm_iters, double* out,
                       double scale = 1.0, double noise = 0.0) {
    RunExt<TF> a;
    a.t = t;
    a.x = ext_par(xp);
    a.init(R0, rad);
    int c; double res;
    for (uint64_t k = 0; k < n_pre; ++k) a.fire_increment(*p, &c, &res, nullptr, 0);
    RunExt<TF> b = a;
    rf_task tb = *t;
    b.t = &tb;
    const uint64_t it_plain = a.fire_increment(*p, &c, &res, nullptr, 0);
    std::vector<double> warm(6 * a.N);
    uint64_t lcg = 0x2545F4914F6CDD1Dull;
    for (uint64_t i = 0; i < a.N; ++i)
        for (int k = 0; k < 3; ++k) {
            lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
            const double u = (double)(lcg >> 11) * (2.0 / 9007199254740992.0) - 1.0;
            const double f = scale + noise * u;
            warm[6 * i + k] = (a.R[i + k * a.N] - a.X0[i + k * a.N]) * f;
            warm[6 * i + 3 + k] = a.ROT[3 * i + k] * f;
        }
    rf_relax_params q = *p;
    q.max_iter = warm_iters;
    int cb; double rb;
    const uint64_t it_warm = b.fire_increment(q, &cb, &rb, nullptr, 0, warm.data());
    double dO = 0, dN = 0, dT = 0, dR = 0, sO = 0, sN = 0, sT = 0, dx = 0;
    for (uint64_t k = 0; k < a.N * a.K; ++k) {
        if (a.type[k] != 1 || b.type[k] != 1) continue;
        auto diff = [](const V3<TF>& u, const V3<TF>& v) {
            return std::max(std::fabs((double)u.x - v.x), std::max(std::fabs((double)u.y - v.y), std::fabs((double)u.z - v.z)));
        };
        auto mag = [](const V3<TF>& u) { return std::max(std::fabs((double)u.x), std::max(std::fabs((double)u.y), std::fabs((double)u.z))); };
        dO = std::max(dO, diff(a.Oijt[k], b.Oijt[k])); sO = std::max(sO, mag(a.Oijt[k]));
        dN = std::max(dN, diff(a.Mijn[k], b.Mijn[k])); sN = std::max(sN, mag(a.Mijn[k]));
        dT = std::max(dT, diff(a.Mijt[k], b.Mijt[k])); sT = std::max(sT, mag(a.Mijt[k]));
        dR = std::max(dR, diff(a.Rij[k], b.Rij[k]));
    }
    for (uint64_t q2 = 0; q2 < 3 * a.N; ++q2) dx = std::max(dx, std::fabs(a.R[q2] - b.R[q2]));
    out[0] = (double)it_plain; out[1] = res; out[2] = rb; out[3] = t->Compress.Stress; out[4] = tb.Compress.Stress;
    out[5] = dO; out[6] = sO; out[7] = dN; out[8] = sN; out[9] = dT; out[10] = sT; out[11] = dR; out[12] = dx;
    out[13] = (double)it_warm; out[14] = (double)cb;
}
}  // namespace rfo

extern "C" {
void rfo_warm_probe_ext_d(rf_task* t, const rf_ext_params* x, const double* R0, const double* rad,
                          const rf_relax_params* p, uint64_t n_pre, uint64_t warm_iters, double* out) {
    rfo::warm_probe<double>(t, x, R0, rad, p, n_pre, warm_iters, out);
}
// The same with float forces (the engine's arithmetic) and an inexact warm start.
void rfo_warm_probe_ext_f(rf_task* t, const rf_ext_params* x, const double* R0, const double* rad,
                          const rf_relax_params* p, uint64_t n_pre, uint64_t warm_iters, double* out, double scale,
                          double noise) {
    rfo::warm_probe<float>(t, x, R0, rad, p, n_pre, warm_iters, out, scale, noise);
}
int rfo_qs_ext_f(rf_task* t, const rf_ext_params* x, double* R_io, const double* rad, const rf_relax_params* p,
                 uint64_t n_inc, uint64_t* iters, int* conv, double* res, double* stress, double* trace,
                 uint64_t trace_cap) {
    return rfo::qs_ext<float>(t, x, R_io, rad, p, n_inc, iters, conv, res, stress, trace, trace_cap);
}
int rfo_qs_ext_d(rf_task* t, const rf_ext_params* x, double* R_io, const double* rad, const rf_relax_params* p,
                 uint64_t n_inc, uint64_t* iters, int* conv, double* res, double* stress, double* trace,
                 uint64_t trace_cap) {
    return rfo::qs_ext<double>(t, x, R_io, rad, p, n_inc, iters, conv, res, stress, trace, trace_cap);
}
// Extended model, float forces (the engine's arithmetic) and FP64 (the FP64 oracle).
// R_io: double[3N] planar in, final positions out (after the pending delete pass).
uint64_t rfo_run_ext_f(rf_task* t, const rf_ext_params* x, double* R_io, const double* rad, uint64_t max_steps,
                       float* V_out, uint64_t* IL_out, uint8_t* type_out, double* curve, uint64_t cap,
                       uint64_t* nsaved, int* status, uint64_t* broken) {
    return rfo::run_ext<float>(t, x, R_io, rad, max_steps, V_out, IL_out, type_out, curve, cap, nsaved, status,
                               broken);
}
void rfo_set_qs_total(int on) { rfo::g_qs_total = on; }
// Float forces with positions as hi/lo float pairs (pos_mode 1) or as floats (2): the
// precision comparison.
uint64_t rfo_run_ext_pos_f(rf_task* t, const rf_ext_params* x, double* R_io, const double* rad, uint64_t max_steps,
                           float* V_out, uint64_t* IL_out, uint8_t* type_out, double* curve, uint64_t cap,
                           uint64_t* nsaved, int* status, uint64_t* broken, int pos_mode) {
    return rfo::run_ext<float>(t, x, R_io, rad, max_steps, V_out, IL_out, type_out, curve, cap, nsaved, status,
                               broken, pos_mode);
}
// Wall time of `steps` explicit steps of the extended model (float forces, FP64 positions)
// on `threads` host threads, after bond construction and rf_engine_affine_strain(strain)
// (strain may be null); the set-up is not timed. The CPU baseline of the benchmark.
double rfo_time_ext_f(rf_task* t, const rf_ext_params* xp, const double* R0, const double* rad, const double* strain,
                      uint64_t steps, int threads, uint64_t* done) {
    rfo::RunExt<float> r;
    r.t = t;
    r.x = rfo::ext_par(xp);
    r.nthreads = threads < 1 ? 1 : threads;
    r.init(R0, rad);
    if (strain) r.affine(strain[0], strain[1], strain[2]);
    uint64_t ns = 0;
    const auto t0 = std::chrono::steady_clock::now();
    while (r.running() && r.steps < steps) r.step(nullptr, 0, &ns);
    const auto t1 = std::chrono::steady_clock::now();
    if (done) *done = r.steps;
    return std::chrono::duration<double>(t1 - t0).count();
}
// rfo_run_ext_f after rf_engine_affine_strain(strain) applied to the built specimen.
uint64_t rfo_run_ext_strained_f(rf_task* t, const rf_ext_params* x, double* R_io, const double* rad,
                                const double* strain, uint64_t max_steps, float* V_out, uint64_t* IL_out,
                                uint8_t* type_out, double* curve, uint64_t cap, uint64_t* nsaved, int* status,
                                uint64_t* broken) {
    return rfo::run_ext<float>(t, x, R_io, rad, max_steps, V_out, IL_out, type_out, curve, cap, nsaved, status,
                               broken, 0, strain);
}
uint64_t rfo_run_ext_d(rf_task* t, const rf_ext_params* x, double* R_io, const double* rad, uint64_t max_steps,
                       double* V_out, uint64_t* IL_out, uint8_t* type_out, double* curve, uint64_t cap,
                       uint64_t* nsaved, int* status, uint64_t* broken) {
    return rfo::run_ext<double>(t, x, R_io, rad, max_steps, V_out, IL_out, type_out, curve, cap, nsaved, status,
                                broken);
}
}  // extern "C"

extern "C" {
int rfo_task_prepare(rf_task* t, const double ss[3], const double ls[3], double cell_a, double vload,
                     double minstress, double maxstrain) {
    return rfo::prepare(t, ss, ls, cell_a, vload, minstress, maxstrain);
}
void rfo_compress(rf_task* t, double pressure) { rfo::compress(t, pressure); }
void rfo_sum_forces(rf_task* t, double sfb, double sft, double sz0) {
    uint64_t n = 0;
    rfo::sum_forces(t, sfb, sft, sz0, nullptr, 0, &n);
}

// Full run in FP32 (reference precision). State in/out arrays are the reference
// layout; R_io holds the initial positions on entry and final ones on exit.
// Returns the number of steps taken; *status gets the first bound/overflow status.
uint64_t rfo_run_f(rf_task* t, float* R_io, uint64_t max_steps, float* V_out, float* W_out,
                   uint64_t* IL_out, uint8_t* type_out, float* iL_out, float* Rij_out, float* Oijt_out,
                   float* Mijn_out, float* Mijt_out, uint8_t* broke_out, double* curve, uint64_t cap,
                   uint64_t* nsaved, int* status) {
    rfo::Run<float> r;
    r.t = t;
    r.init(R_io);
    uint64_t ns = 0;
    while (r.running() && (max_steps == 0 || r.steps < max_steps)) r.step(curve, cap, &ns);
    if (nsaved) *nsaved = ns;
    uint64_t N = r.N, K = r.K;
    std::memcpy(R_io, r.R.data(), sizeof(float) * 3 * N);
    if (V_out) std::memcpy(V_out, r.V.data(), sizeof(float) * 3 * N);
    if (W_out) std::memcpy(W_out, r.W.data(), sizeof(float) * 3 * N);
    if (IL_out) std::memcpy(IL_out, r.IL.data(), sizeof(uint64_t) * N * K);
    if (type_out) std::memcpy(type_out, r.type.data(), N * K);
    if (iL_out) std::memcpy(iL_out, r.iL.data(), sizeof(float) * N * K);
    if (Rij_out) std::memcpy(Rij_out, r.Rij.data(), sizeof(float) * 3 * N * K);
    if (Oijt_out) std::memcpy(Oijt_out, r.Oijt.data(), sizeof(float) * 3 * N * K);
    if (Mijn_out) std::memcpy(Mijn_out, r.Mijn.data(), sizeof(float) * 3 * N * K);
    if (Mijt_out) std::memcpy(Mijt_out, r.Mijt.data(), sizeof(float) * 3 * N * K);
    if (broke_out) std::memcpy(broke_out, r.broke.data(), N * K);
    if (status) *status = r.status;
    return r.steps;
}

// Same run in FP64 (the FP64 oracle): positions, velocities, forces and all
// parameters in double. Outputs are rounded to float for comparison.
uint64_t rfo_run_d(rf_task* t, const float* R_in, uint64_t max_steps, double* R_out, double* curve,
                   uint64_t cap, uint64_t* nsaved, uint8_t* type_out, int* status) {
    rfo::Run<double> r;
    r.t = t;
    r.init(R_in);
    uint64_t ns = 0;
    while (r.running() && (max_steps == 0 || r.steps < max_steps)) r.step(curve, cap, &ns);
    if (nsaved) *nsaved = ns;
    if (R_out) std::memcpy(R_out, r.R.data(), sizeof(double) * 3 * r.N);
    if (type_out) std::memcpy(type_out, r.type.data(), r.N * r.K);
    if (status) *status = r.status;
    return r.steps;
}
}  // extern "C"
// ===========================================================================
// C ABI for the tests (ctypes). Suffix _f = float instance, _d = double instance.
// Slot state arrays are float3/double3 AoS, ids uint64 (uint_fast32_t on Linux).
// ===========================================================================
extern "C" {

int rfo_cell_distribution_f(const float* R, uint64_t N, uint64_t* CI, uint64_t* CIs, uint64_t* pnC,
                            uint64_t CN, float inv_a, rf_uint3 cN) {
    return rfo::cell_distribution<float>(R, N, CI, CIs, pnC, CN, inv_a, cN);
}
int rfo_construct_list_f(const float* R, uint64_t N, const uint64_t* CIs, const uint64_t* pnC, uint64_t* IL,
                         uint64_t K, float a, float inv_a, float aacut, rf_uint3 cN, uint64_t CN) {
    return rfo::construct_list<float>(R, N, CIs, pnC, IL, K, a, inv_a, aacut, cN, CN);
}
int rfo_reconstruct_bpm_f(const float* R, uint64_t N, const uint64_t* CIs, const uint64_t* pnC, uint64_t* IL,
                          uint8_t* ILtype, uint64_t K, float a, float inv_a, float aacut, rf_uint3 cN,
                          uint64_t CN) {
    return rfo::reconstruct_bpm<float>(R, N, CIs, pnC, IL, ILtype, K, a, inv_a, aacut, cN, CN);
}
void rfo_delete_far_links_f(const float* R, uint64_t N, uint64_t* IL, uint8_t* ILtype, float* Rij, float* Oijt,
                            float* Mijn, float* Mijt, uint64_t K, float aacut) {
    typedef rfo::V3<float> v;
    rfo::delete_far_links<float>(R, N, IL, ILtype, (v*)Rij, (v*)Oijt, (v*)Mijn, (v*)Mijt, K, aacut);
}
void rfo_construct_bonds_f(const float* R, uint64_t N, const uint64_t* IL, uint8_t* ILtype, float* iL,
                           float* Rij, float* Oijt, float* Mijn, float* Mijt, uint64_t K, float aa_create) {
    typedef rfo::V3<float> v;
    rfo::construct_bonds<float>(R, N, IL, ILtype, iL, (v*)Rij, (v*)Oijt, (v*)Mijn, (v*)Mijt, K, aa_create);
}
void rfo_forces_22_f(const float* R, const float* V, const float* W, const uint64_t* IL, uint8_t* ILtype,
                     const float* iL, float* Rij, float* Oijt, float* Mijn, float* Mijt, float* F, float* M,
                     uint64_t N, uint64_t K, float dt, float m_E, float m_G, float b_r, float m_Gcritn,
                     float m_Gcritt, uint8_t* broke) {
    typedef rfo::V3<float> v;
    rfo::FP<float> p{};
    p.dt = dt; p.m_E = m_E; p.m_G = m_G; p.b_r = b_r; p.m_Gcritn = m_Gcritn; p.m_Gcritt = m_Gcritt;
    rfo::forces_22<float>(R, V, W, IL, ILtype, iL, (v*)Rij, (v*)Oijt, (v*)Mijn, (v*)Mijt, F, M, N, K, p, broke);
}
// forces_22 with the break criteria of every bond slot: crit[2k] = Sc (tensile stress
// plus bending), crit[2k + 1] = Mc (shear plus torsion), as tested against m_Gcritn / m_Gcritt.
void rfo_forces_22_crit_f(const float* R, const float* V, const float* W, const uint64_t* IL, uint8_t* ILtype,
                          const float* iL, float* Rij, float* Oijt, float* Mijn, float* Mijt, float* F, float* M,
                          uint64_t N, uint64_t K, float dt, float m_E, float m_G, float b_r, float m_Gcritn,
                          float m_Gcritt, uint8_t* broke, float* crit) {
    typedef rfo::V3<float> v;
    rfo::FP<float> p{};
    p.dt = dt; p.m_E = m_E; p.m_G = m_G; p.b_r = b_r; p.m_Gcritn = m_Gcritn; p.m_Gcritt = m_Gcritt;
    rfo::forces_22<float>(R, V, W, IL, ILtype, iL, (v*)Rij, (v*)Oijt, (v*)Mijn, (v*)Mijt, F, M, N, K, p, broke,
                          crit);
}
void rfo_forces_21_f(const float* R, const float* V, const float* W, const uint64_t* IL, const uint8_t* ILtype,
                     float* Oijt, float* F, float* M, uint64_t N, uint64_t K, float dt, float m_E, float m_G,
                     float p_A, float m_mu, float m_muroll, float mP, float rP) {
    typedef rfo::V3<float> v;
    rfo::FP<float> p{};
    p.dt = dt; p.hm_E = m_E; p.hm_G = m_G; p.p_A = p_A; p.m_mu = m_mu; p.m_muroll = m_muroll; p.mP = mP; p.rP = rP;
    rfo::forces_21<float>(R, V, W, IL, ILtype, (v*)Oijt, F, M, N, K, p);
}
void rfo_increments_f(const float* F, float* V, float* R, const float* M, float* W, uint64_t N, float dt_d_m,
                      float dt, float dt_d_I) {
    rfo::increments<float>(F, V, R, M, W, N, dt_d_m, dt, dt_d_I);
}
void rfo_brazil_platen_f(float* R, float* V, float* F, uint64_t N, rf_float3 c, float RR, float Yt, float Yb,
                         float Ytr, float Ybr, float vt, float Zcut, double* sums) {
    rfo::brazil_platen<float>(R, V, F, N, {c.x, c.y, c.z}, RR, Yt, Yb, Ytr, Ybr, vt, Zcut, &sums[0], &sums[1]);
}
void rfo_uniaxial_platen_f(float* R, float* V, float* F, uint64_t N, rf_float3 c, float RR, float Zt, float Zb,
                           float Ztr, float Zbr, float vt, float Zcut, double* sums) {
    rfo::uniaxial_platen<float>(R, V, F, N, {c.x, c.y, c.z}, RR, Zt, Zb, Ztr, Zbr, vt, Zcut, &sums[0], &sums[1]);
}
void rfo_cut_restriction_f(float* R, float* V, float* F, uint64_t N, rf_float3 center, rf_float3 sized2,
                           rf_float3 hp) {
    rfo::cut_restriction<float>(R, V, F, N, {center.x, center.y, center.z}, {sized2.x, sized2.y, sized2.z},
                                {hp.x, hp.y, hp.z});
}
// d_CalculateIncrementsFIRE (md_firerelaxation.cu:18-56): V is replaced by F * dt0/m
// (QUIRK: no memory of the previous V), mixed with F by the per-particle ratio |v|/|F|
// (also a no-op, v being parallel to F), and R advances by V * dt.
void rfo_fire_increments_f(const float* F, float* V, float* R, uint64_t N, float dtm, float dt, float a) {
    for (uint64_t i = 0; i < N; ++i) {
        const float Fx = F[i], Fy = F[i + N], Fz = F[i + 2 * N];
        float vx = Fx * dtm, vy = Fy * dtm, vz = Fz * dtm;
        const float vv = vx * vx + vy * vy + vz * vz;
        const float f = Fx * Fx + Fy * Fy + Fz * Fz;
        float vdf;
        if (f > 1e-12f) vdf = a * std::sqrt(vv * (1.0f / f));
        else vdf = a * std::sqrt(vv) * (float)1e6;
        vx = (1.0f - a) * vx + vdf * Fx;
        vy = (1.0f - a) * vy + vdf * Fy;
        vz = (1.0f - a) * vz + vdf * Fz;
        V[i] = vx; V[i + N] = vy; V[i + 2 * N] = vz;
        R[i] += vx * dt; R[i + N] += vy * dt; R[i + 2 * N] += vz * dt;
    }
}
// d_CalculateDecrementsHalfStepFIRE (md_firerelaxation.cu:58-70)
void rfo_fire_half_f(const float* V, float* R, uint64_t N, float dt2) {
    for (uint64_t q = 0; q < 3 * N; ++q) R[q] -= V[q] * dt2;
}
// d_FdotVEntire (md_firerelaxation.cu:372-490), summed in double.
double rfo_fdotv_f(const float* V, const float* F, uint64_t N) {
    double s = 0.0;
    for (uint64_t q = 0; q < 3 * N; ++q) s += (double)F[q] * (double)V[q];
    return s;
}
float rfo_rsqrt_rn_f(float x) { return rfo::rsqrt_rn<float>(x); }
void rfo_rsqrt_rn_array_f(const float* x, float* y, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) y[i] = rfo::rsqrt_rn<float>(x[i]);
}

}  // extern "C"
