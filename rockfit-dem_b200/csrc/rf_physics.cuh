// Per-slot physics of the bonded-particle model, shared by the md_* drop-in kernels
// (reference layout) and the fused engine (slot-major layout).
//
// Operation order follows the reference's live kernels expression by expression
// (MSMS-LAB/RockFit-DEM md_calculateforcesdem3.cu); with --fmad=false each line is
// the same sequence of IEEE float operations the CPU oracle performs. The
// library-norm call norm3df of the reference is replaced by sqrt(x*x+y*y+z*z).
#pragma once
#include "rf_common.cuh"

namespace rf {

#define RF_PI_F 3.14159265358979f      // MCf_pi, md_math_constants.h:87
#define RF_2D3_F 0.6666666667f         // MCf_2d3, md_math_constants.h:63

struct BondParams {          // scalar arguments of d_CalculateForcesDEM_22
    float dt, m_E, m_G, b_r, m_Gcritn, m_Gcritt;
};
struct ContactParams {       // scalar arguments of d_CalculateForcesDEM_21
    float dt, m_E, m_G, p_A, m_mu, m_muroll, mP, rP;
};

__device__ __forceinline__ float norm3(float x, float y, float z) {
    return __fsqrt_rn(x * x + y * y + z * z);
}

// One bond slot i->j (d_CalculateForcesDEM_22 loop body, :441-473). r = Rj - Ri.
// Accumulates into fs, ms in the reference's order and updates the slot state.
// Returns true when the break check fired (the slot is then type 0 and its
// Oijt, Mijn, Mijt are zero).
__device__ __forceinline__ bool bond_slot(const BondParams& p, const f3 r, const f3 vi, const f3 vj,
                                          const f3 wi, const f3 wj, const float il, f3& Rij, f3& Oijt,
                                          f3& Mijn, f3& Mijt, f3& fs, f3& ms) {
    // dd_Calculate_rijm_nij_2 (:38-52)
    const float rijm = norm3(r.x, r.y, r.z);
    const float inv_rm = __frcp_rn(rijm);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    // dd_Calculate_fijn_bpm_2 (:91-103)
    float cef = p.m_E * (rijm - __frcp_rn(il)) * il;
    float Sc = cef;
    cef *= p.b_r * p.b_r * RF_PI_F;
    fs.x += nx * cef; fs.y += ny * cef; fs.z += nz * cef;
    // dd_Calculate_M123_bpm_2 (:54-89)
    const float tx = Rij.y * nz - Rij.z * ny;
    const float ty = Rij.z * nx - Rij.x * nz;
    const float tz = Rij.x * ny - Rij.y * nx;
    const float wsx = wj.x + wi.x, wsy = wj.y + wi.y, wsz = wj.z + wi.z;
    const float cphi = (wsx * nx + wsy * ny + wsz * nz) * p.dt * 0.5f;
    const float phx = nx * cphi, phy = ny * cphi, phz = nz * cphi;
    Rij = mk3(nx, ny, nz);
    const float M1x = 1.0f + tz * phz + ty * phy;
    const float M1y = phz - tz - ty * phx;
    const float M1z = -phy - tz * phx + ty;
    const float M2x = tz - phz - tx * phy;
    const float M2y = tz * phz + 1.0f + tx * phx;
    const float M2z = -tz * phy + phx - tx;
    const float M3x = -ty - tx * phz + phy;
    const float M3y = -ty * phz + tx - phx;
    const float M3z = ty * phy + tx * phx + 1.0f;
    const float dwx = wj.x - wi.x, dwy = wj.y - wi.y, dwz = wj.z - wi.z;
    // dd_Calculate_mijn_bpm_2 (:105-129)
    {
        float c1 = nx * dwx + ny * dwy + nz * dwz;
        c1 *= p.dt * 0.5f * p.m_G * il;
        const f3 o = Mijn;
        const float mx = M1x * o.x + M1y * o.y + M1z * o.z + nx * c1;
        const float my = M2x * o.x + M2y * o.y + M2z * o.z + ny * c1;
        const float mz = M3x * o.x + M3y * o.y + M3z * o.z + nz * c1;
        Mijn = mk3(mx, my, mz);
        c1 = RF_PI_F * p.b_r * p.b_r * p.b_r * p.b_r;
        ms.x += mx * c1; ms.y += my * c1; ms.z += mz * c1;
    }
    // dd_Calculate_mijt_bpm_2 (:131-152): the summed moment carries dt*E/(4 L0) twice
    {
        const float c1 = nx * dwx + ny * dwy + nz * dwz;
        float c2 = p.dt * 0.25f * p.m_E * il;
        const f3 o = Mijt;
        const float mx = M1x * o.x + M1y * o.y + M1z * o.z + (dwx - nx * c1) * c2;
        const float my = M2x * o.x + M2y * o.y + M2z * o.z + (dwy - ny * c1) * c2;
        const float mz = M3x * o.x + M3y * o.y + M3z * o.z + (dwz - nz * c1) * c2;
        Mijt = mk3(mx, my, mz);
        c2 *= RF_PI_F * p.b_r * p.b_r * p.b_r * p.b_r;
        ms.x += mx * c2; ms.y += my * c2; ms.z += mz * c2;
    }
    // dd_Calculate_fijt_mijunsym_bpm_2 (:154-197)
    float Mc;
    {
        const float hx = 0.5f * wsx, hy = 0.5f * wsy, hz = 0.5f * wsz;
        const float vx = vj.x - vi.x - hy * r.z + hz * r.y;
        const float vy = vj.y - vi.y - hz * r.x + hx * r.z;
        const float vz = vj.z - vi.z - hx * r.y + hy * r.x;
        float c = nx * vx + ny * vy + nz * vz;
        const f3 o = Oijt;
        const float ox = (M1x * o.x + M1y * o.y + M1z * o.z) + (vx - nx * c) * p.dt;
        const float oy = (M2x * o.x + M2y * o.y + M2z * o.z) + (vy - ny * c) * p.dt;
        const float oz = (M3x * o.x + M3y * o.y + M3z * o.z) + (vz - nz * c) * p.dt;
        c = p.m_G * il;
        Mc = c;
        c *= p.b_r * p.b_r * RF_PI_F;
        fs.x += ox * c; fs.y += oy * c; fs.z += oz * c;
        Oijt = mk3(ox, oy, oz);
        ms.x += 0.5f * (r.y * oz - r.z * oy) * c;
        ms.y += 0.5f * (r.z * ox - r.x * oz) * c;
        ms.z += 0.5f * (r.x * oy - r.y * ox) * c;
    }
    // dd_CheckBreakConditionDEM_2 (:20-36)
    Mc *= norm3(Oijt.x, Oijt.y, Oijt.z);
    Sc += norm3(Mijt.x, Mijt.y, Mijt.z) * 4.0f * p.b_r;
    Mc += norm3(Mijn.x, Mijn.y, Mijn.z) * 2.0f * p.b_r;
    if ((Sc > p.m_Gcritn) || (Mc > p.m_Gcritt)) {
        Oijt = mk3(0.f, 0.f, 0.f);
        Mijn = mk3(0.f, 0.f, 0.f);
        Mijt = mk3(0.f, 0.f, 0.f);
        return true;
    }
    return false;
}

// One contact slot of type 0 (d_CalculateForcesDEM_21 loop body, :356-402).
// r = Rj - Ri. Returns true when the pair overlaps (rijm < 2 rP); otherwise the
// caller sets Oijt to zero, as the reference does.
// The overlapping pair (rijm < 2 rP) part of the contact slot; rijm = norm3(r).
__device__ __forceinline__ void contact_pair(const ContactParams& p, const f3 r, const float rijm, const f3 vi,
                                             const f3 vj, const f3 wi, const f3 wj, f3& Oijt, f3& fs, f3& ms);

__device__ __forceinline__ bool contact_slot(const ContactParams& p, const f3 r, const f3 vi, const f3 vj,
                                             const f3 wi, const f3 wj, f3& Oijt, f3& fs, f3& ms) {
    const float rijm = norm3(r.x, r.y, r.z);
    if (!(rijm < 2.0f * p.rP)) return false;
    contact_pair(p, r, rijm, vi, vj, wi, wj, Oijt, fs, ms);
    return true;
}

__device__ __forceinline__ void contact_pair(const ContactParams& p, const f3 r, const float rijm, const f3 vi,
                                             const f3 vj, const f3 wi, const f3 wj, f3& Oijt, f3& fs, f3& ms) {
    const float inv_rm = __frcp_rn(rijm);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    // dd_Calculate_fijn_ppHM_2 (:199-253)
    float c1 = __fsqrt_rn(p.rP * fabsf(p.rP - 0.5f * rijm));
    const float Kn = 2.0f * p.m_E * c1;
    const float Kt = 8.0f * p.m_G * c1;
    const float wsx = wj.x + wi.x, wsy = wj.y + wi.y, wsz = wj.z + wi.z;
    const float vx = vj.x - vi.x + p.rP * (ny * wsz - nz * wsy);
    const float vy = vj.y - vi.y + p.rP * (nz * wsx - nx * wsz);
    const float vz = vj.z - vi.z + p.rP * (nx * wsy - ny * wsx);
    const float vn = nx * vx + ny * vy + nz * vz;
    const float fn = (rijm - 2.0f * p.rP) * Kn * RF_2D3_F;
    c1 = -1.8257f * p.p_A * vn * __fsqrt_rn(Kn * 0.5f * p.mP);
    fs.x += nx * (fn + c1); fs.y += ny * (fn + c1); fs.z += nz * (fn + c1);
    const float vtx = vx - nx * vn, vty = vy - ny * vn, vtz = vz - nz * vn;
    // dd_Calculate_fijtmijt_ppHM_2 (:255-314)
    const f3 o = Oijt;
    float c = nx * o.x + ny * o.y + nz * o.z;
    float ox = o.x - nx * c, oy = o.y - ny * c, oz = o.z - nz * c;
    c = ox * ox + oy * oy + oz * oz;
    if ((double)c > 1e-18) {
        c = __frcp_rn(c);
        c *= o.x * o.x + o.y * o.y + o.z * o.z;
        c = __fsqrt_rn(c);
        ox *= c; oy *= c; oz *= c;
    }
    ox += vtx * p.dt; oy += vty * p.dt; oz += vtz * p.dt;
    float ftx = ox * Kt, fty = oy * Kt, ftz = oz * Kt;
    const float ftm = ftx * ftx + fty * fty + ftz * ftz;
    if (ftm > p.m_mu * p.m_mu * fn * fn) {
        c = p.m_mu * fabsf(fn) * __frsqrt_rn(ftm);
        ftx *= c; fty *= c; ftz *= c;
        c = __frcp_rn(Kt);
        ox = ftx * c; oy = fty * c; oz = ftz * c;
    } else {
        c = -1.8257f * p.p_A * __fsqrt_rn(Kt * 0.5f * p.mP);
        ftx += vtx * c; fty += vty * c; ftz += vtz * c;
    }
    Oijt = mk3(ox, oy, oz);
    fs.x += ftx; fs.y += fty; fs.z += ftz;
    ms.x += (ny * ftz - nz * fty) * p.rP;
    ms.y += (nz * ftx - nx * ftz) * p.rP;
    ms.z += (nx * fty - ny * ftx) * p.rP;
    // dd_Calculate_mijroll_ppHM_2 (:316-336): a (near-)zero spin clears the whole sum
    const float wim = wi.x * wi.x + wi.y * wi.y + wi.z * wi.z;
    if ((double)wim > 1e-18) {
        const float cr = -p.m_muroll * fabsf(fn) * __frsqrt_rn(wim);
        ms.x += wi.x * cr; ms.y += wi.y * cr; ms.z += wi.z * cr;
    } else {
        ms = mk3(0.f, 0.f, 0.f);
    }
}

// rr as the list kernels compute it: __fmul_rn products, summed left to right.
__device__ __forceinline__ float dist2_rn(const f3 a, const f3 b) {
    const float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Cell grid of the reference (cell_data): cell edge a, 1/a, Nr.
struct RefGrid {
    float a, inv_a;
    uint32_t nx, ny, nz;
    uint64_t CN;
};

// d_CalculateCellIndex (md_calculate_cell.cu:39-48): per-axis floorf(x * 1/a) converted
// to unsigned (saturating), linearised x fastest in 32-bit arithmetic.
__device__ __forceinline__ uint32_t ref_cell(const f3 x, const RefGrid& g, uint32_t* cx = nullptr,
                                             uint32_t* cy = nullptr, uint32_t* cz = nullptr) {
    const uint32_t ix = __float2uint_rz(floorf(__fmul_rn(x.x, g.inv_a)));
    const uint32_t iy = __float2uint_rz(floorf(__fmul_rn(x.y, g.inv_a)));
    const uint32_t iz = __float2uint_rz(floorf(__fmul_rn(x.z, g.inv_a)));
    if (cx) { *cx = ix; *cy = iy; *cz = iz; }
    return ix + iy * g.nx + iz * g.ny * g.nx;
}

// The 8 octant cells in the reference's visiting order
// (md_interaction_list_reconstructbpm.cu:91-118): own cell, +x, +y, +z, +xy, +xz, +yz, +xyz,
// each step towards the half of the cell the particle sits in.
__device__ __forceinline__ void octant_cells(const f3 x, const RefGrid& g, int64_t cells[8]) {
    uint32_t ix, iy, iz;
    const uint32_t c = ref_cell(x, g, &ix, &iy, &iz);
    const float hx = __fadd_rn((float)ix, 0.5f), hy = __fadd_rn((float)iy, 0.5f), hz = __fadd_rn((float)iz, 0.5f);
    const int sx = signbit(x.x - __fmul_rn(hx, g.a)) ? -1 : 1;
    const int sy = signbit(x.y - __fmul_rn(hy, g.a)) ? -1 : 1;
    const int sz = signbit(x.z - __fmul_rn(hz, g.a)) ? -1 : 1;
    const int64_t ox = sx, oy = (int64_t)sy * g.nx, oz = (int64_t)sz * g.ny * g.nx;
    const int64_t b = (int64_t)c;
    cells[0] = b;           cells[1] = b + ox;           cells[2] = b + oy;      cells[3] = b + oz;
    cells[4] = b + ox + oy; cells[5] = b + ox + oz;      cells[6] = b + oy + oz; cells[7] = b + ox + oy + oz;
}

// The same 8 cells as base + offsets (compact form for register-tight kernels).
struct Octant {
    int64_t b, ox, oy, oz;
};
__device__ __forceinline__ Octant octant_of(const f3 x, const RefGrid& g) {
    uint32_t ix, iy, iz;
    const uint32_t c = ref_cell(x, g, &ix, &iy, &iz);
    const float hx = __fadd_rn((float)ix, 0.5f), hy = __fadd_rn((float)iy, 0.5f), hz = __fadd_rn((float)iz, 0.5f);
    Octant o;
    o.b = (int64_t)c;
    o.ox = signbit(x.x - __fmul_rn(hx, g.a)) ? -1 : 1;
    o.oy = (signbit(x.y - __fmul_rn(hy, g.a)) ? -1 : 1) * (int64_t)g.nx;
    o.oz = (signbit(x.z - __fmul_rn(hz, g.a)) ? -1 : 1) * (int64_t)g.ny * g.nx;
    return o;
}
// Rank of cell cj in the visiting order own, +x, +y, +z, +xy, +xz, +yz, +xyz, or -1.
__device__ __forceinline__ int octant_rank(const Octant& o, uint32_t cj) {
    const int64_t dlt = (int64_t)cj - o.b;
    if (dlt == 0) return 0;
    if (dlt == o.ox) return 1;
    if (dlt == o.oy) return 2;
    if (dlt == o.oz) return 3;
    if (dlt == o.ox + o.oy) return 4;
    if (dlt == o.ox + o.oz) return 5;
    if (dlt == o.oy + o.oz) return 6;
    if (dlt == o.ox + o.oy + o.oz) return 7;
    return -1;
}

// Rank (0..7) of cell cj among the octant cells of a particle at x, or -1.
__device__ __forceinline__ int octant_rank(const int64_t cells[8], uint32_t cj) {
    const int64_t c = (int64_t)cj;
#pragma unroll
    for (int r = 0; r < 8; ++r)
        if (cells[r] == c) return r;
    return -1;
}

// d_braziltest_simple2 per particle (md_braziltest_simple2.cu:28-92); returns contributions.
__device__ __forceinline__ void brazil_particle(float& Rx, float& Ry, float& Rz, float& Vx, float& Vy, float& Vz,
                                                float& Fx, float& Fy, float& Fz, const rf_float3 c, float RR, float Yt,
                                                float Yb, float Ytr, float Ybr, float vt, float Zcut, double& sfb,
                                                double& sft) {
    const float rx = Rx - c.x, ry = Ry, rz = Rz - c.z;
    if (rx * rx + rz * rz < RR && rz < Zcut) {
        if ((double)(ry - Ytr) > -1e-9) {
            const float fy = Fy;
            if (fy > 0) {
                sft += (double)fy;
                float iv = Vx * Vx + Vz * Vz;
                if ((double)iv > 1e-9) {
                    iv = __frsqrt_rn(iv);
                    Fx -= 0.45f * fy * Vx * iv;
                    Fz -= 0.45f * fy * Vz * iv;
                }
            }
            if ((double)(ry - Yt) > -1e-9) { Ry = Yt; Vy = vt; Fy = 0.f; }
        }
        if ((double)(ry - Ybr) < 1e-9) {
            const float fy = Fy;
            if (fy < 0) {
                sfb += (double)fy;
                float iv = Vx * Vx + Vz * Vz;
                if ((double)iv > 1e-9) {
                    iv = __frsqrt_rn(iv);
                    Fx += 0.45f * fy * Vx * iv;
                    Fz += 0.45f * fy * Vz * iv;
                }
            }
            if ((double)(ry - Yb) < 1e-9) { Ry = Yb; Vy = 0.f; Fy = 0.f; }
        }
    }
}

// d_UniaxialCompression3_simple per particle (md_uniaxialcompression3_simple.cu:28-224).
__device__ __forceinline__ void uniaxial_particle(float& Rx, float& Ry, float& Rz, float& Vz, float& Fz,
                                                  const rf_float3 c, float RR, float Zt, float Zb, float Ztr, float Zbr,
                                                  float vt, float Zcut, double& sfb, double& sft) {
    const float rx = Rx - c.x, ry = Ry - c.y, rz = Rz;
    if (rx * rx + ry * ry < RR && rz < Zcut) {
        if ((double)(rz - Ztr) > -1e-9) {
            const float fz = Fz;
            if (fz > 0) sft += (double)fz;
            if ((double)(rz - Zt) > -1e-9) { Rz = Zt; Vz = vt; Fz = 0.f; }
        }
        if ((double)(rz - Zbr) < 1e-9) {
            const float fz = Fz;
            if (fz < 0) sfb += (double)fz;
            if ((double)(rz - Zb) < 1e-9) { Rz = Zb; Vz = 0.f; Fz = 0.f; }
        }
    }
}

__device__ __forceinline__ bool outside_box(float Rx, float Ry, float Rz, const rf_float3 c, const rf_float3 h) {
    const float dx = Rx - c.x, dy = Ry - c.y, dz = Rz - c.z;
    return (dx - h.x > 0) || (dx + h.x < 0) || (dy - h.y > 0) || (dy + h.y < 0) || (dz - h.z > 0) || (dz + h.z < 0);
}

}  // namespace rf

// ===========================================================================
// Extended model: polydisperse particles, per-bond stiffness and strength, FP64
// positions. Each formula is the reference's with its mono-sized constants replaced:
//   E/L0 -> kn, G/L0 -> ks (normal / shear stiffness per area, kn = E/L0 as the
//   reference's moduli imply), b_r -> the bond's radius (lambda * min(r_i, r_j)),
//   2 rP -> r_i + r_j, rP*(rP - r/2) -> R* delta/2... (equivalent radius),
//   0.5 mP -> m* (equivalent mass), rP lever arms -> r_i.
// Positions are double; r = Rj - Ri and the bond stretch |r| - L0 are formed in
// double and rounded once to float, so small increments and small strains survive.
// ===========================================================================
namespace rf {

struct BondExt {            // per-bond constants of the extended model
    float kn, ks, br, sc, tc;   // stiffness (normal, shear), bond radius, tensile and shear strength
    double L0;                  // initial length
};
struct ExtParams {
    float dt, hm_E, hm_G, p_A, mu, mur;
};

// One bond slot of the extended model (same structure and order as bond_slot).
// rlen = |r| in double; r is the float rounding of the double separation.
// q1: sum the bending moment with the reference's extra dt*E/(4 L0) factor (its Q1,
// md_calculateforcesdem3.cu:131-152), as the reference-constants mode does.
__device__ __forceinline__ bool bond_slot_ext(const ExtParams& p, const BondExt& b, const f3 r, const double rlen,
                                              const f3 vi, const f3 vj, const f3 wi, const f3 wj, f3& Rij, f3& Oijt,
                                              f3& Mijn, f3& Mijt, f3& fs, f3& ms, float& fnabs, float& kt,
                                              float& kr, const bool q1 = false) {
    const float rijm = (float)rlen;
    const float inv_rm = __frcp_rn(rijm);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    const float stretch = (float)(rlen - b.L0);     // in double: no cancellation at small strains
    const float A = b.br * b.br * RF_PI_F;
    const float J = RF_PI_F * b.br * b.br * b.br * b.br;
    // translational and rotational stiffness of the bond (FIRE mass scaling)
    kt += (b.kn + b.ks) * A;
    kr += 0.25f * b.kn * J + 0.5f * b.ks * J + 0.25f * b.ks * A * rijm * rijm;
    float cef = b.kn * stretch;
    float Sc = cef;
    cef *= A;
    fnabs += fabsf(cef);
    fs.x += nx * cef; fs.y += ny * cef; fs.z += nz * cef;
    const float tx = Rij.y * nz - Rij.z * ny;
    const float ty = Rij.z * nx - Rij.x * nz;
    const float tz = Rij.x * ny - Rij.y * nx;
    const float wsx = wj.x + wi.x, wsy = wj.y + wi.y, wsz = wj.z + wi.z;
    const float cphi = (wsx * nx + wsy * ny + wsz * nz) * p.dt * 0.5f;
    const float phx = nx * cphi, phy = ny * cphi, phz = nz * cphi;
    Rij = mk3(nx, ny, nz);
    const float M1x = 1.0f + tz * phz + ty * phy;
    const float M1y = phz - tz - ty * phx;
    const float M1z = -phy - tz * phx + ty;
    const float M2x = tz - phz - tx * phy;
    const float M2y = tz * phz + 1.0f + tx * phx;
    const float M2z = -tz * phy + phx - tx;
    const float M3x = -ty - tx * phz + phy;
    const float M3y = -ty * phz + tx - phx;
    const float M3z = ty * phy + tx * phx + 1.0f;
    const float dwx = wj.x - wi.x, dwy = wj.y - wi.y, dwz = wj.z - wi.z;
    {
        float c1 = nx * dwx + ny * dwy + nz * dwz;
        c1 *= p.dt * 0.5f * b.ks;
        const f3 o = Mijn;
        const float mx = M1x * o.x + M1y * o.y + M1z * o.z + nx * c1;
        const float my = M2x * o.x + M2y * o.y + M2z * o.z + ny * c1;
        const float mz = M3x * o.x + M3y * o.y + M3z * o.z + nz * c1;
        Mijn = mk3(mx, my, mz);
        ms.x += mx * J; ms.y += my * J; ms.z += mz * J;
    }
    {
        const float c1 = nx * dwx + ny * dwy + nz * dwz;
        float c2 = p.dt * 0.25f * b.kn;
        const f3 o = Mijt;
        const float mx = M1x * o.x + M1y * o.y + M1z * o.z + (dwx - nx * c1) * c2;
        const float my = M2x * o.x + M2y * o.y + M2z * o.z + (dwy - ny * c1) * c2;
        const float mz = M3x * o.x + M3y * o.y + M3z * o.z + (dwz - nz * c1) * c2;
        Mijt = mk3(mx, my, mz);
        // bending moment kn * (pi br^4 / 4) * angle = Mijt * J; the reference's extra
        // factor dt*E/(4 L0) here (its Q1) is carried only in the reference-constants mode
        if (q1) {
            const float q = c2 * J;
            ms.x += mx * q; ms.y += my * q; ms.z += mz * q;
        } else {
            ms.x += mx * J; ms.y += my * J; ms.z += mz * J;
        }
    }
    float Mc;
    {
        const float hx = 0.5f * wsx, hy = 0.5f * wsy, hz = 0.5f * wsz;
        const float vx = vj.x - vi.x - hy * r.z + hz * r.y;
        const float vy = vj.y - vi.y - hz * r.x + hx * r.z;
        const float vz = vj.z - vi.z - hx * r.y + hy * r.x;
        float c = nx * vx + ny * vy + nz * vz;
        const f3 o = Oijt;
        const float ox = (M1x * o.x + M1y * o.y + M1z * o.z) + (vx - nx * c) * p.dt;
        const float oy = (M2x * o.x + M2y * o.y + M2z * o.z) + (vy - ny * c) * p.dt;
        const float oz = (M3x * o.x + M3y * o.y + M3z * o.z) + (vz - nz * c) * p.dt;
        c = b.ks;
        Mc = c;
        c *= A;
        fs.x += ox * c; fs.y += oy * c; fs.z += oz * c;
        Oijt = mk3(ox, oy, oz);
        ms.x += 0.5f * (r.y * oz - r.z * oy) * c;
        ms.y += 0.5f * (r.z * ox - r.x * oz) * c;
        ms.z += 0.5f * (r.x * oy - r.y * ox) * c;
    }
    Mc *= norm3(Oijt.x, Oijt.y, Oijt.z);
    Sc += norm3(Mijt.x, Mijt.y, Mijt.z) * 4.0f * b.br;
    Mc += norm3(Mijn.x, Mijn.y, Mijn.z) * 2.0f * b.br;
    if ((Sc > b.sc) || (Mc > b.tc)) {
        Oijt = mk3(0.f, 0.f, 0.f);
        Mijn = mk3(0.f, 0.f, 0.f);
        Mijt = mk3(0.f, 0.f, 0.f);
        return true;
    }
    return false;
}

// One bond record inside a quasi-static increment (FIRE mode). The state is the record's
// state at the start of the increment (Rij0, Oijt0, Mijn0, Mijt0) carried to the current
// configuration in one step -- the start normal to the current one, the particles'
// rotations ti, tj since the increment began, and du, the pair's relative motion since
// then less the mean rotation's part ((r - r0) - ((ti + tj) / 2) x r, formed in double
// by the caller: in float its terms cancel and the relaxation stalls on the rounding) --
// with the formulas of bond_slot_ext. The relaxed state so depends on where the particles
// are, not on the path the relaxation took: an exact warm start lands on it at once.
__device__ __forceinline__ bool bond_slot_ext_total(const ExtParams& p, const BondExt& b, const f3 r,
                                                    const double rlen, const f3 du, const f3 ti, const f3 tj,
                                                    const f3 Rij0, const f3 Oijt0, const f3 Mijn0, const f3 Mijt0,
                                                    f3& Rij, f3& Oijt, f3& Mijn, f3& Mijt, f3& fs, f3& ms,
                                                    float& fnabs, float& kt, float& kr) {
    const float rijm = (float)rlen;
    const float inv_rm = __frcp_rn(rijm);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    const float stretch = (float)(rlen - b.L0);
    const float A = b.br * b.br * RF_PI_F;
    const float J = RF_PI_F * b.br * b.br * b.br * b.br;
    kt += (b.kn + b.ks) * A;
    kr += 0.25f * b.kn * J + 0.5f * b.ks * J + 0.25f * b.ks * A * rijm * rijm;
    float cef = b.kn * stretch;
    float Sc = cef;
    cef *= A;
    fnabs += fabsf(cef);
    fs.x += nx * cef; fs.y += ny * cef; fs.z += nz * cef;
    const float tx = Rij0.y * nz - Rij0.z * ny;
    const float ty = Rij0.z * nx - Rij0.x * nz;
    const float tz = Rij0.x * ny - Rij0.y * nx;
    const float wsx = tj.x + ti.x, wsy = tj.y + ti.y, wsz = tj.z + ti.z;
    const float cphi = (wsx * nx + wsy * ny + wsz * nz) * 0.5f;
    const float phx = nx * cphi, phy = ny * cphi, phz = nz * cphi;
    Rij = mk3(nx, ny, nz);
    const float M1x = 1.0f + tz * phz + ty * phy;
    const float M1y = phz - tz - ty * phx;
    const float M1z = -phy - tz * phx + ty;
    const float M2x = tz - phz - tx * phy;
    const float M2y = tz * phz + 1.0f + tx * phx;
    const float M2z = -tz * phy + phx - tx;
    const float M3x = -ty - tx * phz + phy;
    const float M3y = -ty * phz + tx - phx;
    const float M3z = ty * phy + tx * phx + 1.0f;
    const float dwx = tj.x - ti.x, dwy = tj.y - ti.y, dwz = tj.z - ti.z;
    {
        float c1 = nx * dwx + ny * dwy + nz * dwz;
        c1 *= 0.5f * b.ks;
        const f3 o = Mijn0;
        const float mx = M1x * o.x + M1y * o.y + M1z * o.z + nx * c1;
        const float my = M2x * o.x + M2y * o.y + M2z * o.z + ny * c1;
        const float mz = M3x * o.x + M3y * o.y + M3z * o.z + nz * c1;
        Mijn = mk3(mx, my, mz);
        ms.x += mx * J; ms.y += my * J; ms.z += mz * J;
    }
    {
        const float c1 = nx * dwx + ny * dwy + nz * dwz;
        const float c2 = 0.25f * b.kn;
        const f3 o = Mijt0;
        const float mx = M1x * o.x + M1y * o.y + M1z * o.z + (dwx - nx * c1) * c2;
        const float my = M2x * o.x + M2y * o.y + M2z * o.z + (dwy - ny * c1) * c2;
        const float mz = M3x * o.x + M3y * o.y + M3z * o.z + (dwz - nz * c1) * c2;
        Mijt = mk3(mx, my, mz);
        ms.x += mx * J; ms.y += my * J; ms.z += mz * J;
    }
    float Mc;
    {
        float c = nx * du.x + ny * du.y + nz * du.z;
        const f3 o = Oijt0;
        const float ox = (M1x * o.x + M1y * o.y + M1z * o.z) + (du.x - nx * c);
        const float oy = (M2x * o.x + M2y * o.y + M2z * o.z) + (du.y - ny * c);
        const float oz = (M3x * o.x + M3y * o.y + M3z * o.z) + (du.z - nz * c);
        c = b.ks;
        Mc = c;
        c *= A;
        fs.x += ox * c; fs.y += oy * c; fs.z += oz * c;
        Oijt = mk3(ox, oy, oz);
        ms.x += 0.5f * (r.y * oz - r.z * oy) * c;
        ms.y += 0.5f * (r.z * ox - r.x * oz) * c;
        ms.z += 0.5f * (r.x * oy - r.y * ox) * c;
    }
    Mc *= norm3(Oijt.x, Oijt.y, Oijt.z);
    Sc += norm3(Mijt.x, Mijt.y, Mijt.z) * 4.0f * b.br;
    Mc += norm3(Mijn.x, Mijn.y, Mijn.z) * 2.0f * b.br;
    if ((Sc > b.sc) || (Mc > b.tc)) {
        Oijt = mk3(0.f, 0.f, 0.f);
        Mijn = mk3(0.f, 0.f, 0.f);
        Mijt = mk3(0.f, 0.f, 0.f);
        return true;
    }
    return false;
}

// Overlapping pair of the extended model. delta = r_i + r_j - |r| is formed in double
// by the caller (in float it would cancel to a few significant bits at small overlaps);
// mi, mj are the masses.
__device__ __forceinline__ void contact_pair_ext(const ExtParams& p, const f3 r, const float rijm, const float delta,
                                                 const float ri, const float rj, const float mi, const float mj,
                                                 const f3 vi, const f3 vj, const f3 wi, const f3 wj, f3& Oijt, f3& fs,
                                                 f3& ms, float& fnabs, float& kt, float& kr) {
    const float inv_rm = __frcp_rn(rijm);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    const float Rs = ri * rj / (ri + rj);               // equivalent radius (rP/2 for equal sizes)
    const float ms_ = mi * mj / (mi + mj);             // equivalent mass (mP/2 for equal masses)
    float c1 = __fsqrt_rn(Rs * fabsf(delta));
    const float Kn = 2.0f * p.hm_E * c1;
    const float Kt = 8.0f * p.hm_G * c1;
    kt += Kn + Kt;                                      // contact stiffness (FIRE mass scaling)
    kr += Kt * ri * ri;
    // relative velocity of the contact point: vj - vi + n x (ri wi + rj wj)
    const float ax = ri * wi.x + rj * wj.x, ay = ri * wi.y + rj * wj.y, az = ri * wi.z + rj * wj.z;
    const float vx = vj.x - vi.x + (ny * az - nz * ay);
    const float vy = vj.y - vi.y + (nz * ax - nx * az);
    const float vz = vj.z - vi.z + (nx * ay - ny * ax);
    const float vn = nx * vx + ny * vy + nz * vz;
    const float fn = -delta * Kn * RF_2D3_F;
    fnabs += fabsf(fn);
    c1 = -1.8257f * p.p_A * vn * __fsqrt_rn(Kn * ms_);
    fs.x += nx * (fn + c1); fs.y += ny * (fn + c1); fs.z += nz * (fn + c1);
    const float vtx = vx - nx * vn, vty = vy - ny * vn, vtz = vz - nz * vn;
    const f3 o = Oijt;
    float c = nx * o.x + ny * o.y + nz * o.z;
    float ox = o.x - nx * c, oy = o.y - ny * c, oz = o.z - nz * c;
    c = ox * ox + oy * oy + oz * oz;
    if ((double)c > 1e-18) {
        c = __frcp_rn(c);
        c *= o.x * o.x + o.y * o.y + o.z * o.z;
        c = __fsqrt_rn(c);
        ox *= c; oy *= c; oz *= c;
    }
    ox += vtx * p.dt; oy += vty * p.dt; oz += vtz * p.dt;
    float ftx = ox * Kt, fty = oy * Kt, ftz = oz * Kt;
    const float ftm = ftx * ftx + fty * fty + ftz * ftz;
    if (ftm > p.mu * p.mu * fn * fn) {
        c = p.mu * fabsf(fn) * __frsqrt_rn(ftm);
        ftx *= c; fty *= c; ftz *= c;
        c = __frcp_rn(Kt);
        ox = ftx * c; oy = fty * c; oz = ftz * c;
    } else {
        c = -1.8257f * p.p_A * __fsqrt_rn(Kt * ms_);
        ftx += vtx * c; fty += vty * c; ftz += vtz * c;
    }
    Oijt = mk3(ox, oy, oz);
    fs.x += ftx; fs.y += fty; fs.z += ftz;
    ms.x += (ny * ftz - nz * fty) * ri;
    ms.y += (nz * ftx - nx * ftz) * ri;
    ms.z += (nx * fty - ny * ftx) * ri;
    if (p.mur != 0.f) {           // rolling resistance, with the reference's zero-spin clear
        const float wim = wi.x * wi.x + wi.y * wi.y + wi.z * wi.z;
        if ((double)wim > 1e-18) {
            const float cr = -p.mur * fabsf(fn) * __frsqrt_rn(wim);
            ms.x += wi.x * cr; ms.y += wi.y * cr; ms.z += wi.z * cr;
        } else {
            ms = mk3(0.f, 0.f, 0.f);
        }
    }
}

}  // namespace rf
