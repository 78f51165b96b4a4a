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
//   2 rP -> r_i + r_j, rP*(rP - r/2) -> R* delta (equivalent radius),
//   0.5 mP -> m* (equivalent mass), rP lever arms -> r_i.
// Positions are double; r = Rj - Ri and |r|^2 are formed in double. The bond stretch
// |r| - L0 and the contact overlap r_i + r_j - |r| are taken as differences of squares
// (|r|^2 - L0^2 in double, then divided by |r| + L0 in float), so small strains and
// overlaps keep their precision without a double square root.
// This model's own arithmetic is written with explicit fused multiply-adds (fm, dot3,
// the cross products below): the CPU oracle restates every one with std::fma, so the
// two still agree bit for bit, with about a third fewer floating-point instructions
// than separate multiplies and adds.
// ===========================================================================
namespace rf {

struct BondExt {            // per-bond constants of the extended model
    float kn, ks, br, sc, tc;   // stiffness (normal, shear), bond radius, tensile and shear strength
    double L0;                  // initial length
};
struct ExtParams {
    float dt, hm_E, hm_G, p_A, mu, mur;
};

__device__ __forceinline__ float fm(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// a . b = a.x b.x + (a.y b.y + a.z b.z), fused
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return fm(ax, bx, fm(ay, by, az * bz));
}
// |r| and the stretch |r| - L0 of a pair from the double |r|^2 (see above)
__device__ __forceinline__ float len_from_sq(double rr) { return __fsqrt_rn((float)rr); }
__device__ __forceinline__ float stretch_from_sq(double rr, double L0, float rlen) {
    return (float)fma(-L0, L0, rr) * __frcp_rn(rlen + (float)L0);
}

// The part shared by the explicit and the quasi-static bond update: normal force, the
// incremental rotation matrix built from the previous normal Rp and the rotation
// increment ws = (rotation of i + rotation of j) (times dt/2 in cphi), torsion and
// bending of the moments Mn0, Mt0 by the relative rotation dw, the shear displacement
// Ot0 carried by the same matrix plus the tangential part of du; the break check.
// dts: dt for the explicit step (rates), 1 for the quasi-static total (displacements).
// q1: the bending moment is summed with the reference's extra dt*E/(4 L0) factor.
__device__ __forceinline__ bool bond_core(const BondExt& b, const f3 r, const float rlen, const float stretch,
                                          const float dts, const f3 Rp, const f3 ws, const f3 dw, const f3 du,
                                          const f3 Ot0, const f3 Mn0, const f3 Mt0, f3& Rij, f3& Oijt, f3& Mijn,
                                          f3& Mijt, f3& fs, f3& ms, float& fnabs, float& kt, float& kr, const bool q1) {
    const float inv_rm = __frcp_rn(rlen);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    const float A = b.br * b.br * RF_PI_F;
    const float J = A * (b.br * b.br);
    // translational and rotational stiffness of the bond (FIRE mass scaling)
    kt = fm(b.kn + b.ks, A, kt);
    kr = fm(0.25f * b.ks * A, rlen * rlen, fm(fm(0.25f, b.kn, 0.5f * b.ks), J, kr));
    const float Sn = b.kn * stretch;           // tensile stress
    const float cef = Sn * A;
    fnabs += fabsf(cef);
    fs.x = fm(nx, cef, fs.x); fs.y = fm(ny, cef, fs.y); fs.z = fm(nz, cef, fs.z);
    // rotation-increment matrix: t = Rp x n, phi = n (n . ws) dts / 2
    const float tx = fm(Rp.y, nz, -(Rp.z * ny));
    const float ty = fm(Rp.z, nx, -(Rp.x * nz));
    const float tz = fm(Rp.x, ny, -(Rp.y * nx));
    const float cphi = dot3(ws.x, ws.y, ws.z, nx, ny, nz) * (dts * 0.5f);
    const float phx = nx * cphi, phy = ny * cphi, phz = nz * cphi;
    Rij = mk3(nx, ny, nz);
    const float M1x = fm(tz, phz, fm(ty, phy, 1.0f)), M1y = fm(-ty, phx, phz - tz), M1z = fm(-tz, phx, ty - phy);
    const float M2x = fm(-tx, phy, tz - phz), M2y = fm(tz, phz, fm(tx, phx, 1.0f)), M2z = fm(-tz, phy, phx - tx);
    const float M3x = fm(-tx, phz, phy - ty), M3y = fm(-ty, phz, tx - phx), M3z = fm(ty, phy, fm(tx, phx, 1.0f));
    const float c1 = dot3(nx, ny, nz, dw.x, dw.y, dw.z);
    {   // torsion
        const float ct = c1 * (dts * 0.5f * b.ks);
        const float mx = fm(M1x, Mn0.x, fm(M1y, Mn0.y, fm(M1z, Mn0.z, nx * ct)));
        const float my = fm(M2x, Mn0.x, fm(M2y, Mn0.y, fm(M2z, Mn0.z, ny * ct)));
        const float mz = fm(M3x, Mn0.x, fm(M3y, Mn0.y, fm(M3z, Mn0.z, nz * ct)));
        Mijn = mk3(mx, my, mz);
        ms.x = fm(mx, J, ms.x); ms.y = fm(my, J, ms.y); ms.z = fm(mz, J, ms.z);
    }
    {   // bending: kn * (pi br^4 / 4) * angle = Mijt * J
        const float c2 = dts * 0.25f * b.kn;
        const float mx = fm(M1x, Mt0.x, fm(M1y, Mt0.y, fm(M1z, Mt0.z, fm(-nx, c1, dw.x) * c2)));
        const float my = fm(M2x, Mt0.x, fm(M2y, Mt0.y, fm(M2z, Mt0.z, fm(-ny, c1, dw.y) * c2)));
        const float mz = fm(M3x, Mt0.x, fm(M3y, Mt0.y, fm(M3z, Mt0.z, fm(-nz, c1, dw.z) * c2)));
        Mijt = mk3(mx, my, mz);
        const float q = q1 ? c2 * J : J;      // Q1: the reference's factor again
        ms.x = fm(mx, q, ms.x); ms.y = fm(my, q, ms.y); ms.z = fm(mz, q, ms.z);
    }
    float Mc;
    {   // shear displacement and force, and the moment of the force about the bond's middle
        const float c = dot3(nx, ny, nz, du.x, du.y, du.z);
        const float ox = fm(M1x, Ot0.x, fm(M1y, Ot0.y, fm(M1z, Ot0.z, fm(-nx, c, du.x) * dts)));
        const float oy = fm(M2x, Ot0.x, fm(M2y, Ot0.y, fm(M2z, Ot0.z, fm(-ny, c, du.y) * dts)));
        const float oz = fm(M3x, Ot0.x, fm(M3y, Ot0.y, fm(M3z, Ot0.z, fm(-nz, c, du.z) * dts)));
        Oijt = mk3(ox, oy, oz);
        const float k = b.ks * A;
        fs.x = fm(ox, k, fs.x); fs.y = fm(oy, k, fs.y); fs.z = fm(oz, k, fs.z);
        const float hk = 0.5f * k;
        ms.x = fm(fm(r.y, oz, -(r.z * oy)), hk, ms.x);
        ms.y = fm(fm(r.z, ox, -(r.x * oz)), hk, ms.y);
        ms.z = fm(fm(r.x, oy, -(r.y * ox)), hk, ms.z);
        Mc = b.ks * __fsqrt_rn(dot3(ox, oy, oz, ox, oy, oz));
    }
    // dd_CheckBreakConditionDEM_2's criteria (md_calculateforcesdem3.cu:20-36)
    const float Sc = fm(__fsqrt_rn(dot3(Mijt.x, Mijt.y, Mijt.z, Mijt.x, Mijt.y, Mijt.z)), 4.0f * b.br, Sn);
    Mc = fm(__fsqrt_rn(dot3(Mijn.x, Mijn.y, Mijn.z, Mijn.x, Mijn.y, Mijn.z)), 2.0f * b.br, Mc);
    if ((Sc > b.sc) || (Mc > b.tc)) {
        Oijt = mk3(0.f, 0.f, 0.f);
        Mijn = mk3(0.f, 0.f, 0.f);
        Mijt = mk3(0.f, 0.f, 0.f);
        return true;
    }
    return false;
}

// One bond slot of the extended model in an explicit step (the reference's _22 slot
// with this model's constants): rates v, w integrated over dt. rr = |r|^2 in double.
__device__ __forceinline__ bool bond_slot_ext(const ExtParams& p, const BondExt& b, const f3 r, const double rr,
                                              const f3 vi, const f3 vj, const f3 wi, const f3 wj, f3& Rij, f3& Oijt,
                                              f3& Mijn, f3& Mijt, f3& fs, f3& ms, float& fnabs, float& kt,
                                              float& kr, const bool q1 = false) {
    const float rlen = len_from_sq(rr);
    const float stretch = stretch_from_sq(rr, b.L0, rlen);
    const f3 ws = mk3(wj.x + wi.x, wj.y + wi.y, wj.z + wi.z);
    const f3 dw = mk3(wj.x - wi.x, wj.y - wi.y, wj.z - wi.z);
    // relative velocity of the bond's middle: vj - vi - ((wi + wj) / 2) x r
    const float hx = 0.5f * ws.x, hy = 0.5f * ws.y, hz = 0.5f * ws.z;
    const f3 du = mk3(fm(hz, r.y, fm(-hy, r.z, vj.x - vi.x)), fm(hx, r.z, fm(-hz, r.x, vj.y - vi.y)),
                      fm(hy, r.x, fm(-hx, r.y, vj.z - vi.z)));
    return bond_core(b, r, rlen, stretch, p.dt, Rij, ws, dw, du, Oijt, Mijn, Mijt, Rij, Oijt, Mijn, Mijt, fs, ms,
                     fnabs, kt, kr, q1);
}

// One bond record inside a quasi-static increment (FIRE mode). The state is the record's
// state at the start of the increment (Rij0, Oijt0, Mijn0, Mijt0) carried to the current
// configuration in one step -- the start normal to the current one, the particles'
// rotations ti, tj since the increment began, and du, the pair's relative motion since
// then less the mean rotation's part ((r - r0) - ((ti + tj) / 2) x r, formed in double
// by the caller: in float its terms cancel and the relaxation stalls on the rounding) --
// with the formulas of bond_slot_ext. The relaxed state so depends on where the particles
// are, not on the path the relaxation took: an exact warm start lands on it at once.
__device__ __forceinline__ bool bond_slot_ext_total(const BondExt& b, const f3 r, const double rr, const f3 du,
                                                    const f3 ti, const f3 tj, const f3 Rij0, const f3 Oijt0,
                                                    const f3 Mijn0, const f3 Mijt0, f3& Rij, f3& Oijt, f3& Mijn,
                                                    f3& Mijt, f3& fs, f3& ms, float& fnabs, float& kt, float& kr) {
    const float rlen = len_from_sq(rr);
    const float stretch = stretch_from_sq(rr, b.L0, rlen);
    const f3 ws = mk3(tj.x + ti.x, tj.y + ti.y, tj.z + ti.z);
    const f3 dw = mk3(tj.x - ti.x, tj.y - ti.y, tj.z - ti.z);
    return bond_core(b, r, rlen, stretch, 1.0f, Rij0, ws, dw, du, Oijt0, Mijn0, Mijt0, Rij, Oijt, Mijn, Mijt, fs, ms,
                     fnabs, kt, kr, false);
}

// Overlapping pair of the extended model. rr = |r|^2 and sr = r_i + r_j in double, with
// rr < sr^2; the overlap is (sr^2 - rr) / (sr + |r|). mi, mj are the masses. Returns true
// when the rolling resistance's zero-spin rule cleared the moment sum ms.
__device__ __forceinline__ bool contact_pair_ext(const ExtParams& p, const f3 r, const double rr, const double sr,
                                                 const float ri, const float rj, const float mi, const float mj,
                                                 const f3 vi, const f3 vj, const f3 wi, const f3 wj, f3& Oijt, f3& fs,
                                                 f3& ms, float& fnabs, float& kt, float& kr) {
    const float rijm = len_from_sq(rr);
    const float delta = (float)fma(sr, sr, -rr) * __frcp_rn((float)sr + rijm);
    const float inv_rm = __frcp_rn(rijm);
    const float nx = r.x * inv_rm, ny = r.y * inv_rm, nz = r.z * inv_rm;
    const float Rs = ri * rj * __frcp_rn(ri + rj);      // equivalent radius (rP/2 for equal sizes)
    const float ms_ = mi * mj * __frcp_rn(mi + mj);     // equivalent mass (mP/2 for equal masses)
    const float c0 = __fsqrt_rn(Rs * delta);
    const float Kn = 2.0f * p.hm_E * c0;
    const float Kt = 8.0f * p.hm_G * c0;
    kt += Kn + Kt;                                        // contact stiffness (FIRE mass scaling)
    kr = fm(Kt, ri * ri, kr);
    // relative velocity of the contact point: vj - vi + n x (ri wi + rj wj)
    const float ax = fm(ri, wi.x, rj * wj.x), ay = fm(ri, wi.y, rj * wj.y), az = fm(ri, wi.z, rj * wj.z);
    const float vx = fm(ny, az, fm(-nz, ay, vj.x - vi.x));
    const float vy = fm(nz, ax, fm(-nx, az, vj.y - vi.y));
    const float vz = fm(nx, ay, fm(-ny, ax, vj.z - vi.z));
    const float vn = dot3(nx, ny, nz, vx, vy, vz);
    const float fn = -delta * Kn * RF_2D3_F;
    fnabs += fabsf(fn);
    const float fnd = fm(-1.8257f * p.p_A * vn, __fsqrt_rn(Kn * ms_), fn);
    fs.x = fm(nx, fnd, fs.x); fs.y = fm(ny, fnd, fs.y); fs.z = fm(nz, fnd, fs.z);
    const float vtx = fm(-nx, vn, vx), vty = fm(-ny, vn, vy), vtz = fm(-nz, vn, vz);
    // old tangential overlap: onto the tangent plane, back to its old length
    const f3 o = Oijt;
    float c = dot3(nx, ny, nz, o.x, o.y, o.z);
    float ox = fm(-nx, c, o.x), oy = fm(-ny, c, o.y), oz = fm(-nz, c, o.z);
    c = dot3(ox, oy, oz, ox, oy, oz);
    if ((double)c > 1e-18) {
        c = __fsqrt_rn(dot3(o.x, o.y, o.z, o.x, o.y, o.z) * __frcp_rn(c));
        ox *= c; oy *= c; oz *= c;
    }
    ox = fm(vtx, p.dt, ox); oy = fm(vty, p.dt, oy); oz = fm(vtz, p.dt, oz);
    float ftx = ox * Kt, fty = oy * Kt, ftz = oz * Kt;
    const float ftm = dot3(ftx, fty, ftz, ftx, fty, ftz);
    const float fmax = p.mu * fn;
    if (ftm > fmax * fmax) {                             // Coulomb cap
        c = p.mu * fabsf(fn) * __frsqrt_rn(ftm);
        ftx *= c; fty *= c; ftz *= c;
        c = __frcp_rn(Kt);
        ox = ftx * c; oy = fty * c; oz = ftz * c;
    } else {                                             // tangential damping
        c = -1.8257f * p.p_A * __fsqrt_rn(Kt * ms_);
        ftx = fm(vtx, c, ftx); fty = fm(vty, c, fty); ftz = fm(vtz, c, ftz);
    }
    Oijt = mk3(ox, oy, oz);
    fs.x += ftx; fs.y += fty; fs.z += ftz;
    ms.x = fm(fm(ny, ftz, -(nz * fty)), ri, ms.x);
    ms.y = fm(fm(nz, ftx, -(nx * ftz)), ri, ms.y);
    ms.z = fm(fm(nx, fty, -(ny * ftx)), ri, ms.z);
    if (p.mur != 0.f) {           // rolling resistance, with the reference's zero-spin clear
        const float wim = dot3(wi.x, wi.y, wi.z, wi.x, wi.y, wi.z);
        if ((double)wim > 1e-18) {
            const float cr = -p.mur * fabsf(fn) * __frsqrt_rn(wim);
            ms.x = fm(wi.x, cr, ms.x); ms.y = fm(wi.y, cr, ms.y); ms.z = fm(wi.z, cr, ms.z);
        } else {
            ms = mk3(0.f, 0.f, 0.f);
            return true;
        }
    }
    return false;
}

}  // namespace rf
