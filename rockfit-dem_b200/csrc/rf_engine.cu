// Fused B200 engine for the explicit BPM test loop.
//
// One explicit step of the reference (md_calculationbraziltest.cu:170-190:
// CellDistribution, InteractionListReConstructBPM, F=M=0, _22, _21, platen,
// SumForcesULoading, increments, cut, DeleteFarLinks, CompressB/U) is ONE kernel
// here, one thread per particle:
//
//   delete  -- DeleteFarLinks of the previous step, with this step's positions
//              (the reference runs it at the end of the previous step on the same
//              positions, so the result is identical);
//   add     -- new neighbours inside a_farcut, taken from a Verlet candidate list
//              (cutoff a_farcut + skin, rebuilt only when some particle has moved
//              more than 0.45*skin since the last build) instead of re-binning every
//              step. New links are inserted in the order the reference would insert
//              them: by (octant-cell rank, id), computed from the same float cell
//              arithmetic, into the first free slot;
//   bonds   -- bond slots in slot order (same sums, same rounding as _22);
//   contacts-- contact slots in slot order (as _21), F = (0 + F_bond) + F_contact;
//   platen, increments, cut -- per particle, into the other position buffer;
//   load    -- per-block FP64 partial sums, the last block finishes the scalar
//              step (SumForcesULoading, CompressB/U, fracture, load curve) on device.
//
// Layout in HBM: particle vectors as float4 (x, y, z, 0), double-buffered; rows
// slot-major (ids[k*N + i]) so a warp reading slot k of 32 particles is one
// coalesced 128-byte access; per-slot state as 12 float planes (Rij, Oijt, Mijn,
// Mijt); per-particle 32-bit masks for occupied slots, bond slots and contacts
// with non-zero tangential overlap (so empty and idle slots cost no state reads).
//
// The step loop is a CUDA graph: WHILE(continue) { IF(rebuild) {bin, scan,
// scatter, candidates}; step }, with both conditions set on device by the step
// kernel, so one graph launch advances many steps without host round trips.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>
#include <algorithm>
#include <cuda_bf16.h>
#include "rf_physics.cuh"

#ifndef RF_STEP_MIN_BLOCKS
#define RF_STEP_MIN_BLOCKS 6      // resident 128-thread CTAs per SM the step kernel is compiled for
#endif

#ifndef RF_GRAPH_UNROLL
#define RF_GRAPH_UNROLL 8         // explicit steps per iteration of the graph's WHILE loop
#endif
// outcome of one bond record, handed by the lane that evaluated it to its particle's lane
// (bits 8-12: the record's row slot)
// margin buckets of the candidate lists: a candidate's margin (distance - list cutoff at
// the build) below RF_CB1, RF_CB2, RF_CB3 skins, or above
#define RF_CB1 0.05f
#define RF_CB2 0.15f
#define RF_CB3 0.3f
#define RF_REC_DELETE 1u          // beyond the bond's keep distance: the slot is deleted (partner id in the force word)
#define RF_REC_BROKE 2u           // the bond broke this step
#define RF_REC_PARALLEL 4u        // the pair overlaps: the slot's contact was taken with the bond
#define RF_REC_CLEAR 8u           // that contact's zero-spin rule cleared the particle's moment sum
#ifndef RF_REBUILD_EACH_STEP_N
#define RF_REBUILD_EACH_STEP_N (1u << 20)   // from this many particles the rebuild condition is evaluated every step
#endif

namespace rf {

// Scalar state of the run, device resident (compression_data + result bookkeeping).
struct DevScalars {
    double V, VLoad, Top, Bottom, TopR, BottomR, FractureStress, FractureStrain, MinStress, ZeroStress, Stress,
        Strain, MaxStrain, Size0;
    double size_d[3], center_d[3];
    double sz0;
    double keep_frac;       // post-peak stop: fracture once Stress < keep_frac * peak (0: off)
    float center[3], size[3], sized2[3];
    float RR, _1d_Area, Hd2;
    int32_t Loading, Fracture;
    unsigned long long steps, target, rebuilds, curve_n, broken;
    uint32_t done, err, rebuild, moved, block_counter, pad;
    // largest displacement since the last candidate build of the positions a step reads
    // (FP32 bits of its square, accumulated by the step writing them), for skipping scans
    uint32_t d2max_next;
    float dmax;
    // FIRE relaxation of a quasi-static load increment (extended model)
    double fdt, falpha, fdt0, fdtmax, fdtmin, finc, fdec, falpha0, fshrink, ftol;
    double fresidual, fmean, fpower, fcv, fcf, fcm;
    unsigned long long fiter, fmax_iter, fnpos, fiter_total;
    uint32_t fndelay, fuphill, fconverged, fstop, fcounter, fwarm;
};

struct Consts {
    uint32_t N, K, KC;
    int kind;
    double dt_d, p_r_d;
    BondParams bp;
    ContactParams cp;
    float dtm, dt, dtI;
    float aacut, aa_farcut;
    RefGrid g;
    float zcut;
    rf_float3 box_c, box_h, hp;
    // candidate grid
    float cg_inv_h;
    float cg_ox, cg_oy, cg_oz;
    uint32_t cg_nx, cg_ny, cg_nz, cg_cells;
    float rc2, disp2, hard2;   // rebuild trigger and the displacement the candidate lists cover
    float acut_f;              // sqrt(aacut)
    unsigned long long curve_cap;
    cudaGraphConditionalHandle h_loop, h_rebuild;
    int use_graph;
    // extended model (ext != 0): FP64 positions with radii, per-bond strengths
    int ext;
    ExtParams ep;
    float kn, ks, br_lambda, cmass;     // bond stiffness per area, bond radius / min(r_i, r_j), mass = cmass r^3
    double aa_farcut_d, aacut_d;
    // list rule: lgap_d == 0 lists pairs within a_farcut (add test on the float aacut,
    // delete test on aa_farcut, as the reference); lgap_d > 0 within min(a_farcut, r_i + r_j + g)
    double a_farcut_d, lgap_d;
    float lgap_f, skin_f;
    // reference constants in the extended model (rf_ext_params.ref_mode): per-bond stiffness
    // E/L0, G/L0 from the record's 1/L0, bond radius b_r, the Q1 bending factor, platen
    // coordinates rounded to float as the reference's drivers pass them
    int ref_mode;
    float refE, refG, ref_br;
};

// Per-specimen geometry of a batch (constant during a run): the platen's cut height, the
// cut box and its hidden point, the specimen's particle range and the CTAs touching it.
struct SpecGeom {
    float zcut;
    rf_float3 box_c, box_h, hp;
    uint32_t p0, p1;
    uint32_t b0, b1;
};

struct Dev {
    // batch of specimens (one specimen: spec == sc, geom[0], blk_spec == nullptr)
    DevScalars* spec;           // [nspec] per-specimen platen / result scalars
    const SpecGeom* geom;       // [nspec]
    const uint16_t* blk_spec;   // [blocks] first specimen of each 128-particle CTA
    double2* partial2;          // [blocks] load partials of a CTA's second specimen
    uint32_t nspec;
    double4* posd[2];   // extended model: x, y, z (FP64) and radius
    double* bL0;        // extended model: [QB][N] rest length of each bond record
    float2* bstr;       // extended model: [QB][N] tensile and shear strength of each bond record
    float4* pos[2];
    float4* vel[2];
    float4* ang[2];
    // rows: slot-major, K slots per particle
    uint32_t* ids;      // [N][K] neighbour id of each occupied slot (row-major: a thread walks its own row)
    float* il;          // [K][N] 1/L0 per slot, as the reference layout keeps it (read out only)
    float* cO[2];       // [N][K][3] tangential overlap of type-0 slots, by step parity (read cur, write next)
    uint32_t* live;     // [N] occupied slots
    uint32_t* bond;     // [N] slots holding an intact bond
    uint32_t* cmask;    // [N] type-0 slots whose overlap may be non-zero
    // bond records: the bonds of particle i in slot order, ordinal-major [q][i]
    uint32_t* bj;       // [QB][N] partner id
    uint8_t* bk;        // [QB][N] slot of the record (0xFF: record retired)
    float* bil;         // [QB][N] 1/L0
    float4* bst;        // [3][QB][N] (Rij.xyz Oijt.x) (Oijt.yz Mijn.xy) (Mijn.z Mijt.xyz)
    float4* bst0;       // bst at the start of the current quasi-static increment (FIRE mode)
    uint32_t* nbq;      // [N] records of the particle
    uint32_t* bmask;    // [N] records holding an intact bond
    // Verlet candidates
    uint32_t* cand;     // [KC][N]
    uint32_t* cand_n;   // [N]
    unsigned long long* member;   // [N]
    float4* pos_ref;    // [N]
    float* cmargin;     // [N] smallest (distance - a_farcut) of the non-member candidates at the build
    uint32_t* cbound;   // [N] ends of the candidates' margin buckets (bytes 0-2, see k_rb_cand)
    uint32_t* cg_key;   // [N]
    uint32_t* cg_count; // [cells+1]
    uint32_t* cg_start; // [cells+1]
    uint32_t* cg_fill;  // [cells+1]
    uint32_t* cg_bsum;
    uint32_t* cg_sorted;   // [N]
    double2* partial;   // [blocks]
    // FIRE relaxation (allocated on first use)
    float4* frc;        // [N] net force after the platen clamp
    float4* mom;        // [N] net moment
    double* fpart;      // [blocks][FIRE_SUMS] FP64 block partial sums (of a CTA's first specimen)
    double* fpart2;     // [blocks][FIRE_SUMS] the same for a CTA's second specimen (batches)
    double4* rot;       // [N] accumulated rotation of the increment (sum of w dt)
    double4* x0;        // [N] positions at the start of the increment
    unsigned long long n_particles;
    uint32_t QB;
    double* curve;      // [cap][3]
    DevScalars* sc;
};

__device__ __forceinline__ f3 f4to3(const float4 v) { return mk3(v.x, v.y, v.z); }
// Position of particle j as float4 (x, y, z, radius) in either model.
__device__ __forceinline__ float4 posf(const Dev& d, const Consts& c, uint32_t buf, uint32_t j) {
    if (c.ext) {
        const double4 p = d.posd[buf][j];
        return make_float4((float)p.x, (float)p.y, (float)p.z, (float)p.w);
    }
    return d.pos[buf][j];
}
__device__ __forceinline__ void zero_record(const Dev& d, size_t QN, size_t s) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    d.bst[s] = z; d.bst[s + QN] = z; d.bst[s + 2 * QN] = z;
}

// ---------------------------------------------------------------------------
// Candidate-list rebuild (runs only when the displacement flag is set)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool gate_closed(const Dev& d, const Consts& c) {
    // In graph mode the IF node gates the rebuild; on a plain stream the kernels check.
    return !c.use_graph && (d.sc->rebuild == 0 || d.sc->done);
}

__device__ __forceinline__ uint32_t cg_cell_of(const float4 x, const Consts& c) {
    const float fx = floorf((x.x - c.cg_ox) * c.cg_inv_h);
    const float fy = floorf((x.y - c.cg_oy) * c.cg_inv_h);
    const float fz = floorf((x.z - c.cg_oz) * c.cg_inv_h);
    if (!(fx >= 0.f && fy >= 0.f && fz >= 0.f)) return 0xFFFFFFFFu;
    const uint32_t ix = (uint32_t)fx, iy = (uint32_t)fy, iz = (uint32_t)fz;
    if (ix >= c.cg_nx || iy >= c.cg_ny || iz >= c.cg_nz) return 0xFFFFFFFFu;
    return ix + c.cg_nx * (iy + c.cg_ny * iz);
}

__global__ void k_rb_zero(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= c.cg_cells; q += gridDim.x * blockDim.x) {
        d.cg_count[q] = 0;
        d.cg_fill[q] = 0;
    }
}

__global__ void k_rb_bin(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    const uint32_t cur = (uint32_t)(d.sc->steps & 1);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        uint32_t key = cg_cell_of(posf(d, c, cur, i), c);
        if (key == 0xFFFFFFFFu) key = c.cg_cells;          // parked or outside: tail bin, no candidates
        d.cg_key[i] = key;
        atomicAdd(&d.cg_count[key], 1u);
    }
}

__global__ void k_rb_scan_sums(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    __shared__ uint32_t sh[32];
    const size_t n = (size_t)c.cg_cells + 1, base = (size_t)blockIdx.x * 4096;
    uint32_t s = 0;
    for (int t = threadIdx.x; t < 4096; t += blockDim.x)
        if (base + t < n) s += d.cg_count[base + t];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) d.cg_bsum[blockIdx.x] = v;
    }
}

__global__ void k_rb_scan_totals(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    const uint32_t nb = (c.cg_cells + 1 + 4095) / 4096;
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t b = 0; b < nb; ++b) { uint32_t v = d.cg_bsum[b]; d.cg_bsum[b] = acc; acc += v; }
    }
}

__global__ void k_rb_scan_apply(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    __shared__ uint32_t wsum[32];
    const size_t n = (size_t)c.cg_cells + 1;
    const size_t base = (size_t)blockIdx.x * 4096 + (size_t)threadIdx.x * 4;
    uint32_t v[4], t = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) { v[q] = (base + q < n) ? d.cg_count[base + q] : 0; t += v[q]; }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t incl = t;
    for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += y; }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0, si = s;
        for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, si, o); if (lane >= o) si += y; }
        wsum[lane] = si - s;
    }
    __syncthreads();
    uint32_t run = d.cg_bsum[blockIdx.x] + wsum[w] + incl - t;
#pragma unroll
    for (int q = 0; q < 4; ++q) { if (base + q < n) d.cg_start[base + q] = run; run += v[q]; }
}

__global__ void k_rb_scatter(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const uint32_t key = d.cg_key[i];
        d.cg_sorted[d.cg_start[key] + atomicAdd(&d.cg_fill[key], 1u)] = i;
    }
}

// Candidates: every j != i within rc of i (27 cells), and which of them sit in i's row.
__global__ void k_rb_cand(Dev d, Consts c) {
    if (gate_closed(d, c)) return;
    const uint32_t cur = (uint32_t)(d.sc->steps & 1);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const float4 xi = posf(d, c, cur, i);
        d.pos_ref[i] = xi;
        const uint32_t key = d.cg_key[i];
        uint32_t n = 0;
        if (key < c.cg_cells) {
            const int ix = key % c.cg_nx, iy = (key / c.cg_nx) % c.cg_ny, iz = key / (c.cg_nx * c.cg_ny);
            for (int dz = -1; dz <= 1; ++dz) {
                const int z = iz + dz;
                if (z < 0 || z >= (int)c.cg_nz) continue;
                for (int dy = -1; dy <= 1; ++dy) {
                    const int y = iy + dy;
                    if (y < 0 || y >= (int)c.cg_ny) continue;
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int x = ix + dx;
                        if (x < 0 || x >= (int)c.cg_nx) continue;
                        const uint32_t cell = x + c.cg_nx * (y + c.cg_ny * z);
                        const uint32_t s = d.cg_start[cell], e = s + d.cg_count[cell];
                        for (uint32_t q = s; q < e; ++q) {
                            const uint32_t j = d.cg_sorted[q];
                            if (j == i) continue;
                            const float4 xj = posf(d, c, cur, j);
                            const float ddx = xj.x - xi.x, ddy = xj.y - xi.y, ddz = xj.z - xi.z;
                            const float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            bool near = d2 < c.rc2;
                            if (c.lgap_f > 0.f && near) {
                                const float q = fminf(c.acut_f, (xi.w + xj.w) + c.lgap_f) + c.skin_f;
                                near = d2 < q * q;
                            }
                            if (near) {
                                if (n < c.KC) d.cand[(size_t)n * c.N + i] = j;
                                else raise_status(&d.sc->err, RF_ERR_CAPACITY);
                                ++n;
                            }
                        }
                    }
                }
            }
        }
        if (n > c.KC) n = c.KC;
        d.cand_n[i] = n;
        // candidates in the order of their margin bucket (stable within a bucket): a scan
        // needs no candidate of a bucket whose lower bound the displacements since this
        // build cannot have closed (scan_limit)
        {
            uint32_t jl[64];
            uint8_t bq[64];
            uint32_t cnt[4] = {0u, 0u, 0u, 0u};
            for (uint32_t q = 0; q < n; ++q) {
                const uint32_t j = d.cand[(size_t)q * c.N + i];
                const float4 xj = posf(d, c, cur, j);
                const float ddx = xj.x - xi.x, ddy = xj.y - xi.y, ddz = xj.z - xi.z;
                const float cut = c.lgap_f > 0.f ? fminf(c.acut_f, (xi.w + xj.w) + c.lgap_f) : c.acut_f;
                const float mg = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz) - cut;
                const uint32_t b = mg < RF_CB1 * c.skin_f ? 0u : mg < RF_CB2 * c.skin_f ? 1u : mg < RF_CB3 * c.skin_f ? 2u : 3u;
                jl[q] = j;
                bq[q] = (uint8_t)b;
                ++cnt[b];
            }
            uint32_t pos[4] = {0u, cnt[0], cnt[0] + cnt[1], cnt[0] + cnt[1] + cnt[2]};
            d.cbound[i] = pos[1] | (pos[2] << 8) | (pos[3] << 16);
            for (uint32_t q = 0; q < n; ++q) d.cand[(size_t)(pos[bq[q]]++) * c.N + i] = jl[q];
        }
        // membership: candidates already in the row
        unsigned long long mem = 0ull;
        uint32_t live = d.live[i];
        while (live) {
            const uint32_t k = __ffs(live) - 1;
            live &= live - 1;
            const uint32_t j = d.ids[(size_t)i * c.K + k];
            for (uint32_t q = 0; q < n; ++q)
                if (d.cand[(size_t)q * c.N + i] == j) { mem |= 1ull << q; break; }
        }
        d.member[i] = mem;
        // margin of the nearest non-member candidate: until the displacements since this
        // build add up to it, no candidate can come within its list cutoff
        float mg = 3.0e38f;
        for (uint32_t q = 0; q < n; ++q) {
            if ((mem >> q) & 1ull) continue;
            const float4 xj = posf(d, c, cur, d.cand[(size_t)q * c.N + i]);
            const float ddx = xj.x - xi.x, ddy = xj.y - xi.y, ddz = xj.z - xi.z;
            const float cut = c.lgap_f > 0.f ? fminf(c.acut_f, (xi.w + xj.w) + c.lgap_f) : c.acut_f;
            mg = fminf(mg, sqrtf(ddx * ddx + ddy * ddy + ddz * ddz) - cut);
        }
        d.cmargin[i] = mg;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&d.sc->rebuilds, 1ull);
        d.sc->dmax = 0.f;                     // positions == build positions
    }
}

// ---------------------------------------------------------------------------
// The step kernel
// ---------------------------------------------------------------------------
// Retire the bond record of slot k of particle i, if it has one: its state is
// zeroed (DeleteFarLinks zeroes Rij, Oijt, Mijn, Mijt of the slot) and it stops
// belonging to the slot.
__device__ __forceinline__ void retire_record(const Dev& d, const Consts& c, uint32_t i, uint32_t k, uint32_t nbq,
                                              uint32_t& bmask) {
    const uint32_t N = c.N;
    for (uint32_t q = 0; q < nbq; ++q) {
        const size_t s = (size_t)q * N + i;
        if (d.bk[s] == (uint8_t)k) {
            d.bk[s] = 0xFF;
            zero_record(d, (size_t)d.QB * N, s);
            bmask &= ~(1u << q);
            return;
        }
    }
}

// DeleteFarLinks (md_interaction_list_reconstructbpm.cu:141-186) of one slot.
__device__ __forceinline__ void delete_slot(const Dev& d, const Consts& c, uint32_t i, uint32_t k, uint32_t j,
                                            uint32_t ncand, uint32_t nbq, uint32_t& live, uint32_t& bond, uint32_t& cm,
                                            uint32_t& bmask, unsigned long long& mem) {
    const uint32_t N = c.N;
    const size_t s = (size_t)i * c.K + k;
    d.ids[s] = EMPTY32;                       // its overlap reads as zero once the cmask bit is clear
    d.cmargin[i] = 0.f;                       // the deleted partner may come back: scan until the next build
    retire_record(d, c, i, k, nbq, bmask);
    const uint32_t bit = 1u << k;
    live &= ~bit; bond &= ~bit; cm &= ~bit;
    for (uint32_t q = 0; q < ncand; ++q)
        if (d.cand[(size_t)q * N + i] == j) { mem &= ~(1ull << q); break; }
}

// DeleteFarLinks for every occupied slot of particle i with the current positions.
__device__ __forceinline__ void delete_far(const Dev& d, const Consts& c, const float4* __restrict__ P, uint32_t i,
                                           const f3 xi, uint32_t ncand, uint32_t nbq, uint32_t& live, uint32_t& bond,
                                           uint32_t& cm, uint32_t& bmask, unsigned long long& mem) {
    const uint32_t* row = d.ids + (size_t)i * c.K;
    uint32_t m = live;
    while (m) {
        const uint32_t k = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t j = row[k];
        const float rr = dist2_rn(xi, f4to3(__ldg(&P[j])));
        if (rr > c.aa_farcut || (double)rr < 1e-10) delete_slot(d, c, i, k, j, ncand, nbq, live, bond, cm, bmask, mem);
    }
}

// True when the candidate scan of the add pass cannot find anything: every non-member
// candidate was at least cmargin beyond a_farcut at the last build, and since then this
// particle moved by |x - x_build| and none by more than dmax (the largest displacement
// of the positions this step reads). 10 % and 1e-4 a_farcut of slack cover the float
// rounding of the margins and displacements.
__device__ __forceinline__ bool scan_not_needed(const Dev& d, const Consts& c, uint32_t i, float x, float y, float z) {
    const float4 pr = d.pos_ref[i];
    const float ex = x - pr.x, ey = y - pr.y, ez = z - pr.z;
    const float di = sqrtf(ex * ex + ey * ey + ez * ez);
    return di + d.sc->dmax < 0.9f * d.cmargin[i] - 1e-4f * c.acut_f;
}

// How many of particle i's candidates (in bucket order) a scan must test: the candidates
// of a bucket whose smallest margin the displacements since the build cannot have closed
// (the test of scan_not_needed, with the bucket's lower bound for cmargin) can be skipped.
// After a deletion (cmargin 0) every candidate is tested.
__device__ __forceinline__ uint32_t scan_limit(const Dev& d, const Consts& c, uint32_t i, float x, float y, float z,
                                               uint32_t n) {
    if (!(d.cmargin[i] > 0.f)) return n;
    const float4 pr = d.pos_ref[i];
    const float ex = x - pr.x, ey = y - pr.y, ez = z - pr.z;
    const float reach = sqrtf(ex * ex + ey * ey + ez * ez) + d.sc->dmax + 1e-4f * c.acut_f;
    const uint32_t b = d.cbound[i];
    if (reach < 0.9f * RF_CB1 * c.skin_f) return b & 0xFFu;
    if (reach < 0.9f * RF_CB2 * c.skin_f) return (b >> 8) & 0xFFu;
    if (reach < 0.9f * RF_CB3 * c.skin_f) return (b >> 16) & 0xFFu;
    return n;
}

// Largest squared displacement (since the last build) of the positions a step writes.
__device__ __forceinline__ void note_displacement(const Dev& d, float e2) {
    const uint32_t w = __reduce_max_sync(0xffffffffu, __float_as_uint(e2));
    if ((threadIdx.x & 31) == 0 && w) atomicMax(&d.sc->d2max_next, w);
}

// The delete pass of the last step, applied before the state is read out: the step
// kernel defers each step's DeleteFarLinks to the start of the next step (same
// positions), so a snapshot taken between steps applies it first. Idempotent.
__global__ void k_delete_pending(Dev d, Consts c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < c.N;
    const float4* P = d.pos[d.sc->steps & 1ull];
    f3 xi = mk3(0.f, 0.f, 0.f);
    uint32_t live = 0, bond = 0, cm = 0, ncand = 0, nbq = 0, bmask = 0;
    unsigned long long mem = 0ull;
    if (valid) {
        xi = f4to3(P[i]);
        live = d.live[i]; bond = d.bond[i]; cm = d.cmask[i]; mem = d.member[i]; ncand = d.cand_n[i];
        nbq = d.nbq[i]; bmask = d.bmask[i];
    }
    const uint32_t live0 = live;
    delete_far(d, c, P, i, xi, ncand, nbq, live, bond, cm, bmask, mem);
    if (valid && live != live0) {
        d.live[i] = live; d.bond[i] = bond; d.cmask[i] = cm; d.member[i] = mem; d.bmask[i] = bmask;
    }
}

// End of a step: block partial sums of the platen loads (fixed tree, deterministic);
// the last block to finish does SumForcesULoading (md_results.cu:34-74) and
// CompressB/U (md_data_types.h:223-293) and sets the graph conditions.
template <int KIND>
__device__ __forceinline__ void step_finish(const Dev& d, const Consts& c, double sfb, double sft,
                                            uint32_t nbroken, uint32_t moved) {
    DevScalars* sc = d.sc;
    const uint32_t FULL = 0xffffffffu;
    // ---- block reductions (fixed tree: deterministic)
    __shared__ double s_b[4], s_t[4];
    __shared__ uint32_t s_n[4], s_m[4];
    __shared__ bool s_last;
    for (int o = 16; o; o >>= 1) {
        sfb += __shfl_xor_sync(FULL, sfb, o);
        sft += __shfl_xor_sync(FULL, sft, o);
    }
    const uint32_t wn = __reduce_add_sync(FULL, nbroken), wm = __reduce_or_sync(FULL, moved);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { s_b[w] = sfb; s_t[w] = sft; s_n[w] = wn; s_m[w] = wm; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double b = (s_b[0] + s_b[1]) + (s_b[2] + s_b[3]);
        const double t = (s_t[0] + s_t[1]) + (s_t[2] + s_t[3]);
        d.partial[blockIdx.x] = make_double2(b, t);
        const uint32_t nb = s_n[0] + s_n[1] + s_n[2] + s_n[3];
        if (nb) atomicAdd(&sc->broken, (unsigned long long)nb);
        if (s_m[0] | s_m[1] | s_m[2] | s_m[3]) atomicOr(&sc->moved, 1u);
        __threadfence();
        const uint32_t ticket = atomicAdd(&sc->block_counter, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;

    // ---- last block: SumForcesULoading (md_results.cu:34-74) and CompressB/U
    __threadfence();
    double pb = 0.0, pt = 0.0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double2 v = __ldcg(&d.partial[b]);
        pb += v.x; pt += v.y;
    }
    for (int o = 16; o; o >>= 1) {
        pb += __shfl_xor_sync(FULL, pb, o);
        pt += __shfl_xor_sync(FULL, pt, o);
    }
    __syncthreads();
    if (l == 0) { s_b[w] = pb; s_t[w] = pt; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double sfb_all = (s_b[0] + s_b[1]) + (s_b[2] + s_b[3]);
    const double sft_all = (s_t[0] + s_t[1]) + (s_t[2] + s_t[3]);
    sc->block_counter = 0;
    // curve record and stress
    const double a1 = (double)sc->_1d_Area;
    if (sc->curve_n < c.curve_cap) {
        double* rec = d.curve + 3 * sc->curve_n;
        rec[0] = (sc->size_d[2] - sc->sz0) / sc->sz0;
        rec[1] = sfb_all * a1;
        rec[2] = sft_all * a1;
    }
    sc->curve_n += 1;
    sc->Stress = 0.5 * (fabs(sfb_all) + fabs(sft_all)) * a1;
    if (!sc->Loading && sc->Stress > sc->MinStress) sc->Loading = 1;
    if (sc->FractureStress < sc->Stress) {
        sc->FractureStress = sc->Stress;
        sc->FractureStrain = (sc->sz0 - sc->size_d[2]) / sc->sz0;
    }
    if (sc->Loading && sc->Stress < sc->ZeroStress) sc->Fracture = 1;
    // CompressU / CompressB (md_data_types.h:223-293)
    const int ax = (KIND == RF_TEST_BRAZIL) ? 1 : 2;
    sc->V = (sc->Stress < 1e-9) ? 10.0 * sc->VLoad : sc->VLoad;
    sc->size_d[ax] += sc->V * c.dt_d;
    sc->Top += sc->V * c.dt_d;
    sc->TopR = sc->Top - 2.0 * c.p_r_d;
    sc->size[ax] = (float)sc->size_d[ax];
    sc->sized2[ax] = (float)(0.5 * sc->size_d[ax]);
    sc->center_d[ax] += sc->V * c.dt_d;
    sc->center[ax] = (float)sc->center_d[ax];
    sc->Hd2 = sc->sized2[ax];
    sc->Strain = (sc->size_d[ax] - sc->Size0) / sc->Size0;
    sc->steps += 1;
    sc->dmax = sqrtf(__uint_as_float(sc->d2max_next));
    sc->d2max_next = 0;
    const bool running = (sc->Strain < sc->MaxStrain) && !sc->Fracture;
    sc->done = running ? 0u : 1u;
    const uint32_t mv = sc->moved;
    sc->moved = 0;
    sc->rebuild = mv;
    if (c.use_graph) {
        cudaGraphSetConditional(c.h_rebuild, mv ? 1u : 0u);
        cudaGraphSetConditional(c.h_loop, (running && sc->steps < sc->target) ? 1u : 0u);
    }
}

template <int KIND>
__global__ void __launch_bounds__(128, RF_STEP_MIN_BLOCKS) k_step(Dev d, Consts c) {
    DevScalars* sc = d.sc;
    // Loop safety: clear the WHILE condition first. Only the last block's finalize,
    // which runs after every block has passed this point and advances the step
    // counter towards the target, sets it again, so the device loop always ends.
    if (c.use_graph && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(c.h_loop, 0u);
    if (sc->done || sc->steps >= sc->target) return;
    const uint32_t cur = (uint32_t)(sc->steps & 1ull), nxt = cur ^ 1u;
    const float4* __restrict__ P = d.pos[cur];
    const float4* __restrict__ Vv = d.vel[cur];
    const float4* __restrict__ Wv = d.ang[cur];
    const uint32_t N = c.N;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < N;
    const uint32_t FULL = 0xffffffffu;

    // platen arguments of this step, as the driver passes them (double -> float)
    const float Top = (float)sc->Top, Bottom = (float)sc->Bottom, TopR = (float)sc->TopR,
                BottomR = (float)sc->BottomR, vt = (float)sc->V, RR = sc->RR;
    rf_float3 cc;
    cc.x = sc->center[0]; cc.y = sc->center[1]; cc.z = sc->center[2];

    f3 xi = mk3(0.f, 0.f, 0.f), vi = xi, wi = xi;
    uint32_t live = 0, bond = 0, cm = 0, nbq = 0, bmask = 0;
    unsigned long long mem = 0ull;
    uint32_t ncand = 0;
    if (valid) {
        xi = f4to3(P[i]); vi = f4to3(Vv[i]); wi = f4to3(Wv[i]);
        live = d.live[i]; bond = d.bond[i]; cm = d.cmask[i];
        mem = d.member[i]; ncand = d.cand_n[i];
        nbq = d.nbq[i]; bmask = d.bmask[i];
    }
    const uint32_t live0 = live, bond0 = bond, cm0 = cm, bmask0 = bmask;
    const unsigned long long mem0 = mem;
    const size_t QN = (size_t)d.QB * N;

    // ---- bonds: d_CalculateForcesDEM_22 (md_calculateforcesdem3.cu:424-483) over the bond
    // records in slot order, with the DeleteFarLinks test of each bond slot on the same
    // gathered position (md_interaction_list_reconstructbpm.cu:141-186). The next record
    // is fetched while the current one is computed.
    f3 fsb = mk3(0.f, 0.f, 0.f), msb = fsb;
    uint32_t nbroken = 0;
    {
        const uint32_t wb = __reduce_or_sync(FULL, bmask);
        const uint32_t qend = 32u - __clz(wb);
        uint32_t nj = i;
        float nil = 0.f;
        float4 n0 = make_float4(0.f, 0.f, 0.f, 0.f), n1 = n0, n2 = n0;
        if (qend > 0 && (bmask & 1u)) {
            const size_t s = (size_t)i;
            nj = __ldg(&d.bj[s]); nil = __ldg(&d.bil[s]);
            n0 = d.bst[s]; n1 = d.bst[s + QN]; n2 = d.bst[s + 2 * QN];
        }
        for (uint32_t q = 0; q < qend; ++q) {
            const uint32_t j = nj;
            const float il = nil;
            const float4 s0 = n0, s1 = n1, s2 = n2;
            const bool act = (bmask >> q) & 1u;
            if (q + 1 < qend && ((bmask >> (q + 1)) & 1u)) {
                const size_t s = (size_t)(q + 1) * N + i;
                nj = __ldg(&d.bj[s]); nil = __ldg(&d.bil[s]);
                n0 = d.bst[s]; n1 = d.bst[s + QN]; n2 = d.bst[s + 2 * QN];
            }
            if (!act) continue;
            const size_t s = (size_t)q * N + i;
            const float4 pj = __ldg(&P[j]), vj = __ldg(&Vv[j]), wj = __ldg(&Wv[j]);
            const f3 xj = f4to3(pj);
            const float rr = dist2_rn(xi, xj);
            if (rr > c.aa_farcut || (double)rr < 1e-10) {
                delete_slot(d, c, i, d.bk[s], j, ncand, nbq, live, bond, cm, bmask, mem);
                continue;
            }
            const f3 r = mk3(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z);
            f3 rij = mk3(s0.x, s0.y, s0.z), oijt = mk3(s0.w, s1.x, s1.y);
            f3 mijn = mk3(s1.z, s1.w, s2.x), mijt = mk3(s2.y, s2.z, s2.w);
            const bool broke = bond_slot(c.bp, r, vi, f4to3(vj), wi, f4to3(wj), il, rij, oijt, mijn, mijt, fsb, msb);
            d.bst[s] = make_float4(rij.x, rij.y, rij.z, oijt.x);
            d.bst[s + QN] = make_float4(oijt.y, oijt.z, mijn.x, mijn.y);
            d.bst[s + 2 * QN] = make_float4(mijn.z, mijt.x, mijt.y, mijt.z);
            if (broke) { bmask &= ~(1u << q); bond &= ~(1u << d.bk[s]); ++nbroken; }
        }
    }

    // ---- type-0 slots, one gather each: the rest of the previous step's DeleteFarLinks,
    // then d_CalculateForcesDEM_21 (md_calculateforcesdem3.cu:338-422) in slot order
    // (bonds broken above included). Overlaps are read from this step's buffer and
    // written to the next one, so the pass can be replayed below if a link added by
    // this step's list update turns out to be in contact.
    const uint32_t* row = d.ids + (size_t)i * c.K;
    const float* oin = d.cO[cur] + (size_t)i * c.K * 3;
    float* oout = d.cO[nxt] + (size_t)i * c.K * 3;
    const uint32_t cm_in = cm;
    const float twoR = 2.0f * c.cp.rP;
    f3 fsc = mk3(0.f, 0.f, 0.f), msc = fsc;
    uint32_t cm_out = 0;
    {
        uint32_t m = live & ~bond;
        while (m) {
            const uint32_t k = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t j = row[k];
            const f3 xj = f4to3(__ldg(&P[j]));
            const float rr = dist2_rn(xi, xj);
            if (rr > c.aa_farcut || (double)rr < 1e-10) {
                delete_slot(d, c, i, k, j, ncand, nbq, live, bond, cm, bmask, mem);
                continue;
            }
            const f3 r = mk3(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z);
            const float rijm = norm3(r.x, r.y, r.z);
            if (!(rijm < twoR)) continue;
            const uint32_t bit = 1u << k;
            f3 o = (cm_in & bit) ? mk3(oin[3 * k], oin[3 * k + 1], oin[3 * k + 2]) : mk3(0.f, 0.f, 0.f);
            contact_pair(c.cp, r, rijm, vi, f4to3(__ldg(&Vv[j])), wi, f4to3(__ldg(&Wv[j])), o, fsc, msc);
            oout[3 * k] = o.x; oout[3 * k + 1] = o.y; oout[3 * k + 2] = o.z;
            cm_out |= bit;
        }
    }

    // ---- add: InteractionListReConstructBPM (md_interaction_list_reconstructbpm.cu:13-46,80-139)
    // (skipped when no candidate can have come within a_farcut since the build: the scan
    // would add nothing)
    bool replay = false;
    if (valid && !scan_not_needed(d, c, i, xi.x, xi.y, xi.z)) {
        unsigned long long tried = mem;
        bool have_cells = false;
        Octant oc;
        for (;;) {
            unsigned long long best = ~0ull;
            uint32_t best_q = 0;
            for (uint32_t q = 0; q < ncand; ++q) {
                if ((tried >> q) & 1ull) continue;
                const uint32_t j = __ldg(&d.cand[(size_t)q * N + i]);
                const f3 xj = f4to3(__ldg(&P[j]));
                const float rr = dist2_rn(xi, xj);
                if (!(rr < c.aacut && (double)rr > 1e-10)) continue;
                if (!have_cells) { oc = octant_of(xi, c.g); have_cells = true; }
                const int rank = octant_rank(oc, ref_cell(xj, c.g));
                if (rank < 0) continue;
                const unsigned long long key = ((unsigned long long)rank << 32) | j;
                if (key < best) { best = key; best_q = q; }
            }
            if (best == ~0ull) break;
            tried |= 1ull << best_q;
            const uint32_t free = ~live & (c.K >= 32 ? 0xffffffffu : ((1u << c.K) - 1u));
            if (!free) { raise_status(&sc->err, RF_ERR_ROW_OVERFLOW); continue; }
            uint32_t k;
            if (i == 0 && (free & 1u) && (free & ~1u)) k = __ffs(free & ~1u) - 1;   // kdxfree==0 quirk
            else k = __ffs(free) - 1;
            const uint32_t j = (uint32_t)(best & 0xffffffffull);
            d.ids[(size_t)i * c.K + k] = j;
            live |= 1u << k;
            mem |= 1ull << best_q;
            const f3 xj = f4to3(__ldg(&P[j]));
            if (norm3(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z) < twoR) replay = true;
        }
    }
    // A new link already in contact: _21 would have visited it in slot order among the
    // others, so the contact pass is replayed over the final row from the unchanged
    // overlaps of this step.
    if (replay) {
        fsc = mk3(0.f, 0.f, 0.f); msc = fsc; cm_out = 0;
        uint32_t m = live & ~bond;
        while (m) {
            const uint32_t k = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t j = row[k];
            const f3 xj = f4to3(__ldg(&P[j]));
            const f3 r = mk3(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z);
            const float rijm = norm3(r.x, r.y, r.z);
            if (!(rijm < twoR)) continue;
            const uint32_t bit = 1u << k;
            f3 o = (cm & bit) ? mk3(oin[3 * k], oin[3 * k + 1], oin[3 * k + 2]) : mk3(0.f, 0.f, 0.f);
            contact_pair(c.cp, r, rijm, vi, f4to3(__ldg(&Vv[j])), wi, f4to3(__ldg(&Wv[j])), o, fsc, msc);
            oout[3 * k] = o.x; oout[3 * k + 1] = o.y; oout[3 * k + 2] = o.z;
            cm_out |= bit;
        }
    }
    cm = cm_out;

    float e2max = 0.f;
    double sfb = 0.0, sft = 0.0;
    uint32_t moved = 0;
    if (valid) {
        if (live != live0) d.live[i] = live;
        if (bond != bond0) d.bond[i] = bond;
        if (cm != cm0) d.cmask[i] = cm;
        if (mem != mem0) d.member[i] = mem;
        if (bmask != bmask0) d.bmask[i] = bmask;
        // F = 0 after the memset, then += _22 sums, then += _21 sums
        float Fx = 0.0f + fsb.x, Fy = 0.0f + fsb.y, Fz = 0.0f + fsb.z;
        Fx += fsc.x; Fy += fsc.y; Fz += fsc.z;
        float Mx = 0.0f + msb.x, My = 0.0f + msb.y, Mz = 0.0f + msb.z;
        Mx += msc.x; My += msc.y; Mz += msc.z;
        float Rx = xi.x, Ry = xi.y, Rz = xi.z, Vx = vi.x, Vy = vi.y, Vz = vi.z;
        if (KIND == RF_TEST_BRAZIL)
            brazil_particle(Rx, Ry, Rz, Vx, Vy, Vz, Fx, Fy, Fz, cc, RR, Top, Bottom, TopR, BottomR, vt, c.zcut, sfb, sft);
        else
            uniaxial_particle(Rx, Ry, Rz, Vz, Fz, cc, RR, Top, Bottom, TopR, BottomR, vt, c.zcut, sfb, sft);
        // d_CalculateIncrementsDEM (md_calculateincrementsdem.cu:19-49)
        Vx += __fmul_rn(Fx, c.dtm); Vy += __fmul_rn(Fy, c.dtm); Vz += __fmul_rn(Fz, c.dtm);
        Rx += __fmul_rn(Vx, c.dt); Ry += __fmul_rn(Vy, c.dt); Rz += __fmul_rn(Vz, c.dt);
        float Wx = wi.x + __fmul_rn(Mx, c.dtI), Wy = wi.y + __fmul_rn(My, c.dtI), Wz = wi.z + __fmul_rn(Mz, c.dtI);
        // d_ParallelepipedCutRestriction (md_parallelepipedrestriction.cu:73-159)
        if (outside_box(Rx, Ry, Rz, c.box_c, c.box_h)) {
            Rx = c.hp.x; Ry = c.hp.y; Rz = c.hp.z;
            Vx = 0.f; Vy = 0.f; Vz = 0.f;
        }
        d.pos[nxt][i] = make_float4(Rx, Ry, Rz, 0.f);
        d.vel[nxt][i] = make_float4(Vx, Vy, Vz, 0.f);
        d.ang[nxt][i] = make_float4(Wx, Wy, Wz, 0.f);
        const float4 pr = d.pos_ref[i];
        const float ex = Rx - pr.x, ey = Ry - pr.y, ez = Rz - pr.z;
        const float e2 = ex * ex + ey * ey + ez * ez;
        moved = (e2 > c.disp2) ? 1u : 0u;
        // lists may have missed a neighbour (a particle moved to the hidden point has none)
        const bool hidden = Rx == c.hp.x && Ry == c.hp.y && Rz == c.hp.z;
        if (e2 > c.hard2 && !hidden) raise_status(&d.sc->err, RF_ERR_CAPACITY);
        if (!hidden) e2max = e2;
    }
    note_displacement(d, e2max);
    step_finish<KIND>(d, c, sfb, sft, nbroken, moved);
}

// ===========================================================================
// Extended model step: FP64 positions (x, y, z, radius), per-particle mass and
// inertia from the radius, bond records with an FP64 rest length and their own
// strengths, contacts with equivalent radius and mass. Same structure and order as
// k_step; list maintenance compares FP64 squared distances.
// ===========================================================================
// Read-only load of a 32-byte particle record (two 16-byte loads of one sector pair).
__device__ __forceinline__ double4 ldg_d4(const double4* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
// A read of three floats that the compiler may not merge with an earlier read of the same
// address: the value is fetched again (an L1 hit) instead of being held in registers.
__device__ __forceinline__ f3 reload3(const float4* p) {
    float x, y, z, w;
    asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(x), "=f"(y), "=f"(z), "=f"(w) : "l"(p));
    (void)w;
    return mk3(x, y, z);
}
__device__ __forceinline__ double3 dsub(const double4 a, const double4 b) {
    return make_double3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ double dlen2(const double3 r) { return r.x * r.x + r.y * r.y + r.z * r.z; }

// Squared list cutoffs of a pair of the extended model (radii ri, rj): the add test and
// the delete test. With a list gap g the pair's cutoff is min(a_farcut, ri + rj + g).
__device__ __forceinline__ double cut2_add(const Consts& c, double ri, double rj) {
    if (c.lgap_d > 0.0) {
        const double q = fmin(c.a_farcut_d, (ri + rj) + c.lgap_d);
        return q * q;
    }
    return c.aacut_d;
}
__device__ __forceinline__ double cut2_del(const Consts& c, double ri, double rj) {
    if (c.lgap_d > 0.0) {
        const double q = fmin(c.a_farcut_d, (ri + rj) + c.lgap_d);
        return q * q;
    }
    return c.aa_farcut_d;
}

// The reference removes a listed pair beyond a_farcut = 2.9 p_r, 1.45 times the contact
// distance 2 p_r of its mono-sized particles, intact bonds included
// (md_interaction_list_reconstructbpm.cu:141-186). With a list gap, or radii that span a
// range, a pair cutoff can lie within a bond's failure stretch (a bond of two r_max
// particles sits just inside a_farcut = 2.02 r_max), so list maintenance would remove
// intact bonds that their strengths still hold. In the extended model an intact bond is
// therefore removed by distance only beyond the same relative margin of its own rest
// length, |r| > 1.45 L0; the reference-constants mode keeps the reference's rule.
#define RF_BOND_KEEP_RATIO 1.45
__device__ __forceinline__ double bond_cut2_del(const Consts& c, double ri, double rj, double L0) {
    if (c.ref_mode) return cut2_del(c, ri, rj);
    const double q = RF_BOND_KEEP_RATIO * L0;
    return q * q;
}
// Rest length of the intact bond in slot k of particle i (its record's).
__device__ __forceinline__ double slot_rest_length(const Dev& d, const Consts& c, uint32_t i, uint32_t k, uint32_t nbq) {
    for (uint32_t q = 0; q < nbq; ++q) {
        const size_t s = (size_t)q * c.N + i;
        if (d.bk[s] == (uint8_t)k) return d.bL0[s];
    }
    return 0.0;
}

__device__ __forceinline__ void delete_far_ext(const Dev& d, const Consts& c, const double4* __restrict__ P,
                                               uint32_t i, const double4 xi, uint32_t ncand, uint32_t nbq,
                                               uint32_t& live, uint32_t& bond, uint32_t& cm, uint32_t& bmask,
                                               unsigned long long& mem) {
    const uint32_t* row = d.ids + (size_t)i * c.K;
    uint32_t m = live;
    while (m) {
        const uint32_t k = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t j = row[k];
        const double4 xj = ldg_d4(&P[j]);
        const double rr = dlen2(dsub(xj, xi));
        const double cut = ((bond >> k) & 1u) ? bond_cut2_del(c, xi.w, xj.w, slot_rest_length(d, c, i, k, nbq))
                                              : cut2_del(c, xi.w, xj.w);
        if (rr > cut || rr < 1e-10)
            delete_slot(d, c, i, k, j, ncand, nbq, live, bond, cm, bmask, mem);
    }
}

__global__ void k_delete_pending_ext(Dev d, Consts c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const double4* P = d.posd[d.sc->steps & 1ull];
    uint32_t live = d.live[i], bond = d.bond[i], cm = d.cmask[i], ncand = d.cand_n[i], nbq = d.nbq[i],
             bmask = d.bmask[i];
    unsigned long long mem = d.member[i];
    const uint32_t live0 = live;
    delete_far_ext(d, c, P, i, P[i], ncand, nbq, live, bond, cm, bmask, mem);
    if (live != live0) {
        d.live[i] = live; d.bond[i] = bond; d.cmask[i] = cm; d.member[i] = mem; d.bmask[i] = bmask;
    }
}

// Platen contact and clamp with FP64 positions (d_UniaxialCompression3_simple /
// d_braziltest_simple2 with the coordinates kept in double). The platens act on the
// particle surfaces: the coordinate tested and clamped along the load axis is the
// centre plus (radius - p_r) towards the top platen and minus it towards the bottom
// one, so a polydisperse specimen meets a flat platen with every particle that
// touches it; for radius p_r this is the reference's centre rule.
// hold: inside a quasi-static increment's FIRE iterations a particle held by a platen
// does not slide along it either (removes the specimen's rigid tilting and sliding).
__device__ __forceinline__ void uniaxial_particle_ext(double& Rx, double& Ry, double& Rz, float& Vx, float& Vy,
                                                      float& Vz, float& Fx, float& Fy, float& Fz, const rf_float3 c,
                                                      float RR, double Zt, double Zb, double Ztr, double Zbr, float vt,
                                                      double Zcut, double off, double& sfb, double& sft, bool hold) {
    const float rx = (float)(Rx - c.x), ry = (float)(Ry - c.y);
    const double rz = Rz;
    if (rx * rx + ry * ry < RR && rz < Zcut) {
        if (rz + off - Ztr > -1e-9) {
            if (Fz > 0) sft += (double)Fz;
            if (rz + off - Zt > -1e-9) {
                Rz = Zt - off; Vz = vt; Fz = 0.f;
                if (hold) { Fx = 0.f; Fy = 0.f; Vx = 0.f; Vy = 0.f; }
            }
        }
        if (rz - off - Zbr < 1e-9) {
            if (Fz < 0) sfb += (double)Fz;
            if (rz - off - Zb < 1e-9) {
                Rz = Zb + off; Vz = 0.f; Fz = 0.f;
                if (hold) { Fx = 0.f; Fy = 0.f; Vx = 0.f; Vy = 0.f; }
            }
        }
    }
}
__device__ __forceinline__ void brazil_particle_ext(double& Rx, double& Ry, double& Rz, float& Vx, float& Vy,
                                                    float& Vz, float& Fx, float& Fy, float& Fz, const rf_float3 c,
                                                    float RR, double Yt, double Yb, double Ytr, double Ybr, float vt,
                                                    double Zcut, double off, double& sfb, double& sft, bool hold) {
    const float rx = (float)(Rx - c.x), rz = (float)(Rz - c.z);
    const double ry = Ry;
    if (rx * rx + rz * rz < RR && (double)rz < Zcut) {
        if (ry + off - Ytr > -1e-9) {
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
            if (ry + off - Yt > -1e-9) {
                Ry = Yt - off; Vy = vt; Fy = 0.f;
                if (hold) { Fx = 0.f; Fz = 0.f; Vx = 0.f; Vz = 0.f; }
            }
        }
        if (ry - off - Ybr < 1e-9) {
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
            if (ry - off - Yb < 1e-9) {
                Ry = Yb + off; Vy = 0.f; Fy = 0.f;
                if (hold) { Fx = 0.f; Fz = 0.f; Vx = 0.f; Vz = 0.f; }
            }
        }
    }
}

// End of an extended-model step for a batch of specimens. The platen reaction sums of a
// CTA are kept per specimen (its first and, if it touches one, its second); the last CTA
// adds each specimen's CTA partials in CTA order and runs SumForcesULoading
// (md_results.cu:34-74), the fracture test and CompressB/U (md_data_types.h:223-293)
// for every specimen still running; the loop ends when all are done. With one specimen
// this is step_finish's arithmetic, sum for sum.
template <int KIND>
__device__ __forceinline__ void step_finish_ext(const Dev& d, const Consts& c, double sfb, double sft,
                                                uint32_t nbroken, uint32_t moved, uint32_t second) {
    DevScalars* sc = d.sc;
    const uint32_t FULL = 0xffffffffu;
    __shared__ double s_b[4], s_t[4], s_b2[4], s_t2[4];
    __shared__ uint32_t s_n[4], s_m[4];
    __shared__ bool s_last;
    double b1 = second ? sfb : 0.0, t1 = second ? sft : 0.0;
    if (second) { sfb = 0.0; sft = 0.0; }
    for (int o = 16; o; o >>= 1) {
        sfb += __shfl_xor_sync(FULL, sfb, o);
        sft += __shfl_xor_sync(FULL, sft, o);
        b1 += __shfl_xor_sync(FULL, b1, o);
        t1 += __shfl_xor_sync(FULL, t1, o);
    }
    const uint32_t wn = __reduce_add_sync(FULL, nbroken), wm = __reduce_or_sync(FULL, moved);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { s_b[w] = sfb; s_t[w] = sft; s_b2[w] = b1; s_t2[w] = t1; s_n[w] = wn; s_m[w] = wm; }
    __syncthreads();
    if (threadIdx.x == 0) {
        d.partial[blockIdx.x] = make_double2((s_b[0] + s_b[1]) + (s_b[2] + s_b[3]), (s_t[0] + s_t[1]) + (s_t[2] + s_t[3]));
        d.partial2[blockIdx.x] =
            make_double2((s_b2[0] + s_b2[1]) + (s_b2[2] + s_b2[3]), (s_t2[0] + s_t2[1]) + (s_t2[2] + s_t2[3]));
        const uint32_t nb = s_n[0] + s_n[1] + s_n[2] + s_n[3];
        if (nb) atomicAdd(&sc->broken, (unsigned long long)nb);
        if (s_m[0] | s_m[1] | s_m[2] | s_m[3]) atomicOr(&sc->moved, 1u);
        __threadfence();
        const uint32_t ticket = atomicAdd(&sc->block_counter, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    bool all_done = true;
    for (uint32_t s = 0; s < d.nspec; ++s) {
        DevScalars* S = d.spec + s;
        const SpecGeom& G = d.geom[s];
        if (S->done) continue;                               // uniform across the CTA
        double pb = 0.0, pt = 0.0;
        for (uint32_t b = G.b0 + threadIdx.x; b <= G.b1; b += blockDim.x) {
            const double2 v = (d.blk_spec == nullptr || d.blk_spec[b] == s) ? __ldcg(&d.partial[b])
                                                                             : __ldcg(&d.partial2[b]);
            pb += v.x; pt += v.y;
        }
        for (int o = 16; o; o >>= 1) {
            pb += __shfl_xor_sync(FULL, pb, o);
            pt += __shfl_xor_sync(FULL, pt, o);
        }
        __syncthreads();
        if (l == 0) { s_b[w] = pb; s_t[w] = pt; }
        __syncthreads();
        if (threadIdx.x == 0) {
            const double sfb_all = (s_b[0] + s_b[1]) + (s_b[2] + s_b[3]);
            const double sft_all = (s_t[0] + s_t[1]) + (s_t[2] + s_t[3]);
            const double a1 = (double)S->_1d_Area;
            if (S->curve_n < c.curve_cap) {
                double* rec = d.curve + 3 * ((size_t)s * c.curve_cap + S->curve_n);
                rec[0] = (S->size_d[2] - S->sz0) / S->sz0;
                rec[1] = sfb_all * a1;
                rec[2] = sft_all * a1;
            }
            S->curve_n += 1;
            S->Stress = 0.5 * (fabs(sfb_all) + fabs(sft_all)) * a1;
            if (!S->Loading && S->Stress > S->MinStress) S->Loading = 1;
            if (S->FractureStress < S->Stress) {
                S->FractureStress = S->Stress;
                S->FractureStrain = (S->sz0 - S->size_d[2]) / S->sz0;
            }
            if (S->Loading && S->Stress < S->ZeroStress) S->Fracture = 1;
            if (S->Loading && S->Stress < S->keep_frac * S->FractureStress) S->Fracture = 1;
            const int ax = (KIND == RF_TEST_BRAZIL) ? 1 : 2;
            S->V = (S->Stress < 1e-9) ? 10.0 * S->VLoad : S->VLoad;
            S->size_d[ax] += S->V * c.dt_d;
            S->Top += S->V * c.dt_d;
            S->TopR = S->Top - 2.0 * c.p_r_d;
            S->size[ax] = (float)S->size_d[ax];
            S->sized2[ax] = (float)(0.5 * S->size_d[ax]);
            S->center_d[ax] += S->V * c.dt_d;
            S->center[ax] = (float)S->center_d[ax];
            S->Hd2 = S->sized2[ax];
            S->Strain = (S->size_d[ax] - S->Size0) / S->Size0;
            S->steps += 1;                                    // the specimen's own step count
            const bool running = (S->Strain < S->MaxStrain) && !S->Fracture;
            S->done = running ? 0u : 1u;
        }
        __syncthreads();
        if (!S->done) all_done = false;
    }
    if (threadIdx.x != 0) return;
    sc->block_counter = 0;
    if (d.nspec > 1) sc->steps += 1;                          // (with one specimen sc == spec)
    sc->dmax = sqrtf(__uint_as_float(sc->d2max_next));
    sc->d2max_next = 0;
    sc->done = all_done ? 1u : 0u;
    const uint32_t mv = sc->moved;
    sc->moved = 0;
    sc->rebuild = mv;
    if (c.use_graph) {
        cudaGraphSetConditional(c.h_rebuild, mv ? 1u : 0u);
        cudaGraphSetConditional(c.h_loop, (!all_done && sc->steps < sc->target) ? 1u : 0u);
    }
}

#define FIRE_SUMS 9     // F.v + M.w, |F|^2, |v|^2, |M|^2, |w|^2, sum |f_n|, pair count, platen sums (2)

template <int KIND>
__device__ __forceinline__ void fire_force_finish(const Dev& d, const Consts& c, double (&acc)[FIRE_SUMS],
                                                  uint32_t second);

// MODE 0: explicit step (Verlet increments, platen moving at V). MODE 1: force evaluation
// of one FIRE iteration: the same forces with the FIRE time step, platens at rest; net
// force and moment are stored for k_fire_update and FP64 sums of the FIRE power, the
// squared norms and the mean normal pair force are reduced for the FIRE decision.
// MINB: resident 128-thread CTAs per SM the kernel is compiled for (the register cap);
// rf_engine_autotune picks among the compiled variants by timing them.
template <int KIND, int MODE, int MINB = RF_STEP_MIN_BLOCKS>
__global__ void __launch_bounds__(128, MINB) k_step_ext(Dev d, Consts c) {
    DevScalars* sc = d.sc;
    if (c.use_graph && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(c.h_loop, 0u);
    if (MODE == 0 && (sc->done || sc->steps >= sc->target)) return;
    if (MODE == 1 && sc->fstop) return;
    const uint32_t cur = (uint32_t)(sc->steps & 1ull), nxt = cur ^ 1u;
    const double4* __restrict__ P = d.posd[cur];
    const float4* __restrict__ Vv = d.vel[cur];
    const float4* __restrict__ Wv = d.ang[cur];
    const uint32_t N = c.N;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // specimen of this particle: the CTA's first one, or the next (each specimen has at
    // least 128 particles, so a CTA touches at most two)
    const uint32_t sA = d.blk_spec ? (uint32_t)d.blk_spec[blockIdx.x] : 0u;
    const uint32_t sI = (i < N && i >= d.geom[sA].p1) ? sA + 1u : sA;
    const SpecGeom& G = d.geom[sI];
    const DevScalars* S = d.spec + sI;
    // a finished specimen of a batch is frozen: its state is carried to the next buffer
    // (explicit steps: it reached its stop rule; FIRE: its relaxation of this increment stopped)
    const bool frozen = i < N && (MODE == 0 ? S->done != 0 : S->fstop != 0);
    const bool valid = i < N && !frozen;
    const uint32_t FULL = 0xffffffffu;
    if (frozen) {
        d.posd[nxt][i] = P[i];
        d.vel[nxt][i] = Vv[i];
        d.ang[nxt][i] = Wv[i];
        const float* oi = d.cO[cur] + (size_t)i * c.K * 3;
        float* oo = d.cO[nxt] + (size_t)i * c.K * 3;
        uint32_t m = d.cmask[i];
        while (m) {
            const uint32_t k = __ffs(m) - 1;
            m &= m - 1;
            oo[3 * k] = oi[3 * k]; oo[3 * k + 1] = oi[3 * k + 1]; oo[3 * k + 2] = oi[3 * k + 2];
        }
    }
    ExtParams ep = c.ep;
    if (MODE == 1) {
        // FIRE minimises the conservative part of the model: its own velocity mixing
        // and restarts replace the viscous contact damping, and the constant-torque
        // rolling resistance (a set-valued term at rest) is left out.
        ep.dt = (float)S->fdt;
        ep.p_A = 0.f;
        ep.mur = 0.f;
    }
    float fnabs = 0.f, kt = 0.f, kr = 0.f;
    uint32_t npair = 0;

    uint32_t live = 0, bond = 0, cm = 0, nbq = 0, bmask = 0, ncand = 0;
    unsigned long long mem = 0ull;
    if (valid) {
        live = d.live[i]; bond = d.bond[i]; cm = d.cmask[i];
        mem = d.member[i]; ncand = d.cand_n[i];
        nbq = d.nbq[i]; bmask = d.bmask[i];
    }
    const size_t QN = (size_t)d.QB * N;

    bool dirty = false;          // live, bond, bmask or member changed
    // bond slots whose pair overlaps: their contact (in parallel with the bond) was taken
    // in the bond pass, with its tangential overlap kept in the slot's contact state
    uint32_t pc = 0;
    const uint32_t cm0 = cm;
    constexpr int NA = MODE == 1 ? 9 : 6;         // the particle's bond sums (float)
    __shared__ float s_acc[4][NA][32];
    __shared__ uint32_t s_msk[4][10][32];
    enum { W_LIVE, W_BOND, W_CM, W_BMASK, W_PC, W_NB, W_MEMLO, W_MEMHI, W_NPAIR, W_DIRTY };
    {
        // Bond records, spread over the warp. The warp's active records are listed
        // ordinal-major (every particle's first record, then every second one, ...; lane
        // order within an ordinal), so consecutive lanes read consecutive entries of the
        // [QB][N] record arrays, and in each round every lane takes one record whatever the
        // 32 particles' bond counts. The lane that takes a record forms its force, moment
        // and outcome from zero and hands them to the particle's lane through shared
        // memory; the particle adds them in record order. While the pass runs, each
        // particle's sums and masks wait in shared memory, leaving the registers to the
        // record arithmetic. FIRE mode reads the records' increment-start state and the
        // motion since then.
        constexpr int NO = MODE == 1 ? 10 : 7;        // words of one record's result
        __shared__ float s_res[4][NO][32];
        __shared__ uint32_t s_q0[4][32], s_qb[4][32];  // per ordinal: first list entry, lanes holding one
        extern __shared__ __align__(16) unsigned char rf_step_smem[];
        const uint32_t lane = threadIdx.x & 31u, wp = threadIdx.x >> 5;
        const uint32_t lt = (1u << lane) - 1u;
        const uint32_t wbase = i - lane;
        uint16_t* lst = reinterpret_cast<uint16_t*>(rf_step_smem) + (size_t)wp * 32u * d.QB;
        const uint32_t qend = 32u - __clz(__reduce_or_sync(FULL, bmask));
        uint32_t T = 0;
        for (uint32_t q = 0; q < qend; ++q) {
            const bool has = (bmask >> q) & 1u;
            const uint32_t bal = __ballot_sync(FULL, has);
            if (has) lst[T + __popc(bal & lt)] = (uint16_t)(lane | (q << 5));
            if (lane == q) { s_q0[wp][q] = T; s_qb[wp][q] = bal; }
            T += __popc(bal);
        }
        uint32_t rem = bmask;                          // this particle's records not yet added
#pragma unroll
        for (int a = 0; a < NA; ++a) s_acc[wp][a][lane] = 0.f;   // (read back after the contact pass)
        s_msk[wp][W_NB][lane] = 0u;
        s_msk[wp][W_NPAIR][lane] = 0u;
        if (T) {
            s_msk[wp][W_LIVE][lane] = live; s_msk[wp][W_BOND][lane] = bond; s_msk[wp][W_CM][lane] = cm;
            s_msk[wp][W_BMASK][lane] = bmask; s_msk[wp][W_PC][lane] = 0u;
            s_msk[wp][W_MEMLO][lane] = (uint32_t)mem; s_msk[wp][W_MEMHI][lane] = (uint32_t)(mem >> 32);
            s_msk[wp][W_DIRTY][lane] = 0u;
        }
        __syncwarp();
        const float4* src = MODE == 1 ? d.bst0 : d.bst;
        for (uint32_t base = 0; base < T; base += 32u) {
            const uint32_t p = base + lane;
            if (p < T) {
                const uint32_t e = lst[p];
                const uint32_t ol = e & 31u, q = e >> 5, io = wbase + ol;
                const size_t s = (size_t)q * N + io;
                // every load of the record is issued before the partner's gathers
                const uint32_t j = __ldg(&d.bj[s]);
                const float4 s0 = src[s], s1 = src[s + QN], s2 = src[s + 2 * QN];
                const float2 str = __ldg(&d.bstr[s]);
                const double L0 = __ldg(&d.bL0[s]);
                const uint32_t k = d.bk[s];
                const double4 xo = ldg_d4(&P[io]);
                const double4 xj = ldg_d4(&P[j]);
                const float4 vj = __ldg(&Vv[j]), wj = __ldg(&Wv[j]);
                const double3 rd = dsub(xj, xo);
                const double rr = dlen2(rd);
                uint32_t fl = k << 8;
                f3 fr = mk3(0.f, 0.f, 0.f), mr = fr;
                float fnr = 0.f, ktr = 0.f, krr = 0.f;
                if (rr > bond_cut2_del(c, xo.w, xj.w, L0) || rr < 1e-10) {
                    fl |= RF_REC_DELETE;
                    fr.x = __uint_as_float(j);
                } else {
                    const float ro = (float)xo.w, rj = (float)xj.w;
                    // parallel contact (extended model, explicit steps): an overlapping bonded pair
                    // also carries the Hertz-Mindlin contact, and a broken bond's slot keeps that
                    // contact's state. Its overlap counts from min(r_i + r_j, L0), so a bond formed
                    // between overlapping particles is force-free at its rest length. FIRE
                    // relaxation leaves it out: its state would depend on the path.
                    const double sr = fmin(xo.w + xj.w, L0);
                    const bool pcon = MODE == 0 && !c.ref_mode && rr < sr * sr;
                    BondExt b;
                    b.kn = c.kn; b.ks = c.ks; b.br = c.br_lambda * fminf(ro, rj);
                    b.sc = str.x; b.tc = str.y; b.L0 = L0;
                    if (MODE == 0 && c.ref_mode) {
                        const float il = __ldg(&d.bil[s]);
                        b.kn = c.refE * il; b.ks = c.refG * il; b.br = c.ref_br;
                    }
                    const f3 r = mk3((float)rd.x, (float)rd.y, (float)rd.z);
                    f3 rij = mk3(s0.x, s0.y, s0.z), oijt = mk3(s0.w, s1.x, s1.y);
                    f3 mijn = mk3(s1.z, s1.w, s2.x), mijt = mk3(s2.y, s2.z, s2.w);
                    bool broke;
                    if (MODE == 1) {
                        const double4 xi0 = ldg_d4(&d.x0[io]), ri0 = ldg_d4(&d.rot[io]);
                        const double4 xj0 = ldg_d4(&d.x0[j]), rj0 = ldg_d4(&d.rot[j]);
                        const double hx = 0.5 * (ri0.x + rj0.x), hy = 0.5 * (ri0.y + rj0.y), hz = 0.5 * (ri0.z + rj0.z);
                        const f3 du = mk3((float)(rd.x - (xj0.x - xi0.x) - (hy * rd.z - hz * rd.y)),
                                          (float)(rd.y - (xj0.y - xi0.y) - (hz * rd.x - hx * rd.z)),
                                          (float)(rd.z - (xj0.z - xi0.z) - (hx * rd.y - hy * rd.x)));
                        broke = bond_slot_ext_total(b, r, rr, du, mk3((float)ri0.x, (float)ri0.y, (float)ri0.z),
                                                    mk3((float)rj0.x, (float)rj0.y, (float)rj0.z), rij, oijt, mijn,
                                                    mijt, rij, oijt, mijn, mijt, fr, mr, fnr, ktr, krr);
                    } else {
                        broke = bond_slot_ext(ep, b, r, rr, f4to3(__ldg(&Vv[io])), f4to3(vj), f4to3(__ldg(&Wv[io])),
                                              f4to3(wj), rij, oijt, mijn, mijt, fr, mr, fnr, ktr, krr, c.ref_mode != 0);
                    }
                    d.bst[s] = make_float4(rij.x, rij.y, rij.z, oijt.x);
                    d.bst[s + QN] = make_float4(oijt.y, oijt.z, mijn.x, mijn.y);
                    d.bst[s + 2 * QN] = make_float4(mijn.z, mijt.x, mijt.y, mijt.z);
                    if (broke) fl |= RF_REC_BROKE;
                    if (pcon) {
                        // the pair's velocities and spins are read again (cache hits) rather
                        // than held through the bond arithmetic
                        const size_t so = ((size_t)io * c.K + k) * 3;
                        const float* oi = d.cO[cur] + so;
                        // the particle's contacts at the step's start (its own record's
                        // bit is only cleared after this record is added)
                        const uint32_t cmo = s_msk[wp][W_CM][ol];
                        f3 o = ((cmo >> k) & 1u) ? mk3(oi[0], oi[1], oi[2]) : mk3(0.f, 0.f, 0.f);
                        if (contact_pair_ext(ep, r, rr, sr, ro, rj, c.cmass * ro * ro * ro, c.cmass * rj * rj * rj,
                                             reload3(&Vv[io]), reload3(&Vv[j]), reload3(&Wv[io]), reload3(&Wv[j]), o,
                                             fr, mr, fnr, ktr, krr))
                            fl |= RF_REC_CLEAR;
                        float* oo = d.cO[nxt] + so;
                        oo[0] = o.x; oo[1] = o.y; oo[2] = o.z;
                        fl |= RF_REC_PARALLEL;
                    }
                }
                s_res[wp][0][lane] = fr.x; s_res[wp][1][lane] = fr.y; s_res[wp][2][lane] = fr.z;
                s_res[wp][3][lane] = mr.x; s_res[wp][4][lane] = mr.y; s_res[wp][5][lane] = mr.z;
                s_res[wp][6][lane] = __uint_as_float(fl);
                if (MODE == 1) { s_res[wp][7][lane] = fnr; s_res[wp][8][lane] = ktr; s_res[wp][9][lane] = krr; }
            }
            __syncwarp();
            // this particle's records that fell in this round, in record order
            while (rem) {
                const uint32_t q = __ffs(rem) - 1u;
                const uint32_t x = s_q0[wp][q] + __popc(s_qb[wp][q] & lt) - base;
                if (x >= 32u) break;
                rem &= rem - 1u;
                const uint32_t fl = __float_as_uint(s_res[wp][6][x]);
                const uint32_t k = (fl >> 8) & 31u;
                if (fl & RF_REC_DELETE) {
                    uint32_t lv = s_msk[wp][W_LIVE][lane], bd = s_msk[wp][W_BOND][lane];
                    uint32_t cmm = s_msk[wp][W_CM][lane], bm = s_msk[wp][W_BMASK][lane];
                    unsigned long long mm = (unsigned long long)s_msk[wp][W_MEMLO][lane] |
                                            ((unsigned long long)s_msk[wp][W_MEMHI][lane] << 32);
                    delete_slot(d, c, i, k, __float_as_uint(s_res[wp][0][x]), d.cand_n[i], d.nbq[i], lv, bd, cmm, bm,
                                mm);
                    s_msk[wp][W_LIVE][lane] = lv; s_msk[wp][W_BOND][lane] = bd;
                    s_msk[wp][W_CM][lane] = cmm; s_msk[wp][W_BMASK][lane] = bm;
                    s_msk[wp][W_MEMLO][lane] = (uint32_t)mm; s_msk[wp][W_MEMHI][lane] = (uint32_t)(mm >> 32);
                    s_msk[wp][W_DIRTY][lane] = 1u;
                    continue;
                }
                s_acc[wp][0][lane] += s_res[wp][0][x];
                s_acc[wp][1][lane] += s_res[wp][1][x];
                s_acc[wp][2][lane] += s_res[wp][2][x];
                if (fl & RF_REC_CLEAR) {       // the contact's zero-spin rule clears the moment sum
                    s_acc[wp][3][lane] = 0.f; s_acc[wp][4][lane] = 0.f; s_acc[wp][5][lane] = 0.f;
                } else {
                    s_acc[wp][3][lane] += s_res[wp][3][x];
                    s_acc[wp][4][lane] += s_res[wp][4][x];
                    s_acc[wp][5][lane] += s_res[wp][5][x];
                }
                if (MODE == 1) {
                    s_acc[wp][6][lane] += s_res[wp][7][x];
                    s_acc[wp][7][lane] += s_res[wp][8][x];
                    s_acc[wp][8][lane] += s_res[wp][9][x];
                }
                uint32_t np = 1;
                if (fl & RF_REC_BROKE) {
                    s_msk[wp][W_BMASK][lane] &= ~(1u << q);
                    s_msk[wp][W_BOND][lane] &= ~(1u << k);
                    s_msk[wp][W_NB][lane] += 1u;
                    s_msk[wp][W_DIRTY][lane] = 1u;
                }
                if (fl & RF_REC_PARALLEL) { s_msk[wp][W_PC][lane] |= 1u << k; ++np; }
                else s_msk[wp][W_CM][lane] &= ~(1u << k);    // not in contact: the parallel contact's state ends
                if (MODE == 1) s_msk[wp][W_NPAIR][lane] += np;
            }
            __syncwarp();
        }
        if (T) {
            live = s_msk[wp][W_LIVE][lane]; bond = s_msk[wp][W_BOND][lane]; cm = s_msk[wp][W_CM][lane];
            bmask = s_msk[wp][W_BMASK][lane]; pc = s_msk[wp][W_PC][lane];
            mem = (unsigned long long)s_msk[wp][W_MEMLO][lane] | ((unsigned long long)s_msk[wp][W_MEMHI][lane] << 32);
            dirty = s_msk[wp][W_DIRTY][lane] != 0u;
        }
    }

    // the particle's own position (the bond pass read it through the cache; its velocity
    // and spin are read where they are used)
    double4 xi = make_double4(0, 0, 0, 1);
    if (valid) xi = P[i];
    const float ri = (float)xi.w;
    const float mi = c.cmass * ri * ri * ri;
    const uint32_t* row = d.ids + (size_t)i * c.K;
    const float* oin = d.cO[cur] + (size_t)i * c.K * 3;
    float* oout = d.cO[nxt] + (size_t)i * c.K * 3;

    f3 fsc = mk3(0.f, 0.f, 0.f), msc = fsc;
    uint32_t cm_out = 0;
    float fnc = 0.f, ktc = 0.f, krc = 0.f;   // contact force magnitudes and stiffness (recounted on a replay)
    uint32_t npc = 0;
    auto contact_pass = [&](bool with_delete) {
        uint32_t m = live & ~bond & ~pc;
        while (m) {
            const uint32_t k = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t j = row[k];
            const double4 xj = ldg_d4(&P[j]);
            const double3 rd = dsub(xj, xi);
            const double rr = dlen2(rd);
            if (with_delete && (rr > cut2_del(c, xi.w, xj.w) || rr < 1e-10)) {
                delete_slot(d, c, i, k, j, ncand, nbq, live, bond, cm, bmask, mem);
                dirty = true;
                continue;
            }
            const float rj = (float)xj.w;
            const double sr = xi.w + xj.w;
            if (!(rr < sr * sr)) continue;
            const uint32_t bit = 1u << k;
            // cm: step-start contacts minus slots deleted this step (a refilled slot starts at zero)
            f3 o = (cm & bit) ? mk3(oin[3 * k], oin[3 * k + 1], oin[3 * k + 2]) : mk3(0.f, 0.f, 0.f);
            const f3 r = mk3((float)rd.x, (float)rd.y, (float)rd.z);
            contact_pair_ext(ep, r, rr, sr, ri, rj, mi, c.cmass * rj * rj * rj, f4to3(__ldg(&Vv[i])),
                             f4to3(__ldg(&Vv[j])), f4to3(__ldg(&Wv[i])), f4to3(__ldg(&Wv[j])), o, fsc, msc, fnc, ktc,
                             krc);
            ++npc;
            oout[3 * k] = o.x; oout[3 * k + 1] = o.y; oout[3 * k + 2] = o.z;
            cm_out |= bit;
        }
    };
    contact_pass(true);

    bool replay = false;
    if (valid && !scan_not_needed(d, c, i, (float)xi.x, (float)xi.y, (float)xi.z)) {
        unsigned long long tried = mem;
        bool have_cells = false;
        Octant oc;
        const f3 xif = mk3((float)xi.x, (float)xi.y, (float)xi.z);
        const uint32_t qlim = scan_limit(d, c, i, xif.x, xif.y, xif.z, ncand);
        for (;;) {
            unsigned long long best = ~0ull;
            uint32_t best_q = 0;
            for (uint32_t q = 0; q < qlim; ++q) {
                if ((tried >> q) & 1ull) continue;
                const uint32_t j = __ldg(&d.cand[(size_t)q * N + i]);
                const double4 xj = ldg_d4(&P[j]);
                const double rr = dlen2(dsub(xj, xi));
                if (!(rr < cut2_add(c, xi.w, xj.w) && rr > 1e-10)) continue;
                if (!have_cells) { oc = octant_of(xif, c.g); have_cells = true; }
                const int rank = octant_rank(oc, ref_cell(mk3((float)xj.x, (float)xj.y, (float)xj.z), c.g));
                if (rank < 0) continue;
                const unsigned long long key = ((unsigned long long)rank << 32) | j;
                if (key < best) { best = key; best_q = q; }
            }
            if (best == ~0ull) break;
            tried |= 1ull << best_q;
            const uint32_t free = ~live & (c.K >= 32 ? 0xffffffffu : ((1u << c.K) - 1u));
            if (!free) { raise_status(&sc->err, RF_ERR_ROW_OVERFLOW); continue; }
            uint32_t k;
            if (i == G.p0 && (free & 1u) && (free & ~1u)) k = __ffs(free & ~1u) - 1;   // kdxfree==0 quirk
            else k = __ffs(free) - 1;
            const uint32_t j = (uint32_t)(best & 0xffffffffull);
            d.ids[(size_t)i * c.K + k] = j;
            live |= 1u << k;
            mem |= 1ull << best_q;
            dirty = true;
            const double4 xj = ldg_d4(&P[j]);
            const double sr = xi.w + xj.w;
            if (dlen2(dsub(xj, xi)) < sr * sr) replay = true;
        }
    }
    if (replay) {
        fsc = mk3(0.f, 0.f, 0.f); msc = fsc; cm_out = 0; fnc = 0.f; ktc = 0.f; krc = 0.f; npc = 0;
        contact_pass(false);
    }
    cm = cm_out | pc;
    fnabs += fnc;
    npair += npc;
    kt += ktc;
    kr += krc;

    float e2max = 0.f;
    double sfb = 0.0, sft = 0.0;
    uint32_t moved = 0;
    double acc[FIRE_SUMS];
#pragma unroll
    for (int q = 0; q < FIRE_SUMS; ++q) acc[q] = 0.0;
    if (valid) {
        // the bond pass's sums, waiting in shared memory through the contact pass
        const uint32_t wq = threadIdx.x >> 5, lq = threadIdx.x & 31u;
        const f3 vi = f4to3(Vv[i]), wi = f4to3(Wv[i]);
        const f3 fsb = mk3(s_acc[wq][0][lq], s_acc[wq][1][lq], s_acc[wq][2][lq]);
        const f3 msb = mk3(s_acc[wq][3][lq], s_acc[wq][4][lq], s_acc[wq][5][lq]);
        if (MODE == 1) {
            fnabs += s_acc[wq][6][lq]; kt += s_acc[wq][7][lq]; kr += s_acc[wq][8][lq];
            npair += s_msk[wq][W_NPAIR][lq];
        }
        if (dirty) { d.live[i] = live; d.bond[i] = bond; d.member[i] = mem; d.bmask[i] = bmask; }
        if (cm != cm0) d.cmask[i] = cm;
        // platens of this particle's specimen (with the reference constants their
        // coordinates are rounded to float, as the reference's drivers pass them)
        const double Top = c.ref_mode ? (double)(float)S->Top : S->Top;
        const double Bottom = c.ref_mode ? (double)(float)S->Bottom : S->Bottom;
        const double TopR = c.ref_mode ? (double)(float)S->TopR : S->TopR;
        const double BottomR = c.ref_mode ? (double)(float)S->BottomR : S->BottomR;
        const float vt = MODE == 0 ? (float)S->V : 0.f, RR = S->RR;
        rf_float3 cc;
        cc.x = S->center[0]; cc.y = S->center[1]; cc.z = S->center[2];
        float Fx = 0.0f + fsb.x, Fy = 0.0f + fsb.y, Fz = 0.0f + fsb.z;
        Fx += fsc.x; Fy += fsc.y; Fz += fsc.z;
        float Mx = 0.0f + msb.x, My = 0.0f + msb.y, Mz = 0.0f + msb.z;
        Mx += msc.x; My += msc.y; Mz += msc.z;
        double Rx = xi.x, Ry = xi.y, Rz = xi.z;
        float Vx = vi.x, Vy = vi.y, Vz = vi.z;
        if (KIND == RF_TEST_BRAZIL)
            brazil_particle_ext(Rx, Ry, Rz, Vx, Vy, Vz, Fx, Fy, Fz, cc, RR, Top, Bottom, TopR, BottomR, vt,
                                (double)G.zcut, xi.w - c.p_r_d, sfb, sft, MODE == 1);
        else
            uniaxial_particle_ext(Rx, Ry, Rz, Vx, Vy, Vz, Fx, Fy, Fz, cc, RR, Top, Bottom, TopR, BottomR, vt,
                                  (double)G.zcut, xi.w - c.p_r_d, sfb, sft, MODE == 1);
        if (MODE == 1) {
            // FIRE: keep the clamped state for the update kernel; reduce the FIRE sums
            d.posd[nxt][i] = make_double4(Rx, Ry, Rz, xi.w);
            d.vel[nxt][i] = make_float4(Vx, Vy, Vz, 0.f);
            d.ang[nxt][i] = make_float4(wi.x, wi.y, wi.z, 0.f);
            d.frc[i] = make_float4(Fx, Fy, Fz, kt);
            d.mom[i] = make_float4(Mx, My, Mz, kr);
            acc[0] = (double)Fx * Vx + (double)Fy * Vy + (double)Fz * Vz + (double)Mx * wi.x + (double)My * wi.y +
                     (double)Mz * wi.z;
            acc[1] = (double)Fx * Fx + (double)Fy * Fy + (double)Fz * Fz;
            acc[2] = (double)Vx * Vx + (double)Vy * Vy + (double)Vz * Vz;
            acc[3] = (double)Mx * Mx + (double)My * My + (double)Mz * Mz;
            acc[4] = (double)wi.x * wi.x + (double)wi.y * wi.y + (double)wi.z * wi.z;
            acc[5] = (double)fnabs;
            acc[6] = (double)npair;
            acc[7] = sfb;
            acc[8] = sft;
        }
        if (MODE == 0) {
        const float dtm = ep.dt / mi, dtI = ep.dt / (0.4f * mi * ri * ri);
        Vx += Fx * dtm; Vy += Fy * dtm; Vz += Fz * dtm;
        Rx += (double)(Vx * ep.dt); Ry += (double)(Vy * ep.dt); Rz += (double)(Vz * ep.dt);
        const float Wx = wi.x + Mx * dtI, Wy = wi.y + My * dtI, Wz = wi.z + Mz * dtI;
        const double dx = Rx - G.box_c.x, dy = Ry - G.box_c.y, dz = Rz - G.box_c.z;
        if ((dx - G.box_h.x > 0) || (dx + G.box_h.x < 0) || (dy - G.box_h.y > 0) || (dy + G.box_h.y < 0) ||
            (dz - G.box_h.z > 0) || (dz + G.box_h.z < 0)) {
            Rx = G.hp.x; Ry = G.hp.y; Rz = G.hp.z;
            Vx = 0.f; Vy = 0.f; Vz = 0.f;
        }
        d.posd[nxt][i] = make_double4(Rx, Ry, Rz, xi.w);
        d.vel[nxt][i] = make_float4(Vx, Vy, Vz, 0.f);
        d.ang[nxt][i] = make_float4(Wx, Wy, Wz, 0.f);
        const float4 pr = d.pos_ref[i];
        const float ex = (float)Rx - pr.x, ey = (float)Ry - pr.y, ez = (float)Rz - pr.z;
        const float e2 = ex * ex + ey * ey + ez * ez;
        moved = (e2 > c.disp2) ? 1u : 0u;
        // lists may have missed a neighbour (a particle moved to the hidden point has none)
        const bool hidden = Rx == (double)G.hp.x && Ry == (double)G.hp.y && Rz == (double)G.hp.z;
        if (e2 > c.hard2 && !hidden) raise_status(&d.sc->err, RF_ERR_CAPACITY);
        if (!hidden) e2max = e2;
        }
    }
    const uint32_t nbroken = s_msk[threadIdx.x >> 5][W_NB][threadIdx.x & 31u];
    if (MODE == 0) {
        note_displacement(d, e2max);
        step_finish_ext<KIND>(d, c, sfb, sft, nbroken, moved, sI - sA);
    } else {
        const uint32_t nb = __reduce_add_sync(FULL, nbroken);
        if ((threadIdx.x & 31) == 0 && nb) atomicAdd(&sc->broken, (unsigned long long)nb);
        fire_force_finish<KIND>(d, c, acc, sI - sA);
    }
}

// The FIRE decision of one specimen from its sums tot (FP64; n its particle count), by
// the last CTA's thread 0 (Bitzek et al. 2006):
//   residual = sqrt(sum |F_i|^2 / n) / (mean normal pair force); converged when <= tol;
//   P = F.v + M.w > 0: mixing v <- (1-a) v + a (|v|/|F|) F (same for w with M), and after
//   n_delay such steps dt <- min(dt f_inc, dt_max), a <- a f_alpha;
//   P <= 0: dt <- max(dt f_dec, dt_min), a <- a0, v = w = 0.
__device__ __forceinline__ void fire_decide(DevScalars* S, const Consts& c, const double* tot, uint32_t n) {
    const double P = tot[0], FF = tot[1], VV = tot[2], MM = tot[3], WW = tot[4], FN = tot[5], NP = tot[6];
    const double mean = NP > 0.0 ? FN / NP : 0.0;
    const double rms = sqrt(FF / (double)n);
    S->fmean = mean;
    S->fresidual = mean > 0.0 ? rms / mean : (FF > 0.0 ? 1e300 : 0.0);
    S->fpower = P;
    // platen stress of this configuration (SumForcesULoading's formula)
    const double a1 = (double)S->_1d_Area;
    S->Stress = 0.5 * (fabs(tot[7]) + fabs(tot[8])) * a1;
    S->fiter += 1;
    S->fiter_total += 1;
    if (S->fresidual <= S->ftol) { S->fconverged = 1; S->fstop = 1; return; }
    if (S->fiter >= S->fmax_iter) { S->fstop = 1; return; }
    if (S->fwarm) {
        // first pass of an increment: the velocities only carried the start motion into
        // the state; the dynamics starts from rest
        S->fwarm = 0;
        S->fuphill = 1;
        S->fnpos = 0;
        S->fcv = 0.0; S->fcf = 0.0; S->fcm = 0.0;
    } else if (P > 0.0) {
        const double a = S->falpha;
        S->fcv = 1.0 - a;
        S->fcf = FF > 0.0 ? a * sqrt(VV / FF) : 0.0;
        S->fcm = MM > 0.0 ? a * sqrt(WW / MM) : 0.0;
        S->fuphill = 0;
        S->fnpos += 1;
        if (S->fnpos > S->fndelay) {
            S->fdt = fmin(S->fdt * S->finc, S->fdtmax);
            S->falpha = a * S->fshrink;
        }
    } else {
        S->fnpos = 0;
        S->fdt = fmax(S->fdt * S->fdec, S->fdtmin);
        S->falpha = S->falpha0;
        S->fuphill = 1;
        S->fcv = 0.0; S->fcf = 0.0; S->fcm = 0.0;
    }
}

// Block sums of the FIRE accumulators (fixed tree, per specimen); the last block adds
// each specimen's block partials in block order and makes its FIRE decision.
template <int KIND>
__device__ __forceinline__ void fire_force_finish(const Dev& d, const Consts& c, double (&acc)[FIRE_SUMS],
                                                  uint32_t second) {
    DevScalars* sc = d.sc;
    const uint32_t FULL = 0xffffffffu;
    __shared__ double s_acc[4][FIRE_SUMS], s_acc2[4][FIRE_SUMS];
    __shared__ bool s_last;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    // a CTA touches at most two specimens: its sums are kept apart per specimen
#pragma unroll
    for (int q = 0; q < FIRE_SUMS; ++q) {
        double v = second ? 0.0 : acc[q], v2 = second ? acc[q] : 0.0;
        for (int o = 16; o; o >>= 1) {
            v += __shfl_xor_sync(FULL, v, o);
            v2 += __shfl_xor_sync(FULL, v2, o);
        }
        if (l == 0) { s_acc[w][q] = v; s_acc2[w][q] = v2; }
    }
    __syncthreads();
    if (threadIdx.x < FIRE_SUMS) {
        const int q = threadIdx.x;
        d.fpart[(size_t)blockIdx.x * FIRE_SUMS + q] = (s_acc[0][q] + s_acc[1][q]) + (s_acc[2][q] + s_acc[3][q]);
        if (d.fpart2)
            d.fpart2[(size_t)blockIdx.x * FIRE_SUMS + q] =
                (s_acc2[0][q] + s_acc2[1][q]) + (s_acc2[2][q] + s_acc2[3][q]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&sc->fcounter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the last CTA: per specimen still relaxing, its sums over its CTAs in CTA order, then
    // its FIRE decision
    __shared__ double tot[FIRE_SUMS];
    bool all_stopped = true;
    for (uint32_t sp = 0; sp < d.nspec; ++sp) {
        DevScalars* S = d.spec + sp;
        if (S->fstop) continue;                               // uniform across the CTA
        const SpecGeom& G = d.geom[sp];
        // fixed order: each thread a CTA-strided share of the blocks, then the warp trees,
        // then the four warps
        double v[FIRE_SUMS];
#pragma unroll
        for (int q = 0; q < FIRE_SUMS; ++q) v[q] = 0.0;
        for (uint32_t b = G.b0 + threadIdx.x; b <= G.b1; b += blockDim.x) {
            const double* src = (d.blk_spec == nullptr || d.blk_spec[b] == sp) ? d.fpart : d.fpart2;
#pragma unroll
            for (int q = 0; q < FIRE_SUMS; ++q) v[q] += __ldcg(&src[(size_t)b * FIRE_SUMS + q]);
        }
#pragma unroll
        for (int q = 0; q < FIRE_SUMS; ++q) {
            double x = v[q];
            for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
            if (l == 0) s_acc[w][q] = x;
        }
        __syncthreads();
        if (threadIdx.x < FIRE_SUMS) {
            const int q = threadIdx.x;
            tot[q] = (s_acc[0][q] + s_acc[1][q]) + (s_acc[2][q] + s_acc[3][q]);
        }
        __syncthreads();
        if (threadIdx.x == 0) fire_decide(S, c, tot, G.p1 - G.p0);
        __syncthreads();
        if (!S->fstop) all_stopped = false;
    }
    if (threadIdx.x != 0) return;
    sc->fcounter = 0;
    sc->steps += 1;                     // buffer parity: the update works on what this pass wrote
    if (d.nspec > 1) sc->fstop = all_stopped ? 1u : 0u;      // (with one specimen sc == spec)
}

// FIRE update of one iteration, in place on the buffers the force pass wrote:
// mixing (or, on uphill power, stop), then semi-implicit Euler in FP64
// positions; the rotation of the increment is accumulated for the warm-start data.
__global__ void k_fire_update(Dev d, Consts c) {
    DevScalars* sc = d.sc;
    const uint32_t cur = (uint32_t)(sc->steps & 1ull);
    const bool stop = sc->fstop != 0;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // the particle's specimen (a batch's specimens relax on their own FIRE scalars; one
    // whose relaxation stopped stays where it is)
    const uint32_t sA = d.blk_spec ? (uint32_t)d.blk_spec[blockIdx.x] : 0u;
    const DevScalars* S = d.spec + ((i < c.N && i >= d.geom[sA].p1) ? sA + 1u : sA);
    uint32_t moved = 0;
    float e2max = 0.f;
    if (!stop && i < c.N && !S->fstop) {
        double4 x = d.posd[cur][i];
        float4 v = d.vel[cur][i], w = d.ang[cur][i];
        const float4 F = d.frc[i], M = d.mom[i];
        const float dt = (float)S->fdt;
        const double dtd = (double)dt;
        if (S->fuphill) {
            // stop (no half step back: the bond and contact state integrates v dt, so every
            // position change must be a v dt of the force pass that follows)
            v = make_float4(0.f, 0.f, 0.f, 0.f);
            w = v;
        } else {
            const float cv = (float)S->fcv, cf = (float)S->fcf, cm = (float)S->fcm;
            v.x = cv * v.x + cf * F.x; v.y = cv * v.y + cf * F.y; v.z = cv * v.z + cf * F.z;
            w.x = cv * w.x + cm * M.x; w.y = cv * w.y + cm * M.y; w.z = cv * w.z + cm * M.z;
        }
        // stiffness-scaled (Jacobi) masses: every particle's own frequency is 1, so the
        // FIRE step is dimensionless and stiffness contrasts do not slow the relaxation
        const float dtm = dt / fmaxf(F.w, 1e-30f), dtI = dt / fmaxf(M.w, 1e-30f);
        v.x += F.x * dtm; v.y += F.y * dtm; v.z += F.z * dtm;
        w.x += M.x * dtI; w.y += M.y * dtI; w.z += M.z * dtI;
        x.x += (double)v.x * dtd; x.y += (double)v.y * dtd; x.z += (double)v.z * dtd;
        double4 r = d.rot[i];
        r.x += (double)w.x * dtd; r.y += (double)w.y * dtd; r.z += (double)w.z * dtd;
        d.rot[i] = r;
        d.posd[cur][i] = x;
        d.vel[cur][i] = v;
        d.ang[cur][i] = w;
        const float4 pr = d.pos_ref[i];
        const float ex = (float)x.x - pr.x, ey = (float)x.y - pr.y, ez = (float)x.z - pr.z;
        const float e2 = ex * ex + ey * ey + ez * ez;
        moved = (e2 > c.disp2) ? 1u : 0u;
        if (e2 > c.hard2) raise_status(&d.sc->err, RF_ERR_CAPACITY);   // lists may have missed a neighbour
        e2max = e2;
    }
    note_displacement(d, e2max);           // every lane of the warp takes part
    __shared__ bool s_last;
    __shared__ uint32_t s_m;
    if (threadIdx.x == 0) s_m = 0;
    __syncthreads();
    if (__reduce_or_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(&s_m, 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_m) atomicOr(&sc->moved, 1u);
        __threadfence();
        s_last = (atomicAdd(&sc->block_counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    sc->block_counter = 0;
    // largest displacement since the last candidate build of the positions the next force
    // pass reads (this update wrote them): the force pass's add-pass scan skip uses it
    sc->dmax = sqrtf(__uint_as_float(sc->d2max_next));
    sc->d2max_next = 0;
    const uint32_t mv = sc->moved;
    sc->moved = 0;
    sc->rebuild = mv;
    if (c.use_graph) {
        cudaGraphSetConditional(c.h_rebuild, (mv && !sc->fstop) ? 1u : 0u);
        cudaGraphSetConditional(c.h_loop, sc->fstop ? 0u : 1u);
    }
}

// Start of a quasi-static load increment: advance the loading platen by the increment
// (CompressU / CompressB with V dt replaced by -delta), reset the FIRE state, start
// from rest, remember the start positions, and apply a warm start if given:
// warm[i*6 + 0..2] is added to the position, warm[i*6 + 3..5] / dt0 becomes the
// initial angular velocity (so the first iteration's bond and contact state advance
// by that rotation).
template <int KIND>
__global__ void k_qs_begin_scalars(Dev d, Consts c, double sinc) {
    const int ax = (KIND == RF_TEST_BRAZIL) ? 1 : 2;
    for (uint32_t sp = threadIdx.x; sp < d.nspec; sp += blockDim.x) {
        DevScalars* S = d.spec + sp;
        const double delta = sinc * S->Size0;      // the specimen's platen advance
        S->V = 0.0;
        S->size_d[ax] -= delta;
        S->Top -= delta;
        S->TopR = S->Top - 2.0 * c.p_r_d;
        S->size[ax] = (float)S->size_d[ax];
        S->sized2[ax] = (float)(0.5 * S->size_d[ax]);
        S->center_d[ax] -= delta;
        S->center[ax] = (float)S->center_d[ax];
        S->Hd2 = S->sized2[ax];
        S->Strain = (S->size_d[ax] - S->Size0) / S->Size0;
        S->fdt = S->fdt0;
        S->falpha = S->falpha0;
        S->fnpos = 0; S->fiter = 0; S->fuphill = 0; S->fconverged = 0; S->fstop = 0;
        S->fcv = 1.0; S->fcf = 0.0; S->fcm = 0.0;
        S->fwarm = 1;
        S->done = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DevScalars* sc = d.sc;     // (with one specimen sc == spec)
        sc->fstop = 0;
        sc->fcounter = 0;
        sc->done = 0;
        sc->dmax = 3.0e38f;        // the increment moves particles (platen, warm start): the first pass scans
        sc->d2max_next = 0;
        sc->rebuild = 1;          // positions jumped (platen clamp, warm start): rebuild the candidates
    }
}
template <int KIND>
__global__ void k_qs_begin(Dev d, Consts c, const float* __restrict__ warm, int ldw, int scaled, double sinc) {
    const DevScalars* sc = d.sc;
    const uint32_t cur = (uint32_t)(sc->steps & 1ull);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;      // one particle per thread, 128-thread CTAs
    if (i >= c.N) return;
    const uint32_t sA = d.blk_spec ? (uint32_t)d.blk_spec[blockIdx.x] : 0u;
    const uint32_t sI = i >= d.geom[sA].p1 ? sA + 1u : sA;
    const DevScalars* S = d.spec + sI;
    const double zcut = (double)d.geom[sI].zcut;
    const float idt0 = (float)(1.0 / S->fdt0);
    const double D = sinc * S->Size0;                          // the specimen's platen advance
    const double Top = S->Top, Bottom = S->Bottom, TopR = S->TopR, BottomR = S->BottomR;
    const float RR = S->RR;
    rf_float3 cc;
    cc.x = S->center[0]; cc.y = S->center[1]; cc.z = S->center[2];
    {
        double4 x = d.posd[cur][i];
        d.x0[i] = x;
        float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
        float v0 = 0.f, v1 = 0.f, v2 = 0.f;
        double4 rot = make_double4(0.0, 0.0, 0.0, 0.0);
        if (warm) {
            // predicted displacement and rotation; as velocities over dt0 they make the first
            // force pass advance the bond and contact state by exactly that motion (the
            // first update then starts from rest)
            const float* q = warm + (size_t)i * ldw;
            float u[6];
            for (int a = 0; a < 6; ++a) u[a] = q[a];
            if (scaled) {                   // MLP units: displacement / D, rotation * r / D
                const float sd = (float)D, sr = (float)(D / x.w);
                u[0] *= sd; u[1] *= sd; u[2] *= sd; u[3] *= sr; u[4] *= sr; u[5] *= sr;
            }
            // a particle the platens held at the end of the last increment stays on its
            // platen (the top one has moved by D): the prediction's error along the load
            // axis must not lift it off
            const double off = x.w - c.p_r_d;
            const double a0 = KIND == RF_TEST_BRAZIL ? x.y : x.z;
            const float q0 = (float)(x.x - cc.x), q1 = KIND == RF_TEST_BRAZIL ? (float)(x.z - cc.z) : (float)(x.y - cc.y);
            const bool zone = q0 * q0 + q1 * q1 < RR && (KIND == RF_TEST_BRAZIL ? (double)(float)(x.z - cc.z) : a0) <
                                                          zcut;
            const bool at_top = zone && a0 + off - (Top + D) > -1e-9;
            const bool at_bottom = zone && a0 - off - Bottom < 1e-9;
            x.x += (double)u[0]; x.y += (double)u[1]; x.z += (double)u[2];
            v0 = u[0] * idt0; v1 = u[1] * idt0; v2 = u[2] * idt0;
            w = make_float4(u[3] * idt0, u[4] * idt0, u[5] * idt0, 0.f);
            rot = make_double4(u[3], u[4], u[5], 0.0);
            double& ax = KIND == RF_TEST_BRAZIL ? x.y : x.z;
            if (at_top) ax = Top - off;
            else if (at_bottom) ax = Bottom + off;
        }
        // the platen pushes the particles it passed: clamp them now, so the first force
        // pass (and its convergence test) sees the loaded configuration
        float f0 = 0.f, f1 = 0.f, f2 = 0.f;
        double sb = 0.0, st = 0.0;
        if (KIND == RF_TEST_BRAZIL)
            brazil_particle_ext(x.x, x.y, x.z, v0, v1, v2, f0, f1, f2, cc, RR, Top, Bottom, TopR, BottomR, 0.f,
                                zcut, x.w - c.p_r_d, sb, st, false);
        else
            uniaxial_particle_ext(x.x, x.y, x.z, v0, v1, v2, f0, f1, f2, cc, RR, Top, Bottom, TopR, BottomR, 0.f,
                                  zcut, x.w - c.p_r_d, sb, st, false);
        d.posd[cur][i] = x;
        d.vel[cur][i] = make_float4(v0, v1, v2, 0.f);
        d.ang[cur][i] = w;
        d.rot[i] = rot;
    }
}

// The specimen of particle i in a kernel of 128-thread CTAs, one particle per thread.
__device__ __forceinline__ const DevScalars* spec_of(const Dev& d, uint32_t i) {
    const uint32_t sA = d.blk_spec ? (uint32_t)d.blk_spec[blockIdx.x] : 0u;
    return d.spec + (i >= d.geom[sA].p1 ? sA + 1u : sA);
}

// Warm-start features of each particle from the last increment's motion (layout in the
// header); sinc = strain_inc, D = sinc * the specimen's initial size (its platen advance).
template <int KIND>
__global__ void k_warm_features(Dev d, Consts c, double sinc, __nv_bfloat16* __restrict__ feat) {
    const uint32_t cur = (uint32_t)(d.sc->steps & 1ull);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const DevScalars* sc = spec_of(d, i);
    const double D = sinc * sc->Size0;
    const int ax = (KIND == RF_TEST_BRAZIL) ? 1 : 2;
    const double iD = 1.0 / D;
    const double4 x = d.posd[cur][i], x0 = d.x0[i], r = d.rot[i];
    float f[64];
#pragma unroll
    for (int q = 0; q < 64; ++q) f[q] = 0.f;
    const double dxi = x.x - x0.x, dyi = x.y - x0.y, dzi = x.z - x0.z;
    f[0] = (float)(dxi * iD); f[1] = (float)(dyi * iD); f[2] = (float)(dzi * iD);
    f[3] = (float)(r.x * x.w * iD); f[4] = (float)(r.y * x.w * iD); f[5] = (float)(r.z * x.w * iD);
    const double p[3] = {x.x - sc->center_d[0], x.y - sc->center_d[1], x.z - sc->center_d[2]};
    f[6] = (float)(p[ax] / (0.5 * sc->size_d[ax]));
    const double o0 = p[ax == 2 ? 0 : 0], o1 = p[ax == 2 ? 1 : 2];
    f[7] = (float)(sqrt(o0 * o0 + o1 * o1) / (0.5 * sc->size_d[0]));
    const size_t QN = (size_t)d.QB * c.N;
    (void)QN;
    const uint32_t bm = d.bmask[i], nq = d.nbq[i];
    int nb = 0;
    for (uint32_t q = 0; q < nq && nb < 12; ++q) {
        if (!((bm >> q) & 1u)) continue;
        const size_t s = (size_t)q * c.N + i;
        const uint32_t j = d.bj[s];
        const double4 xj = d.posd[cur][j], xj0 = d.x0[j];
        const double ex = (xj.x - xj0.x) - dxi, ey = (xj.y - xj0.y) - dyi, ez = (xj.z - xj0.z) - dzi;
        const double rx = xj.x - x.x, ry = xj.y - x.y, rz = xj.z - x.z;
        const double L0 = d.bL0[s];
        float* g = f + 8 + 4 * nb;
        g[0] = (float)(ex * iD); g[1] = (float)(ey * iD); g[2] = (float)(ez * iD);
        g[3] = (float)((sqrt(rx * rx + ry * ry + rz * rz) - L0) / (L0 * sinc));
        ++nb;
    }
    f[56] = (float)nb * (1.0f / 12.0f);
    const double xa = ax == 1 ? x.y : x.z, off = x.w - c.p_r_d;
    f[57] = (xa + off - sc->Top > -1e-9 || xa - off - sc->Bottom < 1e-9) ? 1.f : 0.f;
    f[58] = 1.f;
    uint4* out = reinterpret_cast<uint4*>(feat + (size_t)i * 64);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        __nv_bfloat162 h0 = __floats2bfloat162_rn(f[8 * q + 0], f[8 * q + 1]);
        __nv_bfloat162 h1 = __floats2bfloat162_rn(f[8 * q + 2], f[8 * q + 3]);
        __nv_bfloat162 h2 = __floats2bfloat162_rn(f[8 * q + 4], f[8 * q + 5]);
        __nv_bfloat162 h3 = __floats2bfloat162_rn(f[8 * q + 6], f[8 * q + 7]);
        uint4 u;
        u.x = *reinterpret_cast<uint32_t*>(&h0); u.y = *reinterpret_cast<uint32_t*>(&h1);
        u.z = *reinterpret_cast<uint32_t*>(&h2); u.w = *reinterpret_cast<uint32_t*>(&h3);
        out[q] = u;
    }
}

// Targets of the last increment: displacement / D and rotation * r / D.
__global__ void k_warm_targets(Dev d, Consts c, double sinc, float* __restrict__ t) {
    const uint32_t cur = (uint32_t)(d.sc->steps & 1ull);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const double D = sinc * spec_of(d, i)->Size0;
    const double iD = 1.0 / D;
    const double4 x = d.posd[cur][i], x0 = d.x0[i], r = d.rot[i];
    float* o = t + (size_t)i * 6;
    o[0] = (float)((x.x - x0.x) * iD); o[1] = (float)((x.y - x0.y) * iD); o[2] = (float)((x.z - x0.z) * iD);
    o[3] = (float)(r.x * x.w * iD); o[4] = (float)(r.y * x.w * iD); o[5] = (float)(r.z * x.w * iD);
}

// Start positions of the first increment: x0 = x, no rotation.
__global__ void k_fire_buffers_init(Dev d, Consts c) {
    const uint32_t cur = (uint32_t)(d.sc->steps & 1ull);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        d.x0[i] = d.posd[cur][i];
        d.rot[i] = make_double4(0.0, 0.0, 0.0, 0.0);
    }
}

// Sets the FIRE loop's graph conditions at the start of a launch.
__global__ void k_fire_prologue(Dev d, Consts c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        DevScalars* sc = d.sc;
        const bool go = !sc->fstop;
        cudaGraphSetConditional(c.h_rebuild, (go && sc->rebuild) ? 1u : 0u);
        cudaGraphSetConditional(c.h_loop, go ? 1u : 0u);
    }
}

// Sets both graph conditions at the start of a launch.
__global__ void k_prologue(Dev d, Consts c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        DevScalars* sc = d.sc;
        const bool go = !sc->done && sc->steps < sc->target;
        if (c.use_graph) {
            cudaGraphSetConditional(c.h_rebuild, (go && sc->rebuild) ? 1u : 0u);
            cudaGraphSetConditional(c.h_loop, go ? 1u : 0u);
        }
    }
}

// On a plain stream: stop once the target step count is reached.
__global__ void k_stream_gate(Dev d) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        DevScalars* sc = d.sc;
        if (sc->steps >= sc->target) sc->done = sc->done | 2u;
    }
}
__global__ void k_stream_ungate(Dev d) {
    if (threadIdx.x == 0 && blockIdx.x == 0) d.sc->done &= 1u;
}

// ---------------------------------------------------------------------------
// Layout conversion (reference layout <-> engine layout)
// ---------------------------------------------------------------------------
__global__ void k_planar_to_f4(const float* __restrict__ R, uint32_t N, float4* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        out[i] = make_float4(R[i], R[i + N], R[i + 2 * (size_t)N], 0.f);
}
__global__ void k_f4_to_planar(const float4* __restrict__ in, uint32_t N, float* __restrict__ R) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float4 v = in[i];
        R[i] = v.x; R[i + N] = v.y; R[i + 2 * (size_t)N] = v.z;
    }
}

// Bond records a reference-layout row needs: its intact bonds, and broken bonds that
// still carry a bond direction (Rij is kept until the slot is deleted).
__device__ __forceinline__ bool needs_record(uint8_t type, const rf_float3 r) {
    return type == 1 || r.x != 0.f || r.y != 0.f || r.z != 0.f;
}

__global__ void k_count_records(const uint_fast32_t* __restrict__ IL, const uint8_t* __restrict__ type,
                                const rf_float3* __restrict__ Rij, uint32_t N, uint32_t K, uint32_t* maxq) {
    const uint_fast32_t E = empty_id<uint_fast32_t>();
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        uint32_t n = 0;
        for (uint32_t k = 0; k < K; ++k) {
            const size_t r = (size_t)i * K + k;
            if (IL[r] != E && IL[r] < N && needs_record(type[r], Rij[r])) ++n;
        }
        m = max(m, n);
    }
    atomicMax(maxq, m);
}

// Reference-layout rows (uint_fast32_t ids, AoS float3 state) -> engine rows and records.
__global__ void k_rows_import(const uint_fast32_t* __restrict__ IL, const uint8_t* __restrict__ type,
                              const float* __restrict__ iL, const rf_float3* __restrict__ Rij,
                              const rf_float3* __restrict__ Oijt, const rf_float3* __restrict__ Mijn,
                              const rf_float3* __restrict__ Mijt, const double* __restrict__ L0x,
                              const float2* __restrict__ strx, Dev d, Consts c) {
    const uint_fast32_t E = empty_id<uint_fast32_t>();
    const size_t QN = (size_t)d.QB * c.N;
    const uint32_t cur = (uint32_t)(d.sc->steps & 1ull);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        uint32_t live = 0, bond = 0, cm = 0, nq = 0, bmask = 0;
        for (uint32_t k = 0; k < c.K; ++k) {
            const size_t r = (size_t)i * c.K + k, s = (size_t)k * c.N + i;
            const uint_fast32_t j = IL[r];
            const bool ok = (j != E && j < c.N);
            d.ids[r] = ok ? (uint32_t)j : EMPTY32;
            d.il[s] = iL[r];
            const bool t1 = ok && type[r] == 1;
            float* co = d.cO[cur] + 3 * r;
            co[0] = t1 ? 0.f : Oijt[r].x; co[1] = t1 ? 0.f : Oijt[r].y; co[2] = t1 ? 0.f : Oijt[r].z;
            if (!ok) continue;
            live |= 1u << k;
            if (t1) bond |= 1u << k;
            else if (Oijt[r].x != 0.f || Oijt[r].y != 0.f || Oijt[r].z != 0.f) cm |= 1u << k;
            if (needs_record(type[r], Rij[r]) && nq < d.QB) {
                const size_t b = (size_t)nq * c.N + i;
                d.bj[b] = (uint32_t)j; d.bk[b] = (uint8_t)k; d.bil[b] = iL[r];
                const float ox = t1 ? Oijt[r].x : 0.f, oy = t1 ? Oijt[r].y : 0.f, oz = t1 ? Oijt[r].z : 0.f;
                d.bst[b] = make_float4(Rij[r].x, Rij[r].y, Rij[r].z, ox);
                d.bst[b + QN] = make_float4(oy, oz, Mijn[r].x, Mijn[r].y);
                d.bst[b + 2 * QN] = make_float4(Mijn[r].z, Mijt[r].x, Mijt[r].y, Mijt[r].z);
                if (L0x) { d.bL0[b] = L0x[r]; d.bstr[b] = strx[r]; }
                if (t1) bmask |= 1u << nq;
                ++nq;
            }
        }
        for (uint32_t q = nq; q < d.QB; ++q) {          // unused records: retired, zero
            const size_t b = (size_t)q * c.N + i;
            d.bj[b] = 0; d.bk[b] = 0xFF; d.bil[b] = 0.f;
            if (L0x) { d.bL0[b] = 1.0; d.bstr[b] = make_float2(0.f, 0.f); }
            zero_record(d, QN, b);
        }
        d.live[i] = live; d.bond[i] = bond; d.cmask[i] = cm; d.nbq[i] = nq; d.bmask[i] = bmask;
    }
}

__global__ void k_rows_export(uint_fast32_t* __restrict__ IL, uint8_t* __restrict__ type, float* __restrict__ iL,
                              rf_float3* __restrict__ Rij, rf_float3* __restrict__ Oijt, rf_float3* __restrict__ Mijn,
                              rf_float3* __restrict__ Mijt, Dev d, Consts c) {
    const uint_fast32_t E = empty_id<uint_fast32_t>();
    const size_t QN = (size_t)d.QB * c.N;
    const uint32_t cur = (uint32_t)(d.sc->steps & 1ull);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const uint32_t live = d.live[i], bond = d.bond[i], nq = d.nbq[i];
        for (uint32_t k = 0; k < c.K; ++k) {
            const size_t r = (size_t)i * c.K + k, s = (size_t)k * c.N + i;
            IL[r] = ((live >> k) & 1u) ? (uint_fast32_t)d.ids[r] : E;
            type[r] = (uint8_t)((bond >> k) & 1u);
            iL[r] = d.il[s];
            Rij[r].x = 0.f; Rij[r].y = 0.f; Rij[r].z = 0.f;
            Mijn[r] = Rij[r]; Mijt[r] = Rij[r];
            const bool has = ((d.cmask[i] >> k) & 1u) != 0;
            const float* co = d.cO[cur] + 3 * r;
            Oijt[r].x = has ? co[0] : 0.f; Oijt[r].y = has ? co[1] : 0.f; Oijt[r].z = has ? co[2] : 0.f;
        }
        for (uint32_t q = 0; q < nq; ++q) {
            const size_t b = (size_t)q * c.N + i;
            const uint32_t k = d.bk[b];
            if (k == 0xFF) continue;
            const size_t r = (size_t)i * c.K + k;
            const float4 s0 = d.bst[b], s1 = d.bst[b + QN], s2 = d.bst[b + 2 * QN];
            Rij[r].x = s0.x; Rij[r].y = s0.y; Rij[r].z = s0.z;
            Mijn[r].x = s1.z; Mijn[r].y = s1.w; Mijn[r].z = s2.x;
            Mijt[r].x = s2.y; Mijt[r].y = s2.z; Mijt[r].z = s2.w;
            if ((bond >> k) & 1u) { Oijt[r].x = s0.w; Oijt[r].y = s1.x; Oijt[r].z = s1.y; }
        }
    }
}

// Bond construction of the extended model: slot (i, k) -> j becomes a bond when the
// gap |r_ij| - r_i - r_j is below gap_frac * min(r_i, r_j) (distances in double). The
// rest length is |r_ij| in double; tensile and shear strengths are Weibull draws
// scale * (-ln U)^(1/m) keyed on the unordered pair, so both directed slots of a pair
// share them. The slot state starts at zero, as d_ConstructBoundInteractions leaves it.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double pair_uniform(uint64_t seed, uint32_t a, uint32_t b, uint32_t stream) {
    const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
    const uint64_t h = mix64(mix64(seed ^ (0x51ED270B27F3A4C1ull * (stream + 1))) + (hi << 32 | lo));
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);       // in (0, 1)
}
// Bond rule and strength distribution of one specimen of a batch.
struct BondSpec {
    double gap_frac, wm, sig, tau;
    uint64_t seed;
    uint32_t p0, p1;            // its particles
    int ref_mode;               // reference constants: bonds below the centre distance bd, strengths sig, tau
    double bd;
};
// Initial rows of the extended model with a list gap g: the reference's construction
// (md_interaction_list_construct.cu:13-98: the 8 octant cells in visiting order, their
// occupants in cell order, slots filled in order) with the pair test
// rr < min(a_farcut, r_i + r_j + g)^2 on the FP64 positions. IL is preset to empty.
__global__ void k_list_ext(const float* __restrict__ R, const double4* __restrict__ P, uint32_t N,
                           const uint_fast32_t* __restrict__ CIs, const uint_fast32_t* __restrict__ pnC,
                           uint_fast32_t* __restrict__ IL, uint32_t K, RefGrid g, double a_farcut, double gap,
                           uint32_t* err) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        int64_t cells[8];
        octant_cells(mk3(R[i], R[i + N], R[i + 2 * (size_t)N]), g, cells);
        const double4 xi = P[i];
        uint32_t n = 0;
        for (int c = 0; c < 8; ++c) {
            if (cells[c] < 0 || (uint64_t)cells[c] >= g.CN) { raise_status(err, RF_ERR_CELL_RANGE); continue; }
            const uint64_t s = (uint64_t)pnC[cells[c]], cnt = (uint64_t)pnC[cells[c] + g.CN];
            for (uint64_t m = 0; m < cnt; ++m) {
                if (s + m >= N) break;
                const uint_fast32_t j = CIs[s + m + N];
                if (j >= N) continue;
                const double4 xj = P[j];
                const double rr = dlen2(dsub(xj, xi));
                const double q = fmin(a_farcut, (xi.w + xj.w) + gap);
                if (rr < q * q && j != i) {
                    if (n < K) IL[(size_t)i * K + n] = j;
                    else raise_status(err, RF_ERR_ROW_OVERFLOW);
                    ++n;
                }
            }
        }
    }
}

__global__ void k_bond_ext(const double4* __restrict__ P, const uint_fast32_t* __restrict__ IL,
                           uint8_t* __restrict__ type, float* __restrict__ iL, double* __restrict__ L0x,
                           float2* __restrict__ strx, uint32_t N, uint32_t K, const BondSpec* __restrict__ bs,
                           uint32_t nspec) {
    const uint_fast32_t E = empty_id<uint_fast32_t>();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        uint32_t sp = 0;
        while (sp + 1 < nspec && i >= bs[sp].p1) ++sp;
        const double gap_frac = bs[sp].gap_frac, sig = bs[sp].sig, tau = bs[sp].tau;
        const double inv_m = 1.0 / bs[sp].wm;
        const uint64_t seed = bs[sp].seed;
        const uint32_t pbase = bs[sp].p0;       // strengths keyed on specimen-local ids
        const double4 xi = P[i];
        for (uint32_t k = 0; k < K; ++k) {
            const size_t r = (size_t)i * K + k;
            const uint_fast32_t j = IL[r];
            type[r] = 0; iL[r] = 0.f; L0x[r] = 1.0; strx[r] = make_float2(0.f, 0.f);
            if (j == E || j >= N) continue;
            const double4 xj = P[j];
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const double L = sqrt(dx * dx + dy * dy + dz * dz);
            if (bs[sp].ref_mode) {
                // md_boundinteractions_construct.cu:62 (on the FP64 distance), global strengths
                if (!(L < bs[sp].bd) || !(L > 0)) continue;
            } else if (!(L - xi.w - xj.w < gap_frac * fmin(xi.w, xj.w)) || !(L > 0)) {
                continue;
            }
            type[r] = 1;
            iL[r] = (float)(1.0 / L);
            L0x[r] = L;
            if (bs[sp].ref_mode) { strx[r] = make_float2((float)sig, (float)tau); continue; }
            const uint32_t li = i - pbase, lj = (uint32_t)j - pbase;
            const double us = pair_uniform(seed, li, lj, 0), ut = pair_uniform(seed, li, lj, 1);
            strx[r] = make_float2((float)(sig * pow(-log(us), inv_m)), (float)(tau * pow(-log(ut), inv_m)));
        }
    }
}
__global__ void k_posd_from_planar(const double* __restrict__ R, const double* __restrict__ rad, uint32_t N,
                                   double4* __restrict__ out, float* __restrict__ Rf) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double x = R[i], y = R[i + N], z = R[i + 2 * (size_t)N];
        out[i] = make_double4(x, y, z, rad[i]);
        if (Rf) { Rf[i] = (float)x; Rf[i + N] = (float)y; Rf[i + 2 * (size_t)N] = (float)z; }
    }
}
__global__ void k_posd_to_planar(const double4* __restrict__ in, uint32_t N, double* __restrict__ R) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double4 v = in[i];
        R[i] = v.x; R[i + N] = v.y; R[i + 2 * (size_t)N] = v.z;
    }
}
__global__ void k_posd_to_planar_f(const double4* __restrict__ in, uint32_t N, float* __restrict__ R) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double4 v = in[i];
        R[i] = (float)v.x; R[i + N] = (float)v.y; R[i + 2 * (size_t)N] = (float)v.z;
    }
}

__global__ void k_counters(Dev d, Consts c, unsigned long long* out) {
    unsigned long long nb = 0, nc = 0, nl = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const uint32_t l = d.live[i], b = d.bond[i];
        nl += __popc(l); nb += __popc(b); nc += __popc(d.cmask[i]);
    }
    atomicAdd(&out[0], nb); atomicAdd(&out[1], nc); atomicAdd(&out[2], nl);
}


__global__ void k_set_target(DevScalars* sc, unsigned long long n) { sc->target = sc->steps + n; }
__global__ void k_force_rebuild(DevScalars* sc) { sc->rebuild = 1u; }

// Homogeneous strain of the specimen about the platen box's centre: every position (and
// the load axis's platens with them) scaled by 1 + eps per axis; the platen zone's radius
// grows with the larger lateral strain. Rest lengths, slot state and velocities stay, so
// the bonds and contacts carry the strain from the next step on.
__global__ void k_affine_positions(Dev d, Consts c, double ex, double ey, double ez) {
    const uint32_t cur = (uint32_t)(d.sc->steps & 1ull);
    const double cx = d.sc->center_d[0], cy = d.sc->center_d[1], cz = d.sc->center_d[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        if (c.ext) {
            double4 x = d.posd[cur][i];
            x.x = cx + (1.0 + ex) * (x.x - cx); x.y = cy + (1.0 + ey) * (x.y - cy); x.z = cz + (1.0 + ez) * (x.z - cz);
            d.posd[cur][i] = x;
        } else {
            float4 x = d.pos[cur][i];
            x.x = (float)(cx + (1.0 + ex) * ((double)x.x - cx));
            x.y = (float)(cy + (1.0 + ey) * ((double)x.y - cy));
            x.z = (float)(cz + (1.0 + ez) * ((double)x.z - cz));
            d.pos[cur][i] = x;
        }
    }
}
template <int KIND>
__global__ void k_affine_scalars(Dev d, Consts c, double ex, double ey, double ez) {
    DevScalars* sc = d.sc;
    if (blockIdx.x || threadIdx.x) return;
    const int ax = (KIND == RF_TEST_BRAZIL) ? 1 : 2;
    const double e = ax == 1 ? ey : ez, el = ax == 1 ? fmax(ex, ez) : fmax(ex, ey);
    const double ca = sc->center_d[ax];
    const double dtr = sc->TopR - sc->Top, dbr = sc->BottomR - sc->Bottom;
    sc->Top = ca + (1.0 + e) * (sc->Top - ca);
    sc->Bottom = ca + (1.0 + e) * (sc->Bottom - ca);
    sc->TopR = sc->Top + dtr;
    sc->BottomR = sc->Bottom + dbr;
    sc->size_d[ax] *= 1.0 + e;
    sc->size[ax] = (float)sc->size_d[ax];
    sc->sized2[ax] = (float)(0.5 * sc->size_d[ax]);
    sc->Hd2 = sc->sized2[ax];
    sc->Strain = (sc->size_d[ax] - sc->Size0) / sc->Size0;
    sc->RR = (float)((double)sc->RR * (1.0 + el) * (1.0 + el));
    sc->dmax = 3.0e38f;          // positions jumped: the next add pass scans
    sc->d2max_next = 0;
    sc->rebuild = 1;             // and the candidate lists are rebuilt first
}
__global__ void k_planar_to_cur(const float* __restrict__ R, Dev d) {
    const uint32_t N = (uint32_t)(d.n_particles);
    if (d.posd[0]) {                      // extended model: keep the radius
        double4* out = d.posd[d.sc->steps & 1ull];
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
            out[i] = make_double4(R[i], R[i + N], R[i + 2 * (size_t)N], out[i].w);
    } else {
        float4* out = d.pos[d.sc->steps & 1ull];
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
            out[i] = make_float4(R[i], R[i + N], R[i + 2 * (size_t)N], 0.f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) d.sc->rebuild = 1u;
}
__global__ void k_cur_to_planar(Dev d, float* __restrict__ R) {
    const uint32_t N = (uint32_t)(d.n_particles);
    if (d.posd[0]) {
        const double4* in = d.posd[d.sc->steps & 1ull];
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
            const double4 v = in[i];
            R[i] = (float)v.x; R[i + N] = (float)v.y; R[i + 2 * (size_t)N] = (float)v.z;
        }
        return;
    }
    const float4* in = d.pos[d.sc->steps & 1ull];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float4 v = in[i];
        R[i] = v.x; R[i + N] = v.y; R[i + 2 * (size_t)N] = v.z;
    }
}

}  // namespace rf

using namespace rf;

struct rf_engine {
    rf_task task;
    Dev d;
    Consts c;
    int device;
    cudaStream_t stream;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    uint32_t nblocks;
    uint32_t cg_nb;
    bool graph_ok;
    std::vector<void*> allocs;
    std::vector<size_t> alloc_bytes;
    int step_minb = RF_STEP_MIN_BLOCKS;    // register-cap variant of the extended step (autotuned)
    unsigned long long* counters_dev;
    float* staging;
    uint64_t bonds_initial;
    uint32_t* maxq_dev;
    // batch of specimens
    std::vector<rf_task> spec_tasks;   // per specimen, shifted, with the batch's cell grid
    std::vector<uint32_t> spec_p0, spec_n;
    std::vector<double> spec_xoff;
    // FIRE relaxation graph (built on the first load increment)
    Consts cf;
    cudaGraph_t fgraph;
    cudaGraphExec_t fexec;
    bool fire_ready;
};

namespace {

template <class T> rf_status dalloc(rf_engine* e, T** p, size_t n) {
    void* q = nullptr;
    RF_CUDA(cudaMalloc(&q, (n ? n : 1) * sizeof(T)));
    e->allocs.push_back(q);
    e->alloc_bytes.push_back((n ? n : 1) * sizeof(T));
    *p = (T*)q;
    return RF_OK;
}

#define TRY(x) do { rf_status s__ = (x); if (s__ != RF_OK) return s__; } while (0)

// Explicit extended-model step kernels compiled for 5, 6 or 8 CTAs per SM.
void* ext_step_variant(bool brazil, int minb) {
    switch (minb) {
        case 8: return brazil ? (void*)k_step_ext<RF_TEST_BRAZIL, 0, 8> : (void*)k_step_ext<RF_TEST_UNIAXIAL, 0, 8>;
        case 5: return brazil ? (void*)k_step_ext<RF_TEST_BRAZIL, 0, 5> : (void*)k_step_ext<RF_TEST_UNIAXIAL, 0, 5>;
        default: return brazil ? (void*)k_step_ext<RF_TEST_BRAZIL, 0, 6> : (void*)k_step_ext<RF_TEST_UNIAXIAL, 0, 6>;
    }
}

// dynamic shared memory of a step launch: the extended kernel's per-warp record list
// (32 particles x QB records, 2 bytes each, 4 warps)
unsigned step_smem(const rf_engine* e) { return e->c.ext ? 4u * 32u * e->d.QB * 2u : 0u; }

void* step_kernel(const rf_engine* e) {
    const bool br = e->task.kind == RF_TEST_BRAZIL;
    if (e->c.ext) return ext_step_variant(br, e->step_minb);
    return br ? (void*)k_step<RF_TEST_BRAZIL> : (void*)k_step<RF_TEST_UNIAXIAL>;
}

rf_status build_graph(rf_engine* e) {
    cudaGraph_t g;
    RF_CUDA(cudaGraphCreate(&g, 0));
    e->graph = g;
    // The loop body is RF_GRAPH_UNROLL steps, each preceded by IF(rebuild) {rebuild
    // kernels} or, for specimens below RF_REBUILD_EACH_STEP_N particles, only the first:
    // there a conditional node costs as much as a few percent of a step, and the rebuild
    // condition is evaluated once per RF_GRAPH_UNROLL steps. The rebuild trigger is set at
    // 0.3 of the skin so that the particles' motion until the next evaluation stays within
    // the 0.5 skin the candidate lists are complete for; a step that finds a particle beyond
    // 0.5 skin reports RF_ERR_CAPACITY. Evaluating before every step lets particles move 0.2
    // skin per step (fragments of a damaged large specimen), against 0.2 skin per
    // RF_GRAPH_UNROLL steps otherwise. Each IF node has its own conditional handle (a handle
    // drives one conditional node); a step node's parameters carry the handle of the IF
    // node after it (the last step's: the body's first IF, evaluated on the next iteration),
    // the prologue's the first. The WHILE condition is evaluated once per body. A step
    // whose step count has reached the target returns at once, so the target is kept exactly.
    const int every = e->c.N >= RF_REBUILD_EACH_STEP_N ? 1 : RF_GRAPH_UNROLL;
    const int nif = RF_GRAPH_UNROLL / every;
    cudaGraphConditionalHandle hif[RF_GRAPH_UNROLL];
    RF_CUDA(cudaGraphConditionalHandleCreate(&e->c.h_loop, g, 0, 0));
    for (int q = 0; q < nif; ++q) RF_CUDA(cudaGraphConditionalHandleCreate(&hif[q], g, 0, 0));
    e->c.h_rebuild = hif[0];
    e->c.use_graph = 1;
    Dev d = e->d;
    Consts c = e->c;
    void* args[] = {&d, &c};
    auto kparams = [&](void* fn, unsigned grid, unsigned block, void** a) {
        cudaKernelNodeParams kp = {};
        kp.func = fn; kp.gridDim = dim3(grid); kp.blockDim = dim3(block);
        kp.sharedMemBytes = 0; kp.kernelParams = a; kp.extra = nullptr;
        return kp;
    };
    // prologue -> WHILE
    cudaGraphNode_t pro;
    cudaKernelNodeParams kp = kparams((void*)k_prologue, 1, 32, args);
    RF_CUDA(cudaGraphAddKernelNode(&pro, g, nullptr, 0, &kp));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = e->c.h_loop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    RF_CUDA(cudaGraphAddNode(&wnode, g, &pro, 1, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    const unsigned gN = (e->c.N + 255) / 256;
    const unsigned gC = (e->c.cg_cells + 1 + 255) / 256;
    struct { void* fn; unsigned grid, block; } seq[] = {
        {(void*)k_rb_zero, gC, 256},      {(void*)k_rb_bin, gN, 256},
        {(void*)k_rb_scan_sums, e->cg_nb, 1024}, {(void*)k_rb_scan_totals, 1, 32},
        {(void*)k_rb_scan_apply, e->cg_nb, 1024}, {(void*)k_rb_scatter, gN, 256},
        {(void*)k_rb_cand, (e->c.N + 127) / 128, 128},
    };
    void* fn = step_kernel(e);
    // per step node: Consts with the handle of the IF node that follows it (node parameters
    // are copied when the node is added, so one slot per step suffices until then)
    Consts cs[RF_GRAPH_UNROLL];
    void* sargs[RF_GRAPH_UNROLL][2];
    cudaGraphNode_t last = nullptr;
    for (int u = 0; u < RF_GRAPH_UNROLL; ++u) {
        if (u % every == 0) {
            cudaGraphNodeParams ip = {};
            ip.type = cudaGraphNodeTypeConditional;
            ip.conditional.handle = hif[u / every];
            ip.conditional.type = cudaGraphCondTypeIf;
            ip.conditional.size = 1;
            cudaGraphNode_t inode;
            RF_CUDA(cudaGraphAddNode(&inode, body, last ? &last : nullptr, last ? 1 : 0, &ip));
            cudaGraph_t rb = ip.conditional.phGraph_out[0];
            cudaGraphNode_t prev = nullptr;
            for (auto& q : seq) {
                cudaGraphNode_t n;
                kp = kparams(q.fn, q.grid, q.block, args);
                RF_CUDA(cudaGraphAddKernelNode(&n, rb, prev ? &prev : nullptr, prev ? 1 : 0, &kp));
                prev = n;
            }
            last = inode;
        }
        cs[u] = c;
        cs[u].h_rebuild = hif[((u + 1) / every) % nif];
        sargs[u][0] = &d;
        sargs[u][1] = &cs[u];
        cudaGraphNode_t step;
        kp = kparams(fn, e->nblocks, 128, sargs[u]);
        kp.sharedMemBytes = step_smem(e);
        RF_CUDA(cudaGraphAddKernelNode(&step, body, &last, 1, &kp));
        last = step;
    }
    RF_CUDA(cudaGraphInstantiate(&e->exec, g, 0));
    return RF_OK;
}

// FIRE loop graph: prologue -> WHILE(not stopped) { IF(moved) {candidate rebuild}; forces; update }.
rf_status build_fire_graph(rf_engine* e) {
    cudaGraph_t g;
    RF_CUDA(cudaGraphCreate(&g, 0));
    e->fgraph = g;
    Consts& c = e->cf;
    RF_CUDA(cudaGraphConditionalHandleCreate(&c.h_loop, g, 0, 0));
    RF_CUDA(cudaGraphConditionalHandleCreate(&c.h_rebuild, g, 0, 0));
    c.use_graph = 1;
    Dev d = e->d;
    Consts cc = c;
    void* args[] = {&d, &cc};
    auto kparams = [&](void* fn, unsigned grid, unsigned block) {
        cudaKernelNodeParams kp = {};
        kp.func = fn; kp.gridDim = dim3(grid); kp.blockDim = dim3(block);
        kp.sharedMemBytes = 0; kp.kernelParams = args; kp.extra = nullptr;
        return kp;
    };
    cudaGraphNode_t pro;
    cudaKernelNodeParams kp = kparams((void*)k_fire_prologue, 1, 32);
    RF_CUDA(cudaGraphAddKernelNode(&pro, g, nullptr, 0, &kp));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = c.h_loop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    RF_CUDA(cudaGraphAddNode(&wnode, g, &pro, 1, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = c.h_rebuild;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    RF_CUDA(cudaGraphAddNode(&inode, body, nullptr, 0, &ip));
    cudaGraph_t rb = ip.conditional.phGraph_out[0];
    const unsigned gN = (c.N + 255) / 256;
    const unsigned gC = (c.cg_cells + 1 + 255) / 256;
    struct { void* fn; unsigned grid, block; } seq[] = {
        {(void*)k_rb_zero, gC, 256},      {(void*)k_rb_bin, gN, 256},
        {(void*)k_rb_scan_sums, e->cg_nb, 1024}, {(void*)k_rb_scan_totals, 1, 32},
        {(void*)k_rb_scan_apply, e->cg_nb, 1024}, {(void*)k_rb_scatter, gN, 256},
        {(void*)k_rb_cand, (c.N + 127) / 128, 128},
    };
    cudaGraphNode_t prev = nullptr;
    for (auto& q : seq) {
        cudaGraphNode_t n;
        kp = kparams(q.fn, q.grid, q.block);
        RF_CUDA(cudaGraphAddKernelNode(&n, rb, prev ? &prev : nullptr, prev ? 1 : 0, &kp));
        prev = n;
    }
    cudaGraphNode_t fnode, unode;
    void* ff = (e->task.kind == RF_TEST_BRAZIL) ? (void*)k_step_ext<RF_TEST_BRAZIL, 1> : (void*)k_step_ext<RF_TEST_UNIAXIAL, 1>;
    kp = kparams(ff, e->nblocks, 128);
    kp.sharedMemBytes = step_smem(e);
    RF_CUDA(cudaGraphAddKernelNode(&fnode, body, &inode, 1, &kp));
    kp = kparams((void*)k_fire_update, e->nblocks, 128);
    RF_CUDA(cudaGraphAddKernelNode(&unode, body, &fnode, 1, &kp));
    RF_CUDA(cudaGraphInstantiate(&e->fexec, g, 0));
    return RF_OK;
}

// The FIRE loop on a plain stream (no conditional graph nodes): chunks of iterations,
// each kernel returning early once the device has stopped the loop.
rf_status launch_stream_fire(rf_engine* e, uint64_t max_iter) {
    Dev d = e->d;
    Consts c = e->cf;
    c.use_graph = 0;
    const unsigned gN = (c.N + 255) / 256, gC = (c.cg_cells + 1 + 255) / 256;
    cudaStream_t s = e->stream;
    void* ff = (e->task.kind == RF_TEST_BRAZIL) ? (void*)k_step_ext<RF_TEST_BRAZIL, 1> : (void*)k_step_ext<RF_TEST_UNIAXIAL, 1>;
    void* args[] = {&d, &c};
    for (uint64_t q = 0; q < max_iter + 1;) {
        for (int u = 0; u < 32; ++u, ++q) {
            k_rb_zero<<<gC, 256, 0, s>>>(d, c);
            k_rb_bin<<<gN, 256, 0, s>>>(d, c);
            k_rb_scan_sums<<<e->cg_nb, 1024, 0, s>>>(d, c);
            k_rb_scan_totals<<<1, 32, 0, s>>>(d, c);
            k_rb_scan_apply<<<e->cg_nb, 1024, 0, s>>>(d, c);
            k_rb_scatter<<<gN, 256, 0, s>>>(d, c);
            k_rb_cand<<<(c.N + 127) / 128, 128, 0, s>>>(d, c);
            RF_CUDA(cudaLaunchKernel(ff, dim3(e->nblocks), dim3(128), args, step_smem(e), s));
            k_fire_update<<<e->nblocks, 128, 0, s>>>(d, c);
        }
        RF_CHECK_LAUNCH("engine stream FIRE");
        uint32_t stop = 0;
        RF_CUDA(cudaMemcpyAsync(&stop, &e->d.sc->fstop, sizeof(stop), cudaMemcpyDeviceToHost, s));
        RF_CUDA(cudaStreamSynchronize(s));
        if (stop) break;
    }
    return RF_OK;
}

rf_status launch_stream_steps(rf_engine* e, uint64_t nsteps) {
    Dev d = e->d;
    Consts c = e->c;
    c.use_graph = 0;
    const unsigned gN = (c.N + 255) / 256, gC = (c.cg_cells + 1 + 255) / 256;
    cudaStream_t s = e->stream;
    for (uint64_t q = 0; q < nsteps; ++q) {
        k_stream_gate<<<1, 32, 0, s>>>(d);
        k_rb_zero<<<gC, 256, 0, s>>>(d, c);
        k_rb_bin<<<gN, 256, 0, s>>>(d, c);
        k_rb_scan_sums<<<e->cg_nb, 1024, 0, s>>>(d, c);
        k_rb_scan_totals<<<1, 32, 0, s>>>(d, c);
        k_rb_scan_apply<<<e->cg_nb, 1024, 0, s>>>(d, c);
        k_rb_scatter<<<gN, 256, 0, s>>>(d, c);
        k_rb_cand<<<(c.N + 127) / 128, 128, 0, s>>>(d, c);
        void* sargs[] = {&d, &c};
        if (cudaLaunchKernel(step_kernel(e), dim3(e->nblocks), dim3(128), sargs, step_smem(e), s) != cudaSuccess) break;
        k_stream_ungate<<<1, 32, 0, s>>>(d);
    }
    RF_CHECK_LAUNCH("engine stream steps");
    return RF_OK;
}

}  // namespace

// Host-side helpers from the md_* layer.
extern "C" size_t md_CellDistributionScratchBytes(uint_fast32_t N, uint_fast32_t CN);

namespace {

// Host description of a batch: per-specimen tasks (shifted, with the batch's grid), bond
// parameters and particle ranges.
struct BatchIn {
    std::vector<rf_task> tasks;
    std::vector<rf_ext_params> xs;
    std::vector<uint32_t> p0, n;
    std::vector<double> xoff;
};

// post-peak stop rule of an extended-model specimen: the stress fraction of the peak below
// which it counts as fractured (0: the reference's ZeroStress rule alone)
double keep_fraction(const rf_ext_params& x) { return x.post_peak_drop > 0.0 ? 1.0 - x.post_peak_drop : 0.0; }

void fill_scalars(DevScalars& h, const rf_task& t) {
    std::memset(&h, 0, sizeof(h));
    const rf_compression& K_ = t.Compress;
    h.V = K_.V; h.VLoad = K_.VLoad; h.Top = K_.Top; h.Bottom = K_.Bottom; h.TopR = K_.TopR; h.BottomR = K_.BottomR;
    h.FractureStress = K_.FractureStress; h.FractureStrain = K_.FractureStrain; h.MinStress = K_.MinStress;
    h.ZeroStress = K_.ZeroStress; h.Stress = K_.Stress; h.Strain = K_.Strain; h.MaxStrain = K_.MaxStrain;
    h.Size0 = K_.Size0;
    h.size_d[0] = K_.size_d.x; h.size_d[1] = K_.size_d.y; h.size_d[2] = K_.size_d.z;
    h.center_d[0] = K_.center_d.x; h.center_d[1] = K_.center_d.y; h.center_d[2] = K_.center_d.z;
    h.sz0 = t.sz0 != 0.0 ? t.sz0 : (double)K_.size.z;
    h.center[0] = K_.center.x; h.center[1] = K_.center.y; h.center[2] = K_.center.z;
    h.size[0] = K_.size.x; h.size[1] = K_.size.y; h.size[2] = K_.size.z;
    h.sized2[0] = K_.sized2.x; h.sized2[1] = K_.sized2.y; h.sized2[2] = K_.sized2.z;
    h.RR = K_.RR; h._1d_Area = K_._1d_Area; h.Hd2 = K_.Hd2;
    h.Loading = K_.Loading; h.Fracture = K_.Fracture;
    h.done = (K_.Strain < K_.MaxStrain && !K_.Fracture) ? 0u : 1u;
}

// Rows given in the reference layout (a restored checkpoint) instead of built from the
// positions: the engine sizes its bond records for them.
struct RowsIn {
    const uint_fast32_t* IL;
    const uint8_t* ILtype;
    const float* iL;
    const rf_float3 *Rij, *Oijt, *Mijn, *Mijt;
};

rf_status engine_create_impl(const rf_task* t, const float* h_R, const double* h_Rd, const double* h_rad,
                             const rf_ext_params* x, rf_engine** out, const BatchIn* bin = nullptr,
                             const RowsIn* rows = nullptr) {
    const bool ext = x != nullptr;
    if (!t || !out || t->N == 0 || t->K == 0 || (ext ? (!h_Rd || !h_rad) : !h_R)) {
        set_error("rf_engine_create: bad arguments");
        return RF_ERR_INVALID;
    }
    double rmax = 0.0, rmin = 1e300;
    if (ext) {
        for (uint64_t i = 0; i < t->N; ++i) { rmax = std::max(rmax, h_rad[i]); rmin = std::min(rmin, h_rad[i]); }
        if (x->ref_mode != 0 && x->ref_mode != 1) { set_error("rf_engine_create_ext: ref_mode must be 0 or 1"); return RF_ERR_INVALID; }
        if (x->ref_mode) {
            if (rmin != t->Po.p_r || rmax != t->Po.p_r) {
                set_error("rf_engine_create_ext: ref_mode needs every radius equal to Po.p_r (%g)", t->Po.p_r);
                return RF_ERR_INVALID;
            }
        } else if (!(x->kn > 0.0) || !(x->ks >= 0.0) || !(x->bond_lambda > 0.0) || !(x->weibull_m > 0.0) ||
                   !(x->sigma_c > 0.0) || !(x->tau_c > 0.0)) {
            set_error("rf_engine_create_ext: radii and bond parameters must be positive");
            return RF_ERR_INVALID;
        }
        if (!(rmin > 0.0) || !(x->post_peak_drop >= 0.0 && x->post_peak_drop < 1.0) ||
            !(x->list_gap >= 0.0 && x->list_gap < 1e300)) {
            set_error("rf_engine_create_ext: radii must be positive, post_peak_drop in [0, 1), list_gap >= 0");
            return RF_ERR_INVALID;
        }
        if (!(2.0 * rmax < std::sqrt(t->Po.aa_farcut))) {
            set_error("rf_engine_create_ext: a_farcut (%g) must exceed the largest contact distance 2*r_max (%g)",
                      std::sqrt(t->Po.aa_farcut), 2.0 * rmax);
            return RF_ERR_INVALID;
        }
    }
    if (t->K > 32) { set_error("rf_engine_create: the engine keeps slot masks in 32 bits (K <= 32), got K=%u", t->K); return RF_ERR_INVALID; }
    if (t->N >= 0xFFFFFFFFull) { set_error("rf_engine_create: N too large"); return RF_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("rf_engine_create: no CUDA device"); return RF_ERR_NO_DEVICE; }
    rf_engine* e = new rf_engine();
    std::memset(&e->d, 0, sizeof(e->d));
    std::memset(&e->c, 0, sizeof(e->c));
    e->task = *t;
    e->graph = nullptr; e->exec = nullptr; e->graph_ok = false; e->staging = nullptr; e->bonds_initial = 0;
    e->stream = nullptr; e->counters_dev = nullptr; e->maxq_dev = nullptr;
    e->fgraph = nullptr; e->fexec = nullptr; e->fire_ready = false;
    cudaGetDevice(&e->device);
    rf_status st = RF_OK;
    auto fail = [&](rf_status s) { rf_engine_destroy(e); return s; };
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(RF_ERR_CUDA);

    const uint32_t N = (uint32_t)t->N, K = t->K;
    Consts& c = e->c;
    c.N = N; c.K = K; c.KC = 64; c.kind = t->kind;
    const rf_potential& P = t->Po;
    c.dt_d = P.dt; c.p_r_d = P.p_r;
    c.bp = BondParams{(float)P.dt, (float)P.m_E, (float)P.m_G, (float)P.b_r, (float)P.m_Ec, (float)P.m_Gc};
    c.cp = ContactParams{(float)P.dt, (float)P.hm_E, (float)P.hm_G, (float)P.p_A, (float)P.p_mu, (float)P.p_mur,
                         (float)P.p_m, (float)P.p_r};
    c.dtm = (float)P.dt_d_m; c.dt = (float)P.dt; c.dtI = (float)P.dt_d_I;
    if (ext) {
        c.ext = 1;
        c.ep = ExtParams{(float)P.dt, (float)P.hm_E, (float)P.hm_G, (float)P.p_A, (float)P.p_mu, (float)P.p_mur};
        c.kn = (float)x->kn; c.ks = (float)x->ks; c.br_lambda = (float)x->bond_lambda;
        c.cmass = (float)(P.p_m / (P.p_r * P.p_r * P.p_r));     // mass = density * 4/3 pi r^3
        c.aa_farcut_d = P.aa_farcut; c.aacut_d = (double)t->aacut;
        c.a_farcut_d = P.a_farcut;
        c.lgap_d = x->list_gap;
        c.lgap_f = (float)x->list_gap;
        c.ref_mode = x->ref_mode;
        c.refE = (float)P.m_E; c.refG = (float)P.m_G; c.ref_br = (float)P.b_r;
    }
    c.aacut = t->aacut; c.aa_farcut = (float)P.aa_farcut;
    c.g.a = t->C.a; c.g.inv_a = t->C._1d_a; c.g.nx = t->C.Nr.x; c.g.ny = t->C.Nr.y; c.g.nz = t->C.Nr.z; c.g.CN = t->C.N;
    c.zcut = (t->kind == RF_TEST_BRAZIL) ? (float)((double)t->S.center.y + (double)t->S.spacesized2.y)
                                         : (float)((double)t->S.center.z + (double)t->S.spacesized2.z);
    c.box_c = t->S.center; c.box_h = t->S.spacesized2; c.hp = t->S.hidenpoint;
    // candidate grid over the cut box, one cell of margin each side; cell >= rc
    const double acut = std::sqrt((double)t->aacut);
    const double skin = 0.1 * acut;
    const double rc = acut + skin;
    c.rc2 = (float)(rc * rc);
    c.disp2 = (float)((0.3 * skin) * (0.3 * skin));   // checked every RF_GRAPH_UNROLL steps
    c.hard2 = (float)((0.5 * skin) * (0.5 * skin));
    c.acut_f = (float)acut;
    c.skin_f = (float)skin;
    const double hcell = rc * 1.0001;
    c.cg_inv_h = (float)(1.0 / hcell);
    c.cg_ox = (float)(t->S.center.x - t->S.spacesized2.x - hcell);
    c.cg_oy = (float)(t->S.center.y - t->S.spacesized2.y - hcell);
    c.cg_oz = (float)(t->S.center.z - t->S.spacesized2.z - hcell);
    c.cg_nx = (uint32_t)std::ceil((2.0 * t->S.spacesized2.x + 2 * hcell) / hcell) + 1;
    c.cg_ny = (uint32_t)std::ceil((2.0 * t->S.spacesized2.y + 2 * hcell) / hcell) + 1;
    c.cg_nz = (uint32_t)std::ceil((2.0 * t->S.spacesized2.z + 2 * hcell) / hcell) + 1;
    const uint64_t cells = (uint64_t)c.cg_nx * c.cg_ny * c.cg_nz;
    if (cells >= 0x7FFFFFFFull) { set_error("rf_engine_create: candidate grid too large"); return fail(RF_ERR_INVALID); }
    c.cg_cells = (uint32_t)cells;
    e->cg_nb = (uint32_t)((cells + 1 + 4095) / 4096);
    const uint32_t nspec = bin ? (uint32_t)bin->tasks.size() : 1u;
    c.curve_cap = nspec == 1 ? (1u << 20) : std::max(4096u, (1u << 20) / nspec);   // records per specimen
    e->nblocks = (N + 127) / 128;

    Dev& d = e->d;
    d.n_particles = N;
    const size_t NK = (size_t)N * K;
    for (int b = 0; b < 2; ++b) {
        if ((ext ? (st = dalloc(e, &d.posd[b], N)) : (st = dalloc(e, &d.pos[b], N))) ||
            (st = dalloc(e, &d.vel[b], N)) || (st = dalloc(e, &d.ang[b], N)))
            return fail(st);
    }
    if ((st = dalloc(e, &d.ids, NK)) || (st = dalloc(e, &d.il, NK)) || (st = dalloc(e, &d.cO[0], 3 * NK)) || (st = dalloc(e, &d.cO[1], 3 * NK)) ||
        (st = dalloc(e, &d.live, N)) || (st = dalloc(e, &d.bond, N)) || (st = dalloc(e, &d.cmask, N)) ||
        (st = dalloc(e, &d.nbq, N)) || (st = dalloc(e, &d.bmask, N)) || (st = dalloc(e, &e->maxq_dev, 1)) ||
        (st = dalloc(e, &d.cand, (size_t)c.KC * N)) || (st = dalloc(e, &d.cand_n, N)) || (st = dalloc(e, &d.member, N)) ||
        (st = dalloc(e, &d.pos_ref, N)) || (st = dalloc(e, &d.cmargin, N)) || (st = dalloc(e, &d.cbound, N)) || (st = dalloc(e, &d.cg_key, N)) || (st = dalloc(e, &d.cg_count, cells + 1)) ||
        (st = dalloc(e, &d.cg_start, cells + 1)) || (st = dalloc(e, &d.cg_fill, cells + 1)) ||
        (st = dalloc(e, &d.cg_bsum, e->cg_nb)) || (st = dalloc(e, &d.cg_sorted, N)) ||
        (st = dalloc(e, &d.partial, e->nblocks)) || (st = dalloc(e, &d.partial2, e->nblocks)) ||
        (st = dalloc(e, &d.curve, 3 * (size_t)c.curve_cap * nspec)) ||
        (st = dalloc(e, &d.sc, 1)) || (st = dalloc(e, &e->counters_dev, 4)))
        return fail(st);
    cudaStream_t s = e->stream;
    for (int b = 0; b < 2; ++b) {
        if (cudaMemsetAsync(d.vel[b], 0, N * sizeof(float4), s) || cudaMemsetAsync(d.ang[b], 0, N * sizeof(float4), s))
            return fail(cuda_status(cudaGetLastError(), "memset"));
    }
    // specimens: geometry, CTA -> specimen map, per-specimen scalars
    d.nspec = nspec;
    {
        std::vector<SpecGeom> hg(nspec);
        for (uint32_t q = 0; q < nspec; ++q) {
            const rf_task& ts = bin ? bin->tasks[q] : *t;
            SpecGeom& G = hg[q];
            G.zcut = (t->kind == RF_TEST_BRAZIL) ? (float)((double)ts.S.center.y + (double)ts.S.spacesized2.y)
                                                 : (float)((double)ts.S.center.z + (double)ts.S.spacesized2.z);
            G.box_c = ts.S.center; G.box_h = ts.S.spacesized2; G.hp = ts.S.hidenpoint;
            G.p0 = bin ? bin->p0[q] : 0u;
            G.p1 = bin ? bin->p0[q] + bin->n[q] : N;
            G.b0 = G.p0 / 128; G.b1 = (G.p1 - 1) / 128;
        }
        SpecGeom* dg = nullptr;
        if ((st = dalloc(e, &dg, nspec))) return fail(st);
        if (cudaMemcpyAsync(dg, hg.data(), nspec * sizeof(SpecGeom), cudaMemcpyHostToDevice, s)) return fail(RF_ERR_CUDA);
        d.geom = dg;
        d.blk_spec = nullptr;
        if (nspec > 1) {
            std::vector<uint16_t> hb(e->nblocks);
            uint32_t q = 0;
            for (uint32_t b = 0; b < e->nblocks; ++b) {
                while (q + 1 < nspec && hg[q].p1 <= b * 128u) ++q;
                hb[b] = (uint16_t)q;
            }
            uint16_t* db = nullptr;
            if ((st = dalloc(e, &db, e->nblocks))) return fail(st);
            if (cudaMemcpyAsync(db, hb.data(), e->nblocks * sizeof(uint16_t), cudaMemcpyHostToDevice, s))
                return fail(RF_ERR_CUDA);
            d.blk_spec = db;
            if ((st = dalloc(e, &d.spec, nspec))) return fail(st);
            std::vector<DevScalars> hs(nspec);
            for (uint32_t k = 0; k < nspec; ++k) {
                fill_scalars(hs[k], bin->tasks[k]);
                hs[k].keep_frac = keep_fraction(bin->xs[k]);
            }
            if (cudaMemcpyAsync(d.spec, hs.data(), nspec * sizeof(DevScalars), cudaMemcpyHostToDevice, s))
                return fail(RF_ERR_CUDA);
            e->spec_tasks = bin->tasks;
            e->spec_p0 = bin->p0;
            e->spec_n = bin->n;
            e->spec_xoff = bin->xoff;
        } else {
            d.spec = d.sc;
        }
    }
    // the scalar block is read (step parity) by the row import below: start it at zero
    if (cudaMemsetAsync(d.member, 0, N * sizeof(unsigned long long), s) || cudaMemsetAsync(d.cand_n, 0, N * 4, s) ||
        cudaMemsetAsync(d.cmargin, 0, N * sizeof(float), s) ||
        cudaMemsetAsync(d.sc, 0, sizeof(DevScalars), s))
        return fail(RF_ERR_CUDA);

    // Initial rows exactly as the drivers build them (md_calculationbraziltest.cu:132-144),
    // with the md_* kernels on temporary reference-layout buffers.
    {
        float *dR = nullptr, *dV = nullptr, *dIL_f = nullptr;
        uint_fast32_t *dCI = nullptr, *dCIs = nullptr, *dpnC = nullptr, *dIL = nullptr;
        uint8_t* dT = nullptr;
        rf_float3* dS = nullptr;
        double *dRd = nullptr, *dRad = nullptr, *dL0 = nullptr;
        float2* dStr = nullptr;
        void* scratch = nullptr;
        const size_t sb = md_CellDistributionScratchBytes(N, t->C.N);
        cudaError_t ce = cudaSuccess;
        ce = cudaMalloc(&dR, 3 * (size_t)N * sizeof(float));
        if (!ce) ce = cudaMalloc(&dV, 3 * (size_t)N * sizeof(float));
        if (!ce) ce = cudaMalloc(&dCI, N * sizeof(uint_fast32_t));
        if (!ce) ce = cudaMalloc(&dCIs, 2 * (size_t)N * sizeof(uint_fast32_t));
        if (!ce) ce = cudaMalloc(&dpnC, 2 * t->C.N * sizeof(uint_fast32_t));
        if (!ce) ce = cudaMalloc(&dIL, NK * sizeof(uint_fast32_t));
        if (!ce) ce = cudaMalloc(&dT, NK);
        if (!ce) ce = cudaMalloc(&dIL_f, NK * sizeof(float));
        if (!ce) ce = cudaMalloc(&dS, 7 * NK * sizeof(rf_float3));
        if (!ce) ce = cudaMalloc(&scratch, sb);
        if (ext) {
            if (!ce) ce = cudaMalloc(&dRd, 3 * (size_t)N * sizeof(double));
            if (!ce) ce = cudaMalloc(&dRad, (size_t)N * sizeof(double));
            if (!ce) ce = cudaMalloc(&dL0, NK * sizeof(double));
            if (!ce) ce = cudaMalloc(&dStr, NK * sizeof(float2));
            if (!ce) ce = cudaMemcpyAsync(dRd, h_Rd, 3 * (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s);
            if (!ce) ce = cudaMemcpyAsync(dRad, h_rad, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s);
            if (!ce) { k_posd_from_planar<<<(N + 255) / 256, 256, 0, s>>>(dRd, dRad, N, d.posd[0], dR); ce = cudaGetLastError(); }
        } else if (!ce) {
            ce = cudaMemcpyAsync(dR, h_R, 3 * (size_t)N * sizeof(float), cudaMemcpyHostToDevice, s);
        }
        if (!ce) ce = cudaMemsetAsync(dV, 0, 3 * (size_t)N * sizeof(float), s);
        if (!ce) ce = cudaMemsetAsync(dT, 0, NK, s);
        if (!ce) ce = cudaMemsetAsync(dIL_f, 0, NK * sizeof(float), s);
        if (!ce) ce = cudaMemsetAsync(dS, 0, 7 * NK * sizeof(rf_float3), s);
        rf_status st2 = ce ? cuda_status(ce, "engine init buffers") : RF_OK;
        rf_float3 *Rij = dS, *Oijt = dS + NK, *Fijn = dS + 2 * NK, *Fijt = dS + 3 * NK, *Mijn = dS + 4 * NK,
                  *Mijt = dS + 5 * NK, *Mijadd = dS + 6 * NK;
        rf_status init_dev = RF_OK;
        if (!st2) {
            rf_status a = md_CellDistribution(dR, N, dCI, dCIs, dpnC, t->C.N, t->C._1d_a, t->C.Nr, scratch, sb, s);
            if (a != RF_OK && a != RF_ERR_CELL_RANGE && a != RF_ERR_ROW_OVERFLOW) st2 = a; else if (a) init_dev = a;
        }
        const bool pair_cut = ext && x->list_gap > 0.0;
        if (!st2 && rows) {
            ce = cudaMemcpyAsync(dIL, rows->IL, NK * sizeof(uint_fast32_t), cudaMemcpyHostToDevice, s);
            if (!ce) ce = cudaMemcpyAsync(dT, rows->ILtype, NK, cudaMemcpyHostToDevice, s);
            if (!ce) ce = cudaMemcpyAsync(dIL_f, rows->iL, NK * sizeof(float), cudaMemcpyHostToDevice, s);
            const rf_float3* src[4] = {rows->Rij, rows->Oijt, rows->Mijn, rows->Mijt};
            rf_float3* dst[4] = {Rij, Oijt, Mijn, Mijt};
            for (int q = 0; q < 4 && !ce; ++q)
                ce = cudaMemcpyAsync(dst[q], src[q], NK * sizeof(rf_float3), cudaMemcpyHostToDevice, s);
            if (ce) st2 = cuda_status(ce, "engine rows");
        }
        if (!st2 && !pair_cut && !rows) {
            rf_status a = md_InteractionListConstruct(dR, N, dCIs, dpnC, dIL, K, t->C.a, t->C._1d_a, t->aacut,
                                                      t->C.Nr, t->C.N, s);
            if (a != RF_OK && a != RF_ERR_CELL_RANGE && a != RF_ERR_ROW_OVERFLOW) st2 = a; else if (a && !init_dev) init_dev = a;
        }
        if (!st2 && pair_cut) {
            uint32_t w = 0;
            ce = cudaMemsetAsync(dIL, 0xFF, NK * sizeof(uint_fast32_t), s);
            if (!ce) ce = cudaMemsetAsync(e->maxq_dev, 0, sizeof(uint32_t), s);
            if (!ce) {
                k_list_ext<<<(N + 127) / 128, 128, 0, s>>>(dR, d.posd[0], N, dCIs, dpnC, dIL, K, c.g, P.a_farcut,
                                                           x->list_gap, e->maxq_dev);
                ce = cudaGetLastError();
            }
            if (!ce) ce = cudaMemcpyAsync(&w, e->maxq_dev, sizeof(w), cudaMemcpyDeviceToHost, s);
            if (!ce) ce = cudaStreamSynchronize(s);
            if (ce) st2 = cuda_status(ce, "k_list_ext");
            else if (w && !init_dev) init_dev = (rf_status)w;
        }
        if (!st2 && !ext && !rows) st2 = md_ConstructBoundInteractions(dR, dV, dV, dIL, dT, dIL_f, Rij, Oijt, Fijn, Fijt, Mijn, Mijt,
                                                              Mijadd, N, K, (float)P.b_dd, (float)P.b_r, s);
        if (!st2 && ext) {
            std::vector<BondSpec> hbs(nspec);
            for (uint32_t q = 0; q < nspec; ++q) {
                const rf_ext_params& xq = bin ? bin->xs[q] : *x;
                const rf_task& tq = bin ? bin->tasks[q] : *t;
                hbs[q] = BondSpec{xq.gap_frac, xq.weibull_m, xq.sigma_c, xq.tau_c, xq.seed, bin ? bin->p0[q] : 0u,
                                  bin ? bin->p0[q] + bin->n[q] : N, xq.ref_mode, tq.Po.b_d};
                if (xq.ref_mode) { hbs[q].sig = tq.Po.m_Ec; hbs[q].tau = tq.Po.m_Gc; hbs[q].wm = 1.0; }
            }
            BondSpec* dbs = nullptr;
            ce = cudaMalloc(&dbs, nspec * sizeof(BondSpec));
            if (!ce) ce = cudaMemcpyAsync(dbs, hbs.data(), nspec * sizeof(BondSpec), cudaMemcpyHostToDevice, s);
            if (!ce) {
                k_bond_ext<<<(N + 127) / 128, 128, 0, s>>>(d.posd[0], dIL, dT, dIL_f, dL0, dStr, N, K, dbs, nspec);
                ce = cudaGetLastError();
            }
            if (!ce) ce = cudaStreamSynchronize(s);
            cudaFree(dbs);
            if (ce) st2 = cuda_status(ce, "k_bond_ext");
        }
        // (with a list gap every listed pair is within its cutoff: nothing to delete)
        if (!st2 && !pair_cut && !rows)
            st2 = md_DeleteFarLinks(dR, N, dIL, dT, dIL_f, Rij, Oijt, Fijn, Fijt, Mijn, Mijt, Mijadd, K,
                                    (float)P.aa_farcut, s);
        if (!st2) {
            // bond records: as many per particle as its row holds bonds (bonds are never created later)
            uint32_t qb = 0;
            ce = cudaMemsetAsync(e->maxq_dev, 0, sizeof(uint32_t), s);
            if (!ce) { k_count_records<<<148 * 4, 256, 0, s>>>(dIL, dT, Rij, N, K, e->maxq_dev); ce = cudaGetLastError(); }
            if (!ce) ce = cudaMemcpyAsync(&qb, e->maxq_dev, sizeof(qb), cudaMemcpyDeviceToHost, s);
            if (!ce) ce = cudaStreamSynchronize(s);
            if (ce) st2 = cuda_status(ce, "engine bond count");
            if (qb == 0) qb = 1;
            d.QB = qb;
            const size_t QN = (size_t)qb * N;
            if (!st2 && ((st2 = dalloc(e, &d.bj, QN)) || (st2 = dalloc(e, &d.bk, QN)) || (st2 = dalloc(e, &d.bil, QN)) ||
                         (st2 = dalloc(e, &d.bst, 3 * QN)))) {}
            if (!st2 && ext && ((st2 = dalloc(e, &d.bL0, QN)) || (st2 = dalloc(e, &d.bstr, QN)))) {}
        }
        if (!st2) {
            if (!ext) k_planar_to_f4<<<(N + 255) / 256, 256, 0, s>>>(dR, N, d.pos[0]);
            k_rows_import<<<(N + 127) / 128, 128, 0, s>>>(dIL, dT, dIL_f, Rij, Oijt, Mijn, Mijt, dL0, dStr, d, c);
            ce = cudaGetLastError();
            if (ce) st2 = cuda_status(ce, "engine import");
        }
        if (!st2) { ce = cudaStreamSynchronize(s); if (ce) st2 = cuda_status(ce, "engine init"); }
        cudaFree(dR); cudaFree(dV); cudaFree(dCI); cudaFree(dCIs); cudaFree(dpnC); cudaFree(dIL); cudaFree(dT);
        cudaFree(dIL_f); cudaFree(dS); cudaFree(scratch); cudaFree(dRd); cudaFree(dRad); cudaFree(dL0); cudaFree(dStr);
        if (st2) return fail(st2);
        st = init_dev;
    }

    // scalar state (with one specimen the global block is also the specimen's)
    DevScalars h;
    fill_scalars(h, *t);
    if (ext) h.keep_frac = keep_fraction(*x);
    if (nspec > 1) {
        h.done = 0;
        for (uint32_t q = 0; q < nspec; ++q) {
            const rf_compression& Kq = bin->tasks[q].Compress;
            if (Kq.Strain < Kq.MaxStrain && !Kq.Fracture) break;
            if (q + 1 == nspec) h.done = 1;
        }
    }
    h.rebuild = 1;
    h.err = (uint32_t)st;
    if (cudaMemcpyAsync(d.sc, &h, sizeof(h), cudaMemcpyHostToDevice, s) || cudaStreamSynchronize(s))
        return fail(RF_ERR_CUDA);

    {
        uint64_t cnt[5];
        if (rf_engine_counters(e, cnt, 5) == RF_OK) e->bonds_initial = cnt[2];
    }
    // graph with device-driven loop; fall back to plain stream launches if unavailable
    if (!getenv("RF_ENGINE_NO_GRAPH")) {
        rf_status gs = build_graph(e);
        if (gs == RF_OK) e->graph_ok = true;
        else { cudaGetLastError(); e->c.use_graph = 0; }
    }
    *out = e;
    return RF_OK;
}

}  // namespace

extern "C" {

rf_status rf_engine_create(const rf_task* t, const float* h_R, rf_engine** out) {
    return engine_create_impl(t, h_R, nullptr, nullptr, nullptr, out);
}

rf_status rf_engine_create_ext(const rf_task* t, const rf_ext_params* x, const double* h_R, const double* h_radius,
                               rf_engine** out) {
    if (!x) { set_error("rf_engine_create_ext: null parameters"); return RF_ERR_INVALID; }
    return engine_create_impl(t, nullptr, h_R, h_radius, x, out);
}

rf_status rf_engine_create_batch(const rf_task* tasks, const rf_ext_params* xs, const double* const* h_R,
                                 const double* const* h_radius, int nspec, rf_engine** out) {
    if (!tasks || !xs || !h_R || !h_radius || !out || nspec < 1 || nspec > 65535) {
        set_error("rf_engine_create_batch: bad arguments");
        return RF_ERR_INVALID;
    }
    const rf_task& t0 = tasks[0];
    uint64_t total = 0;
    for (int q = 0; q < nspec; ++q) {
        const rf_task& tq = tasks[q];
        if (!h_R[q] || !h_radius[q] || tq.N < 128 || tq.kind != t0.kind || tq.K != t0.K || tq.C.a != t0.C.a ||
            tq.aacut != t0.aacut || tq.Po.dt != t0.Po.dt || tq.Po.p_r != t0.Po.p_r ||
            tq.Po.aa_farcut != t0.Po.aa_farcut || tq.Po.hm_E != t0.Po.hm_E || tq.Po.hm_G != t0.Po.hm_G ||
            tq.Po.p_A != t0.Po.p_A || tq.Po.p_mu != t0.Po.p_mu || tq.Po.p_mur != t0.Po.p_mur ||
            tq.Po.p_m != t0.Po.p_m || xs[q].kn != xs[0].kn || xs[q].ks != xs[0].ks ||
            xs[q].bond_lambda != xs[0].bond_lambda || xs[q].list_gap != xs[0].list_gap ||
            xs[q].ref_mode != xs[0].ref_mode ||
            (xs[0].ref_mode && (tq.Po.m_E != t0.Po.m_E || tq.Po.m_G != t0.Po.m_G || tq.Po.b_r != t0.Po.b_r)) ||
            !(xs[q].post_peak_drop >= 0.0 && xs[q].post_peak_drop < 1.0)) {
            set_error("rf_engine_create_batch: specimen %d must have >= 128 particles and the batch's test kind, "
                      "slots, grid cell, material, time step, bond stiffness and list gap, and a post-peak drop in [0, 1)", q);
            return RF_ERR_INVALID;
        }
        total += tq.N;
    }
    if (total >= 0xFFFFFFFFull) { set_error("rf_engine_create_batch: too many particles"); return RF_ERR_INVALID; }
    // lay the specimens out along x, each shifted by a whole number of cells so that its
    // cell-relative geometry (and so its insertion order) is what it would be alone,
    // with two cells between neighbouring boxes (no cross-specimen links)
    const double a = (double)t0.C.a;
    BatchIn bin;
    bin.tasks.resize(nspec); bin.xs.assign(xs, xs + nspec); bin.p0.resize(nspec); bin.n.resize(nspec);
    bin.xoff.resize(nspec);
    double cursor = 0.0, Bx = 0.0, By = 0.0, Bz = 0.0, lo_y = 1e300, lo_z = 1e300, hi_y = -1e300, hi_z = -1e300;
    uint32_t p = 0;
    for (int q = 0; q < nspec; ++q) {
        const rf_sample& S = tasks[q].S;
        const double lo = (double)S.center.x - (double)S.spacesized2.x, hi = (double)S.center.x + (double)S.spacesized2.x;
        const double off = q == 0 ? 0.0 : std::ceil((cursor - lo) / a) * a;
        bin.xoff[q] = off;
        cursor = hi + off + 2.0 * a;
        rf_task tq = tasks[q];
        tq.S.center.x = (float)((double)S.center.x + off);
        tq.S.A.x = (float)((double)S.A.x + off); tq.S.B.x = (float)((double)S.B.x + off);
        tq.S.hidenpoint.x = (float)((double)S.hidenpoint.x + off);
        tq.S.center_real.x += off; tq.S.A_real.x += off; tq.S.B_real.x += off;
        tq.Compress.center_d.x += off;
        tq.Compress.center.x = (float)tq.Compress.center_d.x;
        bin.tasks[q] = tq;
        bin.p0[q] = p; bin.n[q] = (uint32_t)tq.N;
        p += (uint32_t)tq.N;
        Bx = std::max(Bx, (double)tq.S.B.x); By = std::max(By, (double)S.B.y); Bz = std::max(Bz, (double)S.B.z);
        lo_y = std::min(lo_y, (double)S.center.y - (double)S.spacesized2.y);
        hi_y = std::max(hi_y, (double)S.center.y + (double)S.spacesized2.y);
        lo_z = std::min(lo_z, (double)S.center.z - (double)S.spacesized2.z);
        hi_z = std::max(hi_z, (double)S.center.z + (double)S.spacesized2.z);
    }
    // the batch's cell grid covers every box (cell_data::CalculateParameters on the union corner)
    rf_cells C = t0.C;
    C.Nr.x = (unsigned)(std::floor((float)(Bx * (double)C._1d_a)) + 1.0f);
    C.Nr.y = (unsigned)(std::floor((float)(By * (double)C._1d_a)) + 1.0f);
    C.Nr.z = (unsigned)(std::floor((float)(Bz * (double)C._1d_a)) + 3.0f);
    C.N = (uint64_t)C.Nr.x * C.Nr.y * C.Nr.z;
    for (int q = 0; q < nspec; ++q) bin.tasks[q].C = C;
    rf_task tc = bin.tasks[0];
    tc.N = total;
    tc.C = C;
    const double lo_x = (double)bin.tasks[0].S.center.x - (double)bin.tasks[0].S.spacesized2.x;
    const double hi_x = (double)bin.tasks[nspec - 1].S.center.x + (double)bin.tasks[nspec - 1].S.spacesized2.x;
    tc.S.center = rf_float3{(float)(0.5 * (lo_x + hi_x)), (float)(0.5 * (lo_y + hi_y)), (float)(0.5 * (lo_z + hi_z))};
    tc.S.spacesized2 = rf_float3{(float)(0.5 * (hi_x - lo_x)), (float)(0.5 * (hi_y - lo_y)), (float)(0.5 * (hi_z - lo_z))};
    tc.bloks = total / 1024 + 1;
    std::vector<double> R(3 * total), rad(total);
    for (int q = 0; q < nspec; ++q) {
        const uint64_t n = tasks[q].N, p0 = bin.p0[q];
        for (uint64_t i = 0; i < n; ++i) {
            R[p0 + i] = h_R[q][i] + bin.xoff[q];
            R[total + p0 + i] = h_R[q][n + i];
            R[2 * total + p0 + i] = h_R[q][2 * n + i];
            rad[p0 + i] = h_radius[q][i];
        }
    }
    return engine_create_impl(&tc, nullptr, R.data(), rad.data(), &xs[0], out, &bin);
}

rf_status rf_engine_positions_f64(rf_engine* e, double* R) {
    if (!e || !R) { set_error("rf_engine_positions_f64: bad arguments"); return RF_ERR_INVALID; }
    if (!e->c.ext) { set_error("rf_engine_positions_f64: engine keeps float positions"); return RF_ERR_STATE; }
    const uint32_t N = e->c.N;
    cudaStream_t s = e->stream;
    DevScalars h;
    RF_CUDA(cudaStreamSynchronize(s));
    RF_CUDA(cudaMemcpy(&h, e->d.sc, sizeof(h), cudaMemcpyDeviceToHost));
    double* tmp = nullptr;
    RF_CUDA(cudaMalloc(&tmp, 3 * (size_t)N * sizeof(double)));
    k_posd_to_planar<<<(N + 255) / 256, 256, 0, s>>>(e->d.posd[h.steps & 1ull], N, tmp);
    cudaError_t ce = cudaGetLastError();
    if (!ce) ce = cudaMemcpyAsync(R, tmp, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (!ce) ce = cudaStreamSynchronize(s);
    cudaFree(tmp);
    if (ce) return cuda_status(ce, "rf_engine_positions_f64");
    return RF_OK;
}

rf_status rf_relax_default_params(rf_relax_params* p, const rf_task* t) {
    if (!p || !t) { set_error("rf_relax_default_params: bad arguments"); return RF_ERR_INVALID; }
    std::memset(p, 0, sizeof(*p));
    p->strain_inc = 2.5e-5;
    p->tol = 1e-6;
    p->dt0 = 0.1;
    p->dt_max = 1.0;
    p->dt_min = 1e-3;
    p->alpha0 = 0.1;
    p->f_inc = 1.1;
    p->f_dec = 0.5;
    p->f_alpha = 0.99;
    p->n_delay = 5;
    p->max_iter = 200000;
    return RF_OK;
}

}  // extern "C"

namespace {
rf_status fire_setup(rf_engine* e) {
    if (e->fire_ready) return RF_OK;
    Dev& d = e->d;
    const uint32_t N = e->c.N;
    rf_status st;
    if ((st = dalloc(e, &d.frc, N)) || (st = dalloc(e, &d.mom, N)) ||
        (st = dalloc(e, &d.fpart, (size_t)e->nblocks * FIRE_SUMS)) || (st = dalloc(e, &d.rot, N)) ||
        (d.nspec > 1 && (st = dalloc(e, &d.fpart2, (size_t)e->nblocks * FIRE_SUMS))) ||
        (st = dalloc(e, &d.x0, N)) || (st = dalloc(e, &d.bst0, 3 * (size_t)d.QB * N)))
        return st;
    e->cf = e->c;
    if (!getenv("RF_ENGINE_NO_GRAPH")) {
        if (build_fire_graph(e) != RF_OK) { cudaGetLastError(); e->cf.use_graph = 0; }
    } else {
        e->cf.use_graph = 0;
    }
    k_fire_buffers_init<<<(N + 255) / 256, 256, 0, e->stream>>>(d, e->cf);
    RF_CHECK_LAUNCH("k_fire_buffers_init");
    e->fire_ready = true;
    return RF_OK;
}

// One quasi-static load increment of every specimen of the engine (a batch relaxes its
// specimens together, each on its own FIRE scalars, and a specimen whose relaxation
// stopped stays put until the others stop). r: one result per specimen.
rf_status load_increment(rf_engine* e, const rf_relax_params* p, const float* warm, int ldw, int scaled,
                         rf_relax_result* r) {
    if (!e || !p) { set_error("rf_engine_load_increment: bad arguments"); return RF_ERR_INVALID; }
    if (!e->c.ext) { set_error("rf_engine_load_increment: quasi-static relaxation needs the extended model"); return RF_ERR_STATE; }
    if (e->c.ref_mode) { set_error("rf_engine_load_increment: the reference-constants mode runs explicit steps only"); return RF_ERR_STATE; }
    if (!(p->dt0 > 0) || !(p->dt_max >= p->dt0) || !(p->dt_min > 0) || !(p->dt_min <= p->dt0) || !(p->tol > 0) ||
        p->max_iter == 0 || !(p->alpha0 >= 0 && p->alpha0 < 1) || !(p->f_inc >= 1) || !(p->f_dec > 0 && p->f_dec < 1) ||
        !(p->strain_inc > 0)) {
        set_error("rf_engine_load_increment: bad FIRE parameters");
        return RF_ERR_INVALID;
    }
    cudaStream_t s = e->stream;
    Dev& d = e->d;
    const uint32_t N = e->c.N, ns = d.nspec;
    if (rf_status st = fire_setup(e)) return st;
    // FIRE constants into every specimen's scalar block (host read-modify-write, stream ordered)
    std::vector<DevScalars> hs(ns);
    RF_CUDA(cudaMemcpyAsync(hs.data(), d.spec, ns * sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaStreamSynchronize(s));
    for (DevScalars& h : hs) {
        h.fdt0 = p->dt0; h.fdtmax = p->dt_max; h.fdtmin = p->dt_min; h.falpha0 = p->alpha0; h.finc = p->f_inc;
        h.fdec = p->f_dec; h.fshrink = p->f_alpha; h.fndelay = p->n_delay; h.ftol = p->tol; h.fmax_iter = p->max_iter;
    }
    RF_CUDA(cudaMemcpyAsync(d.spec, hs.data(), ns * sizeof(DevScalars), cudaMemcpyHostToDevice, s));
    // the bond records' state at the start of the increment (FIRE mode computes from it)
    RF_CUDA(cudaMemcpyAsync(d.bst0, d.bst, 3 * (size_t)d.QB * N * sizeof(float4), cudaMemcpyDeviceToDevice, s));
    const unsigned nb = (N + 127) / 128;
    if (e->task.kind == RF_TEST_BRAZIL) {
        k_qs_begin_scalars<RF_TEST_BRAZIL><<<1, 32, 0, s>>>(d, e->cf, p->strain_inc);
        k_qs_begin<RF_TEST_BRAZIL><<<nb, 128, 0, s>>>(d, e->cf, warm, ldw, scaled, p->strain_inc);
    } else {
        k_qs_begin_scalars<RF_TEST_UNIAXIAL><<<1, 32, 0, s>>>(d, e->cf, p->strain_inc);
        k_qs_begin<RF_TEST_UNIAXIAL><<<nb, 128, 0, s>>>(d, e->cf, warm, ldw, scaled, p->strain_inc);
    }
    RF_CHECK_LAUNCH("k_qs_begin");
    if (e->cf.use_graph) RF_CUDA(cudaGraphLaunch(e->fexec, s));
    else if (rf_status st = launch_stream_fire(e, p->max_iter)) return st;
    DevScalars g;
    RF_CUDA(cudaMemcpyAsync(hs.data(), d.spec, ns * sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaMemcpyAsync(&g, d.sc, sizeof(g), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaStreamSynchronize(s));
    if (r) {
        for (uint32_t k = 0; k < ns; ++k) {
            const DevScalars& h = hs[k];
            r[k].iterations = h.fiter;
            r[k].converged = (int32_t)h.fconverged;
            r[k].residual = h.fresidual;
            r[k].mean_force = h.fmean;
            r[k].stress = h.Stress;
            r[k].strain = h.Strain;
            r[k].broken_bonds = g.broken;         // (the engine's total)
            r[k].error = (rf_status)g.err;
        }
    }
    return RF_OK;
}

}  // namespace

extern "C" {

rf_status rf_engine_load_increment(rf_engine* e, const rf_relax_params* p, const float* warm, rf_relax_result* r) {
    if (e && e->d.nspec > 1) { set_error("rf_engine_load_increment: a batch takes rf_engine_load_increment_batch"); return RF_ERR_STATE; }
    return load_increment(e, p, warm, 6, 0, r);
}

rf_status rf_engine_load_increment_batch(rf_engine* e, const rf_relax_params* p, const float* warm, int ldw,
                                         int scaled, rf_relax_result* results) {
    if (warm && ldw < 6) { set_error("rf_engine_load_increment_batch: bad warm-start buffer"); return RF_ERR_INVALID; }
    return load_increment(e, p, warm, ldw, scaled ? 1 : 0, results);
}

rf_status rf_engine_load_increment_pred(rf_engine* e, const rf_relax_params* p, const float* pred, int ldp,
                                        rf_relax_result* r) {
    if (!pred || ldp < 6) { set_error("rf_engine_load_increment_pred: bad prediction buffer"); return RF_ERR_INVALID; }
    if (e && e->d.nspec > 1) { set_error("rf_engine_load_increment_pred: a batch takes rf_engine_load_increment_batch"); return RF_ERR_STATE; }
    return load_increment(e, p, pred, ldp, 1, r);
}

rf_status rf_engine_warm_features(rf_engine* e, double strain_inc, void* feat) {
    if (!e || !feat || !(strain_inc > 0)) { set_error("rf_engine_warm_features: bad arguments"); return RF_ERR_INVALID; }
    if (!e->c.ext) { set_error("rf_engine_warm_features: needs an extended-model engine"); return RF_ERR_STATE; }
    if (rf_status st = fire_setup(e)) return st;
    const uint32_t N = e->c.N, rows = (N + 127) / 128 * 128;
    cudaStream_t s = e->stream;
    if (rows > N) RF_CUDA(cudaMemsetAsync((__nv_bfloat16*)feat + (size_t)N * 64, 0, (size_t)(rows - N) * 64 * 2, s));
    if (e->task.kind == RF_TEST_BRAZIL)
        k_warm_features<RF_TEST_BRAZIL><<<(N + 127) / 128, 128, 0, s>>>(e->d, e->cf, strain_inc, (__nv_bfloat16*)feat);
    else
        k_warm_features<RF_TEST_UNIAXIAL><<<(N + 127) / 128, 128, 0, s>>>(e->d, e->cf, strain_inc, (__nv_bfloat16*)feat);
    RF_CHECK_LAUNCH("k_warm_features");
    return RF_OK;
}

rf_status rf_engine_warm_targets(rf_engine* e, double strain_inc, float* targets) {
    if (!e || !targets || !(strain_inc > 0)) { set_error("rf_engine_warm_targets: bad arguments"); return RF_ERR_INVALID; }
    if (!e->fire_ready) { set_error("rf_engine_warm_targets: no load increment run yet"); return RF_ERR_STATE; }
    cudaStream_t s = e->stream;
    k_warm_targets<<<(e->c.N + 127) / 128, 128, 0, s>>>(e->d, e->cf, strain_inc, targets);
    RF_CHECK_LAUNCH("k_warm_targets");
    return RF_OK;
}

rf_status rf_engine_increment_fields(rf_engine* e, double* x0, double* dx, double* rot) {
    if (!e || !e->fire_ready) { set_error("rf_engine_increment_fields: no load increment run yet"); return RF_ERR_STATE; }
    const uint32_t N = e->c.N;
    cudaStream_t s = e->stream;
    DevScalars h;
    RF_CUDA(cudaMemcpyAsync(&h, e->d.sc, sizeof(h), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaStreamSynchronize(s));
    std::vector<double4> a(N), b(N), c(N);
    RF_CUDA(cudaMemcpy(a.data(), e->d.x0, N * sizeof(double4), cudaMemcpyDeviceToHost));
    RF_CUDA(cudaMemcpy(b.data(), e->d.posd[h.steps & 1ull], N * sizeof(double4), cudaMemcpyDeviceToHost));
    RF_CUDA(cudaMemcpy(c.data(), e->d.rot, N * sizeof(double4), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < N; ++i) {
        if (x0) { x0[3 * i] = a[i].x; x0[3 * i + 1] = a[i].y; x0[3 * i + 2] = a[i].z; }
        if (dx) { dx[3 * i] = b[i].x - a[i].x; dx[3 * i + 1] = b[i].y - a[i].y; dx[3 * i + 2] = b[i].z - a[i].z; }
        if (rot) { rot[3 * i] = c[i].x; rot[3 * i + 1] = c[i].y; rot[3 * i + 2] = c[i].z; }
    }
    return RF_OK;
}

rf_status rf_engine_autotune(rf_engine* e, int steps, int* choice, float* ms_out) {
    if (!e || steps <= 0) { set_error("rf_engine_autotune: bad arguments"); return RF_ERR_INVALID; }
    if (!e->c.ext) {
        if (choice) *choice = RF_STEP_MIN_BLOCKS;
        return RF_OK;                                      // the reference-model step has one variant
    }
    cudaStream_t s = e->stream;
    RF_CUDA(cudaStreamSynchronize(s));
    // snapshot the whole device state: the trials advance it and are undone afterwards
    std::vector<void*> backup(e->allocs.size(), nullptr);
    auto release = [&]() { for (void* p : backup) if (p) cudaFree(p); };
    for (size_t q = 0; q < e->allocs.size(); ++q) {
        if (cudaMalloc(&backup[q], e->alloc_bytes[q]) != cudaSuccess) { release(); return cuda_status(cudaGetLastError(), "rf_engine_autotune"); }
        if (cudaMemcpyAsync(backup[q], e->allocs[q], e->alloc_bytes[q], cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
            release();
            return cuda_status(cudaGetLastError(), "rf_engine_autotune");
        }
    }
    auto restore = [&]() -> cudaError_t {
        for (size_t q = 0; q < e->allocs.size(); ++q) {
            cudaError_t ce = cudaMemcpyAsync(e->allocs[q], backup[q], e->alloc_bytes[q], cudaMemcpyDeviceToDevice, s);
            if (ce) return ce;
        }
        return cudaStreamSynchronize(s);
    };
    const int variants[3] = {8, 6, 5};
    float best = 1e30f;
    int pick = e->step_minb;
    float times[3] = {0, 0, 0};
    Dev d = e->d;
    Consts c = e->c;
    c.use_graph = 0;
    void* args[] = {&d, &c};
    cudaEvent_t a0, a1;
    cudaEventCreate(&a0); cudaEventCreate(&a1);
    cudaError_t ce = cudaSuccess;
    for (int v = 0; v < 3 && !ce; ++v) {
        void* fn = ext_step_variant(e->task.kind == RF_TEST_BRAZIL, variants[v]);
        for (int rep = 0; rep < 2 && !ce; ++rep) {             // first pass warms up
            ce = restore();
            // candidate lists from the current positions (the engine's first step would build them)
            const unsigned gN = (c.N + 255) / 256, gC = (c.cg_cells + 1 + 255) / 256;
            k_force_rebuild<<<1, 1, 0, s>>>(d.sc);
            k_rb_zero<<<gC, 256, 0, s>>>(d, c);
            k_rb_bin<<<gN, 256, 0, s>>>(d, c);
            k_rb_scan_sums<<<e->cg_nb, 1024, 0, s>>>(d, c);
            k_rb_scan_totals<<<1, 32, 0, s>>>(d, c);
            k_rb_scan_apply<<<e->cg_nb, 1024, 0, s>>>(d, c);
            k_rb_scatter<<<gN, 256, 0, s>>>(d, c);
            k_rb_cand<<<(c.N + 127) / 128, 128, 0, s>>>(d, c);
            k_set_target<<<1, 1, 0, s>>>(d.sc, (unsigned long long)steps);
            cudaEventRecord(a0, s);
            for (int q = 0; q < steps && !ce; ++q)
                ce = cudaLaunchKernel(fn, dim3(e->nblocks), dim3(128), args, step_smem(e), s);
            cudaEventRecord(a1, s);
            if (!ce) ce = cudaEventSynchronize(a1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a0, a1);
            times[v] = ms;
        }
        if (!ce && times[v] < best) { best = times[v]; pick = variants[v]; }
    }
    if (!ce) ce = restore();
    cudaEventDestroy(a0); cudaEventDestroy(a1);
    release();
    if (ce) return cuda_status(ce, "rf_engine_autotune");
    if (pick != e->step_minb) {
        e->step_minb = pick;
        if (e->graph_ok) {                                     // rebuild the step graph with the choice
            if (e->exec) cudaGraphExecDestroy(e->exec);
            if (e->graph) cudaGraphDestroy(e->graph);
            e->exec = nullptr; e->graph = nullptr; e->graph_ok = false;
            if (build_graph(e) == RF_OK) e->graph_ok = true;
            else { cudaGetLastError(); e->c.use_graph = 0; }
        }
    }
    if (choice) *choice = pick;
    if (ms_out) for (int v = 0; v < 3; ++v) ms_out[v] = times[v];
    return RF_OK;
}

rf_status rf_engine_destroy(rf_engine* e) {
    if (!e) return RF_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    if (e->fexec) cudaGraphExecDestroy(e->fexec);
    if (e->fgraph) cudaGraphDestroy(e->fgraph);
    for (void* p : e->allocs) cudaFree(p);
    if (e->staging) cudaFree(e->staging);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return RF_OK;
}

rf_status rf_engine_step(rf_engine* e, uint64_t nsteps) {
    if (!e) { set_error("rf_engine_step: null engine"); return RF_ERR_INVALID; }
    if (nsteps == 0) return RF_OK;
    k_set_target<<<1, 1, 0, e->stream>>>(e->d.sc, (unsigned long long)nsteps);
    RF_CHECK_LAUNCH("k_set_target");
    if (e->graph_ok) {
        RF_CUDA(cudaGraphLaunch(e->exec, e->stream));
        return RF_OK;
    }
    return launch_stream_steps(e, nsteps);
}

rf_status rf_engine_affine_strain(rf_engine* e, const double strain[3]) {
    if (!e || !strain) { set_error("rf_engine_affine_strain: bad arguments"); return RF_ERR_INVALID; }
    if (e->d.nspec > 1) { set_error("rf_engine_affine_strain: one specimen per engine"); return RF_ERR_STATE; }
    for (int a = 0; a < 3; ++a)
        if (!(strain[a] > -0.5 && strain[a] < 0.5)) {
            set_error("rf_engine_affine_strain: strain components must lie in (-0.5, 0.5)");
            return RF_ERR_INVALID;
        }
    cudaStream_t s = e->stream;
    const uint32_t N = e->c.N;
    k_affine_positions<<<(N + 255) / 256, 256, 0, s>>>(e->d, e->c, strain[0], strain[1], strain[2]);
    RF_CHECK_LAUNCH("k_affine_positions");
    if (e->c.kind == RF_TEST_BRAZIL) k_affine_scalars<RF_TEST_BRAZIL><<<1, 32, 0, s>>>(e->d, e->c, strain[0], strain[1], strain[2]);
    else k_affine_scalars<RF_TEST_UNIAXIAL><<<1, 32, 0, s>>>(e->d, e->c, strain[0], strain[1], strain[2]);
    RF_CHECK_LAUNCH("k_affine_scalars");
    return RF_OK;
}

rf_status rf_engine_step_host(rf_engine* e, const float* h_R_in, uint64_t nsteps, float* h_R_out) {
    if (!e) { set_error("rf_engine_step_host: null engine"); return RF_ERR_INVALID; }
    const uint32_t N = e->c.N;
    cudaStream_t s = e->stream;
    if (!e->staging) RF_CUDA(cudaMalloc(&e->staging, 3 * (size_t)N * sizeof(float)));
    if (h_R_in) {
        RF_CUDA(cudaMemcpyAsync(e->staging, h_R_in, 3 * (size_t)N * sizeof(float), cudaMemcpyHostToDevice, s));
        k_planar_to_cur<<<(N + 255) / 256, 256, 0, s>>>(e->staging, e->d);
        RF_CHECK_LAUNCH("k_planar_to_cur");
    }
    rf_status st = rf_engine_step(e, nsteps);
    if (st) return st;
    if (h_R_out) {
        k_cur_to_planar<<<(N + 255) / 256, 256, 0, s>>>(e->d, e->staging);
        RF_CHECK_LAUNCH("k_cur_to_planar");
        RF_CUDA(cudaMemcpyAsync(h_R_out, e->staging, 3 * (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, s));
        RF_CUDA(cudaStreamSynchronize(s));
    }
    return RF_OK;
}

rf_status rf_engine_sync_spec(rf_engine* e, int spec, rf_task* t_out, rf_run_result* r_out) {
    if (!e || spec < 0 || (uint32_t)spec >= e->d.nspec) { set_error("rf_engine_sync_spec: bad arguments"); return RF_ERR_INVALID; }
    DevScalars h, g;
    RF_CUDA(cudaMemcpyAsync(&h, e->d.spec + spec, sizeof(h), cudaMemcpyDeviceToHost, e->stream));
    RF_CUDA(cudaMemcpyAsync(&g, e->d.sc, sizeof(g), cudaMemcpyDeviceToHost, e->stream));
    RF_CUDA(cudaStreamSynchronize(e->stream));
    if (t_out) {
        *t_out = e->d.nspec > 1 ? e->spec_tasks[spec] : e->task;
        rf_compression& K = t_out->Compress;
        K.V = h.V; K.Top = h.Top; K.Bottom = h.Bottom; K.TopR = h.TopR; K.BottomR = h.BottomR;
        K.FractureStress = h.FractureStress; K.FractureStrain = h.FractureStrain; K.Stress = h.Stress;
        K.Strain = h.Strain; K.Loading = h.Loading; K.Fracture = h.Fracture; K.Hd2 = h.Hd2;
        K.size_d = rf_double3{h.size_d[0], h.size_d[1], h.size_d[2]};
        K.center_d = rf_double3{h.center_d[0], h.center_d[1], h.center_d[2]};
        K.size = rf_float3{h.size[0], h.size[1], h.size[2]};
        K.sized2 = rf_float3{h.sized2[0], h.sized2[1], h.sized2[2]};
        K.center = rf_float3{h.center[0], h.center[1], h.center[2]};
    }
    if (r_out) {
        r_out->steps = h.steps;                  // the specimen's own steps (all steps for one specimen)
        r_out->FractureStress = h.FractureStress; r_out->FractureStrain = h.FractureStrain;
        r_out->Stress = h.Stress; r_out->Strain = h.Strain; r_out->Fracture = h.Fracture;
        r_out->broken_bonds = g.broken;          // of the whole engine
        r_out->bonds_initial = e->bonds_initial;
        r_out->error = (rf_status)g.err;
    }
    return RF_OK;
}

rf_status rf_engine_sync(rf_engine* e, rf_task* t_out, rf_run_result* r_out) {
    if (!e) { set_error("rf_engine_sync: null engine"); return RF_ERR_INVALID; }
    if (rf_status st = rf_engine_sync_spec(e, 0, t_out, r_out)) return st;
    if (r_out && e->d.nspec > 1) {
        DevScalars g;
        RF_CUDA(cudaMemcpy(&g, e->d.sc, sizeof(g), cudaMemcpyDeviceToHost));
        r_out->steps = g.steps;
    }
    return RF_OK;
}

rf_status rf_engine_export(rf_engine* e, float* R, float* V, float* W, uint_fast32_t* IL, uint8_t* ILtype,
                           float* _1d_iL, rf_float3* Rij, rf_float3* Oijt, rf_float3* Mijn, rf_float3* Mijt) {
    if (!e) { set_error("rf_engine_export: null engine"); return RF_ERR_INVALID; }
    const uint32_t N = e->c.N, K = e->c.K;
    const size_t NK = (size_t)N * K;
    cudaStream_t s = e->stream;
    RF_CUDA(cudaStreamSynchronize(s));
    DevScalars h;
    RF_CUDA(cudaMemcpy(&h, e->d.sc, sizeof(h), cudaMemcpyDeviceToHost));
    const int cur = (int)(h.steps & 1ull);
    if (!e->staging) RF_CUDA(cudaMalloc(&e->staging, 3 * (size_t)N * sizeof(float)));
    if (e->c.ext) k_delete_pending_ext<<<(N + 127) / 128, 128, 0, s>>>(e->d, e->c);
    else k_delete_pending<<<(N + 127) / 128, 128, 0, s>>>(e->d, e->c);
    RF_CHECK_LAUNCH("k_delete_pending");
    const float4* vecs[3] = {e->d.pos[cur], e->d.vel[cur], e->d.ang[cur]};
    float* outs[3] = {R, V, W};
    for (int q = 0; q < 3; ++q) {
        if (!outs[q]) continue;
        if (q == 0 && e->c.ext) k_posd_to_planar_f<<<(N + 255) / 256, 256, 0, s>>>(e->d.posd[cur], N, e->staging);
        else k_f4_to_planar<<<(N + 255) / 256, 256, 0, s>>>(vecs[q], N, e->staging);
        RF_CHECK_LAUNCH("k_f4_to_planar");
        RF_CUDA(cudaMemcpyAsync(outs[q], e->staging, 3 * (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, s));
        RF_CUDA(cudaStreamSynchronize(s));
    }
    if (IL || ILtype || _1d_iL || Rij || Oijt || Mijn || Mijt) {
        uint_fast32_t* dIL = nullptr; uint8_t* dT = nullptr; float* dL = nullptr; rf_float3* dS = nullptr;
        cudaError_t ce = cudaMalloc(&dIL, NK * sizeof(uint_fast32_t));
        if (!ce) ce = cudaMalloc(&dT, NK);
        if (!ce) ce = cudaMalloc(&dL, NK * sizeof(float));
        if (!ce) ce = cudaMalloc(&dS, 4 * NK * sizeof(rf_float3));
        if (!ce) {
            k_rows_export<<<(N + 127) / 128, 128, 0, s>>>(dIL, dT, dL, dS, dS + NK, dS + 2 * NK, dS + 3 * NK, e->d, e->c);
            ce = cudaGetLastError();
        }
        if (!ce && IL) ce = cudaMemcpyAsync(IL, dIL, NK * sizeof(uint_fast32_t), cudaMemcpyDeviceToHost, s);
        if (!ce && ILtype) ce = cudaMemcpyAsync(ILtype, dT, NK, cudaMemcpyDeviceToHost, s);
        if (!ce && _1d_iL) ce = cudaMemcpyAsync(_1d_iL, dL, NK * sizeof(float), cudaMemcpyDeviceToHost, s);
        rf_float3* outs3[4] = {Rij, Oijt, Mijn, Mijt};
        for (int q = 0; q < 4 && !ce; ++q)
            if (outs3[q]) ce = cudaMemcpyAsync(outs3[q], dS + q * NK, NK * sizeof(rf_float3), cudaMemcpyDeviceToHost, s);
        if (!ce) ce = cudaStreamSynchronize(s);
        cudaFree(dIL); cudaFree(dT); cudaFree(dL); cudaFree(dS);
        if (ce) return cuda_status(ce, "rf_engine_export");
    }
    return RF_OK;
}

rf_status rf_engine_import(rf_engine* e, const float* R, const float* V, const float* W, const uint_fast32_t* IL,
                           const uint8_t* ILtype, const float* _1d_iL, const rf_float3* Rij, const rf_float3* Oijt,
                           const rf_float3* Mijn, const rf_float3* Mijt) {
    if (!e || !R || !V || !W || !IL || !ILtype || !_1d_iL || !Rij || !Oijt || !Mijn || !Mijt) {
        set_error("rf_engine_import: bad arguments");
        return RF_ERR_INVALID;
    }
    if (e->c.ext) {
        set_error("rf_engine_import: the extended model resumes from its own state only (no reference layout)");
        return RF_ERR_STATE;
    }
    const uint32_t N = e->c.N, K = e->c.K;
    const size_t NK = (size_t)N * K;
    cudaStream_t s = e->stream;
    RF_CUDA(cudaStreamSynchronize(s));
    DevScalars h;
    RF_CUDA(cudaMemcpy(&h, e->d.sc, sizeof(h), cudaMemcpyDeviceToHost));
    const int cur = (int)(h.steps & 1ull);
    if (!e->staging) RF_CUDA(cudaMalloc(&e->staging, 3 * (size_t)N * sizeof(float)));
    const float* ins[3] = {R, V, W};
    float4* vecs[3] = {e->d.pos[cur], e->d.vel[cur], e->d.ang[cur]};
    for (int q = 0; q < 3; ++q) {
        RF_CUDA(cudaMemcpyAsync(e->staging, ins[q], 3 * (size_t)N * sizeof(float), cudaMemcpyHostToDevice, s));
        k_planar_to_f4<<<(N + 255) / 256, 256, 0, s>>>(e->staging, N, vecs[q]);
        RF_CHECK_LAUNCH("k_planar_to_f4");
        RF_CUDA(cudaStreamSynchronize(s));
    }
    uint_fast32_t* dIL = nullptr; uint8_t* dT = nullptr; float* dL = nullptr; rf_float3* dS = nullptr;
    cudaError_t ce = cudaMalloc(&dIL, NK * sizeof(uint_fast32_t));
    if (!ce) ce = cudaMalloc(&dT, NK);
    if (!ce) ce = cudaMalloc(&dL, NK * sizeof(float));
    if (!ce) ce = cudaMalloc(&dS, 4 * NK * sizeof(rf_float3));
    if (!ce) ce = cudaMemcpyAsync(dIL, IL, NK * sizeof(uint_fast32_t), cudaMemcpyHostToDevice, s);
    if (!ce) ce = cudaMemcpyAsync(dT, ILtype, NK, cudaMemcpyHostToDevice, s);
    if (!ce) ce = cudaMemcpyAsync(dL, _1d_iL, NK * sizeof(float), cudaMemcpyHostToDevice, s);
    const rf_float3* ins3[4] = {Rij, Oijt, Mijn, Mijt};
    for (int q = 0; q < 4 && !ce; ++q)
        ce = cudaMemcpyAsync(dS + q * NK, ins3[q], NK * sizeof(rf_float3), cudaMemcpyHostToDevice, s);
    uint32_t qb = 0;
    if (!ce) ce = cudaMemsetAsync(e->maxq_dev, 0, sizeof(uint32_t), s);
    if (!ce) { k_count_records<<<148 * 4, 256, 0, s>>>(dIL, dT, dS, N, K, e->maxq_dev); ce = cudaGetLastError(); }
    if (!ce) ce = cudaMemcpyAsync(&qb, e->maxq_dev, sizeof(qb), cudaMemcpyDeviceToHost, s);
    if (!ce) ce = cudaStreamSynchronize(s);
    if (!ce && qb > e->d.QB) {
        cudaFree(dIL); cudaFree(dT); cudaFree(dL); cudaFree(dS);
        set_error("rf_engine_import: a row holds %u bond records, the engine was sized for %u", qb, e->d.QB);
        return RF_ERR_CAPACITY;
    }
    if (!ce) {
        k_rows_import<<<(N + 127) / 128, 128, 0, s>>>(dIL, dT, dL, dS, dS + NK, dS + 2 * NK, dS + 3 * NK, nullptr,
                                                      nullptr, e->d, e->c);
        ce = cudaGetLastError();
    }
    if (!ce) {
        k_force_rebuild<<<1, 1, 0, s>>>(e->d.sc);
        ce = cudaGetLastError();
    }
    if (!ce) ce = cudaStreamSynchronize(s);
    cudaFree(dIL); cudaFree(dT); cudaFree(dL); cudaFree(dS);
    if (ce) return cuda_status(ce, "rf_engine_import");
    return RF_OK;
}

rf_status rf_engine_curve_spec(rf_engine* e, int spec, double* curve, uint64_t cap, uint64_t* n) {
    if (!e || spec < 0 || (uint32_t)spec >= e->d.nspec) { set_error("rf_engine_curve: bad arguments"); return RF_ERR_INVALID; }
    DevScalars h;
    RF_CUDA(cudaStreamSynchronize(e->stream));
    RF_CUDA(cudaMemcpy(&h, e->d.spec + spec, sizeof(h), cudaMemcpyDeviceToHost));
    uint64_t m = h.curve_n < e->c.curve_cap ? h.curve_n : e->c.curve_cap;
    if (n) *n = h.curve_n;
    if (curve && cap) {
        if (m > cap) m = cap;
        RF_CUDA(cudaMemcpy(curve, e->d.curve + 3 * (size_t)spec * e->c.curve_cap, 3 * m * sizeof(double),
                           cudaMemcpyDeviceToHost));
    }
    return RF_OK;
}

}  // extern "C"

// Checkpoint files: header, the rf_task, the SaveAllData payload (rf_io.cpp).
namespace rf {
rf_status io_write_all(std::ostream& f, int id_bytes, const rf_sample* S, uint64_t pn, uint64_t N, uint32_t K,
                       float acut, const float* F, const float* V, const float* R, const float* M, const float* W,
                       const float* Q, const uint_fast32_t* IL, const uint8_t* ILtype, const float* _1d_iL,
                       const rf_float3* Rij, const rf_float3* Oijt, const rf_float3* Fijn, const rf_float3* Fijt,
                       const rf_float3* Mijn, const rf_float3* Mijt, const rf_float3* Mijadd);
rf_status io_read_all(std::istream& f, int id_bytes, rf_sample* S, uint64_t* pn, uint64_t* N_out, uint32_t* K_out,
                      float* acut, float* F, float* V, float* R, float* M, float* W, float* Q, uint_fast32_t* IL,
                      uint8_t* ILtype, float* _1d_iL, rf_float3* Rij, rf_float3* Oijt, rf_float3* Fijn,
                      rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd);
}  // namespace rf

namespace {
const char kCkptMagic[8] = {'R', 'F', 'B', '2', 'C', 'K', 'P', 'T'};
struct CkptHeader {
    char magic[8];
    uint32_t version, id_bytes, model, reserved;
    uint64_t task_bytes;
};
}  // namespace

extern "C" {

rf_status rf_engine_checkpoint(rf_engine* e, const char* path) {
    if (!e || !path) { set_error("rf_engine_checkpoint: bad arguments"); return RF_ERR_INVALID; }
    if (e->c.ext) {
        set_error("rf_engine_checkpoint: the reference model only (the extended model has no reference layout)");
        return RF_ERR_STATE;
    }
    rf_task t;
    rf_run_result r;
    TRY(rf_engine_sync(e, &t, &r));
    const uint64_t N = e->c.N, K = e->c.K, NK = N * K;
    std::vector<float> R(3 * N), V(3 * N), W(3 * N), iL(NK);
    std::vector<uint_fast32_t> IL(NK);
    std::vector<uint8_t> ty(NK);
    std::vector<rf_float3> Rij(NK), Oijt(NK), Mijn(NK), Mijt(NK);
    TRY(rf_engine_export(e, R.data(), V.data(), W.data(), IL.data(), ty.data(), iL.data(), Rij.data(), Oijt.data(),
                         Mijn.data(), Mijt.data()));
    std::ofstream f(path, std::ios::out | std::ios::binary | std::ios::trunc);
    if (!f) { set_error("rf_engine_checkpoint: cannot open %s", path); return RF_ERR_INVALID; }
    CkptHeader h;
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = 1; h.id_bytes = (uint32_t)sizeof(uint_fast32_t); h.model = 0; h.reserved = 0;
    h.task_bytes = sizeof(rf_task);
    f.write((const char*)&h, sizeof(h));
    f.write((const char*)&t, sizeof(t));
    TRY(io_write_all(f, (int)sizeof(uint_fast32_t), &t.S, 0, N, (uint32_t)K, t.acut, nullptr, V.data(), R.data(),
                     nullptr, W.data(), nullptr, IL.data(), ty.data(), iL.data(), Rij.data(), Oijt.data(), nullptr,
                     nullptr, Mijn.data(), Mijt.data(), nullptr));
    f.close();
    if (!f) { set_error("rf_engine_checkpoint: write to %s failed", path); return RF_ERR_INVALID; }
    return RF_OK;
}

rf_status rf_engine_restore(const char* path, rf_engine** out) {
    if (!path || !out) { set_error("rf_engine_restore: bad arguments"); return RF_ERR_INVALID; }
    *out = nullptr;
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) { set_error("rf_engine_restore: cannot open %s", path); return RF_ERR_INVALID; }
    CkptHeader h;
    f.read((char*)&h, sizeof(h));
    if (!f || std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1 || h.model != 0 ||
        h.id_bytes != sizeof(uint_fast32_t) || h.task_bytes != sizeof(rf_task)) {
        set_error("rf_engine_restore: %s is not a version-1 checkpoint of this build", path);
        return RF_ERR_INVALID;
    }
    rf_task t;
    f.read((char*)&t, sizeof(t));
    const std::streampos body = f.tellg();
    uint64_t N = 0;
    uint32_t K = 0;
    TRY(io_read_all(f, (int)h.id_bytes, nullptr, nullptr, &N, &K, nullptr, nullptr, nullptr, nullptr, nullptr,
                    nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                    nullptr));
    if (N != t.N || K != t.K) { set_error("rf_engine_restore: the payload does not match the task"); return RF_ERR_INVALID; }
    const uint64_t NK = N * K;
    std::vector<float> R(3 * N), V(3 * N), W(3 * N), iL(NK);
    std::vector<uint_fast32_t> IL(NK);
    std::vector<uint8_t> ty(NK);
    std::vector<rf_float3> Rij(NK), Oijt(NK), Mijn(NK), Mijt(NK);
    f.clear();
    f.seekg(body);
    TRY(io_read_all(f, (int)h.id_bytes, nullptr, nullptr, &N, &K, nullptr, nullptr, V.data(), R.data(), nullptr,
                    W.data(), nullptr, IL.data(), ty.data(), iL.data(), Rij.data(), Oijt.data(), nullptr, nullptr,
                    Mijn.data(), Mijt.data(), nullptr));
    RowsIn rows{IL.data(), ty.data(), iL.data(), Rij.data(), Oijt.data(), Mijn.data(), Mijt.data()};
    rf_engine* e = nullptr;
    TRY(engine_create_impl(&t, R.data(), nullptr, nullptr, nullptr, &e, nullptr, &rows));
    const rf_status st = rf_engine_import(e, R.data(), V.data(), W.data(), IL.data(), ty.data(), iL.data(), Rij.data(),
                                          Oijt.data(), Mijn.data(), Mijt.data());
    if (st != RF_OK) { rf_engine_destroy(e); return st; }
    *out = e;
    return RF_OK;
}

rf_status rf_engine_curve(rf_engine* e, double* curve, uint64_t cap, uint64_t* n) {
    return rf_engine_curve_spec(e, 0, curve, cap, n);
}

int rf_engine_batch_size(rf_engine* e) { return e ? (int)e->d.nspec : 0; }

rf_status rf_engine_spec_info(rf_engine* e, int spec, uint64_t* first, uint64_t* count, double* x_offset,
                              rf_task* task) {
    if (!e || spec < 0 || (uint32_t)spec >= e->d.nspec) { set_error("rf_engine_spec_info: bad arguments"); return RF_ERR_INVALID; }
    const bool b = e->d.nspec > 1;
    if (first) *first = b ? e->spec_p0[spec] : 0;
    if (count) *count = b ? e->spec_n[spec] : e->c.N;
    if (x_offset) *x_offset = b ? e->spec_xoff[spec] : 0.0;
    if (task) *task = b ? e->spec_tasks[spec] : e->task;
    return RF_OK;
}

rf_status rf_engine_counters(rf_engine* e, uint64_t* out, int n) {
    if (!e || !out || n <= 0) { set_error("rf_engine_counters: bad arguments"); return RF_ERR_INVALID; }
    cudaStream_t s = e->stream;
    RF_CUDA(cudaMemsetAsync(e->counters_dev, 0, 4 * sizeof(unsigned long long), s));
    k_counters<<<148 * 4, 256, 0, s>>>(e->d, e->c, e->counters_dev);
    RF_CHECK_LAUNCH("k_counters");
    unsigned long long cnt[4];
    DevScalars h;
    RF_CUDA(cudaMemcpyAsync(cnt, e->counters_dev, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaMemcpyAsync(&h, e->d.sc, sizeof(h), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaStreamSynchronize(s));
    const uint64_t v[5] = {h.steps, h.rebuilds, cnt[0], cnt[1], cnt[2]};
    for (int q = 0; q < n && q < 5; ++q) out[q] = v[q];
    return RF_OK;
}

int rf_engine_launches_per_step(void) { return 1; }
rf_stream rf_engine_stream(rf_engine* e) { return e ? (rf_stream)e->stream : nullptr; }
int rf_engine_uses_graph(rf_engine* e) { return (e && e->graph_ok) ? 1 : 0; }

}  // extern "C"
