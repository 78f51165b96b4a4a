// md_* drop-in kernels: the RockFit-DEM hot-path step operations on buffers in the
// reference's own layout (md_data_types.h), in place, on a caller stream.
//
// Rows are read one particle per thread in slot order, as the reference's row
// loops run, so per-particle force and moment sums are accumulated in the same
// order and round the same way. Cell binning replaces cub's radix sort with a
// counting sort (histogram, scan, scatter, per-cell id order), whose output is
// the same stable (cell, id) order.
#include <cstdio>
#include <mutex>
#include "rf_physics.cuh"

namespace rf {

typedef uint_fast32_t mid_t;   // the reference's id type at this boundary
static_assert(sizeof(mid_t) == 8 || sizeof(mid_t) == 4, "unexpected uint_fast32_t width");

__device__ __forceinline__ f3 ld3p(const float* P, size_t N, size_t i) {   // planar x|y|z
    return mk3(P[i], P[i + N], P[i + 2 * N]);
}
__device__ __forceinline__ f3 ld3(const rf_float3* p, size_t k) { return mk3(p[k].x, p[k].y, p[k].z); }
__device__ __forceinline__ void st3(rf_float3* p, size_t k, f3 v) { p[k].x = v.x; p[k].y = v.y; p[k].z = v.z; }

static inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return (int)g;
}

// ---------------------------------------------------------------------------
// Cells
// ---------------------------------------------------------------------------
__global__ void k_cell_index(const float* __restrict__ R, size_t N, mid_t* __restrict__ CI, RefGrid g,
                             uint32_t* __restrict__ counts, uint32_t* err) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t cx, cy, cz;
        const uint32_t c = ref_cell(ld3p(R, N, i), g, &cx, &cy, &cz);
        CI[i] = (mid_t)c;
        if (cx > g.nx - 1 || cy > g.ny - 1 || cz > g.nz - 1 || (uint64_t)c >= g.CN)
            raise_status(err, RF_ERR_CELL_RANGE);
        // binned by the key, as the sort orders it: a key past the grid goes to the tail
        // bin; an out-of-range cell coordinate whose linear key still lands inside the grid
        // (it wraps into another row) is binned under that key, as the scatter files it
        if (counts) atomicAdd(&counts[(uint64_t)c < g.CN ? (uint64_t)c : g.CN], 1u);
    }
}

// Exclusive scan, three passes: per-block totals, scan of totals, add back.
__global__ void k_scan_block_sums(const uint32_t* __restrict__ in, size_t n, uint32_t* __restrict__ bsum) {
    __shared__ uint32_t sh[32];
    const size_t base = (size_t)blockIdx.x * 4096;
    uint32_t s = 0;
    for (int t = threadIdx.x; t < 4096; t += blockDim.x)
        if (base + t < n) s += in[base + t];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) bsum[blockIdx.x] = v;
    }
}
__global__ void k_scan_totals(uint32_t* __restrict__ bsum, size_t nb) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        uint32_t acc = 0;
        for (size_t b = 0; b < nb; ++b) { uint32_t v = bsum[b]; bsum[b] = acc; acc += v; }
    }
}
// 1024 threads x 4 items per block of 4096
__global__ void k_scan_apply(const uint32_t* __restrict__ in, size_t n, const uint32_t* __restrict__ boff,
                             uint32_t* __restrict__ out) {
    __shared__ uint32_t wsum[32];
    const size_t base = (size_t)blockIdx.x * 4096 + (size_t)threadIdx.x * 4;
    uint32_t v[4], t = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) { v[q] = (base + q < n) ? in[base + q] : 0; t += v[q]; }
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
    uint32_t run = boff[blockIdx.x] + wsum[w] + incl - t;
#pragma unroll
    for (int q = 0; q < 4; ++q) { if (base + q < n) out[base + q] = run; run += v[q]; }
}

__global__ void k_cell_scatter(const mid_t* __restrict__ CI, size_t N, uint64_t CN, const uint32_t* __restrict__ start,
                               uint32_t* __restrict__ fill, mid_t* __restrict__ CIs) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t c = (uint64_t)CI[i];
        const uint64_t b = c < CN ? c : CN;
        const uint32_t p = start[b] + atomicAdd(&fill[b], 1u);
        CIs[N + p] = (mid_t)i;
    }
}

// Order each cell's ids ascending (the stable sort's tie order), write the sorted
// keys and pnC. One thread per cell; cells hold tens of particles.
__global__ void k_cell_finish(const mid_t* __restrict__ CI, size_t N, uint64_t CN, const uint32_t* __restrict__ counts,
                              const uint32_t* __restrict__ start, mid_t* __restrict__ CIs, mid_t* __restrict__ pnC) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c <= CN; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t n = counts[c], s = start[c];
        mid_t* ids = CIs + N + s;
        for (uint32_t a = 1; a < n; ++a) {            // insertion sort by id (for the tail bin: by key, then id)
            mid_t v = ids[a];
            uint64_t kv = (c < CN) ? 0 : (uint64_t)CI[v];
            uint32_t b = a;
            while (b > 0) {
                mid_t u = ids[b - 1];
                uint64_t ku = (c < CN) ? 0 : (uint64_t)CI[u];
                if (ku < kv || (ku == kv && u < v)) break;
                ids[b] = u;
                --b;
            }
            ids[b] = v;
        }
        for (uint32_t a = 0; a < n; ++a) CIs[s + a] = (c < CN) ? (mid_t)c : CI[ids[a]];
        if (c < CN) {
            pnC[c] = n ? (mid_t)s : (mid_t)0;
            pnC[c + CN] = (mid_t)n;
        }
    }
}

// d_DetermineCellPointer's run scan continues past N into the id half of CIs
// (md_calculate_cell.cu:72): the last run's count grows by one when CIs[N] equals
// its key. Reproduced so pnC matches the reference bit for bit.
__global__ void k_cell_last_run(size_t N, uint64_t CN, mid_t* __restrict__ CIs, mid_t* __restrict__ pnC) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && N > 0) {
        const mid_t last = CIs[N - 1];
        if ((uint64_t)last < CN && CIs[N] == last) pnC[last + CN] += 1;
    }
}

// ---------------------------------------------------------------------------
// Rows
// ---------------------------------------------------------------------------
__global__ void k_list_construct(const float* __restrict__ R, size_t N, const mid_t* __restrict__ CIs,
                                 const mid_t* __restrict__ pnC, mid_t* __restrict__ IL, uint32_t K, RefGrid g,
                                 float aacut, uint32_t* err) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const f3 xi = ld3p(R, N, i);
        int64_t cells[8];
        octant_cells(xi, g, cells);
        uint32_t n = 0;
        for (int c = 0; c < 8; ++c) {
            if (cells[c] < 0 || (uint64_t)cells[c] >= g.CN) { raise_status(err, RF_ERR_CELL_RANGE); continue; }
            const uint64_t s = (uint64_t)pnC[cells[c]], cnt = (uint64_t)pnC[cells[c] + g.CN];
            for (uint64_t m = 0; m < cnt; ++m) {
                if (s + m >= N) break;
                const mid_t j = CIs[s + m + N];
                if ((size_t)j >= N) continue;
                const float rr = dist2_rn(xi, ld3p(R, N, j));
                if (rr < aacut && (size_t)j != i) {
                    if (n < K) IL[i * K + n] = j;
                    else raise_status(err, RF_ERR_ROW_OVERFLOW);
                    ++n;
                }
            }
        }
    }
}

__global__ void k_list_reconstruct_bpm(const float* __restrict__ R, size_t N, const mid_t* __restrict__ CIs,
                                       const mid_t* __restrict__ pnC, mid_t* __restrict__ IL, uint8_t* __restrict__ ILtype,
                                       uint32_t K, RefGrid g, float aacut, uint32_t* err) {
    const mid_t E = empty_id<mid_t>();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const f3 xi = ld3p(R, N, i);
        int64_t cells[8];
        octant_cells(xi, g, cells);
        mid_t* row = IL + i * K;
        for (int c = 0; c < 8; ++c) {
            if (cells[c] < 0 || (uint64_t)cells[c] >= g.CN) { raise_status(err, RF_ERR_CELL_RANGE); continue; }
            const uint64_t s = (uint64_t)pnC[cells[c]], cnt = (uint64_t)pnC[cells[c] + g.CN];
            for (uint64_t m = 0; m < cnt; ++m) {
                if (s + m >= N) break;
                const mid_t j = CIs[s + m + N];
                if ((size_t)j >= N) continue;
                const float rr = dist2_rn(xi, ld3p(R, N, j));
                if (!(rr < aacut && (double)rr > 1e-10)) continue;
                // addnewlinkbpm (md_interaction_list_reconstructbpm.cu:25-41): scan the row for
                // j and for the first free slot; slot 0 of particle 0 reads as "none found".
                uint64_t kfree = 0;
                bool any_free = false, found = false;
                for (uint32_t q = 0; q < K; ++q) {
                    const mid_t kj = row[q];
                    if (kj == E) {
                        any_free = true;
                        if (kfree == 0) kfree = i * K + q;
                    }
                    if (kj == j) { found = true; break; }
                }
                if (found) continue;
                // A full row: the reference writes IL[0] here; the row is left unchanged instead.
                if (!any_free) { raise_status(err, RF_ERR_ROW_OVERFLOW); continue; }
                IL[kfree] = j;
                ILtype[kfree] = 0;
            }
        }
    }
}

__global__ void k_delete_far_links(const float* __restrict__ R, size_t N, mid_t* __restrict__ IL,
                                   uint8_t* __restrict__ ILtype, rf_float3* Rij, rf_float3* Oijt, rf_float3* Fijn,
                                   rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd, uint32_t K,
                                   float aacut) {
    const mid_t E = empty_id<mid_t>();
    const f3 z = mk3(0.f, 0.f, 0.f);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const f3 xi = ld3p(R, N, i);
        for (uint32_t q = 0; q < K; ++q) {
            const size_t k = i * K + q;
            const mid_t j = IL[k];
            if (j == E || (size_t)j >= N) continue;
            const float rr = dist2_rn(xi, ld3p(R, N, j));
            if (rr > aacut || (double)rr < 1e-10) {
                IL[k] = E;
                ILtype[k] = 0;
                // 1/L0 is left as it was: the reference's "_1d_iL = 0;" clears its own pointer.
                st3(Rij, k, z); st3(Oijt, k, z); st3(Fijn, k, z); st3(Fijt, k, z);
                st3(Mijn, k, z); st3(Mijt, k, z); st3(Mijadd, k, z);
            }
        }
    }
}

// rm2 with the contraction nvcc gives r.x*r.x + r.y*r.y + r.z*r.z in the reference build.
__device__ __forceinline__ float rm2_bond(float x, float y, float z) {
    return __fmaf_rn(z, z, __fmaf_rn(x, x, __fmul_rn(y, y)));
}

__global__ void k_construct_bonds(const float* __restrict__ R, size_t N, const mid_t* __restrict__ IL,
                                  uint8_t* __restrict__ ILtype, float* __restrict__ iL, rf_float3* Rij, rf_float3* Oijt,
                                  rf_float3* Fijn, rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd,
                                  uint32_t K, float aa_create) {
    const mid_t E = empty_id<mid_t>();
    const f3 z = mk3(0.f, 0.f, 0.f);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const f3 xi = ld3p(R, N, i);
        for (uint32_t q = 0; q < K; ++q) {
            const size_t k = i * K + q;
            const mid_t j = IL[k];
            if (j == E || (size_t)j >= N) continue;
            const f3 xj = ld3p(R, N, j);
            const float rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
            const float rm2 = rm2_bond(rx, ry, rz);
            if (rm2 < aa_create && (double)rm2 > 1e-18) {
                iL[k] = __frsqrt_rn(rm2);
                ILtype[k] = 1;
            } else {
                ILtype[k] = 0;
            }
            st3(Rij, k, z); st3(Oijt, k, z); st3(Fijn, k, z); st3(Fijt, k, z);
            st3(Mijn, k, z); st3(Mijt, k, z); st3(Mijadd, k, z);
        }
    }
}

// ---------------------------------------------------------------------------
// Forces
// ---------------------------------------------------------------------------
__global__ void k_forces_22(const float* __restrict__ R, const float* __restrict__ V, const float* __restrict__ W,
                            const mid_t* __restrict__ IL, uint8_t* __restrict__ ILtype, const float* __restrict__ iL,
                            rf_float3* __restrict__ Rij, rf_float3* __restrict__ Oijt, rf_float3* __restrict__ Mijn,
                            rf_float3* __restrict__ Mijt, float* __restrict__ F, float* __restrict__ M, size_t N,
                            uint32_t K, BondParams p) {
    const mid_t E = empty_id<mid_t>();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const f3 xi = ld3p(R, N, i), vi = ld3p(V, N, i), wi = ld3p(W, N, i);
        f3 fs = mk3(0.f, 0.f, 0.f), ms = mk3(0.f, 0.f, 0.f);
        for (uint32_t q = 0; q < K; ++q) {
            const size_t k = i * K + q;
            const mid_t j = IL[k];
            if (!(j != E && ILtype[k] == 1)) continue;
            const f3 xj = ld3p(R, N, j);
            const f3 r = mk3(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z);
            f3 rij = ld3(Rij, k), oijt = ld3(Oijt, k), mijn = ld3(Mijn, k), mijt = ld3(Mijt, k);
            const bool broke = bond_slot(p, r, vi, ld3p(V, N, j), wi, ld3p(W, N, j), iL[k], rij, oijt, mijn, mijt, fs, ms);
            st3(Rij, k, rij); st3(Oijt, k, oijt); st3(Mijn, k, mijn); st3(Mijt, k, mijt);
            if (broke) ILtype[k] = 0;
        }
        F[i] += fs.x; F[i + N] += fs.y; F[i + 2 * N] += fs.z;
        M[i] += ms.x; M[i + N] += ms.y; M[i + 2 * N] += ms.z;
    }
}

__global__ void k_forces_21(const float* __restrict__ R, const float* __restrict__ V, const float* __restrict__ W,
                            const mid_t* __restrict__ IL, const uint8_t* __restrict__ ILtype,
                            rf_float3* __restrict__ Oijt, float* __restrict__ F, float* __restrict__ M, size_t N,
                            uint32_t K, ContactParams p) {
    const mid_t E = empty_id<mid_t>();
    const f3 z = mk3(0.f, 0.f, 0.f);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const f3 xi = ld3p(R, N, i), vi = ld3p(V, N, i), wi = ld3p(W, N, i);
        f3 fs = mk3(0.f, 0.f, 0.f), ms = mk3(0.f, 0.f, 0.f);
        for (uint32_t q = 0; q < K; ++q) {
            const size_t k = i * K + q;
            const mid_t j = IL[k];
            if (j != E && ILtype[k] == 0) {
                const f3 xj = ld3p(R, N, j);
                const f3 r = mk3(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z);
                f3 o = ld3(Oijt, k);
                if (contact_slot(p, r, vi, ld3p(V, N, j), wi, ld3p(W, N, j), o, fs, ms)) st3(Oijt, k, o);
                else st3(Oijt, k, z);
            } else if (j == E) {
                st3(Oijt, k, z);
            }
        }
        F[i] += fs.x; F[i + N] += fs.y; F[i + 2 * N] += fs.z;
        M[i] += ms.x; M[i + N] += ms.y; M[i + 2 * N] += ms.z;
    }
}

__global__ void k_increments(const float* __restrict__ F, float* __restrict__ V, float* __restrict__ R,
                             const float* __restrict__ M, float* __restrict__ W, size_t N, float dtm, float dt, float dtI) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const size_t q = i + c * N;
            V[q] += __fmul_rn(F[q], dtm);
            R[q] += __fmul_rn(V[q], dt);
            W[q] += __fmul_rn(M[q], dtI);
        }
}

// Block-wide sum of two doubles (deterministic tree).
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sa[32], sb[32];
    for (int o = 16; o; o >>= 1) { a += __shfl_xor_sync(0xffffffffu, a, o); b += __shfl_xor_sync(0xffffffffu, b, o); }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        a = l < (int)(blockDim.x >> 5) ? sa[l] : 0.0;
        b = l < (int)(blockDim.x >> 5) ? sb[l] : 0.0;
        for (int o = 16; o; o >>= 1) { a += __shfl_xor_sync(0xffffffffu, a, o); b += __shfl_xor_sync(0xffffffffu, b, o); }
    }
}

__global__ void k_brazil(float* R, float* V, float* F, float* FL, size_t N, rf_float3 c, float RR, float Yt, float Yb,
                         float Ytr, float Ybr, float vt, float Zcut, uint64_t nblocks) {
    double sfb = 0.0, sft = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        brazil_particle(R[i], R[i + N], R[i + 2 * N], V[i], V[i + N], V[i + 2 * N], F[i], F[i + N], F[i + 2 * N], c,
                        RR, Yt, Yb, Ytr, Ybr, vt, Zcut, sfb, sft);
    block_sum2(sfb, sft);
    if (threadIdx.x == 0) { FL[blockIdx.x] = (float)sfb; FL[nblocks + blockIdx.x] = (float)sft; }
}

__global__ void k_uniaxial(float* R, float* V, float* F, float* FL, size_t N, rf_float3 c, float RR, float Zt, float Zb,
                           float Ztr, float Zbr, float vt, float Zcut, uint64_t nblocks) {
    double sfb = 0.0, sft = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        uniaxial_particle(R[i], R[i + N], R[i + 2 * N], V[i + 2 * N], F[i + 2 * N], c, RR, Zt, Zb, Ztr, Zbr, vt, Zcut,
                          sfb, sft);
    block_sum2(sfb, sft);
    if (threadIdx.x == 0) { FL[blockIdx.x] = (float)sfb; FL[nblocks + blockIdx.x] = (float)sft; }
}

__global__ void k_cut(float* R, float* V, float* F, size_t N, rf_float3 c, rf_float3 h, rf_float3 hp) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        if (outside_box(R[i], R[i + N], R[i + 2 * N], c, h)) {
            R[i] = hp.x; R[i + N] = hp.y; R[i + 2 * N] = hp.z;
            V[i] = 0.f; V[i + N] = 0.f; V[i + 2 * N] = 0.f;
            F[i] = 0.f; F[i + N] = 0.f; F[i + 2 * N] = 0.f;
        }
    }
}

// d_CalculateIncrementsFIRE (md_firerelaxation.cu:18-56)
__global__ void k_fire_inc(const float* __restrict__ F, float* __restrict__ V, float* __restrict__ R, size_t N, float dtm,
                           float dt, float a) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const float Fx = F[i], Fy = F[i + N], Fz = F[i + 2 * N];
        float vx = __fmul_rn(Fx, dtm), vy = __fmul_rn(Fy, dtm), vz = __fmul_rn(Fz, dtm);
        const float vv = vx * vx + vy * vy + vz * vz;
        const float f = Fx * Fx + Fy * Fy + Fz * Fz;
        float vdf;
        if (f > 1e-12f) vdf = a * __fsqrt_rn(vv * __frcp_rn(f));
        else vdf = a * __fsqrt_rn(vv) * 1e6f;
        vx = (1.0f - a) * vx + vdf * Fx;
        vy = (1.0f - a) * vy + vdf * Fy;
        vz = (1.0f - a) * vz + vdf * Fz;
        V[i] = vx; V[i + N] = vy; V[i + 2 * N] = vz;
        R[i] += __fmul_rn(vx, dt); R[i + N] += __fmul_rn(vy, dt); R[i + 2 * N] += __fmul_rn(vz, dt);
    }
}
__global__ void k_fire_half(const float* __restrict__ V, float* __restrict__ R, size_t N, float dt2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 3 * N; i += (size_t)gridDim.x * blockDim.x)
        R[i] -= __fmul_rn(V[i], dt2);
}
__global__ void k_fdotv(const float* __restrict__ V, const float* __restrict__ F, size_t N, double* __restrict__ partial) {
    double s = 0.0, dummy = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 3 * N; i += (size_t)gridDim.x * blockDim.x)
        s += (double)F[i] * (double)V[i];
    block_sum2(s, dummy);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}
// Identity of the CUDA context current on the calling thread, unique within the process
// (cuCtxGetId). A cudaDeviceReset destroys the device's primary context together with
// every device address taken in it; the next runtime call makes a new context with a
// new id, so an address cached with the id of the context it came from is known to be
// stale when the ids differ. cudaSetDevice makes the device's primary context current
// (creating it if needed) and allocates nothing. The driver functions come through
// cudaGetDriverEntryPoint, so the library keeps linking against the runtime only.
static rf_status current_context_id(int dev, unsigned long long* id) {
    typedef int (*ctx_get_current_t)(void**);
    typedef int (*ctx_get_id_t)(void*, unsigned long long*);
    static ctx_get_current_t get_current = nullptr;
    static ctx_get_id_t get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (ctx_get_current_t)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (ctx_get_id_t)f;
    });
    if (!get_current || !get_id) { set_error("driver entry points cuCtxGetCurrent / cuCtxGetId unavailable"); return RF_ERR_CUDA; }
    RF_CUDA(cudaSetDevice(dev));
    void* ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) {
        set_error("no CUDA context current on device %d", dev);
        return RF_ERR_CUDA;
    }
    return RF_OK;
}

// Status word of the md_* launches of one host thread on the current device (one per
// device, re-made when the device's context was reset). nullptr if it cannot be had.
static uint32_t* status_word() {
    const int kMaxDev = 64;
    static thread_local uint32_t* w[kMaxDev] = {nullptr};
    static thread_local unsigned long long ctx[kMaxDev] = {0};
    int dev = 0;
    unsigned long long id = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return nullptr;
    if (current_context_id(dev, &id) != RF_OK) return nullptr;
    if (!w[dev] || ctx[dev] != id) {
        // a word of an earlier context went away with it; a word of this one is kept
        w[dev] = nullptr;
        uint32_t* p = nullptr;
        if (cudaMalloc(&p, sizeof(uint32_t)) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, sizeof(uint32_t)) != cudaSuccess) { cudaFree(p); return nullptr; }
        w[dev] = p;
        ctx[dev] = id;
    }
    return w[dev];
}

// Read and clear the status word after a launch sequence (synchronises the stream).
static rf_status take_status(cudaStream_t s) {
    uint32_t* w = status_word();
    if (!w) { set_error("md_* status word unavailable on the current device"); return RF_ERR_CUDA; }
    uint32_t h = 0;
    RF_CUDA(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaStreamSynchronize(s));
    if (h) {
        RF_CUDA(cudaMemsetAsync(w, 0, sizeof(uint32_t), s));
        RF_CUDA(cudaStreamSynchronize(s));
        set_error("device status %u", h);
        return (rf_status)h;
    }
    return RF_OK;
}

}  // namespace rf

using namespace rf;

static inline cudaStream_t S(rf_stream s) { return (cudaStream_t)s; }
static inline RefGrid make_grid(float a, float inv_a, rf_uint3 cN, uint64_t CN) {
    RefGrid g;
    g.a = a; g.inv_a = inv_a; g.nx = cN.x; g.ny = cN.y; g.nz = cN.z; g.CN = CN;
    return g;
}

extern "C" {

rf_status md_CalculateCellIndex(const float* R, uint_fast32_t N, uint_fast32_t* CI, float _1d_a, rf_uint3 cN,
                                rf_stream stream) {
    if (!R || !CI || N == 0) { set_error("md_CalculateCellIndex: bad arguments"); return RF_ERR_INVALID; }
    RefGrid g = make_grid(0.f, _1d_a, cN, (uint64_t)cN.x * cN.y * cN.z);
    k_cell_index<<<grid_for(N, 256), 256, 0, S(stream)>>>(R, N, CI, g, nullptr, status_word());
    RF_CHECK_LAUNCH("k_cell_index");
    return take_status(S(stream));
}

size_t md_CellDistributionScratchBytes(uint_fast32_t N, uint_fast32_t CN) {
    (void)N;
    const size_t cells = (size_t)CN + 1;                 // + tail bin for out-of-grid keys
    const size_t nb = (cells + 4095) / 4096;
    return (3 * cells + nb) * sizeof(uint32_t) + 256;
}

rf_status md_CellDistribution(const float* R, uint_fast32_t N, uint_fast32_t* CI, uint_fast32_t* CIs,
                              uint_fast32_t* pnC, uint_fast32_t CN, float _1d_a, rf_uint3 cN, void* scratch,
                              size_t scratch_bytes, rf_stream stream) {
    if (!R || !CI || !CIs || !pnC || N == 0 || CN == 0 || !scratch) {
        set_error("md_CellDistribution: bad arguments");
        return RF_ERR_INVALID;
    }
    if (scratch_bytes < md_CellDistributionScratchBytes(N, CN)) {
        set_error("md_CellDistribution: scratch too small (%zu < %zu)", scratch_bytes,
                  md_CellDistributionScratchBytes(N, CN));
        return RF_ERR_INVALID;
    }
    if ((uint64_t)cN.x * cN.y * cN.z != (uint64_t)CN) { set_error("md_CellDistribution: CN != Nr.x*Nr.y*Nr.z"); return RF_ERR_INVALID; }
    cudaStream_t s = S(stream);
    const size_t cells = (size_t)CN + 1, nb = (cells + 4095) / 4096;
    uint32_t* counts = (uint32_t*)scratch;
    uint32_t* start = counts + cells;
    uint32_t* fill = start + cells;
    uint32_t* bsum = fill + cells;
    RefGrid g = make_grid(0.f, _1d_a, cN, CN);
    RF_CUDA(cudaMemsetAsync(counts, 0, cells * sizeof(uint32_t), s));
    RF_CUDA(cudaMemsetAsync(fill, 0, cells * sizeof(uint32_t), s));
    k_cell_index<<<grid_for(N, 256), 256, 0, s>>>(R, N, CI, g, counts, status_word());
    k_scan_block_sums<<<(unsigned)nb, 1024, 0, s>>>(counts, cells, bsum);
    k_scan_totals<<<1, 32, 0, s>>>(bsum, nb);
    k_scan_apply<<<(unsigned)nb, 1024, 0, s>>>(counts, cells, bsum, start);
    k_cell_scatter<<<grid_for(N, 256), 256, 0, s>>>(CI, N, CN, start, fill, CIs);
    k_cell_finish<<<grid_for(cells, 128), 128, 0, s>>>(CI, N, CN, counts, start, CIs, pnC);
    k_cell_last_run<<<1, 32, 0, s>>>(N, CN, CIs, pnC);
    RF_CHECK_LAUNCH("md_CellDistribution");
    return take_status(s);
}

rf_status md_InteractionListConstruct(const float* R, uint_fast32_t N, const uint_fast32_t* CIs,
                                      const uint_fast32_t* pnC, uint_fast32_t* IL, uint_fast32_t K, float a,
                                      float _1d_a, float aacut, rf_uint3 cN, uint_fast32_t CN, rf_stream stream) {
    if (!R || !CIs || !pnC || !IL || N == 0 || K == 0) { set_error("md_InteractionListConstruct: bad arguments"); return RF_ERR_INVALID; }
    cudaStream_t s = S(stream);
    RF_CUDA(cudaMemsetAsync(IL, 0xFF, (size_t)N * K * sizeof(uint_fast32_t), s));
    k_list_construct<<<grid_for(N, 128), 128, 0, s>>>(R, N, CIs, pnC, IL, (uint32_t)K, make_grid(a, _1d_a, cN, CN),
                                                     aacut, status_word());
    RF_CHECK_LAUNCH("k_list_construct");
    return take_status(s);
}

rf_status md_InteractionListReConstructBPM(const float* R, uint_fast32_t N, const uint_fast32_t* CIs,
                                           const uint_fast32_t* pnC, uint_fast32_t* IL, uint8_t* ILtype,
                                           uint_fast32_t K, float a, float _1d_a, float aacut, rf_uint3 cN,
                                           uint_fast32_t CN, rf_stream stream) {
    if (!R || !CIs || !pnC || !IL || !ILtype || N == 0 || K == 0) {
        set_error("md_InteractionListReConstructBPM: bad arguments");
        return RF_ERR_INVALID;
    }
    cudaStream_t s = S(stream);
    k_list_reconstruct_bpm<<<grid_for(N, 128), 128, 0, s>>>(R, N, CIs, pnC, IL, ILtype, (uint32_t)K,
                                                            make_grid(a, _1d_a, cN, CN), aacut, status_word());
    RF_CHECK_LAUNCH("k_list_reconstruct_bpm");
    return take_status(s);
}

rf_status md_DeleteFarLinks(const float* R, uint_fast32_t N, uint_fast32_t* IL, uint8_t* ILtype, float* _1d_iL,
                            rf_float3* Rij, rf_float3* Oijt, rf_float3* Fijn, rf_float3* Fijt, rf_float3* Mijn,
                            rf_float3* Mijt, rf_float3* Mijadd, uint_fast32_t K, float aacut, rf_stream stream) {
    (void)_1d_iL;
    if (!R || !IL || !ILtype || !Rij || !Oijt || !Fijn || !Fijt || !Mijn || !Mijt || !Mijadd || N == 0 || K == 0) {
        set_error("md_DeleteFarLinks: bad arguments");
        return RF_ERR_INVALID;
    }
    k_delete_far_links<<<grid_for(N, 128), 128, 0, S(stream)>>>(R, N, IL, ILtype, Rij, Oijt, Fijn, Fijt, Mijn, Mijt,
                                                               Mijadd, (uint32_t)K, aacut);
    RF_CHECK_LAUNCH("k_delete_far_links");
    return RF_OK;
}

rf_status md_ConstructBoundInteractions(const float* R, const float* V, const float* W, const uint_fast32_t* IL,
                                        uint8_t* ILtype, float* _1d_iL, rf_float3* Rij, rf_float3* Oijt,
                                        rf_float3* Fijn, rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt,
                                        rf_float3* Mijadd, uint_fast32_t N, uint_fast32_t K, float aa_create,
                                        float b_r, rf_stream stream) {
    (void)V; (void)W; (void)b_r;
    if (!R || !IL || !ILtype || !_1d_iL || !Rij || !Oijt || !Fijn || !Fijt || !Mijn || !Mijt || !Mijadd || N == 0 || K == 0) {
        set_error("md_ConstructBoundInteractions: bad arguments");
        return RF_ERR_INVALID;
    }
    k_construct_bonds<<<grid_for(N, 128), 128, 0, S(stream)>>>(R, N, IL, ILtype, _1d_iL, Rij, Oijt, Fijn, Fijt, Mijn,
                                                              Mijt, Mijadd, (uint32_t)K, aa_create);
    RF_CHECK_LAUNCH("k_construct_bonds");
    return RF_OK;
}

rf_status md_CalculateForcesDEM_22(const float* R, const float* V, const float* W, const uint_fast32_t* IL,
                                   uint8_t* ILtype, const float* _1d_iL, rf_float3* Rij, rf_float3* Oijt,
                                   rf_float3* Mijn, rf_float3* Mijt, float* F, float* M, uint_fast32_t N,
                                   uint_fast32_t K, float dt, float m_E, float m_G, float b_r, float m_Gcritn,
                                   float m_Gcritt, rf_stream stream) {
    if (!R || !V || !W || !IL || !ILtype || !_1d_iL || !Rij || !Oijt || !Mijn || !Mijt || !F || !M || N == 0 || K == 0) {
        set_error("md_CalculateForcesDEM_22: bad arguments");
        return RF_ERR_INVALID;
    }
    BondParams p{dt, m_E, m_G, b_r, m_Gcritn, m_Gcritt};
    k_forces_22<<<grid_for(N, 128), 128, 0, S(stream)>>>(R, V, W, IL, ILtype, _1d_iL, Rij, Oijt, Mijn, Mijt, F, M, N,
                                                        (uint32_t)K, p);
    RF_CHECK_LAUNCH("k_forces_22");
    return RF_OK;
}

rf_status md_CalculateForcesDEM_21(const float* R, const float* V, const float* W, const uint_fast32_t* IL,
                                   uint8_t* ILtype, const float* _1d_iL, rf_float3* Rij, rf_float3* Oijt, float* F,
                                   float* M, uint_fast32_t N, uint_fast32_t K, float dt, float m_E, float m_G,
                                   float p_A, float m_mu, float m_muroll, float mP, float rP, rf_stream stream) {
    (void)_1d_iL; (void)Rij;
    if (!R || !V || !W || !IL || !ILtype || !Oijt || !F || !M || N == 0 || K == 0) {
        set_error("md_CalculateForcesDEM_21: bad arguments");
        return RF_ERR_INVALID;
    }
    ContactParams p{dt, m_E, m_G, p_A, m_mu, m_muroll, mP, rP};
    k_forces_21<<<grid_for(N, 128), 128, 0, S(stream)>>>(R, V, W, IL, ILtype, Oijt, F, M, N, (uint32_t)K, p);
    RF_CHECK_LAUNCH("k_forces_21");
    return RF_OK;
}

rf_status md_CalculateIncrementsDEM(const float* F, float* V, float* R, const float* M, float* W, uint_fast32_t N,
                                    float _1d_Mass_m_dt, float dt, float _1d_I_m_dt, rf_stream stream) {
    if (!F || !V || !R || !M || !W || N == 0) { set_error("md_CalculateIncrementsDEM: bad arguments"); return RF_ERR_INVALID; }
    k_increments<<<grid_for(N, 256), 256, 0, S(stream)>>>(F, V, R, M, W, N, _1d_Mass_m_dt, dt, _1d_I_m_dt);
    RF_CHECK_LAUNCH("k_increments");
    return RF_OK;
}

rf_status md_braziltest_simple2(float* R, float* V, float* F, float* FL, uint_fast32_t N, rf_float3 c, float RR,
                                float Yt, float Yb, float Ytr, float Ybr, float vt, float Zcut, uint64_t nblocks,
                                rf_stream stream) {
    if (!R || !V || !F || !FL || N == 0 || nblocks == 0) { set_error("md_braziltest_simple2: bad arguments"); return RF_ERR_INVALID; }
    cudaStream_t s = S(stream);
    const int g = (int)(nblocks < 148 * 4 ? nblocks : 148 * 4);
    RF_CUDA(cudaMemsetAsync(FL, 0, 2 * nblocks * sizeof(float), s));
    k_brazil<<<g, 256, 0, s>>>(R, V, F, FL, N, c, RR, Yt, Yb, Ytr, Ybr, vt, Zcut, nblocks);
    RF_CHECK_LAUNCH("k_brazil");
    return RF_OK;
}

rf_status md_UniaxialCompression3_simple(float* R, float* V, float* F, float* FL, uint_fast32_t N, rf_float3 c,
                                         float RR, float Zt, float Zb, float Ztr, float Zbr, float vt, float Zcut,
                                         uint64_t nblocks, rf_stream stream) {
    if (!R || !V || !F || !FL || N == 0 || nblocks == 0) {
        set_error("md_UniaxialCompression3_simple: bad arguments");
        return RF_ERR_INVALID;
    }
    cudaStream_t s = S(stream);
    const int g = (int)(nblocks < 148 * 4 ? nblocks : 148 * 4);
    RF_CUDA(cudaMemsetAsync(FL, 0, 2 * nblocks * sizeof(float), s));
    k_uniaxial<<<g, 256, 0, s>>>(R, V, F, FL, N, c, RR, Zt, Zb, Ztr, Zbr, vt, Zcut, nblocks);
    RF_CHECK_LAUNCH("k_uniaxial");
    return RF_OK;
}

rf_status md_ParallelepipedCutRestriction(float* R, float* V, float* F, uint_fast32_t N, rf_float3 center,
                                          rf_float3 sized2, rf_float3 hp, rf_stream stream) {
    if (!R || !V || !F || N == 0) { set_error("md_ParallelepipedCutRestriction: bad arguments"); return RF_ERR_INVALID; }
    k_cut<<<grid_for(N, 256), 256, 0, S(stream)>>>(R, V, F, N, center, sized2, hp);
    RF_CHECK_LAUNCH("k_cut");
    return RF_OK;
}

rf_status md_CalculateIncrementsFIRE(const float* F, float* V, float* R, uint_fast32_t N, float _1d_Mass_m_dt, float dt,
                                     float F_alpha, rf_stream stream) {
    if (!F || !V || !R || N == 0) { set_error("md_CalculateIncrementsFIRE: bad arguments"); return RF_ERR_INVALID; }
    k_fire_inc<<<grid_for(N, 256), 256, 0, S(stream)>>>(F, V, R, N, _1d_Mass_m_dt, dt, F_alpha);
    RF_CHECK_LAUNCH("k_fire_inc");
    return RF_OK;
}

rf_status md_CalculateDecrementsHalfStepFIRE(const float* V, float* R, uint_fast32_t N, float dt_d2, rf_stream stream) {
    if (!V || !R || N == 0) { set_error("md_CalculateDecrementsHalfStepFIRE: bad arguments"); return RF_ERR_INVALID; }
    k_fire_half<<<grid_for(3 * (size_t)N, 256), 256, 0, S(stream)>>>(V, R, N, dt_d2);
    RF_CHECK_LAUNCH("k_fire_half");
    return RF_OK;
}

rf_status md_FdotVEntire(const float* V, const float* F, double* FdotV, uint64_t nblocks, uint_fast32_t N,
                         rf_stream stream) {
    if (!V || !F || !FdotV || N == 0 || nblocks == 0) { set_error("md_FdotVEntire: bad arguments"); return RF_ERR_INVALID; }
    const int g = (int)(nblocks < 148 * 8 ? nblocks : 148 * 8);
    cudaStream_t s = S(stream);
    RF_CUDA(cudaMemsetAsync(FdotV, 0, nblocks * sizeof(double), s));
    k_fdotv<<<g, 256, 0, s>>>(V, F, N, FdotV);
    RF_CHECK_LAUNCH("k_fdotv");
    return RF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Cell binning without any allocation.
//
// Some callers cannot allocate device memory at the point where they bin: a host
// framework that owns every device byte through its own allocator and forbids other
// allocations, or a plugin handed only its input and output buffers.
// md_CellDistribution needs caller-provided scratch; md_CellDistributionNoAlloc
// instead uses the file-scope device array below as its scratch, so it allocates
// nothing. The array is fixed in size (cell grids of up to RF_NOALLOC_MAX_CELLS - 1
// cells, about 6.3 MB) and every GPU that loads this library holds it until the
// process exits. Like the other md_* entry points, a call returns only once its work
// on the stream has finished: it reads the device status word back.
// ---------------------------------------------------------------------------
#define RF_NOALLOC_MAX_CELLS (1u << 19)   /* cells + the out-of-grid tail bin */
#define RF_NOALLOC_WORDS (3u * RF_NOALLOC_MAX_CELLS + 256u)
static __device__ __align__(256) uint32_t g_noalloc_scratch[RF_NOALLOC_WORDS];

namespace rf {
namespace {
// Device address of g_noalloc_scratch per device. In host code the symbol name is
// only a host-side stand-in, so the address comes from cudaGetSymbolAddress, once
// per device, with that device current. The address belongs to the context it was
// taken in: after a cudaDeviceReset the array lives at a new address in the new
// context, so the lookup is redone when the context id differs from the cached one.
const int kMaxDevices = 64;
uint32_t* g_noalloc_ptr[kMaxDevices] = {nullptr};
unsigned long long g_noalloc_ctx[kMaxDevices] = {0};
std::mutex g_noalloc_mu;

rf_status noalloc_scratch(uint32_t** out) {
    int dev = 0;
    RF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) { set_error("md_CellDistributionNoAlloc: device %d out of range", dev); return RF_ERR_INVALID; }
    unsigned long long id = 0;
    rf_status st = current_context_id(dev, &id);
    if (st) return st;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev] || g_noalloc_ctx[dev] != id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "md_CellDistributionNoAlloc: cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = (uint32_t*)p;
        g_noalloc_ctx[dev] = id;
    }
    *out = g_noalloc_ptr[dev];
    return RF_OK;
}
}  // namespace
}  // namespace rf

extern "C" rf_status md_CellDistributionNoAlloc(const float* R, uint_fast32_t N, uint_fast32_t* CI,
                                                uint_fast32_t* CIs, uint_fast32_t* pnC, uint_fast32_t CN,
                                                float _1d_a, rf_uint3 cN, rf_stream stream) {
    if (!R || !CI || !CIs || !pnC || N == 0 || CN == 0) {
        set_error("md_CellDistributionNoAlloc: bad arguments");
        return RF_ERR_INVALID;
    }
    if ((uint64_t)cN.x * cN.y * cN.z != (uint64_t)CN) {
        set_error("md_CellDistributionNoAlloc: CN != Nr.x*Nr.y*Nr.z");
        return RF_ERR_INVALID;
    }
    if ((uint64_t)CN + 1 > RF_NOALLOC_MAX_CELLS) {
        set_error("md_CellDistributionNoAlloc: %llu cells exceed the fixed scratch limit of %u cells; "
                  "use md_CellDistribution with caller scratch", (unsigned long long)CN, RF_NOALLOC_MAX_CELLS - 1);
        return RF_ERR_INVALID;
    }
    uint32_t* base = nullptr;
    rf_status st = noalloc_scratch(&base);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t cells = (size_t)CN + 1, nb = (cells + 4095) / 4096;
    uint32_t* counts = base;
    uint32_t* start = counts + cells;
    uint32_t* fill = start + cells;
    uint32_t* bsum = fill + cells;
    uint32_t* status = base + RF_NOALLOC_WORDS - 1;
    RefGrid g = make_grid(0.f, _1d_a, cN, CN);
    // The array keeps the previous call's contents: counters and status start at zero.
    RF_CUDA(cudaMemsetAsync(counts, 0, cells * sizeof(uint32_t), s));
    RF_CUDA(cudaMemsetAsync(fill, 0, cells * sizeof(uint32_t), s));
    RF_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), s));
    k_cell_index<<<grid_for(N, 256), 256, 0, s>>>(R, N, CI, g, counts, status);
    k_scan_block_sums<<<(unsigned)nb, 1024, 0, s>>>(counts, cells, bsum);
    k_scan_totals<<<1, 32, 0, s>>>(bsum, nb);
    k_scan_apply<<<(unsigned)nb, 1024, 0, s>>>(counts, cells, bsum, start);
    k_cell_scatter<<<grid_for(N, 256), 256, 0, s>>>(CI, N, CN, start, fill, CIs);
    k_cell_finish<<<grid_for(cells, 128), 128, 0, s>>>(CI, N, CN, counts, start, CIs, pnC);
    k_cell_last_run<<<1, 32, 0, s>>>(N, CN, CIs, pnC);
    RF_CHECK_LAUNCH("md_CellDistributionNoAlloc");
    uint32_t h = 0;
    RF_CUDA(cudaMemcpyAsync(&h, status, sizeof(h), cudaMemcpyDeviceToHost, s));
    RF_CUDA(cudaStreamSynchronize(s));
    if (h) {
        set_error("md_CellDistributionNoAlloc: device status %u", h);
        return (rf_status)h;
    }
    return RF_OK;
}
