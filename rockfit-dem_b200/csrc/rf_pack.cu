// Seeded polydisperse specimen generator: random positions in a cylindrical container,
// overlaps removed by FIRE with a repulsive (frictionless, undamped) Hertz contact, radii
// grown in stages from a loose start to their targets. FP64 throughout (a one-time
// generator, not the hot path). Neighbour search: a cell grid rebuilt every iteration
// (histogram, scan, scatter). Each FIRE iteration is two fused kernels (forces with the
// power and norm partials; then the per-particle FIRE update), the scalar FIRE state
// lives on the device and batches of iterations are captured in a CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "rf_common.cuh"

namespace rf {
namespace pack {

struct Scal {
    double dt, alpha, fdotv, ff, vv, maxov;
    double scale;          // current radius scale g
    unsigned long long npos, iters;
    uint32_t counter, pad;
};

struct Par {
    uint32_t N, cells, nx, ny, nz;
    double ox, oy, oz, inv_h;       // grid origin and 1 / cell edge
    double Rc, Hh;                  // container radius and half height
    double dtmax, dtmin, finc, fdec, alpha0, falpha;
    uint32_t ndelay;
};

struct Dev {
    double4* x;       // x, y, z, target radius
    double4* v;       // velocity (w unused)
    double4* f;       // force (w unused)
    uint32_t *key, *count, *start, *fill, *sorted, *bsum;
    double4* part;    // per-block (F.v, |F|^2, |v|^2, max overlap)
    Scal* s;
};

__device__ __forceinline__ uint32_t cell_of(const double4 p, const Par& c) {
    long ix = (long)floor((p.x - c.ox) * c.inv_h), iy = (long)floor((p.y - c.oy) * c.inv_h),
         iz = (long)floor((p.z - c.oz) * c.inv_h);
    ix = ix < 0 ? 0 : (ix >= (long)c.nx ? c.nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= (long)c.ny ? c.ny - 1 : iy);
    iz = iz < 0 ? 0 : (iz >= (long)c.nz ? c.nz - 1 : iz);
    return (uint32_t)(ix + c.nx * (iy + c.ny * iz));
}

__global__ void k_zero(Dev d, Par c) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < c.cells; q += gridDim.x * blockDim.x) {
        d.count[q] = 0; d.fill[q] = 0;
    }
}
__global__ void k_bin(Dev d, Par c) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const uint32_t k = cell_of(d.x[i], c);
        d.key[i] = k;
        atomicAdd(&d.count[k], 1u);
    }
}
// single-block exclusive scan of the cell counts (cells are few: N / ~2)
// Exclusive scan of the cell counts into cell starts, in three kernels: per-chunk sums
// (SCAN_CHUNK cells per block), a one-block scan of the chunk sums, and the chunks'
// own scans offset by their sums.
constexpr uint32_t SCAN_CHUNK = 4096;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* wsum, uint32_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) { const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += y; }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        const uint32_t t = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
        uint32_t ti = t;
        for (int o = 1; o < 32; o <<= 1) { const uint32_t y = __shfl_up_sync(0xffffffffu, ti, o); if (lane >= o) ti += y; }
        wsum[lane] = ti - t;
        if (lane == 31) *total = ti;
    }
    __syncthreads();
    const uint32_t r = wsum[w] + incl - v;
    __syncthreads();
    return r;
}

__global__ void k_scan_sums(Dev d, Par c) {
    __shared__ uint32_t sh[32];
    const size_t base = (size_t)blockIdx.x * SCAN_CHUNK;
    uint32_t s = 0;
    for (uint32_t t = threadIdx.x; t < SCAN_CHUNK; t += blockDim.x)
        if (base + t < c.cells) s += d.count[base + t];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) d.bsum[blockIdx.x] = v;
    }
}

// one block: exclusive scan of the nb chunk sums, in place
__global__ void k_scan_chunks(Dev d, uint32_t nb) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t total;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += blockDim.x) {
        const uint32_t q = base + threadIdx.x;
        const uint32_t v = q < nb ? d.bsum[q] : 0;
        const uint32_t ex = block_excl_scan(v, wsum, &total);
        if (q < nb) d.bsum[q] = carry + ex;
        carry += total;
        __syncthreads();
    }
}

__global__ void k_scan_apply(Dev d, Par c) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t total;
    const size_t base = (size_t)blockIdx.x * SCAN_CHUNK;
    uint32_t carry = d.bsum[blockIdx.x];
    for (uint32_t off = 0; off < SCAN_CHUNK; off += blockDim.x) {
        const size_t q = base + off + threadIdx.x;
        const uint32_t v = q < c.cells ? d.count[q] : 0;
        const uint32_t ex = block_excl_scan(v, wsum, &total);
        if (q < c.cells) d.start[q] = carry + ex;
        carry += total;
        __syncthreads();
    }
}
__global__ void k_scatter(Dev d, Par c) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const uint32_t k = d.key[i];
        d.sorted[d.start[k] + atomicAdd(&d.fill[k], 1u)] = i;
    }
}

// Occupants of each cell in id order (the scatter's atomics leave them in arrival
// order), so the force sums below, and with them the whole packing, are deterministic.
__global__ void k_cellsort(Dev d, Par c) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < c.cells; q += gridDim.x * blockDim.x) {
        uint32_t* a = d.sorted + d.start[q];
        const uint32_t n = d.count[q];
        for (uint32_t u = 1; u < n; ++u) {
            const uint32_t v = a[u];
            uint32_t w = u;
            while (w > 0 && a[w - 1] > v) { a[w] = a[w - 1]; --w; }
            a[w] = v;
        }
    }
}

// Forces: repulsive Hertz between overlapping spheres and against the container wall,
// f = 4/3 sqrt(R*) delta^1.5 (unit modulus, unit masses). Partials of F.v, |F|^2,
// |v|^2 and the largest overlap (relative to the smaller radius).
__global__ void k_force(Dev d, Par c) {
    const double g = d.s->scale;
    double fv = 0, ff = 0, vv = 0, mo = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        const double4 xi = d.x[i];
        const double ri = g * xi.w;
        double fx = 0, fy = 0, fz = 0;
        const uint32_t key = d.key[i];
        const int ix = key % c.nx, iy = (key / c.nx) % c.ny, iz = key / (c.nx * c.ny);
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = iz + dz;
            if (z < 0 || z >= (int)c.nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = iy + dy;
                if (y < 0 || y >= (int)c.ny) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = ix + dx;
                    if (x < 0 || x >= (int)c.nx) continue;
                    const uint32_t cell = x + c.nx * (y + c.ny * z);
                    const uint32_t s0 = d.start[cell], e0 = s0 + d.count[cell];
                    for (uint32_t q = s0; q < e0; ++q) {
                        const uint32_t j = d.sorted[q];
                        if (j == i) continue;
                        const double4 xj = d.x[j];
                        const double rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
                        const double rj = g * xj.w;
                        const double r2 = rx * rx + ry * ry + rz * rz, sr = ri + rj;
                        if (r2 >= sr * sr || r2 <= 0) continue;
                        const double r = sqrt(r2), dl = sr - r;
                        const double Rs = ri * rj / sr;
                        const double fn = (4.0 / 3.0) * sqrt(Rs) * dl * sqrt(dl);
                        fx -= fn * rx / r; fy -= fn * ry / r; fz -= fn * rz / r;
                        mo = fmax(mo, dl / fmin(ri, rj));
                    }
                }
            }
        }
        // container wall (cylinder side and end caps)
        const double rho = sqrt(xi.x * xi.x + xi.y * xi.y);
        const double dw = rho + ri - c.Rc;
        if (dw > 0 && rho > 0) {
            const double fn = (4.0 / 3.0) * sqrt(ri) * dw * sqrt(dw);
            fx -= fn * xi.x / rho; fy -= fn * xi.y / rho;
            mo = fmax(mo, dw / ri);
        }
        const double dtop = xi.z + ri - c.Hh, dbot = -xi.z + ri - c.Hh;
        if (dtop > 0) { fz -= (4.0 / 3.0) * sqrt(ri) * dtop * sqrt(dtop); mo = fmax(mo, dtop / ri); }
        if (dbot > 0) { fz += (4.0 / 3.0) * sqrt(ri) * dbot * sqrt(dbot); mo = fmax(mo, dbot / ri); }
        const double4 vi = d.v[i];
        d.f[i] = make_double4(fx, fy, fz, 0.0);
        fv += fx * vi.x + fy * vi.y + fz * vi.z;
        ff += fx * fx + fy * fy + fz * fz;
        vv += vi.x * vi.x + vi.y * vi.y + vi.z * vi.z;
    }
    __shared__ double sh[4][32];
    for (int o = 16; o; o >>= 1) {
        fv += __shfl_xor_sync(0xffffffffu, fv, o);
        ff += __shfl_xor_sync(0xffffffffu, ff, o);
        vv += __shfl_xor_sync(0xffffffffu, vv, o);
        mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[0][w] = fv; sh[1][w] = ff; sh[2][w] = vv; sh[3][w] = mo; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, e = 0, m = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += sh[0][q]; b += sh[1][q]; e += sh[2][q]; m = fmax(m, sh[3][q]); }
        d.part[blockIdx.x] = make_double4(a, b, e, m);
    }
}

// FIRE step decision (one block): sums of the block partials in a fixed order (thread t
// adds partials t, t + blockDim, ...; then a fixed tree), then power, time step and
// mixing factor on thread 0.
__global__ void k_fire_decide(Dev d, Par c, int nblocks) {
    __shared__ double sh[4][32];
    double fv = 0, ff = 0, vv = 0, mo = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double4 p = d.part[b];
        fv += p.x; ff += p.y; vv += p.z; mo = fmax(mo, p.w);
    }
    for (int o = 16; o; o >>= 1) {
        fv += __shfl_xor_sync(0xffffffffu, fv, o);
        ff += __shfl_xor_sync(0xffffffffu, ff, o);
        vv += __shfl_xor_sync(0xffffffffu, vv, o);
        mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[0][w] = fv; sh[1][w] = ff; sh[2][w] = vv; sh[3][w] = mo; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    fv = 0; ff = 0; vv = 0; mo = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { fv += sh[0][q]; ff += sh[1][q]; vv += sh[2][q]; mo = fmax(mo, sh[3][q]); }
    Scal* s = d.s;
    s->fdotv = fv; s->ff = ff; s->vv = vv; s->maxov = mo;
    if (fv > 0) {
        s->npos += 1;
        if (s->npos > c.ndelay) { s->dt = fmin(s->dt * c.finc, c.dtmax); s->alpha *= c.falpha; }
        s->counter = 0;
    } else {
        s->npos = 0;
        s->dt = fmax(s->dt * c.fdec, c.dtmin);
        s->alpha = c.alpha0;
        s->counter = 1;                     // velocity reset this iteration
    }
    s->iters += 1;
}

// FIRE update: back off half a step and stop on uphill power, then semi-implicit Euler
// and the velocity mixing v = (1 - a) v + a |v| F / |F| (per particle).
__global__ void k_fire_update(Dev d, Par c) {
    const Scal s = *d.s;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.N; i += gridDim.x * blockDim.x) {
        double4 x = d.x[i], v = d.v[i];
        const double4 f = d.f[i];
        if (s.counter) {
            x.x -= 0.5 * s.dt * v.x; x.y -= 0.5 * s.dt * v.y; x.z -= 0.5 * s.dt * v.z;
            v = make_double4(0, 0, 0, 0);
        }
        v.x += f.x * s.dt; v.y += f.y * s.dt; v.z += f.z * s.dt;
        const double vn = sqrt(v.x * v.x + v.y * v.y + v.z * v.z), fn = sqrt(f.x * f.x + f.y * f.y + f.z * f.z);
        if (fn > 0) {
            const double a = s.alpha, k = a * vn / fn;
            v.x = (1 - a) * v.x + k * f.x; v.y = (1 - a) * v.y + k * f.y; v.z = (1 - a) * v.z + k * f.z;
        }
        x.x += v.x * s.dt; x.y += v.y * s.dt; x.z += v.z * s.dt;
        d.x[i] = x; d.v[i] = v;
    }
}

inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double unif(uint64_t seed, uint64_t k) {
    return (double)(splitmix64(seed * 0x2545F4914F6CDD1Dull + k) >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace pack
}  // namespace rf

using namespace rf;
using namespace rf::pack;

extern "C" rf_status rf_pack_cylinder(uint64_t seed, uint64_t N, double r0, double rmin, double rmax, double aspect,
                                      double phi, const double center[3], double* R, double* radius,
                                      double* diameter, double* height, double* max_overlap) {
    return rf_pack_cylinder_dist(seed, N, r0, rmin, rmax, RF_RADII_UNIFORM, aspect, phi, center, R, radius, diameter,
                                 height, max_overlap);
}

extern "C" rf_status rf_pack_cylinder_dist(uint64_t seed, uint64_t N, double r0, double rmin, double rmax, int dist,
                                           double aspect, double phi, const double center[3], double* R,
                                           double* radius, double* diameter, double* height, double* max_overlap) {
    if (N < 2 || !(r0 > 0) || !(rmin > 0) || !(rmax >= rmin) || !(aspect > 0) || !(phi > 0.05 && phi < 0.7) || !R ||
        !radius || !center || (dist != RF_RADII_UNIFORM && dist != RF_RADII_LOG_UNIFORM)) {
        set_error("rf_pack_cylinder: bad arguments");
        return RF_ERR_INVALID;
    }
    // work in units of r0; container sized for the target packing fraction
    std::vector<double4> hx(N);
    double vol = 0.0;
    for (uint64_t i = 0; i < N; ++i) {
        const double u = unif(seed, 4 * i + 3);
        const double r = dist == RF_RADII_LOG_UNIFORM ? rmin * std::pow(rmax / rmin, u) : rmin + (rmax - rmin) * u;
        hx[i].w = r;
        vol += 4.0 / 3.0 * M_PI * r * r * r;
    }
    const double Vc = vol / phi;
    const double D = std::cbrt(4.0 * Vc / (M_PI * aspect)), H = aspect * D;
    const double Rc = 0.5 * D, Hh = 0.5 * H;
    for (uint64_t i = 0; i < N; ++i) {      // uniform in the container (rejection on the disc)
        double x, y;
        uint64_t k = 0;
        do {
            x = (2.0 * unif(seed, 4 * i + 0 + 4 * N * k) - 1.0) * Rc;
            y = (2.0 * unif(seed, 4 * i + 1 + 4 * N * k) - 1.0) * Rc;
            ++k;
        } while (x * x + y * y > (Rc - hx[i].w) * (Rc - hx[i].w) && k < 64);
        hx[i].x = x; hx[i].y = y;
        hx[i].z = (2.0 * unif(seed, 4 * i + 2) - 1.0) * (Hh - hx[i].w);
    }
    double rmx = rmax;
    Par c{};
    c.N = (uint32_t)N;
    const double hcell = 2.0 * rmx * 1.0001;
    c.inv_h = 1.0 / hcell;
    c.ox = -Rc - hcell; c.oy = -Rc - hcell; c.oz = -Hh - hcell;
    c.nx = (uint32_t)std::ceil((2 * Rc + 2 * hcell) / hcell) + 1; c.ny = c.nx;
    c.nz = (uint32_t)std::ceil((2 * Hh + 2 * hcell) / hcell) + 1;
    c.cells = c.nx * c.ny * c.nz;
    c.Rc = Rc; c.Hh = Hh;
    c.dtmax = 1.0; c.dtmin = 1e-4; c.finc = 1.1; c.fdec = 0.5; c.alpha0 = 0.1; c.falpha = 0.99; c.ndelay = 5;
    Dev d{};
    std::vector<void*> allocs;
    auto al = [&](void** p, size_t bytes) { cudaError_t e = cudaMalloc(p, bytes); if (!e) allocs.push_back(*p); return e; };
    const int nb = (int)((N + 255) / 256) < 148 * 8 ? (int)((N + 255) / 256) : 148 * 8;
    cudaError_t e = cudaSuccess;
    if (!e) e = al((void**)&d.x, N * sizeof(double4));
    if (!e) e = al((void**)&d.v, N * sizeof(double4));
    if (!e) e = al((void**)&d.f, N * sizeof(double4));
    if (!e) e = al((void**)&d.key, N * 4);
    if (!e) e = al((void**)&d.sorted, N * 4);
    if (!e) e = al((void**)&d.count, (size_t)c.cells * 4);
    if (!e) e = al((void**)&d.start, (size_t)c.cells * 4);
    if (!e) e = al((void**)&d.fill, (size_t)c.cells * 4);
    if (!e) e = al((void**)&d.part, nb * sizeof(double4));
    const uint32_t nchunks = (c.cells + SCAN_CHUNK - 1) / SCAN_CHUNK;
    if (!e) e = al((void**)&d.bsum, (size_t)nchunks * sizeof(uint32_t));
    if (!e) e = al((void**)&d.s, sizeof(Scal));
    cudaStream_t st = nullptr;
    if (!e) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    Scal hs{};
    hs.dt = 0.1; hs.alpha = c.alpha0; hs.scale = 0.5;
    if (!e) e = cudaMemcpyAsync(d.x, hx.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(d.v, 0, N * sizeof(double4), st);
    if (!e) e = cudaMemcpyAsync(d.s, &hs, sizeof(hs), cudaMemcpyHostToDevice, st);
    // one batch of FIRE iterations, captured once and relaunched
    const int BATCH = 50;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (!e) e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (!e) {
        for (int it = 0; it < BATCH; ++it) {
            k_zero<<<(c.cells + 255) / 256, 256, 0, st>>>(d, c);
            k_bin<<<nb, 256, 0, st>>>(d, c);
            k_scan_sums<<<nchunks, 256, 0, st>>>(d, c);
            k_scan_chunks<<<1, 1024, 0, st>>>(d, nchunks);
            k_scan_apply<<<nchunks, 1024, 0, st>>>(d, c);
            k_scatter<<<nb, 256, 0, st>>>(d, c);
            k_cellsort<<<(c.cells + 255) / 256, 256, 0, st>>>(d, c);
            k_force<<<nb, 256, 0, st>>>(d, c);
            k_fire_decide<<<1, 1024, 0, st>>>(d, c, nb);
            k_fire_update<<<nb, 256, 0, st>>>(d, c);
        }
        e = cudaStreamEndCapture(st, &graph);
    }
    if (!e) e = cudaGraphInstantiate(&exec, graph, 0);
    // radius growth: g from 0.5 to 1, relaxing each stage to a small overlap
    double g = 0.5, mo = 0.0;
    const int max_batches_per_stage = 200;
    for (int stage = 0; !e && stage < 400; ++stage) {
        const double tol = (g >= 1.0) ? 2e-4 : 5e-3;
        int b = 0;
        for (; b < max_batches_per_stage && !e; ++b) {
            e = cudaGraphLaunch(exec, st);
            if (!e) e = cudaMemcpyAsync(&hs, d.s, sizeof(hs), cudaMemcpyDeviceToHost, st);
            if (!e) e = cudaStreamSynchronize(st);
            if (hs.maxov < tol) break;
        }
        mo = hs.maxov;
        if (g >= 1.0) break;
        g = std::min(1.0, g * 1.02);
        hs.scale = g;
        // keep dt/alpha, restart the positive-power count
        hs.npos = 0;
        if (!e) e = cudaMemcpyAsync(d.s, &hs, sizeof(hs), cudaMemcpyHostToDevice, st);
        (void)b;
    }
    if (!e) e = cudaMemcpyAsync(hx.data(), d.x, N * sizeof(double4), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (st) cudaStreamDestroy(st);
    for (void* p : allocs) cudaFree(p);
    if (e) return cuda_status(e, "rf_pack_cylinder");
    // number the particles in spatial order (cells of 6 r0, x fastest, then y, then z;
    // packing order within a cell), so that a particle's neighbours sit close to it in
    // memory and the step kernels' neighbour gathers hit the caches
    std::vector<uint64_t> key(N), order(N);
    {
        const double h = 6.0;
        const double x0 = -Rc, y0 = -Rc, z0 = -Hh;
        const uint64_t nx = (uint64_t)std::ceil(2.0 * Rc / h) + 2, ny = nx;
        for (uint64_t i = 0; i < N; ++i) {
            const double fx = std::floor((hx[i].x - x0) / h), fy = std::floor((hx[i].y - y0) / h),
                         fz = std::floor((hx[i].z - z0) / h);
            const uint64_t cx = fx < 0 ? 0 : (uint64_t)fx, cy = fy < 0 ? 0 : (uint64_t)fy, cz = fz < 0 ? 0 : (uint64_t)fz;
            key[i] = cx + nx * (cy + ny * cz);
            order[i] = i;
        }
        std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return key[a] < key[b]; });
    }
    for (uint64_t q = 0; q < N; ++q) {
        const double4& p = hx[order[q]];
        R[q] = center[0] + r0 * p.x;
        R[q + N] = center[1] + r0 * p.y;
        R[q + 2 * N] = center[2] + r0 * p.z;
        radius[q] = r0 * p.w;
    }
    if (diameter) *diameter = r0 * D;
    if (height) *height = r0 * H;
    if (max_overlap) *max_overlap = mo;
    return RF_OK;
}
