// Shared definitions for the B200 DEM engine: error plumbing, id types, small
// vector helpers. Translation units that include this are compiled with
// --fmad=false: every a*b+c below is a separate IEEE multiply and add, the way
// the CPU oracle evaluates it; fused multiply-adds appear only where written as
// __fmaf_rn.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/rockfit_b200.h"

#define RF_WARP 32

namespace rf {

// Empty slot marker for the engine's 32-bit rows.
constexpr uint32_t EMPTY32 = 0xFFFFFFFFu;

template <class IdT> __host__ __device__ constexpr IdT empty_id() { return (IdT)~(IdT)0; }

// Device-side status word: the first non-zero status wins.
__device__ __forceinline__ void raise_status(uint32_t* err, uint32_t code) {
    if (err) atomicCAS(err, 0u, code);
}

struct f3 { float x, y, z; };
__host__ __device__ __forceinline__ f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }

// Host-side error text.
void set_error(const char* fmt, ...);
rf_status cuda_status(cudaError_t e, const char* what);

}  // namespace rf

#define RF_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t e__ = (call);                                       \
        if (e__ != cudaSuccess) return rf::cuda_status(e__, #call);     \
    } while (0)

#define RF_CHECK_LAUNCH(what)                                           \
    do {                                                                \
        cudaError_t e__ = cudaGetLastError();                           \
        if (e__ != cudaSuccess) return rf::cuda_status(e__, what);      \
    } while (0)
