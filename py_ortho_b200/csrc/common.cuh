// Shared helpers of libmvs_b200: status / last-error plumbing and small device utilities.
#pragma once

#include <cuda.h>              // CUtensorMap (the tensor-map type only; the driver is reached at run time)
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>
#include <string.h>

#include "../../include/mvs_b200.h"

namespace mvs {

// Thread-local message of the last failing call (the reference raises with a message; the
// ctypes shim reads this and raises the matching Python exception).
void set_error(const char* fmt, ...);
void clear_error();

inline mvs_status fail(mvs_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return st;
}

inline mvs_status check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return fail(e == cudaErrorMemoryAllocation ? MVS_ERR_MEMORY : MVS_ERR_CUDA,
                    "%s: %s", what, cudaGetErrorString(e));
    }
    return MVS_OK;
}

#define MVS_TRY(expr)                        \
    do {                                     \
        mvs_status st__ = (expr);            \
        if (st__ != MVS_OK) return st__;     \
    } while (0)

#define MVS_CUDA(expr, what)                                                              \
    do {                                                                                  \
        cudaError_t e__ = (expr);                                                         \
        if (e__ != cudaSuccess)                                                           \
            return ::mvs::fail(e__ == cudaErrorMemoryAllocation ? MVS_ERR_MEMORY             \
                                                                : MVS_ERR_CUDA,           \
                               "%s: %s", what, cudaGetErrorString(e__));                  \
    } while (0)

inline int num_sms() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

// Bounds-checked debug build (nvcc -DMVS_DEBUG_BOUNDS; `python -m py_ortho_b200.build
// --debug-bounds` writes libmvs_b200_debug.so): MVS_BOUND(cond) counts every shared-memory or
// global index the instrumented kernels (tile engine, batched / server kernels, PatchMatch) would
// use outside its buffer, in a per-translation-unit device counter that the host reads with
// mvs_debug_bound_violations. The access itself still happens (the counter records, it does not
// trap), so tests run the debug build on small cases only. Release builds compile the checks away.
#ifdef MVS_DEBUG_BOUNDS
static __device__ unsigned g_bound_violations;
#define MVS_BOUND(cond)                                                  \
    do {                                                                 \
        if (!(cond)) atomicAdd(&::mvs::g_bound_violations, 1u);          \
    } while (0)
// host: this translation unit's count, cleared
static inline unsigned take_bound_violations_here() {
    unsigned n = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&n, g_bound_violations, sizeof(n)) != cudaSuccess) return ~0u;
    cudaMemcpyToSymbol(g_bound_violations, &zero, sizeof(zero));
    return n;
}
#else
#define MVS_BOUND(cond) \
    do {                \
    } while (0)
static inline unsigned take_bound_violations_here() { return 0; }
#endif
// per-unit readers (sweep.cu, batch.cu, patchmatch.cu), summed by mvs_debug_bound_violations
unsigned take_bound_violations_sweep();
unsigned take_bound_violations_batch();
unsigned take_bound_violations_pm();

// NaN-propagating max with a float32 floor (np.maximum semantics).
__device__ __forceinline__ float max_nan(float v, float lo) { return (v >= lo || v != v) ? v : lo; }
__device__ __forceinline__ double max_nan(double v, double lo) { return (v >= lo || v != v) ? v : lo; }

}  // namespace mvs
