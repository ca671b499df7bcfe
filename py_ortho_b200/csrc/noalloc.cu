// mvs_sweep_noalloc: the multi-hypothesis sweep for callers that cannot allocate device memory.
//
// mvs_sweep allocates its plane-chunk scratch (the per-chunk winner records merged in
// hypothesis order) with cudaMallocAsync on every call. Some callers cannot do that: a host
// process whose device memory is owned entirely by another allocator (a framework's caching
// pool holding a fixed budget), or a latency-critical loop that must not enter the driver's
// allocator, which can synchronise the device. This entry point takes its scratch from one
// file-scope device array instead and calls no allocating routine.
//
// Limits and behaviour:
//   * the array holds MVS_NOALLOC_SCRATCH_BYTES (32 MiB) per GPU that loads the library, for the
//     life of the process;
//   * with plane_chunks == 0 the chunk count is the automatic one, lowered until the records fit;
//     an explicit plane_chunks whose records do not fit is rejected (MVS_ERR_VALUE);
//   * every call looks up the array's device address on the current device
//     (cudaGetSymbolAddress, which allocates nothing once the array exists); the first call on a
//     device - and the first after that device's context was reset - loads the library's device
//     code there, which is when the array is created: make that first call before any stream
//     capture;
//   * every call shares the array and it keeps the last call's contents; nothing in it needs to
//     start at zero (each chunk record is written in full before it is merged), but calls that
//     overlap on the GPU (different streams, or host threads without ordering) race on it.
#include "sweep_tile.cuh"

#define MVS_NOALLOC_SCRATCH_BYTES (32u << 20)

namespace mvs {

size_t sweep_scratch_bytes(const mvs_sweep_args* a, int* nchunks_out);
mvs_status sweep_with_scratch(const mvs_sweep_args* a, void* scratch, size_t scratch_bytes, cudaStream_t st);

static __device__ __align__(256) float g_noalloc_scratch[MVS_NOALLOC_SCRATCH_BYTES / sizeof(float)];

// The array's name is a host-side stand-in in host code; its device address is looked up on the
// current device at every call, so a context that was reset and recreated is never served a
// stale address.
static mvs_status noalloc_scratch(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(MVS_ERR_CUDA, "sweep_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    *out = p;
    return MVS_OK;
}

}  // namespace mvs

using namespace mvs;

extern "C" mvs_status mvs_sweep_noalloc(const mvs_sweep_args* a, void* stream) {
    clear_error();
    MVS_TRY(validate_sweep(a));
    if (a->H == 0 || a->W == 0 || a->i1 == a->i0) return MVS_OK;
    mvs_sweep_args b = *a;
    int nch = 1;
    size_t need = sweep_scratch_bytes(&b, &nch);
    if (need > MVS_NOALLOC_SCRATCH_BYTES) {
        if (a->plane_chunks > 0)
            return fail(MVS_ERR_VALUE,
                        "sweep_noalloc: %d plane chunks of a %dx%d image need %zu bytes of scratch, above the "
                        "%u-byte static buffer; use fewer plane chunks (0 = automatic) or mvs_sweep",
                        a->plane_chunks, a->H, a->W, need, MVS_NOALLOC_SCRATCH_BYTES);
        // automatic chunking: lower the chunk count until the records fit (one chunk needs none)
        while (nch > 1 && need > MVS_NOALLOC_SCRATCH_BYTES) {
            b.plane_chunks = --nch;
            need = sweep_scratch_bytes(&b, &nch);
        }
    }
    void* ws = nullptr;
    if (need) MVS_TRY(noalloc_scratch(&ws));
    return sweep_with_scratch(&b, ws, need, reinterpret_cast<cudaStream_t>(stream));
}
