// Plane-sweep kernels of one view: the tiled sweep (engine in sweep_tile.cuh), the ordered
// plane-chunk merge and the sub-hypothesis parabola (finalize), plus their C-ABI entry points.
#define MVS_SWEEP_TMA_UNIT 1   // this unit instantiates the TMA kernels and owns their fault counter
#include "sweep_tile.cuh"

#include <atomic>
#include <cudaTypedefs.h>
#include <mutex>

namespace mvs {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        else
            cudaGetLastError();
    });
    return fn;
}

// The reference's 2D tiled map for the tile copy: box = the tile with its halo (Geom<r, th>::JP x
// Geom<r, th>::HR floats). Needs a 16-byte aligned base and a row pitch that is a multiple of 16
// bytes (W % 4 == 0); otherwise the tile is loaded by the threads (same values).
static bool make_ref_map(SweepParams& p, const float* ref, int H, int W, int r, int th) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || !ref || (reinterpret_cast<uintptr_t>(ref) & 15u) || W % 4 != 0 || W < 1 || H < 1) return false;
    const int RA = (r + 3) & ~3;
    const cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
    const cuuint64_t strides[1] = {(cuuint64_t)W * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)(TW + 2 * RA + 4), (cuuint32_t)(th + 2 * r)};
    const cuuint32_t es[2] = {1, 1};
    const CUresult e = enc(&p.ref_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ref), dims, strides, box,
                           es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return e == CUDA_SUCCESS;
}

template <int R, int KMAX, bool PLANES, bool F16, bool X64, bool CMP, int TH = TH_DEFAULT>
__global__ void __launch_bounds__(TileShape<TH>::NT, TileShape<TH>::MIN_CTAS)
    sweep_kernel(const __grid_constant__ SweepParams p) {
    extern __shared__ __align__(128) float4 smem4[];
    const int pa = p.i0 + blockIdx.z * p.ppc;
    const int pb = min(p.i1, pa + p.ppc);
    sweep_tile<R, KMAX, PLANES, F16, true, true, X64, CMP, TH>(p, blockIdx.x * TW, blockIdx.y * TH, pa, pb,
                                                     p.rec ? (int)blockIdx.z : -1, reinterpret_cast<float*>(smem4));
}

__global__ void merge_kernel(long long HW, int nchunks, int i0, int i1, int ppc, const float* __restrict__ rec,
                             float* best, float* prev, float* spb, float* snb, int* idx) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= HW) return;
    float B = best[o], P = prev[o], SP = spb[o], SN = snb[o];
    int I = idx[o];
    merge_pixel(o, HW, nchunks, i0, i1, ppc, rec, B, P, SP, SN, I);
    best[o] = B;
    prev[o] = P;
    spb[o] = SP;
    snb[o] = SN;
    idx[o] = I;
}

__global__ void finalize_kernel(int H, int W, int kind, int n, int t0, const float* __restrict__ hyp_a,
                                const float* __restrict__ hyp_b, long long map_stride, float plane0,
                                float plane1, const float* __restrict__ best, const float* __restrict__ spb,
                                const float* __restrict__ snb, const int* __restrict__ idx, float* depth) {
    const long long HW = (long long)H * W;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= HW) return;
    float inv0, inv1;
    switch (kind) {
        case MVS_HYP_MAPS:
            inv0 = hyp_a[o];
            inv1 = n > 1 ? hyp_a[map_stride + o] : inv0;
            break;
        case MVS_HYP_LINEAR:
            inv0 = __fadd_rn(hyp_a[o], __fmul_rn(0.f, hyp_b[o]));
            inv1 = __fadd_rn(hyp_a[o], __fmul_rn(1.f, hyp_b[o]));
            break;
        case MVS_HYP_REFINE:
            inv0 = max_nan(__fadd_rn(hyp_a[o], __fmul_rn((float)t0, hyp_b[o])), 1e-6f);
            inv1 = max_nan(__fadd_rn(hyp_a[o], __fmul_rn((float)(1 + t0), hyp_b[o])), 1e-6f);
            break;
        default:
            inv0 = plane0;
            inv1 = plane1;
    }
    depth[o] = finalize_pixel(inv0, inv1, n, best[o], spb[o], snb[o], idx[o]);
}

// ------------------------------------------------------------------------------ launcher

template <int R, int KMAX, bool PLANES, bool F16, bool X64, bool CMP, int TH>
static mvs_status launch_sweep(const SweepParams& p, dim3 grid, cudaStream_t st) {
    auto kern = sweep_kernel<R, KMAX, PLANES, F16, X64, CMP, TH>;
    const size_t smem = Geom<R, TH>::smem_bytes() + (CMP ? Geom<R, TH>::count_bytes() : 0);
    // the attribute is per function and per device: set it for the current device every time
    MVS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "sweep: shared memory attribute");
    kern<<<grid, TileShape<TH>::NT, smem, st>>>(p);
    return check_launch("sweep kernel");
}

template <int KMAX, bool PLANES, bool F16, bool X64 = false, bool CMP = false, int TH = TH_DEFAULT>
static mvs_status dispatch_r(int r, const SweepParams& p, dim3 grid, cudaStream_t st) {
    switch (r) {
        case 0: return launch_sweep<0, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 1: return launch_sweep<1, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 2: return launch_sweep<2, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 3: return launch_sweep<3, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 4: return launch_sweep<4, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 5: return launch_sweep<5, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 6: return launch_sweep<6, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
        case 7: return launch_sweep<7, KMAX, PLANES, F16, X64, CMP, TH>(p, grid, st);
    }
    return fail(MVS_ERR_VALUE, "sweep: window radius %d outside 0..%d", r, MVS_MAX_RADIUS);
}

static mvs_status dispatch(int r, int kmax, bool planes, int precision, int th, const SweepParams& p, dim3 grid,
                           cudaStream_t st) {
    const bool f16 = precision == MVS_PREC_FP16 || precision == MVS_PREC_FP16_COMP;
    if (th != TH_DEFAULT) {   // the other tile shapes: FP32 / FP16-storage plane sweeps, 2-entry lists
        if (!planes || kmax > 2 || (precision != MVS_PREC_FP32 && precision != MVS_PREC_FP16))
            return fail(MVS_ERR_UNSUPPORTED, "sweep: tile height %d needs an FP32 or FP16 plane sweep with top_k <= 2", th);
        if (th == 16) return f16 ? dispatch_r<2, true, true, false, false, 16>(r, p, grid, st)
                                 : dispatch_r<2, true, false, false, false, 16>(r, p, grid, st);
        return f16 ? dispatch_r<2, true, true, false, false, 64>(r, p, grid, st)
                   : dispatch_r<2, true, false, false, false, 64>(r, p, grid, st);
    }
    if (precision == MVS_PREC_FP32_COMP || precision == MVS_PREC_FP16_COMP) {
        if (!planes || kmax > 2) return fail(MVS_ERR_UNSUPPORTED, "sweep: compensated sums need MVS_HYP_PLANES and top_k <= 2");
        return f16 ? dispatch_r<2, true, true, false, true>(r, p, grid, st)
                   : dispatch_r<2, true, false, false, true>(r, p, grid, st);
    }
    if (precision == MVS_PREC_FP64_SUMS) {
        if (planes) return kmax <= 2 ? dispatch_r<2, true, false, true>(r, p, grid, st)
                                     : dispatch_r<8, true, false, true>(r, p, grid, st);
        return kmax <= 2 ? dispatch_r<2, false, false, true>(r, p, grid, st) : dispatch_r<8, false, false, true>(r, p, grid, st);
    }
    if (planes) {
        if (f16) return kmax <= 2 ? dispatch_r<2, true, true>(r, p, grid, st) : dispatch_r<8, true, true>(r, p, grid, st);
        return kmax <= 2 ? dispatch_r<2, true, false>(r, p, grid, st) : dispatch_r<8, true, false>(r, p, grid, st);
    }
    if (f16) return fail(MVS_ERR_UNSUPPORTED, "sweep: FP16 storage needs MVS_HYP_PLANES");
    return kmax <= 2 ? dispatch_r<2, false, false>(r, p, grid, st) : dispatch_r<8, false, false>(r, p, grid, st);
}

// 3x3 helpers (row-major, double)
static void mat_mul(const double* a, const double* b, double* o) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

mvs_status validate_sweep(const mvs_sweep_args* a) {
    if (!a) return fail(MVS_ERR_VALUE, "sweep: null arguments");
    if (a->n_src < 1 || a->n_src > MVS_MAX_SOURCES) return fail(MVS_ERR_VALUE, "sweep_hypothesis needs 1..16 sources");
    if (a->H < 0 || a->W < 0) return fail(MVS_ERR_VALUE, "sweep: negative image shape");
    if (a->r < 0) return fail(MVS_ERR_VALUE, "sweep_hypothesis: negative window radius");
    if (a->r > MVS_MAX_RADIUS) return fail(MVS_ERR_UNSUPPORTED, "sweep: window radius %d above %d", a->r, MVS_MAX_RADIUS);
    if (a->top_k < 1) return fail(MVS_ERR_VALUE, "sweep: top_k must be >= 1");
    if (!a->geo) return fail(MVS_ERR_VALUE, "geo must be (n_sources, 18)");
    if (a->i1 < a->i0) return fail(MVS_ERR_VALUE, "sweep: empty or reversed hypothesis range");
    if (a->precision < MVS_PREC_FP32 || a->precision > MVS_PREC_FP16_COMP)
        return fail(MVS_ERR_VALUE, "sweep: unknown precision");
    if (a->tile_h != 0 && a->tile_h != 16 && a->tile_h != 32 && a->tile_h != 64)
        return fail(MVS_ERR_VALUE, "sweep: tile height %d is not 0, 16, 32 or 64", a->tile_h);
    if (tile_height(a) != TH_DEFAULT &&
        (a->hyp.kind != MVS_HYP_PLANES || (a->precision != MVS_PREC_FP32 && a->precision != MVS_PREC_FP16) ||
         (a->top_k < a->n_src ? a->top_k : a->n_src) > 2))
        return fail(MVS_ERR_UNSUPPORTED, "sweep: tile height %d needs an FP32 or FP16 plane sweep with top_k <= 2",
                    a->tile_h);
    const int kind = a->hyp.kind;
    if (kind < MVS_HYP_MAPS || kind > MVS_HYP_PLANES) return fail(MVS_ERR_VALUE, "sweep: unknown hypothesis kind");
    if (a->H == 0 || a->W == 0) return MVS_OK;
    if (!a->ref || !a->mu || !a->sd || !a->best || !a->prev || !a->s_prev_best || !a->s_next_best || !a->idx)
        return fail(MVS_ERR_VALUE, "sweep: null image or state pointer");
    for (int s = 0; s < a->n_src; ++s) {
        if (!a->src[s]) return fail(MVS_ERR_VALUE, "sweep: null source %d", s);
        if (a->src_h[s] < 2 || a->src_w[s] < 2) return fail(MVS_ERR_VALUE, "sweep: source %d smaller than 2x2", s);
    }
    if (kind == MVS_HYP_PLANES) {
        if (!a->hyp.planes || !a->ref_cam) return fail(MVS_ERR_VALUE, "sweep: PLANES needs planes and ref_cam");
        if (a->hyp.n < a->i1) return fail(MVS_ERR_VALUE, "sweep: plane list shorter than i1");
        const double* rc = a->ref_cam;
        if (rc[13] != 0.0 || rc[14] != 0.0 || rc[15] != 0.0 || rc[12] == 0.0)
            return fail(MVS_ERR_VALUE, "sweep: PLANES needs a pinhole reference camera");
        for (int s = 0; s < a->n_src; ++s) {
            const double* g = a->geo + 18 * s;
            if (g[13] != 0.0 || g[14] != 0.0 || g[15] != 0.0)
                return fail(MVS_ERR_VALUE, "sweep: PLANES needs pinhole source cameras (source %d)", s);
        }
    } else {
        if (!a->ray) return fail(MVS_ERR_VALUE, "sweep: ray grid required for per-pixel hypotheses");
        if (kind == MVS_HYP_MAPS && !a->hyp.maps) return fail(MVS_ERR_VALUE, "sweep: null hypothesis maps");
        if ((kind == MVS_HYP_LINEAR || kind == MVS_HYP_REFINE) && (!a->hyp.base || !a->hyp.step))
            return fail(MVS_ERR_VALUE, "sweep: null hypothesis base/step");
    }
    if ((a->precision == MVS_PREC_FP16 || a->precision == MVS_PREC_FP16_COMP) && kind != MVS_HYP_PLANES)
        return fail(MVS_ERR_UNSUPPORTED, "sweep: FP16 storage needs MVS_HYP_PLANES");
    if ((a->precision == MVS_PREC_FP32_COMP || a->precision == MVS_PREC_FP16_COMP) &&
        (kind != MVS_HYP_PLANES || (a->top_k < a->n_src ? a->top_k : a->n_src) > 2))
        return fail(MVS_ERR_UNSUPPORTED, "sweep: compensated sums need MVS_HYP_PLANES and top_k <= 2");
    return MVS_OK;
}

// Fills the plane-invariant part of the kernel parameters (sources, geometry, state pointers).
// try_wait iterations of the sweep's bounded TMA wait (mvs_set_wait_limit; tests only lower it)
static std::atomic<unsigned> g_wait_limit{MVS_WAIT_LIMIT_DEFAULT};

mvs_status fill_params(const mvs_sweep_args* a, SweepParams& p) {
    memset(&p, 0, sizeof(p));
    p.wait_limit = g_wait_limit.load(std::memory_order_relaxed);
    p.H = a->H;
    p.W = a->W;
    p.n_src = a->n_src;
    const int kk = a->top_k < a->n_src ? a->top_k : a->n_src;
    p.kk = kk;
    p.topk_bottom = 0;
    p.hyp_kind = a->hyp.kind;
    p.t0 = a->hyp.t0;
    p.map_stride = a->hyp.map_stride ? a->hyp.map_stride : (long long)a->H * a->W;
    p.ref = a->ref;
    p.mu = a->mu;
    p.sd = a->sd;
    p.ray = a->ray;
    p.hyp_a = a->hyp.kind == MVS_HYP_MAPS ? a->hyp.maps : a->hyp.base;
    p.hyp_b = a->hyp.step;
    p.best = a->best;
    p.prev = a->prev;
    p.spb = a->s_prev_best;
    p.snb = a->s_next_best;
    p.idx = a->idx;
    double Ainv[9] = {0}, RrT[9] = {0};
    if (a->hyp.kind == MVS_HYP_PLANES) {
        const double* rc = a->ref_cam;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) RrT[3 * i + j] = rc[3 * j + i];
        const double f = rc[12], cx = rc[16], cy = rc[17];
        const double Kinv[9] = {1.0 / f, 0.0, -cx / f, 0.0, 1.0 / f, -cy / f, 0.0, 0.0, 1.0};
        mat_mul(RrT, Kinv, Ainv);   // R_ref^T K_ref^-1
    }
    for (int s = 0; s < a->n_src; ++s) {
        const double* g = a->geo + 18 * s;
        SrcGeo& d = p.src[s];
        d.img = a->src[s];
        d.h = a->src_h[s];
        d.w = a->src_w[s];
        if (a->hyp.kind == MVS_HYP_PLANES) mat_mul(g, Ainv, d.m);
        else for (int k = 0; k < 9; ++k) d.m[k] = g[k];
        for (int k = 0; k < 3; ++k) d.b[k] = g[9 + k];
        d.f = g[12]; d.k1 = g[13]; d.k2 = g[14]; d.k3 = g[15]; d.cx = g[16]; d.cy = g[17];
    }
    return MVS_OK;
}

// Picks the top-k representation: keep min(kk, n - kk) values (top list or bottom list).
int pick_kmax(SweepParams& p) {
    const int n = p.n_src, kk = p.kk;
    if (kk <= 2) { p.topk_bottom = 0; return 2; }
    if (kk <= 8) { p.topk_bottom = 0; return 8; }
    p.topk_bottom = 1;   // n - kk < 8 because n <= 16 and kk > 8
    return 8;
}

int auto_plane_chunks(int tiles, int nplanes) {
    const int target = num_sms() * 6;         // ~3 waves of 2 resident CTAs per SM
    if (tiles >= target || nplanes < 8) return 1;
    int c = (target + tiles - 1) / tiles;
    const int maxc = nplanes / 4;             // keep >= 4 planes per chunk
    if (c > maxc) c = maxc;
    return c < 1 ? 1 : c;
}

mvs_status sweep_range(const mvs_sweep_args* a, int i0, int i1, float* rec_ws, int nchunks, cudaStream_t st) {
    SweepParams p;
    MVS_TRY(fill_params(a, p));
    const int kmax = pick_kmax(p);
    p.i0 = i0;
    p.i1 = i1;
    const int n = i1 - i0;
    if (a->hyp.kind == MVS_HYP_PLANES) {
        for (int j = 0; j < n; ++j) p.planes[j] = a->hyp.planes[i0 + j];
    }
    if (a->hyp.kind == MVS_HYP_MAPS) {
        // maps are indexed from the caller's i0; shift the base for later sub-ranges
        p.hyp_a = a->hyp.maps + (long long)(i0 - a->i0) * p.map_stride;
    }
    p.ppc = (n + nchunks - 1) / nchunks;
    const int th = tile_height(a);
    p.ref_tma = make_ref_map(p, a->ref, a->H, a->W, a->r, th) ? 1 : 0;
    const int used = (n + p.ppc - 1) / p.ppc;
    p.rec = used > 1 ? rec_ws : nullptr;
    p.nchunks = used;
    p.r = a->r;
    dim3 grid((a->W + TW - 1) / TW, (a->H + th - 1) / th, used);
    MVS_TRY(dispatch(a->r, kmax, a->hyp.kind == MVS_HYP_PLANES, a->precision, th, p, grid, st));
    if (used > 1) {
        const long long HW = (long long)a->H * a->W;
        merge_kernel<<<(unsigned)((HW + 255) / 256), 256, 0, st>>>(HW, used, i0, i1, p.ppc, rec_ws, a->best, a->prev,
                                                       a->s_prev_best, a->s_next_best, a->idx);
        MVS_TRY(check_launch("sweep merge kernel"));
    }
    return MVS_OK;
}

// Bytes of chunk-record scratch one sweep call needs (0 when a single chunk suffices).
size_t sweep_scratch_bytes(const mvs_sweep_args* a, int* nchunks_out) {
    const int th = tile_height(a);
    const int tiles = ((a->W + TW - 1) / TW) * ((a->H + th - 1) / th);
    const int nplanes = a->i1 - a->i0;
    const int per_call = nplanes < MVS_MAX_PLANES_PER_CALL ? nplanes : MVS_MAX_PLANES_PER_CALL;
    int nch = a->plane_chunks > 0 ? a->plane_chunks : auto_plane_chunks(tiles, per_call);
    if (nch > per_call) nch = per_call < 1 ? 1 : per_call;
    *nchunks_out = nch;
    if (nch <= 1) return 0;
    return (size_t)6 * nch * a->H * a->W * sizeof(float);
}

mvs_status sweep_with_scratch(const mvs_sweep_args* a, void* scratch, size_t scratch_bytes, cudaStream_t st) {
    int nch = 1;
    const size_t need = sweep_scratch_bytes(a, &nch);
    if (need > scratch_bytes) return fail(MVS_ERR_VALUE, "sweep: scratch of %zu bytes below the %zu needed", scratch_bytes, need);
    for (int i = a->i0; i < a->i1; i += MVS_MAX_PLANES_PER_CALL) {
        const int e = (a->i1 - i) < MVS_MAX_PLANES_PER_CALL ? a->i1 : i + MVS_MAX_PLANES_PER_CALL;
        int nc = nch;
        if (nc > e - i) nc = e - i;
        MVS_TRY(sweep_range(a, i, e, reinterpret_cast<float*>(scratch), nc, st));
    }
    return MVS_OK;
}

}  // namespace mvs

using namespace mvs;

extern "C" mvs_status mvs_sweep(const mvs_sweep_args* a, void* stream) {
    clear_error();
    MVS_TRY(validate_sweep(a));
    if (a->H == 0 || a->W == 0 || a->i1 == a->i0) return MVS_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int nch = 1;
    const size_t need = sweep_scratch_bytes(a, &nch);
    void* ws = nullptr;
    if (need) MVS_CUDA(cudaMallocAsync(&ws, need, st), "sweep: chunk-record scratch");
    mvs_status s = sweep_with_scratch(a, ws, need, st);
    if (ws) cudaFreeAsync(ws, st);
    return s;
}

extern "C" mvs_status mvs_sweep_hypothesis(int32_t H, int32_t W, const float* ref, const float* mu_i,
                                           const float* sd_i, int32_t n_src, const float* const* srcs,
                                           const int32_t* src_h, const int32_t* src_w, const float* ray,
                                           const double* geo, const float* inv, int32_t r, int32_t top_k,
                                           int32_t i, float* best, float* prev, float* s_prev_best,
                                           float* s_next_best, int32_t* idx, void* stream) {
    clear_error();
    if (n_src < 1 || n_src > MVS_MAX_SOURCES) return fail(MVS_ERR_VALUE, "sweep_hypothesis needs 1..16 sources");
    if (!srcs || !src_h || !src_w) return fail(MVS_ERR_VALUE, "sweep_hypothesis: null source table");
    mvs_sweep_args a;
    memset(&a, 0, sizeof(a));
    a.H = H; a.W = W; a.ref = ref; a.mu = mu_i; a.sd = sd_i; a.ray = ray; a.n_src = n_src;
    a.precision = MVS_PREC_FP32;
    for (int s = 0; s < n_src; ++s) { a.src[s] = srcs[s]; a.src_h[s] = src_h[s]; a.src_w[s] = src_w[s]; }
    a.geo = geo;
    a.hyp.kind = MVS_HYP_MAPS; a.hyp.n = i + 1; a.hyp.maps = inv; a.hyp.map_stride = (int64_t)H * W;
    a.i0 = i; a.i1 = i + 1; a.r = r; a.top_k = top_k; a.plane_chunks = 1;
    a.best = best; a.prev = prev; a.s_prev_best = s_prev_best; a.s_next_best = s_next_best; a.idx = idx;
    MVS_TRY(validate_sweep(&a));
    if (H == 0 || W == 0) return MVS_OK;
    if (!inv) return fail(MVS_ERR_VALUE, "sweep_hypothesis: null inverse-depth map");
    return sweep_range(&a, i, i + 1, nullptr, 1, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" mvs_status mvs_sweep_finalize(int32_t H, int32_t W, const mvs_hyp* hyp, const float* best,
                                         const float* s_prev_best, const float* s_next_best, const int32_t* idx,
                                         float* depth, void* stream) {
    clear_error();
    if (!hyp) return fail(MVS_ERR_VALUE, "finalize: null hypothesis description");
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "finalize: negative shape");
    if (H == 0 || W == 0) return MVS_OK;
    if (hyp->n < 1) return fail(MVS_ERR_VALUE, "finalize: needs at least one hypothesis");
    if (!best || !s_prev_best || !s_next_best || !idx || !depth) return fail(MVS_ERR_VALUE, "finalize: null pointer");
    float p0 = 0.f, p1 = 0.f;
    if (hyp->kind == MVS_HYP_PLANES) {
        if (!hyp->planes) return fail(MVS_ERR_VALUE, "finalize: null plane list");
        p0 = hyp->planes[0];
        p1 = hyp->n > 1 ? hyp->planes[1] : p0;
    } else if (hyp->kind == MVS_HYP_MAPS) {
        if (!hyp->maps) return fail(MVS_ERR_VALUE, "finalize: null maps");
    } else if (hyp->kind == MVS_HYP_LINEAR || hyp->kind == MVS_HYP_REFINE) {
        if (!hyp->base || !hyp->step) return fail(MVS_ERR_VALUE, "finalize: null base/step");
    } else {
        return fail(MVS_ERR_VALUE, "finalize: unknown hypothesis kind");
    }
    const long long HW = (long long)H * W;
    const long long stride = hyp->map_stride ? hyp->map_stride : HW;
    const float* a = hyp->kind == MVS_HYP_MAPS ? hyp->maps : hyp->base;
    finalize_kernel<<<(unsigned)((HW + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        H, W, hyp->kind, hyp->n, hyp->t0, a, hyp->step, stride, p0, p1, best, s_prev_best, s_next_best, idx, depth);
    return check_launch("finalize kernel");
}

extern "C" uint32_t mvs_set_wait_limit(uint32_t iterations) {
    return g_wait_limit.exchange(iterations);
}

extern "C" mvs_status mvs_device_faults(uint32_t* count) {
    clear_error();
    unsigned n = 0;
    MVS_CUDA(cudaMemcpyFromSymbol(&n, g_ref_copy_faults, sizeof(n)), "device faults: read");
    if (n) {
        const unsigned zero = 0;
        MVS_CUDA(cudaMemcpyToSymbol(g_ref_copy_faults, &zero, sizeof(zero)), "device faults: clear");
    }
    if (count) *count = n;
    return n ? fail(MVS_ERR_TIMEOUT, "%u sweep tile(s) gave up waiting for their reference copy", n) : MVS_OK;
}

unsigned mvs::take_bound_violations_sweep() { return take_bound_violations_here(); }
