// Batched plane sweep: many reference views of uneven size, source count, plane count and
// window radius in ONE persistent launch.
//
// The plan is a device work list of (job, tile_x, tile_y, plane-chunk) items ordered by cost,
// largest first (longest-processing-time order). Persistent CTAs (a multiple of the SM count)
// take items with one atomicAdd each, so no CTA waits on another and uneven jobs balance. A
// job's result does not depend on what else is in the batch: its per-pixel reduction order is
// fixed by hypothesis index (chunk records are merged in hypothesis order afterwards).
// run = [reset counter] -> [persistent sweep] -> [ordered chunk merge + parabola finalize],
// captured once into a CUDA graph and replayed.
#include <vector>
#include <algorithm>

#include "sweep_tile.cuh"

namespace mvs {

struct JobFin {                        // per-job table of the merge / finalize pass
    long long block0;                  // first block of this job in the finalize grid
    long long HW;
    int nchunks, ppc, i0, i1, n;
    float p0, p1;
    const float* rec;
    float* best;
    float* prev;
    float* spb;
    float* snb;
    int* idx;
    float* depth;
};

// One radius of the tile engine as an out-of-line call: the persistent kernel dispatches on the
// work item's radius, and keeping each instance out of line gives each its own register
// allocation (inlined together, the largest instance's pressure spilled the others).
template <int R, int KMAX, bool F16, bool WIDE, int TH>
__device__ __noinline__ void batch_tile(const SweepParams& p, int tx, int ty, int pa, int pb, int ch, float* smem) {
    sweep_tile<R, KMAX, true, F16, WIDE, false, false, false, TH>(p, tx, ty, pa, pb, ch, smem);
}

// TH: the plan's tile height (one shape per persistent launch; 64 x TH tiles on 8 TH threads)
template <int RMAX, int KMAX, bool F16, int TH = TH_DEFAULT>
__global__ void __launch_bounds__(TileShape<TH>::NT, TileShape<TH>::MIN_CTAS)
    batch_kernel(const SweepParams* __restrict__ jobs, const int4* __restrict__ items, int n_items, int* counter) {
    extern __shared__ float4 smem4[];
    __shared__ int s_item;
    float* smem = reinterpret_cast<float*>(smem4);
    for (;;) {
        __syncthreads();                   // everyone has read the previous s_item
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const int4 w = items[it];
        const SweepParams& p = jobs[w.x];
        const int pa = p.i0 + w.w * p.ppc;
        const int pb = min(p.i1, pa + p.ppc);
        // a job with one record buffer (nchunks == 1: serving) always writes record 0
        const int ch = p.rec ? (p.nchunks == 1 ? 0 : w.w) : -1;
        const int tx = w.y * TW, ty = w.z * TH;
        // the radius is uniform per work item: each case is the single-view instance itself
        switch (p.r) {
            case 0: batch_tile<0, KMAX, F16, false, TH>(p, tx, ty, pa, pb, ch, smem); break;
            case 1: batch_tile<1, KMAX, F16, false, TH>(p, tx, ty, pa, pb, ch, smem); break;
            case 2: batch_tile<2, KMAX, F16, true, TH>(p, tx, ty, pa, pb, ch, smem); break;
            case 3: batch_tile<3, KMAX, F16, true, TH>(p, tx, ty, pa, pb, ch, smem); break;
            default:
                if constexpr (RMAX > 3) {
                    switch (p.r) {
                        case 4: batch_tile<4, KMAX, F16, true, TH>(p, tx, ty, pa, pb, ch, smem); break;
                        case 5: batch_tile<5, KMAX, F16, true, TH>(p, tx, ty, pa, pb, ch, smem); break;
                        case 6: batch_tile<6, KMAX, F16, true, TH>(p, tx, ty, pa, pb, ch, smem); break;
                        default: batch_tile<7, KMAX, F16, true, TH>(p, tx, ty, pa, pb, ch, smem); break;
                    }
                }
        }
    }
}

__global__ void batch_finalize_kernel(const JobFin* __restrict__ jobs, int n_jobs) {
    // locate the job of this block (jobs are few; binary search over block0)
    int lo = 0, hi = n_jobs - 1;
    const long long blk = blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (jobs[mid].block0 <= blk) lo = mid; else hi = mid - 1;
    }
    const JobFin& j = jobs[lo];
    const long long o = (blk - j.block0) * blockDim.x + threadIdx.x;
    if (o >= j.HW) return;
    float B, P, SP, SN;
    int I;
    if (j.rec) {
        B = -2.f; P = -2.f; SP = -2.f; SN = -2.f; I = -1;
        merge_pixel(o, j.HW, j.nchunks, j.i0, j.i1, j.ppc, j.rec, B, P, SP, SN, I);
        j.best[o] = B;
        j.prev[o] = P;
        j.spb[o] = SP;
        j.snb[o] = SN;
        j.idx[o] = I;
    } else {
        B = j.best[o]; SP = j.spb[o]; SN = j.snb[o]; I = j.idx[o];
    }
    if (j.depth) j.depth[o] = finalize_pixel(j.p0, j.p1, j.n, B, SP, SN, I);
}

template <int RMAX, int KMAX, bool F16, int TH = TH_DEFAULT>
static mvs_status batch_attr(int* max_ctas_per_sm) {
    auto kern = batch_kernel<RMAX, KMAX, F16, TH>;
    const size_t smem = smem_bytes_upto<RMAX, TH>();
    MVS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "batch: smem attribute");
    MVS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(max_ctas_per_sm, kern, TileShape<TH>::NT, smem),
             "batch: occupancy");
    return MVS_OK;
}

template <int RMAX, int KMAX, bool F16, int TH = TH_DEFAULT>
static void batch_launch(dim3 grid, cudaStream_t st, const SweepParams* jobs, const int4* items, int n, int* counter) {
    batch_kernel<RMAX, KMAX, F16, TH><<<grid, TileShape<TH>::NT, smem_bytes_upto<RMAX, TH>(), st>>>(jobs, items, n,
                                                                                                 counter);
}

// The plan's kernel for radius class RMAX (3 or 7), list size KMAX (2 or 8), storage and tile
// height: attribute query (Q) or launch. Tile heights 16 and 64 exist for 2-entry lists only.
template <int RMAX, int KMAX, bool F16>
static mvs_status batch_select(int th, bool query, int* cps, dim3 grid, cudaStream_t st, const SweepParams* jobs,
                               const int4* items, int n, int* counter) {
    if constexpr (KMAX == 2) {
        if (th == 16) {
            if (query) return batch_attr<RMAX, 2, F16, 16>(cps);
            batch_launch<RMAX, 2, F16, 16>(grid, st, jobs, items, n, counter);
            return MVS_OK;
        }
        if (th == 64) {
            if (query) return batch_attr<RMAX, 2, F16, 64>(cps);
            batch_launch<RMAX, 2, F16, 64>(grid, st, jobs, items, n, counter);
            return MVS_OK;
        }
    }
    if (th != TH_DEFAULT) return fail(MVS_ERR_UNSUPPORTED, "batch: tile height %d needs top_k <= 2", th);
    if (query) return batch_attr<RMAX, KMAX, F16>(cps);
    batch_launch<RMAX, KMAX, F16>(grid, st, jobs, items, n, counter);
    return MVS_OK;
}

static mvs_status batch_kernel_for(int rmax, int kmax, bool f16, int th, bool query, int* cps, dim3 grid,
                                   cudaStream_t st, const SweepParams* jobs, const int4* items, int n, int* counter) {
    if (rmax <= 3) {
        if (kmax <= 2) return f16 ? batch_select<3, 2, true>(th, query, cps, grid, st, jobs, items, n, counter)
                                  : batch_select<3, 2, false>(th, query, cps, grid, st, jobs, items, n, counter);
        return f16 ? batch_select<3, 8, true>(th, query, cps, grid, st, jobs, items, n, counter)
                   : batch_select<3, 8, false>(th, query, cps, grid, st, jobs, items, n, counter);
    }
    if (kmax <= 2) return f16 ? batch_select<7, 2, true>(th, query, cps, grid, st, jobs, items, n, counter)
                              : batch_select<7, 2, false>(th, query, cps, grid, st, jobs, items, n, counter);
    return f16 ? batch_select<7, 8, true>(th, query, cps, grid, st, jobs, items, n, counter)
               : batch_select<7, 8, false>(th, query, cps, grid, st, jobs, items, n, counter);
}

}  // namespace mvs

using namespace mvs;

struct mvs_batch {
    int n_jobs = 0;
    int rmax = 3, kmax = 2;
    bool f16 = false;
    int th = TH_DEFAULT;               // tile height of the plan
    int grid = 0;
    int n_items = 0;
    long long evals = 0;
    long long fin_blocks = 0;
    SweepParams* d_params = nullptr;
    int4* d_items = nullptr;
    int* d_counter = nullptr;
    float* d_rec = nullptr;
    JobFin* d_fin = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static mvs_status batch_enqueue(mvs_batch* b, cudaStream_t st) {
    MVS_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(int), st), "batch: reset counter");
    const dim3 grid(b->grid);
    MVS_TRY(batch_kernel_for(b->rmax, b->kmax, b->f16, b->th, false, nullptr, grid, st, b->d_params, b->d_items,
                             b->n_items, b->d_counter));
    MVS_TRY(check_launch("batch persistent kernel"));
    batch_finalize_kernel<<<(unsigned)b->fin_blocks, 256, 0, st>>>(b->d_fin, b->n_jobs);
    return check_launch("batch finalize kernel");
}

static void batch_free(mvs_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    cudaFree(b->d_params);
    cudaFree(b->d_items);
    cudaFree(b->d_counter);
    cudaFree(b->d_rec);
    cudaFree(b->d_fin);
    delete b;
}

extern "C" mvs_status mvs_batch_create(const mvs_batch_job* jobs, int32_t n_jobs, const mvs_batch_tuning* tuning,
                                       mvs_batch** out) {
    clear_error();
    if (!out) return fail(MVS_ERR_VALUE, "batch: null output handle");
    *out = nullptr;
    if (!jobs || n_jobs < 1) return fail(MVS_ERR_VALUE, "batch: needs at least one job");
    const int pc_req = tuning ? tuning->plane_chunk : 0;
    const int cps_req = tuning ? tuning->ctas_per_sm : 0;
    const int th = tuning && tuning->tile_h ? tuning->tile_h : TH_DEFAULT;
    if (pc_req < 0 || cps_req < 0) return fail(MVS_ERR_VALUE, "batch: negative tuning value");
    if (th != 16 && th != 32 && th != 64) return fail(MVS_ERR_VALUE, "batch: tile height %d is not 0, 16, 32 or 64", th);
    std::vector<SweepParams> params(n_jobs);
    std::vector<JobFin> fin(n_jobs);
    std::vector<int4> items;
    std::vector<long long> cost;
    long long rec_floats = 0;
    mvs_batch* b = new mvs_batch();
    b->n_jobs = n_jobs;
    b->th = th;
    b->f16 = jobs[0].sweep.precision == MVS_PREC_FP16;
    int rmax = 0, kmax = 2;
    std::vector<long long> rec_off(n_jobs, -1);
    for (int j = 0; j < n_jobs; ++j) {
        // the plan's tile height applies to every job (the jobs' own tile_h is not read)
        mvs_sweep_args ja = jobs[j].sweep;
        ja.tile_h = 0;
        const mvs_sweep_args* a = &ja;
        mvs_status st = validate_sweep(a);
        if (st != MVS_OK) { batch_free(b); return st; }
        if (a->hyp.kind != MVS_HYP_PLANES) { batch_free(b); return fail(MVS_ERR_VALUE, "batch: job %d must use MVS_HYP_PLANES", j); }
        if (a->precision == MVS_PREC_FP64_SUMS || a->precision == MVS_PREC_FP32_COMP || a->precision == MVS_PREC_FP16_COMP) {
            batch_free(b);
            return fail(MVS_ERR_UNSUPPORTED, "batch: float64 and compensated window sums run on the single-view kernel (mvs_sweep) only");
        }
        if ((a->precision == MVS_PREC_FP16) != b->f16) { batch_free(b); return fail(MVS_ERR_VALUE, "batch: all jobs need the same precision"); }
        if (a->i1 - a->i0 > MVS_MAX_PLANES_PER_CALL) { batch_free(b); return fail(MVS_ERR_VALUE, "batch: job %d has more than %d planes", j, MVS_MAX_PLANES_PER_CALL); }
        if (a->H == 0 || a->W == 0 || a->i1 == a->i0) { batch_free(b); return fail(MVS_ERR_VALUE, "batch: job %d is empty", j); }
        SweepParams& p = params[j];
        st = fill_params(a, p);
        if (st != MVS_OK) { batch_free(b); return st; }
        kmax = std::max(kmax, pick_kmax(p));
        rmax = std::max(rmax, a->r);
        const int n = a->i1 - a->i0;
        for (int k = 0; k < n; ++k) p.planes[k] = a->hyp.planes[a->i0 + k];
        p.i0 = a->i0;
        p.i1 = a->i1;
        p.r = a->r;
        p.fresh = 1;
        const int pc = pc_req > 0 ? std::min(pc_req, n) : n;
        p.ppc = pc;
        p.nchunks = (n + pc - 1) / pc;
        const int tx = (a->W + TW - 1) / TW, ty = (a->H + th - 1) / th;
        if (p.nchunks > 1) {
            rec_off[j] = rec_floats;
            rec_floats += (long long)6 * p.nchunks * a->H * a->W;
        }
        for (int ch = 0; ch < p.nchunks; ++ch) {
            const int planes = std::min(pc, n - ch * pc);
            for (int y = 0; y < ty; ++y)
                for (int x = 0; x < tx; ++x) {
                    items.push_back(make_int4(j, x, y, ch));
                    cost.push_back((long long)planes * a->n_src * (TW + 2 * a->r) * (th + 2 * a->r));
                }
        }
        b->evals += (long long)a->H * a->W * n * a->n_src;
        JobFin& f = fin[j];
        f.HW = (long long)a->H * a->W;
        f.nchunks = p.nchunks; f.ppc = pc; f.i0 = a->i0; f.i1 = a->i1; f.n = a->hyp.n;
        f.p0 = a->hyp.planes[0];
        f.p1 = a->hyp.n > 1 ? a->hyp.planes[1] : f.p0;
        f.best = a->best; f.prev = a->prev; f.spb = a->s_prev_best; f.snb = a->s_next_best; f.idx = a->idx;
        f.depth = jobs[j].depth;
    }
    b->rmax = rmax <= 3 ? 3 : 7;
    b->kmax = kmax;
    if (th != TH_DEFAULT && kmax > 2) {
        batch_free(b);
        return fail(MVS_ERR_UNSUPPORTED, "batch: tile height %d needs top_k <= 2 in every job", th);
    }
    // largest items first
    std::vector<int> order(items.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    std::vector<int4> sorted(items.size());
    for (size_t i = 0; i < order.size(); ++i) sorted[i] = items[order[i]];
    b->n_items = (int)sorted.size();

    int max_cps = 0;
    mvs_status st = batch_kernel_for(b->rmax, b->kmax, b->f16, th, true, &max_cps, dim3(1), nullptr, nullptr, nullptr,
                                     0, nullptr);
    if (st != MVS_OK) { batch_free(b); return st; }
    if (max_cps < 1) { batch_free(b); return fail(MVS_ERR_CUDA, "batch: kernel does not fit on an SM"); }
    const int cps = cps_req > 0 ? std::min(cps_req, max_cps) : max_cps;
    b->grid = num_sms() * cps;

#define BATCH_ALLOC(ptr, bytes, what)                                                       \
    do {                                                                                    \
        cudaError_t e__ = cudaMalloc((void**)&(ptr), (bytes));                              \
        if (e__ != cudaSuccess) { batch_free(b); return fail(MVS_ERR_MEMORY, "batch: %s: %s", what, cudaGetErrorString(e__)); } \
    } while (0)
    BATCH_ALLOC(b->d_params, sizeof(SweepParams) * n_jobs, "job table");
    BATCH_ALLOC(b->d_items, sizeof(int4) * sorted.size(), "work list");
    BATCH_ALLOC(b->d_counter, sizeof(int), "counter");
    if (rec_floats) BATCH_ALLOC(b->d_rec, sizeof(float) * rec_floats, "chunk records");
    BATCH_ALLOC(b->d_fin, sizeof(JobFin) * n_jobs, "finalize table");
#undef BATCH_ALLOC
    long long blocks = 0;
    for (int j = 0; j < n_jobs; ++j) {
        if (rec_off[j] >= 0) {
            params[j].rec = b->d_rec + rec_off[j];
            fin[j].rec = params[j].rec;
        } else {
            params[j].rec = nullptr;
            fin[j].rec = nullptr;
        }
        fin[j].block0 = blocks;
        blocks += (fin[j].HW + 255) / 256;
    }
    b->fin_blocks = blocks;
    cudaError_t e = cudaMemcpy(b->d_params, params.data(), sizeof(SweepParams) * n_jobs, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_items, sorted.data(), sizeof(int4) * sorted.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_fin, fin.data(), sizeof(JobFin) * n_jobs, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { batch_free(b); return fail(MVS_ERR_CUDA, "batch: upload: %s", cudaGetErrorString(e)); }
    *out = b;
    return MVS_OK;
}

extern "C" mvs_status mvs_batch_run(mvs_batch* b, int32_t use_graph, void* stream) {
    clear_error();
    if (!b) return fail(MVS_ERR_VALUE, "batch: null handle");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);   // NULL = legacy default stream
    if (!use_graph) return batch_enqueue(b, st);
    if (!b->exec) {
        // capture on the private stream (capture is not possible on the legacy default stream);
        // the instantiated graph then runs on the caller's stream
        MVS_CUDA(cudaStreamBeginCapture(b->own_stream, cudaStreamCaptureModeThreadLocal), "batch: begin capture");
        mvs_status s = batch_enqueue(b, b->own_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->own_stream, &g);
        if (s != MVS_OK) { if (g) cudaGraphDestroy(g); return s; }
        if (e != cudaSuccess) return fail(MVS_ERR_CUDA, "batch: end capture: %s", cudaGetErrorString(e));
        b->graph = g;
        MVS_CUDA(cudaGraphInstantiate(&b->exec, g, 0), "batch: instantiate graph");
    }
    MVS_CUDA(cudaGraphLaunch(b->exec, st), "batch: graph launch");
    return MVS_OK;
}

extern "C" mvs_status mvs_batch_stats(const mvs_batch* b, int64_t* work_items, int64_t* evals) {
    clear_error();
    if (!b) return fail(MVS_ERR_VALUE, "batch: null handle");
    if (work_items) *work_items = b->n_items;
    if (evals) *evals = b->evals;
    return MVS_OK;
}

extern "C" void mvs_batch_destroy(mvs_batch* b) { batch_free(b); }

// ------------------------------------------------------------------------------ serving engine

namespace mvs {

struct StepMerge {                     // one (job, chunk) of a serving step
    long long block0;
    long long HW;
    int pa, pb;
    const float* rec;
    float* best;
    float* prev;
    float* spb;
    float* snb;
    int* idx;
};

__global__ void server_merge_kernel(const StepMerge* __restrict__ m, int n) {
    int lo = 0, hi = n - 1;
    const long long blk = blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (m[mid].block0 <= blk) lo = mid; else hi = mid - 1;
    }
    const StepMerge& j = m[lo];
    const long long o = (blk - j.block0) * blockDim.x + threadIdx.x;
    if (o >= j.HW) return;
    float B = j.best[o], P = j.prev[o], SP = j.spb[o], SN = j.snb[o];
    int I = j.idx[o];
    merge_pixel(o, j.HW, 1, j.pa, j.pb, j.pb - j.pa, j.rec, B, P, SP, SN, I);
    j.best[o] = B;
    j.prev[o] = P;
    j.spb[o] = SP;
    j.snb[o] = SN;
    j.idx[o] = I;
}

}  // namespace mvs

struct mvs_server {
    int max_slots = 0, max_items = 0, rmax = 3;
    bool f16 = false;
    int kmax = 2;
    int grid = 0;
    SweepParams* d_params = nullptr;
    std::vector<SweepParams> h_params;
    std::vector<char> used;
    int4* d_items = nullptr;
    int4* h_items = nullptr;           // pinned
    StepMerge* d_merge = nullptr;
    StepMerge* h_merge = nullptr;      // pinned
    int* d_counter = nullptr;
    cudaEvent_t uploaded = nullptr;
};

static void server_free(mvs_server* s) {
    if (!s) return;
    if (s->uploaded) cudaEventDestroy(s->uploaded);
    cudaFree(s->d_params);
    cudaFree(s->d_items);
    cudaFree(s->d_merge);
    cudaFree(s->d_counter);
    cudaFreeHost(s->h_items);
    cudaFreeHost(s->h_merge);
    delete s;
}

extern "C" mvs_status mvs_server_create(int32_t max_slots, int32_t max_items, int32_t max_radius, int32_t precision,
                                        mvs_server** out) {
    clear_error();
    if (!out) return fail(MVS_ERR_VALUE, "server: null output handle");
    *out = nullptr;
    if (max_slots < 1 || max_items < 1) return fail(MVS_ERR_VALUE, "server: needs slots and items");
    if (max_radius < 0 || max_radius > MVS_MAX_RADIUS) return fail(MVS_ERR_VALUE, "server: radius outside 0..%d", MVS_MAX_RADIUS);
    if (precision == MVS_PREC_FP64_SUMS || precision == MVS_PREC_FP32_COMP || precision == MVS_PREC_FP16_COMP)
        return fail(MVS_ERR_UNSUPPORTED, "server: float64 and compensated window sums run on the single-view kernel (mvs_sweep) only");
    if (precision != MVS_PREC_FP32 && precision != MVS_PREC_FP16) return fail(MVS_ERR_VALUE, "server: unknown precision");
    mvs_server* s = new mvs_server();
    s->max_slots = max_slots;
    s->max_items = max_items;
    s->rmax = max_radius <= 3 ? 3 : 7;
    s->f16 = precision == MVS_PREC_FP16;
    s->h_params.resize(max_slots);
    s->used.assign(max_slots, 0);
    int cps = 0;
    mvs_status st = s->rmax <= 3 ? (s->f16 ? batch_attr<3, 2, true>(&cps) : batch_attr<3, 2, false>(&cps))
                                 : (s->f16 ? batch_attr<7, 2, true>(&cps) : batch_attr<7, 2, false>(&cps));
    if (st != MVS_OK) { server_free(s); return st; }
    s->grid = num_sms() * (cps > 0 ? cps : 1);
    cudaError_t e = cudaMalloc((void**)&s->d_params, sizeof(SweepParams) * max_slots);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->d_items, sizeof(int4) * max_items);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->d_merge, sizeof(StepMerge) * max_slots);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->d_counter, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_items, sizeof(int4) * max_items);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_merge, sizeof(StepMerge) * max_slots);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming);
    if (e != cudaSuccess) { server_free(s); return fail(MVS_ERR_MEMORY, "server: allocation: %s", cudaGetErrorString(e)); }
    *out = s;
    return MVS_OK;
}

extern "C" mvs_status mvs_server_set_job(mvs_server* s, int32_t slot, const mvs_sweep_args* job, float* chunk_rec,
                                         int32_t plane_chunk) {
    clear_error();
    if (!s || !job) return fail(MVS_ERR_VALUE, "server: null argument");
    if (slot < 0 || slot >= s->max_slots) return fail(MVS_ERR_VALUE, "server: slot %d outside 0..%d", slot, s->max_slots - 1);
    MVS_TRY(validate_sweep(job));
    if (job->hyp.kind != MVS_HYP_PLANES) return fail(MVS_ERR_VALUE, "server: jobs must use MVS_HYP_PLANES");
    if (job->precision == MVS_PREC_FP64_SUMS || job->precision == MVS_PREC_FP32_COMP || job->precision == MVS_PREC_FP16_COMP)
        return fail(MVS_ERR_UNSUPPORTED, "server: float64 and compensated window sums run on the single-view kernel (mvs_sweep) only");
    if ((job->precision == MVS_PREC_FP16) != s->f16) return fail(MVS_ERR_VALUE, "server: job precision differs from the server's");
    if (job->r > (s->rmax <= 3 ? 3 : 7)) return fail(MVS_ERR_VALUE, "server: job radius above the server's");
    if (job->i1 - job->i0 > MVS_MAX_PLANES_PER_CALL || job->i1 <= job->i0) return fail(MVS_ERR_VALUE, "server: bad plane range");
    if (job->H == 0 || job->W == 0) return fail(MVS_ERR_VALUE, "server: empty job");
    if (!chunk_rec || plane_chunk < 1) return fail(MVS_ERR_VALUE, "server: needs a chunk record buffer and plane_chunk >= 1");
    SweepParams p;
    MVS_TRY(fill_params(job, p));
    if (pick_kmax(p) > 2) return fail(MVS_ERR_UNSUPPORTED, "server: top_k needs more than 2 list entries");
    const int n = job->i1 - job->i0;
    for (int k = 0; k < n; ++k) p.planes[k] = job->hyp.planes[job->i0 + k];
    p.i0 = job->i0;
    p.i1 = job->i1;
    p.r = job->r;
    p.fresh = 1;
    p.ppc = plane_chunk;
    p.nchunks = 1;                     // one record buffer: chunk records always land in record 0
    p.rec = chunk_rec;
    s->h_params[slot] = p;
    s->used[slot] = 1;
    MVS_CUDA(cudaMemcpy(s->d_params + slot, &p, sizeof(SweepParams), cudaMemcpyHostToDevice), "server: upload job");
    return MVS_OK;
}

extern "C" mvs_status mvs_server_step(mvs_server* s, const int32_t* slots, const int32_t* chunks, int32_t n,
                                      void* stream) {
    clear_error();
    if (!s) return fail(MVS_ERR_VALUE, "server: null handle");
    if (n <= 0) return MVS_OK;
    if (!slots || !chunks || n > s->max_slots) return fail(MVS_ERR_VALUE, "server: bad step list");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    MVS_CUDA(cudaEventSynchronize(s->uploaded), "server: previous upload");   // host buffers free again
    int items = 0;
    long long blocks = 0;
    for (int k = 0; k < n; ++k) {
        const int sl = slots[k];
        if (sl < 0 || sl >= s->max_slots || !s->used[sl]) return fail(MVS_ERR_VALUE, "server: slot %d holds no job", sl);
        for (int q = 0; q < k; ++q)
            if (slots[q] == sl) return fail(MVS_ERR_VALUE, "server: slot %d twice in one step", sl);
        const SweepParams& p = s->h_params[sl];
        const int pa = p.i0 + chunks[k] * p.ppc;
        if (chunks[k] < 0 || pa >= p.i1) return fail(MVS_ERR_VALUE, "server: chunk %d beyond job %d", chunks[k], sl);
        const int tx = (p.W + TW - 1) / TW, ty = (p.H + TH_DEFAULT - 1) / TH_DEFAULT;
        if (items + tx * ty > s->max_items) return fail(MVS_ERR_VALUE, "server: step exceeds %d work items", s->max_items);
        for (int y = 0; y < ty; ++y)
            for (int x = 0; x < tx; ++x) s->h_items[items++] = make_int4(sl, x, y, chunks[k]);
        StepMerge& m = s->h_merge[k];
        m.block0 = blocks;
        m.HW = (long long)p.H * p.W;
        m.pa = pa;
        m.pb = std::min(p.i1, pa + p.ppc);
        m.rec = p.rec;
        m.best = p.best; m.prev = p.prev; m.spb = p.spb; m.snb = p.snb; m.idx = p.idx;
        blocks += (m.HW + 255) / 256;
    }
    MVS_CUDA(cudaMemcpyAsync(s->d_items, s->h_items, sizeof(int4) * items, cudaMemcpyHostToDevice, st), "server: items");
    MVS_CUDA(cudaMemcpyAsync(s->d_merge, s->h_merge, sizeof(StepMerge) * n, cudaMemcpyHostToDevice, st), "server: merge table");
    MVS_CUDA(cudaEventRecord(s->uploaded, st), "server: record upload");
    MVS_CUDA(cudaMemsetAsync(s->d_counter, 0, sizeof(int), st), "server: counter");
    const dim3 grid(s->grid);
    if (s->rmax <= 3) {
        if (s->f16) batch_launch<3, 2, true>(grid, st, s->d_params, s->d_items, items, s->d_counter);
        else batch_launch<3, 2, false>(grid, st, s->d_params, s->d_items, items, s->d_counter);
    } else {
        if (s->f16) batch_launch<7, 2, true>(grid, st, s->d_params, s->d_items, items, s->d_counter);
        else batch_launch<7, 2, false>(grid, st, s->d_params, s->d_items, items, s->d_counter);
    }
    MVS_TRY(check_launch("server persistent kernel"));
    server_merge_kernel<<<(unsigned)blocks, 256, 0, st>>>(s->d_merge, n);
    return check_launch("server merge kernel");
}

extern "C" void mvs_server_destroy(mvs_server* s) { server_free(s); }

unsigned mvs::take_bound_violations_batch() { return take_bound_violations_here(); }
