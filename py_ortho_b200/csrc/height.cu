// The legacy ground-grid height sweep of the reference (mvs.dense_reconstruct, mvs.py:138-434) on
// the device: the view sampler (_mvs.sample_view, _mvs.pyx:13-58, the CPU twin of the CuPy kernel
// in _cuda.py:88-124), the float64 summed-area box mean (_fast.box_sat_mean, _fast.pyx:897-942),
// the photo-consistency score of a stack of height hypotheses (score_at, mvs.py:254-304) and the
// 8-path semi-global aggregation (_mvs.sgm, _mvs.pyx:98-251).
//
// This file is compiled with -fmad=false: every float64 / float32 expression is evaluated with one
// rounding per operation in the written order, as the reference's C and NumPy evaluate it, so the
// sampler, the box means and the aggregation are bit-identical to the reference's.
#include "common.cuh"

namespace mvs {

// ---------------------------------------------------------------- sampler
struct SampleParams {
    int h, w, nch, D, H, W;
    double R[9], C[3], f, k1, k2, k3, cx, cy, X0, Y0, gsd;
    const float* img;
    const float* Z;
    float* out;
    unsigned char* valid;
};

__global__ void __launch_bounds__(256) sample_view_kernel(const __grid_constant__ SampleParams p) {
    const long long n = (long long)p.D * p.H * p.W;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)(i % p.W);
    const int r = (int)((i / p.W) % p.H);
    const double Y = p.Y0 - ((double)r + 0.5) * p.gsd;
    const double X = p.X0 + ((double)c + 0.5) * p.gsd;
    const double dx = X - p.C[0], dy = Y - p.C[1], dz = (double)p.Z[i] - p.C[2];
    const double zc = p.R[6] * dx + p.R[7] * dy + p.R[8] * dz;
    float* o = p.out + i * p.nch;
    bool ok = zc > 1e-6;
    double u = 0.0, v = 0.0;
    if (ok) {
        const double xc = p.R[0] * dx + p.R[1] * dy + p.R[2] * dz;
        const double yc = p.R[3] * dx + p.R[4] * dy + p.R[5] * dz;
        const double nx = xc / zc, ny = yc / zc;
        const double r2 = nx * nx + ny * ny;
        const double d = 1.0 + r2 * (p.k1 + r2 * (p.k2 + r2 * p.k3));
        u = p.f * d * nx + p.cx;
        v = p.f * d * ny + p.cy;
        // NaN positions fail every comparison of the reference's test and are sampled there as
        // garbage; here they are invalid
        ok = u >= 0.0 && v >= 0.0 && u <= (double)(p.w - 1) && v <= (double)(p.h - 1);
    }
    if (!ok) {
        for (int ch = 0; ch < p.nch; ++ch) o[ch] = 0.f;
        p.valid[i] = 0;
        return;
    }
    const int x0 = (int)u, y0 = (int)v;
    const int x1 = x0 + 1 < p.w ? x0 + 1 : x0, y1 = y0 + 1 < p.h ? y0 + 1 : y0;
    const double fx = u - (double)x0, fy = v - (double)y0;
    for (int ch = 0; ch < p.nch; ++ch) {
        const double a00 = p.img[((long long)y0 * p.w + x0) * p.nch + ch];
        const double a01 = p.img[((long long)y0 * p.w + x1) * p.nch + ch];
        const double a10 = p.img[((long long)y1 * p.w + x0) * p.nch + ch];
        const double a11 = p.img[((long long)y1 * p.w + x1) * p.nch + ch];
        o[ch] = (float)((1 - fy) * ((1 - fx) * a00 + fx * a01) + fy * ((1 - fx) * a10 + fx * a11));
    }
    p.valid[i] = 1;
}

// ---------------------------------------------------------------- float64 summed-area box mean
// Padded table S (PH = H + 2r + 1 rows, PW = W + 2r + 1 columns) per plane, built as the reference
// builds its ring rows: column sums down the rows (one thread per column), then a running total of
// those along each row (one thread per row); the window mean takes the four corners in the
// reference's order.
__global__ void box_cols_kernel(int B, int H, int W, int r, const float* __restrict__ a, double* __restrict__ cs) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)B * W) return;
    const int b = (int)(t / W), x = (int)(t - (long long)b * W);
    const int PH = H + 2 * r + 1;
    const float* ab = a + (long long)b * H * W;
    double* cb = cs + (long long)b * PH * W;
    double col = 0.0;
    for (int i = 0; i < PH; ++i) {
        const int ay = i - r - 1;
        const double val = (ay >= 0 && ay < H) ? (double)ab[(long long)ay * W + x] : 0.0;
        col = col + val;
        cb[(long long)i * W + x] = col;
    }
}

__global__ void box_rows_kernel(int B, int H, int W, int r, const double* __restrict__ cs, double* __restrict__ sat) {
    const int PH = H + 2 * r + 1, PW = W + 2 * r + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)B * PH) return;
    const long long b = t / PH, i = t - b * PH;
    const double* row = cs + (b * PH + i) * W;
    double* cur = sat + (b * PH + i) * PW;
    double total = 0.0;
    for (int x = 0; x < r + 1; ++x) cur[x] = 0.0;
    for (int x = 0; x < W; ++x) {
        total = total + row[x];
        cur[x + r + 1] = total;
    }
    for (int x = r + 1 + W; x < PW; ++x) cur[x] = total;
}

__global__ void box_mean_kernel(int B, int H, int W, int r, const double* __restrict__ sat, float* __restrict__ out) {
    const long long n = (long long)B * H * W;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = 2 * r + 1, PH = H + 2 * r + 1, PW = W + 2 * r + 1;
    const int x = (int)(t % W);
    const int y = (int)((t / W) % H);
    const long long b = t / ((long long)H * W);
    const double* cur = sat + (b * PH + y + k) * PW;
    const double* old = sat + (b * PH + y) * PW;
    double val = cur[x + k] - old[x + k];
    val = val - cur[x];
    val = val + old[x];
    out[t] = (float)(val / ((double)k * (double)k));
}

// ---------------------------------------------------------------- score of height hypotheses
// score_at (mvs.py:254-304) after the sampling and the box means, for every cell of a (D, H, W)
// hypothesis stack and V views: the cell's reference view is the nearest camera (in X, Y) among
// those whose window is fully valid; the NCC of every other view against it (box statistics,
// variance floor 1e-6, -1 where either window is not full), the mean of the topk largest, scaled
// by the reference's texture strength. Arrays are (V or pairs, D, H, W) float32 planes:
//   M (box of S), S2 (box of S*S), VA (box of the valid mask), PP (box of S_a * S_b for the pairs
//   a < b in np.triu_indices order).
struct ScoreParams {
    int V, D, H, W, topk;
    float full, min_texture, full_texture;
    const float* M;
    const float* S2;
    const float* VA;
    const float* PP;
    const float* cxs;                 // (W) float32 cell centres, X
    const float* cys;                 // (H) float32 cell centres, Y
    float camx[16], camy[16];         // the views' centres, rounded to float32
    float* score;                     // (D, H, W)
    float* st;                        // (V, D, H, W) NCC against the cell's reference (-2: itself), or null
    int* ref;                         // (D, H, W) reference view, or null
};

__device__ __forceinline__ int pair_slot(int a, int b, int V) {   // np.triu_indices(V, 1) order, a < b
    return a * V - a * (a + 1) / 2 + (b - a - 1);
}

__global__ void __launch_bounds__(256) height_score_kernel(const __grid_constant__ ScoreParams p) {
    const long long plane = (long long)p.D * p.H * p.W;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= plane) return;
    const int x = (int)(i % p.W);
    const int y = (int)((i / p.W) % p.H);
    const int V = p.V;
    float var[16];
    bool full[16];
    // reference: argmin over views of (full ? d2 : inf), first index on ties (np.argmin)
    int ref = 0;
    float dmin = INFINITY;
    for (int v = 0; v < V; ++v) {
        const float m = p.M[v * plane + i];
        var[v] = __fsub_rn(p.S2[v * plane + i], __fmul_rn(m, m));
        full[v] = p.VA[v * plane + i] >= p.full;
        const float ey = __fsub_rn(p.cys[y], p.camy[v]), ex = __fsub_rn(p.cxs[x], p.camx[v]);
        const float d2 = __fadd_rn(__fmul_rn(ey, ey), __fmul_rn(ex, ex));
        const float dist = full[v] ? d2 : INFINITY;
        if (v == 0 || dist < dmin) {
            dmin = dist;
            ref = v;
        }
    }
    // NCC(ref, v) for every view
    float st[16];
    for (int v = 0; v < V; ++v) {
        if (v == ref) {
            st[v] = -2.f;
            continue;
        }
        const int a = min(ref, v), b = max(ref, v);
        const float cov = __fsub_rn(p.PP[pair_slot(a, b, V) * plane + i], __fmul_rn(p.M[a * plane + i], p.M[b * plane + i]));
        const float va = fmaxf(var[a], 1e-6f), vb = fmaxf(var[b], 1e-6f);
        const float ncc = __fdiv_rn(cov, __fsqrt_rn(__fmul_rn(va, vb)));
        st[v] = (full[a] && full[b]) ? ncc : -1.f;
    }
    if (p.st)
        for (int v = 0; v < V; ++v) p.st[v * plane + i] = st[v];
    // mean of the topk largest (summed in descending order)
    float top[16];
    for (int v = 0; v < V; ++v) top[v] = st[v];
    for (int a = 1; a < V; ++a) {                        // insertion sort, descending
        const float t = top[a];
        int b = a - 1;
        while (b >= 0 && top[b] < t) {
            top[b + 1] = top[b];
            --b;
        }
        top[b + 1] = t;
    }
    float sum = 0.f;
    for (int k = 0; k < p.topk; ++k) sum = __fadd_rn(sum, top[k]);
    float score = __fdiv_rn(sum, (float)p.topk);
    const float varR = var[ref];
    float tex = __fdiv_rn(__fsqrt_rn(fmaxf(varR, 0.f)), p.full_texture);
    tex = fminf(fmaxf(tex, 0.f), 1.f);
    const bool ok = isfinite(dmin) && varR > p.min_texture;
    p.score[i] = ok ? __fmul_rn(score, tex) : 0.f;
    if (p.ref) p.ref[i] = ref;
}

// ---------------------------------------------------------------- semi-global aggregation
// One direction of _mvs.sgm: a warp per line of cells along the direction (lanes over the depth
// values of a cell), the cells of a line in the reference's scan order; the previous cell's
// values are read back from L. agg += L for every cell as the reference adds the directions.
__global__ void __launch_bounds__(128) sgm_dir_kernel(int D, int H, int W, int dy, int dx, float P1, float P2,
                                                      const float* __restrict__ cost, float* __restrict__ L,
                                                      float* __restrict__ agg, int first) {
    const int lane = threadIdx.x & 31;
    const int line = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const long long HW = (long long)H * W;
    // lines: dy == 0 -> rows; dx == 0 -> columns; diagonals -> cells with a common x*dy - y*dx
    int nlines, y, x, len;
    if (dy == 0) {
        nlines = H;
        if (line >= nlines) return;
        y = line;
        x = dx > 0 ? 0 : W - 1;
        len = W;
    } else if (dx == 0) {
        nlines = W;
        if (line >= nlines) return;
        x = line;
        y = dy > 0 ? 0 : H - 1;
        len = H;
    } else {
        nlines = H + W - 1;
        if (line >= nlines) return;
        // start cells: the first row (scan side) for lines that start there, then the first column
        const int ys = dy > 0 ? 0 : H - 1, xs = dx > 0 ? 0 : W - 1;
        if (line < W) {
            y = ys;
            x = dx > 0 ? line : W - 1 - line;
        } else {
            x = xs;
            y = dy > 0 ? line - W + 1 : H - 1 - (line - W + 1);
        }
        const int ny = dy > 0 ? H - y : y + 1, nx = dx > 0 ? W - x : x + 1;
        len = ny < nx ? ny : nx;
    }
    const unsigned full = 0xffffffffu;
    for (int s = 0; s < len; ++s, y += dy, x += dx) {
        const long long o = (long long)y * W + x;
        if (s == 0) {
            for (int d = lane; d < D; d += 32) L[d * HW + o] = cost[d * HW + o];
        } else {
            const long long po = o - (long long)dy * W - dx;
            float best = INFINITY;
            for (int d = lane; d < D; d += 32) best = fminf(best, L[d * HW + po]);
            for (int m = 16; m > 0; m >>= 1) best = fminf(best, __shfl_xor_sync(full, best, m));
            for (int d = lane; d < D; d += 32) {
                float v = L[d * HW + po];
                if (d > 0) {
                    const float a = __fadd_rn(L[(d - 1) * HW + po], P1);
                    if (a < v) v = a;
                }
                if (d < D - 1) {
                    const float b = __fadd_rn(L[(d + 1) * HW + po], P1);
                    if (b < v) v = b;
                }
                const float bp = __fadd_rn(best, P2);
                if (bp < v) v = bp;
                L[d * HW + o] = __fsub_rn(__fadd_rn(cost[d * HW + o], v), best);
            }
        }
        for (int d = lane; d < D; d += 32) {
            const float l = L[d * HW + o];
            agg[d * HW + o] = first ? __fadd_rn(0.f, l) : __fadd_rn(agg[d * HW + o], l);
        }
        __syncwarp();
    }
}

}  // namespace mvs

using namespace mvs;

extern "C" mvs_status mvs_sample_view(const mvs_sample_view_args* a, void* stream) {
    clear_error();
    if (!a) return fail(MVS_ERR_VALUE, "sample_view: null arguments");
    if (a->h < 1 || a->w < 1 || a->nch < 1 || a->D < 0 || a->H < 0 || a->W < 0)
        return fail(MVS_ERR_VALUE, "sample_view: bad shapes");
    const long long n = (long long)a->D * a->H * a->W;
    if (n == 0) return MVS_OK;
    if (!a->img || !a->cam || !a->Z || !a->out || !a->valid) return fail(MVS_ERR_VALUE, "sample_view: null pointer");
    SampleParams p;
    memset(&p, 0, sizeof(p));
    p.h = a->h; p.w = a->w; p.nch = a->nch; p.D = a->D; p.H = a->H; p.W = a->W;
    for (int k = 0; k < 9; ++k) p.R[k] = a->cam[k];
    for (int k = 0; k < 3; ++k) p.C[k] = a->cam[9 + k];
    p.f = a->cam[12]; p.k1 = a->cam[13]; p.k2 = a->cam[14]; p.k3 = a->cam[15]; p.cx = a->cam[16]; p.cy = a->cam[17];
    p.X0 = a->X0; p.Y0 = a->Y0; p.gsd = a->gsd;
    p.img = a->img; p.Z = a->Z; p.out = a->out; p.valid = a->valid;
    sample_view_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p);
    return check_launch("sample_view kernel");
}

extern "C" mvs_status mvs_box_sat_mean(int32_t B, int32_t H, int32_t W, const float* a, int32_t r, float* out,
                                       void* stream) {
    clear_error();
    if (r < 0) return fail(MVS_ERR_VALUE, "radius must be nonnegative");
    if (B < 0 || H < 0 || W < 0) return fail(MVS_ERR_VALUE, "box_sat_mean: negative shape");
    if ((long long)B * H * W == 0) return MVS_OK;
    if (!a || !out) return fail(MVS_ERR_VALUE, "box_sat_mean: null pointer");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long PH = H + 2LL * r + 1, PW = W + 2LL * r + 1;
    const size_t cs_bytes = sizeof(double) * (size_t)B * PH * W, sat_bytes = sizeof(double) * (size_t)B * PH * PW;
    void* ws = nullptr;
    MVS_CUDA(cudaMallocAsync(&ws, cs_bytes + sat_bytes, st), "box_sat_mean: scratch");
    double* cs = reinterpret_cast<double*>(ws);
    double* sat = cs + (size_t)B * PH * W;
    box_cols_kernel<<<(unsigned)(((long long)B * W + 127) / 128), 128, 0, st>>>(B, H, W, r, a, cs);
    mvs_status s = check_launch("box columns");
    if (s == MVS_OK) {
        box_rows_kernel<<<(unsigned)(((long long)B * PH + 127) / 128), 128, 0, st>>>(B, H, W, r, cs, sat);
        s = check_launch("box rows");
    }
    if (s == MVS_OK) {
        const long long n = (long long)B * H * W;
        box_mean_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(B, H, W, r, sat, out);
        s = check_launch("box mean");
    }
    cudaFreeAsync(ws, st);
    return s;
}

extern "C" mvs_status mvs_height_score(const mvs_height_score_args* a, void* stream) {
    clear_error();
    if (!a) return fail(MVS_ERR_VALUE, "height_score: null arguments");
    if (a->V < 2 || a->V > 16) return fail(MVS_ERR_VALUE, "height_score: %d views (2..16)", a->V);
    if (a->topk < 1 || a->topk > a->V) return fail(MVS_ERR_VALUE, "height_score: topk %d outside 1..%d", a->topk, a->V);
    const long long n = (long long)a->D * a->H * a->W;
    if (n == 0) return MVS_OK;
    if (!a->M || !a->S2 || !a->VA || !a->PP || !a->cxs || !a->cys || !a->cam_xy || !a->score)
        return fail(MVS_ERR_VALUE, "height_score: null pointer");
    ScoreParams p;
    memset(&p, 0, sizeof(p));
    p.V = a->V; p.D = a->D; p.H = a->H; p.W = a->W; p.topk = a->topk;
    p.full = (float)a->full; p.min_texture = (float)a->min_texture; p.full_texture = (float)a->full_texture;
    p.M = a->M; p.S2 = a->S2; p.VA = a->VA; p.PP = a->PP; p.cxs = a->cxs; p.cys = a->cys;
    for (int v = 0; v < a->V; ++v) {
        p.camx[v] = (float)a->cam_xy[2 * v];
        p.camy[v] = (float)a->cam_xy[2 * v + 1];
    }
    p.score = a->score; p.st = a->st; p.ref = a->ref;
    height_score_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p);
    return check_launch("height score kernel");
}

extern "C" mvs_status mvs_sgm(int32_t D, int32_t H, int32_t W, const float* cost, float P1, float P2, float* agg,
                              void* stream) {
    clear_error();
    if (D < 0 || H < 0 || W < 0) return fail(MVS_ERR_VALUE, "sgm: negative shape");
    if ((long long)D * H * W == 0) return MVS_OK;
    if (!cost || !agg) return fail(MVS_ERR_VALUE, "sgm: null pointer");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    void* ws = nullptr;
    MVS_CUDA(cudaMallocAsync(&ws, sizeof(float) * (size_t)D * H * W, st), "sgm: scratch");
    float* L = reinterpret_cast<float*>(ws);
    static const int dirs[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    mvs_status s = MVS_OK;
    for (int k = 0; k < 8 && s == MVS_OK; ++k) {
        const int dy = dirs[k][0], dx = dirs[k][1];
        const int nlines = dy == 0 ? H : (dx == 0 ? W : H + W - 1);
        const long long threads = (long long)nlines * 32;
        sgm_dir_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(D, H, W, dy, dx, P1, P2, cost, L, agg,
                                                                          k == 0);
        s = check_launch("sgm direction");
    }
    cudaFreeAsync(ws, st);
    return s;
}
