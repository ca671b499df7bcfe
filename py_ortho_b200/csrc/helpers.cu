// Per-view helpers of the depth-map path: reference window statistics, ray grid, hypothesis
// maps, image preparation and the 2x2 pyramid. Each reproduces the reference helper's float32 /
// float64 rounding steps (no contraction: explicit _rn intrinsics), so results are identical
// to _fast.pyx / densify.py on the same inputs.
#include "common.cuh"

namespace mvs {

static thread_local char g_err[512];

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void clear_error() { g_err[0] = 0; }

// ---- _fast.box_zero_mean (_fast.pyx:661-713): column cumsum over rows padded (r+1, r), window
// difference c[y+k] - c[y]; then the same along each row; times float32(1/k^2). The two
// cumulative sums are sequential float32 sums, so each column / row is one thread (the lead and
// lag values c[y+k], c[y] follow the identical add sequence, so no table is stored).
__device__ __forceinline__ float box_in(const float* a, long long o, int sq) {
    const float v = a[o];
    return sq ? __fmul_rn(v, v) : v;
}

__global__ void box_col_kernel(int H, int W, const float* __restrict__ a, int r, int sq, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W) return;
    const int k = 2 * r + 1;
    auto val = [&](int i) -> float {       // padded row i
        const int ay = i - (r + 1);
        return (ay < 0 || ay >= H) ? 0.f : box_in(a, (long long)ay * W + x, sq);
    };
    float lag = val(0), lead = val(0);
    for (int i = 1; i <= k; ++i) lead = __fadd_rn(lead, val(i));
    for (int y = 0; y < H; ++y) {
        out[(long long)y * W + x] = __fsub_rn(lead, lag);
        lag = __fadd_rn(lag, val(y + 1));
        lead = __fadd_rn(lead, val(y + k + 1));
    }
}

// one CTA per row: stage the row in shared memory, scan sequentially, write back coalesced
__global__ void box_row_kernel(int H, int W, int r, float scale, float* __restrict__ io) {
    extern __shared__ float row[];        // 2 * W
    float* res = row + W;
    const int y = blockIdx.x;
    float* p = io + (long long)y * W;
    for (int x = threadIdx.x; x < W; x += blockDim.x) row[x] = p[x];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int k = 2 * r + 1;
        auto t = [&](int j) -> float {     // padded (r+1 left, r right)
            const int ax = j - (r + 1);
            return (ax < 0 || ax >= W) ? 0.f : row[ax];
        };
        float lag = t(0), lead = t(0);
        for (int j = 1; j <= k; ++j) lead = __fadd_rn(lead, t(j));
        for (int x = 0; x < W; ++x) {
            res[x] = __fmul_rn(__fsub_rn(lead, lag), scale);
            lag = __fadd_rn(lag, t(x + 1));
            lead = __fadd_rn(lead, t(x + k + 1));
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < W; x += blockDim.x) p[x] = res[x];
}

// sd = sqrt(max(b2 - mu*mu, 1e-6)) in float32 (densify.py:328), in place over b2.
__global__ void sd_kernel(long long n, const float* __restrict__ mu, float* b2sd) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float m = mu[i];
    const float v = __fsub_rn(b2sd[i], __fmul_rn(m, m));
    b2sd[i] = __fsqrt_rn(max_nan(v, 1e-6f));
}

mvs_status box_zero_mean(int H, int W, const float* a, int r, int sq, float* out, cudaStream_t st) {
    if (H == 0 || W == 0) return MVS_OK;
    box_col_kernel<<<(W + 127) / 128, 128, 0, st>>>(H, W, a, r, sq, out);
    MVS_TRY(check_launch("box column pass"));
    const int k = 2 * r + 1;
    const float scale = (float)(1.0 / ((double)k * k));
    const size_t smem = (size_t)2 * W * sizeof(float);
    if (smem > 48 * 1024) {
        MVS_CUDA(cudaFuncSetAttribute(box_row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "box: shared memory attribute");
    }
    box_row_kernel<<<H, 128, smem, st>>>(H, W, r, scale, out);
    return check_launch("box row pass");
}

// ---- rays: _fast._undistort (_fast.pyx:145-164) + densify._rays_world (densify.py:288-297)
__global__ void rays_kernel(int H, int W, double R0, double R1, double R2, double R3, double R4, double R5,
                            double R6, double R7, double R8, double f, double k1, double k2, double k3, double cx,
                            double cy, float* __restrict__ ray) {
    const long long HW = (long long)H * W;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= HW) return;
    const int row = (int)(o / W), col = (int)(o - (long long)row * W);
    const double nx = __ddiv_rn(__dsub_rn((double)col, cx), f);
    const double ny = __ddiv_rn(__dsub_rn((double)row, cy), f);
    double x = nx, y = ny;
    for (int it = 0; it < 8; ++it) {
        double r2 = __dmul_rn(x, x);
        const double t = __dmul_rn(y, y);
        r2 = __dadd_rn(r2, t);
        double d = __dmul_rn(r2, k3);
        d = __dadd_rn(k2, d);
        d = __dmul_rn(r2, d);
        d = __dadd_rn(k1, d);
        d = __dmul_rn(r2, d);
        d = __dadd_rn(1.0, d);
        x = __ddiv_rn(nx, d);
        y = __ddiv_rn(ny, d);
    }
    // ray_w[i] = sum_j R[j][i] * (x, y, 1)[j]
    const double Rm[9] = {R0, R1, R2, R3, R4, R5, R6, R7, R8};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double acc = __dmul_rn(Rm[i], x);
        acc = __dadd_rn(acc, __dmul_rn(Rm[3 + i], y));
        acc = __dadd_rn(acc, Rm[6 + i]);
        ray[i * HW + o] = (float)acc;
    }
}

__global__ void hyp_linear_kernel(long long n, const float* __restrict__ base, const float* __restrict__ step,
                                  float fi, float* __restrict__ out) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    out[o] = __fadd_rn(base[o], __fmul_rn(fi, step[o]));
}

__global__ void hyp_refine_kernel(long long n, const float* __restrict__ iu, const float* __restrict__ ds,
                                  float ft, float* __restrict__ out) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const float v = __fadd_rn(iu[o], __fmul_rn(ft, ds[o]));
    out[o] = max_nan(v, 1e-6f);
}

// _fast.depth_view (_fast.pyx:577-624)
__global__ void depth_view_kernel(long long n, const uint8_t* __restrict__ rgb, int has_g, float g0, float g1,
                                  float g2, int has_b, float b0, float b1, float b2, const uint8_t* __restrict__ mask,
                                  float* __restrict__ grey, uint8_t* __restrict__ rgb8) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    float v[3];
    const float g[3] = {g0, g1, g2}, b[3] = {b0, b1, b2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        v[c] = (float)rgb[3 * o + c];
        if (has_g) v[c] = __fmul_rn(v[c], g[c]);
        if (has_b) v[c] = __fadd_rn(v[c], b[c]);
    }
    float s = __fadd_rn(v[0], v[1]);
    s = __fadd_rn(s, v[2]);
    s = __fdiv_rn(s, 3.0f);
    s = __fsub_rn(s, 128.0f);
    s = __fdiv_rn(s, 64.0f);
    grey[o] = (mask && !mask[o]) ? __int_as_float(0x7fc00000) : s;
    if (rgb8) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float t = __fadd_rn(v[c], 0.5f);
            // _clip32 then the C cast to unsigned char (truncation); NaN clips to 0
            t = (t > 255.f) ? 255.f : (t >= 0.f ? t : 0.f);
            rgb8[3 * o + c] = (uint8_t)t;
        }
    }
}

// densify._half (densify.py:127-130) over `planes` stacked images
__global__ void half_kernel(int planes, int h, int w, const float* __restrict__ in, float* __restrict__ out) {
    const int h2 = h / 2, w2 = w / 2;
    const long long n = (long long)planes * h2 * w2;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int pl = (int)(o / ((long long)h2 * w2));
    const long long rem = o - (long long)pl * h2 * w2;
    const int y = (int)(rem / w2), x = (int)(rem - (long long)y * w2);
    const float* p = in + (long long)pl * h * w;
    const float a00 = p[(long long)(2 * y) * w + 2 * x], a10 = p[(long long)(2 * y + 1) * w + 2 * x];
    const float a01 = p[(long long)(2 * y) * w + 2 * x + 1], a11 = p[(long long)(2 * y + 1) * w + 2 * x + 1];
    float s = __fadd_rn(a00, a10);
    s = __fadd_rn(s, a01);
    s = __fadd_rn(s, a11);
    out[o] = __fmul_rn(s, 0.25f);
}

__global__ void to_fp16_kernel(long long n, const float* __restrict__ in, __half* __restrict__ out) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    out[o] = __float2half_rn(in[o]);
}

// ---- tie-point geometry of the coarse-to-fine driver (densify._depth_range / _depth_band)

// Camera coordinates of a world point as NumPy's (X - C) @ R^T: OpenBLAS's dgemm accumulates each
// output as a = d0 r0; a = fma(d1, r1, a); a = fma(d2, r2, a).
__device__ __forceinline__ void tie_cam_coords(const double* cam, const double* X, double* xc) {
    const double d0 = __dsub_rn(X[0], cam[9]), d1 = __dsub_rn(X[1], cam[10]), d2 = __dsub_rn(X[2], cam[11]);
#pragma unroll
    for (int j = 0; j < 3; ++j)
        xc[j] = __fma_rn(d2, cam[3 * j + 2], __fma_rn(d1, cam[3 * j + 1], __dmul_rn(d0, cam[3 * j])));
}

struct TieCam {
    double c[18];   // R(9) C(3) f k1 k2 k3 cx cy
};

// One tie point: its camera-axis depth if it lands inside the w x h view under the pinhole map
// u = f x / z + cx (the range census), else NaN.
__global__ void tie_depths_kernel(int n, const double* __restrict__ X, const TieCam cam, int w, int h,
                                  double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xc[3];
    tie_cam_coords(cam.c, X + 3LL * i, xc);
    const double f = cam.c[12], cx = cam.c[16], cy = cam.c[17];
    const double u = __dadd_rn(__ddiv_rn(__dmul_rn(f, xc[0]), xc[2]), cx);
    const double v = __dadd_rn(__ddiv_rn(__dmul_rn(f, xc[1]), xc[2]), cy);
    const bool in = xc[2] > 0.0 && u >= 0.0 && v >= 0.0 && u < (double)w && v < (double)h;
    out[i] = in ? xc[2] : __longlong_as_double(0x7ff8000000000000LL);
}

// NumPy's floor division of a non-negative double by a positive integer: exact (the remainder
// from fmod is exact, so a - fmod(a, b) is a multiple of b).
__device__ __forceinline__ int floor_div_pos(double a, int b) {
    const double bd = (double)b;
    return (int)__ddiv_rn(__dsub_rn(a, fmod(a, bd)), bd);
}

// Scatter of the observed tie points into block x block cells of the sweep image: per cell the
// count and the min / max camera depth. Depths are > 0 here, so their bit patterns order like the
// values and the extrema are integer atomics (order-independent: the same cell values in any
// order).
__global__ void band_scatter_kernel(int n, const double* __restrict__ X, const TieCam cam, int H, int W, int block,
                                    int gw, unsigned long long* __restrict__ zlo, unsigned long long* __restrict__ zhi,
                                    int* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xc[3];
    tie_cam_coords(cam.c, X + 3LL * i, xc);
    if (!(xc[2] > 0.0)) return;
    // _Cam.project_cam: pinhole + radial k1..k3, z floored at 1e-6
    const double* c = cam.c;
    const double z = fmax(xc[2], 1e-6);
    const double x = __ddiv_rn(xc[0], z), y = __ddiv_rn(xc[1], z);
    const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    const double poly =
        __dadd_rn(1.0, __dmul_rn(r2, __dadd_rn(c[13], __dmul_rn(r2, __dadd_rn(c[14], __dmul_rn(r2, c[15]))))));
    const double d = __dmul_rn(c[12], poly);
    const double u = __dadd_rn(__dmul_rn(d, x), c[16]), v = __dadd_rn(__dmul_rn(d, y), c[17]);
    if (!(u >= 0.0 && v >= 0.0 && u < (double)W && v < (double)H)) return;
    const int bx = floor_div_pos(fmin(u, (double)(W - 1)), block);
    const int by = floor_div_pos(fmin(v, (double)(H - 1)), block);
    const int b = by * gw + bx;
    const unsigned long long zb = (unsigned long long)__double_as_longlong(xc[2]);
    atomicMin(zlo + b, zb);
    atomicMax(zhi + b, zb);
    atomicAdd(cnt + b, 1);
}

__global__ void band_init_kernel(int nb, unsigned long long* zlo, unsigned long long* zhi, int* cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    zlo[i] = 0x7FF0000000000000ULL;   // +inf
    zhi[i] = 0ULL;                    // +0 (every scattered depth is larger)
    cnt[i] = 0;
}

// Per pixel: the band of its cell. A cell with >= 5 points takes the depth extent of the points
// in its 3 x 3 cell neighbourhood (cells with >= 5 points only), widened by margin + 5 % of that
// extent and clipped to the view's range; other cells take the view's range. Out: float32
// base = 1 / hi and step = (1 / max(lo, 1e-6) - base) / max(nd - 1, 1) of the coarse sweep.
__global__ void band_fill_kernel(int H, int W, int block, int gh, int gw, const unsigned long long* __restrict__ zlo,
                                 const unsigned long long* __restrict__ zhi, const int* __restrict__ cnt, double lo_g,
                                 double hi_g, double margin, int nd, int uniform, float* __restrict__ base,
                                 float* __restrict__ step, float* __restrict__ inv_hi) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    float il, ih;
    if (uniform) {
        il = __double2float_rn(__ddiv_rn(1.0, hi_g));
        ih = __double2float_rn(__ddiv_rn(1.0, lo_g));
    } else {
        const int bx = x / block, by = y / block;
        double lo3 = __longlong_as_double(0x7FF0000000000000LL), hi3 = -lo3;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int cy = by + dy, cx = bx + dx;
                if (cy < 0 || cx < 0 || cy >= gh || cx >= gw) continue;
                const int b = cy * gw + cx;
                if (cnt[b] < 5) continue;
                lo3 = fmin(lo3, __longlong_as_double((long long)zlo[b]));
                hi3 = fmax(hi3, __longlong_as_double((long long)zhi[b]));
            }
        const bool has = cnt[by * gw + bx] >= 5 && isfinite(lo3) && isfinite(hi3);
        double lob = lo_g, hib = hi_g;
        if (has) {
            const double pad = __dadd_rn(margin, __dmul_rn(0.05, __dsub_rn(hi3, lo3)));
            lob = fmin(fmax(__dsub_rn(lo3, pad), lo_g), hi_g);
            hib = fmin(fmax(__dadd_rn(hi3, pad), lo_g), hi_g);
        }
        il = __double2float_rn(__ddiv_rn(1.0, hib));
        ih = __double2float_rn(__ddiv_rn(1.0, fmax(lob, 1e-6)));
    }
    const long long o = (long long)y * W + x;
    base[o] = il;
    step[o] = __fdiv_rn(__fsub_rn(ih, il), (float)max(nd - 1, 1));
    if (inv_hi) inv_hi[o] = ih;
}

static inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace mvs

using namespace mvs;

extern "C" size_t mvs_last_error(char* buf, size_t cap) {
    const size_t n = strlen(g_err);
    if (buf && cap) {
        const size_t m = n < cap - 1 ? n : cap - 1;
        memcpy(buf, g_err, m);
        buf[m] = 0;
    }
    return n;
}

extern "C" const char* mvs_version(void) { return "libmvs_b200 0.1.0 (sm_100a)"; }

extern "C" mvs_status mvs_box_zero_mean(int32_t H, int32_t W, const float* a, int32_t r, int32_t square,
                                        float* out, void* stream) {
    clear_error();
    if (r < 0) return fail(MVS_ERR_VALUE, "box_zero_mean needs r >= 0");
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "box_zero_mean: negative shape");
    if (H == 0 || W == 0) return MVS_OK;
    if (!a || !out) return fail(MVS_ERR_VALUE, "box_zero_mean: null pointer");
    if (a == out) return fail(MVS_ERR_VALUE, "box_zero_mean: input and output must differ");
    return box_zero_mean(H, W, a, r, square, out, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" mvs_status mvs_ref_stats(int32_t H, int32_t W, const float* ref, int32_t r, float* mu, float* sd,
                                    void* stream) {
    clear_error();
    if (r < 0) return fail(MVS_ERR_VALUE, "ref_stats: negative window radius");
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "ref_stats: negative shape");
    if (H == 0 || W == 0) return MVS_OK;
    if (!ref || !mu || !sd || mu == sd || ref == mu || ref == sd) return fail(MVS_ERR_VALUE, "ref_stats: bad pointers");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    MVS_TRY(box_zero_mean(H, W, ref, r, 0, mu, st));
    MVS_TRY(box_zero_mean(H, W, ref, r, 1, sd, st));
    const long long n = (long long)H * W;
    sd_kernel<<<blocks(n, 256), 256, 0, st>>>(n, mu, sd);
    return check_launch("ref_stats sd");
}

extern "C" mvs_status mvs_rays_grid(int32_t H, int32_t W, const double* c, float* ray, void* stream) {
    clear_error();
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "rays_grid: negative shape");
    if (H == 0 || W == 0) return MVS_OK;
    if (!c || !ray) return fail(MVS_ERR_VALUE, "rays_grid: null pointer");
    const long long n = (long long)H * W;
    rays_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        H, W, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[12], c[13], c[14], c[15], c[16], c[17], ray);
    return check_launch("rays_grid");
}

extern "C" mvs_status mvs_hyp_linear(int32_t H, int32_t W, const float* base, const float* step, int64_t i,
                                     float* out, void* stream) {
    clear_error();
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "hyp_linear: shapes differ");
    const long long n = (long long)H * W;
    if (!n) return MVS_OK;
    if (!base || !step || !out) return fail(MVS_ERR_VALUE, "hyp_linear: null pointer");
    hyp_linear_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, base, step, (float)i, out);
    return check_launch("hyp_linear");
}

extern "C" mvs_status mvs_hyp_refine(int32_t H, int32_t W, const float* iu, const float* ds, int64_t t,
                                     float* out, void* stream) {
    clear_error();
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "hyp_refine: shapes differ");
    const long long n = (long long)H * W;
    if (!n) return MVS_OK;
    if (!iu || !ds || !out) return fail(MVS_ERR_VALUE, "hyp_refine: null pointer");
    hyp_refine_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, iu, ds, (float)t, out);
    return check_launch("hyp_refine");
}

extern "C" mvs_status mvs_depth_view(int32_t h, int32_t w, const uint8_t* rgb, const float* gain, const float* bias,
                                     const uint8_t* mask, float* grey, uint8_t* rgb8, void* stream) {
    clear_error();
    if (h < 0 || w < 0) return fail(MVS_ERR_VALUE, "depth_view: negative shape");
    const long long n = (long long)h * w;
    if (!n) return MVS_OK;
    if (!rgb || !grey) return fail(MVS_ERR_VALUE, "depth_view: null pointer");
    depth_view_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        n, rgb, gain != nullptr, gain ? gain[0] : 1.f, gain ? gain[1] : 1.f, gain ? gain[2] : 1.f, bias != nullptr,
        bias ? bias[0] : 0.f, bias ? bias[1] : 0.f, bias ? bias[2] : 0.f, mask, grey, rgb8);
    return check_launch("depth_view");
}

extern "C" mvs_status mvs_half(int32_t planes, int32_t h, int32_t w, const float* in, float* out, void* stream) {
    clear_error();
    if (planes < 0 || h < 0 || w < 0) return fail(MVS_ERR_VALUE, "half: negative shape");
    const long long n = (long long)planes * (h / 2) * (w / 2);
    if (!n) return MVS_OK;
    if (!in || !out) return fail(MVS_ERR_VALUE, "half: null pointer");
    half_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(planes, h, w, in, out);
    return check_launch("half");
}

extern "C" mvs_status mvs_to_fp16(int64_t n, const float* in, void* out, void* stream) {
    clear_error();
    if (n < 0) return fail(MVS_ERR_VALUE, "to_fp16: negative size");
    if (!n) return MVS_OK;
    if (!in || !out) return fail(MVS_ERR_VALUE, "to_fp16: null pointer");
    to_fp16_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, in, reinterpret_cast<__half*>(out));
    return check_launch("to_fp16");
}

extern "C" mvs_status mvs_tie_depths(int32_t n, const double* X, const double* cam, int32_t w, int32_t h, double* out,
                                     void* stream) {
    clear_error();
    if (n < 0 || w < 0 || h < 0) return fail(MVS_ERR_VALUE, "tie_depths: negative size");
    if (n == 0) return MVS_OK;
    if (!X || !cam || !out) return fail(MVS_ERR_VALUE, "tie_depths: null pointer");
    TieCam c;
    memcpy(c.c, cam, sizeof(c.c));
    tie_depths_kernel<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, X, c, w, h, out);
    return check_launch("tie_depths");
}

extern "C" mvs_status mvs_depth_band(const mvs_depth_band_args* a, void* stream) {
    clear_error();
    if (!a) return fail(MVS_ERR_VALUE, "depth_band: null arguments");
    if (a->H < 0 || a->W < 0 || a->n_pts < 0) return fail(MVS_ERR_VALUE, "depth_band: negative size");
    if (a->block < 1) return fail(MVS_ERR_VALUE, "depth_band: block must be >= 1");
    if (a->H == 0 || a->W == 0) return MVS_OK;
    if (!a->cam || !a->base || !a->step || (a->n_pts >= MVS_BAND_MIN_POINTS && !a->X))
        return fail(MVS_ERR_VALUE, "depth_band: null pointer");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int gh = (a->H + a->block - 1) / a->block, gw = (a->W + a->block - 1) / a->block;
    const int nb = gh * gw;
    const bool uniform = a->n_pts < MVS_BAND_MIN_POINTS;
    char* cells = nullptr;
    if (!uniform) {
        MVS_CUDA(cudaMallocAsync((void**)&cells, (size_t)nb * 20, st), "depth_band: cell table");
        unsigned long long* zlo = reinterpret_cast<unsigned long long*>(cells);
        unsigned long long* zhi = zlo + nb;
        int* cnt = reinterpret_cast<int*>(zhi + nb);
        TieCam c;
        memcpy(c.c, a->cam, sizeof(c.c));
        band_init_kernel<<<blocks(nb, 256), 256, 0, st>>>(nb, zlo, zhi, cnt);
        band_scatter_kernel<<<blocks(a->n_pts, 256), 256, 0, st>>>(a->n_pts, a->X, c, a->H, a->W, a->block, gw, zlo,
                                                                   zhi, cnt);
    }
    const unsigned long long* zlo = reinterpret_cast<const unsigned long long*>(cells);
    const unsigned long long* zhi = uniform ? nullptr : zlo + nb;
    const int* cnt = uniform ? nullptr : reinterpret_cast<const int*>(zhi + nb);
    band_fill_kernel<<<dim3(blocks(a->W, 256), a->H), 256, 0, st>>>(a->H, a->W, a->block, gh, gw, zlo, zhi, cnt, a->lo,
                                                                   a->hi, a->margin, a->nd, uniform ? 1 : 0, a->base,
                                                                   a->step, a->inv_hi);
    const mvs_status s = check_launch("depth_band");
    if (cells) cudaFreeAsync(cells, st);
    return s;
}

extern "C" mvs_status mvs_debug_bound_violations(uint32_t* count) {
    clear_error();
#ifdef MVS_DEBUG_BOUNDS
    MVS_CUDA(cudaDeviceSynchronize(), "debug bounds: synchronise");
    const unsigned n = take_bound_violations_sweep() + take_bound_violations_batch() + take_bound_violations_pm();
    if (count) *count = n;
    return MVS_OK;
#else
    if (count) *count = 0;
    return fail(MVS_ERR_UNSUPPORTED, "this library was built without bounds checks (MVS_DEBUG_BOUNDS)");
#endif
}
