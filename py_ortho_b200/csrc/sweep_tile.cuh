// The plane-sweep tile engine shared by the single-view kernel (sweep.cu) and the persistent
// batched kernel (batch.cu): warp + windowed ZNCC + best-k over sources + streaming
// winner-take-all for one TW x TH output tile and one contiguous range of hypotheses.
//
// Semantics follow the reference's fused CPU step (_dense.pyx:740-838 with _sweep.h) and its
// definitional form (_dense.ncc_warp + _dense.combine, _dense.pyx:13-144):
//   * a source sample is valid when its camera-frame Z > 1e-6, 0 <= u <= w - 1.001,
//     0 <= v <= h - 1.001 and the bilinear value is finite (NaN pixels are masks);
//   * window sums run over the (2r+1)^2 window clipped to the reference image;
//     count/k^2 <= 0.9 gives NCC = -1; otherwise
//     NCC = (mean(JI) - mu mean(J)) / (sd * sdj), sdj = sqrt(var(J)) if var > 1e-6 else 1e-3,
//     clipped to [-1, 1];
//   * the hypothesis score is the float32 mean of the top_k source NCCs (summed in descending
//     order); the winner update is strict '>' in hypothesis order (first index wins ties),
//     tracking the score of the previous hypothesis and of the one after the winner.
//
// Work of one CTA per (hypothesis, source):
//   A. warp the source into a shared-memory tile with an r-pixel halo (NaN = invalid sample);
//   B. horizontal window sums of (V, J, J^2, J*I): each thread runs along a 16-column row
//      segment (inputs from 16-byte shared loads, products formed once per input) and stores
//      one float4 per output;
//   C. vertical running sums down each column (TH/SEG rows per thread) from float4 loads, NCC,
//      insertion into a per-pixel top-k list in registers.
// After the last source the winner-take-all state of each pixel is updated in registers; it
// leaves the SM once per hypothesis chunk. Window sums are short FP32 sums (at most TH/SEG
// add/subtract steps): within the parity bar wherever the window has texture, but on bright
// low-texture windows at r <= 2 their rounding, amplified by 1 / (sd_ref sd_src), can reach
// ~1e-3 in NCC. X64 (MVS_PREC_FP64_SUMS) keeps the sums in float64 as the reference does
// (stage_b64 / stage_c64).
#pragma once

#include "common.cuh"

namespace mvs {

constexpr int TW = 64;                 // output tile width (columns)
constexpr int ROWS = 8;                // output rows per thread in stage C
constexpr int TH_DEFAULT = 32;         // output tile height of the default shape

// A TW x TH output tile runs on NT = 8 TH threads: thread t keeps column t mod TW and the ROWS rows
// of segment t / TW in stage C, so every thread's rows start on a multiple of 8 in each of the
// three shapes (TH = 16, 32, 64; 128, 256, 512 threads).
template <int TH>
struct TileShape {
    static_assert(TH == 16 || TH == 32 || TH == 64, "tile height 16, 32 or 64");
    static constexpr int NT = 8 * TH;              // threads per CTA
    static constexpr int SEG = NT / TW;            // row segments (= TH / ROWS)
    static constexpr int MIN_CTAS = TH == 16 ? 3 : (TH == 32 ? 2 : 1);   // resident CTAs per SM
};

struct SrcGeo {
    const void* img;                   // float or __half, (h, w) row-major
    int h, w;
    double m[9];                       // PLANES: A = Rs R_ref^T K_ref^-1; ray path: Rs
    double b[3];                       // Rs (C_ref - C_src)
    double f, k1, k2, k3, cx, cy;
};

struct SweepParams {
    CUtensorMap ref_map;               // 2D tiled map of `ref` (single-view kernel, ref_tma = 1)
    int ref_tma;                       // 1: the reference tile is copied by TMA
    int H, W, n_src, kk;
    int topk_bottom;                   // 1: keep the n-kk lowest and subtract from the total
    int i0, i1, ppc;                   // hypotheses [i0, i1), planes per chunk
    int hyp_kind, t0;
    int r, nchunks;
    int fresh;                         // 1: start from the initial state instead of loading it
    unsigned wait_limit;               // try_wait iterations of the TMA tile wait
    long long map_stride;
    const float* ref;
    const float* mu;
    const float* sd;
    const float* ray;
    const float* hyp_a;                // MAPS: maps; LINEAR/REFINE: base
    const float* hyp_b;                // LINEAR/REFINE: step
    float* best;
    float* prev;
    float* spb;
    float* snb;
    int* idx;
    float* rec;                        // chunk records (6, nchunks, H, W) or nullptr
    SrcGeo src[MVS_MAX_SOURCES];
    float planes[MVS_MAX_PLANES_PER_CALL];   // PLANES: inverse depth of hypothesis i0 + j
};

// Per (hypothesis, source, tile) projective map in tile-local coordinates (a, b) of the halo
// origin, composed in FP64 and rounded once: u_l = (nu0 + nu1 a + nu2 b) / dz, v_l likewise,
// dz = dz0 + dz1 a + dz2 b; the source pixel is (U0 + u_l, V0 + v_l) and the camera-frame
// depth is zs * dz. Small local magnitudes keep the FP32 evaluation at ~1e-5 px.
struct Coef {
    float nu0, nu1, nu2, nv0, nv1, nv2, dz0, dz1, dz2, zs;
    float lo_u, hi_u, lo_v, hi_v;
    int U0, V0;
    int inside;       // every sample of the halo rectangle maps inside the source (with margin)
    int pad_[3];
};

template <int R, int TH = TH_DEFAULT>
struct Geom {
    static constexpr int K = 2 * R + 1;
    static constexpr int RA = (R + 3) & ~3;        // halo rounded up to a float4
    static constexpr int HR = TH + 2 * R;          // sampled rows
    static constexpr int HC = TW + 2 * R;          // sampled columns
    static constexpr int JP = TW + 2 * RA + 4;     // shared row pitch (floats): odd in float4 units
    static constexpr int P = 16;                   // stage-B outputs per thread (one row segment)
    static constexpr int NSEG = TW / P;
    static constexpr int NIN = P + 2 * RA;         // stage-B inputs per segment
    static constexpr size_t count_bytes() {      // compensated mode: uint8 horizontal window counts
        return ((size_t)HR * TW + 15) & ~(size_t)15;
    }
    static constexpr size_t smem_bytes() {       // sJ, sI, sH, winner state (6 planes), sC
        return (size_t)HR * JP * 4 * 2 + (size_t)HR * TW * 16 + (size_t)6 * TH * TW * 4 +
               sizeof(Coef) * MVS_MAX_SOURCES;
    }
};

// Largest shared-memory footprint over radii 0..RMAX (a persistent CTA serves any of them).
template <int RMAX, int TH = TH_DEFAULT>
constexpr size_t smem_bytes_upto() {
    size_t m = 0;
    if constexpr (RMAX >= 0) m = Geom<0, TH>::smem_bytes() > m ? Geom<0, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 1) m = Geom<1, TH>::smem_bytes() > m ? Geom<1, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 2) m = Geom<2, TH>::smem_bytes() > m ? Geom<2, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 3) m = Geom<3, TH>::smem_bytes() > m ? Geom<3, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 4) m = Geom<4, TH>::smem_bytes() > m ? Geom<4, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 5) m = Geom<5, TH>::smem_bytes() > m ? Geom<5, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 6) m = Geom<6, TH>::smem_bytes() > m ? Geom<6, TH>::smem_bytes() : m;
    if constexpr (RMAX >= 7) m = Geom<7, TH>::smem_bytes() > m ? Geom<7, TH>::smem_bytes() : m;
    return m;
}

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fc00000); }

// Position of the horizontal-sum float4 of (row, col) in shared memory: an XOR swizzle of the
// column's low 3 bits by (segment + row), so that the row-segment writers of stage B (32 lanes =
// 8 rows x 4 segments) and the column readers of stage C (32 consecutive columns) both touch 8
// distinct 16-byte bank groups per quarter-warp.
__device__ __forceinline__ int hs_index(int row, int col) {
    return row * TW + (col ^ (((col >> 4) + row) & 7));
}

__device__ __forceinline__ float hyp_value(const SweepParams& p, int i, int gx, int gy) {
    const long long o = (long long)gy * p.W + gx;
    switch (p.hyp_kind) {
        case MVS_HYP_MAPS:
            return __ldg(p.hyp_a + (long long)(i - p.i0) * p.map_stride + o);
        case MVS_HYP_LINEAR: {      // (base + (float)i * step), two float32 roundings
            const float t = __fmul_rn((float)i, __ldg(p.hyp_b + o));
            return __fadd_rn(__ldg(p.hyp_a + o), t);
        }
        case MVS_HYP_REFINE: {      // max(iu + (float)t * ds, 1e-6), NaN propagating
            const float t = __fmul_rn((float)(i + p.t0), __ldg(p.hyp_b + o));
            return max_nan(__fadd_rn(__ldg(p.hyp_a + o), t), 1e-6f);
        }
        default:
            return p.planes[i - p.i0];
    }
}

template <bool F16>
__device__ __forceinline__ float tap(const void* img, long long i) {
    if constexpr (F16) {
        return __half2float(__ldg(reinterpret_cast<const __half*>(img) + i));
    } else {
        return __ldg(reinterpret_cast<const float*>(img) + i);
    }
}

// floor(x) for |x| < 2^22 on the FMA pipe: adding 1.5 * 2^23 rounded toward -inf leaves floor(x)
// in the low mantissa bits. Returns the integer; `f` receives floor(x) as a float.
__device__ __forceinline__ int floor_fma(float x, float& f) {
    const float t = __fadd_rd(x, 12582912.0f);
    f = __fsub_rn(t, 12582912.0f);
    return __float_as_int(t) - 0x4B400000;
}

// Homography path sample (pinhole, constant inverse depth per hypothesis), branch-free so that
// the loads of several samples can be in flight together. Invalid samples read a safe address
// and return NaN.
template <bool F16>
__device__ __forceinline__ float sample_plane(const Coef& c, const void* img, int w, int h, float a, float b, bool in) {
    const float dz = fmaf(c.dz1, a, fmaf(c.dz2, b, c.dz0));
    const float rz = __fdividef(1.0f, dz);
    const float ul = fmaf(c.nu1, a, fmaf(c.nu2, b, c.nu0)) * rz;
    const float vl = fmaf(c.nv1, a, fmaf(c.nv2, b, c.nv0)) * rz;
    bool ok = in && (c.zs * dz > 1e-6f) && (ul >= c.lo_u) && (ul <= c.hi_u) && (vl >= c.lo_v) && (vl <= c.hi_v);
    float fu, fv;
    const int x0 = c.U0 + floor_fma(ok ? ul : 0.f, fu);
    const int y0 = c.V0 + floor_fma(ok ? vl : 0.f, fv);
    // integer guard: every tap stays inside the image whatever the float rounding did
    ok = ok && (unsigned)x0 < (unsigned)(w - 1) && (unsigned)y0 < (unsigned)(h - 1);
    const long long o = ok ? (long long)y0 * w + x0 : 0;
    MVS_BOUND(o >= 0 && o + w + 1 < (long long)h * w);
    const float fx = ul - fu, fy = vl - fv;
    const float a00 = tap<F16>(img, o), a01 = tap<F16>(img, o + 1);
    const float a10 = tap<F16>(img, o + w), a11 = tap<F16>(img, o + w + 1);
    const float top = fmaf(fx, a01 - a00, a00);
    const float bot = fmaf(fx, a11 - a10, a10);
    const float val = fmaf(fy, bot - top, top);
    return (ok && isfinite(val)) ? val : qnan();
}

// Homography sample when the whole halo rectangle is known to map inside the source and to lie
// inside the reference image: no per-sample bounds; a non-finite value becomes NaN (invalid).
// (Evaluating the maps column part first, so that a thread walking down one halo column keeps
// fmaf(x1, a, x0), and clamping the linear tap offset once instead of each coordinate measured
// 1.3 % slower at C2: 167.5 vs 165.2 ms.)
template <bool F16>
__device__ __forceinline__ float sample_plane_inside(const Coef& c, const void* img, int w, int h, float a, float b) {
    const float dz = fmaf(c.dz1, a, fmaf(c.dz2, b, c.dz0));
    const float rz = __fdividef(1.0f, dz);
    const float ul = fmaf(c.nu1, a, fmaf(c.nu2, b, c.nu0)) * rz;
    const float vl = fmaf(c.nv1, a, fmaf(c.nv2, b, c.nv0)) * rz;
    float fu, fv;
    // the clamp is a no-op when the corner test holds; it keeps every tap inside the image even if
    // an extreme geometry defeated that test
    const unsigned x0 = min((unsigned)(c.U0 + floor_fma(ul, fu)), (unsigned)(w - 2));
    const unsigned y0 = min((unsigned)(c.V0 + floor_fma(vl, fv)), (unsigned)(h - 2));
    const long long o = (long long)y0 * w + x0;
    MVS_BOUND(o >= 0 && o + w + 1 < (long long)h * w);
    const float fx = ul - fu, fy = vl - fv;
    const float a00 = tap<F16>(img, o), a01 = tap<F16>(img, o + 1);
    const float a10 = tap<F16>(img, o + w), a11 = tap<F16>(img, o + w + 1);
    const float top = fmaf(fx, a01 - a00, a00);
    const float bot = fmaf(fx, a11 - a10, a10);
    const float val = fmaf(fy, bot - top, top);
    return fmaf(val, 0.0f, val);   // finite: val; inf: NaN; NaN: NaN
}

// Ray path sample: per-pixel inverse depth and world ray, FP64 projection with radial
// distortion and FP64 bilinear, as _sweep.h:49-80.
__device__ __forceinline__ float sample_ray(const SweepParams& p, const SrcGeo& g, int i, int gx, int gy) {
    const float inv = hyp_value(p, i, gx, gy);
    const long long HW = (long long)p.H * p.W, o = (long long)gy * p.W + gx;
    const double d = 1.0 / (double)inv;
    const double rx = __ldg(p.ray + o), ry = __ldg(p.ray + HW + o), rz = __ldg(p.ray + 2 * HW + o);
    const double X = g.b[0] + d * ((g.m[0] * rx + g.m[1] * ry) + g.m[2] * rz);
    const double Y = g.b[1] + d * ((g.m[3] * rx + g.m[4] * ry) + g.m[5] * rz);
    const double Z = g.b[2] + d * ((g.m[6] * rx + g.m[7] * ry) + g.m[8] * rz);
    if (!(Z > 1e-6)) return qnan();
    const double nx = X / Z, ny = Y / Z;
    const double r2 = nx * nx + ny * ny;
    const double dd = g.f * (1.0 + r2 * (g.k1 + r2 * (g.k2 + r2 * g.k3)));
    const double u = dd * nx + g.cx, v = dd * ny + g.cy;
    // NaN u / v (NaN hypotheses) count as invalid; the reference leaves them undefined
    if (!(u >= 0.0 && v >= 0.0 && u <= (double)g.w - 1.001 && v <= (double)g.h - 1.001)) return qnan();
    const int x0 = (int)u, y0 = (int)v;
    const double fx = u - (double)x0, fy = v - (double)y0;
    const long long so = (long long)y0 * g.w + x0;
    MVS_BOUND(so >= 0 && so + g.w + 1 < (long long)g.h * g.w);
    const double a00 = tap<false>(g.img, so), a01 = tap<false>(g.img, so + 1);
    const double a10 = tap<false>(g.img, so + g.w), a11 = tap<false>(g.img, so + g.w + 1);
    const double val = (a00 * (1.0 - fx) + a01 * fx) * (1.0 - fy) + (a10 * (1.0 - fx) + a11 * fx) * fy;
    return isfinite(val) ? (float)val : qnan();
}

// The plane map of one (hypothesis, source, tile), composed in FP64 and rounded once (Coef),
// by the 4 lanes of an aligned lane group: lane k tests corner k of the halo rectangle, lane 0
// also forms the map, so the four corner tests' divisions run in parallel. A projective map whose
// depth stays positive maps the halo rectangle onto the convex hull of its corner images, so four
// corners strictly inside (a 1e-3 px margin absorbs the FP32 evaluation error of ~1e-5 px) put
// every sample inside. Every lane of the calling warps must call it (width-4 shuffles); `write`
// selects the groups that store their source's Coef.
__device__ inline void make_coef_group(Coef& c, const SrcGeo& g, float inv, int ox, int oy, int hc_span, int hr_span,
                                       bool write) {
    const int k = threadIdx.x & 3;
    const double d = 1.0 / (double)inv;
    double g0[3], g1[3], g2[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        g1[q] = d * g.m[3 * q + 0];
        g2[q] = d * g.m[3 * q + 1];
        g0[q] = d * (g.m[3 * q + 0] * (double)ox + g.m[3 * q + 1] * (double)oy + g.m[3 * q + 2]) + g.b[q];
    }
    const double Z0 = g0[2];
    const bool norm = fabs(Z0) > 1e-9;
    // corner k of the halo rectangle: (0, 0), (w - 1, 0), (0, h - 1), (w - 1, h - 1)
    const double ca = (k & 1) ? (double)(hc_span - 1) : 0.0, cb = (k & 2) ? (double)(hr_span - 1) : 0.0;
    const double Xc = g0[0] + ca * g1[0] + cb * g2[0];
    const double Yc = g0[1] + ca * g1[1] + cb * g2[1];
    const double Zc = g0[2] + ca * g1[2] + cb * g2[2];
    const double uc = g.f * Xc / Zc + g.cx, vc = g.f * Yc / Zc + g.cy;
    int in = Zc > 1e-5 && uc >= 1e-3 && vc >= 1e-3 && uc <= (double)g.w - 1.001 - 1e-3 &&
             vc <= (double)g.h - 1.001 - 1e-3;
    in &= __shfl_xor_sync(0xffffffffu, in, 1, 4);
    in &= __shfl_xor_sync(0xffffffffu, in, 2, 4);
    if (k != 0 || !write) return;
    const double zs = norm ? Z0 : 1.0;
    const double rzs = 1.0 / zs;
    double U0 = 0.0, V0 = 0.0;
    if (norm) {
        const double u00 = g.f * g0[0] * rzs + g.cx, v00 = g.f * g0[1] * rzs + g.cy;
        if (isfinite(u00)) U0 = fmin(fmax(floor(u00), -1048576.0), 1048576.0);
        if (isfinite(v00)) V0 = fmin(fmax(floor(v00), -1048576.0), 1048576.0);
    }
    const double au = g.cx - U0, av = g.cy - V0;
    c.nu0 = (float)((g.f * g0[0] + au * g0[2]) * rzs);
    c.nu1 = (float)((g.f * g1[0] + au * g1[2]) * rzs);
    c.nu2 = (float)((g.f * g2[0] + au * g2[2]) * rzs);
    c.nv0 = (float)((g.f * g0[1] + av * g0[2]) * rzs);
    c.nv1 = (float)((g.f * g1[1] + av * g1[2]) * rzs);
    c.nv2 = (float)((g.f * g2[1] + av * g2[2]) * rzs);
    c.dz0 = (float)(g0[2] * rzs);
    c.dz1 = (float)(g1[2] * rzs);
    c.dz2 = (float)(g2[2] * rzs);
    c.zs = (float)zs;
    c.lo_u = (float)(-U0);
    c.lo_v = (float)(-V0);
    c.hi_u = (float)(((double)g.w - 1.001) - U0);
    c.hi_v = (float)(((double)g.h - 1.001) - V0);
    c.U0 = (int)U0;
    c.V0 = (int)V0;
    c.inside = (norm && in) ? 1 : 0;
}

// Stage B: horizontal window sums of (V, J, J^2, J I) for one 16-column row segment per thread:
// products formed once per input, running sums along the segment, one float4 per output.
// WITHV = false when every sample is valid: the count column is not formed (it would be k).
template <int R, bool WITHV, int TH = TH_DEFAULT>
__device__ __forceinline__ void stage_b(const float* sJ, const float* sI, float4* sH, int tid) {
    using G = Geom<R, TH>;
    constexpr int RA = G::RA, HR = G::HR, JP = G::JP, P = G::P, NSEG = G::NSEG, NIN = G::NIN;
    if (tid >= HR * NSEG) return;
    // consecutive threads take consecutive rows of one segment: a quarter-warp's 16-byte loads then
    // start (19 hy + 4 sg) mod 8 float4 units into the bank space - 8 distinct groups (JP = 76)
    const int sg = tid / HR, hy = tid - sg * HR;
    MVS_BOUND(hy < HR && P * sg + P <= TW && hy * JP + P * sg + NIN <= HR * JP);
    const float4* jr = reinterpret_cast<const float4*>(sJ + hy * JP + P * sg);
    const float4* ir = reinterpret_cast<const float4*>(sI + hy * JP + P * sg);
    float v[NIN], s1[NIN], s2[NIN], s3[NIN];
#pragma unroll
    for (int q = 0; q < NIN / 4; ++q) {
        const float4 a = jr[q], b = ir[q];
        const float jv[4] = {a.x, a.y, a.z, a.w}, iv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = 4 * q + u;
            float jz = jv[u];
            if constexpr (WITHV) {
                const bool ok = jz == jz;
                jz = ok ? jz : 0.f;
                v[t] = ok ? 1.f : 0.f;
            }
            s1[t] = jz;
            s2[t] = __fmul_rn(jz, jz);
            s3[t] = __fmul_rn(jz, iv[u]);
        }
    }
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
    for (int t = RA - R; t <= RA + R; ++t) {
        if constexpr (WITHV) a0 = __fadd_rn(a0, v[t]);
        a1 = __fadd_rn(a1, s1[t]);
        a2 = __fadd_rn(a2, s2[t]);
        a3 = __fadd_rn(a3, s3[t]);
    }
    // hs_index(hy, P sg + j) = hy TW + P sg + (j ^ kx): the segment's columns share (col >> 4) = sg
    float4* row = sH + hy * TW + P * sg;
    const int kx = (sg + hy) & 7;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (j > 0) {
            const int tn = RA + R + j, to = RA - R + j - 1;
            if constexpr (WITHV) a0 = __fadd_rn(a0, __fsub_rn(v[tn], v[to]));
            a1 = __fadd_rn(a1, __fsub_rn(s1[tn], s1[to]));
            a2 = __fadd_rn(a2, __fsub_rn(s2[tn], s2[to]));
            a3 = __fadd_rn(a3, __fsub_rn(s3[tn], s3[to]));
        }
        row[j ^ kx] = make_float4(a0, a1, a2, a3);
    }
}

// Stage C for one thread: vertical running sums down column c (rows y0 .. y0 + ROWS - 1), ZNCC,
// insertion into the per-pixel top-k lists. WITHV = false: every window count is k^2.
template <int R, int KMAX, bool WITHV, int TH = TH_DEFAULT>
__device__ __forceinline__ void stage_c(const float4* sH, int c, int y0, const float* mu, const float* rsd,
                                        float (&topk)[ROWS][KMAX], float* total, bool bottom, int nlist) {
    constexpr int K = 2 * R + 1;
    const float k2 = (float)(K * K), inv_k2 = 1.0f / (float)(K * K);
    // y0 is a multiple of 8 (ROWS = 8), so hs_index(y0 + t, c) = (y0 + t) TW + sw[t & 7]
    static_assert(ROWS % 8 == 0, "stage C rows must start on a multiple of 8");
    int sw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) sw[k] = c ^ (((c >> 4) + k) & 7);
    const float4* col = sH + y0 * TW;
    MVS_BOUND(y0 + ROWS + 2 * R <= (Geom<R, TH>::HR) && c < TW);
    float cv = 0.f, cj = 0.f, cjj = 0.f, cji = 0.f;
#pragma unroll
    for (int t = 0; t < K; ++t) {
        const float4 h = col[t * TW + sw[t & 7]];
        if constexpr (WITHV) cv = __fadd_rn(cv, h.x);
        cj = __fadd_rn(cj, h.y);
        cjj = __fadd_rn(cjj, h.z);
        cji = __fadd_rn(cji, h.w);
    }
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        if (j > 0) {
            const float4 hn = col[(j + 2 * R) * TW + sw[(j + 2 * R) & 7]];
            const float4 ho = col[(j - 1) * TW + sw[(j - 1) & 7]];
            if constexpr (WITHV) cv = __fadd_rn(cv, __fsub_rn(hn.x, ho.x));
            cj = __fadd_rn(cj, __fsub_rn(hn.y, ho.y));
            cjj = __fadd_rn(cjj, __fsub_rn(hn.z, ho.z));
            cji = __fadd_rn(cji, __fsub_rn(hn.w, ho.w));
        }
        float ncc;
        if (WITHV && cv * 10.f <= 9.f * k2) {
            ncc = -1.f;
        } else {
            const float rc = (!WITHV || cv == k2) ? inv_k2 : __frcp_rn(cv);
            const float mj = __fmul_rn(cj, rc), m2 = __fmul_rn(cjj, rc), mij = __fmul_rn(cji, rc);
            const float var = __fsub_rn(m2, __fmul_rn(mj, mj));
            const float rsdj = var > 1e-6f ? rsqrtf(var) : 1000.f;
            ncc = __fmul_rn(__fsub_rn(mij, __fmul_rn(mu[j], mj)), __fmul_rn(rsd[j], rsdj));
            ncc = ncc > 1.f ? 1.f : (ncc < -1.f ? -1.f : ncc);
        }
        if (bottom) total[j] = __fadd_rn(total[j], ncc);
        float x = ncc;
#pragma unroll
        for (int q = 0; q < KMAX; ++q) {
            if (q < nlist) {
                const float hi = fmaxf(topk[j][q], x), lo = fminf(topk[j][q], x);
                topk[j][q] = bottom ? lo : hi;
                x = bottom ? hi : lo;
            }
        }
    }
}

// ---- float64 window sums (MVS_PREC_FP64_SUMS): the reference's arithmetic for the sums
// (_sweep.h:85-178): the products J J and J I formed in float32 (float times float, as there),
// horizontal window sums accumulated in float64 - the new column added, then the old one
// subtracted - and stored rounded to float32, as the reference stores its hs rows; vertical sums
// in float64 (add, then subtract), the moments scaled by 1 / k^2 and divided by the scaled count,
// the count gate, variance and NCC in float64 (om_sw_ncc_row), the NCC rounded to float32 once.
// On bright low-texture windows, where the NCC divides by sd_ref * sd_src ~ 1e-3, float32 running
// sums differ from the reference by up to ~1e-3; these track it to the last float32 bit or so.

template <int R, bool WITHV, int TH = TH_DEFAULT>
__device__ __forceinline__ void stage_b64(const float* sJ, const float* sI, float4* sH, int tid) {
    using G = Geom<R, TH>;
    constexpr int RA = G::RA, HR = G::HR, JP = G::JP, P = G::P, NSEG = G::NSEG, NIN = G::NIN;
    if (tid >= HR * NSEG) return;
    const int sg = tid / HR, hy = tid - sg * HR;
    MVS_BOUND(hy < HR && P * sg + P <= TW && hy * JP + P * sg + NIN <= HR * JP);
    const float4* jr = reinterpret_cast<const float4*>(sJ + hy * JP + P * sg);
    const float4* ir = reinterpret_cast<const float4*>(sI + hy * JP + P * sg);
    float v[NIN], jz[NIN], q2[NIN], q3[NIN];
#pragma unroll
    for (int q = 0; q < NIN / 4; ++q) {
        const float4 a = jr[q], b = ir[q];
        const float jv[4] = {a.x, a.y, a.z, a.w}, iv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = 4 * q + u;
            float x = jv[u];
            if constexpr (WITHV) {
                const bool ok = x == x;
                x = ok ? x : 0.f;
                v[t] = ok ? 1.f : 0.f;
            }
            jz[t] = x;
            q2[t] = __fmul_rn(x, x);
            q3[t] = __fmul_rn(x, iv[u]);
        }
    }
    float a0 = 0.f;                       // counts are small integers: exact in float32
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
    for (int t = RA - R; t <= RA + R; ++t) {
        if constexpr (WITHV) a0 = __fadd_rn(a0, v[t]);
        a1 = __dadd_rn(a1, (double)jz[t]);
        a2 = __dadd_rn(a2, (double)q2[t]);
        a3 = __dadd_rn(a3, (double)q3[t]);
    }
    float4* row = sH + hy * TW + P * sg;
    const int kx = (sg + hy) & 7;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (j > 0) {
            const int tn = RA + R + j, to = RA - R + j - 1;
            if constexpr (WITHV) a0 = __fadd_rn(a0, __fsub_rn(v[tn], v[to]));
            a1 = __dsub_rn(__dadd_rn(a1, (double)jz[tn]), (double)jz[to]);
            a2 = __dsub_rn(__dadd_rn(a2, (double)q2[tn]), (double)q2[to]);
            a3 = __dsub_rn(__dadd_rn(a3, (double)q3[tn]), (double)q3[to]);
        }
        row[j ^ kx] = make_float4(a0, (float)a1, (float)a2, (float)a3);
    }
}

// `sdv` holds the reference's window deviation itself (not its reciprocal) in this mode.
template <int R, int KMAX, bool WITHV, int TH = TH_DEFAULT>
__device__ __forceinline__ void stage_c64(const float4* sH, int c, int y0, const float* mu, const float* sdv,
                                          float (&topk)[ROWS][KMAX], float* total, bool bottom, int nlist) {
    constexpr int K = 2 * R + 1;
    const double kkd = 1.0 / (double)(K * K);
    static_assert(ROWS % 8 == 0, "stage C rows must start on a multiple of 8");
    int sw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) sw[k] = c ^ (((c >> 4) + k) & 7);
    const float4* col = sH + y0 * TW;
    MVS_BOUND(y0 + ROWS + 2 * R <= (Geom<R, TH>::HR) && c < TW);
    float cv = 0.f;
    double cj = 0.0, cjj = 0.0, cji = 0.0;
#pragma unroll
    for (int t = 0; t < K; ++t) {
        const float4 h = col[t * TW + sw[t & 7]];
        if constexpr (WITHV) cv = __fadd_rn(cv, h.x);
        cj = __dadd_rn(cj, (double)h.y);
        cjj = __dadd_rn(cjj, (double)h.z);
        cji = __dadd_rn(cji, (double)h.w);
    }
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        if (j > 0) {
            const float4 hn = col[(j + 2 * R) * TW + sw[(j + 2 * R) & 7]];
            const float4 ho = col[(j - 1) * TW + sw[(j - 1) & 7]];
            if constexpr (WITHV) cv = __fadd_rn(cv, __fsub_rn(hn.x, ho.x));
            cj = __dsub_rn(__dadd_rn(cj, (double)hn.y), (double)ho.y);
            cjj = __dsub_rn(__dadd_rn(cjj, (double)hn.z), (double)ho.z);
            cji = __dsub_rn(__dadd_rn(cji, (double)hn.w), (double)ho.w);
        }
        float ncc;
        const double cov = __dmul_rn(WITHV ? (double)cv : (double)(K * K), kkd);
        if (cov <= 0.9) {
            ncc = -1.f;
        } else {
            const double mj = __ddiv_rn(__dmul_rn(cj, kkd), cov), m2 = __ddiv_rn(__dmul_rn(cjj, kkd), cov);
            const double mij = __ddiv_rn(__dmul_rn(cji, kkd), cov);
            const double var = __dsub_rn(m2, __dmul_rn(mj, mj));
            const double sdj = var > 1e-6 ? __dsqrt_rn(var) : 1e-3;
            double x = __ddiv_rn(__dsub_rn(mij, __dmul_rn((double)mu[j], mj)), __dmul_rn((double)sdv[j], sdj));
            x = x > 1.0 ? 1.0 : (x < -1.0 ? -1.0 : x);
            ncc = (float)x;
        }
        if (bottom) total[j] = __fadd_rn(total[j], ncc);
        float x = ncc;
#pragma unroll
        for (int q = 0; q < KMAX; ++q) {
            if (q < nlist) {
                const float hi = fmaxf(topk[j][q], x), lo = fminf(topk[j][q], x);
                topk[j][q] = bottom ? lo : hi;
                x = bottom ? hi : lo;
            }
        }
    }
}

// ---- compensated window sums (MVS_PREC_FP32_COMP / MVS_PREC_FP16_COMP)
//
// A bright, low-texture window (grey ~1.5, deviations ~0.05) makes the plain form's moments
// m2 - mj^2 and mij - mu mj differences of numbers ~2.25 that agree to ~3 digits, so float32
// rounding of the sums (and of the reference statistics) reaches the NCC a thousand-fold. This form
// removes the large common part before anything is summed: the tile's reference values and every
// warped source value are shifted by one pivot per tile (the mean reference value of the tile's
// pixels), the window sums of the shifted values are accumulated with Kahan compensation in the
// vertical direction (the variance and covariance terms), and the reference window statistics are
// formed from the shifted tile (zero padding outside the image, divided by k^2, floor 1e-6 on the
// variance: the reference's definitions). With I' = I - p and J' = J - p:
//   var(J) = E[J'^2] - E[J']^2,   E[IJ] - mu E[J] = E[I'J'] - mu' E[J'] + p (E[I'] - mu'),
// mu' = mu - p; E[] over the window's valid samples. When every sample of the tile is valid the
// windows are full and E[I'] = mu' exactly, so the last term is zero and is not formed; otherwise
// the masked sum of I' is accumulated as a fifth quantity (the counts then move to a byte array).

template <int R, bool WITHV, int TH = TH_DEFAULT>
__device__ __forceinline__ void stage_b_cmp(const float* sJ, const float* sI, float4* sH, unsigned char* sV, int tid) {
    using G = Geom<R, TH>;
    constexpr int RA = G::RA, HR = G::HR, JP = G::JP, P = G::P, NSEG = G::NSEG, NIN = G::NIN;
    if (tid >= HR * NSEG) return;
    const int sg = tid / HR, hy = tid - sg * HR;
    MVS_BOUND(hy < HR && P * sg + P <= TW && hy * JP + P * sg + NIN <= HR * JP);
    const float4* jr = reinterpret_cast<const float4*>(sJ + hy * JP + P * sg);
    const float4* ir = reinterpret_cast<const float4*>(sI + hy * JP + P * sg);
    float v[NIN], s0[NIN], s1[NIN], s2[NIN], s3[NIN];
#pragma unroll
    for (int q = 0; q < NIN / 4; ++q) {
        const float4 a = jr[q], b = ir[q];
        const float jv[4] = {a.x, a.y, a.z, a.w}, iv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = 4 * q + u;
            float jz = jv[u];
            if constexpr (WITHV) {
                const bool ok = jz == jz;
                jz = ok ? jz : 0.f;
                v[t] = ok ? 1.f : 0.f;
                s0[t] = ok ? iv[u] : 0.f;
            }
            s1[t] = jz;
            s2[t] = __fmul_rn(jz, jz);
            s3[t] = __fmul_rn(jz, iv[u]);
        }
    }
    float a0 = 0.f, a4 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
    for (int t = RA - R; t <= RA + R; ++t) {
        if constexpr (WITHV) {
            a0 = __fadd_rn(a0, v[t]);
            a4 = __fadd_rn(a4, s0[t]);
        }
        a1 = __fadd_rn(a1, s1[t]);
        a2 = __fadd_rn(a2, s2[t]);
        a3 = __fadd_rn(a3, s3[t]);
    }
    float4* row = sH + hy * TW + P * sg;
    unsigned char* crow = sV + hy * TW + P * sg;
    const int kx = (sg + hy) & 7;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (j > 0) {
            const int tn = RA + R + j, to = RA - R + j - 1;
            if constexpr (WITHV) {
                a0 = __fadd_rn(a0, __fsub_rn(v[tn], v[to]));
                a4 = __fadd_rn(a4, __fsub_rn(s0[tn], s0[to]));
            }
            a1 = __fadd_rn(a1, __fsub_rn(s1[tn], s1[to]));
            a2 = __fadd_rn(a2, __fsub_rn(s2[tn], s2[to]));
            a3 = __fadd_rn(a3, __fsub_rn(s3[tn], s3[to]));
        }
        row[j ^ kx] = make_float4(a4, a1, a2, a3);
        if constexpr (WITHV) crow[j] = (unsigned char)a0;
    }
}

// Kahan step: s += x with the running compensation c (s - c is the better estimate).
__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
}

// `mu` holds the pivoted window mean mu' = mu - p and `rsd` the reciprocal window deviation, both
// formed from the pivoted reference tile.
template <int R, int KMAX, bool WITHV, int TH = TH_DEFAULT>
__device__ __forceinline__ void stage_c_cmp(const float4* sH, const unsigned char* sV, int c, int y0, const float* mu,
                                            const float* rsd, float pv, float (&topk)[ROWS][KMAX], float* total,
                                            bool bottom, int nlist) {
    constexpr int K = 2 * R + 1;
    const float k2 = (float)(K * K), inv_k2 = 1.0f / (float)(K * K);
    static_assert(ROWS % 8 == 0, "stage C rows must start on a multiple of 8");
    int sw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) sw[k] = c ^ (((c >> 4) + k) & 7);
    const float4* col = sH + y0 * TW;
    MVS_BOUND(y0 + ROWS + 2 * R <= (Geom<R, TH>::HR) && c < TW);
    const unsigned char* ccol = sV + y0 * TW + c;
    float cv = 0.f, ci = 0.f, cj = 0.f, cjj = 0.f, cji = 0.f;
    float ej = 0.f, ejj = 0.f, eji = 0.f;            // Kahan compensations
#pragma unroll
    for (int t = 0; t < K; ++t) {
        const float4 h = col[t * TW + sw[t & 7]];
        if constexpr (WITHV) {
            cv = __fadd_rn(cv, (float)ccol[t * TW]);
            ci = __fadd_rn(ci, h.x);
        }
        kahan_add(cj, ej, h.y);
        kahan_add(cjj, ejj, h.z);
        kahan_add(cji, eji, h.w);
    }
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        if (j > 0) {
            const float4 hn = col[(j + 2 * R) * TW + sw[(j + 2 * R) & 7]];
            const float4 ho = col[(j - 1) * TW + sw[(j - 1) & 7]];
            if constexpr (WITHV) {
                cv = __fadd_rn(cv, __fsub_rn((float)ccol[(j + 2 * R) * TW], (float)ccol[(j - 1) * TW]));
                ci = __fadd_rn(ci, __fsub_rn(hn.x, ho.x));
            }
            kahan_add(cj, ej, hn.y);
            kahan_add(cj, ej, -ho.y);
            kahan_add(cjj, ejj, hn.z);
            kahan_add(cjj, ejj, -ho.z);
            kahan_add(cji, eji, hn.w);
            kahan_add(cji, eji, -ho.w);
        }
        float ncc;
        if (WITHV && cv * 10.f <= 9.f * k2) {
            ncc = -1.f;
        } else {
            const float rc = (!WITHV || cv == k2) ? inv_k2 : __frcp_rn(cv);
            const float mj = __fmul_rn(__fsub_rn(cj, ej), rc), m2 = __fmul_rn(__fsub_rn(cjj, ejj), rc);
            const float mij = __fmul_rn(__fsub_rn(cji, eji), rc);
            const float var = __fsub_rn(m2, __fmul_rn(mj, mj));
            const float rsdj = var > 1e-6f ? rsqrtf(var) : 1000.f;
            float cov = __fsub_rn(mij, __fmul_rn(mu[j], mj));
            if (WITHV) cov = __fadd_rn(cov, __fmul_rn(pv, __fsub_rn(__fmul_rn(ci, rc), mu[j])));
            ncc = __fmul_rn(cov, __fmul_rn(rsd[j], rsdj));
            ncc = ncc > 1.f ? 1.f : (ncc < -1.f ? -1.f : ncc);
        }
        if (bottom) total[j] = __fadd_rn(total[j], ncc);
        float x = ncc;
#pragma unroll
        for (int q = 0; q < KMAX; ++q) {
            if (q < nlist) {
                const float hi = fmaxf(topk[j][q], x), lo = fminf(topk[j][q], x);
                topk[j][q] = bottom ? lo : hi;
                x = bottom ? hi : lo;
            }
        }
    }
}

// ---- the reference tile by TMA (single-view kernel): one 2D tiled bulk copy per CTA, completed
// on an mbarrier. The copy's box is the tile with its halo, JP x HR floats starting at
// (tx - RA, ty - R): x is a multiple of 4 floats (16 bytes), rows outside the image read as 0,
// as the per-thread loads give.

// Tiles whose reference-tile copy did not complete within the bounded wait (read and cleared by
// mvs_device_faults). The counter exists in the one translation unit that instantiates the TMA
// kernels (sweep.cu defines MVS_SWEEP_TMA_UNIT before including this header); elsewhere a
// REF_TMA instantiation does not compile, so no second, unread copy of the counter can arise.
#ifdef MVS_SWEEP_TMA_UNIT
static __device__ unsigned g_ref_copy_faults;
#endif

constexpr unsigned MVS_WAIT_LIMIT_DEFAULT = 1u << 20;   // try_wait iterations of a bounded wait

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar,
                                            unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Bounded wait for phase `parity` of an mbarrier: false if it did not complete within `limit`
// try_wait iterations.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned limit) {
    for (unsigned it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One tile x hypothesis range at window radius R. `chunk` >= 0 writes the chunk record `chunk`
// of p.nchunks instead of the caller's state. Explicit _rn arithmetic in stages B and C fixes
// every rounding, so the result never depends on how the compiler scheduled this instance.
// WIDE: interior tiles gather all of a thread's warp samples before storing any (more loads in
// flight; more registers - the single-view kernel, whose radius is a template argument, uses it).
// REF_TMA: the reference tile arrives by TMA when p.ref_tma is set (the single-view kernel, whose
// parameters hold the tensor map; `smem` must then be 128-byte aligned).
template <int R, int KMAX, bool PLANES, bool F16, bool WIDE = false, bool REF_TMA = false, bool X64 = false,
          bool CMP = false, int TH = TH_DEFAULT>
__device__ void sweep_tile(const SweepParams& p, int tx, int ty, int pa, int pb, int chunk, float* smem) {
    using G = Geom<R, TH>;
    constexpr int NT = TileShape<TH>::NT, SEG = TileShape<TH>::SEG;
    constexpr int K = G::K, RA = G::RA, HR = G::HR, HC = G::HC, JP = G::JP, P = G::P, NSEG = G::NSEG,
                  NIN = G::NIN;
    float* sI = smem;                                  // HR x JP reference (0 outside); TMA destination
    float* sJ = sI + HR * JP;                          // HR x JP warped source (NaN = invalid)
    float4* sH = reinterpret_cast<float4*>(sJ + HR * JP);   // HR x TW (V, J, J^2, J I), swizzled
    const int H = p.H, W = p.W;
    const int tid = threadIdx.x;

    __syncthreads();   // a previous tile of a persistent CTA is done with shared memory
    bool tma = false;
    __shared__ __align__(8) unsigned long long s_ref_bar;
#ifndef MVS_SWEEP_TMA_UNIT
    static_assert(!REF_TMA, "REF_TMA kernels are instantiated in sweep.cu only (it owns the fault counter)");
#else
    if constexpr (REF_TMA) {
        tma = p.ref_tma != 0;
        if (tma && tid == 0) {
            mbar_init(&s_ref_bar, 1);
            tma_load_2d(sI, &p.ref_map, tx - RA, ty - R, &s_ref_bar, (unsigned)(HR * JP * sizeof(float)));
        }
    }
#endif
    for (int e = tid; e < HR * JP; e += NT) {
        if (!tma) {
            const int hy = e / JP, hc = e - hy * JP;
            const int gy = ty - R + hy, gx = tx - RA + hc;
            float v = 0.f;
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) v = __ldg(p.ref + (long long)gy * W + gx);
            sI[e] = v;
        }
        sJ[e] = qnan();
    }

    // winner-take-all state of the tile's pixels: touched once per hypothesis, so it lives in
    // shared memory (planes: best, prev, s_prev_best, s_next_best, first score, idx bits)
    float* sW = reinterpret_cast<float*>(sH + HR * TW);
    Coef* sC = reinterpret_cast<Coef*>(sW + 6 * TH * TW);
    const int c = tid % TW, seg = tid / TW;
    const float fcol = (float)c, fseg = (float)seg;
    const int gx = tx + c;
    float mu[ROWS], rsd[ROWS];
    const bool to_rec = chunk >= 0;
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int ly = seg * ROWS + j, gy = ty + ly;
        const bool in = gx < W && gy < H;
        const long long o = (long long)gy * W + gx;
        // (compensated mode: formed from the pivoted tile below instead)
        mu[j] = in && !CMP ? __ldg(p.mu + o) : 0.f;
        // X64: the deviation itself (stage C divides in float64); else its reciprocal
        rsd[j] = in && !CMP ? (X64 ? __ldg(p.sd + o) : 1.0f / __ldg(p.sd + o)) : 0.f;
        const bool load = in && !to_rec && !p.fresh;
        const int w = ly * TW + c;
        sW[w] = load ? p.best[o] : -2.f;
        sW[TH * TW + w] = load ? p.prev[o] : -2.f;
        sW[2 * TH * TW + w] = load ? p.spb[o] : -2.f;
        sW[3 * TH * TW + w] = load ? p.snb[o] : -2.f;
        sW[4 * TH * TW + w] = -2.f;
        sW[5 * TH * TW + w] = __int_as_float(load ? p.idx[o] : -1);
    }
    const int nsrc = p.n_src, kk = p.kk;
    const bool bottom = KMAX > 2 && p.topk_bottom != 0;   // the 2-entry list is always a top list
    const int nlist = bottom ? nsrc - kk : kk;
    // every halo sample lies inside the reference image (interior tile)
    const bool tile_inside = tx - R >= 0 && ty - R >= 0 && tx + TW + R <= W && ty + TH + R <= H;
#ifdef MVS_SWEEP_TMA_UNIT
    if constexpr (REF_TMA) {
        if (tma) {
            __syncthreads();   // the barrier's initialisation is visible to every thread
            const bool arrived = mbar_wait_bounded(&s_ref_bar, 0, p.wait_limit);
            // a copy that did not complete in time: count it and leave the tile's state untouched.
            // Before the CTA (and its shared memory) goes, wait once more, with the default
            // bound, for the copy that may still be in flight into that memory.
            if (__syncthreads_or(!arrived)) {
                if (tid == 0) {
                    atomicAdd(&g_ref_copy_faults, 1u);
                    mbar_wait_bounded(&s_ref_bar, 0, MVS_WAIT_LIMIT_DEFAULT);
                }
                __syncthreads();
                return;
            }
        }
    }
#endif
    // compensated mode: pivot the reference tile and form its window statistics from it
    float pv = 0.f;
    unsigned char* sV = reinterpret_cast<unsigned char*>(sC + MVS_MAX_SOURCES);   // byte counts
    if constexpr (CMP) {
        __shared__ float red[2 * (NT / 32)];
        __syncthreads();                       // the reference tile is complete (thread loads or TMA)
        float su = 0.f, nn = 0.f;
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            const int ly = seg * ROWS + j;
            if (gx < W && ty + ly < H) {
                su = __fadd_rn(su, sI[(ly + R) * JP + RA + c]);
                nn += 1.f;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            su = __fadd_rn(su, __shfl_xor_sync(0xffffffffu, su, o));
            nn += __shfl_xor_sync(0xffffffffu, nn, o);
        }
        if ((tid & 31) == 0) {
            red[tid >> 5] = su;
            red[NT / 32 + (tid >> 5)] = nn;
        }
        __syncthreads();
        su = 0.f;
        nn = 0.f;
        for (int w = 0; w < NT / 32; ++w) {   // every thread sums the warp totals in the same order
            su = __fadd_rn(su, red[w]);
            nn += red[NT / 32 + w];
        }
        pv = nn > 0.f ? __fdiv_rn(su, nn) : 0.f;
        for (int e = tid; e < HR * JP; e += NT) sI[e] = __fsub_rn(sI[e], pv);
        __syncthreads();
        // mu' = sum(I') / k^2 over the zero-padded window (I' = -p outside the image), var =
        // sum(I'^2) / k^2 - mu'^2, sd = sqrt(max(var, 1e-6)): the reference's statistics, pivoted
        const float inv_k2 = 1.0f / (float)(K * K);
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            const int ly = seg * ROWS + j;
            float s1 = 0.f, s2 = 0.f;
#pragma unroll 1
            for (int dy = 0; dy < K; ++dy) {
                const float* rowp = sI + (ly + dy) * JP + (RA - R) + c;
#pragma unroll
                for (int dx = 0; dx < K; ++dx) {
                    const float v = rowp[dx];
                    s1 = __fadd_rn(s1, v);
                    s2 = __fmaf_rn(v, v, s2);
                }
            }
            const float m = __fmul_rn(s1, inv_k2);
            const float var = __fsub_rn(__fmul_rn(s2, inv_k2), __fmul_rn(m, m));
            const bool in = gx < W && ty + ly < H;
            mu[j] = in ? m : 0.f;
            rsd[j] = in ? __frcp_rn(__fsqrt_rn(var > 1e-6f ? var : 1e-6f)) : 0.f;
        }
    }

    for (int i = pa; i < pb; ++i) {
        float topk[ROWS][KMAX];
        float total[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            total[j] = 0.f;
#pragma unroll
            for (int q = 0; q < KMAX; ++q) topk[j][q] = bottom ? INFINITY : -INFINITY;
        }
        if constexpr (PLANES) {
            __syncthreads();   // the previous hypothesis is done reading sC
            if (tid < 4 * MVS_MAX_SOURCES && (tid >> 5) * 8 < nsrc) {   // the warps that hold a source
                const int sg_ = tid >> 2;
                make_coef_group(sC[sg_ < nsrc ? sg_ : 0], p.src[sg_ < nsrc ? sg_ : 0], p.planes[i - p.i0], tx - R,
                                ty - R, HC, HR, sg_ < nsrc);
            }
        }
        for (int s = 0; s < nsrc; ++s) {
            __syncthreads();   // sC ready; the previous stage B is done with sJ
            // ---- A: warp the source into the halo tile
            const void* img = p.src[s].img;
            const int sw = p.src[s].w, sh = p.src[s].h;
            bool any_invalid = false;
            if constexpr (PLANES) {
                const Coef cf = sC[s];
                constexpr int PER = (HR * HC + NT - 1) / NT;
                if (WIDE && cf.inside && tile_inside) {
                    // every sample of the thread gathered before any is stored: the gathers are
                    // independent and in flight together. The thread keeps halo column c and
                    // rows seg, seg + SEG, ... (positions and shared offsets fixed per thread, so
                    // no per-sample index arithmetic); the 2R right-hand halo columns are spread
                    // over all threads. A surplus row repeats the last row and is not stored.
                    constexpr int MR = (HR + SEG - 1) / SEG;
                    constexpr int XW = R > 0 ? 2 * R : 1, XS = 2 * R * HR, PX = (XS + NT - 1) / NT;
                    float Jv[MR + PX];
#pragma unroll
                    for (int k = 0; k < MR; ++k) {
                        const float b = (k + 1) * SEG > HR ? fminf(fseg + (float)(k * SEG), (float)(HR - 1))
                                                           : fseg + (float)(k * SEG);
                        Jv[k] = sample_plane_inside<F16>(cf, img, sw, sh, fcol, b);
                    }
#pragma unroll
                    for (int m = 0; m < PX; ++m) {
                        const int e0 = tid + m * NT;
                        const int e = e0 < XS ? e0 : XS - 1;
                        const int hy = e / XW, hc = TW + (e - hy * XW);
                        Jv[MR + m] = sample_plane_inside<F16>(cf, img, sw, sh, (float)hc, (float)hy);
                    }
                    float* col = sJ + seg * JP + (RA - R) + c;
#pragma unroll
                    for (int k = 0; k < MR; ++k) {
                        if ((k + 1) * SEG <= HR || seg + k * SEG < HR) {
                            MVS_BOUND((seg + k * SEG) * JP + (RA - R) + c < HR * JP);
                            any_invalid |= Jv[k] != Jv[k];
                            col[k * SEG * JP] = CMP ? __fsub_rn(Jv[k], pv) : Jv[k];
                        }
                    }
#pragma unroll
                    for (int m = 0; m < PX; ++m) {
                        const int e0 = tid + m * NT;
                        if (e0 < XS) {
                            const int hy = e0 / XW, hc = TW + (e0 - hy * XW);
                            MVS_BOUND(hy * JP + (RA - R) + hc < HR * JP);
                            any_invalid |= Jv[MR + m] != Jv[MR + m];
                            sJ[hy * JP + (RA - R) + hc] = CMP ? __fsub_rn(Jv[MR + m], pv) : Jv[MR + m];
                        }
                    }
                } else if (cf.inside && tile_inside) {
#pragma unroll 4
                    for (int k = 0; k < PER; ++k) {
                        const int e = tid + k * NT;
                        if (e < HR * HC) {
                            const int hy = e / HC, hc = e - hy * HC;
                            const float J = sample_plane_inside<F16>(cf, img, sw, sh, (float)hc, (float)hy);
                            MVS_BOUND(hy * JP + (RA - R) + hc < HR * JP);
                            any_invalid |= J != J;
                            sJ[hy * JP + (RA - R) + hc] = CMP ? __fsub_rn(J, pv) : J;
                        }
                    }
                } else {
#pragma unroll 4
                    for (int k = 0; k < PER; ++k) {
                        const int e = tid + k * NT;
                        if (e < HR * HC) {
                            const int hy = e / HC, hc = e - hy * HC;
                            const int gy = ty - R + hy, gxx = tx - R + hc;
                            const bool in = gy >= 0 && gy < H && gxx >= 0 && gxx < W;
                            const float J = sample_plane<F16>(cf, img, sw, sh, (float)hc, (float)hy, in);
                            MVS_BOUND(hy * JP + (RA - R) + hc < HR * JP);
                            any_invalid |= J != J;
                            sJ[hy * JP + (RA - R) + hc] = CMP ? __fsub_rn(J, pv) : J;
                        }
                    }
                }
            } else {
                any_invalid = true;
                for (int e = tid; e < HR * HC; e += NT) {
                    const int hy = e / HC, hc = e - hy * HC;
                    const int gy = ty - R + hy, gxx = tx - R + hc;
                    float J = qnan();
                    if (gy >= 0 && gy < H && gxx >= 0 && gxx < W) J = sample_ray(p, p.src[s], i, gxx, gy);
                    sJ[hy * JP + (RA - R) + hc] = CMP ? __fsub_rn(J, pv) : J;
                }
            }
            // every sample of this (hypothesis, source) valid -> the count is k^2 everywhere and
            // stages B and C skip it (block-wide vote; uniform branch)
            const bool all_valid = !__syncthreads_or(any_invalid);
            // ---- B: horizontal window sums of (V, J, J^2, J I), one 16-column row segment per
            // thread: products once per input, running sums along the segment
            if constexpr (CMP) {
                if (all_valid) {
                    stage_b_cmp<R, false, TH>(sJ, sI, sH, sV, tid);
                } else {
                    stage_b_cmp<R, true, TH>(sJ, sI, sH, sV, tid);
                }
            } else if constexpr (X64) {
                if (all_valid) {
                    stage_b64<R, false, TH>(sJ, sI, sH, tid);
                } else {
                    stage_b64<R, true, TH>(sJ, sI, sH, tid);
                }
            } else if (all_valid) {
                stage_b<R, false, TH>(sJ, sI, sH, tid);
            } else {
                stage_b<R, true, TH>(sJ, sI, sH, tid);
            }
            __syncthreads();
            // ---- C: vertical running sums down the column, NCC, top-k insertion
            if constexpr (CMP) {
                if (all_valid) {
                    stage_c_cmp<R, KMAX, false, TH>(sH, sV, c, seg * ROWS, mu, rsd, pv, topk, total, bottom, nlist);
                } else {
                    stage_c_cmp<R, KMAX, true, TH>(sH, sV, c, seg * ROWS, mu, rsd, pv, topk, total, bottom, nlist);
                }
            } else if constexpr (X64) {
                if (all_valid) {
                    stage_c64<R, KMAX, false, TH>(sH, c, seg * ROWS, mu, rsd, topk, total, bottom, nlist);
                } else {
                    stage_c64<R, KMAX, true, TH>(sH, c, seg * ROWS, mu, rsd, topk, total, bottom, nlist);
                }
            } else if (all_valid) {
                stage_c<R, KMAX, false, TH>(sH, c, seg * ROWS, mu, rsd, topk, total, bottom, nlist);
            } else {
                stage_c<R, KMAX, true, TH>(sH, c, seg * ROWS, mu, rsd, topk, total, bottom, nlist);
            }
        }
        // ---- winner-take-all update for hypothesis i
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            float sc = 0.f;
#pragma unroll
            for (int q = 0; q < KMAX; ++q)
                if (q < nlist) sc = __fadd_rn(sc, topk[j][q]);
            if (bottom) sc = __fsub_rn(total[j], sc);
            sc = __fdiv_rn(sc, (float)kk);
            const int w = (seg * ROWS + j) * TW + c;
            MVS_BOUND(w < TH * TW);
            float best = sW[w], prv = sW[TH * TW + w];
            const int id = __float_as_int(sW[5 * TH * TW + w]);
            if (id == i - 1) sW[3 * TH * TW + w] = sc;
            if (sc > best) {
                sW[w] = sc;
                sW[2 * TH * TW + w] = prv;
                sW[3 * TH * TW + w] = -2.f;
                sW[5 * TH * TW + w] = __int_as_float(i);
            }
            sW[TH * TW + w] = sc;
            if (i == pa) sW[4 * TH * TW + w] = sc;
        }
    }

    // ---- write back: caller state (single chunk) or the chunk record
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int gy = ty + seg * ROWS + j;
        if (gx >= W || gy >= H) continue;
        const long long o = (long long)gy * W + gx;
        const int w = (seg * ROWS + j) * TW + c;
        if (!to_rec) {
            p.best[o] = sW[w];
            p.prev[o] = sW[TH * TW + w];
            p.spb[o] = sW[2 * TH * TW + w];
            p.snb[o] = sW[3 * TH * TW + w];
            p.idx[o] = __float_as_int(sW[5 * TH * TW + w]);
        } else {
            const long long HW = (long long)H * W;
            const long long plane = (long long)p.nchunks * HW;
            float* rc = p.rec + (long long)chunk * HW + o;
            rc[0] = sW[w];
            rc[plane] = sW[5 * TH * TW + w];
            rc[2 * plane] = sW[2 * TH * TW + w];
            rc[3 * plane] = sW[3 * TH * TW + w];
            rc[4 * plane] = sW[4 * TH * TW + w];
            rc[5 * plane] = sW[TH * TW + w];
        }
    }
}

// Ordered merge of one pixel's chunk records into its state (hypothesis order, first wins).
__device__ __forceinline__ void merge_pixel(long long o, long long HW, int nchunks, int i0, int i1, int ppc,
                                            const float* __restrict__ rec, float& B, float& P, float& SP,
                                            float& SN, int& I) {
    const long long plane = (long long)nchunks * HW;
    for (int ch = 0; ch < nchunks; ++ch) {
        const int a = i0 + ch * ppc, b = min(i1, a + ppc);
        if (a >= b) break;
        const float* r = rec + (long long)ch * HW + o;
        const float cb = r[0];
        const int ci = __float_as_int(r[plane]);
        const float cp = r[2 * plane], cn = r[3 * plane], cf = r[4 * plane], cl = r[5 * plane];
        if (I == a - 1) SN = cf;
        if (cb > B) {
            B = cb;
            I = ci;
            SP = (ci > a) ? cp : P;
            SN = (ci < b - 1) ? cn : -2.f;
        }
        P = cl;
    }
}

// densify.py:354-361: parabola through (idx-1, idx, idx+1) in float32, depth in float64.
__device__ __forceinline__ float finalize_pixel(float inv0, float inv1, int n, float bb, float sp, float sn, int id) {
    const float dinv = n > 1 ? __fsub_rn(inv1, inv0) : 0.f;
    const float den = __fadd_rn(__fsub_rn(sp, __fmul_rn(2.f, bb)), sn);
    const bool interior = id > 0 && id < n - 1 && den < -1e-6f;
    float off = 0.f;
    if (interior) off = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(sp, sn)), den);
    off = off < -0.5f ? -0.5f : (off > 0.5f ? 0.5f : off);
    const double t = __dadd_rn((double)id, (double)off);
    const double inv = __dadd_rn((double)inv0, __dmul_rn(t, (double)dinv));
    const double m = max_nan(inv, 1e-9);
    return (float)__ddiv_rn(1.0, m);
}

// host-side helpers shared by sweep.cu and batch.cu
inline int tile_height(const mvs_sweep_args* a) { return a->tile_h ? a->tile_h : TH_DEFAULT; }
mvs_status validate_sweep(const mvs_sweep_args* a);
mvs_status fill_params(const mvs_sweep_args* a, SweepParams& p);
int pick_kmax(SweepParams& p);

}  // namespace mvs
