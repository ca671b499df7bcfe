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
//   A. warp the source into a shared-memory tile with an r-pixel halo (NaN = invalid sample),
//   B. horizontal window sums of (V, J, J^2, J*I) for groups of 4 columns from 16-byte
//      shared-memory loads,
//   C. vertical running sums down each column (TH/SEG rows per thread), NCC, insertion into a
//      per-pixel top-k list in registers.
// After the last source the winner-take-all state of each pixel is updated in registers; it
// leaves the SM once per hypothesis chunk. Window sums are short FP32 sums (at most TH/SEG
// add/subtract steps), so the reference's float64 running sums are not needed.
#pragma once

#include "common.cuh"

namespace mvs {

constexpr int TW = 64;                 // output tile width (columns)
constexpr int TH = 32;                 // output tile height (rows)
constexpr int NT = 256;                // threads per CTA
constexpr int SEG = NT / TW;           // row segments in stage C
constexpr int ROWS = TH / SEG;         // output rows per thread in stage C

struct SrcGeo {
    const void* img;                   // float or __half, (h, w) row-major
    int h, w;
    double m[9];                       // PLANES: A = Rs R_ref^T K_ref^-1; ray path: Rs
    double b[3];                       // Rs (C_ref - C_src)
    double f, k1, k2, k3, cx, cy;
};

struct SweepParams {
    int H, W, n_src, kk;
    int topk_bottom;                   // 1: keep the n-kk lowest and subtract from the total
    int i0, i1, ppc;                   // hypotheses [i0, i1), planes per chunk
    int hyp_kind, t0;
    int r, nchunks;
    int fresh;                         // 1: start from the initial state instead of loading it
    int pad_;
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
};

template <int RMAX>
struct Geom {
    static constexpr int RA = (RMAX + 3) & ~3;     // halo rounded up to a float4
    static constexpr int HRM = TH + 2 * RMAX;      // sampled rows (maximum)
    static constexpr int HCM = TW + 2 * RMAX;      // sampled columns (maximum)
    static constexpr int JP = TW + 2 * RA;         // shared row pitch
    static constexpr int NG = TW / 4;              // stage-B column groups
    static constexpr int NIN = 2 * RA + 4;         // stage-B inputs per group
    static constexpr size_t smem_bytes() {
        return (size_t)HRM * JP * 4 * 2 + (size_t)4 * HRM * TW * 4 + sizeof(Coef) * MVS_MAX_SOURCES;
    }
};

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fc00000); }

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

// Homography path sample (pinhole, constant inverse depth per hypothesis).
template <bool F16>
__device__ __forceinline__ float sample_plane(const Coef& c, const void* img, int w, int h, float a, float b) {
    const float dz = fmaf(c.dz1, a, fmaf(c.dz2, b, c.dz0));
    if (!(c.zs * dz > 1e-6f)) return qnan();
    const float rz = __fdividef(1.0f, dz);
    const float ul = fmaf(c.nu1, a, fmaf(c.nu2, b, c.nu0)) * rz;
    const float vl = fmaf(c.nv1, a, fmaf(c.nv2, b, c.nv0)) * rz;
    if (!(ul >= c.lo_u && ul <= c.hi_u && vl >= c.lo_v && vl <= c.hi_v)) return qnan();
    const float fu = floorf(ul), fv = floorf(vl);
    const int x0 = c.U0 + (int)fu, y0 = c.V0 + (int)fv;
    // integer guard: every tap stays inside the image whatever the float rounding did
    if ((unsigned)x0 >= (unsigned)(w - 1) || (unsigned)y0 >= (unsigned)(h - 1)) return qnan();
    const float fx = ul - fu, fy = vl - fv;
    const long long o = (long long)y0 * w + x0;
    const float a00 = tap<F16>(img, o), a01 = tap<F16>(img, o + 1);
    const float a10 = tap<F16>(img, o + w), a11 = tap<F16>(img, o + w + 1);
    const float top = fmaf(fx, a01 - a00, a00);
    const float bot = fmaf(fx, a11 - a10, a10);
    const float val = fmaf(fy, bot - top, top);
    return isfinite(val) ? val : qnan();
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
    const double a00 = tap<false>(g.img, so), a01 = tap<false>(g.img, so + 1);
    const double a10 = tap<false>(g.img, so + g.w), a11 = tap<false>(g.img, so + g.w + 1);
    const double val = (a00 * (1.0 - fx) + a01 * fx) * (1.0 - fy) + (a10 * (1.0 - fx) + a11 * fx) * fy;
    return isfinite(val) ? (float)val : qnan();
}

__device__ inline void make_coef(Coef& c, const SrcGeo& g, float inv, int ox, int oy) {
    const double d = 1.0 / (double)inv;
    double g0[3], g1[3], g2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        g1[k] = d * g.m[3 * k + 0];
        g2[k] = d * g.m[3 * k + 1];
        g0[k] = d * (g.m[3 * k + 0] * (double)ox + g.m[3 * k + 1] * (double)oy + g.m[3 * k + 2]) + g.b[k];
    }
    const double Z0 = g0[2];
    const bool norm = fabs(Z0) > 1e-9;
    const double zs = norm ? Z0 : 1.0;
    double U0 = 0.0, V0 = 0.0;
    if (norm) {
        const double u00 = g.f * g0[0] / Z0 + g.cx, v00 = g.f * g0[1] / Z0 + g.cy;
        if (isfinite(u00)) U0 = fmin(fmax(floor(u00), -1048576.0), 1048576.0);
        if (isfinite(v00)) V0 = fmin(fmax(floor(v00), -1048576.0), 1048576.0);
    }
    const double au = g.cx - U0, av = g.cy - V0;
    c.nu0 = (float)((g.f * g0[0] + au * g0[2]) / zs);
    c.nu1 = (float)((g.f * g1[0] + au * g1[2]) / zs);
    c.nu2 = (float)((g.f * g2[0] + au * g2[2]) / zs);
    c.nv0 = (float)((g.f * g0[1] + av * g0[2]) / zs);
    c.nv1 = (float)((g.f * g1[1] + av * g1[2]) / zs);
    c.nv2 = (float)((g.f * g2[1] + av * g2[2]) / zs);
    c.dz0 = (float)(g0[2] / zs);
    c.dz1 = (float)(g1[2] / zs);
    c.dz2 = (float)(g2[2] / zs);
    c.zs = (float)zs;
    c.lo_u = (float)(-U0);
    c.lo_v = (float)(-V0);
    c.hi_u = (float)(((double)g.w - 1.001) - U0);
    c.hi_v = (float)(((double)g.h - 1.001) - V0);
    c.U0 = (int)U0;
    c.V0 = (int)V0;
}

// One tile x hypothesis range. DYN = false: r == RMAX at compile time (fully unrolled windows);
// DYN = true: runtime r <= RMAX (batched jobs of mixed radius). `chunk` >= 0 writes the chunk
// record `chunk` of p.nchunks instead of the caller's state.
template <int RMAX, bool DYN, int KMAX, bool PLANES, bool F16>
__device__ void sweep_tile(const SweepParams& p, int r_dyn, int tx, int ty, int pa, int pb, int chunk, float* smem) {
    using G = Geom<RMAX>;
    constexpr int RA = G::RA, HRM = G::HRM, HCM = G::HCM, JP = G::JP, NG = G::NG, NIN = G::NIN;
    const int r = DYN ? r_dyn : RMAX;
    const int K = 2 * r + 1;
    const int HR = TH + 2 * r;
    float* sJ = smem;                                  // HRM x JP warped source (NaN = invalid)
    float* sI = sJ + HRM * JP;                         // HRM x JP reference (0 outside)
    float* sH = sI + HRM * JP;                         // 4 x HRM x TW horizontal sums
    Coef* sC = reinterpret_cast<Coef*>(sH + 4 * HRM * TW);
    const int H = p.H, W = p.W;
    const int tid = threadIdx.x;

    __syncthreads();   // a previous tile of a persistent CTA is done with shared memory
    for (int e = tid; e < HRM * JP; e += NT) {
        const int hy = e / JP, hc = e - hy * JP;
        const int gy = ty - r + hy, gx = tx - RA + hc;
        float v = 0.f;
        if (hy < HR && gy >= 0 && gy < H && gx >= 0 && gx < W) v = __ldg(p.ref + (long long)gy * W + gx);
        sI[e] = v;
        sJ[e] = qnan();
    }

    const int c = tid % TW, seg = tid / TW;
    const int gx = tx + c;
    float mu[ROWS], rsd[ROWS], best[ROWS], prv[ROWS], spb[ROWS], snb[ROWS], first[ROWS];
    int idx[ROWS];
    const bool to_rec = chunk >= 0;
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int gy = ty + seg * ROWS + j;
        const bool in = gx < W && gy < H;
        const long long o = (long long)gy * W + gx;
        mu[j] = in ? __ldg(p.mu + o) : 0.f;
        rsd[j] = in ? 1.0f / __ldg(p.sd + o) : 0.f;
        if (in && !to_rec && !p.fresh) {
            best[j] = p.best[o];
            prv[j] = p.prev[o];
            spb[j] = p.spb[o];
            snb[j] = p.snb[o];
            idx[j] = p.idx[o];
        } else {
            best[j] = -2.f;
            prv[j] = -2.f;
            spb[j] = -2.f;
            snb[j] = -2.f;
            idx[j] = -1;
        }
        first[j] = -2.f;
    }
    const float k2 = (float)(K * K), inv_k2 = 1.0f / (float)(K * K);
    const int nsrc = p.n_src, kk = p.kk;
    const bool bottom = p.topk_bottom != 0;
    const int nlist = bottom ? nsrc - kk : kk;

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
            if (tid < nsrc) make_coef(sC[tid], p.src[tid], p.planes[i - p.i0], tx - r, ty - r);
        }
        for (int s = 0; s < nsrc; ++s) {
            __syncthreads();   // sC ready; the previous stage B is done with sJ
            // ---- A: warp the source into the halo tile
            const void* img = p.src[s].img;
            const int sw = p.src[s].w, sh = p.src[s].h;
            for (int e = tid; e < HRM * HCM; e += NT) {
                const int hy = e / HCM, hc = e - hy * HCM;
                if (hy >= HR || hc >= TW + 2 * r) continue;
                const int gy = ty - r + hy, gxx = tx - r + hc;
                float J = qnan();
                if (gy >= 0 && gy < H && gxx >= 0 && gxx < W) {
                    if constexpr (PLANES) {
                        J = sample_plane<F16>(sC[s], img, sw, sh, (float)hc, (float)hy);
                    } else {
                        J = sample_ray(p, p.src[s], i, gxx, gy);
                    }
                }
                sJ[hy * JP + (RA - r) + hc] = J;
            }
            __syncthreads();
            // ---- B: horizontal sums of V, J, J^2, J*I for 4 output columns per item
            for (int e = tid; e < HRM * NG; e += NT) {
                const int hy = e / NG, gi = e - hy * NG;
                if (hy >= HR) continue;
                const float4* jr = reinterpret_cast<const float4*>(sJ + hy * JP + 4 * gi);
                const float4* ir = reinterpret_cast<const float4*>(sI + hy * JP + 4 * gi);
                float jv[NIN], iv[NIN];
#pragma unroll
                for (int q = 0; q < NIN / 4; ++q) {
                    const float4 a = jr[q], b = ir[q];
                    jv[4 * q] = a.x; jv[4 * q + 1] = a.y; jv[4 * q + 2] = a.z; jv[4 * q + 3] = a.w;
                    iv[4 * q] = b.x; iv[4 * q + 1] = b.y; iv[4 * q + 2] = b.z; iv[4 * q + 3] = b.w;
                }
                // explicit rounding (no contraction) so that every instantiation - static or
                // runtime radius - produces the same bits
                float v[NIN], s1[NIN], s2[NIN], s3[NIN];
#pragma unroll
                for (int t = 0; t < NIN; ++t) {
                    const bool ok = jv[t] == jv[t];
                    const float jz = ok ? jv[t] : 0.f;
                    v[t] = ok ? 1.f : 0.f;
                    s1[t] = jz;
                    s2[t] = __fmul_rn(jz, jz);
                    s3[t] = __fmul_rn(jz, iv[t]);
                }
                float o0[4], o1[4], o2[4], o3[4];
                float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
                for (int t = -RMAX; t <= RMAX; ++t) {
                    if (t >= -r && t <= r) {
                        a0 = __fadd_rn(a0, v[RA + t]);
                        a1 = __fadd_rn(a1, s1[RA + t]);
                        a2 = __fadd_rn(a2, s2[RA + t]);
                        a3 = __fadd_rn(a3, s3[RA + t]);
                    }
                }
                o0[0] = a0; o1[0] = a1; o2[0] = a2; o3[0] = a3;
#pragma unroll
                for (int j = 1; j < 4; ++j) {
                    float n0, n1, n2, n3, d0, d1, d2, d3;
                    if constexpr (DYN) {
                        // runtime radius: select the entering / leaving columns
                        n0 = 0.f; n1 = 0.f; n2 = 0.f; n3 = 0.f; d0 = 0.f; d1 = 0.f; d2 = 0.f; d3 = 0.f;
#pragma unroll
                        for (int rr = 0; rr <= RMAX; ++rr) {
                            if (rr == r) {
                                n0 = v[RA + rr + j]; n1 = s1[RA + rr + j]; n2 = s2[RA + rr + j]; n3 = s3[RA + rr + j];
                                d0 = v[RA - rr + j - 1]; d1 = s1[RA - rr + j - 1]; d2 = s2[RA - rr + j - 1]; d3 = s3[RA - rr + j - 1];
                            }
                        }
                    } else {
                        const int tn = RA + RMAX + j, to = RA - RMAX + j - 1;
                        n0 = v[tn]; n1 = s1[tn]; n2 = s2[tn]; n3 = s3[tn];
                        d0 = v[to]; d1 = s1[to]; d2 = s2[to]; d3 = s3[to];
                    }
                    a0 = __fadd_rn(a0, __fsub_rn(n0, d0));
                    a1 = __fadd_rn(a1, __fsub_rn(n1, d1));
                    a2 = __fadd_rn(a2, __fsub_rn(n2, d2));
                    a3 = __fadd_rn(a3, __fsub_rn(n3, d3));
                    o0[j] = a0; o1[j] = a1; o2[j] = a2; o3[j] = a3;
                }
                float4* hp = reinterpret_cast<float4*>(sH + hy * TW + 4 * gi);
                hp[0] = make_float4(o0[0], o0[1], o0[2], o0[3]);
                hp[(HRM * TW) / 4] = make_float4(o1[0], o1[1], o1[2], o1[3]);
                hp[(2 * HRM * TW) / 4] = make_float4(o2[0], o2[1], o2[2], o2[3]);
                hp[(3 * HRM * TW) / 4] = make_float4(o3[0], o3[1], o3[2], o3[3]);
            }
            __syncthreads();
            // ---- C: vertical sums, NCC, top-k insertion
            {
                const float* h0 = sH + c;
                const float* h1 = sH + HRM * TW + c;
                const float* h2 = sH + 2 * HRM * TW + c;
                const float* h3 = sH + 3 * HRM * TW + c;
                const int y0 = seg * ROWS;
                float cv = 0.f, cj = 0.f, cjj = 0.f, cji = 0.f;
#pragma unroll
                for (int t = 0; t <= 2 * RMAX; ++t) {
                    if (t <= 2 * r) {
                        const int o = (y0 + t) * TW;
                        cv = __fadd_rn(cv, h0[o]);
                        cj = __fadd_rn(cj, h1[o]);
                        cjj = __fadd_rn(cjj, h2[o]);
                        cji = __fadd_rn(cji, h3[o]);
                    }
                }
#pragma unroll
                for (int j = 0; j < ROWS; ++j) {
                    if (j > 0) {
                        const int on = (y0 + j + 2 * r) * TW, oo = (y0 + j - 1) * TW;
                        cv = __fadd_rn(cv, __fsub_rn(h0[on], h0[oo]));
                        cj = __fadd_rn(cj, __fsub_rn(h1[on], h1[oo]));
                        cjj = __fadd_rn(cjj, __fsub_rn(h2[on], h2[oo]));
                        cji = __fadd_rn(cji, __fsub_rn(h3[on], h3[oo]));
                    }
                    float ncc;
                    if (cv * 10.f <= 9.f * k2) {
                        ncc = -1.f;
                    } else {
                        const float rc = (cv == k2) ? inv_k2 : __frcp_rn(cv);
                        const float mj = __fmul_rn(cj, rc), m2 = __fmul_rn(cjj, rc), mij = __fmul_rn(cji, rc);
                        const float var = __fsub_rn(m2, __fmul_rn(mj, mj));
                        const float rsdj = var > 1e-6f ? rsqrtf(var) : 1000.f;
                        ncc = __fmul_rn(__fsub_rn(mij, __fmul_rn(mu[j], mj)), __fmul_rn(rsd[j], rsdj));
                        ncc = ncc > 1.f ? 1.f : (ncc < -1.f ? -1.f : ncc);
                    }
                    total[j] = __fadd_rn(total[j], ncc);
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
        }
        // ---- winner-take-all update for hypothesis i
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            float s = 0.f;
#pragma unroll
            for (int q = 0; q < KMAX; ++q)
                if (q < nlist) s = __fadd_rn(s, topk[j][q]);
            if (bottom) s = __fsub_rn(total[j], s);
            s = __fdiv_rn(s, (float)kk);
            if (idx[j] == i - 1) snb[j] = s;
            if (s > best[j]) {
                best[j] = s;
                spb[j] = prv[j];
                snb[j] = -2.f;
                idx[j] = i;
            }
            prv[j] = s;
            if (i == pa) first[j] = s;
        }
    }

    // ---- write back: caller state (single chunk) or the chunk record
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int gy = ty + seg * ROWS + j;
        if (gx >= W || gy >= H) continue;
        const long long o = (long long)gy * W + gx;
        if (!to_rec) {
            p.best[o] = best[j];
            p.prev[o] = prv[j];
            p.spb[o] = spb[j];
            p.snb[o] = snb[j];
            p.idx[o] = idx[j];
        } else {
            const long long HW = (long long)H * W;
            const long long plane = (long long)p.nchunks * HW;
            float* rc = p.rec + (long long)chunk * HW + o;
            rc[0] = best[j];
            rc[plane] = __int_as_float(idx[j]);
            rc[2 * plane] = spb[j];
            rc[3 * plane] = snb[j];
            rc[4 * plane] = first[j];
            rc[5 * plane] = prv[j];
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
mvs_status validate_sweep(const mvs_sweep_args* a);
mvs_status fill_params(const mvs_sweep_args* a, SweepParams& p);
int pick_kmax(SweepParams& p);

}  // namespace mvs
