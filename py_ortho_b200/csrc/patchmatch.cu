// Red-black slanted-plane PatchMatch repair (reference: _dense.pm_refine, _dense.pyx:405-666).
//
// This file is compiled with -fmad=false: every float64 expression below is evaluated with one
// rounding per operation in the written order, which is how the reference's C (x86-64, no FMA)
// evaluates it. The float64 mode is bit-identical to the reference's pm_refine.
//
// Parallel schedule. The reference visits the pixels of one colour ((x + y) % 2) in raster order,
// but every pixel reads only its own plane, pixels of the other colour (all 8 neighbour offsets,
// (+-1, 0), (0, +-1), (+-5, 0), (0, +-5), have odd parity) and static inputs. So all pixels of a
// colour are independent: one thread (or lane group) per pixel per colour pass.
//
// Random trials. The reference draws from ONE xorshift32 stream (_rnd, _dense.pyx:559-563,
// started at seed | 1 per call, :606): 8 draws, in raster order, for every active pixel of the
// colour whose depth is finite once propagation is done (:646-652). Which pixels draw is known
// only after propagation, so a colour pass runs as
//   1. propagation (pm_kernel / pm_lane_kernel, PHASE 0): current plane + 8 neighbour planes;
//      the pixel's best cost, score and a flag "draws" go to per-pass scratch;
//   2. the exclusive prefix count of drawing pixels in raster order (pm_count_kernel,
//      pm_scan_kernel, pm_state_kernel): pixel p's first draw is stream element
//      base + 8 * prefix(p); xorshift32 is linear over GF(2), so its state there is
//      A^(8 prefix(p)) s_base with A the 32 x 32 step matrix, applied as a product of the
//      precomputed powers A^(8 * 2^j) (jump-ahead for F2-linear generators: Haramoto,
//      Matsumoto, Nishimura, Panneton, L'Ecuyer 2008); the pass advances the stream by 8 * total;
//   3. the two random trials (PHASE 1) from the pixel's own stream state.
// The stream state lives on the device from pass to pass (and, with mvs_pm_args.rng_state, from
// call to call), so no step waits for the host.
#include "common.cuh"

#include <algorithm>

namespace mvs {

struct PMParams {
    int H, W, S, r, step, top_k, it, colour;
    double cr0, cr1, cr2, geo_w, geo_tol, dmin, dmax, dd_scale, nn_scale;
    const float* ref;
    const float* ray;
    float* depth;
    float* normal;
    float* score;
    const unsigned char* active;
    unsigned long long* changed;
    double* cost_cache;                // per pixel; NaN = recompute (valid within one call)
    double* score_cache;
    // per colour pass, indexed by the pass's pixel number t = y * ceil(W / 2) + x / 2
    unsigned char* flags;              // bit 0: the pixel draws; bits 1-4: propagation changes
    double* pbest;                     // cost of the plane kept by propagation
    double* psc;                       // its photo score
    const unsigned* pstate;            // xorshift32 state before the pixel's first draw
    unsigned win_smem;                 // dynamic shared bytes of the lane kernel (bounds checks)
    const float* img[MVS_MAX_SOURCES];
    const float* dep[MVS_MAX_SOURCES];
    int iw[MVS_MAX_SOURCES], ih[MVS_MAX_SOURCES];
    int pinhole[MVS_MAX_SOURCES];       // k1 = k2 = k3 = 0
    double par[MVS_MAX_SOURCES * 18];
    double bsrc[MVS_MAX_SOURCES * 3];   // R_s (C_ref - C_s)
    // float32 lane kernel: per source its 2 x 2 bilinear footprints, quad[y w + x] =
    // (I(y, x), I(y, x + 1), I(y + 1, x), I(y + 1, x + 1)), one 16-byte load per sample
    const float4* quad[MVS_MAX_SOURCES];
};

// ---------------------------------------------------------------- the reference's stream

// _rnd (_dense.pyx:559-563): one xorshift32 step, then the low 24 bits as a uniform in [0, 1).
__host__ __device__ __forceinline__ unsigned xs_step(unsigned s) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
}
__device__ __forceinline__ double xs_draw(unsigned& s) {
    s = xs_step(s);
    return (double)(s & 0xFFFFFFu) / 16777216.0;
}

// A 32 x 32 matrix over GF(2) by columns: col[i] = M e_i, so M s = XOR of col[i] over set bits i.
struct Gf2 {
    unsigned col[32];
};
__host__ __device__ __forceinline__ unsigned gf2_apply(const Gf2& m, unsigned s) {
    unsigned r = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) r ^= m.col[i] & (0u - ((s >> i) & 1u));
    return r;
}

// Jump table of the stream: t[j] = A^(8 * 2^j), A = one xorshift32 step.
struct PMJump {
    Gf2 t[32];
};

// State after 8 k steps from s.
__device__ __forceinline__ unsigned jump8(const PMJump& J, unsigned s, unsigned k) {
    for (int j = 0; k != 0; ++j, k >>= 1)
        if (k & 1u) s = gf2_apply(J.t[j], s);
    return s;
}

// _proj (_dense.pyx:429-445): world point -> pixel and camera depth.
__device__ __forceinline__ bool pm_proj(const double* p, double X, double Y, double Z, double& u, double& v,
                                        double& z) {
    const double dx = X - p[9], dy = Y - p[10], dz = Z - p[11];
    const double xc = p[0] * dx + p[1] * dy + p[2] * dz;
    const double yc = p[3] * dx + p[4] * dy + p[5] * dz;
    const double zc = p[6] * dx + p[7] * dy + p[8] * dz;
    if (zc <= 1e-6) return false;
    const double nx = xc / zc, ny = yc / zc;
    const double r2 = nx * nx + ny * ny;
    const double dd = p[12] * (1.0 + r2 * (p[13] + r2 * (p[14] + r2 * p[15])));
    u = dd * nx + p[16];
    v = dd * ny + p[17];
    z = zc;
    return true;
}

// _bil (_dense.pyx:448-458); NaN outside [0, w-1.001] x [0, h-1.001] (also for NaN u, v, whose
// behaviour the reference leaves undefined).
__device__ __forceinline__ double pm_bil(const float* im, int w, int h, double u, double v) {
    if (!(u >= 0.0 && v >= 0.0 && u <= (double)w - 1.001 && v <= (double)h - 1.001)) return __longlong_as_double(0x7ff8000000000000LL);
    const int x0 = (int)u, y0 = (int)v;
    const double fx = u - (double)x0, fy = v - (double)y0;
    const long long o = (long long)y0 * w + x0;
    const double a00 = __ldg(im + o), a01 = __ldg(im + o + 1), a10 = __ldg(im + o + w), a11 = __ldg(im + o + w + 1);
    return (a00 * (1.0 - fx) + a01 * fx) * (1.0 - fy) + (a10 * (1.0 - fx) + a11 * fx) * fy;
}

// _pm_cost (_dense.pyx:461-556). Window samples are the outer loop as in the reference; the
// sources of a pass (PM_SRC_PASS at a time) are unrolled inside it with their five sums in
// registers, so each sample's world point (one division) is formed once per pass instead of once
// per source. Each source's work is branch-free (invalid samples read a safe address and add 0.0,
// which leaves a sum that started at +0.0 unchanged), so the sources' float64 dependency chains
// interleave. Every per-source sum still accumulates in window order: no result changes.
#ifndef PM_SRC_PASS
#define PM_SRC_PASS 2
#endif

// Geometric term of _pm_cost (_dense.pyx:532-555): mean over the sources with depth maps of
// min(1, |z - d_j| / d_j / geo_tol) at the rounded projection of the window centre.
__device__ __forceinline__ double pm_geo(const PMParams& c, double d, double rpx, double rpy, double rpz) {
    double geo = 0.0;
    if (c.geo_w > 0.0) {
        const double X = c.cr0 + d * rpx, Y = c.cr1 + d * rpy, Z = c.cr2 + d * rpz;
        int ng = 0;
        for (int s = 0; s < c.S; ++s) {
            if (c.dep[s] == nullptr) continue;
            ++ng;
            double e = 1.0, u, v, z;
            if (pm_proj(c.par + 18 * s, X, Y, Z, u, v, z)) {
                const int ui = (int)(u + 0.5), vv = (int)(v + 0.5);
                if (ui >= 0 && vv >= 0 && ui < c.iw[s] && vv < c.ih[s]) {
                    const double dj = __ldg(c.dep[s] + (long long)vv * c.iw[s] + ui);
                    if (isfinite(dj) && dj > 0.0) {
                        e = fabs(z - dj) / dj / c.geo_tol;
                        if (e > 1.0) e = 1.0;
                    }
                }
            }
            geo = geo + e;
        }
        if (ng) geo = geo / (double)ng;
    }
    return geo;
}

__device__ double pm_cost(const PMParams& c, int y, int x, double d, const double* n, double& ncc_out) {
    const int H = c.H, W = c.W;
    const long long HW = (long long)H * W, idx = (long long)y * W + x;
    const double rpx = __ldg(c.ray + idx), rpy = __ldg(c.ray + HW + idx), rpz = __ldg(c.ray + 2 * HW + idx);
    const double ndr = n[0] * rpx + n[1] * rpy + n[2] * rpz;
    if (ndr >= -1e-6 || d <= 0.0) {
        ncc_out = 0.0;   // unused by the caller for cost 10 (never accepted over a real cost)
        return 10.0;
    }
    const double num = d * ndr;
    double ncc[MVS_MAX_SOURCES];
    int nsamp = 0;
    for (int s0 = 0; s0 < c.S; s0 += PM_SRC_PASS) {
        double sI[PM_SRC_PASS], sJ[PM_SRC_PASS], sII[PM_SRC_PASS], sJJ[PM_SRC_PASS], sIJ[PM_SRC_PASS];
        int cnt[PM_SRC_PASS];
#pragma unroll
        for (int k = 0; k < PM_SRC_PASS; ++k) {
            sI[k] = 0.0; sJ[k] = 0.0; sII[k] = 0.0; sJJ[k] = 0.0; sIJ[k] = 0.0; cnt[k] = 0;
        }
        const int npass = min(PM_SRC_PASS, c.S - s0);
        int ns = 0;
        for (int a = -c.r; a <= c.r; a += c.step) {
            const int yy = y + a;
            if (yy < 0 || yy >= H) continue;
            for (int b = -c.r; b <= c.r; b += c.step) {
                const int xx = x + b;
                if (xx < 0 || xx >= W) continue;
                const long long q = (long long)yy * W + xx;
                const double I = __ldg(c.ref + q);
                if (!isfinite(I)) continue;
                const double qx = __ldg(c.ray + q), qy = __ldg(c.ray + HW + q), qz = __ldg(c.ray + 2 * HW + q);
                const double den = n[0] * qx + n[1] * qy + n[2] * qz;
                if (den >= -1e-9) continue;
                const double t = num / den;
                const double X = c.cr0 + t * qx, Y = c.cr1 + t * qy, Z = c.cr2 + t * qz;
                ++ns;
                const double II = I * I;
#pragma unroll
                for (int k = 0; k < PM_SRC_PASS; ++k) {
                    if (k < npass) {
                        const int s = s0 + k;
                        const double* p = c.par + 18 * s;
                        // _proj
                        const double dx = X - p[9], dy = Y - p[10], dz = Z - p[11];
                        const double xc = p[0] * dx + p[1] * dy + p[2] * dz;
                        const double yc = p[3] * dx + p[4] * dy + p[5] * dz;
                        const double zc = p[6] * dx + p[7] * dy + p[8] * dz;
                        const bool front = zc > 1e-6;
                        const double zq = front ? zc : 1.0;
                        const double nx = xc / zq, ny = yc / zq;
                        // pinhole source: the reference's factor f (1 + r2 (k1 + r2 (k2 + r2 k3)))
                        // evaluates to exactly f (r2 >= 0 finite, so every product with 0 is +0)
                        double dd = p[12];
                        if (!c.pinhole[s]) {
                            const double r2 = nx * nx + ny * ny;
                            dd = p[12] * (1.0 + r2 * (p[13] + r2 * (p[14] + r2 * p[15])));
                        }
                        const double u = dd * nx + p[16], v = dd * ny + p[17];
                        // _bil with its bounds (NaN u / v count as outside)
                        const int iw = c.iw[s], ih = c.ih[s];
                        const bool in = front && u >= 0.0 && v >= 0.0 && u <= (double)iw - 1.001 && v <= (double)ih - 1.001;
                        const double us = in ? u : 0.0, vs = in ? v : 0.0;
                        const int x0 = (int)us, y0 = (int)vs;
                        const double fx = us - (double)x0, fy = vs - (double)y0;
                        MVS_BOUND((long long)y0 * iw + x0 >= 0 && (long long)y0 * iw + x0 + iw + 1 < (long long)iw * ih);
                        const float* im = c.img[s] + ((long long)y0 * iw + x0);
                        const double a00 = __ldg(im), a01 = __ldg(im + 1), a10 = __ldg(im + iw), a11 = __ldg(im + iw + 1);
                        const double J = (a00 * (1.0 - fx) + a01 * fx) * (1.0 - fy) + (a10 * (1.0 - fx) + a11 * fx) * fy;
                        const bool ok = in && isfinite(J);
                        sI[k] += ok ? I : 0.0;
                        sJ[k] += ok ? J : 0.0;
                        sII[k] += ok ? II : 0.0;
                        sJJ[k] += ok ? J * J : 0.0;
                        sIJ[k] += ok ? I * J : 0.0;
                        cnt[k] += ok ? 1 : 0;
                    }
                }
            }
        }
        nsamp = ns;   // identical for every pass
#pragma unroll
        for (int k = 0; k < PM_SRC_PASS; ++k) {
            const int s = s0 + k;
            if (k < npass) {
                if (ns < 4 || (double)cnt[k] < 0.7 * (double)ns) {
                    ncc[s] = -1.0;
                } else {
                    const double dc = (double)cnt[k];
                    const double mi = sI[k] / dc, mj = sJ[k] / dc;
                    const double vi = sII[k] / dc - mi * mi;
                    const double vj = sJJ[k] / dc - mj * mj;
                    const double cv = sIJ[k] / dc - mi * mj;
                    ncc[s] = (vi < 1e-8 || vj < 1e-8) ? 0.0 : cv / sqrt(vi * vj);
                }
            }
        }
    }
    (void)nsamp;
    // descending insertion sort (S <= 16), then the mean of the first top_k
    for (int a = 1; a < c.S; ++a) {
        const double tmp = ncc[a];
        int b = a - 1;
        while (b >= 0 && ncc[b] < tmp) {
            ncc[b + 1] = ncc[b];
            --b;
        }
        ncc[b + 1] = tmp;
    }
    const int kk = c.top_k < c.S ? c.top_k : c.S;
    double photo = 0.0;
    for (int a = 0; a < kk; ++a) photo = photo + ncc[a];
    photo = photo / (double)kk;
    ncc_out = photo;
    return (1.0 - photo) + c.geo_w * pm_geo(c, d, rpx, rpy, rpz);
}

// 8 resident blocks of 128 threads per SM (64 registers): the float64 chains are latency-bound,
// so occupancy beats the spills (measured on B200, 2000 x 1500, 8 sources, 2 iterations: 2 sources
// per pass and 8 blocks 224 ms; 6 blocks 240 ms; 8 sources per pass at 168 registers 334 ms)
#ifndef PM_MIN_BLOCKS
#define PM_MIN_BLOCKS 8
#endif
// Pixel of pass number t (raster order of the colour's pixels): false past the image.
__device__ __forceinline__ bool pm_pixel(const PMParams& c, long long t, int& y, int& x) {
    const int half_w = (c.W + 1) / 2;
    if (t >= (long long)c.H * half_w) return false;
    y = (int)(t / half_w);
    x = 2 * (int)(t - (long long)y * half_w) + ((y + c.colour) & 1);
    return x < c.W;
}

// The two random trials of _dense.pyx:646-663 in the order of the reference: 4 draws per trial
// (depth, then the three normal components), all 8 drawn even when a trial is skipped.
template <typename CostFn>
__device__ __forceinline__ void pm_trials(const PMParams& c, unsigned st, float& dcur, float* ncur, double& best,
                                          double& sc, unsigned long long& changed, CostFn&& cost) {
    for (int tr = 0; tr < 2; ++tr) {
        const double u0 = xs_draw(st);
        const double u1 = xs_draw(st);
        const double u2 = xs_draw(st);
        const double u3 = xs_draw(st);
        const double dp = (double)dcur * (1.0 + c.dd_scale * (2.0 * u0 - 1.0));
        double nb[3];
        nb[0] = (double)ncur[0] + c.nn_scale * (2.0 * u1 - 1.0);
        nb[1] = (double)ncur[1] + c.nn_scale * (2.0 * u2 - 1.0);
        nb[2] = (double)ncur[2] + c.nn_scale * (2.0 * u3 - 1.0);
        const double nn = sqrt(nb[0] * nb[0] + nb[1] * nb[1] + nb[2] * nb[2]);
        if (nn < 1e-9 || dp < c.dmin || dp > c.dmax) continue;
        nb[0] = nb[0] / nn;
        nb[1] = nb[1] / nn;
        nb[2] = nb[2] / nn;
        double ph;
        const double cst = cost(dp, nb, ph);
        if (cst < best) {
            best = cst;
            sc = ph;
            dcur = (float)dp;
            ncur[0] = (float)nb[0];
            ncur[1] = (float)nb[1];
            ncur[2] = (float)nb[2];
            ++changed;
        }
    }
}

// End of a pixel's visit: score, cost cache, change count (depth / normal written by the caller).
__device__ __forceinline__ void pm_finish(const PMParams& c, long long idx, float dcur, double best, double sc,
                                          unsigned long long changed) {
    if (c.cost_cache) {
        const bool keep = changed == 0 && isfinite(dcur);
        c.cost_cache[idx] = keep ? best : __longlong_as_double(0x7ff8000000000000LL);
        if (keep) c.score_cache[idx] = sc;
    }
    c.score[idx] = (float)sc;
    if (changed && c.changed) atomicAdd(c.changed, changed);
}

// PHASE 0: current plane and propagation; PHASE 1: the random trials.
template <int PHASE>
__global__ void __launch_bounds__(128, PM_MIN_BLOCKS) pm_kernel(const __grid_constant__ PMParams c) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int y, x;
    const bool in = pm_pixel(c, t, y, x);
    const long long HW = (long long)c.H * c.W, idx = (long long)y * c.W + x;
    if (!in || !c.active[idx]) {
        if (PHASE == 0 && t < (long long)c.H * ((c.W + 1) / 2)) c.flags[t] = 0;
        return;
    }
    auto cost = [&](double d, const double* nb, double& ph) { return pm_cost(c, y, x, d, nb, ph); };
    float dcur = c.depth[idx];
    float ncur[3] = {c.normal[idx], c.normal[HW + idx], c.normal[2 * HW + idx]};
    double best, sc, ncc;
    unsigned long long changed = 0;
    if (PHASE == 1) {
        const unsigned f = c.flags[t];
        best = c.pbest[t];
        sc = c.psc[t];
        changed = f >> 1;
        if (f & 1u) {
            pm_trials(c, c.pstate[t], dcur, ncur, best, sc, changed, cost);
            c.depth[idx] = dcur;
            c.normal[idx] = ncur[0];
            c.normal[HW + idx] = ncur[1];
            c.normal[2 * HW + idx] = ncur[2];
        }
        pm_finish(c, idx, dcur, best, sc, changed);
        return;
    }
    const int H = c.H, W = c.W;
    const int offy[8] = {-1, 1, 0, 0, -5, 5, 0, 0};
    const int offx[8] = {0, 0, -1, 1, 0, 0, -5, 5};
    // cost of the pixel's current plane: reused from its previous visit when that visit kept the
    // plane it started with (the cost was then computed from these very float32 values)
    const double cached = c.cost_cache ? c.cost_cache[idx] : __longlong_as_double(0x7ff8000000000000LL);
    if (isfinite(dcur) && cached == cached) {
        best = cached;
        sc = c.score_cache[idx];
    } else if (isfinite(dcur)) {
        const double n[3] = {ncur[0], ncur[1], ncur[2]};
        best = pm_cost(c, y, x, (double)dcur, n, ncc);
        sc = ncc;
    } else {
        best = 1e9;
        sc = -1.0;
    }
    const double rx = __ldg(c.ray + idx), ry = __ldg(c.ray + HW + idx), rz = __ldg(c.ray + 2 * HW + idx);
    for (int k = 0; k < 8; ++k) {
        const int yn = y + offy[k], xn = x + offx[k];
        if (yn < 0 || xn < 0 || yn >= H || xn >= W) continue;
        const long long nidx = (long long)yn * W + xn;
        const float dnb = c.depth[nidx];
        if (!isfinite(dnb)) continue;
        const double nb[3] = {c.normal[nidx], c.normal[HW + nidx], c.normal[2 * HW + nidx]};
        const double dn = nb[0] * __ldg(c.ray + nidx) + nb[1] * __ldg(c.ray + HW + nidx) + nb[2] * __ldg(c.ray + 2 * HW + nidx);
        const double ndr = nb[0] * rx + nb[1] * ry + nb[2] * rz;
        if (ndr >= -1e-6) continue;
        const double dp = (double)dnb * dn / ndr;
        if (dp < c.dmin || dp > c.dmax) continue;
        const double cst = pm_cost(c, y, x, dp, nb, ncc);
        if (cst < best) {
            best = cst;
            sc = ncc;
            dcur = (float)dp;
            ncur[0] = (float)nb[0];
            ncur[1] = (float)nb[1];
            ncur[2] = (float)nb[2];
            ++changed;
        }
    }
    if (changed) {
        c.depth[idx] = dcur;
        c.normal[idx] = ncur[0];
        c.normal[HW + idx] = ncur[1];
        c.normal[2 * HW + idx] = ncur[2];
    }
    c.pbest[t] = best;
    c.psc[t] = sc;
    c.flags[t] = (unsigned char)((isfinite(dcur) ? 1u : 0u) | ((unsigned)changed << 1));
}

// ---------------------------------------------------------------- draw offsets of a colour pass

constexpr int PM_SCAN_BLOCK = 1024;

// Exclusive prefix sum over a block of PM_SCAN_BLOCK (32 warps) threads; `total` = the block's
// sum. Called once per kernel (its shared words are not reused).
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned& total) {
    __shared__ unsigned warp_off[32];
    __shared__ unsigned tot_s;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_off[w] = inc;
    __syncthreads();
    if (w == 0) {
        const unsigned wt = warp_off[lane];
        unsigned wi = wt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        warp_off[lane] = wi - wt;
        if (lane == 31) tot_s = wi;
    }
    __syncthreads();
    total = tot_s;
    return warp_off[w] + inc - v;
}

// Drawing pixels per block of PM_SCAN_BLOCK pass pixels.
__global__ void __launch_bounds__(PM_SCAN_BLOCK) pm_count_kernel(const unsigned char* flags, long long n,
                                                                  unsigned* bsum) {
    const long long t = (long long)blockIdx.x * PM_SCAN_BLOCK + threadIdx.x;
    const int f = t < n ? (flags[t] & 1) : 0;
    const int cnt = __syncthreads_count(f);
    if (threadIdx.x == 0) bsum[blockIdx.x] = (unsigned)cnt;
}

// One block: block counts -> exclusive block offsets (in place); the stream state after the
// pass's 8 * total draws goes to rng[nxt].
__global__ void __launch_bounds__(PM_SCAN_BLOCK) pm_scan_kernel(unsigned* bsum, int nb, unsigned* rng, int cur,
                                                                 int nxt, const __grid_constant__ PMJump J) {
    const int per = (nb + PM_SCAN_BLOCK - 1) / PM_SCAN_BLOCK;
    const int beg = min(nb, (int)threadIdx.x * per), end = min(nb, beg + per);
    unsigned s = 0;
    for (int i = beg; i < end; ++i) s += bsum[i];
    unsigned total = 0;
    unsigned run = block_exclusive_scan(s, total);
    for (int i = beg; i < end; ++i) {
        const unsigned v = bsum[i];
        bsum[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) rng[nxt] = jump8(J, rng[cur], total);
}

// Per drawing pixel: the stream state before its first draw (0 for pixels that do not draw; a
// xorshift32 state is never 0).
__global__ void __launch_bounds__(PM_SCAN_BLOCK) pm_state_kernel(const unsigned char* flags, long long n,
                                                                  const unsigned* boff, const unsigned* rng, int cur,
                                                                  const __grid_constant__ PMJump J, unsigned* pstate) {
    const long long t = (long long)blockIdx.x * PM_SCAN_BLOCK + threadIdx.x;
    const unsigned f = t < n ? (flags[t] & 1u) : 0u;
    unsigned total;
    const unsigned excl = block_exclusive_scan(f, total);
    __shared__ unsigned base;
    if (threadIdx.x == 0) base = jump8(J, rng[cur], boff[blockIdx.x]);
    __syncthreads();
    if (t < n) pstate[t] = f ? jump8(J, base, excl) : 0u;
}

__global__ void pm_rng_init_kernel(unsigned* rng, const unsigned* from, unsigned seed) {
    rng[0] = from ? *from : seed;
}

// The 2 x 2 bilinear footprints of a source image (PMParams::quad). The last row and column, which
// are never a footprint's top-left tap (every tap offset is clamped to (h - 2) w + w - 2), repeat
// the edge.
__global__ void __launch_bounds__(256) pm_quad_kernel(const float* __restrict__ im, int w, int h,
                                                      float4* __restrict__ quad) {
    const long long n = (long long)w * h;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / w), x = (int)(i - (long long)y * w);
        const long long r0 = (long long)y * w, r1 = (long long)min(y + 1, h - 1) * w;
        const int x1 = min(x + 1, w - 1);
        quad[i] = make_float4(__ldg(im + r0 + x), __ldg(im + r0 + x1), __ldg(im + r1 + x), __ldg(im + r1 + x1));
    }
}

// ---------------------------------------------------------------- float32 evaluation (MVS_PM_FP32)
//
// The same visits, candidates, draws and acceptance rule as pm_kernel, with the window costs
// evaluated in float32 and the work of one pixel spread over a group of L lanes, one per source:
//
//   * geometry: for a plane (d, n) and a pinhole source s, the camera point of window sample q is
//     M_s ray_q / (n . ray_q) with M_s = b_s n^T + d (n . ray_p) R_s and b_s = R_s (C_ref - C_s)
//     (the reference's ray-plane intersection followed by _proj, multiplied through by
//     n . ray_q). Per (candidate, source) M_s is composed in float64, folded with f, cx, cy and an
//     integer source anchor (U0, V0) at the window centre, and rounded once; per sample only
//     ray_q - ray_p enters, in float32, so source positions carry ~1e-6 px of rounding error;
//   * validity: when the four corners of the (clipped) window map inside the source with a 1 px
//     margin and in front of it, every sample does (a projective map keeps the window inside the
//     convex hull of its corner images) and the per-sample tests are skipped; otherwise each
//     sample is tested as in the reference (camera depth > 1e-6, 0 <= u <= w - 1.001, ...);
//   * sums: reference values are shifted by the window mean of the reference and source values
//     by the source's value at the window centre, so the float32 variance terms do not cancel;
//   * the lanes of a pixel sort their NCCs with a shuffle network (top-k mean) and sum the
//     geometric term; every lane follows the same candidate sequence and decision.
// Float32 costs differ from the float64 ones by ~1e-7 (measured 99.9th percentile 2e-6), so the
// strict '<' can decide near-ties differently; the float64 mode is the bit-exact reference.

// Resident blocks of 256 threads per SM for the lane kernel (propagation; trials). On B200, 2 iterations
// of a 2000 x 1500, 8-source case with one 16-byte footprint load per sample: 5 / 5 blocks (48
// registers, spills) 54.4 ms, 4 / 5 55.2 ms, 4 / 4 (64 registers) 55.5 ms, 4 / 3 57.4 ms, 3 / 4
// 58.6 ms. (With four scalar tap loads 4 blocks had been best: 58.7 ms against 61.7 ms at 3 and
// 64.5 ms at 5; rolling or partly unrolling a window row's samples was slower.)
#ifndef PM_LANE_MIN_BLOCKS
#define PM_LANE_MIN_BLOCKS 5
#endif
#ifndef PM_LANE_MIN_BLOCKS_TRIALS
#define PM_LANE_MIN_BLOCKS_TRIALS PM_LANE_MIN_BLOCKS
#endif
#ifndef PM_UNIT_INLINE
#define PM_UNIT_INLINE __forceinline__
#endif

__device__ __forceinline__ int pmf_floor(float x, float& f) {   // |x| < 2^22
    const float t = __fadd_rd(x, 12582912.0f);
    f = __fsub_rn(t, 12582912.0f);
    return __float_as_int(t) - 0x4B400000;
}

// The same floor, returning the raw bits of x + 1.5 * 2^23 (floor(x) + 0x4B400000).
__device__ __forceinline__ unsigned pmf_floor_bits(float x, float& f) {   // |x| < 2^22
    const float t = __fadd_rd(x, 12582912.0f);
    f = __fsub_rn(t, 12582912.0f);
    return (unsigned)__float_as_int(t);
}

// A pixel's window as the cost code reads it: sample (row, k) = e-th of the window as
// (ray_q - ray_p, I_q - mI) with I = NaN where there is no sample (outside the image or a
// non-finite reference value), and the ray offsets of the clipped window's four corners.
//   PMWinStaged: staged once per visit in shared memory by the pixel's lane group;
//   PMWinTile:   read from the warp's shared tile of raw rays and reference values (one lane per
//                pixel), the offsets formed on each read - the same float32 operations, so the
//                same values (positions outside the image hold masked samples either way).
struct PMWinStaged {
    const float4* w;      // NW samples, then the 4 corners
    __device__ __forceinline__ float4 at(int, int, int e) const { return w[e]; }
    __device__ __forceinline__ float4 corner(int k4, int nw) const { return w[nw + k4]; }
};
struct PMWinTile {
    const float4* t;      // tile entry of the window's first sample (row y - r, column x - r)
    int rs, cs;           // tile offsets of one window row and one window column
    int cy0, cy1, cx0, cx1;   // tile offsets of the clipped corners' rows and columns
    float rpx, rpy, rpz, mI;
    __device__ __forceinline__ float4 at(int row, int k, int) const {
        const float4 v = t[row * rs + k * cs];
        return make_float4(v.x - rpx, v.y - rpy, v.z - rpz, v.w - mI);
    }
    __device__ __forceinline__ float4 corner(int k4, int) const {
        const float4 v = t[(k4 < 2 ? cy0 : cy1) + ((k4 & 1) ? cx1 : cx0)];
        return make_float4(v.x - rpx, v.y - rpy, v.z - rpz, 0.f);
    }
};

// Window statistics of a pixel, fixed for one visit.
template <class Acc>
struct PMWinT {
    Acc acc;
    int side, nw;         // samples along a side, in the window
    float nfin;           // samples with a finite reference value inside the image
    float si, sii;        // sum of (I - mI) and (I - mI)^2 over those samples
    bool allfin;          // every sample has a finite reference value inside the image
};
using PMWin = PMWinT<PMWinStaged>;

// One source's window sums. CHECKED: every sample tested as in the reference (camera depth,
// source bounds, finite value) and the reference sums formed per source; otherwise (the whole
// window maps inside the source, no sample near a test) only the three source sums are formed.
// ALLFIN: no reference sample is missing (no masking of the reference terms).
template <int NSIDE, bool CHECKED, bool ALLFIN, class Acc>
__device__ __forceinline__ void pm_window_sums(const Acc& win, int side_rt, const float* A, const float* B,
                                               const float* C, float a0, float b0, float c0, float n0, float n1,
                                               float n2, float denp, float lou, float hiu, float lov, float hiv,
                                               unsigned kb, const float4* qd, int sw, unsigned last,
                                               float mJ,
                                               float& T1, float& T2, float& X, float& S1, float& S2, float& cnt,
                                               float& ns) {
    // rows rolled, the samples of a row unrolled when the side is known (the checked form, rare,
    // stays rolled to keep the instruction footprint small)
    const int side = NSIDE > 0 ? NSIDE : side_rt;
#pragma unroll 1
    for (int row = 0; row < side; ++row)
#pragma unroll((NSIDE > 0 && !CHECKED) ? NSIDE : 1)
    for (int k = 0; k < side; ++k) {
        const float4 w = win.at(row, k, row * side + k);
        const float cq = fmaf(C[0], w.x, fmaf(C[1], w.y, fmaf(C[2], w.z, c0)));
        const float aq = fmaf(A[0], w.x, fmaf(A[1], w.y, fmaf(A[2], w.z, a0)));
        const float bq = fmaf(B[0], w.x, fmaf(B[1], w.y, fmaf(B[2], w.z, b0)));
        const float rc = __fdividef(1.0f, cq);
        float ul = aq * rc, vl = bq * rc;
        bool ok = ALLFIN || w.w == w.w;
        if (CHECKED) {
            const float den = fmaf(n0, w.x, fmaf(n1, w.y, fmaf(n2, w.z, denp)));
            ok = ok && den < -1e-9f;                    // the reference skips den >= -1e-9
            ns += ok ? 1.f : 0.f;
            ok = ok && cq * __fdividef(1.0f, den) > 1e-6f && ul >= lou && ul <= hiu && vl >= lov && vl <= hiv;
            ul = ok ? ul : 0.f;
            vl = ok ? vl : 0.f;
        }
        float fu, fv;
        // top-left tap offset (floor(v) + V0) sw + floor(u) + U0 from the floor bits: one
        // multiply-add and one add of the unit's constant, wrapping exactly in 32 bits; the clamp
        // (an offset below 0 wraps above `last`) keeps every tap inside the image whatever the inputs
        const unsigned xb = pmf_floor_bits(ul, fu), yb = pmf_floor_bits(vl, fv);
        const unsigned o = min(yb * (unsigned)sw + xb + kb, last);
        MVS_BOUND(o <= last);
        const float fx = ul - fu, fy = vl - fv;
        const float4 q4 = __ldg(qd + o);
        const float t00 = q4.x, t01 = q4.y, t10 = q4.z, t11 = q4.w;
        const float top = fmaf(fx, t01 - t00, t00), bot = fmaf(fx, t11 - t10, t10);
        const float J = fmaf(fy, bot - top, top);
        if (CHECKED) ok = ok && fabsf(J) <= 3.4e38f;
        float Jp = J - mJ, Iv = w.w;
        if (CHECKED || !ALLFIN) {
            Jp = ok ? Jp : 0.f;
            Iv = ok ? Iv : 0.f;
        }
        T1 += Jp;
        T2 = fmaf(Jp, Jp, T2);
        X = fmaf(Iv, Jp, X);
        if (CHECKED) {
            S1 += Iv;
            S2 = fmaf(Iv, Iv, S2);
            cnt += ok ? 1.f : 0.f;
        }
    }
}

// float32 NCC of one (candidate, source) unit: plane (d, n) at the window's pixel, source s
// (s < S); n . ray_p = ndr < -1e-6. Follows _pm_cost: -1 below the count gate, 0 below the
// variance floor.
template <int NSIDE, class Acc>
__device__ PM_UNIT_INLINE float pm_unit_ncc(const PMParams& c, const PMWinT<Acc>& wn, float rpx, float rpy, float rpz,
                                            double d, const double* n, double ndr, int sl) {
    const double num = d * ndr;
    const float n0 = (float)n[0], n1 = (float)n[1], n2 = (float)n[2], denp = (float)ndr;
    const int NW = NSIDE > 0 ? NSIDE * NSIDE : wn.nw;
    const Acc& win = wn.acc;
    const int SIDE = NSIDE > 0 ? NSIDE : wn.side;
    // ---- per (candidate, source) local map. The camera point of sample q is M ray_q / (n.ray_q),
    // M = b n^T + num R. The window centre is formed in float64 (b (n.ray_p) + num R ray_p), the
    // rows of M (which only multiply ray_q - ray_p) in float32.
    const double* p = c.par + 18 * sl;
    const double* bs = c.bsrc + 3 * sl;
    const double rp[3] = {rpx, rpy, rpz};
    double cen[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double Rr = fma(p[3 * i], rp[0], fma(p[3 * i + 1], rp[1], p[3 * i + 2] * rp[2]));
        cen[i] = fma(bs[i], ndr, num * Rr);
    }
    const double xp = cen[0], yp = cen[1], zp = cen[2];
    const double f = p[12], pcx = p[16], pcy = p[17];
    // the centre's camera depth is zp / ndr: in front of the source needs zp < 0
    const bool front = zp < 0.0;
    const float ff = (float)f, rzf = front ? __fdividef(1.0f, (float)zp) : 0.f;
    const float ucf = fmaf(ff, (float)xp * rzf, (float)pcx), vcf = fmaf(ff, (float)yp * rzf, (float)pcy);
    const float Uf = fminf(fmaxf(floorf(ucf), -1048576.f), 1048576.f);
    const float Vf = fminf(fmaxf(floorf(vcf), -1048576.f), 1048576.f);
    const bool anchor = front && Uf == Uf && Vf == Vf;
    const double U0d = anchor ? (double)Uf : 0.0, V0d = anchor ? (double)Vf : 0.0;
    const double au = pcx - U0d, av = pcy - V0d;
    const float a0 = (float)fma(f, xp, au * zp), b0 = (float)fma(f, yp, av * zp), c0 = (float)zp;
    const float auf = (float)au, avf = (float)av, numf = (float)num;
    float A[3], B[3], C[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float nj = j == 0 ? n0 : (j == 1 ? n1 : n2);
        const float mx = fmaf((float)bs[0], nj, numf * (float)p[j]);
        const float my = fmaf((float)bs[1], nj, numf * (float)p[3 + j]);
        const float mz = fmaf((float)bs[2], nj, numf * (float)p[6 + j]);
        A[j] = fmaf(ff, mx, auf * mz);
        B[j] = fmaf(ff, my, avf * mz);
        C[j] = mz;
    }
    const int sw = c.iw[sl], sh = c.ih[sl];
    const float lou = (float)(-U0d), lov = (float)(-V0d);
    const float hiu = (float)(((double)sw - 1.001) - U0d), hiv = (float)(((double)sh - 1.001) - V0d);
    // integer tap position = floor bits + (U0 - magic): one add per coordinate
    const int ub = (int)U0d - 0x4B400000, vb = (int)V0d - 0x4B400000;
    const int last = sh * sw - sw - 2;                    // largest valid top-left tap offset
    // the window sums' tap offset: yb sw + xb + kb for floor bits xb, yb (unsigned, wrapping)
    const unsigned kb = (unsigned)vb * (unsigned)sw + (unsigned)ub;
    const float4* qd = c.quad[sl];
    // ---- corners: the whole window in front and inside (outside) the source
    bool den_ok = true, inside = anchor, front_all = true;
    int out_lo_u = 0, out_hi_u = 0, out_lo_v = 0, out_hi_v = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 w = win.corner(k, NW);
        const float den = fmaf(n0, w.x, fmaf(n1, w.y, fmaf(n2, w.z, denp)));
        const float cq = fmaf(C[0], w.x, fmaf(C[1], w.y, fmaf(C[2], w.z, c0)));
        const float aq = fmaf(A[0], w.x, fmaf(A[1], w.y, fmaf(A[2], w.z, a0)));
        const float bq = fmaf(B[0], w.x, fmaf(B[1], w.y, fmaf(B[2], w.z, b0)));
        const float rc = __fdividef(1.0f, cq);
        const float ul = aq * rc, vl = bq * rc;
        den_ok = den_ok && den < -1e-3f;
        front_all = front_all && cq < 1e-2f * den;
        inside = inside && ul >= lou + 1.f && ul <= hiu - 1.f && vl >= lov + 1.f && vl <= hiv - 1.f;
        out_lo_u += ul < lou - 1.f;
        out_hi_u += ul > hiu + 1.f;
        out_lo_v += vl < lov - 1.f;
        out_hi_v += vl > hiv + 1.f;
    }
    inside = inside && den_ok && front_all;
    const bool outside = den_ok && front_all && anchor &&
                         (out_lo_u == 4 || out_hi_u == 4 || out_lo_v == 4 || out_hi_v == 4);
    // ---- source shift: the source at the window centre (the anchor), else 0
    float mJ = 0.f;
    if (anchor && !outside) {
        const float ul = a0 / c0, vl = b0 / c0;
        if (ul >= lou && ul <= hiu && vl >= lov && vl <= hiv) {
            float fu, fv;
            const int xi = pmf_floor(ul, fu) + ub + 0x4B400000, yi = pmf_floor(vl, fv) + vb + 0x4B400000;
            const int o = min(max(yi * sw + xi, 0), last);
            const float fx = ul - fu, fy = vl - fv;
            const float4 q4 = __ldg(qd + o);
            const float t00 = q4.x, t01 = q4.y, t10 = q4.z, t11 = q4.w;
            const float top = fmaf(fx, t01 - t00, t00), bot = fmaf(fx, t11 - t10, t10);
            const float J = fmaf(fy, bot - top, top);
            if (fabsf(J) <= 3.4e38f) mJ = J;
        }
    }
    // ---- window sums
    float T1 = 0.f, T2 = 0.f, X = 0.f, S1 = 0.f, S2 = 0.f, cnt = 0.f, ns = 0.f;
    bool checked = !den_ok;                   // the count of samples needs the per-sample test
    if (!outside && inside) {
        if (wn.allfin) {
            pm_window_sums<NSIDE, false, true>(win, SIDE, A, B, C, a0, b0, c0, n0, n1, n2, denp, lou, hiu, lov, hiv,
                                               kb, qd, sw, (unsigned)last, mJ, T1, T2, X, S1, S2, cnt, ns);
        } else {
            pm_window_sums<NSIDE, false, false>(win, SIDE, A, B, C, a0, b0, c0, n0, n1, n2, denp, lou, hiu, lov, hiv,
                                                kb, qd, sw, (unsigned)last, mJ, T1, T2, X, S1, S2, cnt, ns);
        }
        // a non-finite source value in the window poisons the sums: redo the source checked
        if (fabsf(T2) <= 3.4e38f && fabsf(X) <= 3.4e38f) {
            S1 = wn.si; S2 = wn.sii; cnt = wn.nfin;
        } else {
            checked = true;
        }
    } else if (!outside) {
        checked = true;
    }
    if (checked) {
        T1 = T2 = X = S1 = S2 = cnt = ns = 0.f;
        pm_window_sums<NSIDE, true, false>(win, SIDE, A, B, C, a0, b0, c0, n0, n1, n2, denp, lou, hiu, lov, hiv,
                                           kb, qd, sw, (unsigned)last, mJ, T1, T2, X, S1, S2, cnt, ns);
    }
    // samples counted by the reference (finite reference value, n.ray_q < -1e-9): with every
    // corner's n.ray_q < -1e-3 that is every finite sample; otherwise each lane counted them
    if (den_ok) ns = wn.nfin;
    float ncc;
    {
        if (ns < 4.f || (double)cnt < 0.7 * (double)ns) {
            ncc = -1.f;
        } else {
            const float rc = 1.0f / cnt;
            const float mi = S1 * rc, mj = T1 * rc;
            const float vi = fmaf(-mi, mi, S2 * rc), vj = fmaf(-mj, mj, T2 * rc);
            const float cv = fmaf(-mi, mj, X * rc);
            ncc = (vi < 1e-8f || vj < 1e-8f) ? 0.f : cv * rsqrtf(vi * vj);
            if (!(fabsf(ncc) <= 3.4e38f)) ncc = 0.f;
        }
    }
    return ncc;
}

// float32 photo term (top-k mean NCC) of plane (d, n): the L lanes of a pixel group evaluate one
// source each and sort their NCCs with a shuffle network; every lane returns the same value.
template <int L, int NSIDE, class Acc>
__device__ float pm_photo_lane(const PMParams& c, const PMWinT<Acc>& wn, float rpx, float rpy, float rpz, double d,
                               const double* n, double ndr, int s, unsigned gmask) {
    float ncc = s < c.S ? pm_unit_ncc<NSIDE>(c, wn, rpx, rpy, rpz, d, n, ndr, s) : -INFINITY;   // idle lanes sort last
    // ---- descending bitonic sort over the group, then the mean of the first top_k
    const int lane = threadIdx.x & (L - 1);
#pragma unroll
    for (int k = 2; k <= L; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const float o = __shfl_xor_sync(gmask, ncc, j, L);
            const bool keep_max = ((lane & k) == 0) == ((lane & j) == 0);
            ncc = keep_max ? fmaxf(ncc, o) : fminf(ncc, o);
        }
    }
    const int kk = c.top_k < c.S ? c.top_k : c.S;
    float sum = lane < kk ? ncc : 0.f;
#pragma unroll
    for (int o = L >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(gmask, sum, o, L);
    return sum / (float)kk;
}

// float32 photo term of plane (d, n) evaluated by one lane over all sources (the propagation
// step gives each lane its own candidate); the top-k list is kept sorted in registers.
template <int NSIDE, int KM, class Acc>
__device__ __forceinline__ float pm_photo_cand_k(const PMParams& c, const PMWinT<Acc>& wn, float rpx, float rpy, float rpz,
                                                 double d, const double* n, double ndr) {
    const int kk = c.top_k < c.S ? c.top_k : c.S;
    float top[KM];
#pragma unroll
    for (int q = 0; q < KM; ++q) top[q] = -INFINITY;
#pragma unroll 1
    for (int s = 0; s < c.S; ++s) {
        float x = pm_unit_ncc<NSIDE>(c, wn, rpx, rpy, rpz, d, n, ndr, s);
#pragma unroll
        for (int q = 0; q < KM; ++q) {
            if (q < kk) {
                const float hi = fmaxf(top[q], x), lo = fminf(top[q], x);
                top[q] = hi;
                x = lo;
            }
        }
    }
    float sum = 0.f;
#pragma unroll
    for (int q = 0; q < KM; ++q) sum += q < kk ? top[q] : 0.f;
    return sum / (float)kk;
}

template <int NSIDE, class Acc>
__device__ __noinline__ float pm_photo_cand_wide(const PMParams& c, const PMWinT<Acc>& wn, float rpx, float rpy, float rpz,
                                                 double d, const double* n, double ndr) {
    return pm_photo_cand_k<NSIDE, MVS_MAX_SOURCES, Acc>(c, wn, rpx, rpy, rpz, d, n, ndr);
}

// top_k <= 2 (the reference's default) keeps a 2-entry list; wider lists take an out-of-line call
template <int NSIDE, class Acc>
__device__ __forceinline__ float pm_photo_cand(const PMParams& c, const PMWinT<Acc>& wn, float rpx, float rpy, float rpz,
                                               double d, const double* n, double ndr) {
    if (c.top_k <= 2) return pm_photo_cand_k<NSIDE, 2, Acc>(c, wn, rpx, rpy, rpz, d, n, ndr);
    return pm_photo_cand_wide<NSIDE, Acc>(c, wn, rpx, rpy, rpz, d, n, ndr);
}

// Geometric term over the group: lane s contributes source s's error (float64, as pm_geo).
template <int L>
__device__ __forceinline__ double pm_geo_lane(const PMParams& c, double d, double rpx, double rpy, double rpz, int s,
                                              unsigned gmask, int ng) {
    double e = 0.0;
    if (s < c.S && c.dep[s] != nullptr) {
        const double X = c.cr0 + d * rpx, Y = c.cr1 + d * rpy, Z = c.cr2 + d * rpz;
        double u, v, z;
        e = 1.0;
        if (pm_proj(c.par + 18 * s, X, Y, Z, u, v, z)) {
            const int ui = (int)(u + 0.5), vv = (int)(v + 0.5);
            if (ui >= 0 && vv >= 0 && ui < c.iw[s] && vv < c.ih[s]) {
                const double dj = __ldg(c.dep[s] + (long long)vv * c.iw[s] + ui);
                if (isfinite(dj) && dj > 0.0) {
                    e = fabs(z - dj) / dj / c.geo_tol;
                    if (e > 1.0) e = 1.0;
                }
            }
        }
    }
#pragma unroll
    for (int o = L >> 1; o > 0; o >>= 1) e += __shfl_xor_sync(gmask, e, o, L);
    return e / (double)ng;
}

// Samples along one side of the window: offsets -r, -r + step, ... <= r.
__host__ __device__ inline int pm_side(int r, int step) { return (2 * r) / step + 1; }

// PHASE 0: current plane and propagation; PHASE 1: the random trials.
template <int L, int NSIDE, int PHASE>
__global__ void __launch_bounds__(256, PHASE == 0 ? PM_LANE_MIN_BLOCKS : PM_LANE_MIN_BLOCKS_TRIALS)
    pm_lane_kernel(const __grid_constant__ PMParams c) {
    extern __shared__ float4 pm_win[];
    const int H = c.H, W = c.W;
    const int lane = threadIdx.x & (L - 1);
    const unsigned gmask = (L == 32 ? 0xffffffffu : ((1u << L) - 1u)) << (threadIdx.x & 31 & ~(L - 1));
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / L;
    int y, x;
    const bool in_img = pm_pixel(c, t, y, x);
    const long long HW = (long long)H * W, idx = (long long)y * W + x;
    if (!in_img || !c.active[idx]) {
        if (PHASE == 0 && lane == 0 && t < (long long)H * ((W + 1) / 2)) c.flags[t] = 0;
        return;
    }
    unsigned pflag = 0;
    if (PHASE == 1) {
        pflag = c.flags[t];
        if (!(pflag & 1u)) {           // no draws: the visit ends with propagation's result
            if (lane == 0) pm_finish(c, idx, c.depth[idx], c.pbest[t], c.psc[t], pflag >> 1);
            return;
        }
    }
    int ng = 0;
    for (int s = 0; s < c.S; ++s) ng += c.dep[s] != nullptr;
    const bool use_geo = c.geo_w > 0.0 && ng > 0;
    // ---- stage the window once per visit: ray offsets and reference values (NaN = no sample),
    // then the four corners of the clipped window; the window mean of the reference is the
    // shift of the float32 sums
    const int side = NSIDE > 0 ? NSIDE : pm_side(c.r, c.step);
    const int nw = side * side;
    float4* win = pm_win + (threadIdx.x / L) * (nw + 4);
    MVS_BOUND((threadIdx.x / L + 1) * (nw + 4) * sizeof(float4) <= c.win_smem);
    const float rpx = __ldg(c.ray + idx), rpy = __ldg(c.ray + HW + idx), rpz = __ldg(c.ray + 2 * HW + idx);
    PMWin wn;
    wn.acc.w = win;
    wn.side = side;
    wn.nw = nw;
    {
        float sum = 0.f, k = 0.f;
        for (int e = lane; e < nw + 4; e += L) {
            int yy, xx;
            if (e < nw) {
                yy = y - c.r + (e / side) * c.step;
                xx = x - c.r + (e % side) * c.step;
            } else {
                const int k4 = e - nw;
                yy = k4 < 2 ? max(y - c.r, 0) : min(y + c.r, H - 1);
                xx = (k4 & 1) ? min(x + c.r, W - 1) : max(x - c.r, 0);
            }
            float4 v = make_float4(0.f, 0.f, 0.f, __int_as_float(0x7fc00000));
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
                const long long q = (long long)yy * W + xx;
                v.x = __ldg(c.ray + q) - rpx;
                v.y = __ldg(c.ray + HW + q) - rpy;
                v.z = __ldg(c.ray + 2 * HW + q) - rpz;
                const float I = __ldg(c.ref + q);
                if (e < nw && fabsf(I) <= 3.4e38f) {
                    v.w = I;
                    sum += I;
                    k += 1.f;
                }
            }
            win[e] = v;
        }
#pragma unroll
        for (int o = L >> 1; o > 0; o >>= 1) {
            sum += __shfl_xor_sync(gmask, sum, o, L);
            k += __shfl_xor_sync(gmask, k, o, L);
        }
        // shift of the float32 sums: the window mean of the reference
        const float mI = k > 0.f ? sum / k : 0.f;
        float si = 0.f, sii = 0.f;
        for (int e = lane; e < nw; e += L) {
            const float I = win[e].w;
            if (I == I) {
                const float Ip = I - mI;
                win[e].w = Ip;
                si += Ip;
                sii = fmaf(Ip, Ip, sii);
            }
        }
#pragma unroll
        for (int o = L >> 1; o > 0; o >>= 1) {
            si += __shfl_xor_sync(gmask, si, o, L);
            sii += __shfl_xor_sync(gmask, sii, o, L);
        }
        wn.nfin = k;
        wn.si = si;
        wn.sii = sii;
        wn.allfin = k == (float)nw;
        __syncwarp(gmask);
    }
    const double rx = rpx, ry = rpy, rz = rpz;
    // cost of a candidate: _pm_cost's 10 for an invalid plane, else (1 - photo) + geo_w * geo
    auto cost = [&](double d, const double* nb, double& photo) -> double {
        const double ndr = nb[0] * rx + nb[1] * ry + nb[2] * rz;
        if (ndr >= -1e-6 || d <= 0.0) {
            photo = 0.0;
            return 10.0;
        }
        photo = (double)pm_photo_lane<L, NSIDE>(c, wn, rpx, rpy, rpz, d, nb, ndr, lane, gmask);
        const double geo = use_geo ? pm_geo_lane<L>(c, d, rx, ry, rz, lane, gmask, ng) : 0.0;
        return (1.0 - photo) + c.geo_w * geo;
    };
    float dcur = c.depth[idx];
    float ncur[3] = {c.normal[idx], c.normal[HW + idx], c.normal[2 * HW + idx]};
    double best, sc, ph;
    unsigned long long changed = 0;
    if (PHASE == 1) {
        best = c.pbest[t];
        sc = c.psc[t];
        changed = pflag >> 1;
        pm_trials(c, c.pstate[t], dcur, ncur, best, sc, changed, cost);
        if (lane != 0) return;
        c.depth[idx] = dcur;
        c.normal[idx] = ncur[0];
        c.normal[HW + idx] = ncur[1];
        c.normal[2 * HW + idx] = ncur[2];
        pm_finish(c, idx, dcur, best, sc, changed);
        return;
    }
    const int offy[8] = {-1, 1, 0, 0, -5, 5, 0, 0};
    const int offx[8] = {0, 0, -1, 1, 0, 0, -5, 5};
    const double cached = c.cost_cache ? c.cost_cache[idx] : __longlong_as_double(0x7ff8000000000000LL);
    if (isfinite(dcur) && cached == cached) {
        best = cached;
        sc = c.score_cache[idx];
    } else if (isfinite(dcur)) {
        const double n[3] = {ncur[0], ncur[1], ncur[2]};
        best = cost((double)dcur, n, ph);
        sc = ph;
    } else {
        best = 1e9;
        sc = -1.0;
    }
    // propagation: the neighbours' planes do not change during a colour pass, so the 8 candidate
    // costs are independent of one another. Lane k (mod L) evaluates candidate k over all sources;
    // then every lane takes the decisions in the reference's order from the shared results.
    auto cost_cand = [&](double d, const double* nb, double& photo) -> double {
        const double ndr = nb[0] * rx + nb[1] * ry + nb[2] * rz;
        if (ndr >= -1e-6 || d <= 0.0) {
            photo = 0.0;
            return 10.0;
        }
        photo = (double)pm_photo_cand<NSIDE>(c, wn, rpx, rpy, rpz, d, nb, ndr);
        const double geo = use_geo ? pm_geo(c, d, rx, ry, rz) : 0.0;
        return (1.0 - photo) + c.geo_w * geo;
    };
    constexpr int PR = (8 + L - 1) / L;          // candidates per lane
    double pcost[PR];
    float pphoto[PR], pd[PR], pn[PR][3];
    bool pok[PR];
#pragma unroll
    for (int r0 = 0; r0 < PR; ++r0) {
        const int k = r0 * L + lane;
        pok[r0] = false;
        pcost[r0] = 0.0;
        pphoto[r0] = pd[r0] = pn[r0][0] = pn[r0][1] = pn[r0][2] = 0.f;
        if (k >= 8) continue;
        const int yn = y + offy[k], xn = x + offx[k];
        if (yn < 0 || xn < 0 || yn >= H || xn >= W) continue;
        const long long nidx = (long long)yn * W + xn;
        const float dnb = c.depth[nidx];
        if (!isfinite(dnb)) continue;
        const double nb[3] = {c.normal[nidx], c.normal[HW + nidx], c.normal[2 * HW + nidx]};
        const double dn = nb[0] * __ldg(c.ray + nidx) + nb[1] * __ldg(c.ray + HW + nidx) + nb[2] * __ldg(c.ray + 2 * HW + nidx);
        const double ndr = nb[0] * rx + nb[1] * ry + nb[2] * rz;
        if (ndr >= -1e-6) continue;
        const double dp = (double)dnb * dn / ndr;
        if (dp < c.dmin || dp > c.dmax) continue;
        double phc;
        pcost[r0] = cost_cand(dp, nb, phc);
        pphoto[r0] = (float)phc;
        pd[r0] = (float)dp;
        pn[r0][0] = (float)nb[0]; pn[r0][1] = (float)nb[1]; pn[r0][2] = (float)nb[2];
        pok[r0] = true;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int from = k % L, r0 = k / L;
        const bool ok = __shfl_sync(gmask, (int)pok[r0], from, L) != 0;
        const double cst = __shfl_sync(gmask, pcost[r0], from, L);
        const float phk = __shfl_sync(gmask, pphoto[r0], from, L);
        const float dk = __shfl_sync(gmask, pd[r0], from, L);
        const float n0 = __shfl_sync(gmask, pn[r0][0], from, L);
        const float n1 = __shfl_sync(gmask, pn[r0][1], from, L);
        const float n2 = __shfl_sync(gmask, pn[r0][2], from, L);
        if (ok && cst < best) {
            best = cst;
            sc = phk;
            dcur = dk;
            ncur[0] = n0; ncur[1] = n1; ncur[2] = n2;
            ++changed;
        }
    }
    if (lane != 0) return;
    if (changed) {
        c.depth[idx] = dcur;
        c.normal[idx] = ncur[0];
        c.normal[HW + idx] = ncur[1];
        c.normal[2 * HW + idx] = ncur[2];
    }
    c.pbest[t] = best;
    c.psc[t] = sc;
    c.flags[t] = (unsigned char)((isfinite(dcur) ? 1u : 0u) | ((unsigned)changed << 1));
}

// ---------------------------------------------------------------- float32 trials, one lane per pixel
//
// In pm_lane_kernel the trials' lanes are the sources, and a pixel is seen by only some of them
// (5.1 of 8 on average in a 3 x 3 flight at 60-75 % overlap): the other lanes idle. Here a warp
// takes 32 consecutive pixels of one colour in one row and each lane evaluates its own pixel's
// two trials over all sources, as propagation evaluates its candidates; neighbouring pixels see
// the same sources, so the lanes skip the same ones together. The warp stages one tile of raw
// rays and reference values (rows y - r .. y + r, columns x_first - r .. x_last + r: 2r + 1 rows
// of 64 + 2r) in place of a window per pixel, and the window statistics are summed in the lane
// kernel's order (L strided partial sums, then its butterfly), so a trial's cost has the lane
// kernel's bits when top_k <= 2 and no source has a depth map (otherwise the top-k and geometric
// sums add the same terms in another order).
// Blocks of 4 warps; resident blocks per SM measured on B200 (2 iterations of a 2000 x 1500,
// 8-source case, the whole PatchMatch call): 3 (168 registers) 50.9 ms, 4 (128) 50.1 ms, 5 (96,
// spills) 53.0 ms, 6 (80) 52.6 ms, 8 (64) 57.6 ms; the lane groups' trials 54.0-54.4 ms.
constexpr int PM_TRIAL_WARPS = 4;   // warps per block
#ifndef PM_TRIAL_MIN_BLOCKS
#define PM_TRIAL_MIN_BLOCKS 4
#endif
#ifndef PM_TRIAL_LANE_GROUPS
#define PM_TRIAL_LANE_GROUPS 0      // 1: the trials on the lane groups' kernel (comparisons)
#endif

__host__ __device__ inline int pm_tile_pitch(int r) { return 64 + 2 * r; }
__host__ __device__ inline size_t pm_tile_entries(int r) { return (size_t)(2 * r + 1) * pm_tile_pitch(r); }

// Sums over the window's samples e = 0 .. nw - 1 as an L-lane group forms them: lane l adds
// e = l, l + L, ... in order, then the xor butterfly (every lane ends with the same value).
template <int L, class F>
__device__ __forceinline__ void pm_group_sums(int nw, F&& term, float& a, float& b) {
    float pa[L], pb[L];
#pragma unroll
    for (int l = 0; l < L; ++l) {
        pa[l] = 0.f;
        pb[l] = 0.f;
        for (int e = l; e < nw; e += L) term(e, pa[l], pb[l]);
    }
#pragma unroll
    for (int o = L >> 1; o > 0; o >>= 1)
#pragma unroll
        for (int l = 0; l < L; ++l)
            if (!(l & o)) {
                const float sa = pa[l] + pa[l | o], sb = pb[l] + pb[l | o];
                pa[l] = sa; pa[l | o] = sa;
                pb[l] = sb; pb[l | o] = sb;
            }
    a = pa[0];
    b = pb[0];
}

template <int L, int NSIDE>
__global__ void __launch_bounds__(32 * PM_TRIAL_WARPS, PM_TRIAL_MIN_BLOCKS)
    pm_trial_kernel(const __grid_constant__ PMParams c) {
    extern __shared__ float4 pm_tiles[];
    const int H = c.H, W = c.W, r = c.r, step = c.step;
    const int half_w = (W + 1) / 2, wpr = (half_w + 31) >> 5;            // warps per row
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * PM_TRIAL_WARPS + warp;
    if (gw >= (long long)H * wpr) return;                                 // the whole warp
    const int y = (int)(gw / wpr), k0 = (int)(gw - (long long)y * wpr) * 32;
    const int par = (y + c.colour) & 1;
    const int pitch = pm_tile_pitch(r), rows = 2 * r + 1;
    const int xs0 = 2 * k0 + par - r;                                     // image column of tile column 0
    float4* tile = pm_tiles + (size_t)warp * rows * pitch;
    MVS_BOUND((size_t)(warp + 1) * rows * pitch * sizeof(float4) <= c.win_smem);
    const long long HW = (long long)H * W;
    for (int e = lane; e < rows * pitch; e += 32) {
        const int ty = e / pitch, tx = e - ty * pitch;
        const int yy = y - r + ty, xx = xs0 + tx;
        float4 v = make_float4(0.f, 0.f, 0.f, __int_as_float(0x7fc00000));
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
            const long long q = (long long)yy * W + xx;
            v.x = __ldg(c.ray + q);
            v.y = __ldg(c.ray + HW + q);
            v.z = __ldg(c.ray + 2 * HW + q);
            const float I = __ldg(c.ref + q);
            if (fabsf(I) <= 3.4e38f) v.w = I;
        }
        tile[e] = v;
    }
    __syncwarp();
    const int k = k0 + lane, x = 2 * k + par;
    if (k >= half_w || x >= W) return;
    const long long t = (long long)y * half_w + k, idx = (long long)y * W + x;
    if (!c.active[idx]) return;
    const unsigned pflag = c.flags[t];
    if (!(pflag & 1u)) {               // no draws: the visit ends with propagation's result
        pm_finish(c, idx, c.depth[idx], c.pbest[t], c.psc[t], pflag >> 1);
        return;
    }
    int ng = 0;
    for (int s = 0; s < c.S; ++s) ng += c.dep[s] != nullptr;
    const bool use_geo = c.geo_w > 0.0 && ng > 0;
    const int side = NSIDE > 0 ? NSIDE : pm_side(r, step);
    const int nw = side * side;
    const float rpx = __ldg(c.ray + idx), rpy = __ldg(c.ray + HW + idx), rpz = __ldg(c.ray + 2 * HW + idx);
    // this pixel's window in the tile: sample (row, col) at w0[row * step * pitch + col * step]
    const float4* w0 = tile + 2 * lane;
    const int rs = step * pitch;
    float sum, kc, si, sii;
    pm_group_sums<L>(nw, [&](int e, float& a, float& b) {
        const int row = e / side, col = e - row * side;
        const float I = w0[row * rs + col * step].w;
        if (I == I) {
            a += I;
            b += 1.f;
        }
    }, sum, kc);
    const float mI = kc > 0.f ? sum / kc : 0.f;
    pm_group_sums<L>(nw, [&](int e, float& a, float& b) {
        const int row = e / side, col = e - row * side;
        const float I = w0[row * rs + col * step].w;
        if (I == I) {
            const float Ip = I - mI;
            a += Ip;
            b = fmaf(Ip, Ip, b);
        }
    }, si, sii);
    PMWinT<PMWinTile> wn;
    wn.acc.t = w0;
    wn.acc.rs = rs;
    wn.acc.cs = step;
    wn.acc.cy0 = (max(y - r, 0) - (y - r)) * pitch;
    wn.acc.cy1 = (min(y + r, H - 1) - (y - r)) * pitch;
    wn.acc.cx0 = max(x - r, 0) - (x - r);
    wn.acc.cx1 = min(x + r, W - 1) - (x - r);
    wn.acc.rpx = rpx;
    wn.acc.rpy = rpy;
    wn.acc.rpz = rpz;
    wn.acc.mI = mI;
    wn.side = side;
    wn.nw = nw;
    wn.nfin = kc;
    wn.si = si;
    wn.sii = sii;
    wn.allfin = kc == (float)nw;
    const double rx = rpx, ry = rpy, rz = rpz;
    auto cost = [&](double d, const double* nb, double& photo) -> double {
        const double ndr = nb[0] * rx + nb[1] * ry + nb[2] * rz;
        if (ndr >= -1e-6 || d <= 0.0) {
            photo = 0.0;
            return 10.0;
        }
        photo = (double)pm_photo_cand<NSIDE>(c, wn, rpx, rpy, rpz, d, nb, ndr);
        const double geo = use_geo ? pm_geo(c, d, rx, ry, rz) : 0.0;
        return (1.0 - photo) + c.geo_w * geo;
    };
    float dcur = c.depth[idx];
    float ncur[3] = {c.normal[idx], c.normal[HW + idx], c.normal[2 * HW + idx]};
    double best = c.pbest[t], sc = c.psc[t];
    unsigned long long changed = pflag >> 1;
    pm_trials(c, c.pstate[t], dcur, ncur, best, sc, changed, cost);
    c.depth[idx] = dcur;
    c.normal[idx] = ncur[0];
    c.normal[HW + idx] = ncur[1];
    c.normal[2 * HW + idx] = ncur[2];
    pm_finish(c, idx, dcur, best, sc, changed);
}

}  // namespace mvs

using namespace mvs;

namespace {

// Powers of the xorshift32 step matrix: P[j] = A^(2^j), j < 64 (A^(2^j) for the stream jumps).
struct StreamTables {
    Gf2 P[64];
    PMJump J;   // J.t[j] = A^(8 * 2^j) = P[j + 3]
};

Gf2 gf2_mul(const Gf2& a, const Gf2& b) {   // (a b) e_i = a (b e_i)
    Gf2 m;
    for (int i = 0; i < 32; ++i) m.col[i] = gf2_apply(a, b.col[i]);
    return m;
}

const StreamTables& stream_tables() {
    static const StreamTables T = [] {
        StreamTables t;
        for (int i = 0; i < 32; ++i) t.P[0].col[i] = xs_step(1u << i);   // the step is linear
        for (int j = 1; j < 64; ++j) t.P[j] = gf2_mul(t.P[j - 1], t.P[j - 1]);
        for (int j = 0; j < 32; ++j) t.J.t[j] = t.P[j + 3];
        return t;
    }();
    return T;
}

}  // namespace

extern "C" uint32_t mvs_pm_stream_advance(uint32_t state, uint64_t n) {
    const StreamTables& T = stream_tables();
    for (int j = 0; n != 0; ++j, n >>= 1)
        if (n & 1u) state = gf2_apply(T.P[j], state);
    return state;
}

extern "C" mvs_status mvs_pm_refine(const mvs_pm_args* a, void* stream) {
    clear_error();
    if (!a) return fail(MVS_ERR_VALUE, "pm_refine: null arguments");
    if (a->S == 0 || a->S > MVS_MAX_SOURCES) return MVS_OK;   // the reference returns 0 here
    if (a->S < 0) return fail(MVS_ERR_VALUE, "pm_refine: negative source count");
    if (a->H < 0 || a->W < 0) return fail(MVS_ERR_VALUE, "pm_refine: negative shape");
    if (a->r < 0 || a->step < 1) return fail(MVS_ERR_VALUE, "pm_refine: needs r >= 0 and step >= 1");
    if (a->top_k < 1) return fail(MVS_ERR_VALUE, "pm_refine: top_k must be >= 1");
    if (a->H == 0 || a->W == 0 || a->iters <= 0) return MVS_OK;
    if (!a->ref || !a->ray || !a->Cr || !a->par || !a->depth || !a->normal || !a->score || !a->active)
        return fail(MVS_ERR_VALUE, "pm_refine: null pointer");
    if ((long long)a->H * ((a->W + 1) / 2) >= (1LL << 31))
        return fail(MVS_ERR_VALUE, "pm_refine: image of %d x %d pixels is too large", a->W, a->H);
    PMParams p;
    memset(&p, 0, sizeof(p));
    p.H = a->H; p.W = a->W; p.S = a->S; p.r = a->r; p.step = a->step; p.top_k = a->top_k;
    p.cr0 = a->Cr[0]; p.cr1 = a->Cr[1]; p.cr2 = a->Cr[2];
    p.geo_w = a->geo_w; p.geo_tol = a->geo_tol; p.dmin = a->dmin; p.dmax = a->dmax;
    p.ref = a->ref; p.ray = a->ray; p.depth = a->depth; p.normal = a->normal; p.score = a->score;
    p.active = a->active;
    p.changed = reinterpret_cast<unsigned long long*>(a->changed);
    for (int s = 0; s < a->S; ++s) {
        if (!a->src[s]) return fail(MVS_ERR_VALUE, "pm_refine: null source %d", s);
        if (a->src_h[s] < 2 || a->src_w[s] < 2) return fail(MVS_ERR_VALUE, "pm_refine: source %d smaller than 2x2", s);
        p.img[s] = a->src[s];
        p.dep[s] = a->src_depth[s];
        p.iw[s] = a->src_w[s];
        p.ih[s] = a->src_h[s];
        for (int k = 0; k < 18; ++k) p.par[18 * s + k] = a->par[18 * s + k];
        p.pinhole[s] = a->par[18 * s + 13] == 0.0 && a->par[18 * s + 14] == 0.0 && a->par[18 * s + 15] == 0.0;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long HW = (long long)a->H * a->W;
    if (a->precision != MVS_PM_FP64 && a->precision != MVS_PM_FP32)
        return fail(MVS_ERR_VALUE, "pm_refine: unknown precision %d", a->precision);
    // float32 evaluation needs pinhole sources (the local map is a homography)
    bool fast = a->precision == MVS_PM_FP32;
    for (int s = 0; s < a->S && fast; ++s) fast = p.pinhole[s] != 0;
    if (fast) {
        for (int s = 0; s < a->S; ++s) {
            const double* q = a->par + 18 * s;
            // b_s = R_s (C_ref - C_s)
            const double e0 = a->Cr[0] - q[9], e1 = a->Cr[1] - q[10], e2 = a->Cr[2] - q[11];
            for (int i = 0; i < 3; ++i) p.bsrc[3 * s + i] = q[3 * i] * e0 + q[3 * i + 1] * e1 + q[3 * i + 2] * e2;
        }
    }
    // scratch, one stream-ordered allocation: per pass pixel the propagation result, its flag and
    // stream state; per scan block a count; the stream state (two words, alternating passes);
    // from the second iteration on, the per-pixel cost cache
    const long long n = (long long)a->H * ((a->W + 1) / 2);
    const int nb = (int)((n + PM_SCAN_BLOCK - 1) / PM_SCAN_BLOCK);
    const bool use_cache = a->iters > 1;
    auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t o_best = 0, o_sc = o_best + up(n * 8), o_state = o_sc + up(n * 8), o_flags = o_state + up(n * 4);
    const size_t o_bsum = o_flags + up(n), o_rng = o_bsum + up((size_t)nb * 4), o_cache = o_rng + 256;
    const size_t o_quad = o_cache + up(use_cache ? (size_t)HW * 2 * sizeof(double) : 0);
    size_t quad_bytes = 0;
    if (fast)
        for (int s = 0; s < a->S; ++s) quad_bytes += up((size_t)a->src_w[s] * a->src_h[s] * sizeof(float4));
    const size_t bytes = o_quad + quad_bytes;
    char* scratch = nullptr;
    MVS_CUDA(cudaMallocAsync((void**)&scratch, bytes, st), "pm_refine: scratch");
    p.pbest = reinterpret_cast<double*>(scratch + o_best);
    p.psc = reinterpret_cast<double*>(scratch + o_sc);
    unsigned* pstate = reinterpret_cast<unsigned*>(scratch + o_state);
    p.pstate = pstate;
    p.flags = reinterpret_cast<unsigned char*>(scratch + o_flags);
    unsigned* bsum = reinterpret_cast<unsigned*>(scratch + o_bsum);
    unsigned* rng = reinterpret_cast<unsigned*>(scratch + o_rng);
    if (use_cache) {
        p.cost_cache = reinterpret_cast<double*>(scratch + o_cache);
        p.score_cache = p.cost_cache + HW;
        cudaMemsetAsync(p.cost_cache, 0xFF, (size_t)HW * sizeof(double), st);   // all-ones = NaN: recompute
    }
    if (fast) {
        size_t off = o_quad;
        for (int s = 0; s < a->S; ++s) {
            float4* q = reinterpret_cast<float4*>(scratch + off);
            p.quad[s] = q;
            off += up((size_t)a->src_w[s] * a->src_h[s] * sizeof(float4));
            const long long ns = (long long)a->src_w[s] * a->src_h[s];
            const int qb = (int)std::min<long long>((ns + 255) / 256, 148LL * 8);
            pm_quad_kernel<<<qb, 256, 0, st>>>(a->src[s], a->src_w[s], a->src_h[s], q);
        }
    }
    const PMJump& J = stream_tables().J;
    // float32 lanes: one per source; a block holds as many pixel groups as its staged windows fit
    const int lanes = a->S <= 4 ? 4 : (a->S <= 8 ? 8 : 16);
    const int side = pm_side(a->r, a->step);
    const size_t win_bytes = (size_t)(side * side + 4) * sizeof(float4);
    int groups = 256 / lanes;
    while (groups > 1 && (size_t)groups * win_bytes > 96 * 1024) groups >>= 1;
    const int block = fast ? groups * lanes : 128;
    const size_t smem = fast ? (size_t)groups * win_bytes : 0;
    p.win_smem = (unsigned)smem;
    void (*lane_kernel[2])(PMParams) = {nullptr, nullptr};
    mvs_status status = MVS_OK;
    if (fast) {
#define PM_PICK(LN, PH)                                                                           \
    lane_kernel[PH] = side == 7 ? pm_lane_kernel<LN, 7, PH> : side == 5 ? pm_lane_kernel<LN, 5, PH> \
                                                            : pm_lane_kernel<LN, 0, PH>;
        if (lanes == 4) { PM_PICK(4, 0) PM_PICK(4, 1) }
        else if (lanes == 8) { PM_PICK(8, 0) PM_PICK(8, 1) }
        else { PM_PICK(16, 0) PM_PICK(16, 1) }
#undef PM_PICK
        for (int ph = 0; ph < 2 && status == MVS_OK; ++ph) {
            if (cudaFuncSetAttribute(lane_kernel[ph], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
                status = fail(MVS_ERR_CUDA, "pm_refine: shared-memory carve-out");
        }
    }
    // the trials: one lane per pixel (pm_trial_kernel) when the warps' tiles fit in shared memory,
    // else the lane groups' kernel
    void (*trial_kernel)(PMParams) = nullptr;
    const size_t smem_trial = (size_t)PM_TRIAL_WARPS * pm_tile_entries(a->r) * sizeof(float4);
    const int wpr = (int)(((a->W + 1) / 2 + 31) / 32);
    const unsigned grid_trial = (unsigned)(((long long)a->H * wpr + PM_TRIAL_WARPS - 1) / PM_TRIAL_WARPS);
#if !PM_TRIAL_LANE_GROUPS
    if (fast && status == MVS_OK && smem_trial <= 227 * 1024) {
#define PM_PICK_TRIAL(LN)                                                                        \
    trial_kernel = side == 7 ? pm_trial_kernel<LN, 7> : side == 5 ? pm_trial_kernel<LN, 5> : pm_trial_kernel<LN, 0>;
        if (lanes == 4) { PM_PICK_TRIAL(4) }
        else if (lanes == 8) { PM_PICK_TRIAL(8) }
        else { PM_PICK_TRIAL(16) }
#undef PM_PICK_TRIAL
        if (cudaFuncSetAttribute(trial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_trial) !=
            cudaSuccess) {
            cudaGetLastError();
            trial_kernel = nullptr;
        }
    }
#endif
    const unsigned grid = fast ? (unsigned)((n * lanes + block - 1) / block) : (unsigned)((n + 127) / 128);
    if (status == MVS_OK) {
        pm_rng_init_kernel<<<1, 1, 0, st>>>(rng, a->rng_state, a->seed | 1u);
        status = check_launch("pm_refine: stream start");
    }
    int cur = 0;
    for (int it = 0; it < a->iters && status == MVS_OK; ++it) {
        const int git = a->it0 + it;
        p.it = git;
        p.dd_scale = 0.05 / (double)(git + 1);
        p.nn_scale = 0.3 / (double)(git + 1);
        for (int colour = 0; colour < 2 && status == MVS_OK; ++colour) {
            p.colour = colour;
            p.win_smem = (unsigned)smem;
            if (fast) lane_kernel[0]<<<grid, block, smem, st>>>(p);
            else pm_kernel<0><<<grid, 128, 0, st>>>(p);
            pm_count_kernel<<<nb, PM_SCAN_BLOCK, 0, st>>>(p.flags, n, bsum);
            pm_scan_kernel<<<1, PM_SCAN_BLOCK, 0, st>>>(bsum, nb, rng, cur, cur ^ 1, J);
            pm_state_kernel<<<nb, PM_SCAN_BLOCK, 0, st>>>(p.flags, n, bsum, rng, cur, J, pstate);
            if (trial_kernel) {
                p.win_smem = (unsigned)smem_trial;
                trial_kernel<<<grid_trial, 32 * PM_TRIAL_WARPS, smem_trial, st>>>(p);
            } else if (fast) {
                lane_kernel[1]<<<grid, block, smem, st>>>(p);
            }
            else pm_kernel<1><<<grid, 128, 0, st>>>(p);
            cur ^= 1;
            status = check_launch("pm_refine kernels");
        }
    }
    if (status == MVS_OK && a->rng_state) {
        if (cudaMemcpyAsync(a->rng_state, rng + cur, sizeof(unsigned), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            status = fail(MVS_ERR_CUDA, "pm_refine: stream state copy");
    }
    cudaFreeAsync(scratch, st);
    return status;
}

unsigned mvs::take_bound_violations_pm() { return take_bound_violations_here(); }
