// Red-black slanted-plane PatchMatch repair (reference: _dense.pm_refine, _dense.pyx:405-666).
//
// This file is compiled with -fmad=false: every float64 expression below is evaluated with one
// rounding per operation in the written order, which is how the reference's C (x86-64, no FMA)
// evaluates it. With the same random draws, results are bit-identical to a sequential CPU
// evaluation of the same algorithm.
//
// Parallel schedule. The reference visits the pixels of one colour ((x + y) % 2) in raster order,
// but every pixel reads only its own plane, pixels of the other colour (all 8 neighbour offsets,
// (+-1, 0), (0, +-1), (+-5, 0), (0, +-5), have odd parity) and static inputs. So all pixels of a
// colour are independent: one thread per pixel per colour pass, two passes per iteration.
// The only sequential dependence in the reference is its xorshift32 stream (_dense.pyx:559-563);
// here each draw comes from a counter-based hash of (seed, iteration, pixel, draw index).
#include "common.cuh"

namespace mvs {

struct PMParams {
    int H, W, S, r, step, top_k, it, colour;
    double cr0, cr1, cr2, geo_w, geo_tol, dmin, dmax, dd_scale, nn_scale;
    unsigned seed;
    const float* ref;
    const float* ray;
    float* depth;
    float* normal;
    float* score;
    const unsigned char* active;
    unsigned long long* changed;
    double* cost_cache;                // per pixel; NaN = recompute (valid within one call)
    double* score_cache;
    const float* img[MVS_MAX_SOURCES];
    const float* dep[MVS_MAX_SOURCES];
    int iw[MVS_MAX_SOURCES], ih[MVS_MAX_SOURCES];
    int pinhole[MVS_MAX_SOURCES];       // k1 = k2 = k3 = 0
    double par[MVS_MAX_SOURCES * 18];
};

__host__ __device__ inline unsigned long long mix64(unsigned long long x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBULL;
    x ^= x >> 31;
    return x;
}

// Uniform draw in [0, 1) with 24-bit resolution (the reference's _rnd resolution).
__host__ __device__ inline double pm_uniform(unsigned seed, int it, long long pixel, int draw) {
    unsigned long long x = mix64((unsigned long long)seed + 0x9E3779B97F4A7C15ULL);
    x = mix64(x ^ ((unsigned long long)(unsigned)it * 0xD1B54A32D192ED03ULL));
    x = mix64(x ^ ((unsigned long long)pixel * 0x8CB92BA72F3D8DD7ULL));
    x = mix64(x ^ (unsigned long long)(unsigned)draw);
    return (double)(unsigned)(x >> 40) / 16777216.0;
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
    return (1.0 - photo) + c.geo_w * geo;
}

// 8 resident blocks of 128 threads per SM (64 registers): the float64 chains are latency-bound,
// so occupancy beats the spills (measured on B200, 2000 x 1500, 8 sources, 2 iterations: 2 sources
// per pass and 8 blocks 224 ms; 6 blocks 240 ms; 8 sources per pass at 168 registers 334 ms)
#ifndef PM_MIN_BLOCKS
#define PM_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(128, PM_MIN_BLOCKS) pm_kernel(const __grid_constant__ PMParams c) {
    const int H = c.H, W = c.W;
    const int half_w = (W + 1) / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int y = (int)(t / half_w);
    if (y >= H) return;
    const int x = 2 * (int)(t - (long long)y * half_w) + ((y + c.colour) & 1);
    if (x >= W) return;
    const long long HW = (long long)H * W, idx = (long long)y * W + x;
    if (!c.active[idx]) return;
    const int offy[8] = {-1, 1, 0, 0, -5, 5, 0, 0};
    const int offx[8] = {0, 0, -1, 1, 0, 0, -5, 5};
    float dcur = c.depth[idx];
    float ncur[3] = {c.normal[idx], c.normal[HW + idx], c.normal[2 * HW + idx]};
    double n[3] = {ncur[0], ncur[1], ncur[2]};
    double best, sc, ncc;
    unsigned long long changed = 0;
    // cost of the pixel's current plane: reused from its previous visit when that visit kept the
    // plane it started with (the cost was then computed from these very float32 values)
    const double cached = c.cost_cache ? c.cost_cache[idx] : __longlong_as_double(0x7ff8000000000000LL);
    if (isfinite(dcur) && cached == cached) {
        best = cached;
        sc = c.score_cache[idx];
    } else if (isfinite(dcur)) {
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
    if (isfinite(dcur)) {
        for (int tr = 0; tr < 2; ++tr) {
            const double u0 = pm_uniform(c.seed, c.it, idx, 4 * tr + 0);
            const double u1 = pm_uniform(c.seed, c.it, idx, 4 * tr + 1);
            const double u2 = pm_uniform(c.seed, c.it, idx, 4 * tr + 2);
            const double u3 = pm_uniform(c.seed, c.it, idx, 4 * tr + 3);
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
    }
    if (c.cost_cache) {
        const bool keep = changed == 0 && isfinite(dcur);
        c.cost_cache[idx] = keep ? best : __longlong_as_double(0x7ff8000000000000LL);
        if (keep) c.score_cache[idx] = sc;
    }
    c.depth[idx] = dcur;
    c.normal[idx] = ncur[0];
    c.normal[HW + idx] = ncur[1];
    c.normal[2 * HW + idx] = ncur[2];
    c.score[idx] = (float)sc;
    if (changed && c.changed) atomicAdd(c.changed, changed);
}

}  // namespace mvs

using namespace mvs;

extern "C" double mvs_pm_uniform(uint32_t seed, int32_t it, int64_t pixel, int32_t draw) {
    return pm_uniform(seed, it, pixel, draw);
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
    PMParams p;
    memset(&p, 0, sizeof(p));
    p.H = a->H; p.W = a->W; p.S = a->S; p.r = a->r; p.step = a->step; p.top_k = a->top_k;
    p.cr0 = a->Cr[0]; p.cr1 = a->Cr[1]; p.cr2 = a->Cr[2];
    p.geo_w = a->geo_w; p.geo_tol = a->geo_tol; p.dmin = a->dmin; p.dmax = a->dmax;
    p.seed = a->seed | 1u;
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
    void* cache = nullptr;
    if (a->iters > 1) {   // the cache pays off from the second iteration on
        if (cudaMallocAsync(&cache, (size_t)HW * 2 * sizeof(double), st) == cudaSuccess) {
            cudaMemsetAsync(cache, 0xFF, (size_t)HW * sizeof(double), st);   // all-ones = NaN: recompute
            p.cost_cache = reinterpret_cast<double*>(cache);
            p.score_cache = p.cost_cache + HW;
        } else {
            cudaGetLastError();   // no cache: every visit recomputes (same results)
        }
    }
    const long long nthreads = (long long)a->H * ((a->W + 1) / 2);
    const unsigned grid = (unsigned)((nthreads + 127) / 128);
    for (int it = 0; it < a->iters; ++it) {
        const int git = a->it0 + it;
        p.it = git;
        p.dd_scale = 0.05 / (double)(git + 1);
        p.nn_scale = 0.3 / (double)(git + 1);
        for (int colour = 0; colour < 2; ++colour) {
            p.colour = colour;
            pm_kernel<<<grid, 128, 0, st>>>(p);
            mvs_status ks = check_launch("pm_refine kernel");
            if (ks != MVS_OK) {
                if (cache) cudaFreeAsync(cache, st);
                return ks;
            }
        }
    }
    if (cache) cudaFreeAsync(cache, st);
    return MVS_OK;
}
