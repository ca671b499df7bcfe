/*
 * CPU oracle for the depth-map path - TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs
 * as the checker. It is never part of the product: libmvs_b200 does not link, load or call it.
 *
 * A plain-C restatement of the reference algorithm (pyOrthomosaic 0.9.3), written from its
 * definitional kernels and with the same float32 / float64 rounding points, so that on the same
 * inputs it reproduces the reference bit for bit (pinned by tests/test_oracle.py against the
 * reference itself, compiled into oracle/_ref, and against tests/golden/ fixtures):
 *   oracle_ncc_warp         <- _dense.ncc_warp          (_dense.pyx:13-110)
 *   oracle_combine          <- _dense.combine           (_dense.pyx:113-144)
 *   oracle_box_zero_mean    <- _fast.box_zero_mean      (_fast.pyx:661-713)
 *   oracle_pm_refine        <- _dense.pm_refine         (_dense.pyx:405-666), with the
 *                              reference's sequential xorshift32 draws (_rnd, :559-563)
 *   oracle_consistency      <- densify._consistency     (densify.py:441-478; _fast.pyx:201-268)
 *   oracle_init_normals     <- densify._init_normals    (densify.py:481-496)
 *   oracle_fuse_view        <- one reference image of densify._fuse_loop (densify.py:688-762;
 *                              _fast.ref_points / neighbour_sample / agreement / accumulate,
 *                              _fast.pyx:201-284)
 * plus an all-float64 variant of the sweep (oracle_sweep_fp64) used as the precision reference:
 * every sum, NCC, score and the parabola in double, no float32 rounding anywhere.
 *
 * Build: oracle/Makefile (gcc -ffp-contract=off: one rounding per written operation).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ ncc_warp (_dense.pyx:13-110) */
EXPORT int oracle_ncc_warp(int H, int W, const float* ref, const float* mu_i, const float* sd_i,
                           const float* src, int h, int w, const float* ray, const double* Rs, const double* b,
                           double f, double k1, double k2, double k3, double cx, double cy, const float* inv,
                           int r, float* out, float* J, float* V, float* hs)
{
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    const int k = 2 * r + 1;
    const double kk = 1.0 / (k * k);
    double* cs;
    int y, x;
    /* 1. warp */
    for (y = 0; y < H; y++) {
        for (x = 0; x < W; x++) {
            const ptrdiff_t o = (ptrdiff_t)y * W + x;
            double d = 1.0 / inv[o];
            double rx = ray[o], ry = ray[HW + o], rz = ray[2 * HW + o];
            double X = b[0] + d * ((Rs[0] * rx + Rs[1] * ry) + Rs[2] * rz);
            double Y = b[1] + d * ((Rs[3] * rx + Rs[4] * ry) + Rs[5] * rz);
            double Z = b[2] + d * ((Rs[6] * rx + Rs[7] * ry) + Rs[8] * rz);
            double nx, ny, r2, dd, u, v, fx, fy, a00, a01, a10, a11, val;
            ptrdiff_t x0, y0;
            J[o] = 0;
            V[o] = 0;
            if (Z <= 1e-6) continue;
            nx = X / Z;
            ny = Y / Z;
            r2 = nx * nx + ny * ny;
            dd = f * (1 + r2 * (k1 + r2 * (k2 + r2 * k3)));
            u = dd * nx + cx;
            v = dd * ny + cy;
            if (u < 0 || v < 0 || u > w - 1.001 || v > h - 1.001) continue;
            x0 = (ptrdiff_t)u;
            y0 = (ptrdiff_t)v;
            fx = u - x0;
            fy = v - y0;
            a00 = src[y0 * w + x0];
            a01 = src[y0 * w + x0 + 1];
            a10 = src[(y0 + 1) * w + x0];
            a11 = src[(y0 + 1) * w + x0 + 1];
            val = (a00 * (1 - fx) + a01 * fx) * (1 - fy) + (a10 * (1 - fx) + a11 * fx) * fy;
            if (isfinite(val)) {
                J[o] = (float)val;
                V[o] = 1;
            }
        }
    }
    /* 2. horizontal running sums (float products, double accumulators, float rows) */
    for (y = 0; y < H; y++) {
        const float* Jr = J + (ptrdiff_t)y * W;
        const float* Vr = V + (ptrdiff_t)y * W;
        const float* Ir = ref + (ptrdiff_t)y * W;
        double sv = 0, sj = 0, sjj = 0, sij = 0;
        for (x = 0; x < (r < W ? r : W); x++) {
            sv += Vr[x];
            sj += Jr[x];
            sjj += (float)(Jr[x] * Jr[x]);
            sij += (float)(Jr[x] * Ir[x]);
        }
        for (x = 0; x < W; x++) {
            if (x + r < W) {
                sv += Vr[x + r];
                sj += Jr[x + r];
                sjj += (float)(Jr[x + r] * Jr[x + r]);
                sij += (float)(Jr[x + r] * Ir[x + r]);
            }
            if (x - r - 1 >= 0) {
                sv -= Vr[x - r - 1];
                sj -= Jr[x - r - 1];
                sjj -= (float)(Jr[x - r - 1] * Jr[x - r - 1]);
                sij -= (float)(Jr[x - r - 1] * Ir[x - r - 1]);
            }
            hs[(ptrdiff_t)y * W + x] = (float)sv;
            hs[HW + (ptrdiff_t)y * W + x] = (float)sj;
            hs[2 * HW + (ptrdiff_t)y * W + x] = (float)sjj;
            hs[3 * HW + (ptrdiff_t)y * W + x] = (float)sij;
        }
    }
    /* 3. vertical running sums (double) -> NCC */
    cs = (double*)calloc((size_t)4 * W, sizeof(double));
    if (!cs) return -1;
    for (y = 0; y < (r < H ? r : H); y++)
        for (x = 0; x < W; x++) {
            int q;
            for (q = 0; q < 4; q++) cs[q * W + x] += hs[q * HW + (ptrdiff_t)y * W + x];
        }
    for (y = 0; y < H; y++) {
        for (x = 0; x < W; x++) {
            int q;
            double cov, mj, m2, mij, sdj, ncc;
            if (y + r < H)
                for (q = 0; q < 4; q++) cs[q * W + x] += hs[q * HW + (ptrdiff_t)(y + r) * W + x];
            if (y - r - 1 >= 0)
                for (q = 0; q < 4; q++) cs[q * W + x] -= hs[q * HW + (ptrdiff_t)(y - r - 1) * W + x];
            cov = cs[x] * kk;
            if (cov <= 0.9) {
                out[(ptrdiff_t)y * W + x] = -1;
                continue;
            }
            mj = cs[W + x] * kk / cov;
            m2 = cs[2 * W + x] * kk / cov;
            mij = cs[3 * W + x] * kk / cov;
            sdj = m2 - mj * mj;
            sdj = sdj > 1e-6 ? sqrt(sdj) : 1e-3;
            ncc = (mij - mu_i[(ptrdiff_t)y * W + x] * mj) / (sd_i[(ptrdiff_t)y * W + x] * sdj);
            out[(ptrdiff_t)y * W + x] = (float)(ncc > 1 ? 1.0 : (ncc < -1 ? -1.0 : ncc));
        }
    }
    free(cs);
    return 0;
}

/* ------------------------------------------------------------------ combine (_dense.pyx:113-144) */
EXPORT void oracle_combine(int n, int H, int W, const float* S, int top_k, int i, float* best, float* prev,
                           float* s_prev_best, float* s_next_best, int* idx)
{
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    const int kk = top_k < n ? top_k : n;
    ptrdiff_t o;
    for (o = 0; o < HW; o++) {
        float buf[16], t, s;
        int a, c;
        for (a = 0; a < n; a++) buf[a] = S[a * HW + o];
        for (a = 1; a < n; a++) {
            t = buf[a];
            c = a - 1;
            while (c >= 0 && buf[c] < t) {
                buf[c + 1] = buf[c];
                c -= 1;
            }
            buf[c + 1] = t;
        }
        s = 0;
        for (a = 0; a < kk; a++) s += buf[a];
        s /= kk;
        if (idx[o] == i - 1) s_next_best[o] = s;
        if (s > best[o]) {
            best[o] = s;
            s_prev_best[o] = prev[o];
            s_next_best[o] = -2;
            idx[o] = i;
        }
        prev[o] = s;
    }
}

/* One hypothesis for all sources: ncc_warp per source, then combine (the unfused definition of
 * _dense.sweep_hypothesis). srcs: n pointers, geo: (n, 18) Rs(9) b(3) f k1 k2 k3 cx cy.
 * If S_out is non-NULL the per-source NCC (n, H, W) is copied there. */
EXPORT int oracle_sweep_hypothesis(int H, int W, const float* ref, const float* mu, const float* sd, int n,
                                   const float* const* srcs, const int* src_h, const int* src_w, const float* ray,
                                   const double* geo, const float* inv, int r, int top_k, int i, float* best,
                                   float* prev, float* s_prev_best, float* s_next_best, int* idx, float* S_out)
{
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    float* S = (float*)malloc(sizeof(float) * (size_t)(n * HW + 6 * HW));
    int s, rc = 0;
    if (!S) return -1;
    for (s = 0; s < n && rc == 0; s++) {
        const double* g = geo + 18 * s;
        rc = oracle_ncc_warp(H, W, ref, mu, sd, srcs[s], src_h[s], src_w[s], ray, g, g + 9, g[12], g[13], g[14],
                             g[15], g[16], g[17], inv, r, S + s * HW, S + n * HW, S + (n + 1) * HW, S + (n + 2) * HW);
    }
    if (rc == 0) {
        oracle_combine(n, H, W, S, top_k, i, best, prev, s_prev_best, s_next_best, idx);
        if (S_out) memcpy(S_out, S, sizeof(float) * (size_t)(n * HW));
    }
    free(S);
    return rc;
}

/* ------------------------------------------------------------------ all-float64 sweep */
/* The same sweep with no float32 rounding: warped values, window sums, NCC, top-k mean, winner
 * state and the parabola in double; depth = 1 / max(inv0 + (idx + off) dinv, 1e-9). inv maps are
 * given per hypothesis as double (n_hyp, H, W); ray and images as float inputs. Outputs: depth and
 * best score (double), idx. Direct window sums (no running add/subtract). */
EXPORT int oracle_sweep_fp64(int H, int W, const float* ref, const double* mu, const double* sd, int n,
                             const float* const* srcs, const int* src_h, const int* src_w, const double* ray,
                             const double* geo, const double* inv, int n_hyp, int r, int top_k, double* depth_out,
                             double* best_out, int* idx_out)
{
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    const int kk = top_k < n ? top_k : n;
    double *J = (double*)malloc(sizeof(double) * HW), *S = (double*)malloc(sizeof(double) * n * HW);
    unsigned char* V = (unsigned char*)malloc(HW);
    double *best = (double*)malloc(sizeof(double) * HW), *prev = (double*)malloc(sizeof(double) * HW);
    double *spb = (double*)malloc(sizeof(double) * HW), *snb = (double*)malloc(sizeof(double) * HW);
    int* idx = idx_out;
    int i, s, y, x;
    ptrdiff_t o;
    if (!J || !S || !V || !best || !prev || !spb || !snb) {
        free(J); free(S); free(V); free(best); free(prev); free(spb); free(snb);
        return -1;
    }
    for (o = 0; o < HW; o++) {
        best[o] = prev[o] = spb[o] = snb[o] = -2.0;
        idx[o] = -1;
    }
    for (i = 0; i < n_hyp; i++) {
        const double* iv = inv + (ptrdiff_t)i * HW;
        for (s = 0; s < n; s++) {
            const double* g = geo + 18 * s;
            const float* src = srcs[s];
            const int h = src_h[s], w = src_w[s];
            for (o = 0; o < HW; o++) {
                double d = 1.0 / iv[o], rx = ray[o], ry = ray[HW + o], rz = ray[2 * HW + o];
                double X = g[9] + d * (g[0] * rx + g[1] * ry + g[2] * rz);
                double Y = g[10] + d * (g[3] * rx + g[4] * ry + g[5] * rz);
                double Z = g[11] + d * (g[6] * rx + g[7] * ry + g[8] * rz);
                double nx, ny, r2, dd, u, v, fx, fy, val;
                ptrdiff_t x0, y0;
                V[o] = 0;
                J[o] = 0;
                if (!(Z > 1e-6)) continue;
                nx = X / Z;
                ny = Y / Z;
                r2 = nx * nx + ny * ny;
                dd = g[12] * (1 + r2 * (g[13] + r2 * (g[14] + r2 * g[15])));
                u = dd * nx + g[16];
                v = dd * ny + g[17];
                if (!(u >= 0 && v >= 0 && u <= w - 1.001 && v <= h - 1.001)) continue;
                x0 = (ptrdiff_t)u;
                y0 = (ptrdiff_t)v;
                fx = u - x0;
                fy = v - y0;
                val = ((double)src[y0 * w + x0] * (1 - fx) + (double)src[y0 * w + x0 + 1] * fx) * (1 - fy) +
                      ((double)src[(y0 + 1) * w + x0] * (1 - fx) + (double)src[(y0 + 1) * w + x0 + 1] * fx) * fy;
                if (isfinite(val)) {
                    J[o] = val;
                    V[o] = 1;
                }
            }
            for (y = 0; y < H; y++)
                for (x = 0; x < W; x++) {
                    double cnt = 0, sj = 0, sjj = 0, sij = 0, mj, m2, mij, var, sdj, ncc;
                    int a, b;
                    const int k = 2 * r + 1;
                    for (a = -r; a <= r; a++) {
                        const int yy = y + a;
                        if (yy < 0 || yy >= H) continue;
                        for (b = -r; b <= r; b++) {
                            const int xx = x + b;
                            const ptrdiff_t q = (ptrdiff_t)yy * W + xx;
                            if (xx < 0 || xx >= W || !V[q]) continue;
                            cnt += 1;
                            sj += J[q];
                            sjj += J[q] * J[q];
                            sij += J[q] * (double)ref[q];
                        }
                    }
                    o = (ptrdiff_t)y * W + x;
                    if (cnt / (k * k) <= 0.9) {
                        S[s * HW + o] = -1;
                        continue;
                    }
                    mj = sj / cnt;
                    m2 = sjj / cnt;
                    mij = sij / cnt;
                    var = m2 - mj * mj;
                    sdj = var > 1e-6 ? sqrt(var) : 1e-3;
                    ncc = (mij - mu[o] * mj) / (sd[o] * sdj);
                    S[s * HW + o] = ncc > 1 ? 1.0 : (ncc < -1 ? -1.0 : ncc);
                }
        }
        for (o = 0; o < HW; o++) {
            double buf[16], t, sc = 0;
            int a, c;
            for (a = 0; a < n; a++) buf[a] = S[a * HW + o];
            for (a = 1; a < n; a++) {
                t = buf[a];
                c = a - 1;
                while (c >= 0 && buf[c] < t) {
                    buf[c + 1] = buf[c];
                    c--;
                }
                buf[c + 1] = t;
            }
            for (a = 0; a < kk; a++) sc += buf[a];
            sc /= kk;
            if (idx[o] == i - 1) snb[o] = sc;
            if (sc > best[o]) {
                best[o] = sc;
                spb[o] = prev[o];
                snb[o] = -2;
                idx[o] = i;
            }
            prev[o] = sc;
        }
    }
    for (o = 0; o < HW; o++) {
        const double inv0 = inv[o], dinv = n_hyp > 1 ? inv[HW + o] - inv[o] : 0.0;
        const double den = spb[o] - 2 * best[o] + snb[o];
        const int in = idx[o] > 0 && idx[o] < n_hyp - 1 && den < -1e-6;
        double off = in ? 0.5 * (spb[o] - snb[o]) / den : 0.0, iv;
        off = off < -0.5 ? -0.5 : (off > 0.5 ? 0.5 : off);
        iv = inv0 + (idx[o] + off) * dinv;
        depth_out[o] = 1.0 / (iv > 1e-9 ? iv : 1e-9);
        best_out[o] = best[o];
    }
    free(J); free(S); free(V); free(best); free(prev); free(spb); free(snb);
    return 0;
}

/* ------------------------------------------------------------------ box_zero_mean (_fast.pyx:661-713) */
EXPORT int oracle_box_zero_mean(int H, int W, const float* a, int r, float* out)
{
    const int k = 2 * r + 1, PH = H + 2 * r + 1, PW = W + 2 * r + 1, R = k + 1;
    const float scale = (float)(1.0 / (k * k));
    float *col, *ring, *rowc;
    int i, x, y;
    if (H == 0 || W == 0) return 0;
    col = (float*)malloc(sizeof(float) * W);
    ring = (float*)malloc(sizeof(float) * (size_t)R * W);
    rowc = (float*)malloc(sizeof(float) * PW);
    if (!col || !ring || !rowc) {
        free(col); free(ring); free(rowc);
        return -1;
    }
    for (x = 0; x < W; x++) col[x] = 0;
    for (i = 0; i < PH; i++) {
        const int ay = i - (r + 1);
        float* cur = ring + (size_t)(i % R) * W;
        for (x = 0; x < W; x++) {
            const float v = (ay < 0 || ay >= H) ? 0.0f : a[(ptrdiff_t)ay * W + x];
            col[x] = (i == 0) ? v : col[x] + v;
            cur[x] = col[x];
        }
        y = i - k;
        if (y >= 0) {
            const float* old = ring + (size_t)(y % R) * W;
            for (x = 0; x < PW; x++) {
                const float t = (x < r + 1 || x >= r + 1 + W) ? 0.0f : cur[x - r - 1] - old[x - r - 1];
                rowc[x] = (x == 0) ? t : rowc[x - 1] + t;
            }
            for (x = 0; x < W; x++) out[(ptrdiff_t)y * W + x] = (rowc[x + k] - rowc[x]) * scale;
        }
    }
    free(col); free(ring); free(rowc);
    return 0;
}

/* ------------------------------------------------------------------ PatchMatch (_dense.pyx:405-666) */
typedef struct {
    const float* ref;
    int H, W;
    const float* ray;
    double cr0, cr1, cr2;
    int S;
    const float* const* img;
    const float* const* dep;
    const int* iw;
    const int* ih;
    const double* par;
    int r, step, top_k;
    double geo_w, geo_tol;
} pm_ctx;

static int pm_proj(const double* p, double X, double Y, double Z, double* u, double* v, double* z)
{
    double dx = X - p[9], dy = Y - p[10], dz = Z - p[11];
    double xc = p[0] * dx + p[1] * dy + p[2] * dz;
    double yc = p[3] * dx + p[4] * dy + p[5] * dz;
    double zc = p[6] * dx + p[7] * dy + p[8] * dz;
    double nx, ny, r2, dd;
    if (zc <= 1e-6) return 0;
    nx = xc / zc;
    ny = yc / zc;
    r2 = nx * nx + ny * ny;
    dd = p[12] * (1 + r2 * (p[13] + r2 * (p[14] + r2 * p[15])));
    *u = dd * nx + p[16];
    *v = dd * ny + p[17];
    *z = zc;
    return 1;
}

static double pm_bil(const float* im, int w, int h, double u, double v)
{
    int x0, y0;
    double fx, fy;
    if (!(u >= 0 && v >= 0 && u <= w - 1.001 && v <= h - 1.001)) return NAN;
    x0 = (int)u;
    y0 = (int)v;
    fx = u - x0;
    fy = v - y0;
    return (((double)im[y0 * w + x0] * (1 - fx) + (double)im[y0 * w + x0 + 1] * fx) * (1 - fy) +
            ((double)im[(y0 + 1) * w + x0] * (1 - fx) + (double)im[(y0 + 1) * w + x0 + 1] * fx) * fy);
}

static double pm_cost(const pm_ctx* c, int y, int x, double d, const double* n, double* ncc_out)
{
    const int H = c->H, W = c->W;
    const ptrdiff_t HW = (ptrdiff_t)H * W, idx = (ptrdiff_t)y * W + x;
    const double rpx = c->ray[idx], rpy = c->ray[HW + idx], rpz = c->ray[2 * HW + idx];
    const double ndr = n[0] * rpx + n[1] * rpy + n[2] * rpz;
    double sI[16], sJ[16], sII[16], sJJ[16], sIJ[16], ncc[16], num, photo, geo;
    int cnt[16], nsamp = 0, s, a, b, kk;
    if (ndr >= -1e-6 || d <= 0) {
        *ncc_out = 0;
        return 10.0;
    }
    num = d * ndr;
    for (s = 0; s < c->S; s++) {
        sI[s] = sJ[s] = sII[s] = sJJ[s] = sIJ[s] = 0;
        cnt[s] = 0;
    }
    for (a = -c->r; a <= c->r; a += c->step) {
        const int yy = y + a;
        if (yy < 0 || yy >= H) continue;
        for (b = -c->r; b <= c->r; b += c->step) {
            const int xx = x + b;
            ptrdiff_t q;
            double I, den, t, X, Y, Z;
            if (xx < 0 || xx >= W) continue;
            q = (ptrdiff_t)yy * W + xx;
            I = c->ref[q];
            if (!isfinite(I)) continue;
            den = n[0] * c->ray[q] + n[1] * c->ray[HW + q] + n[2] * c->ray[2 * HW + q];
            if (den >= -1e-9) continue;
            t = num / den;
            X = c->cr0 + t * c->ray[q];
            Y = c->cr1 + t * c->ray[HW + q];
            Z = c->cr2 + t * c->ray[2 * HW + q];
            nsamp += 1;
            for (s = 0; s < c->S; s++) {
                double u, v, z, J;
                if (pm_proj(c->par + 18 * s, X, Y, Z, &u, &v, &z)) {
                    J = pm_bil(c->img[s], c->iw[s], c->ih[s], u, v);
                    if (isfinite(J)) {
                        sI[s] += I;
                        sJ[s] += J;
                        sII[s] += I * I;
                        sJJ[s] += J * J;
                        sIJ[s] += I * J;
                        cnt[s] += 1;
                    }
                }
            }
        }
    }
    for (s = 0; s < c->S; s++) {
        double mi, mj, vi, vj, cv;
        if (nsamp < 4 || cnt[s] < 0.7 * nsamp) {
            ncc[s] = -1;
            continue;
        }
        mi = sI[s] / cnt[s];
        mj = sJ[s] / cnt[s];
        vi = sII[s] / cnt[s] - mi * mi;
        vj = sJJ[s] / cnt[s] - mj * mj;
        cv = sIJ[s] / cnt[s] - mi * mj;
        ncc[s] = (vi < 1e-8 || vj < 1e-8) ? 0 : cv / sqrt(vi * vj);
    }
    for (a = 1; a < c->S; a++) {
        double tmp = ncc[a];
        b = a - 1;
        while (b >= 0 && ncc[b] < tmp) {
            ncc[b + 1] = ncc[b];
            b--;
        }
        ncc[b + 1] = tmp;
    }
    kk = c->top_k < c->S ? c->top_k : c->S;
    photo = 0;
    for (a = 0; a < kk; a++) photo += ncc[a];
    photo /= kk;
    *ncc_out = photo;
    geo = 0;
    if (c->geo_w > 0) {
        const double X = c->cr0 + d * rpx, Y = c->cr1 + d * rpy, Z = c->cr2 + d * rpz;
        int ng = 0;
        for (s = 0; s < c->S; s++) {
            double e = 1.0, u, v, z;
            if (c->dep[s] == NULL) continue;
            ng++;
            if (pm_proj(c->par + 18 * s, X, Y, Z, &u, &v, &z)) {
                const int ui = (int)(u + 0.5), vv = (int)(v + 0.5);
                if (ui >= 0 && vv >= 0 && ui < c->iw[s] && vv < c->ih[s]) {
                    const double dj = c->dep[s][(ptrdiff_t)vv * c->iw[s] + ui];
                    if (isfinite(dj) && dj > 0) {
                        e = fabs(z - dj) / dj / c->geo_tol;
                        if (e > 1) e = 1;
                    }
                }
            }
            geo += e;
        }
        if (ng) geo /= ng;
    }
    return (1 - photo) + c->geo_w * geo;
}

static double rnd_xorshift(uint32_t* st)
{
    st[0] ^= st[0] << 13;
    st[0] ^= st[0] >> 17;
    st[0] ^= st[0] << 5;
    return (st[0] & 0xFFFFFF) / 16777216.0;
}

/* The stream carried across calls: state NULL starts at seed | 1 as the reference does; otherwise
 * the stream starts at *state and the state after the call's draws is written back (a job split
 * over calls with it0 = iterations done). Returns the change count. */
EXPORT int64_t oracle_pm_refine(int H, int W, const float* ref, const float* ray, const double* Cr, int S,
                                const float* const* srcs, const float* const* src_depths, const int* src_h,
                                const int* src_w, const double* par, float* depth, float* normal, float* score,
                                const unsigned char* active, int r, int step, int top_k, double geo_w, double geo_tol,
                                int iters, double dmin, double dmax, uint32_t seed, uint32_t* state, int it0)
{
    static const int offy[8] = {-1, 1, 0, 0, -5, 5, 0, 0};
    static const int offx[8] = {0, 0, -1, 1, 0, 0, -5, 5};
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    pm_ctx c;
    uint32_t st = state ? *state : (seed | 1u);
    int64_t changed = 0;
    int it, colour, y, x, k, tr;
    if (S == 0 || S > 16) return 0;
    c.ref = ref; c.H = H; c.W = W; c.ray = ray; c.cr0 = Cr[0]; c.cr1 = Cr[1]; c.cr2 = Cr[2]; c.S = S;
    c.img = srcs; c.dep = src_depths; c.iw = src_w; c.ih = src_h; c.par = par;
    c.r = r; c.step = step; c.top_k = top_k; c.geo_w = geo_w; c.geo_tol = geo_tol;
    for (it = 0; it < iters; it++) {
        const int git = it0 + it;
        const double dd_scale = 0.05 / (git + 1), nn_scale = 0.3 / (git + 1);
        for (colour = 0; colour < 2; colour++) {
            for (y = 0; y < H; y++) {
                for (x = 0; x < W; x++) {
                    const ptrdiff_t idx = (ptrdiff_t)y * W + x;
                    double n[3], nb[3], best, cst, ncc, sc;
                    if (!active[idx] || (x + y) % 2 != colour) continue;
                    n[0] = normal[idx]; n[1] = normal[HW + idx]; n[2] = normal[2 * HW + idx];
                    if (isfinite(depth[idx])) {
                        best = pm_cost(&c, y, x, depth[idx], n, &ncc);
                        sc = ncc;
                    } else {
                        best = 1e9;
                        sc = -1;
                    }
                    for (k = 0; k < 8; k++) {
                        const int yn = y + offy[k], xn = x + offx[k];
                        ptrdiff_t nidx;
                        double dn, ndr, dp;
                        if (yn < 0 || xn < 0 || yn >= H || xn >= W || !isfinite(depth[(ptrdiff_t)yn * W + xn])) continue;
                        nidx = (ptrdiff_t)yn * W + xn;
                        nb[0] = normal[nidx]; nb[1] = normal[HW + nidx]; nb[2] = normal[2 * HW + nidx];
                        dn = nb[0] * ray[nidx] + nb[1] * ray[HW + nidx] + nb[2] * ray[2 * HW + nidx];
                        ndr = nb[0] * ray[idx] + nb[1] * ray[HW + idx] + nb[2] * ray[2 * HW + idx];
                        if (ndr >= -1e-6) continue;
                        dp = depth[nidx] * dn / ndr;
                        if (dp < dmin || dp > dmax) continue;
                        cst = pm_cost(&c, y, x, dp, nb, &ncc);
                        if (cst < best) {
                            best = cst;
                            sc = ncc;
                            depth[idx] = (float)dp;
                            normal[idx] = (float)nb[0]; normal[HW + idx] = (float)nb[1]; normal[2 * HW + idx] = (float)nb[2];
                            changed++;
                        }
                    }
                    if (isfinite(depth[idx])) {
                        for (tr = 0; tr < 2; tr++) {
                            double u0, u1, u2, u3, dp, nn;
                            u0 = rnd_xorshift(&st); u1 = rnd_xorshift(&st); u2 = rnd_xorshift(&st); u3 = rnd_xorshift(&st);
                            dp = depth[idx] * (1 + dd_scale * (2 * u0 - 1));
                            nb[0] = normal[idx] + nn_scale * (2 * u1 - 1);
                            nb[1] = normal[HW + idx] + nn_scale * (2 * u2 - 1);
                            nb[2] = normal[2 * HW + idx] + nn_scale * (2 * u3 - 1);
                            nn = sqrt(nb[0] * nb[0] + nb[1] * nb[1] + nb[2] * nb[2]);
                            if (nn < 1e-9 || dp < dmin || dp > dmax) continue;
                            nb[0] /= nn; nb[1] /= nn; nb[2] /= nn;
                            cst = pm_cost(&c, y, x, dp, nb, &ncc);
                            if (cst < best) {
                                best = cst;
                                sc = ncc;
                                depth[idx] = (float)dp;
                                normal[idx] = (float)nb[0]; normal[HW + idx] = (float)nb[1]; normal[2 * HW + idx] = (float)nb[2];
                                changed++;
                            }
                        }
                    }
                    score[idx] = (float)sc;
                }
            }
        }
    }
    if (state) *state = st;
    return changed;
}

/* ------------------------------------------------------------------ pass-2 geometry (densify.py:441-496) */
/* The 3 x 3 products of the reference's consistency check are NumPy matmuls of (n, 3) rows by a
 * 3 x 3 matrix; NumPy hands them to OpenBLAS, whose dgemm accumulates each output as
 * a = m0 * r0; a = fma(m1, r1, a); a = fma(m2, r2, a) (checked against NumPy on this machine). */
static double dot3_blas(double m0, double m1, double m2, double r0, double r1, double r2)
{
    double a = m0 * r0;
    a = fma(m1, r1, a);
    return fma(m2, r2, a);
}

/* _fast._undistort (_fast.pyx:145-164) */
static void undistort(double u, double v, const double* cam, double* xo, double* yo)
{
    const double f = cam[12], k1 = cam[13], k2 = cam[14], k3 = cam[15], cx = cam[16], cy = cam[17];
    const double nx = (u - cx) / f, ny = (v - cy) / f;
    double x = nx, y = ny, r2, d, t;
    int it;
    for (it = 0; it < 8; it++) {
        r2 = x * x;
        t = y * y;
        r2 = r2 + t;
        d = r2 * k3;
        d = k2 + d;
        d = r2 * d;
        d = k1 + d;
        d = r2 * d;
        d = 1.0 + d;
        x = nx / d;
        y = ny / d;
    }
    *xo = x;
    *yo = y;
}

/* _fast._project (_fast.pyx:167-185) */
static void project(double xc0, double xc1, double xc2, const double* cam, double* uo, double* vo)
{
    const double f = cam[12], k1 = cam[13], k2 = cam[14], k3 = cam[15], cx = cam[16], cy = cam[17];
    const double z = (xc2 >= 1e-6 || isnan(xc2)) ? xc2 : 1e-6;
    const double x = xc0 / z, y = xc1 / z;
    double r2 = x * x, t = y * y, d;
    r2 = r2 + t;
    d = r2 * k3;
    d = k2 + d;
    d = r2 * d;
    d = k1 + d;
    d = r2 * d;
    d = 1.0 + d;
    d = f * d;
    t = d * x;
    *uo = t + cx;
    t = d * y;
    *vo = t + cy;
}

/* densify._consistency (densify.py:441-478) through its compiled path (_fast.ref_points,
 * neighbour_sample, agreement, _fast.pyx:201-268): per finite pixel of the reference depth map D,
 * the number of neighbour depth maps that agree (forward-backward reprojection within px_tol
 * pixels and relative depth within rel_tol[j]). Camera rows: R (9), C (3), f, k1, k2, k3, cx, cy.
 * The optional active mask is pass 2's PatchMatch selection (densify.py:621):
 * finite(grey) & ((count < min_views - 1) | (score < min_ncc) | !finite(D)), with min_ncc
 * compared in float32 as NumPy does for a float32 array. */
EXPORT void oracle_consistency(int H, int W, const float* D, const double* cam, int n_nb, const float* const* nb_depth,
                               const int* nb_h, const int* nb_w, const double* nb_cam, const double* rel_tol,
                               double px_tol, int16_t* count, const float* grey, const float* score, double min_ncc,
                               int min_views, uint8_t* active)
{
    const double* R = cam;
    const double* C = cam + 9;
    const float min_ncc_f = (float)min_ncc;
    int y, x, j, i;
    for (y = 0; y < H; y++) {
        for (x = 0; x < W; x++) {
            const ptrdiff_t idx = (ptrdiff_t)y * W + x;
            const float Dv = D[idx];
            int c = 0;
            if (isfinite(Dv)) {
                const double d = Dv;
                double rx, ry, M[3], X[3];
                undistort((double)x, (double)y, cam, &rx, &ry);
                M[0] = rx * d; M[1] = ry * d; M[2] = d;
                for (i = 0; i < 3; i++) X[i] = C[i] + dot3_blas(M[0], M[1], M[2], R[i], R[3 + i], R[6 + i]);
                for (j = 0; j < n_nb; j++) {
                    const double* cj = nb_cam + 18 * j;
                    const double* Rj = cj;
                    const double* Cj = cj + 9;
                    double dx[3], xc[3], u, v, dd, xj, yj, Mj[3], Xj[3], dk[3], xk[3], ub, vb;
                    int64_t a, b;
                    for (i = 0; i < 3; i++) dx[i] = X[i] - Cj[i];
                    for (i = 0; i < 3; i++) xc[i] = dot3_blas(dx[0], dx[1], dx[2], Rj[3 * i], Rj[3 * i + 1], Rj[3 * i + 2]);
                    project(xc[0], xc[1], xc[2], cj, &u, &v);
                    a = (int64_t)rint(u);
                    b = (int64_t)rint(v);
                    if (xc[2] > 0 && a >= 0 && b >= 0 && a < nb_w[j] && b < nb_h[j])
                        dd = nb_depth[j][(ptrdiff_t)b * nb_w[j] + a];
                    else
                        dd = NAN;
                    undistort((double)a, (double)b, cj, &xj, &yj);
                    Mj[0] = xj * dd; Mj[1] = yj * dd; Mj[2] = dd;
                    for (i = 0; i < 3; i++) Xj[i] = Cj[i] + dot3_blas(Mj[0], Mj[1], Mj[2], Rj[i], Rj[3 + i], Rj[6 + i]);
                    for (i = 0; i < 3; i++) dk[i] = Xj[i] - C[i];
                    for (i = 0; i < 3; i++) xk[i] = dot3_blas(dk[0], dk[1], dk[2], R[3 * i], R[3 * i + 1], R[3 * i + 2]);
                    project(xk[0], xk[1], xk[2], cam, &ub, &vb);
                    {
                        const double t = rel_tol[j] * dd;
                        if (isfinite(dd) && hypot(ub - (double)x, vb - (double)y) <= px_tol && fabs(dd - xc[2]) <= t) c++;
                    }
                }
            }
            if (count) count[idx] = (int16_t)c;
            if (active) {
                const int fin_g = isfinite(grey[idx]);
                active[idx] = (uint8_t)(fin_g && (c < min_views - 1 || score[idx] < min_ncc_f || !isfinite(Dv)));
            }
        }
    }
}

/* densify._init_normals (densify.py:481-496), float32 NumPy semantics: P = ray * D (NaN where D is
 * not finite), 2-px central differences along columns (tu) and rows (tv), n = tu x tv
 * (np.cross: a1 b2 - a2 b1, ...), |n| = sqrt((n0^2 + n1^2) + n2^2), n / |n| or (0, 0, 1) where
 * |n| is not finite or < 1e-12, negated where n . ray = (n0 r0 + n1 r1) + n2 r2 > 0. */
EXPORT void oracle_init_normals(int H, int W, const float* D, const float* ray, float* normal)
{
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    int y, x, k;
    for (y = 0; y < H; y++) {
        for (x = 0; x < W; x++) {
            const ptrdiff_t idx = (ptrdiff_t)y * W + x;
            float tu[3], tv[3], n[3], nn, s;
            const float nanf_ = NAN;
            for (k = 0; k < 3; k++) {
                tu[k] = nanf_;
                tv[k] = nanf_;
            }
            if (x >= 2 && x < W - 2) {
                const float da = D[idx + 2], db = D[idx - 2];
                const float pa = isfinite(da) ? da : nanf_, pb = isfinite(db) ? db : nanf_;
                for (k = 0; k < 3; k++) tu[k] = ray[k * HW + idx + 2] * pa - ray[k * HW + idx - 2] * pb;
            }
            if (y >= 2 && y < H - 2) {
                const float da = D[idx + 2 * (ptrdiff_t)W], db = D[idx - 2 * (ptrdiff_t)W];
                const float pa = isfinite(da) ? da : nanf_, pb = isfinite(db) ? db : nanf_;
                for (k = 0; k < 3; k++) tv[k] = ray[k * HW + idx + 2 * (ptrdiff_t)W] * pa - ray[k * HW + idx - 2 * (ptrdiff_t)W] * pb;
            }
            {
                const float p0 = tu[1] * tv[2], q0 = tu[2] * tv[1];
                const float p1 = tu[2] * tv[0], q1 = tu[0] * tv[2];
                const float p2 = tu[0] * tv[1], q2 = tu[1] * tv[0];
                n[0] = p0 - q0;
                n[1] = p1 - q1;
                n[2] = p2 - q2;
            }
            {
                const float s0 = n[0] * n[0], s1 = n[1] * n[1], s2 = n[2] * n[2];
                nn = sqrtf((s0 + s1) + s2);
            }
            if (!isfinite(nn) || nn < 1e-12f) {
                n[0] = 0.0f; n[1] = 0.0f; n[2] = 1.0f;
            } else {
                for (k = 0; k < 3; k++) n[k] = n[k] / nn;
            }
            {
                const float s0 = n[0] * ray[idx], s1 = n[1] * ray[HW + idx], s2 = n[2] * ray[2 * HW + idx];
                s = (s0 + s1) + s2;
            }
            if (s > 0.0f)
                for (k = 0; k < 3; k++) n[k] = -n[k];
            for (k = 0; k < 3; k++) normal[k * HW + idx] = n[k];
        }
    }
}

/* One reference image k of densify._fuse_loop (densify.py:688-762) on its compiled path
 * (_fast.ref_points, neighbour_sample, agreement, accumulate; _fast.pyx:201-284):
 * candidates are the finite, not yet used pixels of D on the point_stride grid (rows and columns
 * multiples of the stride); for each the world point X (acc starts at X, cnt at 1), then for
 * every neighbour j in order the forward-backward check of oracle_consistency, adding j's
 * back-projected point to acc (component by component) when it agrees. Pixels with
 * cnt >= min_views are kept: keep = 1, xyz = acc / cnt, and for every agreeing neighbour the
 * stride-grid pixel ((vi / st) st, (ui / st) st) of j's used mask is set. Outputs: keep (H, W),
 * xyz (3, H, W) (where keep), count (H, W). */
EXPORT void oracle_fuse_view(int H, int W, const float* D, uint8_t* used, const double* cam, int n_nb,
                             const float* const* nb_depth, uint8_t* const* nb_used, const int* nb_h, const int* nb_w,
                             const double* nb_cam, const double* rel_tol, double px_tol, int min_views,
                             int point_stride, uint8_t* keep, double* xyz, int32_t* count)
{
    const double* R = cam;
    const double* C = cam + 9;
    const int st = point_stride > 1 ? point_stride : 1;
    const ptrdiff_t HW = (ptrdiff_t)H * W;
    int y, x, j, i;
    for (y = 0; y < H; y++) {
        for (x = 0; x < W; x++) {
            const ptrdiff_t idx = (ptrdiff_t)y * W + x;
            const float Dv = D[idx];
            int64_t ui_[16], vi_[16];
            int ok_[16];
            double X[3], acc[3], M[3], rx, ry, d;
            int32_t cnt = 1;
            keep[idx] = 0;
            count[idx] = 0;
            if (!isfinite(Dv) || used[idx] || (st > 1 && (y % st != 0 || x % st != 0))) continue;
            d = Dv;
            undistort((double)x, (double)y, cam, &rx, &ry);
            M[0] = rx * d; M[1] = ry * d; M[2] = d;
            for (i = 0; i < 3; i++) X[i] = C[i] + dot3_blas(M[0], M[1], M[2], R[i], R[3 + i], R[6 + i]);
            for (i = 0; i < 3; i++) acc[i] = X[i];
            for (j = 0; j < n_nb; j++) {
                const double* cj = nb_cam + 18 * j;
                const double* Rj = cj;
                const double* Cj = cj + 9;
                double dx[3], xc[3], u, v, dd, xj, yj, Mj[3], Xj[3], dk[3], xk[3], ub, vb;
                int64_t a, b;
                for (i = 0; i < 3; i++) dx[i] = X[i] - Cj[i];
                for (i = 0; i < 3; i++) xc[i] = dot3_blas(dx[0], dx[1], dx[2], Rj[3 * i], Rj[3 * i + 1], Rj[3 * i + 2]);
                project(xc[0], xc[1], xc[2], cj, &u, &v);
                a = (int64_t)rint(u);
                b = (int64_t)rint(v);
                if (xc[2] > 0 && a >= 0 && b >= 0 && a < nb_w[j] && b < nb_h[j])
                    dd = nb_depth[j][(ptrdiff_t)b * nb_w[j] + a];
                else
                    dd = NAN;
                undistort((double)a, (double)b, cj, &xj, &yj);
                Mj[0] = xj * dd; Mj[1] = yj * dd; Mj[2] = dd;
                for (i = 0; i < 3; i++) Xj[i] = Cj[i] + dot3_blas(Mj[0], Mj[1], Mj[2], Rj[i], Rj[3 + i], Rj[6 + i]);
                for (i = 0; i < 3; i++) dk[i] = Xj[i] - C[i];
                for (i = 0; i < 3; i++) xk[i] = dot3_blas(dk[0], dk[1], dk[2], R[3 * i], R[3 * i + 1], R[3 * i + 2]);
                project(xk[0], xk[1], xk[2], cam, &ub, &vb);
                ui_[j] = a;
                vi_[j] = b;
                {
                    const double t = rel_tol[j] * dd;
                    ok_[j] = isfinite(dd) && hypot(ub - (double)x, vb - (double)y) <= px_tol && fabs(dd - xc[2]) <= t;
                }
                if (ok_[j]) {
                    for (i = 0; i < 3; i++) acc[i] = acc[i] + Xj[i];
                    cnt = cnt + 1;
                }
            }
            count[idx] = cnt;
            if (cnt < min_views) continue;
            keep[idx] = 1;
            for (i = 0; i < 3; i++) xyz[i * HW + idx] = acc[i] / (double)cnt;
            for (j = 0; j < n_nb; j++)
                if (ok_[j]) nb_used[j][(ptrdiff_t)((vi_[j] / st) * st) * nb_w[j] + (ui_[j] / st) * st] = 1;
        }
    }
}

/* ------------------------------------------------------------------ legacy height sweep (mvs.py) */

/* _mvs.sample_view (_mvs.pyx:13-58): ground cell (r, c) of a (H, W) grid at height Z[r, c] is
 * (X0 + (c + .5) gsd, Y0 - (r + .5) gsd, Z); projected with the camera (R row-major, C, f, k1..k3,
 * cx, cy in img pixels), bilinear in float64 over nch channels of img (h, w, nch) with the last
 * row / column repeated; out (H, W, nch) is written only where valid (the caller zeroes it). */
EXPORT void oracle_sample_view(int h, int w, int nch, const float* img, const double* R, const double* C, double f,
                               double k1, double k2, double k3, double cx, double cy, double X0, double Y0,
                               double gsd, int H, int W, const float* Z, float* out, uint8_t* valid)
{
    int r, c, ch;
    for (r = 0; r < H; r++) {
        const double Y = Y0 - (r + 0.5) * gsd;
        for (c = 0; c < W; c++) {
            const double X = X0 + (c + 0.5) * gsd;
            const double dx = X - C[0], dy = Y - C[1], dz = (double)Z[(ptrdiff_t)r * W + c] - C[2];
            const double zc = R[6] * dx + R[7] * dy + R[8] * dz;
            double xc, yc, nx, ny, r2, d, u, v, fx, fy;
            ptrdiff_t x0, y0, x1, y1;
            valid[(ptrdiff_t)r * W + c] = 0;
            if (zc <= 1e-6) continue;
            xc = R[0] * dx + R[1] * dy + R[2] * dz;
            yc = R[3] * dx + R[4] * dy + R[5] * dz;
            nx = xc / zc;
            ny = yc / zc;
            r2 = nx * nx + ny * ny;
            d = 1.0 + r2 * (k1 + r2 * (k2 + r2 * k3));
            u = f * d * nx + cx;
            v = f * d * ny + cy;
            if (u < 0 || v < 0 || u > (double)(w - 1) || v > (double)(h - 1)) continue;
            x0 = (ptrdiff_t)u;
            y0 = (ptrdiff_t)v;
            x1 = x0 + 1 < w ? x0 + 1 : x0;
            y1 = y0 + 1 < h ? y0 + 1 : y0;
            fx = u - (double)x0;
            fy = v - (double)y0;
            for (ch = 0; ch < nch; ch++) {
                const double a00 = img[(y0 * w + x0) * nch + ch], a01 = img[(y0 * w + x1) * nch + ch];
                const double a10 = img[(y1 * w + x0) * nch + ch], a11 = img[(y1 * w + x1) * nch + ch];
                out[((ptrdiff_t)r * W + c) * nch + ch] =
                    (float)((1 - fy) * ((1 - fx) * a00 + fx * a01) + fy * ((1 - fx) * a10 + fx * a11));
            }
            valid[(ptrdiff_t)r * W + c] = 1;
        }
    }
}

/* _fast.box_sat_mean (_fast.pyx:897-942): float64 summed-area mean over a (2r+1)^2 window with
 * zero padding, B planes of (H, W) float32: column sums down the rows, then a running row total
 * of those, window = ((S[y+k][x+k] - S[y][x+k]) - S[y+k][x]) + S[y][x], divided by k^2. */
EXPORT int oracle_box_sat_mean(int B, int H, int W, const float* a, int r, float* out)
{
    const int k = 2 * r + 1, PW = W + 2 * r + 1, PH = H + 2 * r + 1;
    const double denom = (double)k * (double)k;
    double* col;
    double* sat;
    int b, i, x, y;
    if (r < 0) return -1;
    if (B == 0 || H == 0 || W == 0) return 0;
    col = (double*)malloc(sizeof(double) * W);
    sat = (double*)malloc(sizeof(double) * (size_t)PH * PW);
    if (!col || !sat) { free(col); free(sat); return -2; }
    for (b = 0; b < B; b++) {
        const float* ab = a + (size_t)b * H * W;
        for (x = 0; x < W; x++) col[x] = 0.0;
        for (i = 0; i < PH; i++) {
            const int ay = i - r - 1;
            double* cur = sat + (size_t)i * PW;
            double total = 0.0;
            for (x = 0; x < r + 1; x++) cur[x] = 0.0;
            for (x = 0; x < W; x++) {
                const double val = (ay >= 0 && ay < H) ? (double)ab[(size_t)ay * W + x] : 0.0;
                col[x] = col[x] + val;
                total = total + col[x];
                cur[x + r + 1] = total;
            }
            for (x = r + 1 + W; x < PW; x++) cur[x] = total;
        }
        for (y = 0; y < H; y++) {
            const double* cur = sat + (size_t)(y + k) * PW;
            const double* old = sat + (size_t)y * PW;
            for (x = 0; x < W; x++) {
                double val = cur[x + k] - old[x + k];
                val = val - cur[x];
                val = val + old[x];
                out[(size_t)b * H * W + (size_t)y * W + x] = (float)(val / denom);
            }
        }
    }
    free(col);
    free(sat);
    return 0;
}

/* _mvs.sgm (_mvs.pyx:98-251): semi-global aggregation of a (D, H, W) float32 cost volume along the
 * 8 directions (0,1) (0,-1) (1,0) (-1,0) (1,1) (1,-1) (-1,1) (-1,-1), summed in that order:
 * L(p, d) = C(p, d) + min(L(q, d), L(q, d+-1) + P1, min_k L(q, k) + P2) - min_k L(q, k), q = p - dir. */
EXPORT int oracle_sgm(int D, int H, int W, const float* cost, float P1, float P2, float* agg)
{
    static const int dirs[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    const size_t HW = (size_t)H * W;
    float* L = (float*)malloc(sizeof(float) * (size_t)D * HW);
    int k, yy, xx, d;
    if (!L) return -2;
    for (size_t q = 0; q < (size_t)D * HW; q++) agg[q] = 0.0f;
    for (k = 0; k < 8; k++) {
        const int dy = dirs[k][0], dx = dirs[k][1];
        for (yy = 0; yy < H; yy++) {
            const int y = dy >= 0 ? yy : H - 1 - yy;
            for (xx = 0; xx < W; xx++) {
                const int x = dx >= 0 ? xx : W - 1 - xx;
                const int py = y - dy, px = x - dx;
                const size_t o = (size_t)y * W + x;
                if (py < 0 || py >= H || px < 0 || px >= W) {
                    for (d = 0; d < D; d++) L[d * HW + o] = cost[d * HW + o];
                } else {
                    const size_t po = (size_t)py * W + px;
                    float best = L[po];
                    for (d = 1; d < D; d++) if (L[d * HW + po] < best) best = L[d * HW + po];
                    for (d = 0; d < D; d++) {
                        float v = L[d * HW + po], a, bb;
                        if (d > 0) { a = L[(d - 1) * HW + po] + P1; if (a < v) v = a; }
                        if (d < D - 1) { bb = L[(d + 1) * HW + po] + P1; if (bb < v) v = bb; }
                        if (best + P2 < v) v = best + P2;
                        L[d * HW + o] = cost[d * HW + o] + v - best;
                    }
                }
                for (d = 0; d < D; d++) agg[d * HW + o] += L[d * HW + o];
            }
        }
    }
    free(L);
    return 0;
}
