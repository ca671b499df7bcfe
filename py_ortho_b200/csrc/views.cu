// Passes 2 and 3 of the multi-view depth maps on the device: the geometric consistency check that
// selects the pixels PatchMatch repairs (densify._consistency, densify.py:441-478, through the
// compiled helpers of _fast.pyx:201-268), the initial PatchMatch normals (densify._init_normals,
// densify.py:481-496) and the point fusion of one reference image (densify._fuse_loop,
// densify.py:688-762, with _fast.accumulate, _fast.pyx:271-284).
//
// This file is compiled with -fmad=false and writes every rounding explicitly: each double
// operation is rounded once in the reference's order, and the reference's 3 x 3 products - NumPy
// matmuls that OpenBLAS evaluates as m0 r0, then two fused multiply-adds - use __fma_rn in the
// same order. The counts and normals are bit-identical to the reference's.
#include "common.cuh"

namespace mvs {

struct ConsParams {
    int H, W, n_nb, min_views;
    float min_ncc;
    double px_tol;
    const float* depth;
    const float* grey;
    const float* score;
    short* count;
    unsigned char* active;
    double cam[18];
    int pinhole;                               // the view's k1 = k2 = k3 = 0
    const float* nb_depth[MVS_MAX_SOURCES];
    int nb_h[MVS_MAX_SOURCES], nb_w[MVS_MAX_SOURCES], nb_pinhole[MVS_MAX_SOURCES];
    double nb_cam[MVS_MAX_SOURCES * 18];
    double rel_tol[MVS_MAX_SOURCES];
};

// m0 r0 + m1 r1 + m2 r2 as OpenBLAS's dgemm forms it for a NumPy (n, 3) @ (3, 3) product.
__device__ __forceinline__ double dot3_blas(double m0, double m1, double m2, double r0, double r1, double r2) {
    double a = __dmul_rn(m0, r0);
    a = __fma_rn(m1, r1, a);
    return __fma_rn(m2, r2, a);
}

// _fast._undistort (_fast.pyx:145-164): 8 fixed-point iterations. For a pinhole camera every
// iteration's factor is exactly 1 (r2 finite: r2 * 0 = +0, 0 + +0 = +0, 1 + +0 = 1), so x = nx.
__device__ __forceinline__ void undistort(double u, double v, const double* cam, bool pinhole, double& xo,
                                          double& yo) {
    const double f = cam[12], cx = cam[16], cy = cam[17];
    const double nx = __ddiv_rn(__dsub_rn(u, cx), f), ny = __ddiv_rn(__dsub_rn(v, cy), f);
    double x = nx, y = ny;
    const double r20 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    if (!(pinhole && isfinite(r20))) {
        const double k1 = cam[13], k2 = cam[14], k3 = cam[15];
        for (int it = 0; it < 8; ++it) {
            const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
            double d = __dmul_rn(r2, k3);
            d = __dadd_rn(k2, d);
            d = __dmul_rn(r2, d);
            d = __dadd_rn(k1, d);
            d = __dmul_rn(r2, d);
            d = __dadd_rn(1.0, d);
            x = __ddiv_rn(nx, d);
            y = __ddiv_rn(ny, d);
        }
    }
    xo = x;
    yo = y;
}

// _fast._project (_fast.pyx:167-185), z = max(xc2, 1e-6) with NaN propagating.
__device__ __forceinline__ void project(double xc0, double xc1, double xc2, const double* cam, bool pinhole,
                                        double& uo, double& vo) {
    const double f = cam[12], cx = cam[16], cy = cam[17];
    const double z = (xc2 >= 1e-6 || isnan(xc2)) ? xc2 : 1e-6;
    const double x = __ddiv_rn(xc0, z), y = __ddiv_rn(xc1, z);
    const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    double d;
    if (pinhole && isfinite(r2)) {
        d = f;                                     // f * (1 + r2 (0 + r2 (0 + r2 0))) = f exactly
    } else {
        d = __dmul_rn(r2, cam[15]);
        d = __dadd_rn(cam[14], d);
        d = __dmul_rn(r2, d);
        d = __dadd_rn(cam[13], d);
        d = __dmul_rn(r2, d);
        d = __dadd_rn(1.0, d);
        d = __dmul_rn(f, d);
    }
    uo = __dadd_rn(__dmul_rn(d, x), cx);
    vo = __dadd_rn(__dmul_rn(d, y), cy);
}

__global__ void __launch_bounds__(256) consistency_kernel(const __grid_constant__ ConsParams c) {
    const long long HW = (long long)c.H * c.W;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= HW) return;
    const int y = (int)(idx / c.W), x = (int)(idx - (long long)y * c.W);
    const float Dv = c.depth[idx];
    int cnt = 0;
    if (isfinite(Dv)) {
        const double* R = c.cam;
        const double* C = c.cam + 9;
        const double d = (double)Dv;
        double rx, ry;
        undistort((double)x, (double)y, c.cam, c.pinhole, rx, ry);
        const double m0 = __dmul_rn(rx, d), m1 = __dmul_rn(ry, d);
        const double X0 = __dadd_rn(C[0], dot3_blas(m0, m1, d, R[0], R[3], R[6]));
        const double X1 = __dadd_rn(C[1], dot3_blas(m0, m1, d, R[1], R[4], R[7]));
        const double X2 = __dadd_rn(C[2], dot3_blas(m0, m1, d, R[2], R[5], R[8]));
        for (int j = 0; j < c.n_nb; ++j) {
            const double* cj = c.nb_cam + 18 * j;
            const double* Cj = cj + 9;
            const bool pj = c.nb_pinhole[j];
            const double dx0 = __dsub_rn(X0, Cj[0]), dx1 = __dsub_rn(X1, Cj[1]), dx2 = __dsub_rn(X2, Cj[2]);
            const double xc0 = dot3_blas(dx0, dx1, dx2, cj[0], cj[1], cj[2]);
            const double xc1 = dot3_blas(dx0, dx1, dx2, cj[3], cj[4], cj[5]);
            const double xc2 = dot3_blas(dx0, dx1, dx2, cj[6], cj[7], cj[8]);
            double u, v;
            project(xc0, xc1, xc2, cj, pj, u, v);
            // <int64_t>rint(u): out-of-range values fail the bounds test either way
            const double ur = rint(u), vr = rint(v);
            const long long a = (ur > -9.0e18 && ur < 9.0e18) ? (long long)ur : -1;
            const long long b = (vr > -9.0e18 && vr < 9.0e18) ? (long long)vr : -1;
            double dd = __longlong_as_double(0x7ff8000000000000LL);
            if (xc2 > 0.0 && a >= 0 && b >= 0 && a < c.nb_w[j] && b < c.nb_h[j])
                dd = (double)__ldg(c.nb_depth[j] + b * c.nb_w[j] + a);
            if (!isfinite(dd)) continue;               // agreement needs a finite neighbour depth
            double xj, yj;
            undistort((double)a, (double)b, cj, pj, xj, yj);
            const double n0 = __dmul_rn(xj, dd), n1 = __dmul_rn(yj, dd);
            const double Y0 = __dadd_rn(Cj[0], dot3_blas(n0, n1, dd, cj[0], cj[3], cj[6]));
            const double Y1 = __dadd_rn(Cj[1], dot3_blas(n0, n1, dd, cj[1], cj[4], cj[7]));
            const double Y2 = __dadd_rn(Cj[2], dot3_blas(n0, n1, dd, cj[2], cj[5], cj[8]));
            const double e0 = __dsub_rn(Y0, C[0]), e1 = __dsub_rn(Y1, C[1]), e2 = __dsub_rn(Y2, C[2]);
            const double xk0 = dot3_blas(e0, e1, e2, R[0], R[1], R[2]);
            const double xk1 = dot3_blas(e0, e1, e2, R[3], R[4], R[5]);
            const double xk2 = dot3_blas(e0, e1, e2, R[6], R[7], R[8]);
            double ub, vb;
            project(xk0, xk1, xk2, c.cam, c.pinhole, ub, vb);
            const double t = __dmul_rn(c.rel_tol[j], dd);
            if (hypot(__dsub_rn(ub, (double)x), __dsub_rn(vb, (double)y)) <= c.px_tol &&
                fabs(__dsub_rn(dd, xc2)) <= t)
                ++cnt;
        }
    }
    if (c.count) c.count[idx] = (short)cnt;
    if (c.active) {
        const bool fin_g = isfinite(c.grey[idx]);
        c.active[idx] = (unsigned char)(fin_g && (cnt < c.min_views - 1 || c.score[idx] < c.min_ncc || !isfinite(Dv)));
    }
}

// densify._init_normals in float32 NumPy semantics (one rounding per ufunc, np.cross as
// a1 b2 - a2 b1, ..., norm and dot product summed as (0 + 1) + 2).
__global__ void __launch_bounds__(256) init_normals_kernel(int H, int W, const float* __restrict__ D,
                                                           const float* __restrict__ ray,
                                                           float* __restrict__ normal) {
    const long long HW = (long long)H * W;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= HW) return;
    const int y = (int)(idx / W), x = (int)(idx - (long long)y * W);
    const float qnan = __int_as_float(0x7fc00000);
    float tu[3] = {qnan, qnan, qnan}, tv[3] = {qnan, qnan, qnan};
    if (x >= 2 && x < W - 2) {
        const float da = D[idx + 2], db = D[idx - 2];
        const float pa = isfinite(da) ? da : qnan, pb = isfinite(db) ? db : qnan;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            tu[k] = __fsub_rn(__fmul_rn(ray[k * HW + idx + 2], pa), __fmul_rn(ray[k * HW + idx - 2], pb));
    }
    if (y >= 2 && y < H - 2) {
        const long long o = 2LL * W;
        const float da = D[idx + o], db = D[idx - o];
        const float pa = isfinite(da) ? da : qnan, pb = isfinite(db) ? db : qnan;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            tv[k] = __fsub_rn(__fmul_rn(ray[k * HW + idx + o], pa), __fmul_rn(ray[k * HW + idx - o], pb));
    }
    float n0 = __fsub_rn(__fmul_rn(tu[1], tv[2]), __fmul_rn(tu[2], tv[1]));
    float n1 = __fsub_rn(__fmul_rn(tu[2], tv[0]), __fmul_rn(tu[0], tv[2]));
    float n2 = __fsub_rn(__fmul_rn(tu[0], tv[1]), __fmul_rn(tu[1], tv[0]));
    const float nn = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(n0, n0), __fmul_rn(n1, n1)), __fmul_rn(n2, n2)));
    if (!isfinite(nn) || nn < 1e-12f) {
        n0 = 0.0f;
        n1 = 0.0f;
        n2 = 1.0f;
    } else {
        n0 = __fdiv_rn(n0, nn);
        n1 = __fdiv_rn(n1, nn);
        n2 = __fdiv_rn(n2, nn);
    }
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(n0, ray[idx]), __fmul_rn(n1, ray[HW + idx])),
                              __fmul_rn(n2, ray[2 * HW + idx]));
    if (s > 0.0f) {
        n0 = -n0;
        n1 = -n1;
        n2 = -n2;
    }
    normal[idx] = n0;
    normal[HW + idx] = n1;
    normal[2 * HW + idx] = n2;
}


// Fusion of one reference image (densify._fuse_loop, densify.py:688-762): the forward-backward
// check of consistency_kernel for every neighbour in order, the agreeing neighbours' points added
// to the pixel's own (acc starts at X, cnt at 1), kept when cnt >= min_views, and the agreeing
// neighbours' stride-grid pixels marked as used. Views run one launch after another (the marks
// of a view gate the candidates of the later ones); within a launch only other views' masks are
// written, and only with 1.
struct FuseParams {
    int H, W, n_nb, min_views, stride;
    double px_tol;
    const float* depth;
    const unsigned char* used;
    unsigned char* keep;
    double* xyz;
    int* count;
    double cam[18];
    int pinhole;
    const float* nb_depth[MVS_MAX_SOURCES];
    unsigned char* nb_used[MVS_MAX_SOURCES];
    int nb_h[MVS_MAX_SOURCES], nb_w[MVS_MAX_SOURCES], nb_pinhole[MVS_MAX_SOURCES];
    double nb_cam[MVS_MAX_SOURCES * 18];
    double rel_tol[MVS_MAX_SOURCES];
};

__global__ void __launch_bounds__(256) fuse_kernel(const __grid_constant__ FuseParams c) {
    const long long HW = (long long)c.H * c.W;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= HW) return;
    const int y = (int)(idx / c.W), x = (int)(idx - (long long)y * c.W);
    const int st = c.stride;
    const float Dv = c.depth[idx];
    c.keep[idx] = 0;
    c.count[idx] = 0;
    if (!isfinite(Dv) || c.used[idx] || (st > 1 && (y % st != 0 || x % st != 0))) return;
    const double* R = c.cam;
    const double* C = c.cam + 9;
    const double d = (double)Dv;
    double rx, ry;
    undistort((double)x, (double)y, c.cam, c.pinhole, rx, ry);
    const double m0 = __dmul_rn(rx, d), m1 = __dmul_rn(ry, d);
    const double X0 = __dadd_rn(C[0], dot3_blas(m0, m1, d, R[0], R[3], R[6]));
    const double X1 = __dadd_rn(C[1], dot3_blas(m0, m1, d, R[1], R[4], R[7]));
    const double X2 = __dadd_rn(C[2], dot3_blas(m0, m1, d, R[2], R[5], R[8]));
    double a0 = X0, a1 = X1, a2 = X2;
    int cnt = 1;
    unsigned okbits = 0;
    int mark[MVS_MAX_SOURCES];
    for (int j = 0; j < c.n_nb; ++j) {
        const double* cj = c.nb_cam + 18 * j;
        const double* Cj = cj + 9;
        const bool pj = c.nb_pinhole[j];
        const double dx0 = __dsub_rn(X0, Cj[0]), dx1 = __dsub_rn(X1, Cj[1]), dx2 = __dsub_rn(X2, Cj[2]);
        const double xc0 = dot3_blas(dx0, dx1, dx2, cj[0], cj[1], cj[2]);
        const double xc1 = dot3_blas(dx0, dx1, dx2, cj[3], cj[4], cj[5]);
        const double xc2 = dot3_blas(dx0, dx1, dx2, cj[6], cj[7], cj[8]);
        double u, v;
        project(xc0, xc1, xc2, cj, pj, u, v);
        const double ur = rint(u), vr = rint(v);
        const long long a = (ur > -9.0e18 && ur < 9.0e18) ? (long long)ur : -1;
        const long long b = (vr > -9.0e18 && vr < 9.0e18) ? (long long)vr : -1;
        double dd = __longlong_as_double(0x7ff8000000000000LL);
        if (xc2 > 0.0 && a >= 0 && b >= 0 && a < c.nb_w[j] && b < c.nb_h[j])
            dd = (double)__ldg(c.nb_depth[j] + b * c.nb_w[j] + a);
        if (!isfinite(dd)) continue;               // agreement needs a finite neighbour depth
        double xj, yj;
        undistort((double)a, (double)b, cj, pj, xj, yj);
        const double n0 = __dmul_rn(xj, dd), n1 = __dmul_rn(yj, dd);
        const double Y0 = __dadd_rn(Cj[0], dot3_blas(n0, n1, dd, cj[0], cj[3], cj[6]));
        const double Y1 = __dadd_rn(Cj[1], dot3_blas(n0, n1, dd, cj[1], cj[4], cj[7]));
        const double Y2 = __dadd_rn(Cj[2], dot3_blas(n0, n1, dd, cj[2], cj[5], cj[8]));
        const double e0 = __dsub_rn(Y0, C[0]), e1 = __dsub_rn(Y1, C[1]), e2 = __dsub_rn(Y2, C[2]);
        const double xk0 = dot3_blas(e0, e1, e2, R[0], R[1], R[2]);
        const double xk1 = dot3_blas(e0, e1, e2, R[3], R[4], R[5]);
        const double xk2 = dot3_blas(e0, e1, e2, R[6], R[7], R[8]);
        double ub, vb;
        project(xk0, xk1, xk2, c.cam, c.pinhole, ub, vb);
        const double t = __dmul_rn(c.rel_tol[j], dd);
        if (hypot(__dsub_rn(ub, (double)x), __dsub_rn(vb, (double)y)) <= c.px_tol && fabs(__dsub_rn(dd, xc2)) <= t) {
            // _fast.accumulate: acc[i] = acc[i] + Xj[i]; cnt = cnt + 1
            a0 = __dadd_rn(a0, Y0);
            a1 = __dadd_rn(a1, Y1);
            a2 = __dadd_rn(a2, Y2);
            ++cnt;
            okbits |= 1u << j;
            // the stride-grid pixel of j that would emit this surface sample (a, b >= 0 here)
            mark[j] = (int)((b / st) * st) * c.nb_w[j] + (int)((a / st) * st);
        }
    }
    c.count[idx] = cnt;
    if (cnt < c.min_views) return;
    c.keep[idx] = 1;
    const double dc = (double)cnt;
    c.xyz[idx] = __ddiv_rn(a0, dc);
    c.xyz[HW + idx] = __ddiv_rn(a1, dc);
    c.xyz[2 * HW + idx] = __ddiv_rn(a2, dc);
    for (int j = 0; j < c.n_nb; ++j)
        if (okbits & (1u << j)) c.nb_used[j][mark[j]] = 1;
}

static bool is_pinhole(const double* row) { return row[13] == 0.0 && row[14] == 0.0 && row[15] == 0.0; }

}  // namespace mvs

using namespace mvs;

extern "C" mvs_status mvs_consistency(const mvs_consistency_args* a, void* stream) {
    clear_error();
    if (!a) return fail(MVS_ERR_VALUE, "consistency: null arguments");
    if (a->H < 0 || a->W < 0) return fail(MVS_ERR_VALUE, "consistency: negative shape");
    if (a->n_nb < 0 || a->n_nb > MVS_MAX_SOURCES)
        return fail(MVS_ERR_VALUE, "consistency: %d neighbours (at most %d)", a->n_nb, MVS_MAX_SOURCES);
    if (a->H == 0 || a->W == 0) return MVS_OK;
    if (!a->depth || !a->cam || (a->n_nb > 0 && (!a->nb_cam || !a->rel_tol)))
        return fail(MVS_ERR_VALUE, "consistency: null pointer");
    if (!a->count && !a->active) return MVS_OK;
    if (a->active && (!a->grey || !a->score)) return fail(MVS_ERR_VALUE, "consistency: the mask needs grey and score");
    ConsParams p;
    memset(&p, 0, sizeof(p));
    p.H = a->H; p.W = a->W; p.n_nb = a->n_nb; p.min_views = a->min_views;
    p.min_ncc = (float)a->min_ncc;
    p.px_tol = a->px_tol;
    p.depth = a->depth; p.grey = a->grey; p.score = a->score;
    p.count = a->count; p.active = a->active;
    for (int k = 0; k < 18; ++k) p.cam[k] = a->cam[k];
    p.pinhole = is_pinhole(a->cam);
    for (int j = 0; j < a->n_nb; ++j) {
        if (!a->nb_depth[j]) return fail(MVS_ERR_VALUE, "consistency: null neighbour map %d", j);
        if (a->nb_h[j] < 1 || a->nb_w[j] < 1) return fail(MVS_ERR_VALUE, "consistency: empty neighbour map %d", j);
        p.nb_depth[j] = a->nb_depth[j];
        p.nb_h[j] = a->nb_h[j];
        p.nb_w[j] = a->nb_w[j];
        for (int k = 0; k < 18; ++k) p.nb_cam[18 * j + k] = a->nb_cam[18 * j + k];
        p.nb_pinhole[j] = is_pinhole(a->nb_cam + 18 * j);
        p.rel_tol[j] = a->rel_tol[j];
    }
    const long long HW = (long long)a->H * a->W;
    consistency_kernel<<<(unsigned)((HW + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p);
    return check_launch("consistency kernel");
}

extern "C" mvs_status mvs_init_normals(int32_t H, int32_t W, const float* depth, const float* ray, float* normal,
                                       void* stream) {
    clear_error();
    if (H < 0 || W < 0) return fail(MVS_ERR_VALUE, "init_normals: negative shape");
    if (H == 0 || W == 0) return MVS_OK;
    if (!depth || !ray || !normal) return fail(MVS_ERR_VALUE, "init_normals: null pointer");
    const long long HW = (long long)H * W;
    init_normals_kernel<<<(unsigned)((HW + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        H, W, depth, ray, normal);
    return check_launch("init_normals kernel");
}

extern "C" mvs_status mvs_fuse_view(const mvs_fuse_args* a, void* stream) {
    clear_error();
    if (!a) return fail(MVS_ERR_VALUE, "fuse: null arguments");
    if (a->H < 0 || a->W < 0) return fail(MVS_ERR_VALUE, "fuse: negative shape");
    if (a->n_nb < 0 || a->n_nb > MVS_MAX_SOURCES)
        return fail(MVS_ERR_VALUE, "fuse: %d neighbours (at most %d)", a->n_nb, MVS_MAX_SOURCES);
    if (a->H == 0 || a->W == 0) return MVS_OK;
    if (!a->depth || !a->used || !a->cam || !a->keep || !a->xyz || !a->count ||
        (a->n_nb > 0 && (!a->nb_cam || !a->rel_tol)))
        return fail(MVS_ERR_VALUE, "fuse: null pointer");
    FuseParams p;
    memset(&p, 0, sizeof(p));
    p.H = a->H; p.W = a->W; p.n_nb = a->n_nb; p.min_views = a->min_views;
    p.stride = a->point_stride > 1 ? a->point_stride : 1;
    p.px_tol = a->px_tol;
    p.depth = a->depth; p.used = a->used; p.keep = a->keep; p.xyz = a->xyz; p.count = a->count;
    for (int k = 0; k < 18; ++k) p.cam[k] = a->cam[k];
    p.pinhole = is_pinhole(a->cam);
    for (int j = 0; j < a->n_nb; ++j) {
        if (!a->nb_depth[j] || !a->nb_used[j]) return fail(MVS_ERR_VALUE, "fuse: null neighbour map %d", j);
        if (a->nb_h[j] < 1 || a->nb_w[j] < 1) return fail(MVS_ERR_VALUE, "fuse: empty neighbour map %d", j);
        if (a->nb_used[j] == a->used) return fail(MVS_ERR_VALUE, "fuse: neighbour %d is the view itself", j);
        p.nb_depth[j] = a->nb_depth[j];
        p.nb_used[j] = a->nb_used[j];
        p.nb_h[j] = a->nb_h[j];
        p.nb_w[j] = a->nb_w[j];
        for (int k = 0; k < 18; ++k) p.nb_cam[18 * j + k] = a->nb_cam[18 * j + k];
        p.nb_pinhole[j] = is_pinhole(a->nb_cam + 18 * j);
        p.rel_tol[j] = a->rel_tol[j];
    }
    const long long HW = (long long)a->H * a->W;
    fuse_kernel<<<(unsigned)((HW + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p);
    return check_launch("fuse kernel");
}
