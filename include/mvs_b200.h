/*
 * mvs_b200.h - C ABI of the B200 multi-view-stereo depth-map engine (libmvs_b200.so).
 *
 * Drop-in replacement for the depth-map path of pyOrthomosaic 0.9.3: the plane sweep
 * (`_dense.sweep_hypothesis`, `densify._sweep`) and the slanted-plane PatchMatch repair
 * (`_dense.pm_refine`), plus the small per-view helpers that feed them (`_fast.*`).
 *
 * Conventions (the reference's, kept on purpose):
 *   - the caller allocates every input and output; state arrays are updated in place;
 *   - images are C-contiguous row-major, pixel centres at integer coordinates;
 *   - cameras use the reference's 18-double rows (R(9, world->camera, row-major) C(3) f k1 k2 k3
 *     cx cy) or the sweep's geo rows (Rs(9) b(3) f k1 k2 k3 cx cy, b = Rs (C_ref - C_src));
 *   - every image/state pointer is a DEVICE pointer (cudaMalloc / torch CUDA tensor storage);
 *     camera rows, plane lists and other small tables are HOST pointers;
 *   - `stream` is a cudaStream_t (NULL = legacy default stream). Work is enqueued
 *     asynchronously; the call returns after launch (errors found at launch are returned).
 *   - status codes map to Python exceptions in the ctypes shim: MVS_ERR_VALUE -> ValueError,
 *     MVS_ERR_MEMORY -> MemoryError, MVS_ERR_TIMEOUT -> TimeoutError, others -> RuntimeError.
 *     mvs_last_error() returns the message of the calling thread's last failure.
 *
 * No function here falls back to the CPU.
 */
#ifndef MVS_B200_H
#define MVS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MVS_MAX_SOURCES 16
#define MVS_MAX_RADIUS 7          /* window (2r+1)^2 up to 15x15 */
#define MVS_MAX_PLANES_PER_CALL 1024

typedef enum mvs_status {
    MVS_OK = 0,
    MVS_ERR_VALUE = 1,        /* bad shapes / arguments (reference: ValueError) */
    MVS_ERR_MEMORY = 2,       /* device allocation failed (reference: MemoryError) */
    MVS_ERR_CUDA = 3,         /* CUDA launch or runtime error */
    MVS_ERR_TIMEOUT = 4,      /* a bounded device-side wait ran out */
    MVS_ERR_UNSUPPORTED = 5   /* valid request outside what this build implements */
} mvs_status;

/* Hypothesis families of the sweep. Each yields one float32 inverse depth per pixel and
 * hypothesis index i (0 <= i < n). */
typedef enum mvs_hyp_kind {
    MVS_HYP_MAPS = 0,    /* explicit maps: inv_i = maps[(i - i0) * map_stride + y * W + x]      */
    MVS_HYP_LINEAR = 1,  /* inv_i = base + (float)i * step          (_fast.hyp_linear)          */
    MVS_HYP_REFINE = 2,  /* inv_i = max(base + (float)(i + t0) * step, 1e-6f) (_fast.hyp_refine) */
    MVS_HYP_PLANES = 3   /* inv_i = planes[i], constant: fronto-parallel to the reference camera;
                            pinhole cameras only (k1 = k2 = k3 = 0); evaluated as one FP64-composed
                            homography per (plane, source, tile) instead of per-pixel rays        */
} mvs_hyp_kind;

typedef struct mvs_hyp {
    int32_t kind;            /* mvs_hyp_kind */
    int32_t n;               /* hypotheses in the whole sweep (finalize: interior test)           */
    const float* maps;       /* MAPS: device (n_maps, H, W) volume, map 0 <-> hypothesis i0       */
    int64_t map_stride;      /* MAPS: elements between consecutive maps (0 -> H * W)              */
    const float* base;       /* LINEAR / REFINE: device (H, W)                                    */
    const float* step;       /* LINEAR / REFINE: device (H, W)                                    */
    int32_t t0;              /* REFINE: offset added to i                                          */
    int32_t pad_;
    const float* planes;     /* PLANES: HOST array of n float32 inverse depths                    */
} mvs_hyp;

/* Storage precision of source images and warped tiles. */
typedef enum mvs_precision {
    MVS_PREC_FP32 = 0,      /* plain: float32 images and tiles, FP32 window sums                   */
    MVS_PREC_FP16 = 1,      /* FP16 images (src pointers are __half), FP32 window sums; PLANES only;
                               FP64 homography and parabola                                        */
    MVS_PREC_FP64_SUMS = 2, /* float32 images and tiles, window sums in float64 as the reference
                               keeps them (_sweep.h:85-178): its NCC to ~1 float32 ulp even on
                               bright low-texture windows, where FP32 sums differ by up to ~1e-3;
                               single-view calls (mvs_sweep*) only, slower stages B and C        */
    MVS_PREC_FP32_COMP = 3, /* compensated FP32 window sums: reference and warped values shifted by
                               one pivot per tile (the tile's mean reference value), vertical sums
                               of the variance / covariance terms with Kahan compensation, and the
                               reference window statistics formed from the pivoted tile (the `mu`
                               and `sd` arguments are not read). Closer to an all-float64 sweep than
                               the reference's own float32 statistics; PLANES, top_k <= 2,
                               single-view calls only                                              */
    MVS_PREC_FP16_COMP = 4  /* MVS_PREC_FP32_COMP with FP16 source storage (src are __half)        */
} mvs_precision;

typedef struct mvs_sweep_args {
    int32_t H, W;                          /* reference image                                   */
    const float* ref;                      /* (H, W) grey, masked pixels already 0              */
    const float* mu;                       /* (H, W) zero-padded window mean of ref             */
    const float* sd;                       /* (H, W) window standard deviation of ref           */
    const float* ray;                      /* (3, H, W) world rays; NULL allowed for PLANES     */
    int32_t n_src;                         /* 1 .. MVS_MAX_SOURCES                              */
    int32_t precision;                     /* mvs_precision                                     */
    const void* src[MVS_MAX_SOURCES];      /* (src_h[s], src_w[s]) images, NaN = masked         */
    int32_t src_h[MVS_MAX_SOURCES];
    int32_t src_w[MVS_MAX_SOURCES];
    const double* geo;                     /* HOST (n_src, 18): Rs(9) b(3) f k1 k2 k3 cx cy     */
    const double* ref_cam;                 /* HOST 18: R(9) C(3) f k1 k2 k3 cx cy (PLANES only) */
    mvs_hyp hyp;
    int32_t i0, i1;                        /* hypotheses [i0, i1) are swept by this call        */
    int32_t r;                             /* window radius, 0 .. MVS_MAX_RADIUS                */
    int32_t top_k;                         /* score = mean of the best top_k source NCCs        */
    int32_t plane_chunks;                  /* 0 = automatic; else CTAs per tile along planes   */
    int32_t tile_h;                        /* output tile rows: 0 (= 32), 16, 32 or 64; tiles are
                                              64 columns wide. 16 and 64: FP32 / FP16 PLANES
                                              sweeps with top_k <= 2 (other forms: 0 or 32)      */
    float* best;                           /* (H, W) in/out winner-take-all state               */
    float* prev;
    float* s_prev_best;
    float* s_next_best;
    int32_t* idx;
} mvs_sweep_args;

/* ---------------------------------------------------------------- plane sweep */

/* Multi-hypothesis plane sweep: hypotheses [i0, i1) of `hyp` for every source, streaming
 * winner-take-all state update (same per-hypothesis semantics as sweep_hypothesis, applied in
 * hypothesis order). Replaces the hypothesis loop of densify._sweep (densify.py:336-342).
 * Plane chunks that run in parallel are merged in hypothesis order (first index wins ties).
 * Needs device scratch when plane_chunks > 1 (allocated stream-ordered per call). */
mvs_status mvs_sweep(const mvs_sweep_args* args, void* stream);

/* mvs_sweep for callers that cannot allocate device memory - a process whose device memory is
 * owned by another allocator with a fixed budget, or a latency-critical loop that must not enter
 * the driver's allocator (cudaMalloc can synchronise the device). No counterpart in the
 * reference (its CPU kernel mallocs per call). Same arguments and results as mvs_sweep, but the
 * plane-chunk scratch is one 32 MiB file-scope device array per GPU, held until the process
 * exits: with plane_chunks = 0 the chunk count is lowered until the records fit; an explicit
 * plane_chunks whose records (6 floats per pixel per chunk) exceed 32 MiB gives MVS_ERR_VALUE.
 * Every call looks the array's address up on the current device; the first call on a device
 * (and the first after its context was reset) loads the array there: make it before any stream
 * capture. All calls share the array and it keeps the last call's contents (none of
 * it needs to start at zero); calls that overlap on the GPU race on it. Calls no cudaMalloc,
 * cudaFree or other allocating routine. */
mvs_status mvs_sweep_noalloc(const mvs_sweep_args* args, void* stream);

/* One hypothesis `i` given as an explicit inverse-depth map `inv` (H, W), ray-grid geometry
 * with radial distortion. Replaces _dense.sweep_hypothesis (_dense.pyx:740-838); argument
 * order and meaning as there (srcs: n_src device pointers with their shapes). */
mvs_status mvs_sweep_hypothesis(int32_t H, int32_t W, const float* ref, const float* mu_i,
                                const float* sd_i, int32_t n_src, const float* const* srcs,
                                const int32_t* src_h, const int32_t* src_w, const float* ray,
                                const double* geo, const float* inv, int32_t r, int32_t top_k,
                                int32_t i, float* best, float* prev, float* s_prev_best,
                                float* s_next_best, int32_t* idx, void* stream);

/* Sub-hypothesis parabola and depth (camera-axis metres) from the winner-take-all state:
 * den = spb - 2 best + snb; interior = 0 < idx < n-1 and den < -1e-6;
 * off = clip(0.5 (spb - snb) / den, +-0.5); inv = inv_0 + (idx + off) (inv_1 - inv_0);
 * depth = 1 / max(inv, 1e-9). Replaces densify.py:354-361 (same float32 / float64 steps). */
mvs_status mvs_sweep_finalize(int32_t H, int32_t W, const mvs_hyp* hyp, const float* best,
                              const float* s_prev_best, const float* s_next_best,
                              const int32_t* idx, float* depth, void* stream);

/* ---------------------------------------------------------------- per-view helpers */

/* Zero-padded (2r+1)^2 window mean with float32 cumulative sums (columns, then rows), times
 * float32(1/(2r+1)^2). Bit-identical to _fast.box_zero_mean (_fast.pyx:661-713). When
 * `square` != 0 the input is a*a (float32), i.e. densify._box(ref * ref, r). */
mvs_status mvs_box_zero_mean(int32_t H, int32_t W, const float* a, int32_t r, int32_t square,
                             float* out, void* stream);

/* mu = box(ref), sd = sqrt(max(box(ref*ref) - mu*mu, 1e-6)) in float32 (densify.py:327-328). */
mvs_status mvs_ref_stats(int32_t H, int32_t W, const float* ref, int32_t r, float* mu, float* sd,
                         void* stream);

/* World ray grid (3, H, W) float32 of a camera row R(9) C(3) f k1 k2 k3 cx cy: 8 fixed-point
 * undistortion iterations in float64, then R^T (x, y, 1). Replaces densify._rays_world with
 * _fast.rays_grid (densify.py:288-297, _fast.pyx:145-198). */
mvs_status mvs_rays_grid(int32_t H, int32_t W, const double* cam, float* ray, void* stream);

/* out = base + (float)i * step in float32 (_fast.hyp_linear, _fast.pyx:628-641). */
mvs_status mvs_hyp_linear(int32_t H, int32_t W, const float* base, const float* step, int64_t i,
                          float* out, void* stream);

/* out = max(iu + (float)t * ds, 1e-6f), NaN propagating (_fast.hyp_refine, _fast.pyx:644-658). */
mvs_status mvs_hyp_refine(int32_t H, int32_t W, const float* iu, const float* ds, int64_t t,
                          float* out, void* stream);

/* uint8 RGB (h, w, 3) -> grey ((mean - 128) / 64, NaN where mask == 0) and clip(rgb+.5) uint8,
 * with optional per-channel gain / bias (host float[3] or NULL) and mask (device uint8 or NULL).
 * Replaces _fast.depth_view (_fast.pyx:577-624). */
mvs_status mvs_depth_view(int32_t h, int32_t w, const uint8_t* rgb, const float* gain,
                          const float* bias, const uint8_t* mask, float* grey, uint8_t* rgb8,
                          void* stream);

/* 2x2 mean pyramid step of `planes` stacked (h, w) float32 images: out (planes, h/2, w/2) =
 * ((a00 + a10 + a01 + a11) * 0.25) in float32 (densify._half, densify.py:127-130; the ray
 * pyramid at densify.py:398-403 is the same with planes = 3). */
mvs_status mvs_half(int32_t planes, int32_t h, int32_t w, const float* in, float* out,
                    void* stream);

/* Camera-axis depth of every tie point that lands inside a view: X (n, 3) world points (device),
 * `cam` a HOST camera row R(9) C(3) f k1 k2 k3 cx cy, pinhole map u = f x / z + cx, v = f y / z + cy;
 * out[i] = z_i where z_i > 0, 0 <= u < w and 0 <= v < h, else NaN (device, float64). The census
 * of densify._depth_range (densify.py:208-230; the host takes its percentiles), float64 in the
 * reference's NumPy / BLAS rounding order. */
mvs_status mvs_tie_depths(int32_t n, const double* X, const double* cam, int32_t w, int32_t h, double* out,
                          void* stream);

#define MVS_BAND_MIN_POINTS 50    /* fewer observed tie points: the band is the view's whole range */

typedef struct mvs_depth_band_args {
    int32_t H, W;                          /* sweep image (the coarse pyramid level)            */
    int32_t block;                         /* cell side in pixels                               */
    int32_t n_pts;                         /* tie points the view observes                      */
    const double* X;                       /* DEVICE (n_pts, 3) world points                    */
    const double* cam;                     /* HOST 18: the view's camera row at this level      */
    double lo, hi;                         /* the view's depth range (metres)                   */
    double margin;                         /* metres added on each side of a cell's range       */
    int32_t nd, pad_;                      /* hypotheses of the sweep over the band             */
    float* base;                           /* out (H, W): 1 / hi_px, inverse depth of hyp. 0   */
    float* step;                           /* out (H, W): (1 / max(lo_px, 1e-6) - base) / max(nd - 1, 1) */
    float* inv_hi;                         /* out (H, W) 1 / max(lo_px, 1e-6), or NULL          */
} mvs_depth_band_args;

/* Per-pixel inverse-depth band of the coarse sweep from the tie points the view observes, and
 * the linear hypothesis maps over it (densify._depth_band, densify.py:233-274, and the step map
 * of densify.depth_map, :409-411): the points are scattered into block x block cells (count,
 * min and max depth); a cell with >= 5 points takes the extent of its 3 x 3 neighbourhood's
 * counted cells, widened by margin + 5 % and clipped to [lo, hi]; other cells (and every cell
 * when n_pts < MVS_BAND_MIN_POINTS) take [lo, hi]. Bit-identical to the reference's NumPy
 * values. Allocates its cell table stream-ordered. */
mvs_status mvs_depth_band(const mvs_depth_band_args* args, void* stream);

/* float32 -> FP16 image conversion for MVS_PREC_FP16 sources (round to nearest; NaN kept). */
mvs_status mvs_to_fp16(int64_t n, const float* in, void* out_half, void* stream);

/* ---------------------------------------------------------------- PatchMatch */

/* Arithmetic of the PatchMatch cost. */
typedef enum mvs_pm_precision {
    MVS_PM_FP64 = 0,     /* the reference's float64 cost, operation for operation: bit-identical
                            results to a sequential evaluation with the same draws               */
    MVS_PM_FP32 = 1      /* window samples and sums in float32, one float64-composed local
                            homography per candidate and source (pinhole sources; otherwise as
                            MVS_PM_FP64); the lanes of a pixel group evaluate its sources in
                            parallel. Costs differ from float64 by ~1e-7, so near-ties (candidates
                            whose costs differ by less) can be decided differently              */
} mvs_pm_precision;

typedef struct mvs_pm_args {
    int32_t H, W;
    const float* ref;                      /* (H, W) grey, NaN = masked                         */
    const float* ray;                      /* (3, H, W) world rays                              */
    const double* Cr;                      /* HOST (3) reference camera centre                  */
    int32_t S;                             /* sources, 1 .. MVS_MAX_SOURCES (else no-op, 0)     */
    int32_t precision;                     /* mvs_pm_precision (0 = MVS_PM_FP64)                */
    const float* src[MVS_MAX_SOURCES];     /* (src_h, src_w) float32 images                     */
    const float* src_depth[MVS_MAX_SOURCES]; /* same shapes or NULL (no geometric term)         */
    int32_t src_h[MVS_MAX_SOURCES];
    int32_t src_w[MVS_MAX_SOURCES];
    const double* par;                     /* HOST (S, 18): R(9) C(3) f k1 k2 k3 cx cy          */
    float* depth;                          /* (H, W) in/out                                     */
    float* normal;                         /* (3, H, W) in/out, world frame, facing the camera  */
    float* score;                          /* (H, W) in/out                                     */
    const uint8_t* active;                 /* (H, W) pixels to re-estimate                      */
    int32_t r, step, top_k, iters;
    double geo_w, geo_tol, dmin, dmax;
    uint32_t seed;
    int32_t it0;                           /* first iteration index (resumable jobs), usually 0;
                                              sets the trial scales 0.05 / (it0 + it + 1) and
                                              0.3 / (it0 + it + 1)                              */
    int64_t* changed;                      /* DEVICE int64 counter, incremented (may be NULL)   */
    uint32_t* rng_state;                   /* DEVICE uint32 or NULL: the xorshift32 state of the
                                              random trials' stream. NULL: the stream starts at
                                              seed | 1, as the reference's pm_refine does per
                                              call. Otherwise it starts at *rng_state and the
                                              state after the call is written back, so a job
                                              split over calls (it0) draws what one call would
                                              (initialise it to seed | 1)                       */
} mvs_pm_args;

/* Red-black slanted-plane PatchMatch (_dense.pm_refine, _dense.pyx:566-666). Same cost,
 * propagation pattern, trial scales and acceptance rule, and the reference's own random stream:
 * one xorshift32 sequence (_dense.pyx:559-563) from which every active pixel whose depth is
 * finite after propagation takes 8 draws in raster order, colour pass after colour pass. Each
 * pass runs propagation for all its pixels in parallel, counts the drawing pixels (a prefix sum
 * in raster order) and jumps the stream to each pixel's offset (GF(2) matrix powers), then runs
 * the trials in parallel. With MVS_PM_FP64 the result is bit-identical to the reference's.
 * Scratch (about 21 bytes per pixel, plus 16 per pixel when iters > 1, plus 16 per source pixel
 * with MVS_PM_FP32: each source's 2 x 2 bilinear footprints, one 16-byte load per sample) is
 * allocated stream-ordered per call. */
mvs_status mvs_pm_refine(const mvs_pm_args* args, void* stream);

/* The xorshift32 state after n steps of the PatchMatch stream from `state` (host; jump-ahead by
 * GF(2) matrix powers, n up to 2^64 - 1). mvs_pm_refine's trials use the same jumps. */
uint32_t mvs_pm_stream_advance(uint32_t state, uint64_t n);

/* ---------------------------------------------------------------- batched sweep */

typedef struct mvs_batch_job {
    mvs_sweep_args sweep;                  /* hyp must be MVS_HYP_PLANES (one view = one job)   */
    float* depth;                          /* (H, W) output of the fused finalize, or NULL     */
} mvs_batch_job;

typedef struct mvs_batch_tuning {
    int32_t plane_chunk;                   /* planes per work item (0 = autotuned)             */
    int32_t ctas_per_sm;                   /* persistent CTAs per SM (0 = occupancy maximum)  */
    int32_t tile_h;                        /* rows of the plan's 64-column output tiles: 0 (= 32),
                                              16, 32 or 64 (16 and 64: top_k <= 2 in every job);
                                              the jobs' own mvs_sweep_args.tile_h is not read    */
} mvs_batch_tuning;

typedef struct mvs_batch mvs_batch;        /* opaque: device work list, job table, graph       */

/* Build a persistent batched plan over `n_jobs` views (uneven sizes, source and plane counts,
 * radii). All device tables are allocated here; mvs_batch_run then only launches. */
mvs_status mvs_batch_create(const mvs_batch_job* jobs, int32_t n_jobs,
                            const mvs_batch_tuning* tuning, mvs_batch** out);
/* Run every job: one persistent launch over all (job, tile, plane-chunk) work items, then the
 * ordered chunk merge and the finalize; captured once into a CUDA graph and replayed. */
mvs_status mvs_batch_run(mvs_batch* b, int32_t use_graph, void* stream);
/* Number of work items and ZNCC evaluations (pixel x plane x source) in the plan. */
mvs_status mvs_batch_stats(const mvs_batch* b, int64_t* work_items, int64_t* evals);
void mvs_batch_destroy(mvs_batch* b);

/* ---------------------------------------------------------------- continuous batching */

/* A serving engine: a device table of `max_slots` resident jobs (MVS_HYP_PLANES sweeps) and a
 * work-item buffer. Each step runs the next plane chunk of any set of resident jobs - all their
 * tiles - in ONE persistent launch, then merges each chunk into that job's winner state in
 * hypothesis order. Jobs join and leave between steps; a job's result does not depend on which
 * other jobs share its steps. */
typedef struct mvs_server mvs_server;

mvs_status mvs_server_create(int32_t max_slots, int32_t max_items, int32_t max_radius, int32_t precision,
                             mvs_server** out);
/* Installs `job` in `slot`: its images, state arrays (initialised by the caller to the sweep's
 * initial state) and hypotheses stay where the caller put them; `chunk_rec` is a device buffer
 * of 6 * H * W floats for one chunk record; planes are processed `plane_chunk` at a time. */
mvs_status mvs_server_set_job(mvs_server* s, int32_t slot, const mvs_sweep_args* job, float* chunk_rec,
                              int32_t plane_chunk);
/* Runs chunk chunks[k] of the job in slots[k], for k < n, in one launch and merges them. */
mvs_status mvs_server_step(mvs_server* s, const int32_t* slots, const int32_t* chunks, int32_t n, void* stream);
void mvs_server_destroy(mvs_server* s);

/* ---------------------------------------------------------------- pass 2: geometric check */

/* Camera rows here and in mvs_pm_args.par: R (9, world -> camera), C (3), f, k1, k2, k3, cx, cy. */
typedef struct mvs_consistency_args {
    int32_t H, W;
    const float* depth;                    /* (H, W) the view's pass-1 depth map, NaN = none    */
    const double* cam;                     /* host, 18 doubles: the view's camera row           */
    int32_t n_nb, pad_;
    const float* nb_depth[MVS_MAX_SOURCES];   /* neighbours' pass-1 depth maps (device)         */
    int32_t nb_h[MVS_MAX_SOURCES], nb_w[MVS_MAX_SOURCES];
    const double* nb_cam;                  /* host, n_nb x 18 camera rows                       */
    const double* rel_tol;                 /* host, n_nb relative depth tolerances              */
    double px_tol;                         /* forward-backward reprojection tolerance, pixels   */
    int16_t* count;                        /* out (H, W) agreeing neighbours, or NULL           */
    const float* grey;                     /* (H, W) grey (NaN = masked), or NULL: no mask      */
    const float* score;                    /* (H, W) pass-1 NCC score                           */
    double min_ncc;                        /* compared in float32                               */
    int32_t min_views, pad2_;
    uint8_t* active;                       /* out (H, W) PatchMatch selection, or NULL          */
} mvs_consistency_args;

/* Replaces densify._consistency (densify.py:441-478, with _fast.ref_points / neighbour_sample /
 * agreement, _fast.pyx:201-268): per finite pixel, the number of neighbours whose depth map
 * agrees under forward-backward reprojection. With `grey`, also pass 2's PatchMatch mask
 * (densify.py:621): finite(grey) & (count < min_views - 1 | score < min_ncc | !finite(depth)).
 * Bit-exact with the reference, whose 3 x 3 products NumPy evaluates as fused multiply-add
 * chains (a = m0 r0; a = fma(m1, r1, a); a = fma(m2, r2, a)). */
mvs_status mvs_consistency(const mvs_consistency_args* args, void* stream);

/* Replaces densify._init_normals (densify.py:481-496): (3, H, W) float32 world normals of a depth
 * map from 2-px central differences, (0, 0, 1) where undefined, facing the camera. Bit-exact. */
mvs_status mvs_init_normals(int32_t H, int32_t W, const float* depth, const float* ray, float* normal,
                            void* stream);

/* ---------------------------------------------------------------- pass 3: point fusion */

typedef struct mvs_fuse_args {
    int32_t H, W;
    const float* depth;                    /* (H, W) the view's final depth map, NaN = none     */
    const uint8_t* used;                   /* (H, W) the view's used mask (read)                */
    const double* cam;                     /* host, 18 doubles: the view's camera row           */
    int32_t n_nb;                          /* neighbours with a depth map, in the view's order  */
    int32_t point_stride;                  /* candidates on the stride grid (<= 1: every pixel) */
    const float* nb_depth[MVS_MAX_SOURCES];
    uint8_t* nb_used[MVS_MAX_SOURCES];     /* neighbours' used masks (written: 1 where marked)  */
    int32_t nb_h[MVS_MAX_SOURCES], nb_w[MVS_MAX_SOURCES];
    const double* nb_cam;                  /* host, n_nb x 18 camera rows                       */
    const double* rel_tol;                 /* host, n_nb relative depth tolerances              */
    double px_tol;                         /* forward-backward reprojection tolerance, pixels   */
    int32_t min_views, pad_;
    uint8_t* keep;                         /* out (H, W): 1 = the pixel emits a fused point     */
    double* xyz;                           /* out (3, H, W) float64 fused point where keep      */
    int32_t* count;                        /* out (H, W) agreeing views + 1 (0 = no candidate)  */
} mvs_fuse_args;

/* One reference image of the point fusion (densify._fuse_loop, densify.py:688-762, on the
 * compiled path _fast.ref_points / neighbour_sample / agreement / accumulate,
 * _fast.pyx:201-284): candidates are the finite pixels not yet used, on the stride grid; each
 * accumulates the back-projected points of the neighbours that pass the forward-backward check
 * (in neighbour order) onto its own, is kept with at least min_views views (xyz = sum / count)
 * and marks the agreeing neighbours' stride-grid pixels as used. Views must be fused one call
 * after another in the reference's order (sorted view index) on one stream. Bit-exact. */
mvs_status mvs_fuse_view(const mvs_fuse_args* args, void* stream);

/* ---------------------------------------------------------------- legacy height sweep (mvs.py) */

typedef struct mvs_sample_view_args {
    int32_t h, w, nch;                     /* image (h, w, nch) float32, device                 */
    const float* img;
    const double* cam;                     /* host, 18 doubles: R(9) C(3) f k1 k2 k3 cx cy, in
                                              the pixel units of img                            */
    double X0, Y0, gsd;                    /* grid: cell (r, c) at (X0 + (c+.5) gsd, Y0 - (r+.5) gsd) */
    int32_t D, H, W;                       /* heights Z (D, H, W) float32, device               */
    const float* Z;
    float* out;                            /* out (D, H, W, nch) float32: 0 where not valid     */
    uint8_t* valid;                        /* out (D, H, W)                                     */
} mvs_sample_view_args;

/* Projects a ground grid at per-cell heights into a view and samples it bilinearly (float64 as
 * the reference's CPU sampler). Replaces _mvs.sample_view (_mvs.pyx:13-58) / the CuPy kernel
 * sample_view (_cuda.py:88-124) behind backend.sample_view. Bit-exact with _mvs.sample_view. */
mvs_status mvs_sample_view(const mvs_sample_view_args* args, void* stream);

/* Float64 summed-area (2r+1)^2 window mean with zero padding of B stacked (H, W) float32 planes.
 * Replaces _fast.box_sat_mean (_fast.pyx:897-942), the CPU backend's box (backend.py:102-114).
 * Bit-exact. Allocates its table stream-ordered. */
mvs_status mvs_box_sat_mean(int32_t B, int32_t H, int32_t W, const float* a, int32_t r, float* out, void* stream);

typedef struct mvs_height_score_args {
    int32_t V, D, H, W;                    /* views (2..16), hypothesis stack (D, H, W)         */
    int32_t topk;                          /* mean of the topk largest NCCs                     */
    int32_t pad_;
    double full, min_texture, full_texture;   /* compared / divided in float32, as NumPy does  */
    const float* M;                        /* (V, D, H, W) box(S)                               */
    const float* S2;                       /* (V, D, H, W) box(S * S)                           */
    const float* VA;                       /* (V, D, H, W) box(valid)                           */
    const float* PP;                       /* (V(V-1)/2, D, H, W) box(S_a S_b), np.triu_indices */
    const float* cxs;                      /* (W) float32 cell-centre X                         */
    const float* cys;                      /* (H) float32 cell-centre Y                         */
    const double* cam_xy;                  /* host, V x 2 camera centres (X, Y)                 */
    float* score;                          /* out (D, H, W)                                     */
    float* st;                             /* out (V, D, H, W) NCC vs the cell's reference, or NULL */
    int32_t* ref;                          /* out (D, H, W) reference view, or NULL             */
} mvs_height_score_args;

/* The photo-consistency of every hypothesis cell (mvs.dense_reconstruct's score_at,
 * mvs.py:254-304) after the sampling and the box means: nearest fully-valid camera as the cell's
 * reference, NCC of every other view against it, mean of the topk largest (summed in descending
 * order), times the reference's texture weight. */
mvs_status mvs_height_score(const mvs_height_score_args* args, void* stream);

/* Semi-global aggregation of a (D, H, W) float32 cost volume along 8 directions, summed in the
 * reference's direction order. Replaces _mvs.sgm (_mvs.pyx:98-251); bit-exact. */
mvs_status mvs_sgm(int32_t D, int32_t H, int32_t W, const float* cost, float P1, float P2, float* agg,
                   void* stream);

/* ---------------------------------------------------------------- misc */

/* Device-side waits that gave up since the last call (the sweep's TMA copy of the reference
 * tile waits on an mbarrier with an iteration limit; a tile whose copy never completes leaves its
 * state untouched and is counted here). Synchronises with the device; clears the count.
 * Returns MVS_ERR_TIMEOUT when the count was non-zero. No counterpart in the reference. */
mvs_status mvs_device_faults(uint32_t* count);

/* Iterations of the sweep's bounded wait for its reference-tile copy (default 2^20 try_wait
 * iterations, far above a copy's latency); returns the previous value. For tests of the give-up
 * path: with 0 every tile gives up at once - it counts a fault, waits (with the default bound)
 * for its copy in flight to land and returns with its state untouched. Applies to calls made
 * after it, from any thread. No counterpart in the reference. */
uint32_t mvs_set_wait_limit(uint32_t iterations);

/* Bounds-checked debug build only (libmvs_b200_debug.so, compiled with MVS_DEBUG_BOUNDS): the
 * number of shared-memory and global indices the tile engine, the batched kernels and PatchMatch
 * used outside their buffers since the last call (synchronises; clears the counts). Release
 * builds return MVS_ERR_UNSUPPORTED. No counterpart in the reference (its Cython kernels are
 * compiled with boundscheck=False). */
mvs_status mvs_debug_bound_violations(uint32_t* count);

/* Message of this thread's last failing call ("" if none). Returns the message length. */
size_t mvs_last_error(char* buf, size_t cap);
/* Library version string. */
const char* mvs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MVS_B200_H */
