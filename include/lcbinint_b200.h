/*
 * lcbinint_b200 -- C ABI of the B200 implementation of lcbinint's
 * magnification hot path (binary-lens point-source and finite-source
 * magnification).  Plain pointers and sizes only; no C++ or torch types.
 *
 * Every entry point names the reference interface it replaces
 * (NunotaKansuke/lcbinint, file:line).  Arrays are host pointers unless the
 * call's `flags` include LCBI_GPU_DEVICE_POINTERS, in which case every array
 * argument of that call is a device pointer on the context's device.  Calls
 * are synchronous with respect to the host unless documented otherwise, and
 * a context may be used by one host thread at a time; distinct contexts are
 * independent (no global mutable state).
 */
#ifndef LCBININT_B200_H
#define LCBININT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef LCBININT_H
/* Status codes, same names and values as include/lcbinint/lcbinint.h:8-13. */
typedef enum lcbi_status {
    LCBI_OK = 0,
    LCBI_INVALID_ARGUMENT = 1,
    LCBI_NUMERICAL_ERROR = 2,
    LCBI_UNSUPPORTED = 3
} lcbi_status;
#endif

/* Extra status returned by the GPU calls only. */
#define LCBI_GPU_ERROR 16

/* flags */
#define LCBI_GPU_DEVICE_POINTERS 1u

typedef struct lcbi_gpu_context lcbi_gpu_context;

/* Creates a context on CUDA device `device` with its own stream and device
 * workspace.  No reference counterpart: the reference keeps per-thread state
 * in thread_local caches (python/lcbinint_pybind.cpp:927-943). */
int lcbi_gpu_create(int device, lcbi_gpu_context **ctx);
void lcbi_gpu_destroy(lcbi_gpu_context *ctx);
/* Message of the last failed call on this context ("" if none). */
const char *lcbi_gpu_last_error(const lcbi_gpu_context *ctx);
/* Number of kernels this context has launched (instrumentation). */
int64_t lcbi_gpu_launch_count(const lcbi_gpu_context *ctx);
/* Device bytes the context's workspaces hold now (they grow with the batches
 * and are kept for the next call; no reference counterpart). */
int64_t lcbi_gpu_workspace_bytes(lcbi_gpu_context *ctx);
/* The compute capability the library's device code was built for, as the
 * driver reports it for the current device (cudaFuncAttributes::binaryVersion,
 * 100 for sm_100a); LCBI_GPU_ERROR when no device can run it.  No reference
 * counterpart. */
int lcbi_gpu_kernel_binary_version(int32_t *version);
/* Runs the context's work on a caller's cudaStream_t (NULL: the context's own
 * stream), so callers can order and time it with their own events. */
int lcbi_gpu_set_stream(lcbi_gpu_context *ctx, void *cuda_stream);
/* Enables (and resets) per-stage kernel timing with CUDA events. */
int lcbi_gpu_set_timing(lcbi_gpu_context *ctx, int enable);
/* Accumulated device milliseconds and launch counts per stage since timing was
 * enabled: 0 caustics + limb-darkening tables, 1 decision, 2 seeding,
 * 3 Cartesian inverse ray, 4 polar inverse ray, 5 point source. */
int lcbi_gpu_stage_times(const lcbi_gpu_context *ctx, double *ms, int64_t *launches, int32_t n);
/* Enables stream marks (instrumentation, no reference counterpart): every
 * finite-source call records timing events where its inverse-ray streams end,
 * without changing how they overlap. */
int lcbi_gpu_set_stream_marks(lcbi_gpu_context *ctx, int enable);
/* Device milliseconds from the start of the last call's seeding stage to the
 * end of, in order, the early stream (the largest Cartesian points' seeding
 * and block pass), the side stream (the first and second Cartesian passes and
 * its blocks' share of the early pass) and the context's stream (the polar
 * passes); -1 for a stream that did not run.  n entries (at most 3) are
 * written.  Waits for the call's work to finish. */
int lcbi_gpu_stream_marks(lcbi_gpu_context *ctx, double *ms, int32_t n);
/* Enables per-point clock64 cycle counts of seeding + inverse-ray integration
 * (instrumentation, read back with lcbi_gpu_last_item_cycles). */
int lcbi_gpu_set_item_cycles(lcbi_gpu_context *ctx, int enable);
int lcbi_gpu_last_item_cycles(lcbi_gpu_context *ctx, int64_t n, int64_t *cycles);
/* Load balance of the finite-source scans (no reference counterpart): a point
 * whose Cartesian or polar scan passes `cells` lattice cells on its one warp
 * is moved to a second pass that runs it on a whole block with a larger
 * scratch.  0 disables the move (points then change pass only when they
 * outgrow the per-warp scratch); the default is 524288, and 1 (every point on
 * a block) for calls of at most 4 points per SM until this is called.  Results
 * are the same for every value. */
int lcbi_gpu_set_cell_budget(lcbi_gpu_context *ctx, int64_t cells);
/* Seeding of inverse-ray points (no reference counterpart): a point whose
 * caustic-crossing phase scan reaches `sources` critical-curve source points
 * inside its disk (each probed with up to 88 lens-equation solves) is seeded
 * again by a pass that gives each such point a whole block and probes eight
 * critical sources at a time.  0 keeps every point on its one warp; the
 * default is 32.  The seeds, and so the results, are the same for every
 * value. */
int lcbi_gpu_set_seed_block_after(lcbi_gpu_context *ctx, int32_t sources);
/* Precision of the inverse-ray lens map (no reference counterpart; the
 * reference maps every cell in FP64).  64 (the default): the reference's FP64
 * map, bit-exact.  32: each Cartesian scan maps its cells in FP32 about its
 * seed, and each polar tile column about its middle radius -- the map at the
 * anchor in FP64 plus the difference to the cell in FP32, so the rounding is
 * relative to the cell's offset from the anchor -- while every sum stays
 * FP64.  Cells within about 1e-7 rho of the source's limb can change sides, so
 * magnifications differ from the FP64 ones by ~1e-7 relative, the limb-darkening
 * table index by a few 1e-3 of a step.  Seeds, decisions and the start cells
 * stay FP64. */
int lcbi_gpu_set_ray_precision(lcbi_gpu_context *ctx, int32_t bits);

/* Polar inverse ray in the first pass: 1 (default) the tile-parallel flood
 * fill spread over the whole GPU, 0 the one-warp-per-point segment flood fill.
 * Both count the same cells; results are the same.  No reference counterpart. */
int lcbi_gpu_set_polar_tiles(lcbi_gpu_context *ctx, int enable);
/* Load balance of the largest Cartesian points (no reference counterpart):
 * with 1 (the default), once the first and second Cartesian passes have
 * finished, their stream's blocks join the early block pass of the points
 * predicted largest and take the units it has not started; 0 leaves that
 * pass to its own blocks.  Results are the same for both values. */
int lcbi_gpu_set_early_helpers(lcbi_gpu_context *ctx, int enable);
/* Device workspace of the finite-source scans (no reference counterpart):
 * first-pass warps per SM (default 8; about 7 MB of scratch each), second-pass
 * blocks (default 0: one per SM; about 100 MB each; a number set here also
 * sets the early pass of the largest Cartesian points to as many blocks, at
 * least 2 and at most 96, of 40 MB each, with 32 unit row areas of 2.5 MB per
 * block, at most 256) and the polar tile table's
 * capacity (a power of two, default 1048576 tiles of 400 B).  Smaller values
 * trade speed for memory; results do not change.  A value <= 0 keeps the
 * current setting, except second-pass blocks, where 0 means one per SM. */
int lcbi_gpu_set_workspace(lcbi_gpu_context *ctx, int32_t warps_per_sm, int32_t second_pass_blocks,
                           int64_t tile_capacity);
/* Device-measured FP64 fused-multiply-add throughput of this GPU in TFLOP/s
 * (2 flop per FMA), the denominator of the FP64 roofline; no reference counterpart. */
int lcbi_gpu_measure_fp64_peak(lcbi_gpu_context *ctx, double *tflops);

/* Point-source magnification of n source positions.
 * Replaces PointSourceMagnifier::binary_mag0
 * (src/lcbinint/magnification/point_source_magnifier.cpp:652-693) and the
 * Python free function lcbinint.binary_mag0 (python/lcbinint_pybind.cpp:3819-3824):
 * separation s, mass ratio q in the core convention (q < 1: heavier lens at -s;
 * q > 1 is inverted), source (y1, y2) in the centre-of-mass frame.
 * Outputs A[n] and, if not NULL, image_count[n] (3 or 5) and status[n]
 * (LCBI_OK, or LCBI_NUMERICAL_ERROR with A = NaN when the source sits exactly
 * on the lighter lens, where the reference's solver does not terminate). */
int lcbi_gpu_binary_mag0(lcbi_gpu_context *ctx, int64_t n, const double *s, const double *q,
                         const double *y1, const double *y2, double *A, int32_t *image_count,
                         int32_t *status, unsigned flags);

/* Point-source magnification summed over the physical images of
 * PointSourceMagnifier::binary_images
 * (src/lcbinint/magnification/point_source_magnifier.cpp:723-778), in their
 * order, as LensModel forms it (src/lcbinint/model/lens_model.cpp:209-216);
 * image_count = number of those images (0 when s == 0 or q <= 0).  This can
 * differ from lcbi_gpu_binary_mag0 in the last bits (another root selection). */
int lcbi_gpu_binary_images_mag(lcbi_gpu_context *ctx, int64_t n, const double *s, const double *q,
                               const double *y1, const double *y2, double *A, int32_t *image_count,
                               unsigned flags);

/* The five image candidates of PointSourceMagnifier::binary_image_candidates
 * (src/lcbinint/magnification/point_source_magnifier.cpp:739-778), sorted by
 * residual, for n source positions (the conventions of lcbi_gpu_binary_mag0).
 * candidates[20 i + 4 k ...] = {x, y, jacobian determinant, sqrt residual} of
 * candidate k of position i, in the frame of the lens-equation roots;
 * n_physical[i] = how many lead the list as physical images (3 or 5;
 * PointSourceMagnifier::binary_images keeps those).  n_physical[i] = 0 (and
 * position i's records untouched) when s == 0 or q <= 0, where the reference
 * returns no candidate; -1 when the source sits exactly on the lighter lens,
 * where the reference's solver does not terminate. */
int lcbi_gpu_binary_image_candidates(lcbi_gpu_context *ctx, int64_t n, const double *s, const double *q,
                                     const double *y1, const double *y2, double *candidates,
                                     int32_t *n_physical, unsigned flags);

/* Point-source magnification plus the smoothness indicator the finite-source
 * decision tree uses.  Replaces PointSourceMagnifier::binary_mag0_with_derivatives
 * (src/lcbinint/magnification/point_source_magnifier.cpp:583-611). */
int lcbi_gpu_binary_mag0_derivatives(lcbi_gpu_context *ctx, int64_t n, const double *s,
                                     const double *q, const double *y1, const double *y2,
                                     double *A, int32_t *image_count, double *indicator,
                                     unsigned flags);

/* ------------------------------------------------------------------ */
/* Finite source                                                       */
/* ------------------------------------------------------------------ */

/* FiniteSourceSettings (src/lcbinint/magnification/finite_source_magnifier.hpp:22-38). */
typedef struct lcbi_fs_settings {
    int32_t source_bins;             /* nbin: cells per source radius */
    int32_t caustic_bins;            /* caustic phase samples (>= 32 used) */
    double grid_ratio;
    int32_t polar_source_bins;       /* 0: use source_bins */
    double polar_grid_ratio;         /* <= 0: use grid_ratio */
    int32_t finite_mode;             /* 1 cartesian, 2 polar, 4 auto */
    double kinji_threshold;          /* bounding-box margin for the point-source exit, in rho */
    double hex_threshold;            /* caustic-distance threshold, in rho */
    double adaptive_hex_threshold;   /* hexadecapole tolerance */
    double limb_darkening_c;
    double limb_darkening_d;
    int32_t adaptive_source_bins;    /* nonzero with a tolerance below: local adaptive refinement
                                        (finite_source_magnifier.cpp:3074-3289) of Cartesian points */
    int32_t max_source_bins;         /* below 4096 when refining (the tape holds at most 4096 cells) */
    double finite_source_tol;
    double finite_source_reltol;
} lcbi_fs_settings;

/* One evaluation of FiniteSourceMagnifier::binary_mag
 * (src/lcbinint/magnification/finite_source_magnifier.cpp:4633-4642):
 * core convention (q < 1: heavier lens at -s; q > 1 inverted), source (y1, y2)
 * in the centre-of-mass frame, radius rho. */
typedef struct lcbi_fs_point {
    double s, q, y1, y2, rho;
    double point_source_magnification;  /* ignored with LCBI_FS_PS_ON_DEVICE */
    int32_t settings;                   /* index into the settings table */
    int32_t model;                      /* index into the lens-model table (LCBI_GPU_MODELS_GIVEN) */
    int32_t flags;                      /* LCBI_FS_PS_EXACT | LCBI_FS_PS_ON_DEVICE */
    int32_t reserved;
} lcbi_fs_point;

#define LCBI_FS_PS_EXACT 1      /* point_source_magnification_is_exact */
#define LCBI_FS_PS_ON_DEVICE 2  /* point_source_magnification = binary_mag0(s, q, y1, y2), on the GPU */
#define LCBI_FS_SEED_HINTS 4    /* seed the inverse ray with the point images that map inside the source,
                                   as LensModel passes them (src/lcbinint/model/lens_model.cpp:209-226) */

/* A caustic model (s, q, caustic_bins), the key of the reference's caustic
 * cache (finite_source_magnifier.cpp:4014-4022). */
typedef struct lcbi_lens_model {
    double s, q;
    int32_t caustic_bins;
    int32_t reserved;
} lcbi_lens_model;

/* FiniteSourceResult (finite_source_magnifier.hpp:53-60). */
typedef struct lcbi_fs_result {
    double magnification;
    double error_estimate;
    int32_t method;       /* 0 point source, 1 hexadecapole, 2 Cartesian, 3 polar */
    int32_t converged;
    int32_t status;       /* LCBI_OK, LCBI_NUMERICAL_ERROR, or LCBI_GPU_LIMIT_* */
    int32_t seed_count;   /* inverse-ray image seeds used */
} lcbi_fs_result;

/* Per-item device limits (the item's magnification is NaN). */
#define LCBI_GPU_LIMIT_SEEDS 17
#define LCBI_GPU_LIMIT_ROWS 18
#define LCBI_GPU_LIMIT_QUEUE 19
/* No longer returned: a point that meets needs_global_topology_retry
 * (finite_source_magnifier.cpp:1108-1121: adaptive_source_bins set, fewer than
 * 50 bins, rho < 1e-2, at least 16 seeds, 100 overlaps, 1,000 gap repairs and
 * a 1,000-cell jump) is scanned again at min(max_source_bins, max(50, 2 nbin))
 * bins as the reference does (:3168-3196), refinement level 1.  The value
 * stays reserved. */
#define LCBI_GPU_TOPOLOGY_RETRY 21

#define LCBI_GPU_MODELS_GIVEN 2u  /* points carry model indices into `models` */

/* Finite-source magnification of n points in one batched launch sequence.
 * Replaces FiniteSourceMagnifier::binary_mag
 * (src/lcbinint/magnification/finite_source_magnifier.cpp:4633-4843): the same
 * decision tree (caustic bounding box, derivative check, hexadecapole,
 * Cartesian or polar inverse ray) evaluated per point.  `settings` and
 * `models` are host arrays; without LCBI_GPU_MODELS_GIVEN the library derives
 * the models from the points (host `points` required).  Returns LCBI_OK when
 * the batch ran; per-point failures are in results[i].status. */
int lcbi_gpu_binary_mag(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int32_t n_settings,
                        const lcbi_lens_model *models, int32_t n_models, int64_t n,
                        const lcbi_fs_point *points, lcbi_fs_result *results, unsigned flags);

/* Launch-shape autotuner (no reference counterpart).  Runs
 * lcbi_gpu_binary_mag on the given batch (same arguments and flags) under a
 * coordinate search of three launch shapes -- blocks per SM of the polar tile
 * flood fill (1, 2, 4 or the occupancy limit), first-pass warps per SM (4 or
 * 8) and second-pass blocks (one or two per SM) -- timing each with CUDA events
 * after one untimed call, and leaves the fastest set on the context.  The
 * results do not depend on the shapes.  shape (optional) receives {flood
 * blocks per SM, warps per SM, second-pass blocks}, best_ms the fastest time;
 * results holds the last call's output. */
int lcbi_gpu_autotune(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int32_t n_settings,
                      const lcbi_lens_model *models, int32_t n_models, int64_t n, const lcbi_fs_point *points,
                      lcbi_fs_result *results, unsigned flags, int32_t *shape, double *best_ms);


/* lcbinint.binary_inverse_ray over n source positions
 * (python/lcbinint_pybind.cpp:3826-3847): the decision thresholds are forced
 * (kinji_threshold 1e18, hex thresholds 0) so every point is integrated by
 * inverse ray; q is passed to the core unchanged.  Host arrays only. */
int lcbi_gpu_binary_inverse_ray(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int64_t n,
                                const double *s, const double *q, const double *y1, const double *y2,
                                const double *rho, double *A, int32_t *method, int32_t *status);

/* Static binary light curves, VBM convention: the fast path of
 * lcbinint.LightCurve.__call__ (python/lcbinint_pybind.cpp:1087-1174).
 * params[m] = {t0, tE, u0, alpha, s, q, rho} (q in VBM convention, inverted
 * internally); times[first[m] .. first[m]+count[m]) are model m's epochs.
 * Host arrays only; A has one value per epoch. */
int lcbi_gpu_light_curves(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int32_t n_models,
                          const double *params, const int64_t *first, const int32_t *count,
                          const double *times, int64_t n_times, double *A, int32_t *method, int32_t *status);

/* Adjoint (no reference counterpart: the reference has no gradient; its
 * users difference the forward).  As lcbi_gpu_binary_mag, plus grads[8 * n]:
 * per point dA/d(y1, y2, s, q, rho, c) in the point's own parameters (core
 * convention, linear limb-darkening coefficient c), then the value that was
 * differentiated and the method.  Point source and hexadecapole: exact
 * derivatives of the forward's closed forms (implicit differentiation of the
 * lens-equation roots).  Inverse ray: derivatives of the continuum
 * magnification the lattice approximates -- image-boundary contour integrals
 * at rho and six Gauss-Legendre radii, which carry the limb-darkening term
 * without its interior singularity, on a lattice of rho/48 cells (slot 6 holds
 * the continuum value); quadratic limb darkening (d != 0) adds six radii
 * rho sqrt(1 - u^4) at Gauss-Legendre nodes u of [0, 1].  The contour sums
 * are accumulated with FP64 atomic additions in an order that varies between
 * calls, so inverse-ray gradients repeat to rounding, not bit for bit (the
 * magnifications do repeat bit for bit). */
int lcbi_gpu_binary_mag_grad(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int32_t n_settings,
                             const lcbi_lens_model *models, int32_t n_models, int64_t n,
                             const lcbi_fs_point *points, lcbi_fs_result *results, double *grads,
                             unsigned flags);

/* Resolution of the inverse-ray gradients' lattice (no reference
 * counterpart): cells of rho / cells_per_radius (default 48, accepted 8 to
 * 512).  The gradient is that of a piecewise-linear approximation of the
 * continuum magnification on this lattice, whose error falls as the square
 * of the cell, so a finer lattice brings the gradient (and the continuum
 * value in its slot 6) closer to the continuum's; time and tile-table use
 * grow as the square of cells_per_radius, and a point whose tiles do not fit
 * the table gets NaN gradients. */
int lcbi_gpu_set_grad_resolution(lcbi_gpu_context *ctx, int32_t cells_per_radius);

/* Light curves with gradients: params[m] = {t0, tE, u0, alpha, s, q, rho,
 * Gamma} (VBM convention, Gamma the linear limb-darkening coefficient, which
 * replaces settings->limb_darkening_c per model); A[n_times] and, if dA is not
 * NULL, dA[8 * n_times] = dA/d(t0, tE, u0, alpha, s, q, rho, Gamma) per epoch.
 * The forward is lcbi_gpu_light_curves' (same magnifications). */
int lcbi_gpu_light_curves_grad(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int32_t n_models,
                               const double *params, const int64_t *first, const int32_t *count,
                               const double *times, int64_t n_times, double *A, double *dA, int32_t *method,
                               int32_t *status);
/* As lcbi_gpu_light_curves_grad, with the per-epoch arrays in device memory:
 * times, A, dA (optional), method and status (optional) are DEVICE arrays of
 * the context's device, so training loops keep them resident; params, first
 * and count stay host arrays (they define the caustic models the host plans,
 * 64 bytes per model).  No reference counterpart (the reference has no
 * gradient). */
int lcbi_gpu_light_curves_grad_device(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, int32_t n_models,
                                      const double *params, const int64_t *first, const int32_t *count,
                                      const double *times, int64_t n_times, double *A, double *dA,
                                      int32_t *method, int32_t *status);

/* Caustic (caustic != 0) or critical curve (caustic == 0) of a binary lens
 * (python/lcbinint_pybind.cpp:1882-1926, LightCurve.caustics /
 * critical_curves): the critical-curve quartic at n_points phases
 * 2 pi i / n_points (n_points >= 8), its four roots, mapped through the lens
 * equation for the caustic, tracked into four branches by the first
 * least-cost assignment to each branch's last point (the first phase sorted
 * by polar angle).  q is the core-convention mass ratio the magnification
 * entry points take (1/q of VBM parameters); critical points are in the lens
 * frame of the quartic (heavier mass at -s or s, lighter at the origin),
 * caustic points in the source frame.  xy[2 * (b * n_points + j)] = (x, y) of
 * point j of branch b; points_per_branch (optional) receives n_points. */
int lcbi_gpu_binary_geometry(lcbi_gpu_context *ctx, double s, double q, int32_t n_points, int32_t caustic,
                             double *xy, int32_t *points_per_branch);

/* Lattice cells counted by the last finite-source call (one count per point,
 * cells whose centre maps inside the source disk), for ray-throughput
 * accounting; no reference counterpart.  n must not exceed that call's size. */
int lcbi_gpu_last_ray_counts(lcbi_gpu_context *ctx, int64_t n, uint64_t *rays);

/* Bounded device waits (no reference counterpart).  The tile-parallel flood
 * fills (polar inverse ray, gradient lattice) hand tiles between persistent
 * warps through a FIFO; a warp waiting for its ticket gives up after `polls`
 * polls (0 restores the default, seconds of polling) and stops that flood.
 * The polar flood's points are then integrated again by the
 * one-block-per-point second pass, which does not wait on other warps, so
 * magnifications never depend on whether a wait gave up (the gradients of a
 * stopped gradient flood are NaN).  lcbi_gpu_last_wait_timeouts reports how
 * many waits gave up during the last finite-source call on the context. */
int lcbi_gpu_set_wait_limit(lcbi_gpu_context *ctx, uint32_t polls);
int lcbi_gpu_last_wait_timeouts(lcbi_gpu_context *ctx, int32_t *count);

/* FiniteSourceResult::refinement_level of each point of the last
 * finite-source call (finite_source_magnifier.hpp:58; 0 unless the point was
 * refined adaptively or scanned again at twice the bins).  n must not exceed
 * that call's size. */
int lcbi_gpu_last_refinement_levels(lcbi_gpu_context *ctx, int64_t n, int32_t *levels);

/* Finite-source magnification that allocates nothing.  No reference
 * counterpart: the reference allocates freely on the host, and the entry
 * points above grow per-context device workspaces (cudaMalloc, and cudaFree of
 * the smaller buffer, which waits for the whole device) whenever a batch
 * outgrows them.  Callers that cannot allow that -- a sampler that has reserved
 * all free device memory for its own pool, or one whose other streams must not
 * be stalled by a device-wide wait -- use this entry point instead.
 *
 * It runs the pipeline of lcbi_gpu_binary_mag for one lens model (s, q) and one
 * settings struct, with the point-source magnification computed on the device
 * (LCBI_FS_PS_ON_DEVICE | LCBI_FS_PS_EXACT), and gives the same results as
 * lcbi_gpu_binary_mag on those points.  y1, y2, rho and results are DEVICE
 * arrays of n entries; settings is a host pointer.  All working memory is one
 * fixed device array of LCBI_NOALLOC_AREA_BYTES (48 MiB) per device, reserved
 * when the library's device code is loaded on that device:
 *   - settings->caustic_bins above LCBI_NOALLOC_MAX_CAUSTIC_BINS is rejected
 *     with LCBI_INVALID_ARGUMENT and a message in lcbi_gpu_last_error;
 *   - adaptive local refinement (adaptive_source_bins with a tolerance) is
 *     refused with LCBI_UNSUPPORTED: its tapes and heaps do not fit the array;
 *   - a point whose Cartesian scan needs more than 65536 rows per seed, or
 *     whose polar flood fill visits more than 262144 segments (or queues more
 *     than 131072 at once), gets status 18 / 19 and NaN (the workspace entry
 *     points go on to 524288 rows and 2097152 segments).
 * The first call on a device sets up: it looks up the fixed array's device
 * address (which loads the library's device code on that device) and uploads
 * constant angle tables with a synchronous copy.  Make that first call -- n = 0
 * is enough -- before any stream capture begins.  Every later call checks the
 * set-up again and repeats it after a cudaDeviceReset.  Calls on one device
 * share the one array and each leaves its contents behind (every call clears
 * what must start empty): calls that overlap in time (two host threads, or two
 * streams without ordering between them) race on it, so serialise them.  The
 * call returns after its work on the context's stream has finished. */
#define LCBI_NOALLOC_MAX_CAUSTIC_BINS 2048
#define LCBI_NOALLOC_AREA_BYTES (48u << 20)
int lcbi_gpu_binary_mag_noalloc(lcbi_gpu_context *ctx, const lcbi_fs_settings *settings, double s, double q,
                                int64_t n, const double *y1, const double *y2, const double *rho,
                                lcbi_fs_result *results);

/* ------------------------------------------------------------------ */
/* The reference's own C ABI (include/lcbinint/lcbinint.h:15-136)       */
/* ------------------------------------------------------------------ */

/* Same types, field order, names and semantics as include/lcbinint/lcbinint.h,
 * so a program written against the reference's header links against this
 * library unchanged.  The magnification runs on the calling thread's current
 * CUDA device, through a context kept per host thread.  Built: binary lenses
 * (q2 <= 0, no parallax, no xallarap), static or with circular or Keplerian
 * lens orbital motion (src/lcbinint/model/orbital_motion.cpp:69-206),
 * annual and terrestrial parallax and xallarap
 * (src/lcbinint/model/trajectory.cpp:185-463; see lcbi_set_earth_ephemeris),
 * in both coordinate conventions, point and finite source, bit-identical to
 * the reference.  Triple lenses return LCBI_UNSUPPORTED, with the result
 * filled as the reference fills unsupported input (NaN magnifications, the
 * source position). */
#ifndef LCBININT_H
typedef enum lcbi_orbital_motion_mode {
    LCBI_ORBIT_STATIC = 0,
    LCBI_ORBIT_CIRCULAR = 1,
    LCBI_ORBIT_KEPLER = 2
} lcbi_orbital_motion_mode;

typedef struct lcbi_params {
    double t0;
    double tE;
    double umin;
    double q;
    double sep;
    double theta;
    double rho;
    double omega;
    double piEN;
    double piEE;
    double piEN_xa;
    double piEE_xa;
    double ra_xa;
    double dec_xa;
    double period_xa;
    double ecc_xa;
    double peri_xa;
    double v_sep;
    double q2;
    double sep2;
    double ang;
    double ra;
    double dec;
    double earth_axis;
    double tfix;
    double obs_lat;
    double obs_lon;
    double limb_darkening_c;
    double limb_darkening_d;
    lcbi_orbital_motion_mode orbital_motion_mode;
    double g1;
    double g2;
    double g3;
    double lom_szs;
    double lom_ar;
    double xi_1;
    double xi_2;
    double omega_xa;
    double inc_xa;
    double phi_xa;
} lcbi_params;

typedef enum lcbi_xallarap_param_type {
    LCBI_XALLARAP_NONE = 0,
    LCBI_XALLARAP_ANGULAR_VELOCITY = 1,
    LCBI_XALLARAP_ORBITAL_ELEMENTS = 2
} lcbi_xallarap_param_type;

typedef struct lcbi_options {
    int parallax_mode;
    int orbit_pair;
    int center_of_mass;
    int caustic_bins;
    int source_bins;
    int mode;                 /* 1 cartesian, 2 polar, 4 auto */
    int vbm_compatible;       /* 0 original convention, 1 VBM convention */
    lcbi_xallarap_param_type xallarap_param_type;
    double grid_ratio;
    int polar_source_bins;
    double polar_grid_ratio;
    double point_source_threshold;
    double hexadecapole_threshold;
    double adaptive_hex_threshold;
    int adaptive_source_bins;
    int max_source_bins;
    double finite_source_tol;
    double finite_source_reltol;
} lcbi_options;

typedef struct lcbi_result {
    double magnification;
    double point_source_magnification;
    double finite_source_magnification;
    double source_x;
    double source_y;
    int image_count;
    double finite_source_error_estimate;
    int finite_source_refinement_level;
    int finite_source_converged;
} lcbi_result;

/* lcbinint.h:118-119: the reference's defaults. */
lcbi_params lcbi_default_params(void);
lcbi_options lcbi_default_options(void);
/* lcbinint.h:121-126: one epoch (a batch of one). */
lcbi_status lcbi_magnification(double time, const lcbi_params *params, const lcbi_options *options,
                               lcbi_result *result);
/* lcbinint.h:128-134: all epochs in one batch on the GPU; like the reference,
 * results are written up to and including the first epoch that fails, whose
 * status is returned. */
lcbi_status lcbi_magnification_array(const double *times, int count, const lcbi_params *params,
                                     const lcbi_options *options, lcbi_result *results);
/* lcbinint.h:136. */
const char *lcbi_status_string(lcbi_status status);
#endif

/* lcbi_magnification_array for many parameter sets in one batched GPU pass
 * (no reference counterpart: the reference evaluates one set per call, one
 * epoch at a time).  Set m covers times[first[m] .. first[m] + count[m]) and
 * writes results[first[m] ...] and status[m] exactly as
 * lcbi_magnification_array(times + first[m], count[m], params + m, options,
 * results + first[m]) would.  Sets may differ in every parameter, lens orbital
 * motion and limb darkening included; options (NULL: the defaults) is shared.
 * Lens orbital motion gives every epoch its own separation, hence its own
 * caustic sampling (1,400 quartics by default), as in the reference.
 * With LCBI_ARRAYS_KEYWORD_ROUTE the source is turned into the orbit's frame
 * as the Python module's keyword-argument light curves turn it
 * (python/lcbinint_pybind.cpp:1985-2008: the trajectory point rotated back
 * by alpha and forward by the orbit's angle) instead of as LensModel does
 * (src/lcbinint/model/lens_model.cpp:172-190); the two differ in rounding
 * only.  Returns LCBI_OK once every set has its status, else the error that
 * stopped the batch (LCBI_INVALID_ARGUMENT for bad array arguments,
 * LCBI_GPU_ERROR). */
/* Lens orbital motion at `time` (src/lcbinint/model/orbital_motion.cpp:69-183;
 * Python lcbinint.circular_orbital_motion / kepler_orbital_motion,
 * python/lcbinint_pybind.cpp:3896-3925): state = {projected separation,
 * angle of the binary axis, line-of-sight separation}.  Host arithmetic,
 * bit-identical to the reference's. */
int lcbi_circular_orbital_motion(double time, double separation, double angle, double g1, double g2, double g3,
                                 double reference_time, double *state);
int lcbi_kepler_orbital_motion(double time, double separation, double angle, double g1, double g2, double g3,
                               double szs, double ar, double reference_time, double *state);

/* LightCurve.source_trajectory (python/lcbinint_pybind.cpp:3292-3330 over
 * PyLightCurveEvaluator::dynamic_source_trajectory, :1819-1880): the source
 * position in the lens frame at each of n times, x[i], y[i].  The straight
 * line in the options' coordinates, moved by annual (and terrestrial) parallax
 * when piEN or piEE is non-zero, and turned into the frame of the binary's
 * axis at that time under lens orbital motion.  Host arithmetic, bit-identical
 * to the reference's.  options NULL means the defaults. */
int lcbi_source_trajectory(const lcbi_params *params, const lcbi_options *options, const double *times, int64_t n,
                           double *x, double *y);

/* The Earth ephemeris for annual parallax (no counterpart in the reference's
 * ABI: the reference reads the file named by the LCBININT_EARTH_EPHEMERIS
 * environment variable, else its compiled-in data/earth_orbital_parallax_table.txt,
 * once per process; src/lcbinint/model/trajectory.cpp:128-183).  This library
 * reads the same environment variable on first use; this call loads a JPL
 * Horizons vector table (JD, x, y, z, vx, vy, vz in AU and AU/day, between
 * $$SOE and $$EOE) explicitly instead.  Returns the number of states read, or
 * -1 if the file cannot be opened.  Without a table every parallax epoch is a
 * numerical error, as in the reference. */
int lcbi_set_earth_ephemeris(const char *path);

#define LCBI_ARRAYS_KEYWORD_ROUTE 1u
int lcbi_gpu_magnification_arrays(lcbi_gpu_context *ctx, int32_t n_sets, const lcbi_params *params,
                                  const lcbi_options *options, const int64_t *first, const int32_t *count,
                                  const double *times, int64_t n_times, unsigned flags, lcbi_result *results,
                                  int32_t *status);

#ifdef __cplusplus
}
#endif

#endif /* LCBININT_B200_H */
