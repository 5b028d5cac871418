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

/* Point-source magnification plus the smoothness indicator the finite-source
 * decision tree uses.  Replaces PointSourceMagnifier::binary_mag0_with_derivatives
 * (src/lcbinint/magnification/point_source_magnifier.cpp:583-611). */
int lcbi_gpu_binary_mag0_derivatives(lcbi_gpu_context *ctx, int64_t n, const double *s,
                                     const double *q, const double *y1, const double *y2,
                                     double *A, int32_t *image_count, double *indicator,
                                     unsigned flags);

#ifdef __cplusplus
}
#endif

#endif /* LCBININT_B200_H */
