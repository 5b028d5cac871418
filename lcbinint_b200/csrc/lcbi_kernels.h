// Internal launch interface between the C-ABI host runtime (capi.cu) and the
// kernel translation units.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

namespace lcbi {

cudaError_t launch_ps_batch(const double* s, const double* q, const double* y1, const double* y2, double* A,
                            int* nimg, int* status, long long n, int sm_count, cudaStream_t stream);

cudaError_t launch_ps_deriv(const double* s, const double* q, const double* y1, const double* y2, double* A,
                            int* nimg, double* indicator, long long n, int sm_count, cudaStream_t stream);

cudaError_t launch_ps_images(const double* s, const double* q, const double* y1, const double* y2, double* A,
                             int* nimg, long long n, int sm_count, cudaStream_t stream);

cudaError_t launch_ps_candidates(const double* s, const double* q, const double* y1, const double* y2, double4* out,
                                 int* nphys, long long n, int sm_count, cudaStream_t stream);

cudaError_t kernel_binary_version(int* version);

} // namespace lcbi
