// Point-source kernels: one thread per source position, FP64 throughout.
//
// A warp holds 32 independent source positions.  The root solver is serial
// within a position (each deflation needs the previous root), so lanes take
// separate positions instead of sharing one; with 1e6 positions that keeps all
// 148 SMs busy and every coefficient in registers.
#include "lcbi_kernels.h"
#include "lcbi_ps.cuh"

namespace lcbi {

__global__ void __launch_bounds__(128, 4) ps_batch_kernel(const double* __restrict__ s, const double* __restrict__ q,
                                                      const double* __restrict__ y1, const double* __restrict__ y2,
                                                      double* __restrict__ A, int* __restrict__ nimg,
                                                      int* __restrict__ status, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const PsResult r = point_source(s[i], q[i], y1[i], y2[i]);
        A[i] = r.magnification;
        if (nimg) nimg[i] = r.image_count;
        if (status) status[i] = r.status;
    }
}

// Same, returning the derivative indicator used by the finite-source decision
// tree (binary_mag0_with_derivatives, point_source_magnifier.cpp:583-611).
__global__ void __launch_bounds__(128) ps_deriv_kernel(const double* __restrict__ s, const double* __restrict__ q,
                                                      const double* __restrict__ y1, const double* __restrict__ y2,
                                                      double* __restrict__ A, int* __restrict__ nimg,
                                                      double* __restrict__ indicator, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double a = 0.0, ind = 0.0;
        int cnt = 0;
        if (s[i] != 0.0 && q[i] > 0.0) {
            const BinaryGeom g = make_geom(s[i], q[i], y1[i], y2[i]);
            dc roots[5];
            if (solve_images(g, roots)) {
                const unsigned mask = physical_mask(g, roots);
                a = sum_inverse_jacobians(g, roots, mask, &cnt);
                ind = derivative_indicator(g, roots, mask);
            } else {
                a = __longlong_as_double(0x7ff8000000000000ll);
            }
        }
        A[i] = a;
        nimg[i] = cnt;
        indicator[i] = ind;
    }
}

// Magnification summed over the physical images of binary_images
// (point_source_magnifier.cpp:723-778) in their residual order, as LensModel
// forms the finite-source decision's point-source value
// (lens_model.cpp:209-216).
__global__ void __launch_bounds__(128) ps_images_kernel(const double* __restrict__ s, const double* __restrict__ q,
                                                       const double* __restrict__ y1, const double* __restrict__ y2,
                                                       double* __restrict__ A, int* __restrict__ nimg, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double a = 0.0;
        int cnt = 0;
        if (s[i] != 0.0 && q[i] > 0.0) {
            const BinaryGeom g = make_geom(s[i], q[i], y1[i], y2[i]);
            dc pos[5];
            double res[5], det[5];
            cnt = image_candidates(g, pos, res, det);
            for (int k = 0; k < cnt; ++k) a += 1.0 / fabs(det[k]);
        }
        A[i] = a;
        if (nimg) nimg[i] = cnt;
    }
}

// The five image candidates of binary_image_candidates
// (point_source_magnifier.cpp:739-778), sorted by residual: per position five
// records {x, y, jacobian determinant, sqrt residual} and the number of
// physical ones (the first 3 or 5; 0 when s == 0 or q <= 0, and then no
// record is written; -1 when the solver cannot run: the source exactly on
// the lighter lens).
__global__ void __launch_bounds__(128) ps_candidates_kernel(const double* __restrict__ s,
                                                           const double* __restrict__ q,
                                                           const double* __restrict__ y1,
                                                           const double* __restrict__ y2,
                                                           double4* __restrict__ out, int* __restrict__ nphys,
                                                           long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int cnt = 0;
        if (s[i] != 0.0 && q[i] > 0.0) {
            const BinaryGeom g = make_geom(s[i], q[i], y1[i], y2[i]);
            dc pos[5];
            double res[5], det[5];
            cnt = image_candidates(g, pos, res, det);
            if (cnt == 0) cnt = -1;
            for (int k = 0; k < 5 && cnt > 0; ++k)
                out[5 * i + k] = make_double4(pos[k].re, pos[k].im, det[k], res[k]);
        }
        nphys[i] = cnt;
    }
}

cudaError_t launch_ps_candidates(const double* s, const double* q, const double* y1, const double* y2, double4* out,
                                 int* nphys, long long n, int sm_count, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    long long blocks = (n + threads - 1) / threads;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    ps_candidates_kernel<<<(unsigned)blocks, threads, 0, stream>>>(s, q, y1, y2, out, nphys, n);
    return cudaGetLastError();
}

// The compute capability the library's device code was built for
// (cudaFuncAttributes::binaryVersion of one of its kernels, e.g. 100 for sm_100a).
cudaError_t kernel_binary_version(int* version)
{
    cudaFuncAttributes a{};
    const cudaError_t e = cudaFuncGetAttributes(&a, ps_batch_kernel);
    if (e == cudaSuccess) *version = a.binaryVersion;
    return e;
}

cudaError_t launch_ps_images(const double* s, const double* q, const double* y1, const double* y2, double* A,
                             int* nimg, long long n, int sm_count, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    long long blocks = (n + threads - 1) / threads;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    ps_images_kernel<<<(unsigned)blocks, threads, 0, stream>>>(s, q, y1, y2, A, nimg, n);
    return cudaGetLastError();
}

cudaError_t launch_ps_batch(const double* s, const double* q, const double* y1, const double* y2, double* A,
                            int* nimg, int* status, long long n, int sm_count, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    long long blocks = (n + threads - 1) / threads;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    ps_batch_kernel<<<(unsigned)blocks, threads, 0, stream>>>(s, q, y1, y2, A, nimg, status, n);
    return cudaGetLastError();
}

cudaError_t launch_ps_deriv(const double* s, const double* q, const double* y1, const double* y2, double* A,
                            int* nimg, double* indicator, long long n, int sm_count, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    long long blocks = (n + threads - 1) / threads;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    ps_deriv_kernel<<<(unsigned)blocks, threads, 0, stream>>>(s, q, y1, y2, A, nimg, indicator, n);
    return cudaGetLastError();
}

} // namespace lcbi
