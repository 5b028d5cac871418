// Light-curve prologue: one finite-source item per (model, epoch).
//
// Source trajectory of the static-binary VBM-convention fast path of
// LightCurve.__call__ (python/lcbinint_pybind.cpp:1140-1157):
//   tau = (t - t0) * (1 / tE),  y1 = tau cos(alpha) - u0 sin(alpha),
//   y2 = tau sin(alpha) + u0 cos(alpha),  q_core = 1 / q.
// cos(alpha) and sin(alpha) come from the host C library, as in the reference.
#include "lcbi_fs_kernels.h"

namespace lcbi {

__global__ void lc_items_kernel(const LcModel* __restrict__ models, int n_models, const double* __restrict__ times,
                                FsItem* __restrict__ items, long long n_items)
{
    const int m = blockIdx.y;
    if (m >= n_models) return;
    const LcModel md = models[m];
    const double inverse_tE = 1.0 / md.tE;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < md.count; i += gridDim.x * blockDim.x) {
        const long long k = md.first + i;
        if (k >= n_items) break;
        const double tau = (times[k] - md.t0) * inverse_tE;
        FsItem it;
        it.s = md.s;
        it.q = md.q_core;
        it.x = tau * md.cos_alpha - md.u0 * md.sin_alpha;
        it.y = tau * md.sin_alpha + md.u0 * md.cos_alpha;
        it.rho = fabs(md.rho);
        it.a_ps = 0.0;
        it.settings = md.settings;
        it.model = md.model;
        it.flags = kItemPsExact | kItemPsOnDevice;
        it.pad = 0;
        items[k] = it;
    }
}

cudaError_t launch_lc_items(const LcModel* models, int n_models, const double* times, FsItem* items,
                            long long n_items, cudaStream_t stream)
{
    if (n_models <= 0) return cudaSuccess;
    dim3 grid(4, n_models);
    lc_items_kernel<<<grid, 256, 0, stream>>>(models, n_models, times, items, n_items);
    return cudaGetLastError();
}

// Point-source value and image count of each item, written into the item as
// the decision's a_ps.  A finite source takes them from binary_images
// (point_source_magnifier.cpp:723-778), whose images also seed the inverse
// ray, as LensModel forms its finite-source call (lens_model.cpp:209-226); a
// point source (rho == 0) from binary_mag0 (lens_model.cpp:43-46).
__global__ void __launch_bounds__(128) item_images_kernel(FsItem* __restrict__ items, long long n,
                                                         double* __restrict__ a_ps, int* __restrict__ nimg)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double s = items[i].s, q = items[i].q, x = items[i].x, y = items[i].y;
        double a = 0.0;
        int cnt = 0;
        if (items[i].rho > 0.0) {
            if (s != 0.0 && q > 0.0) {
                const BinaryGeom g = make_geom(s, q, x, y);
                dc pos[5];
                double res[5], det[5];
                cnt = image_candidates(g, pos, res, det);
                for (int k = 0; k < cnt; ++k) a += 1.0 / fabs(det[k]);
            }
        } else {
            const PsResult r = point_source(s, q, x, y);
            a = r.magnification;
            cnt = r.image_count;
        }
        items[i].a_ps = a;
        a_ps[i] = a;
        nimg[i] = cnt;
    }
}

cudaError_t launch_item_images(FsItem* items, long long n, double* a_ps, int* nimg, int sm_count, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    long long blocks = (n + threads - 1) / threads;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    item_images_kernel<<<(unsigned)blocks, threads, 0, stream>>>(items, n, a_ps, nimg);
    return cudaGetLastError();
}

// Chain rule from the point parameters (y1, y2, s, q_core, rho, c) to the
// light-curve parameters (t0, tE, u0, alpha, s, q, rho, Gamma), with
// q_core = 1 / q and Gamma = c.
__global__ void lc_grad_chain_kernel(const LcModel* __restrict__ models, int n_models,
                                     const double* __restrict__ times, const double* __restrict__ pg,
                                     double* __restrict__ out, long long n_items)
{
    const int m = blockIdx.y;
    if (m >= n_models) return;
    const LcModel md = models[m];
    const double inverse_tE = 1.0 / md.tE;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < md.count; i += gridDim.x * blockDim.x) {
        const long long k = md.first + i;
        if (k >= n_items) break;
        const double tau = (times[k] - md.t0) * inverse_tE;
        const double* g = pg + k * 8;
        const double along = g[0] * md.cos_alpha + g[1] * md.sin_alpha;
        double* o = out + k * 8;
        o[0] = -along * inverse_tE;
        o[1] = -along * tau * inverse_tE;
        o[2] = -g[0] * md.sin_alpha + g[1] * md.cos_alpha;
        o[3] = g[0] * (-tau * md.sin_alpha - md.u0 * md.cos_alpha) + g[1] * (tau * md.cos_alpha - md.u0 * md.sin_alpha);
        o[4] = g[2];
        o[5] = -g[3] * md.q_core * md.q_core;
        o[6] = md.rho < 0.0 ? -g[4] : g[4];
        o[7] = g[5];
    }
}

cudaError_t launch_lc_grad_chain(const LcModel* models, int n_models, const double* times, const double* point_grads,
                                 double* grads, long long n_items, cudaStream_t stream)
{
    if (n_models <= 0) return cudaSuccess;
    dim3 grid(4, n_models);
    lc_grad_chain_kernel<<<grid, 256, 0, stream>>>(models, n_models, times, point_grads, grads, n_items);
    return cudaGetLastError();
}

// Result records into separate device arrays (any of them may be null):
// magnification, method and status of each point, as the host entry points
// hand them back.
__global__ void unpack_results_kernel(const FsOut* __restrict__ out, double* __restrict__ A, int* __restrict__ method,
                                      int* __restrict__ status, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const FsOut o = out[i];
        if (A) A[i] = o.A;
        if (method) method[i] = o.method;
        if (status) status[i] = o.status;
    }
}

cudaError_t launch_unpack_results(const FsOut* out, double* A, int* method, int* status, long long n,
                                  cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    long long blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    unpack_results_kernel<<<(unsigned)blocks, 256, 0, stream>>>(out, A, method, status, n);
    return cudaGetLastError();
}

} // namespace lcbi
