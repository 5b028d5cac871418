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

} // namespace lcbi
