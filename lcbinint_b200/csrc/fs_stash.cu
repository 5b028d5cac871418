// Copies of the caustic models that inverse-ray points need after their pass.
//
// binary_mag_images runs the caustic sampling and the decision pass by pass
// (every point of a pass may have its own separation, so a pass's caustic
// samples are dropped once it is decided), then seeds and integrates all
// inverse-ray points of the batch together.  Seeding reads each point's
// caustic model and its tracked branches, so those are copied out of the
// pass's tables first: one block per model.
#include "lcbi_fs_kernels.h"

namespace lcbi {

__global__ void __launch_bounds__(256) stash_kernel(const CausticModel* __restrict__ src_models,
                                                    const P2* __restrict__ src_branches,
                                                    const StashJob* __restrict__ jobs, int n_jobs,
                                                    CausticModel* __restrict__ dst_models, P2* __restrict__ dst_branches,
                                                    const StashRemap* __restrict__ remaps, int n_remaps,
                                                    FsItem* __restrict__ items)
{
    for (int j = blockIdx.x; j < n_jobs; j += gridDim.x) {
        const StashJob job = jobs[j];
        CausticModel md = src_models[job.src_model];
        const P2* src = src_branches + md.branch_offset;
        P2* dst = dst_branches + job.dst_offset;
        const int n = 4 * md.bins;
        for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
        if (threadIdx.x == 0) {
            md.branch_offset = job.dst_offset;
            dst_models[job.dst_model] = md;
        }
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_remaps; r += gridDim.x * blockDim.x)
        items[remaps[r].item].model = remaps[r].dst_model;
}

cudaError_t launch_stash(const CausticModel* src_models, const P2* src_branches, const StashJob* jobs, int n_jobs,
                         CausticModel* dst_models, P2* dst_branches, const StashRemap* remaps, int n_remaps,
                         FsItem* items, cudaStream_t stream)
{
    if (n_jobs <= 0 && n_remaps <= 0) return cudaSuccess;
    int blocks = n_jobs > 0 ? n_jobs : 1;
    const int by_remaps = (n_remaps + 255) / 256;
    if (by_remaps > blocks) blocks = by_remaps;
    if (blocks > 4096) blocks = 4096;
    stash_kernel<<<blocks, 256, 0, stream>>>(src_models, src_branches, jobs, n_jobs, dst_models, dst_branches, remaps,
                                            n_remaps, items);
    return cudaGetLastError();
}

} // namespace lcbi
