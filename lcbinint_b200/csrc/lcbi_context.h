// Host-side state of one lcbi_gpu_context: device, stream, and growable
// device workspaces reused across calls (no allocation on the steady path).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace lcbi {

struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct Context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    int64_t launches = 0;

    Buffer in[8];
    Buffer out[8];
    Buffer work[8];

    // finite-source pipeline
    Buffer fs_settings, fs_models, fs_raw_offset, fs_phases, fs_items, fs_out, fs_raw, fs_branches, fs_ld;
    Buffer fs_ir, fs_counters, fs_seeds, fs_cand_keys, fs_cand_probes, fs_scratch, fs_scratch_polar;
    Buffer fs_trig, fs_lc_models, fs_times, fs_ld_coeffs, fs_rays, fs_retry, fs_scratch_big, fs_scratch_polar_big;
    Buffer fs_cycles, fs_tiles, fs_grad_tiles, fs_grad, fs_grad_lc;
    Buffer fs_all_aps, fs_all_nimg;  // whole-batch point-source values of binary_mag_images
    // binary_mag_images: caustic samples and work lists of two passes in
    // flight, and the store of what the inverse-ray points need after their
    // pass (their caustic models, work lists and seeds).
    Buffer pass_raw[2], pass_branches[2], pass_lists[2], pass_counters[2], pass_jobs[2];
    Buffer ir_models, ir_branches, ir_lists, ir_counters, ir_retry;
    Buffer fs_needed, fs_model_base;  // caustic models some point needs; first model of each pass
    Buffer fs_tape, fs_levels;        // adaptive refinement: boundary-cell tapes; refinement level per point
    Buffer fs_seed_block;             // block seeding pass: candidate scratch per block
    Buffer fs_route;                  // early block routing: candidate list
    Buffer fs_waits;                  // device waits that gave up during the last call (one int)
    unsigned wait_limit = 0;          // polls before a device wait gives up (0: the kernels' default)
    Buffer fs_seed_early;             // seeding of the early points: candidate scratch per warp
    Buffer fs_split, fs_split_info;   // units of the split early points: row scratch and results
    Buffer fs_seed_info;              // their seeds after the gap repairs
    bool early_live = false;          // the early stream holds work that stage_integrate joins
    bool early_serial = false;        // stage timing on: stage_integrate runs the early block pass
    int seed_block_after = 32;        // in-disk critical sources that move a point's seeding to a block (0: never)
    bool tape_on = false;             // the current plan has settings that refine
    void* pinned = nullptr;     // page-locked staging of the passes' work lists and jobs
    size_t pinned_bytes = 0;
    bool trig_ready = false;
    unsigned long long epoch = 0;
    int fs_warps = 0;          // persistent warps the scratch areas are sized for
    int row_cap = 32768;       // Cartesian rows per seed scan
    int queue_cap = 1 << 16;   // polar FIFO of segments
    int hash_cap = 1 << 17;    // polar visited-segment slots
    int seed_cap = 2048;       // seeds per inverse-ray item
    int cand_cap = 4 * 1400;   // caustic-branch probe candidates per warp
    bool item_cycles = false;  // record per-item seeding + integration cycles
    int warps_per_sm = 8;
    // Second pass, one block of kBigWarps warps per point, for the points that
    // pass the first pass's cell budget or overflow its per-warp scratch.
    long long cell_budget = 1 << 19;
    bool cell_budget_set = false;  // set by the caller; else small batches send every point to blocks
    int retry_blocks = 0;      // 0: one per SM
    bool early_helpers = true;  // the side stream's blocks join the early pass after the Cartesian passes
    int row_cap_big = 1 << 19;
    int queue_cap_big = 1 << 19;
    int hash_cap_big = 1 << 21;
    bool big_ready = false;
    // Tile-parallel polar flood fill: table and FIFO capacity (power of two).
    bool polar_tiles = true;
    bool f32_rays = false;     // inverse-ray cells mapped in FP32 about image-centred anchors
    long long tile_capacity = 1 << 20;
    int tile_blocks = 0;       // persistent flood blocks (0: occupancy x SMs)
    // Adjoint: cells per source radius of the gradient lattice, flood blocks.
    int grad_bins = 48;
    int grad_blocks = 0;
    cudaStream_t own_stream = nullptr;  // the context's stream; `stream` may be a caller's
    // Side stream (highest priority) for the second Cartesian pass, which runs
    // beside the polar passes; fork/join events order it against `stream`.
    cudaStream_t side_stream = nullptr;
    cudaEvent_t fork_event = nullptr, join_event = nullptr;
    // Early stream (highest priority) for the Cartesian points routed to
    // blocks from the start, beside the first pass.
    cudaStream_t early_stream = nullptr;
    cudaEvent_t early_fork = nullptr, early_join = nullptr;
    // Recorded on the early stream once the early points are seeded: the
    // side stream waits for it before its own blocks join the early pass.
    cudaEvent_t early_seeded = nullptr;
    // Stream marks (lcbi_gpu_set_stream_marks): timing events at the start of
    // the seeding stage [0] and where the early [1], side [2] and context [3]
    // streams' inverse-ray work ends; bit i of marks_set: event i recorded.
    bool marks_on = false;
    cudaEvent_t marks[4] = {};
    unsigned marks_set = 0;
    void mark(int i, cudaStream_t s)
    {
        if (marks_on && marks[i] != nullptr && cudaEventRecord(marks[i], s) == cudaSuccess) marks_set |= 1u << i;
    }

    // Optional per-stage kernel timing with CUDA events on the launch stream.
    static constexpr int kStages = 8;  // 0 caustics+LD, 1 decide, 2 seeds, 3 cartesian, 4 polar, 5 point source
    bool timing = false;
    double stage_ms[kStages] = {};
    long long stage_launches[kStages] = {};
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    void stage_begin(int stage, cudaEvent_t* ev);
    void stage_end(int stage, cudaEvent_t begin);
    void collect_timing();

    std::vector<Buffer*> all_buffers()
    {
        std::vector<Buffer*> v;
        for (auto& b : in) v.push_back(&b);
        for (auto& b : out) v.push_back(&b);
        for (auto& b : work) v.push_back(&b);
        for (Buffer* b : {&fs_settings, &fs_models, &fs_raw_offset, &fs_phases, &fs_items, &fs_out, &fs_raw,
                          &fs_branches, &fs_ld, &fs_ir, &fs_counters, &fs_seeds, &fs_cand_keys, &fs_cand_probes,
                          &fs_scratch, &fs_scratch_polar, &fs_trig, &fs_lc_models, &fs_times, &fs_ld_coeffs,
                          &fs_rays, &fs_retry, &fs_scratch_big, &fs_scratch_polar_big, &fs_cycles, &fs_tiles, &fs_grad_tiles, &fs_grad, &fs_grad_lc,
                          &fs_all_aps, &fs_all_nimg, &pass_raw[0], &pass_raw[1], &pass_branches[0],
                          &pass_branches[1], &pass_lists[0], &pass_lists[1], &pass_counters[0], &pass_counters[1],
                          &pass_jobs[0], &pass_jobs[1], &ir_models, &ir_branches, &ir_lists, &ir_counters, &ir_retry, &fs_seed_block, &fs_route, &fs_waits, &fs_seed_early, &fs_split, &fs_split_info, &fs_seed_info,
                          &fs_needed, &fs_model_base, &fs_tape, &fs_levels})
            v.push_back(b);
        return v;
    }

    ~Context();
    bool fail(const char* what, cudaError_t e);
    bool fail(const std::string& what);
    bool check(const char* what, cudaError_t e);
    bool ensure(Buffer& b, size_t bytes);
    bool finish();

    template <typename T>
    bool stage_in(Buffer& buf, const T* src, size_t count, bool device_ptrs, const T** out);
    template <typename T>
    bool stage_out(Buffer& buf, T* dst, size_t count, bool device_ptrs, T** out);
    template <typename T>
    bool copy_back(T* dst, const T* dev, size_t count, bool device_ptrs);
};

} // namespace lcbi
