// Internal launch interface of the finite-source kernels (not public ABI).
#pragma once

#include <cuda_runtime.h>

#include "lcbi_fs.cuh"

namespace lcbi {

// One finite-source evaluation: FiniteSourceMagnifier::binary_mag arguments
// (finite_source_magnifier.cpp:4633-4642) plus table indices.
struct FsItem {
    double s, q, x, y, rho, a_ps;
    int settings;   // index into the FsSettingsDev table
    int model;      // index into the CausticModel table
    int flags;      // kItemPsExact | kItemPsOnDevice
    int pad;
};

enum : int {
    kItemPsExact = 1,     // point_source_magnification_is_exact (hexadecapole reuses a_ps)
    kItemPsOnDevice = 2,  // a_ps = binary_mag0(s, q, x, y), computed by the decision kernel
    kItemSeedHints = 4,   // the point images are seed hints, kept only if they map inside the source
    kItemOutsideBox = 8,  // set by launch_certify: the source is outside the outer caustic box by the margin
};

// Per-item outputs.
struct FsOut {
    double A;
    double err;
    int method;     // FiniteSourceMethod value
    int converged;
    int status;     // 0 ok, 2 numerical error, 16+ device-side limit hit
    int n_seeds;
};

// Device-side limits; exceeding one sets FsOut::status and the item's A to NaN.
enum FsStatus {
    kFsOk = 0,
    kFsNumerical = 2,
    kFsSeedOverflow = 17,
    kFsRowOverflow = 18,
    kFsQueueOverflow = 19,
    kFsHashOverflow = 20,
    kFsTopologyRetry = 21,  // adaptive refinement would rerun the scan at twice the bins (not built)
};

// Adaptive local refinement: the boundary cells a Cartesian scan records
// (LocalRefinementTape, finite_source_magnifier.cpp:977-1004), at most
// kTapeMax per point.
constexpr int kTapeMax = 4096;
struct TapeCell {
    double x, y, w;
    long long kx, ky;
};

struct FsWork {
    const FsItem* items;
    const FsSettingsDev* settings;
    const CausticModel* models;
    const long long* raw_offset;
    const P2* raw;
    const P2* branches;
    const double* ld_tables;
    TrigTables trig;
    FsOut* out;
    int n_items;
    // inverse-ray work lists written by the decision kernel
    int* ir_count;   // [0] cartesian, [1] polar
    int* ir_cart;
    int* ir_polar;
    // seeds
    P2* seeds;       // seed_cap per inverse-ray item, indexed by item
    int seed_cap;
    // per-warp scratch for the Cartesian row scan and the polar flood fill
    char* scratch;
    long long scratch_per_warp;
    char* scratch_polar;
    long long scratch_polar_per_warp;
    int row_cap;     // Cartesian rows per seed scan
    int queue_cap;   // polar FIFO of segments (power of two)
    int hash_cap;    // polar visited-segment hash slots (power of two)
    int* next_item;  // dynamic work counters: [0] seeds, [1] cartesian, [2] polar, [3] cart retry, [4] polar retry
    unsigned long long* rays;  // per item: lattice cells whose centre maps inside the source disk
    // Items whose scratch overflowed, or that passed the cell budget, in the
    // first pass are queued here and run again on whole blocks with a larger
    // scratch per block (retry_pass = 1); counts in ir_count[2..3].
    int retry_pass;
    int* retry_cart;
    int* retry_polar;
    int cand_cap;                  // caustic-branch probe candidates per warp (4 x max caustic bins)
    long long* cycles;             // optional per-item clock64 cycles of seeding + integration
    // First pass only: a point whose scan passes this many cells (0: no limit)
    // is handed to the second pass, which runs each point on a block of
    // kBigWarps warps.
    long long cell_budget;
    // First pass only: when a list holds at most this many points (0: never),
    // the budget is one cell, so every point of the list runs on a block.
    int few_points;
    // Inverse-ray cells mapped in FP32 about an image-centred anchor (sums
    // stay FP64); 0: the reference's FP64 map, bit-exact.
    int f32_rays;
    // Adaptive local refinement (settings with adaptive_source_bins and a
    // tolerance): one tape of kTapeMax cells per scratch group (indexed as the
    // scratch areas; null: refinement off), and each point's refinement level
    // (null: not recorded).
    TapeCell* tape;
    int* levels;
    // Seeding: a point whose caustic-crossing phase scan reaches this many
    // critical sources inside its disk (0: no limit) is handed from the
    // one-warp seeding pass to the block seeding pass (launch_seeds_blocks),
    // which probes several critical sources at once.  Its list position goes
    // to retry_seeds (count in ir_count[4]); each block of that pass has
    // seed_scratch_per_block bytes of candidate scratch at seed_scratch.
    int seed_block_after;
    int* retry_seeds;
    char* seed_scratch;
    long long seed_scratch_per_block;
    // Cartesian points predicted to pass the first pass's budget many times
    // over (launch_route_early) run on blocks from the start, beside the first
    // pass, which skips them: their list positions, largest first, at
    // early_cart (count in ir_count[5], at most kEarlyMax).  early_pass = 1
    // makes the block kernel take that list (work counter next_item[6]).
    int* early_cart;
    int early_pass;
    // Seeding of a given list of Cartesian list positions (null: every point
    // of the work lists), e.g. the early points on their own stream, with its
    // own work counter; seed_skip_early = 1 leaves the early points out.
    const int* seed_slots;
    const int* seed_count;
    int* seed_next;
    int seed_skip_early;
    // Bounded device waits (the tile flood fills' FIFO tickets): a wait gives
    // up after wait_limit polls (0: the default, seconds of polling), sets the
    // flood's error word, and counts itself in *wait_timeouts (if not null);
    // the points of a flood that gave up are integrated again by the second
    // pass, which has no such waits.
    unsigned wait_limit;
    int* wait_timeouts;
    // Early points split into units (early pass only; split_info null: off):
    // the up and the down scan of each of the first kSplitSeeds seeds of
    // every early point run as separate work items, each on its own block
    // (unit u = (point * kSplitSeeds + seed) * 2 + half, its SplitInfo at
    // split_info[u]).  A unit that runs takes the next of split_slots row
    // scratch areas of kSplitRowCap rows (split_bytes each at split_scratch;
    // ir_count[kSplitAlloc] counts the slots taken), and the block that
    // completes a point's last unit (the point's counter at
    // ir_count[kSplitCounter + point]) finishes the point from their rows.
    char* split_scratch;
    long long split_bytes;
    struct SplitInfo* split_info;
    int split_slots;   // row areas in the pool (at most kSplitSlots)
    // Per seed of a split point (kEarlyMax * kSplitSeeds): the block that
    // completes a seed's second half (the seed's counter at
    // ir_count[kSeedCounter + point * kSplitSeeds + seed]) merges the halves,
    // runs the seed's gap repairs and leaves its rows in the up half's area.
    struct SeedInfo* seed_info;
    // Row-key generations of this launch's scans start above gen_base, so a
    // launch whose blocks reuse scratch areas that an earlier launch of the
    // same epoch scanned in (the side stream's blocks joining the early pass
    // in the second pass's areas) never takes that launch's rows for its own.
    unsigned gen_base;
};

constexpr int kEarlyMax = 512;

// One unit of a split early point: what its half scan left.
struct SplitInfo {
    double area;              // the half's image_area value
    unsigned long long rays;  // its inside cells
    int yi_final;             // the scan's row index when it returned
    int pred;                 // down half: index of the predecessor row (rows the first row's scan completed)
    int ok;                   // 1: the point, seed and scan exist and fit the unit's rows
    int slot;                 // its row scratch area
    double row0[3];           // down half: xmin, xmax and y of the first row of the up scan
};

// One seed of a split point after its gap repairs.
struct SeedInfo {
    double areai;             // the seed's area
    double max_jump;          // its rows' largest jump, in cells
    unsigned long long rays;  // its inside cells
    int nyi;                  // rows [0, nyi] in the up half's area: the walk's row count
    int repairs;              // its gap repairs
    int ok;                   // 1: complete; 0: the finishing block scans the seed itself
    int pad;
};
constexpr int kSplitSeeds = 6;
constexpr int kSplitUnits = kEarlyMax * kSplitSeeds * 2;  // SplitInfo entries
constexpr int kSplitSlots = 256;                           // unit row scratch areas (see split_slots)
constexpr int kSplitRowCap = 32768;
// The counters array: ir_count [0, 8), next_item [8, 16), the route's
// candidate count [48], the unit slots taken [kSplitAlloc], early_cart
// [kEarlyOff, kEarlyOff + kEarlyMax), completed seeds per early point
// [kSplitCounter, kSplitCounter + kEarlyMax), completed halves per seed
// [kSeedCounter, kSeedCounter + kEarlyMax * kSplitSeeds).
constexpr int kSplitAlloc = 49;
constexpr int kEarlyOff = 64;
constexpr int kSplitCounter = kEarlyOff + kEarlyMax;
constexpr int kSeedCounter = kSplitCounter + kEarlyMax;
constexpr int kCounterInts = kSeedCounter + kEarlyMax * kSplitSeeds;
constexpr int kEarlyWarps = 4;     // warps per block of the early pass (one block per SM: its LD table)
constexpr int kEarlyBlocks = 96;   // blocks of the early pass

constexpr int kBigWarps = 8;

cudaError_t launch_ld_tables(const double2* coeffs, int n_tables, double* tables, cudaStream_t stream);
// needed (optional): models whose flag is 0 are not sampled.  critical_points:
// track the critical-curve roots themselves (lens frame) instead of their
// images on the source plane.
cudaError_t launch_caustics(CausticModel* models, int n_models, int max_bins, const double2* phases,
                            const long long* raw_offset, P2* raw, P2* branches, cudaStream_t stream,
                            const unsigned char* needed = nullptr, bool critical_points = false);
// Points (rho > 0, finite_mode > 0) whose source is outside the outer caustic
// box (caustic_outer_box) by the decision's margin get kItemOutsideBox; the
// others set needed[model_base[i / pass] + model].  needed must be zeroed.
cudaError_t launch_certify(FsItem* items, long long n, const FsSettingsDev* settings, const int* model_base, int pass,
                           unsigned char* needed, int sm_count, cudaStream_t stream);
cudaError_t launch_decide(const FsWork& w, int sm_count, cudaStream_t stream);
cudaError_t launch_seeds(const FsWork& w, int sm_count, cudaStream_t stream, long long* cand_keys, P2* cand_probes,
                         int n_warps);
cudaError_t launch_cartesian(const FsWork& w, int n_warps, cudaStream_t stream, unsigned long long epoch);
// Picks the early Cartesian points (predicted in-source cells
// pi nbin^2 max(|A_ps|, 1) above min_cells), at most kEarlyMax, largest first,
// into w.early_cart and ir_count[5]; `cand` holds route_bytes() of candidates,
// counted in ir_count[48] (zero beforehand).
constexpr int kRouteCands = 1024;
size_t route_bytes();
cudaError_t launch_route_early(const FsWork& w, double min_cells, void* cand, int max_points, int sm_count,
                               cudaStream_t stream);
cudaError_t launch_polar(const FsWork& w, int n_warps, cudaStream_t stream, unsigned long long epoch);
// Tile-parallel polar flood fill of every polar point of the work lists
// (first pass); points that do not fit go to the second-pass retry list.
cudaError_t launch_polar_tiles(const FsWork& w, void* area, long long capacity, int max_items, int flood_blocks,
                               cudaStream_t stream);
size_t tile_bytes(long long capacity, int max_items);
int polar_tile_blocks_per_sm();
size_t seed_candidate_bytes_per_warp(int cand_cap);
// Block seeding pass over w.retry_seeds: n_blocks blocks of kBigWarps warps.
cudaError_t launch_seeds_blocks(const FsWork& w, int n_blocks, cudaStream_t stream);
// Adjoint: dA/d(y1, y2, s, q, rho, c), the value differentiated and the method
// of every point of the work lists (8 doubles per point).
cudaError_t launch_grad(const FsWork& w, void* area, long long capacity, int max_items, int flood_blocks,
                        int grad_bins, int sm_count, double* grads, cudaStream_t stream);
size_t grad_tile_bytes(long long capacity, int max_items);
int grad_flood_blocks_per_sm();
size_t cartesian_scratch_bytes(int row_cap, int seed_cap);
size_t polar_scratch_bytes(int queue_cap, int hash_cap);

// Source positions of static-binary light curves in VBM convention
// (python/lcbinint_pybind.cpp:1140-1157): one item per epoch.
struct LcModel {
    double t0, tE, u0, cos_alpha, sin_alpha, s, q_core, rho;
    long long first;  // first epoch index in the times array
    int count;
    int settings;
    int model;        // caustic model index
    int pad;
};
cudaError_t launch_lc_items(const LcModel* models, int n_models, const double* times, FsItem* items,
                            long long n_items, cudaStream_t stream);
// What an inverse-ray point needs after its pass of the deferred pipeline:
// its caustic model copied from the pass's tables into the inverse-ray store
// (jobs), and the point's model index pointed at the copy (remaps).
struct StashJob {
    int src_model;          // index in the pass's model table
    int dst_model;          // index in the store
    long long dst_offset;   // first branch point of the copy in the store
};
struct StashRemap {
    long long item;         // index of the point in the whole batch
    int dst_model;
    int pad;
};
cudaError_t launch_stash(const CausticModel* src_models, const P2* src_branches, const StashJob* jobs, int n_jobs,
                         CausticModel* dst_models, P2* dst_branches, const StashRemap* remaps, int n_remaps,
                         FsItem* items, cudaStream_t stream);
// a_ps and image count per item from binary_images (rho > 0) or binary_mag0
// (rho == 0), written into the items and into a_ps[n], nimg[n].
cudaError_t launch_item_images(FsItem* items, long long n, double* a_ps, int* nimg, int sm_count, cudaStream_t stream);
// Per-epoch gradients of light curves, (t0, tE, u0, alpha, s, q, rho, Gamma),
// from the per-point gradients of launch_grad; `rho_sign` per model.
cudaError_t launch_unpack_results(const FsOut* out, double* A, int* method, int* status, long long n,
                                  cudaStream_t stream);
cudaError_t launch_lc_grad_chain(const LcModel* models, int n_models, const double* times, const double* point_grads,
                                 double* grads, long long n_items, cudaStream_t stream);

} // namespace lcbi
