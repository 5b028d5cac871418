// Image seeding for inverse-ray integration, one warp per evaluation:
// augmented_image_seeds (finite_source_magnifier.cpp:1709-1871) followed by
// augment_seeds_from_caustic_branches (:4845-4926), as fixed_inverse_ray_binary
// runs them (:3055-3064).
//
// The reference's seed list is built by a long serial loop of small root
// solves.  Here the solves are batched across lanes -- 32 critical-curve
// phases or 32 probe positions at a time -- and the serial bookkeeping (seed
// de-duplication against the list as it stood before each probe, early exits
// on the seed count) is replayed in the reference's order over the batched
// results, so the final list is identical element by element.
#include "lcbi_fs_kernels.h"
#include "lcbi_warp.cuh"

namespace lcbi {

namespace {

constexpr int kPhaseSamples = 1400;  // FSM:1741
constexpr int kSkip = 40;            // FSM:1745
constexpr int kMaxBoundarySeeds = 128;


// Caustic-branch probe candidates per warp: at most one per sampled caustic
// point, so 4 x caustic_bins (FsWork::cand_cap) always suffices.

struct WarpShared {
    P2 img[32][5];
    int cnt[32];
    int n_cand;
};

struct SeedState {
    P2* seeds;
    int cap;
    int n;
    bool ovf;
    P2 src;
    double rho, rho2;
    double s, q;
    Mapper m;
    WarpShared* sh;
};

__device__ __forceinline__ void push_seed(SeedState& S, P2 v)
{
    if (lane_id() == 0 && S.n < S.cap) S.seeds[S.n] = v;
    S.n += 1;
    if (S.n > S.cap) S.ovf = true;
    __syncwarp();
}

__device__ __forceinline__ bool probe_in_disk(const SeedState& S, P2 p)
{
    return !(S.rho <= 0.0 || dist2(p, S.src) >= S.rho2 * (1.0 + 1.0e-10));
}

// Each active lane solves the lens quintic at its probe and keeps the
// candidates with residual^2 < 1e-12 (selected_point_images, FSM:1873-1889).
__device__ __forceinline__ void probe_batch(SeedState& S, P2 probe, bool active)
{
    const int lane = lane_id();
    int k = 0;
    if (active) {
        const BinaryGeom g = make_geom(S.s, S.q, probe.x, probe.y);
        dc pos[5];
        double res[5], det[5];
        const int nphys = (S.s == 0.0 || S.q <= 0.0) ? -1 : image_candidates(g, pos, res, det);
        if (nphys > 0) {
#pragma unroll
            for (int i = 0; i < 5; ++i) {
                if (res[i] * res[i] < 1.0e-12) S.sh->img[lane][k++] = P2{pos[i].re, pos[i].im};
            }
        }
    }
    S.sh->cnt[lane] = k;
    __syncwarp();
}

// append_valid_probe_image_seeds (FSM:1449-1498) on one probe's k candidate
// images (shared memory, read by the whole warp).
__device__ void replay_images(SeedState& S, int k, const P2* imgs)
{
    if (k <= 3) return;
    const int before = S.n;
    const int lim = before < S.cap ? before : S.cap;
    for (int j = 0; j < k; ++j) {
        const P2 img = imgs[j];
        const double md2 = dist2(map_real(S.m, img.x, img.y), S.src);
        if (md2 > S.rho2 * (1.0 + 1.0e-8)) continue;
        int first = -1;
        for (int base = 0; base < lim; base += 32) {
            const int si = base + lane_id();
            const bool hit = si < lim && dist2(img, S.seeds[si]) < 0.0625 * S.rho2;
            const unsigned b = __ballot_sync(kFull, hit);
            if (b) {
                first = base + __ffs(b) - 1;
                break;
            }
        }
        if (first >= 0) {
            const P2 e = S.seeds[first];
            const double ed2 = dist2(map_real(S.m, e.x, e.y), S.src);
            if (md2 + 1.0e-16 < ed2) {
                if (lane_id() == 0) S.seeds[first] = img;
                __syncwarp();
            }
        } else {
            push_seed(S, img);
        }
    }
}

// The same on the solved batch slot `l`.
__device__ __forceinline__ void replay_probe(SeedState& S, int l) { replay_images(S, S.sh->cnt[l], S.sh->img[l]); }

// append_caustic_probe_image_seeds (FSM:1500-1563).
__device__ void caustic_probe(SeedState& S, P2 cs, const TrigTables& trig)
{
    const double dx = cs.x - S.src.x;
    const double dy = cs.y - S.src.y;
    const double dist = hypot_borges(dx, dy);
    if (dist <= 0.0 || dist >= S.rho) return;
    const double ux = dx / dist;
    const double uy = dy / dist;
    const int lane = lane_id();
    {
        const double steps[4] = {0.02 * S.rho, 0.05 * S.rho, 0.15 * S.rho, 0.35 * S.rho};
        P2 p{0.0, 0.0};
        bool act = false;
        if (lane < 8) {
            const double st = steps[lane >> 1];
            p = (lane & 1) ? P2{cs.x - ux * st, cs.y - uy * st} : P2{cs.x + ux * st, cs.y + uy * st};
            act = probe_in_disk(S, p);
        }
        const unsigned am = __ballot_sync(kFull, act);
        probe_batch(S, p, act);
        for (int l = 0; l < 8; ++l)
            if (am & (1u << l)) replay_probe(S, l);
    }
    if (S.n <= 3) {
        const double radial[5] = {0.02 * S.rho, 0.05 * S.rho, 0.10 * S.rho, 0.20 * S.rho, 0.35 * S.rho};
        for (int base = 0; base < 80; base += 32) {
            const int idx = base + lane;
            P2 p{0.0, 0.0};
            bool act = false;
            if (idx < 80) {
                const double st = radial[idx >> 4];
                const double2 cssn = trig.angular[idx & 15];
                p = P2{cs.x + st * cssn.x, cs.y + st * cssn.y};
                act = probe_in_disk(S, p);
            }
            const unsigned am = __ballot_sync(kFull, act);
            probe_batch(S, p, act);
            for (int l = 0; l < 32 && base + l < 80; ++l) {
                if (am & (1u << l)) replay_probe(S, l);
                if (S.n > 3) return;
            }
        }
    }
}

// Critical-curve source points at an arbitrary phase (golden-section refine only).
__device__ double nearest_critical(SeedState& S, double phi, P2* nearest)
{
    double sn, cs;
    sincos(phi, &sn, &cs);
    dc roots[4];
    critical_roots(S.s, S.q, dc{cs, sn}, roots);
    double best = dinf();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const P2 c = map_real(S.m, roots[k].re, roots[k].im);
        const double d2 = dist2(c, S.src);
        if (d2 < best) {
            best = d2;
            *nearest = c;
        }
    }
    return best;
}

// refine_nearest_critical_source (FSM:1666-1707).
__device__ P2 refine_critical(SeedState& S, double center, double step)
{
    double left = center - step;
    double right = center + step;
    const double g = 0.61803398874989484820;
    double x1 = right - g * (right - left);
    double x2 = left + g * (right - left);
    P2 n1{0.0, 0.0}, n2{0.0, 0.0};
    double f1 = nearest_critical(S, x1, &n1);
    double f2 = nearest_critical(S, x2, &n2);
    for (int it = 0; it < 32; ++it) {
        if (f1 > f2) {
            left = x1;
            x1 = x2;
            f1 = f2;
            n1 = n2;
            x2 = left + g * (right - left);
            f2 = nearest_critical(S, x2, &n2);
        } else {
            right = x2;
            x2 = x1;
            f2 = f1;
            n2 = n1;
            x1 = right - g * (right - left);
            f1 = nearest_critical(S, x1, &n1);
        }
    }
    return f1 < f2 ? n1 : n2;
}

// Probes on a circle of radius pr about the source, in table order, stopping
// when `limit` seeds exist (limit <= 0: no limit).
__device__ void ring_probes(SeedState& S, double pr, const double2* table, int count, int limit)
{
    for (int base = 0; base < count; base += 32) {
        if (limit > 0 && !(S.n < limit)) return;
        const int i = base + lane_id();
        P2 p{0.0, 0.0};
        bool act = false;
        if (i < count) {
            const double2 t = table[i];
            p = P2{S.src.x + pr * t.x, S.src.y + pr * t.y};
            act = probe_in_disk(S, p);
        }
        const unsigned am = __ballot_sync(kFull, act);
        probe_batch(S, p, act);
        for (int l = 0; l < 32 && base + l < count; ++l) {
            if (limit > 0 && !(S.n < limit)) return;
            if (am & (1u << l)) replay_probe(S, l);
        }
    }
}

// augment_seeds_from_caustic_branches (FSM:4845-4926).
__device__ void augment_from_branches(SeedState& S, const CausticModel& md, const P2* __restrict__ br,
                                      long long* cand_key, P2* cand_probe, int kCandCap)
{
    if (S.n >= 5) return;
    const double R = S.rho + md.max_seg_len;
    const int ix0 = grid_cell(S.src.x - R, md.min_x, md.step_x), ix1 = grid_cell(S.src.x + R, md.min_x, md.step_x);
    const int iy0 = grid_cell(S.src.y - R, md.min_y, md.step_y), iy1 = grid_cell(S.src.y + R, md.min_y, md.step_y);
    const int bins = md.bins;
    if (lane_id() == 0) S.sh->n_cand = 0;
    __syncwarp();
    for (int t = lane_id(); t < 4 * bins; t += 32) {
        const int b = t / bins;
        const int pos = t - b * bins;
        if (bins < 2) continue;
        const int next = (pos + 1) % bins;
        if (next == 0) continue;
        const P2 p0 = br[(long long)b * bins + pos];
        const int ix = grid_cell(p0.x, md.min_x, md.step_x);
        const int iy = grid_cell(p0.y, md.min_y, md.step_y);
        if (ix < ix0 || ix > ix1 || iy < iy0 || iy > iy1) continue;
        const P2 p1 = br[(long long)b * bins + next];
        if (seg_dist(S.src, p0, p1) >= S.rho) continue;
        const double sx = p1.x - p0.x;
        const double sy = p1.y - p0.y;
        const double l2 = sx * sx + sy * sy;
        const double tt =
            l2 > 0.0 ? clampd(((S.src.x - p0.x) * sx + (S.src.y - p0.y) * sy) / l2, 0.0, 1.0) : 0.0;
        const P2 nearest{p0.x + tt * sx, p0.y + tt * sy};
        const double dist = sqrt(dist2(nearest, S.src));
        if (dist <= 0.0 || dist >= S.rho) continue;
        const double step = S.rho * 0.05 / dist;
        const P2 probe{nearest.x + (nearest.x - S.src.x) * step, nearest.y + (nearest.y - S.src.y) * step};
        if (dist2(probe, S.src) >= S.rho * S.rho) continue;
        const int slot = atomicAdd(&S.sh->n_cand, 1);
        if (slot < kCandCap) {
            // Visiting order of the reference: bucket (row-major), then branch, then position.
            cand_key[slot] = ((long long)(iy * kCausticGrid + ix) << 32) | (long long)(b * bins + pos);
            cand_probe[slot] = probe;
        }
    }
    __syncwarp();
    int nc = S.sh->n_cand;
    if (nc > kCandCap) {
        S.ovf = true;
        nc = kCandCap;
    }
    if (nc == 0) return;
    // Rank sort of the (unique) keys into visiting order.
    long long* sorted_key = cand_key + kCandCap;
    P2* sorted_probe = cand_probe + kCandCap;
    for (int i = lane_id(); i < nc; i += 32) {
        const long long k = cand_key[i];
        int rank = 0;
        for (int j = 0; j < nc; ++j) rank += (cand_key[j] < k) ? 1 : 0;
        sorted_key[rank] = k;
        sorted_probe[rank] = cand_probe[i];
    }
    __syncwarp();
    long long prev_cell = -1;
    for (int base = 0; base < nc; base += 32) {
        const int i = base + lane_id();
        probe_batch(S, i < nc ? sorted_probe[i] : P2{0.0, 0.0}, i < nc);
        for (int l = 0; l < 32 && base + l < nc; ++l) {
            const long long cell = sorted_key[base + l] >> 32;
            if (cell != prev_cell) {
                if (S.n >= 5) return;
                prev_cell = cell;
            }
            const int k = S.sh->cnt[l];
            if (k > S.n) {
                if (lane_id() < k) S.seeds[lane_id()] = S.sh->img[l][lane_id()];
                S.n = k;
                __syncwarp();
            }
        }
    }
}

// Scan position pp of the interleaved caustic-crossing phase scan -> phase sample (FSM:1757-1787).
__device__ __forceinline__ int phase_sample(int pp)
{
    return (pp % (kPhaseSamples / kSkip)) * kSkip + pp / (kPhaseSamples / kSkip);
}

__device__ __forceinline__ void init_state(SeedState& S, const FsWork& w, int k, const FsItem& item, WarpShared* sh)
{
    S.seeds = w.seeds + (long long)k * w.seed_cap;
    S.cap = w.seed_cap;
    S.n = 0;
    S.ovf = false;
    S.src = P2{item.x, item.y};
    S.rho = item.rho;
    S.rho2 = item.rho * item.rho;
    S.s = item.s;
    S.q = item.q;
    S.m = make_mapper(item.s, item.q);
    S.sh = sh;
}

// Point images at the source centre (binary_images, point_source_magnifier.cpp:723-737).
// As seed hints (LensModel, lens_model.cpp:209-226) only the images that
// map inside the source are kept (append_valid_seed, FSM:1430-1447), all
// of them if none does (FSM:1722-1727).
__device__ void initial_seeds(SeedState& S, const FsItem& item)
{
    int cnt = 0;
    if (lane_id() == 0 && item.s != 0.0 && item.q > 0.0) {
        const BinaryGeom g = make_geom(item.s, item.q, item.x, item.y);
        dc pos[5];
        double res[5], det[5];
        const int all = image_candidates(g, pos, res, det);
        if (item.flags & kItemSeedHints) {
            for (int i = 0; i < all; ++i) {
                if (!(S.rho > 0.0)) break;
                const P2 mp = map_real(S.m, pos[i].re, pos[i].im);
                if (dist2(mp, S.src) > S.rho2 * (1.0 + 1.0e-8)) continue;
                S.seeds[cnt++] = P2{pos[i].re, pos[i].im};
            }
        }
        if (cnt == 0) {
            for (int i = 0; i < all; ++i) S.seeds[i] = P2{pos[i].re, pos[i].im};
            cnt = all;
        }
    }
    S.n = shfl_i(cnt, 0);
    __syncwarp();
}

// Everything after the caustic-crossing phase scan, on one warp: the refined
// nearest critical source, the boundary and interior probe rings, the
// caustic-branch augmentation, and the point's seed count.
__device__ void finish_seeding(SeedState& S, const FsWork& w, int it, const CausticModel& md, bool found,
                               double best_d2, double best_phase, long long* ck, P2* cp, long long t_item)
{
    if (S.rho > 0.0) {
        const double phase_step = 2.0 * kPi / static_cast<double>(kPhaseSamples);
        if (!found && best_d2 < S.rho2 && best_d2 > 0.0) {
            caustic_probe(S, refine_critical(S, best_phase, phase_step), w.trig);
        }
        // Phase 2 (FSM:1800-1865) is not run: its branches start at the
        // sentinel (1e30, 1e30), whose squared distance to any finite
        // critical source (about 2e60) never beats the initial bound 1e60,
        // so no branch is ever assigned and the scan adds no seed.
        if (S.n < kMaxBoundarySeeds) ring_probes(S, S.rho * (1.0 - 0.02), w.trig.boundary, 400, kMaxBoundarySeeds);
        if (S.rho >= 2.0e-2) {
            const double fr[3] = {0.25, 0.5, 0.75};
            for (int r = 0; r < 3; ++r) ring_probes(S, S.rho * fr[r], w.trig.interior, 64, 0);
        }
    }
    augment_from_branches(S, md, w.branches + md.branch_offset, ck, cp, w.cand_cap);
    if (lane_id() == 0) {
        FsOut* o = w.out + it;
        o->n_seeds = S.n;
        if (S.ovf) o->status = kFsSeedOverflow;
        if (w.cycles) w.cycles[it] = clock64() - t_item;
    }
    __syncwarp();
}

// ----- block seeding pass -----
//
// A point whose disk holds much of a caustic probes every critical source
// inside it (8 probes, and 80 more while at most three seeds exist), one
// source after another; on one warp that is four rounds of lens-quintic
// solves per source.  The block pass computes the critical sources of all
// scan positions at once, then the probes of kWinSources consecutive
// in-disk sources at a time on all its warps, while warp 0 replays the
// reference's sequential bookkeeping over the solved probes in the
// reference's order (caustic_probe's early exits included), so the seed list
// is the same element by element.  Probes solved for sources after the scan
// stopped are discarded.

constexpr int kScanPositions = kPhaseSamples * 4;
constexpr int kWinSources = 8;
constexpr int kProbesPerSource = 88;  // 8 along the caustic normal, 80 on rings (FSM:1500-1563)
constexpr int kWinProbes = kWinSources * kProbesPerSource;
constexpr int kCmdWindow = 1, kCmdDone = 2;

struct BlockSeedShared {
    P2 cs[kPhaseSamples * 4];   // critical source of scan position pp, root i at pp * 4 + i
    P2 img[kWinProbes][5];      // the window's probe images
    int cnt[kWinProbes];        // their counts; -1: probe not taken (outside the disk)
    int win[kWinSources];       // scan positions of the window's sources
    int n_win;
    int cmd;
    int item;
    WarpShared warp0;
};

// Named barrier 1 between warp 0 (replay) and the other warps (window
// solves); the two sides reach it from different places, so it is the
// unaligned form.
__device__ __forceinline__ void window_barrier() { asm volatile("barrier.sync 1;" ::: "memory"); }

// Probe j of window source m, as caustic_probe forms and solves it.
__device__ void window_probe(const SeedState& S, BlockSeedShared& B, int m, int j, const TrigTables& trig)
{
    const P2 cs = B.cs[B.win[m]];
    const double dx = cs.x - S.src.x;
    const double dy = cs.y - S.src.y;
    const double dist = hypot_borges(dx, dy);
    const int slot = m * kProbesPerSource + j;
    int k = -1;
    if (dist > 0.0 && dist < S.rho) {
        P2 p;
        if (j < 8) {
            const double steps[4] = {0.02 * S.rho, 0.05 * S.rho, 0.15 * S.rho, 0.35 * S.rho};
            const double ux = dx / dist;
            const double uy = dy / dist;
            const double st = steps[j >> 1];
            p = (j & 1) ? P2{cs.x - ux * st, cs.y - uy * st} : P2{cs.x + ux * st, cs.y + uy * st};
        } else {
            const int idx = j - 8;
            const double radial[5] = {0.02 * S.rho, 0.05 * S.rho, 0.10 * S.rho, 0.20 * S.rho, 0.35 * S.rho};
            const double st = radial[idx >> 4];
            const double2 cssn = trig.angular[idx & 15];
            p = P2{cs.x + st * cssn.x, cs.y + st * cssn.y};
        }
        if (probe_in_disk(S, p)) {
            k = 0;
            const BinaryGeom g = make_geom(S.s, S.q, p.x, p.y);
            dc pos[5];
            double res[5], det[5];
            const int nphys = (S.s == 0.0 || S.q <= 0.0) ? -1 : image_candidates(g, pos, res, det);
            if (nphys > 0) {
#pragma unroll
                for (int i = 0; i < 5; ++i) {
                    if (res[i] * res[i] < 1.0e-12) B.img[slot][k++] = P2{pos[i].re, pos[i].im};
                }
            }
        }
    }
    B.cnt[slot] = k;
}

// caustic_probe (FSM:1500-1563) of window source m on its solved probes (warp 0).
__device__ void replay_source(SeedState& S, const BlockSeedShared& B, int m)
{
    const P2 cs = B.cs[B.win[m]];
    const double dist = hypot_borges(cs.x - S.src.x, cs.y - S.src.y);
    if (dist <= 0.0 || dist >= S.rho) return;
    const int base = m * kProbesPerSource;
    for (int l = 0; l < 8; ++l)
        if (B.cnt[base + l] >= 0) replay_images(S, B.cnt[base + l], B.img[base + l]);
    if (S.n <= 3) {
        for (int idx = 0; idx < 80; ++idx) {
            const int sl = base + 8 + idx;
            if (B.cnt[sl] >= 0) replay_images(S, B.cnt[sl], B.img[sl]);
            if (S.n > 3) return;
        }
    }
}

__device__ __forceinline__ bool in_disk_source(const SeedState& S, P2 cs)
{
    const double d2 = dist2(cs, S.src);
    return !(d2 >= S.rho2 || d2 <= 0.0);
}

} // namespace

__global__ void __launch_bounds__(128) seeds_kernel(FsWork w, long long* cand_keys, P2* cand_probes)
{
    extern __shared__ __align__(16) unsigned char smem[];
    WarpShared* sh = reinterpret_cast<WarpShared*>(smem) + warp_in_block();
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long* ck = cand_keys + (long long)gw * 2 * w.cand_cap;
    P2* cp = cand_probes + (long long)gw * 2 * w.cand_cap;
    const int n_cart = w.ir_count[0];
    const int total = n_cart + w.ir_count[1];
    const bool can_hand_over = w.seed_block_after > 0 && w.retry_seeds != nullptr;
    for (;;) {
        int k = 0;
        if (lane_id() == 0) {
            if (w.seed_slots != nullptr) {
                const int idx = atomicAdd(w.seed_next, 1);
                k = idx < *w.seed_count ? w.seed_slots[idx] : total;
            } else {
                k = atomicAdd(&w.next_item[0], 1);
            }
        }
        k = shfl_i(k, 0);
        if (k >= total) break;
        if (w.seed_skip_early && k < n_cart) {
            // Seeded on the early stream, with the early block pass.
            const int ne = w.ir_count[5];
            bool routed = false;
            for (int e = 0; e < ne; ++e) routed |= w.early_cart[e] == k;
            if (routed) continue;
        }
        const int it = (k < n_cart) ? w.ir_cart[k] : w.ir_polar[k - n_cart];
        const long long t_item = clock64();
        const FsItem item = w.items[it];
        const CausticModel md = w.models[item.model];
        SeedState S;
        init_state(S, w, k, item, sh);
        initial_seeds(S, item);
        double best_d2 = dinf();
        double best_phase = 0.0;
        bool found = false;
        bool hand_over = false;
        if (S.rho > 0.0) {
            // Phase 1: interleaved phase scan for the first caustic crossing (FSM:1757-1787).
            const double phase_step = 2.0 * kPi / static_cast<double>(kPhaseSamples);
            int reached = 0;  // critical sources inside the disk met so far
            for (int p0 = 0; p0 < kPhaseSamples && !found && !hand_over; p0 += 32) {
                const int pl = p0 + lane_id();
                P2 c[4];
                if (pl < kPhaseSamples) {
                    const double2 ph = w.trig.seed_phase[phase_sample(pl)];
                    dc roots[4];
                    critical_roots(S.s, S.q, dc{ph.x, ph.y}, roots);
#pragma unroll
                    for (int i = 0; i < 4; ++i) c[i] = map_real(S.m, roots[i].re, roots[i].im);
                }
                for (int l = 0; l < 32 && p0 + l < kPhaseSamples && !found && !hand_over; ++l) {
                    const int pp = p0 + l;
                    const double phi = phase_step * static_cast<double>(phase_sample(pp));
                    for (int i = 0; i < 4; ++i) {
                        const P2 cs{shfl_d(c[i].x, l), shfl_d(c[i].y, l)};
                        const double d2 = dist2(cs, S.src);
                        if (d2 < best_d2) {
                            best_d2 = d2;
                            best_phase = phi;
                        }
                        if (d2 >= S.rho2 || d2 <= 0.0) continue;
                        if (can_hand_over && ++reached >= w.seed_block_after) {
                            hand_over = true;
                            break;
                        }
                        const int before = S.n;
                        caustic_probe(S, cs, w.trig);
                        found = S.n > before;
                    }
                }
            }
        }
        if (hand_over) {
            // The block pass seeds the point again from the start.
            if (lane_id() == 0) w.retry_seeds[atomicAdd(&w.ir_count[4], 1)] = k;
            __syncwarp();
            continue;
        }
        finish_seeding(S, w, it, md, found, best_d2, best_phase, ck, cp, t_item);
    }
}

__global__ void __launch_bounds__(32 * kBigWarps, 1) seeds_block_kernel(FsWork w)
{
    extern __shared__ __align__(16) unsigned char smem[];
    BlockSeedShared& B = *reinterpret_cast<BlockSeedShared*>(smem);
    const int t = threadIdx.x;
    const int nt = blockDim.x;
    long long* ck = reinterpret_cast<long long*>(w.seed_scratch + (long long)blockIdx.x * w.seed_scratch_per_block);
    P2* cp = reinterpret_cast<P2*>(ck + 2 * (long long)w.cand_cap);
    const int n = w.ir_count[4];
    const int n_cart = w.ir_count[0];
    for (;;) {
        __syncthreads();
        if (t == 0) B.item = atomicAdd(&w.next_item[5], 1);
        __syncthreads();
        const int r = B.item;
        if (r >= n) break;
        const int k = w.retry_seeds[r];
        const int it = (k < n_cart) ? w.ir_cart[k] : w.ir_polar[k - n_cart];
        const long long t_item = clock64();
        const FsItem item = w.items[it];
        SeedState S;
        init_state(S, w, k, item, &B.warp0);
        // Critical sources of every scan position, all threads.
        for (int pp = t; pp < kPhaseSamples; pp += nt) {
            const double2 ph = w.trig.seed_phase[phase_sample(pp)];
            dc roots[4];
            critical_roots(S.s, S.q, dc{ph.x, ph.y}, roots);
#pragma unroll
            for (int i = 0; i < 4; ++i) B.cs[pp * 4 + i] = map_real(S.m, roots[i].re, roots[i].im);
        }
        __syncthreads();
        if (warp_in_block() != 0) {
            // Window solves on request of warp 0.
            for (;;) {
                window_barrier();
                if (B.cmd == kCmdDone) break;
                for (int g = t; g < B.n_win * kProbesPerSource; g += nt)
                    window_probe(S, B, g / kProbesPerSource, g % kProbesPerSource, w.trig);
                window_barrier();
            }
            continue;
        }
        const CausticModel md = w.models[item.model];
        initial_seeds(S, item);
        double best_d2 = dinf();
        double best_phase = 0.0;
        bool found = false;
        if (S.rho > 0.0) {
            const double phase_step = 2.0 * kPi / static_cast<double>(kPhaseSamples);
            int win_end = 0;  // scan positions before win_end that lie in the disk are in the window
            int m = 0;        // window source the replay is at
            for (int pp = 0; pp < kPhaseSamples && !found; ++pp) {
                const double phi = phase_step * static_cast<double>(phase_sample(pp));
                for (int i = 0; i < 4; ++i) {
                    const int pos = pp * 4 + i;
                    const P2 cs = B.cs[pos];
                    const double d2 = dist2(cs, S.src);
                    if (d2 < best_d2) {
                        best_d2 = d2;
                        best_phase = phi;
                    }
                    if (d2 >= S.rho2 || d2 <= 0.0) continue;
                    if (pos >= win_end) {
                        // The next kWinSources in-disk sources from pos on, in scan order.
                        int nw = 0, last_pos = pos;
                        for (int q = pos; q < kScanPositions && nw < kWinSources; q += 32) {
                            const int qq = q + lane_id();
                            const bool in = qq < kScanPositions && in_disk_source(S, B.cs[qq]);
                            unsigned bal = __ballot_sync(kFull, in);
                            while (__popc(bal) > kWinSources - nw) bal &= ~(1u << (31 - __clz(bal)));
                            if ((bal >> lane_id()) & 1u) B.win[nw + __popc(bal & ((1u << lane_id()) - 1u))] = qq;
                            if (bal) last_pos = q + 31 - __clz(bal);
                            nw += __popc(bal);
                        }
                        // In-disk positions before win_end are all in the window.
                        win_end = nw == kWinSources ? last_pos + 1 : kScanPositions;
                        if (lane_id() == 0) {
                            B.n_win = nw;
                            B.cmd = kCmdWindow;
                        }
                        __syncwarp();
                        window_barrier();
                        for (int g = t; g < nw * kProbesPerSource; g += nt)
                            window_probe(S, B, g / kProbesPerSource, g % kProbesPerSource, w.trig);
                        window_barrier();
                        m = 0;
                    }
                    while (m + 1 < B.n_win && B.win[m] != pos) ++m;
                    const int before = S.n;
                    replay_source(S, B, m);
                    found = S.n > before;
                }
            }
        }
        if (lane_id() == 0) B.cmd = kCmdDone;
        __syncwarp();
        window_barrier();
        finish_seeding(S, w, it, md, found, best_d2, best_phase, ck, cp, t_item);
    }
}

cudaError_t launch_seeds(const FsWork& w, int sm_count, cudaStream_t stream, long long* cand_keys,
                         P2* cand_probes, int n_warps)
{
    const int blocks = (n_warps + 3) / 4;
    const size_t smem = 4 * sizeof(WarpShared);
    seeds_kernel<<<blocks, 128, smem, stream>>>(w, cand_keys, cand_probes);
    (void)sm_count;
    return cudaGetLastError();
}

cudaError_t launch_seeds_blocks(const FsWork& w, int n_blocks, cudaStream_t stream)
{
    const int smem = static_cast<int>(sizeof(BlockSeedShared));
    cudaError_t e = cudaFuncSetAttribute(seeds_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    seeds_block_kernel<<<n_blocks, 32 * kBigWarps, smem, stream>>>(w);
    return cudaGetLastError();
}

size_t seed_candidate_bytes_per_warp(int cand_cap) { return (size_t)2 * cand_cap * (sizeof(long long) + sizeof(P2)); }

} // namespace lcbi
