// Polar inverse ray as a tile-parallel flood fill over the whole GPU
// (inverse_ray_polar_boundary_binary, finite_source_magnifier.cpp:1156-1319).
//
// The cells the reference's polar BFS counts are exactly the inside cells
// 4-connected (r +- 1 with r >= 0, phi +- 1 periodic) to the starting cells of
// the seeds (see fs_polar.cu).  That set does not depend on the order of the
// visits, so it is computed here on 32 x 32 tiles of the (r, phi) lattice by
// every warp of the GPU at once, for every polar point of the batch together:
//   * a tile is processed by one warp, lane j owning phi row j of the tile.
//     On its first visit the 1,024 cells are evaluated (each lane sweeps its
//     row, whose sine and cosine are computed once) into a 32-bit inside mask
//     per row;
//   * pending entry cells, ORed in by neighbouring tiles, seed an in-tile
//     closure: Kogge-Stone occluded fills along r inside each row word,
//     alternating with phi steps through warp shuffles, until nothing changes;
//   * newly visited cells (atomicOr on the visited words) are summed, and the
//     ones on a tile edge are ORed into the neighbouring tile's entry words,
//     queuing that tile if it is not queued already;
//   * tiles live in a hash table keyed by (point, phi tile, r tile) and in one
//     global ticketed FIFO; persistent warps pop tiles until no tile is queued
//     or in process.
// Sums are accumulated exactly (128-bit fixed point), so the magnification is
// identical to the one-warp and block flood fills.  A point whose tiles do not
// fit the table is handed to the block flood fill of the second pass.
#include "lcbi_fs_kernels.h"
#include "lcbi_group.cuh"
#include "lcbi_trig.cuh"

#include <cstdint>

namespace lcbi {

namespace {

constexpr int kKeyBits = 25;                      // bits of each tile coordinate in a key
constexpr unsigned long long kKeyMask = (1ull << kKeyBits) - 1;
constexpr int kMaxProbe = 4096;
constexpr unsigned kSpinLimit = 1u << 25;         // bounded waits (seconds with the sleeps below)

struct TileSlot {
    unsigned long long key;   // 0: empty; else 1 + (point << 50 | phi tile << 25 | r tile)
    int queued;
    int mready;
    unsigned m[32];           // inside mask of each phi row (bit c: r cell 32 * r tile + c)
    unsigned v[32];           // visited
    unsigned p[32];           // pending entry cells
};

enum : int { kTileActive = 0, kTileDone = 1, kTileOverflow = 2 };

struct TileItem {
    Mapper m;
    P2 src;
    double rho2, inv_rho2, dr, dphi, flux;
    const double* ld;
    int phi_bins;
    int uniform;
    int state;
    int f32;                 // cells mapped in FP32 about a per-column anchor
    unsigned long long acc_lo;
    long long acc_hi;
    unsigned long long cells;
};

struct TileCtl {
    unsigned long long head, tail;
    long long in_flight;
    int error;
    int pad;
};

struct TileCtx {
    TileItem* items;
    TileSlot* slots;
    unsigned* ring;
    TileCtl* ctl;
    unsigned long long mask;  // capacity - 1 (table and ring)
    unsigned spin_limit;      // polls before a wait gives up
    int* timeouts;            // waits that gave up (null: not counted)
};

__device__ __forceinline__ unsigned long long tile_key(int item, int tphi, int tr)
{
    return 1ull + (((unsigned long long)item << (2 * kKeyBits)) | ((unsigned long long)tphi << kKeyBits) |
                   (unsigned long long)tr);
}

__device__ __forceinline__ unsigned long long ld_cg_u64(const unsigned long long* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_cg_u32(const unsigned* p) { return __ldcg(p); }
__device__ __forceinline__ int ld_cg_i32(const int* p) { return __ldcg(p); }

// Slot of `key`, inserted if absent; -1 when the probe sequence is full.
__device__ long long find_or_insert(const TileCtx& G, unsigned long long key)
{
    unsigned long long h = (key * 0x9e3779b97f4a7c15ull) >> 20;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        h &= G.mask;
        TileSlot* s = G.slots + h;
        const unsigned long long k = ld_cg_u64(&s->key);
        if (k == key) return (long long)h;
        if (k == 0) {
            const unsigned long long prev = atomicCAS(&s->key, 0ull, key);
            if (prev == 0 || prev == key) return (long long)h;
        }
        ++h;
    }
    return -1;
}

__device__ __forceinline__ void push_slot(const TileCtx& G, unsigned slot)
{
    atomicAdd(reinterpret_cast<unsigned long long*>(&G.ctl->in_flight), 1ull);
    const unsigned long long pos = atomicAdd(&G.ctl->tail, 1ull);
    __threadfence();
    atomicExch(G.ring + (pos & G.mask), slot + 1u);
}

// ORs entry bits into row `row` of tile (item, tphi, tr) and queues the tile
// unless it is queued already.  Called by one thread.
__device__ void send_row(const TileCtx& G, int item, int tphi, int tr, int row, unsigned bits)
{
    if (tr >= (1 << kKeyBits) || tphi >= (1 << kKeyBits)) {
        atomicExch(&G.items[item].state, kTileOverflow);
        return;
    }
    const long long s = find_or_insert(G, tile_key(item, tphi, tr));
    if (s < 0) {
        atomicExch(&G.items[item].state, kTileOverflow);
        return;
    }
    TileSlot* T = G.slots + s;
    atomicOr(&T->p[row], bits);
    __threadfence();
    if (atomicExch(&T->queued, 1) == 0) push_slot(G, (unsigned)s);
}

// Cells reachable from g by moving up, then down, through set bits of p
// (Kogge-Stone occluded fills; g must be a subset of p).
__device__ __forceinline__ unsigned fill_row(unsigned g, unsigned p)
{
    unsigned gu = g, pu = p;
    gu |= pu & (gu << 1);
    pu &= pu << 1;
    gu |= pu & (gu << 2);
    pu &= pu << 2;
    gu |= pu & (gu << 4);
    pu &= pu << 4;
    gu |= pu & (gu << 8);
    pu &= pu << 8;
    gu |= pu & (gu << 16);
    unsigned gd = g, pd = p;
    gd |= pd & (gd >> 1);
    pd &= pd >> 1;
    gd |= pd & (gd >> 2);
    pd &= pd >> 2;
    gd |= pd & (gd >> 4);
    pd &= pd >> 4;
    gd |= pd & (gd >> 8);
    pd &= pd >> 8;
    gd |= pd & (gd >> 16);
    return gu | gd;
}

__device__ __forceinline__ double cell_dz2(const TileItem& I, double cs, double sn, int ir)
{
    const double radius = (static_cast<double>(ir) + 0.5) * I.dr;
    const P2 mp = map_real(I.m, radius * cs, radius * sn);
    return dist2(mp, I.src);
}

// As cell_dz2, in FP32 about the anchor A when the item asks for FP32 rays.
__device__ __forceinline__ double cell_dz2_rays(const TileItem& I, const Anchor32& A, double cs, double sn, int ir)
{
    if (!I.f32) return cell_dz2(I, cs, sn, ir);
    const double radius = (static_cast<double>(ir) + 0.5) * I.dr;
    return static_cast<double>(anchored_dist2(A, radius * cs, radius * sn));
}

// One visit of one tile by one warp.
__device__ void process_tile(const TileCtx& G, unsigned slot, double* d2s)
{
    const int j = lane_id();
    TileSlot* T = G.slots + slot;
    // The queued flag is cleared before the pending bits are taken (a sender
    // ORs its bits, then sets the flag), so bits that arrive after the take
    // queue the tile again.  The key, the item and the mask flag do not
    // depend on either and are read meanwhile, so a visit starts after about
    // three L2 round trips instead of six.
    if (j == 0) atomicExch(&T->queued, 0);
    const unsigned long long key = ld_cg_u64(&T->key) - 1ull;
    __syncwarp();
    __threadfence();
    const unsigned pend = atomicExch(&T->p[j], 0u);
    int ready = 0;
    if (j == 0) ready = ld_cg_i32(&T->mready);
    const int item = static_cast<int>(key >> (2 * kKeyBits));
    const int tphi = static_cast<int>((key >> kKeyBits) & kKeyMask);
    const int tr = static_cast<int>(key & kKeyMask);
    const int state = ld_cg_i32(&G.items[item].state);
    const TileItem I = G.items[item];
    if (state != kTileActive) return;
    const int g = tphi * 32 + j;
    const bool valid = g < I.phi_bins;
    double cs = 0.0, sn = 0.0;
    if (valid) {
        const double phi = (static_cast<double>(g) + 0.5) * I.dphi;
        trig::sincos_cr(phi, &sn, &cs);
    }
    // FP32 rays: one anchor per lattice column of the tile, at its middle radius.
    Anchor32 A{};
    if (I.f32 && valid) {
        const double ra = (static_cast<double>(tr * 32) + 16.0) * I.dr;
        A = make_anchor32(I.m, ra * cs, ra * sn, I.src);
    }
    ready = __shfl_sync(kFull, ready, 0);
    unsigned M = 0;
    const bool fresh = ready == 0;
    if (fresh) {
        if (valid) {
            const int base = tr * 32;
#pragma unroll 4
            for (int c = 0; c < 32; ++c) {
                const double d2 = cell_dz2_rays(I, A, cs, sn, base + c);
                d2s[c * 32 + j] = d2;
                if (d2 <= I.rho2) M |= 1u << c;
            }
        }
        T->m[j] = M;
        __threadfence();
        __syncwarp();
        if (j == 0) atomicExch(&T->mready, 1);
    } else {
        M = ld_cg_u32(&T->m[j]);
    }
    const unsigned S = pend & M;
    if (!__any_sync(kFull, S != 0u)) return;
    // In-tile closure of the entry cells.
    unsigned F = S;
    for (int it = 0; it < 1100; ++it) {
        F = fill_row(F, M);
        unsigned up = __shfl_up_sync(kFull, F, 1);
        unsigned dn = __shfl_down_sync(kFull, F, 1);
        if (j == 0) up = 0u;
        if (j == 31) dn = 0u;
        const unsigned Fn = F | ((up | dn) & M);
        if (!__any_sync(kFull, Fn != F)) break;
        F = Fn;
    }
    const unsigned old = atomicOr(&T->v[j], F);
    const unsigned nw = F & ~old;
    // Brightness-weighted radius of the new cells.
    Fixed128 acc{0ull, 0ll};
    unsigned bits = nw;
    while (bits) {
        const int c = __ffs(bits) - 1;
        bits &= bits - 1u;
        const int ir = tr * 32 + c;
        const double radius = (static_cast<double>(ir) + 0.5) * I.dr;
        double b = 1.0;
        if (!I.uniform) {
            const double d2 = fresh ? d2s[c * 32 + j] : cell_dz2_rays(I, A, cs, sn, ir);
            b = ld_lookup(I.ld, d2 * I.inv_rho2);
        }
        fx_add_double(acc, b * radius);
    }
    int cnt = __popc(nw);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long lo = __shfl_xor_sync(kFull, acc.lo, o);
        const long long hi = __shfl_xor_sync(kFull, acc.hi, o);
        fx_add(acc, lo, hi);
        cnt += __shfl_xor_sync(kFull, cnt, o);
    }
    if (cnt == 0) return;
    if (j == 0) {
        TileItem* Ig = G.items + item;
        const unsigned long long prev = atomicAdd(&Ig->acc_lo, acc.lo);
        const long long carry = (prev + acc.lo < prev) ? 1 : 0;
        atomicAdd(reinterpret_cast<unsigned long long*>(&Ig->acc_hi), (unsigned long long)(acc.hi + carry));
        atomicAdd(&Ig->cells, (unsigned long long)cnt);
    }
    // Exits, at most four neighbour tiles: along r outwards (the rows' last
    // cells) and inwards (their first cells), along phi upwards from the
    // tile's last row (or the lattice's last row; phi is periodic) and
    // downwards from its first row.  Lane k of lanes 0-3 looks up exit k's
    // tile, every lane ORs its bits into the r exits' rows, lanes 2 and 3
    // into the phi exits' rows, and lane k queues tile k: the four exits
    // cost the round trips of one.
    const int P = I.phi_bins;
    const int ju = (tphi * 32 + 31 < P) ? 31 : P - 1 - tphi * 32;  // the lattice row below the upward exit
    const unsigned nw_up = __shfl_sync(kFull, valid ? nw : 0u, ju);
    const unsigned nw_dn = __shfl_sync(kFull, valid ? nw : 0u, 0);
    const bool out_r = __any_sync(kFull, (nw >> 31) != 0u);
    const bool in_r = tr > 0 && __any_sync(kFull, (nw & 1u) != 0u);
    const int g_up = tphi * 32 + ju, g_dn = tphi * 32;
    const int gu = (g_up + 1 == P) ? 0 : g_up + 1;
    const int gd = (g_dn == 0) ? P - 1 : g_dn - 1;
    long long s_mine = -1;
    if (j < 4) {
        const bool active = j == 0 ? out_r : (j == 1 ? in_r : (j == 2 ? nw_up != 0u : nw_dn != 0u));
        const int xr = j == 0 ? tr + 1 : (j == 1 ? tr - 1 : tr);
        const int xphi = j < 2 ? tphi : (j == 2 ? gu >> 5 : gd >> 5);
        if (active) {
            if (xr < (1 << kKeyBits) && xphi < (1 << kKeyBits)) s_mine = find_or_insert(G, tile_key(item, xphi, xr));
            if (s_mine < 0) atomicExch(&G.items[item].state, kTileOverflow);
        }
    }
    const long long s0 = __shfl_sync(kFull, s_mine, 0), s1 = __shfl_sync(kFull, s_mine, 1);
    if (s0 >= 0 && (nw >> 31)) atomicOr(&G.slots[s0].p[j], 1u);
    if (s1 >= 0 && (nw & 1u)) atomicOr(&G.slots[s1].p[j], 0x80000000u);
    if (j == 2 && s_mine >= 0) atomicOr(&G.slots[s_mine].p[gu & 31], nw_up);
    if (j == 3 && s_mine >= 0) atomicOr(&G.slots[s_mine].p[gd & 31], nw_dn);
    __threadfence();
    __syncwarp();
    if (s_mine >= 0 && atomicExch(&G.slots[s_mine].queued, 1) == 0) push_slot(G, (unsigned)s_mine);
}

// Persistent warps.  A warp takes a ticket (one atomicAdd on the FIFO head, so
// idle warps do not contend on a compare-and-swap) and waits for the entry of
// its ticket; it leaves when no tile is queued or in process.
__global__ void __launch_bounds__(128) tile_flood_kernel(TileCtx G)
{
    __shared__ double d2s[4][32 * 32];
    double* mine = d2s[warp_in_block()];
    for (;;) {
        unsigned v = 0;
        int stop = 0;
        if (lane_id() == 0) {
            const unsigned long long h = atomicAdd(&G.ctl->head, 1ull);
            volatile unsigned* e = G.ring + (h & G.mask);
            for (unsigned spin = 0;; ++spin) {
                v = *e;
                if (v) {
                    *e = 0u;
                    break;
                }
                if (__ldcg(reinterpret_cast<const long long*>(&G.ctl->in_flight)) == 0 ||
                    ld_cg_i32(&G.ctl->error)) {
                    stop = 1;
                    break;
                }
                if (spin >= G.spin_limit) {
                    atomicExch(&G.ctl->error, 1);
                    if (G.timeouts) atomicAdd(G.timeouts, 1);
                    stop = 1;
                    break;
                }
                __nanosleep(spin < 64 ? 32 : 256);
            }
        }
        stop = __shfl_sync(kFull, stop, 0);
        if (stop) return;
        v = __shfl_sync(kFull, v, 0);
        process_tile(G, v - 1u, mine);
        __syncwarp();
        __threadfence();
        if (lane_id() == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&G.ctl->in_flight), ~0ull);
    }
}

// Warp per polar point: lattice parameters (as in fs_polar.cu) and the start
// cells of its seeds.
__global__ void __launch_bounds__(128) tile_start_kernel(FsWork w, TileCtx G)
{
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int n = w.ir_count[1];
    if (k >= n) return;
    const int n_cart = w.ir_count[0];
    const int it = w.ir_polar[k];
    const FsItem item = w.items[it];
    const FsOut o = w.out[it];
    TileItem I{};
    I.state = kTileDone;
    I.flux = dnan();
    if (o.status == kFsOk && o.n_seeds > 0) {
        const FsSettingsDev st = w.settings[item.settings];
        const P2* seeds = w.seeds + (long long)(n_cart + k) * w.seed_cap;
        const int ns = o.n_seeds;
        const double rho = item.rho;
        const int bins = max(st.polar_source_bins > 0 ? st.polar_source_bins : st.source_bins, 1);
        double ratio = dmax_(st.polar_grid_ratio > 0.0 ? st.polar_grid_ratio : st.grid_ratio, 1.0e-12);
        if (st.finite_mode == 4) ratio = dmax_(dmax_(ratio, 1.0e-12), 12.0);
        I.dr = rho / static_cast<double>(bins);
        double max_r = 1.0;
        for (int i = 0; i < ns; ++i) max_r = dmax_(max_r, hypot_borges(seeds[i].x, seeds[i].y) + 4.0 * rho);
        const double pb = ceil(2.0 * kPi * max_r / (I.dr * ratio));
        I.phi_bins = max(16, to_int_x86(pb));
        I.dphi = 2.0 * kPi / static_cast<double>(I.phi_bins);
        I.flux = source_flux(rho, st.ld_c, st.ld_d);
        I.m = make_mapper(item.s, item.q);
        I.src = P2{item.x, item.y};
        I.rho2 = rho * rho;
        I.inv_rho2 = 1.0 / I.rho2;
        I.uniform = (st.ld_c == 0.0 && st.ld_d == 0.0) ? 1 : 0;
        I.ld = w.ld_tables + (long long)st.ld_table * (kLdTable + 1);
        I.f32 = w.f32_rays;
        if (isfinite(I.flux)) I.state = (I.phi_bins >= (1 << 30)) ? kTileOverflow : kTileActive;
    }
    if (lane_id() == 0) G.items[k] = I;
    __syncwarp();
    __threadfence();
    if (I.state != kTileActive || lane_id() != 0) return;
    // find_polar_inside_start (FSM:1321-1364) for each seed, then the
    // reference's own check that the start cell is inside (FSM:1285-1287).
    const P2* seeds = w.seeds + (long long)(n_cart + k) * w.seed_cap;
    for (int i = 0; i < o.n_seeds; ++i) {
        const P2 seed = seeds[i];
        const double seed_r = hypot_borges(seed.x, seed.y);
        double seed_phi = atan2(seed.y, seed.x);
        while (seed_phi < 0.0) seed_phi += 2.0 * kPi;
        while (seed_phi >= 2.0 * kPi) seed_phi -= 2.0 * kPi;
        const int seed_ir = static_cast<int>(floor(seed_r / I.dr));
        const int seed_iphi = clampi(static_cast<int>(seed_phi / I.dphi), 0, I.phi_bins - 1);
        bool found = false;
        int fir = 0, fiphi = 0;
        for (int shell = 0; shell <= 10 && !found; ++shell) {
            for (int dir = -1; dir <= 1 && !found; dir += 2) {
                for (int d_ir = -shell; d_ir <= shell; ++d_ir) {
                    const int d_iphi = (shell - abs(d_ir)) * dir;
                    const int ir = seed_ir + d_ir;
                    if (ir < 0) continue;
                    int iphi = (seed_iphi + d_iphi) % I.phi_bins;
                    if (iphi < 0) iphi += I.phi_bins;
                    const double phi = (static_cast<double>(iphi) + 0.5) * I.dphi;
                    double sn, cs;
                    trig::sincos_cr(phi, &sn, &cs);
                    if (cell_dz2(I, cs, sn, ir) <= I.rho2) {
                        const double radius = (static_cast<double>(ir) + 0.5) * I.dr;
                        fir = max(0, static_cast<int>(floor(radius / I.dr)));
                        fiphi = clampi(static_cast<int>(phi / I.dphi), 0, I.phi_bins - 1);
                        found = true;
                        break;
                    }
                }
            }
        }
        if (!found) continue;
        {
            const double phi = (static_cast<double>(fiphi) + 0.5) * I.dphi;
            double sn, cs;
            trig::sincos_cr(phi, &sn, &cs);
            if (!(cell_dz2(I, cs, sn, fir) <= I.rho2)) continue;
        }
        if (fir >= (1 << 30)) {
            atomicExch(&G.items[k].state, kTileOverflow);
            return;
        }
        send_row(G, k, fiphi >> 5, fir >> 5, fiphi & 31, 1u << (fir & 31));
    }
}

// Thread per polar point: magnification, status, or hand-off to the second pass.
__global__ void tile_finish_kernel(FsWork w, TileCtx G)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = w.ir_count[1];
    if (k >= n) return;
    const int it = w.ir_polar[k];
    FsOut o = w.out[it];
    if (o.status != kFsOk) return;
    const TileItem I = G.items[k];
    const bool failed = G.ctl->error != 0;
    if (I.state == kTileOverflow || (failed && I.state == kTileActive)) {
        w.retry_polar[atomicAdd(&w.ir_count[3], 1)] = k;
        return;
    }
    double A = dnan();
    if (I.state == kTileActive) {
        const Fixed128 total{I.acc_lo, I.acc_hi};
        A = fx_to_double(total) * I.dr * I.dphi / I.flux;
    }
    o.A = A;
    o.err = isfinite(A) ? 0.0 : dnan();
    o.converged = isfinite(A) ? 1 : 0;
    if (!isfinite(A)) o.status = kFsNumerical;
    w.out[it] = o;
    w.rays[it] = I.cells;
}

} // namespace

size_t tile_bytes(long long capacity, int max_items)
{
    return (size_t)capacity * sizeof(TileSlot) + (size_t)capacity * sizeof(unsigned) +
           (size_t)max_items * sizeof(TileItem) + sizeof(TileCtl) + 1024;
}

int polar_tile_blocks_per_sm()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, tile_flood_kernel, 128, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 4;
    }
    return nb;
}

// Start, flood and finish on `stream`; `area` holds the tile table, the FIFO,
// the per-point state and the control words (tile_bytes), `capacity` a power
// of two.  The area is cleared here.
cudaError_t launch_polar_tiles(const FsWork& w, void* area, long long capacity, int max_items, int flood_blocks,
                               cudaStream_t stream)
{
    char* a = static_cast<char*>(area);
    TileCtx G;
    G.slots = reinterpret_cast<TileSlot*>(a);
    a += (size_t)capacity * sizeof(TileSlot);
    G.ring = reinterpret_cast<unsigned*>(a);
    a += (size_t)capacity * sizeof(unsigned);
    a = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(a) + 255) & ~uintptr_t(255));
    G.items = reinterpret_cast<TileItem*>(a);
    a += (size_t)max_items * sizeof(TileItem);
    a = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(a) + 255) & ~uintptr_t(255));
    G.ctl = reinterpret_cast<TileCtl*>(a);
    G.mask = (unsigned long long)capacity - 1ull;
    G.spin_limit = w.wait_limit ? w.wait_limit : kSpinLimit;
    G.timeouts = w.wait_timeouts;
    cudaError_t e = cudaMemsetAsync(area, 0, (size_t)capacity * (sizeof(TileSlot) + sizeof(unsigned)), stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(G.ctl, 0, sizeof(TileCtl), stream);
    if (e != cudaSuccess) return e;
    tile_start_kernel<<<(max_items * 32 + 127) / 128, 128, 0, stream>>>(w, G);
    tile_flood_kernel<<<flood_blocks, 128, 0, stream>>>(G);
    tile_finish_kernel<<<(max_items + 127) / 128, 128, 0, stream>>>(w, G);
    return cudaGetLastError();
}

} // namespace lcbi
