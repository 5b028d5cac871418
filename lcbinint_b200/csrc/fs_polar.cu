// Polar inverse-ray integration, one warp per evaluation
// (inverse_ray_polar_boundary_binary, finite_source_magnifier.cpp:1156-1319).
//
// The reference flood-fills the global (r, phi) lattice from the cell nearest
// each seed: a FIFO of cells, radial runs grown until an outside or visited
// cell, +-phi neighbours of every run cell enqueued.  Every run it grows is a
// maximal segment of inside cells of its phi row (a visited cell can never
// border an unvisited inside one in the same row), so the cells it counts are
// exactly the inside cells 4-connected (r +- 1, phi +- 1, phi periodic, r >= 0)
// to a starting cell.  The warp computes that same set segment by segment:
// a FIFO of segments, each neighbouring row scanned over the segment's range
// 32 cells at a time, new segments recognised by their (phi, left end) key in
// a per-warp hash set whose slots carry a generation tag (no clearing between
// evaluations).  The counted cells, and so the magnification up to the order
// of the FP64 sum (about 1e-15 relative), match the reference.
#include "lcbi_fs_kernels.h"
#include "lcbi_warp.cuh"

namespace lcbi {

namespace {

struct Slot {
    unsigned long long key;   // iphi << 20 | 64-cell word index
    unsigned long long gen;   // evaluation tag; a slot with another tag is free
    unsigned long long bits;
};

struct Polar {
    Mapper m;
    P2 src;
    double rho2, inv_rho2, dr, dphi;
    int phi_bins;
    bool uniform;
    const double* ld;
    // scratch
    int4* queue;      // FIFO of segments (iphi, L, R, -)
    unsigned qmask;
    Slot* slots;
    unsigned hmask;
    unsigned long long gen;
    bool ovf;
};

__device__ __forceinline__ int wrap_phi(const Polar& P, int i)
{
    i %= P.phi_bins;
    if (i < 0) i += P.phi_bins;
    return i;
}

__device__ __forceinline__ unsigned long long slot_key(int iphi, int word)
{
    return ((unsigned long long)iphi << 20) | (unsigned long long)word;
}

__device__ __forceinline__ unsigned hash_slot(int iphi, int word, unsigned mask)
{
    unsigned long long k = ((unsigned long long)iphi << 20) ^ (unsigned long long)word;
    k *= 0x9e3779b97f4a7c15ull;
    return (unsigned)(k >> 40) & mask;
}

// cell_inside (FSM:1255-1269); returns dz2 through `d2`.
__device__ __forceinline__ bool inside(const Polar& P, int ir, int iphi, double* d2)
{
    if (ir < 0) return false;
    iphi = wrap_phi(P, iphi);
    const double radius = (static_cast<double>(ir) + 0.5) * P.dr;
    const double phi = (static_cast<double>(iphi) + 0.5) * P.dphi;
    double sn, cs;
    sincos(phi, &sn, &cs);
    const P2 mp = map_real(P.m, radius * cs, radius * sn);
    const double dz2 = dist2(mp, P.src);
    *d2 = dz2;
    return dz2 <= P.rho2;
}

// find_polar_inside_start (FSM:1321-1364): diamond search of up to 10 shells.
__device__ bool polar_start(const Polar& P, P2 seed, double rho, int* out_ir, int* out_iphi)
{
    const double seed_r = hypot_borges(seed.x, seed.y);
    double seed_phi = atan2(seed.y, seed.x);
    while (seed_phi < 0.0) seed_phi += 2.0 * kPi;
    while (seed_phi >= 2.0 * kPi) seed_phi -= 2.0 * kPi;
    const int seed_ir = static_cast<int>(floor(seed_r / P.dr));
    const int seed_iphi = clampi(static_cast<int>(seed_phi / P.dphi), 0, P.phi_bins - 1);
    (void)rho;
    for (int shell = 0; shell <= 10; ++shell) {
        for (int dir = -1; dir <= 1; dir += 2) {
            for (int d_ir = -shell; d_ir <= shell; ++d_ir) {
                const int d_iphi = (shell - abs(d_ir)) * dir;
                const int ir = seed_ir + d_ir;
                if (ir < 0) continue;
                int iphi = (seed_iphi + d_iphi) % P.phi_bins;
                if (iphi < 0) iphi += P.phi_bins;
                double d2;
                if (inside(P, ir, iphi, &d2)) {
                    // The reference converts the cell centre back to indices (FSM:1279-1280).
                    const double radius = (static_cast<double>(ir) + 0.5) * P.dr;
                    const double phi = (static_cast<double>(iphi) + 0.5) * P.dphi;
                    *out_ir = max(0, static_cast<int>(floor(radius / P.dr)));
                    *out_iphi = clampi(static_cast<int>(phi / P.dphi), 0, P.phi_bins - 1);
                    return true;
                }
            }
        }
    }
    return false;
}

// Left end of the maximal inside segment of row iphi through inside cell x
// (cells below 0 do not exist).
__device__ int extend_left(const Polar& P, int iphi, int x)
{
    for (;;) {
        const int c = x - 1 - lane_id();
        double d2;
        const bool ok = c >= 0 && inside(P, c, iphi, &d2);
        const unsigned b = __ballot_sync(kFull, ok);
        if (~b == 0u) {
            x -= 32;
            continue;
        }
        return x - (__ffs(~b) - 1);
    }
}

// Right end of the maximal inside segment of row iphi through inside cell x;
// -1 if the segment outgrows the lattice the visited keys can address.
__device__ int extend_right(const Polar& P, int iphi, int x)
{
    for (;;) {
        const int c = x + 1 + lane_id();
        double d2;
        const bool ok = inside(P, c, iphi, &d2);
        const unsigned b = __ballot_sync(kFull, ok);
        if (~b == 0u) {
            x += 32;
            if (x >= (1 << 26)) return -1;
            continue;
        }
        return x + (__ffs(~b) - 1);
    }
}

// Records segment (iphi, L, R) and queues it, unless a segment starting at
// (iphi, L) was recorded before.  All lanes call it with the same arguments.
__device__ void push_run(Polar& P, int iphi, int L, int R, long long head, long long& tail)
{
    bool fresh = false, full = false;
    if (lane_id() == 0) {
        const unsigned long long key = slot_key(iphi, L);
        unsigned h = hash_slot(iphi, L, P.hmask);
        full = true;
        for (unsigned probe = 0; probe <= P.hmask; ++probe) {
            Slot& sl = P.slots[h];
            if (sl.gen != P.gen) {
                sl.key = key;
                sl.bits = (unsigned long long)(unsigned)R;
                sl.gen = P.gen;
                fresh = true;
                full = false;
                break;
            }
            if (sl.key == key) {
                full = false;
                break;
            }
            h = (h + 1) & P.hmask;
        }
        if (fresh) P.queue[tail & P.qmask] = make_int4(iphi, L, R, 0);
    }
    fresh = __shfl_sync(kFull, fresh, 0);
    full = __shfl_sync(kFull, full, 0);
    if (full) P.ovf = true;
    if (fresh) {
        ++tail;
        if (tail - head > (long long)P.qmask) P.ovf = true;
    }
    __syncwarp();
}

// Finds, in order, the maximal inside segments of row nb that intersect
// [L, R] and queues the new ones.  A segment touching L or R is extended past
// the window to its true ends.
__device__ void scan_neighbour_row(Polar& P, int nb, int L, int R, long long head, long long& tail)
{
    bool in_seg = false;
    int seg_start = 0;
    for (int c0 = L; c0 <= R && !P.ovf; c0 += 32) {
        const int cell = c0 + lane_id();
        double d2;
        const bool valid = cell <= R;
        const bool in = valid && inside(P, cell, nb, &d2);
        const unsigned m = __ballot_sync(kFull, in);
        const unsigned vm = __ballot_sync(kFull, valid);
        int pos = 0;
        while (pos < 32) {
            const unsigned from = (pos == 0) ? kFull : (kFull << pos);
            if (in_seg) {
                const unsigned out = ~m & vm & from;
                if (!out) break;
                const int o = __ffs(out) - 1;
                const int s0 = seg_start;
                const int e0 = c0 + o - 1;
                const int Ls = (s0 == L) ? extend_left(P, nb, s0) : s0;
                push_run(P, nb, Ls, e0, head, tail);
                in_seg = false;
                pos = o;
            } else {
                const unsigned nx = m & from;
                if (!nx) break;
                const int i = __ffs(nx) - 1;
                seg_start = c0 + i;
                in_seg = true;
                pos = i;
            }
        }
    }
    if (in_seg && !P.ovf) {
        const int Ls = (seg_start == L) ? extend_left(P, nb, seg_start) : seg_start;
        const int Rs = extend_right(P, nb, R);
        if (Rs < 0) {
            P.ovf = true;
            return;
        }
        push_run(P, nb, Ls, Rs, head, tail);
    }
}

} // namespace

__global__ void __launch_bounds__(128) polar_kernel(FsWork w, unsigned long long epoch)
{
    const int lane = lane_id();
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    char* base = w.scratch_polar + (long long)gw * w.scratch_polar_per_warp;
    unsigned long long local_gen = 0;
    const int n = w.retry_pass ? w.ir_count[3] : w.ir_count[1];
    const int n_cart = w.ir_count[0];
    for (;;) {
        int k = 0;
        if (lane == 0) k = atomicAdd(&w.next_item[w.retry_pass ? 4 : 2], 1);
        k = shfl_i(k, 0);
        if (k >= n) break;
        if (w.retry_pass) k = w.retry_polar[k];
        const int it = w.ir_polar[k];
        const long long t_item = clock64();
        const FsItem item = w.items[it];
        FsOut o = w.out[it];
        if (o.status != kFsOk) continue;
        const FsSettingsDev st = w.settings[item.settings];
        const P2* seeds = w.seeds + (long long)(n_cart + k) * w.seed_cap;
        const int ns = o.n_seeds;
        const double rho = item.rho;
        double A = dnan();
        Polar P;
        P.ovf = false;
        if (ns > 0) {
            const int bins = max(st.polar_source_bins > 0 ? st.polar_source_bins : st.source_bins, 1);
            double ratio = dmax_(st.polar_grid_ratio > 0.0 ? st.polar_grid_ratio : st.grid_ratio, 1.0e-12);
            // Auto mode widens the angular cells for high magnification (FSM:4812-4820).
            if (st.finite_mode == 4) ratio = dmax_(dmax_(ratio, 1.0e-12), 12.0);
            P.dr = rho / static_cast<double>(bins);
            double max_r = 1.0;
            for (int i = 0; i < ns; ++i) max_r = dmax_(max_r, hypot_borges(seeds[i].x, seeds[i].y) + 4.0 * rho);
            const double pb = ceil(2.0 * kPi * max_r / (P.dr * ratio));
            P.phi_bins = max(16, to_int_x86(pb));
            P.dphi = 2.0 * kPi / static_cast<double>(P.phi_bins);
            const double flux = source_flux(rho, st.ld_c, st.ld_d);
            if (isfinite(flux)) {
                P.m = make_mapper(item.s, item.q);
                P.src = P2{item.x, item.y};
                P.rho2 = rho * rho;
                P.inv_rho2 = 1.0 / P.rho2;
                P.uniform = st.ld_c == 0.0 && st.ld_d == 0.0;
                P.ld = w.ld_tables + (long long)st.ld_table * (kLdTable + 1);
                P.queue = reinterpret_cast<int4*>(base);
                P.qmask = (unsigned)w.queue_cap - 1u;
                P.slots = reinterpret_cast<Slot*>(base + (long long)w.queue_cap * sizeof(int4));
                P.hmask = (unsigned)w.hash_cap - 1u;
                ++local_gen;
                P.gen = (epoch << 32) | (local_gen & 0xffffffffull);
                if (P.phi_bins >= (1 << 24)) P.ovf = true;
                long long head = 0, tail = 0;
                // Start segments: the maximal inside segment through each seed's
                // starting cell (find_polar_inside_start, FSM:1271-1282), in seed order.
                for (int i = 0; i < ns && !P.ovf; ++i) {
                    int ir = 0, iphi = 0;
                    bool ok = false;
                    if (lane == 0) ok = polar_start(P, seeds[i], rho, &ir, &iphi);
                    ok = __shfl_sync(kFull, ok, 0);
                    if (!ok) continue;
                    ir = shfl_i(ir, 0);
                    iphi = wrap_phi(P, shfl_i(iphi, 0));
                    const int L = extend_left(P, iphi, ir);
                    const int R = extend_right(P, iphi, ir);
                    if (R < 0) break;
                    push_run(P, iphi, L, R, head, tail);
                }
                double total = 0.0;
                unsigned long long rays = 0;
                while (head < tail && !P.ovf) {
                    const int4 run = P.queue[head & P.qmask];
                    ++head;
                    const int iphi = run.x, L = run.y, R = run.z;
                    // Brightness-weighted radius of the segment's cells, left to right.
                    for (int c0 = L; c0 <= R; c0 += 32) {
                        const int cur = c0 + lane;
                        double v = 0.0;
                        if (cur <= R) {
                            double d2;
                            inside(P, cur, iphi, &d2);
                            const double radius = (static_cast<double>(cur) + 0.5) * P.dr;
                            const double b = P.uniform ? 1.0 : ld_lookup(P.ld, d2 * P.inv_rho2);
                            v = b * radius;
                        }
                        const int m = min(32, R - c0 + 1);
                        for (int t = 0; t < m; ++t) total += shfl_d(v, t);
                    }
                    rays += (unsigned long long)(R - L + 1);
                    // Segments of the rows phi-1 and phi+1 that touch [L, R].
                    scan_neighbour_row(P, wrap_phi(P, iphi - 1), L, R, head, tail);
                    if (P.ovf) break;
                    scan_neighbour_row(P, wrap_phi(P, iphi + 1), L, R, head, tail);
                }
                if (!P.ovf) A = total * P.dr * P.dphi / flux;
                if (lane == 0) w.rays[it] = rays;
            }
        }
        if (P.ovf && !w.retry_pass) {
            if (lane == 0) w.retry_polar[atomicAdd(&w.ir_count[3], 1)] = k;
            __syncwarp();
            continue;
        }
        o.A = A;
        o.err = isfinite(A) ? 0.0 : dnan();
        o.converged = isfinite(A) ? 1 : 0;
        if (P.ovf) o.status = kFsQueueOverflow;
        else if (!isfinite(A)) o.status = kFsNumerical;
        if (lane == 0) {
            w.out[it] = o;
            if (w.cycles) w.cycles[it] += clock64() - t_item;
        }
        __syncwarp();
    }
}

size_t polar_scratch_bytes(int queue_cap, int hash_cap)
{
    return (size_t)queue_cap * sizeof(int4) + (size_t)hash_cap * sizeof(Slot) + 256;
}

cudaError_t launch_polar(const FsWork& w, int n_warps, cudaStream_t stream, unsigned long long epoch)
{
    const int blocks = (n_warps + 3) / 4;
    polar_kernel<<<blocks, 128, 0, stream>>>(w, epoch);
    return cudaGetLastError();
}

} // namespace lcbi
