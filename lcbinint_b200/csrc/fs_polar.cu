// Polar inverse-ray integration
// (inverse_ray_polar_boundary_binary, finite_source_magnifier.cpp:1156-1319).
//
// The reference flood-fills the global (r, phi) lattice from the cell nearest
// each seed: a FIFO of cells, radial runs grown until an outside or visited
// cell, +-phi neighbours of every run cell enqueued.  Every run it grows is a
// maximal segment of inside cells of its phi row (a visited cell can never
// border an unvisited inside one in the same row), so the cells it counts are
// exactly the inside cells 4-connected (r +- 1, phi +- 1, phi periodic, r >= 0)
// to a starting cell.  A group of W warps computes that same set segment by
// segment: a FIFO of segments, each neighbouring row scanned over the
// segment's range 32 W cells at a time, new segments recognised by their
// (phi, left end) key in a hash set whose slots carry a generation tag (no
// clearing between evaluations).  Ordinary points run on one warp; a point
// whose flood fill passes a cell budget (or outgrows the per-warp scratch) is
// handed to a second pass that runs each such point on a whole block.
//
// The brightness-weighted sum is accumulated exactly in 128-bit fixed point, so
// the result does not depend on the group width or on the visiting order; it
// differs from the reference's running FP64 sum only by that sum's own
// rounding (about 1e-16 relative per term).
#include "lcbi_fs_kernels.h"
#include "lcbi_group.cuh"
#include "lcbi_trig.cuh"

namespace lcbi {

namespace {

struct Slot {
    unsigned long long key;   // iphi << 32 | left end
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

// One phi row of the lattice with its direction cosines (the cell centres of
// a row share one angle, so its sine and cosine are evaluated once).
struct Row {
    int iphi;
    double cs, sn;
};

__device__ __forceinline__ int wrap_phi(const Polar& P, int i)
{
    i %= P.phi_bins;
    if (i < 0) i += P.phi_bins;
    return i;
}

__device__ __forceinline__ Row make_row(const Polar& P, int iphi)
{
    Row r;
    r.iphi = wrap_phi(P, iphi);
    const double phi = (static_cast<double>(r.iphi) + 0.5) * P.dphi;
    trig::sincos_cr(phi, &r.sn, &r.cs);
    return r;
}

__device__ __forceinline__ unsigned hash_slot(int iphi, int left, unsigned mask)
{
    unsigned long long k = ((unsigned long long)(unsigned)iphi << 32) ^ (unsigned long long)(unsigned)left;
    k *= 0x9e3779b97f4a7c15ull;
    return (unsigned)(k >> 40) & mask;
}

// cell_inside (FSM:1255-1269) for a cell of row `r`; returns dz2 through `d2`.
__device__ __forceinline__ bool inside_row(const Polar& P, const Row& r, int ir, double* d2)
{
    if (ir < 0) return false;
    const double radius = (static_cast<double>(ir) + 0.5) * P.dr;
    const P2 mp = map_real(P.m, radius * r.cs, radius * r.sn);
    const double dz2 = dist2(mp, P.src);
    *d2 = dz2;
    return dz2 <= P.rho2;
}

__device__ __forceinline__ bool inside(const Polar& P, int ir, int iphi, double* d2)
{
    if (ir < 0) return false;
    return inside_row(P, make_row(P, iphi), ir, d2);
}

// find_polar_inside_start (FSM:1321-1364): diamond search of up to 10 shells.
__device__ bool polar_start(const Polar& P, P2 seed, int* out_ir, int* out_iphi)
{
    const double seed_r = hypot_borges(seed.x, seed.y);
    double seed_phi = atan2(seed.y, seed.x);
    while (seed_phi < 0.0) seed_phi += 2.0 * kPi;
    while (seed_phi >= 2.0 * kPi) seed_phi -= 2.0 * kPi;
    const int seed_ir = static_cast<int>(floor(seed_r / P.dr));
    const int seed_iphi = clampi(static_cast<int>(seed_phi / P.dphi), 0, P.phi_bins - 1);
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

// Left end of the maximal inside segment of row r through inside cell x
// (cells below 0 do not exist).
template <int W>
__device__ int extend_left(const Polar& P, GroupShared<W>& S, int& phase, const Row& r, int x)
{
    for (;;) {
        const int c = x - 1 - Grp<W>::rank();
        double d2;
        const bool ok = c >= 0 && inside_row(P, r, c, &d2);
        unsigned m[W];
        group_ballot<W>(S, phase, !ok, m);
        const int z = first_set<W>(m, 0);
        if (z == Grp<W>::N) {
            x -= Grp<W>::N;
            continue;
        }
        return x - z;
    }
}

// Right end of the maximal inside segment of row r through inside cell x;
// -1 if the segment outgrows the lattice the keys can address.
template <int W>
__device__ int extend_right(const Polar& P, GroupShared<W>& S, int& phase, const Row& r, int x)
{
    for (;;) {
        const int c = x + 1 + Grp<W>::rank();
        double d2;
        const bool ok = inside_row(P, r, c, &d2);
        unsigned m[W];
        group_ballot<W>(S, phase, !ok, m);
        const int z = first_set<W>(m, 0);
        if (z == Grp<W>::N) {
            x += Grp<W>::N;
            if (x >= (1 << 30)) return -1;
            continue;
        }
        return x + z;
    }
}

// Records segment (iphi, L, R) and queues it, unless a segment starting at
// (iphi, L) was recorded before.  The whole group calls it with the same
// arguments; rank 0 touches the table.
template <int W>
__device__ void push_run(Polar& P, GroupShared<W>& S, int iphi, int L, int R, long long head, long long& tail)
{
    int res = 0;  // 1 fresh, 2 table full
    if (Grp<W>::rank() == 0) {
        const unsigned long long key = ((unsigned long long)(unsigned)iphi << 32) | (unsigned long long)(unsigned)L;
        unsigned h = hash_slot(iphi, L, P.hmask);
        res = 2;
        for (unsigned probe = 0; probe <= P.hmask; ++probe) {
            Slot& sl = P.slots[h];
            if (sl.gen != P.gen) {
                sl.key = key;
                sl.bits = (unsigned long long)(unsigned)R;
                sl.gen = P.gen;
                res = 1;
                break;
            }
            if (sl.key == key) {
                res = 0;
                break;
            }
            h = (h + 1) & P.hmask;
        }
        if (res == 1) P.queue[tail & P.qmask] = make_int4(iphi, L, R, 0);
    }
    res = static_cast<int>(group_bcast<W>(S, res));
    if (res == 2) P.ovf = true;
    if (res == 1) {
        ++tail;
        if (tail - head > (long long)P.qmask) P.ovf = true;
    }
}

// Finds, in order, the maximal inside segments of row nb that intersect
// [L, R] and queues the new ones.  A segment touching L or R is extended past
// the window to its true ends.
template <int W>
__device__ void scan_neighbour_row(Polar& P, GroupShared<W>& S, int& phase, const Row& nb, int L, int R,
                                   long long head, long long& tail)
{
    constexpr int N = Grp<W>::N;
    bool in_seg = false;
    int seg_start = 0;
    for (int c0 = L; c0 <= R && !P.ovf; c0 += N) {
        const int cell = c0 + Grp<W>::rank();
        double d2;
        const bool valid = cell <= R;
        const bool in = valid && inside_row(P, nb, cell, &d2);
        unsigned inw[W], outw[W];
        group_ballot2<W>(S, phase, in, valid && !in, inw, outw);
        int pos = 0;
        while (pos < N) {
            if (in_seg) {
                const int o = first_set<W>(outw, pos);
                if (o == N) break;
                const int s0 = seg_start;
                const int e0 = c0 + o - 1;
                const int Ls = (s0 == L) ? extend_left<W>(P, S, phase, nb, s0) : s0;
                push_run<W>(P, S, nb.iphi, Ls, e0, head, tail);
                in_seg = false;
                pos = o;
            } else {
                const int i = first_set<W>(inw, pos);
                if (i == N) break;
                seg_start = c0 + i;
                in_seg = true;
                pos = i;
            }
        }
    }
    if (in_seg && !P.ovf) {
        const int Ls = (seg_start == L) ? extend_left<W>(P, S, phase, nb, seg_start) : seg_start;
        const int Rs = extend_right<W>(P, S, phase, nb, R);
        if (Rs < 0) {
            P.ovf = true;
            return;
        }
        push_run<W>(P, S, nb.iphi, Ls, Rs, head, tail);
    }
}

// The list a kernel instance works through.
struct PolarList {
    const int* slots;   // inverse-ray polar slot of each entry (null: the identity)
    const int* count;
    int* next;
};

template <int W>
__device__ void polar_body(const FsWork& w, unsigned long long epoch, PolarList Lst, char* base, GroupShared<W>& S)
{
    const int t = Grp<W>::rank();
    unsigned long long local_gen = 0;
    const int n = *Lst.count;
    const int n_cart = w.ir_count[0];
    int phase = 0;
    for (;;) {
        int k = 0;
        if (t == 0) k = atomicAdd(Lst.next, 1);
        k = static_cast<int>(group_bcast<W>(S, k));
        if (k >= n) break;
        if (Lst.slots) k = Lst.slots[k];
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
        bool over_budget = false;
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
                if (P.phi_bins >= (1 << 30)) P.ovf = true;
                long long head = 0, tail = 0;
                // Start segments: the maximal inside segment through each seed's
                // starting cell (find_polar_inside_start, FSM:1271-1282), in seed order.
                for (int i = 0; i < ns && !P.ovf; ++i) {
                    long long packed = -1;
                    if (t == 0) {
                        int ir = 0, iphi = 0;
                        if (polar_start(P, seeds[i], &ir, &iphi))
                            packed = ((long long)(unsigned)ir << 32) | (long long)(unsigned)iphi;
                    }
                    packed = group_bcast<W>(S, packed);
                    if (packed < 0) continue;
                    const int ir = static_cast<int>(packed >> 32);
                    const Row r = make_row(P, static_cast<int>(packed & 0xffffffffll));
                    const int L = extend_left<W>(P, S, phase, r, ir);
                    const int R = extend_right<W>(P, S, phase, r, ir);
                    if (R < 0) {
                        P.ovf = true;
                        break;
                    }
                    push_run<W>(P, S, r.iphi, L, R, head, tail);
                }
                Fixed128 acc{0ull, 0ll};
                unsigned long long rays = 0;
                while (head < tail && !P.ovf) {
                    const int4 run = P.queue[head & P.qmask];
                    ++head;
                    const int L = run.y, R = run.z;
                    const Row r = make_row(P, run.x);
                    // Brightness-weighted radius of the segment's cells.
                    for (int c0 = L; c0 <= R; c0 += Grp<W>::N) {
                        const int cur = c0 + t;
                        if (cur <= R) {
                            const double radius = (static_cast<double>(cur) + 0.5) * P.dr;
                            double b = 1.0;
                            if (!P.uniform) {
                                double d2;
                                inside_row(P, r, cur, &d2);
                                b = ld_lookup(P.ld, d2 * P.inv_rho2);
                            }
                            fx_add_double(acc, b * radius);
                        }
                    }
                    rays += (unsigned long long)(R - L + 1);
                    if (W == 1 && !w.retry_pass &&
                        rays > (unsigned long long)(n <= w.few_points ? 1 : w.cell_budget)) {
                        over_budget = true;
                        break;
                    }
                    // Segments of the rows phi-1 and phi+1 that touch [L, R].
                    scan_neighbour_row<W>(P, S, phase, make_row(P, run.x - 1), L, R, head, tail);
                    if (P.ovf) break;
                    scan_neighbour_row<W>(P, S, phase, make_row(P, run.x + 1), L, R, head, tail);
                }
                const Fixed128 total = group_fx_sum<W>(S, acc);
                if (!P.ovf && !over_budget) A = fx_to_double(total) * P.dr * P.dphi / flux;
                if (t == 0) w.rays[it] = rays;
            }
        }
        if ((P.ovf || over_budget) && !w.retry_pass) {
            // Too large for one warp or for this pass's scratch: the second pass
            // runs it again on a whole block with the large scratch.
            if (t == 0) w.retry_polar[atomicAdd(&w.ir_count[3], 1)] = k;
            Grp<W>::sync();
            continue;
        }
        o.A = A;
        o.err = isfinite(A) ? 0.0 : dnan();
        o.converged = isfinite(A) ? 1 : 0;
        if (P.ovf) o.status = kFsQueueOverflow;
        else if (!isfinite(A)) o.status = kFsNumerical;
        if (t == 0) {
            w.out[it] = o;
            if (w.cycles) w.cycles[it] += clock64() - t_item;
        }
        Grp<W>::sync();
    }
}

__global__ void __launch_bounds__(128) polar_warp_kernel(FsWork w, unsigned long long epoch)
{
    __shared__ GroupShared<1> sh[4];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const PolarList L{nullptr, w.ir_count + 1, w.next_item + 2};
    polar_body<1>(w, epoch, L, w.scratch_polar + (long long)gw * w.scratch_polar_per_warp, sh[warp_in_block()]);
}

__global__ void __launch_bounds__(32 * kBigWarps) polar_block_kernel(FsWork w, unsigned long long epoch)
{
    __shared__ GroupShared<kBigWarps> sh;
    const PolarList L{w.retry_polar, w.ir_count + 3, w.next_item + 4};
    polar_body<kBigWarps>(w, epoch, L, w.scratch_polar + (long long)blockIdx.x * w.scratch_polar_per_warp, sh);
}

} // namespace

size_t polar_scratch_bytes(int queue_cap, int hash_cap)
{
    return (size_t)queue_cap * sizeof(int4) + (size_t)hash_cap * sizeof(Slot) + 256;
}

// First pass: one warp per point.  Second pass (w.retry_pass): one block of
// kBigWarps warps per point, n_groups blocks, each with its own scratch.
cudaError_t launch_polar(const FsWork& w, int n_groups, cudaStream_t stream, unsigned long long epoch)
{
    if (w.retry_pass) {
        polar_block_kernel<<<n_groups, 32 * kBigWarps, 0, stream>>>(w, epoch);
    } else {
        polar_warp_kernel<<<(n_groups + 3) / 4, 128, 0, stream>>>(w, epoch);
    }
    return cudaGetLastError();
}

} // namespace lcbi
