// Cartesian inverse-ray integration (inverse_ray_cartesian_binary_mag,
// finite_source_magnifier.cpp:2470-2768, with the row-scan flood fill
// cartesian_image_area_impl, :1891-2014).
//
// The reference walks the image plane one cell at a time: each row runs right
// from the previous row's right edge, then left, with gap repairs and overlap
// bookkeeping that depend on the order of visits.  A group of W warps (one
// warp for ordinary points; a block of kBigWarps warps in the second pass, for
// points whose scan passed the first pass's cell budget or scratch) reproduces
// that walk exactly:
//   * the lens map of the next 32 W cells along the current scan direction is
//     evaluated in parallel.  The reference reaches the cell t steps ahead by t
//     successive additions x += dx; inside one binade every such rounded sum
//     adds the same step, so the abscissa is formed in closed form, one binade
//     stretch at a time (constant_run), with the single additions that cross
//     binade boundaries done as the reference does them;
//   * the scan state machine consumes those results in order: runs of cells
//     that only accumulate, or only step on, are consumed from ballot masks in
//     one go; every other cell goes through the reference's loop body;
//   * row bookkeeping lives in per-group global scratch with the reference's
//     zero-on-growth vector semantics, and the same-row overlap test uses a
//     generation-tagged hash of the reference's integer row keys.
// The brightness sum keeps the reference's summation order, so the
// magnification is bit-identical.
#include "lcbi_fs_kernels.h"
#include "lcbi_group.cuh"

#include <atomic>
#include <cstdint>

namespace lcbi {

namespace {

template <int W>
struct CartShared {
    double d[32 * W];   // dz2 of each chunk cell (rho^2 + 1 on the wrong parity)
    double b[32 * W];   // brightness of inside cells
    double x[32 * W];   // abscissa of each chunk cell
    unsigned in[W];     // inside masks
    unsigned cont[W];   // left scan: abscissa >= xmin(previous row) - dx
    int item;
    int red[W];
    unsigned ev[W];     // gap-repair check: rows with a repair, per warp
    double mx[W];       // and each warp's largest row jump
};

struct RowScratch {
    double* xmin;
    double* xmax;
    double* ax;
    double* y;
    double* dys;
    int* next;                  // chain of rows sharing a row key
    ulonglong2* table;          // open-addressing map row key -> newest row: {generation, key << 32 | row + 1}
    unsigned tmask;             // table slots - 1 (power of two, at least twice the row capacity)
    int cap;
    int hw;                     // rows [0, hw) exist (vector size in the reference)
    unsigned long long gen;
    bool ovf;
};

__device__ __forceinline__ unsigned key_hash(int key, unsigned mask)
{
    unsigned long long k = (unsigned long long)(unsigned)key * 0x9e3779b97f4a7c15ull;
    return (unsigned)(k >> 32) & mask;
}

// Newest row with this key in the current scan generation, or -1; *slot receives
// the table slot to update (its own, or the first free one on the probe path).
__device__ __forceinline__ int key_lookup(const RowScratch& R, int key, unsigned* slot)
{
    unsigned h = key_hash(key, R.tmask);
    for (unsigned probe = 0; probe <= R.tmask; ++probe) {
        const ulonglong2 e = R.table[h];
        if (e.x != R.gen) {
            *slot = h;
            return -1;
        }
        if ((int)(e.y >> 32) == key) {
            *slot = h;
            return (int)(e.y & 0xffffffffull) - 1;
        }
        h = (h + 1) & R.tmask;
    }
    *slot = 0xffffffffu;
    return -1;
}

// Rows [0, i] exist afterwards, rows that come into existence being zero (the
// reference's vector resize).  Rows are zeroed ahead in batches of one per
// thread: a row is only ever written after it exists, so the rows zeroed
// ahead are still zero when they come into existence.
template <int W>
__device__ __forceinline__ void rows_ensure(RowScratch& R, int i)
{
    if (i < R.hw) return;
    if (i >= R.cap) {
        R.ovf = true;
        return;
    }
    const int end = min(R.cap, max(i + 1, R.hw + Grp<W>::N));
    for (int r = R.hw + Grp<W>::rank(); r < end; r += Grp<W>::N) {
        R.xmin[r] = 0.0;
        R.xmax[r] = 0.0;
        R.ax[r] = 0.0;
        R.y[r] = 0.0;
        R.dys[r] = 0.0;
    }
    R.hw = end;
    Grp<W>::sync();
}

// Row values are written by rank 0; every thread keeps the same control flow.
template <int W>
__device__ __forceinline__ void wset(double* a, int i, double v)
{
    if (Grp<W>::rank() == 0) a[i] = v;
}

struct Ctx {
    unsigned long long rays;  // inside cells consumed (identical in every thread)
    long long evals;          // cells evaluated (budget accounting)
    long long budget;         // 0: none
    bool bulk;                // every inside cell has brightness > 0 (run consumption allowed)
    Mapper m;
    P2 src;
    double rho, rho2, inv_rho2;
    bool uniform;
    const double* ld;
    const double* lds;        // the block's shared-memory copy of the same table (null: read ld)
    int max_steps;
    bool f32;                 // FP32 map about the current seed (A)
    Anchor32 A;
    // Adaptive local refinement: the point's tape (null: off), kept by rank 0.
    TapeCell* tape;
    int tape_n, tape_max;
    double band, step;
};

// LocalRefinementTape::add (FSM:993-1003): the first tape_max distinct cells,
// keyed by their lattice indices, in the order the scan visits them.
__device__ __noinline__ void tape_add(Ctx& C, double x, double y, double weight)
{
    if (C.tape_n >= C.tape_max) return;
    const long long kx = llround(x / C.step), ky = llround(y / C.step);
    for (int i = 0; i < C.tape_n; ++i)
        if (C.tape[i].kx == kx && C.tape[i].ky == ky) return;
    C.tape[C.tape_n++] = TapeCell{x, y, weight, kx, ky};
}

// Lens map of one cell, as the reference evaluates it for the current scan.
__device__ __forceinline__ void eval_for_scan(const Ctx& C, double x, double y, int jsign, double* dz2, double* bright)
{
    double md2;
    bool ok = true;
    if (C.f32) {
        md2 = static_cast<double>(anchored_dist2(C.A, x, y));
        if (jsign != 0) {
            const float j = anchored_jacobian(C.A, x, y);
            const int es = j > 0.0f ? 1 : (j < 0.0f ? -1 : 0);
            ok = es != -jsign;
        }
    } else if (jsign == 0) {
        md2 = mapped_dist2(C.m, x, y, C.src);
    } else {
        double jac;
        md2 = eval_cell(C.m, x, y, C.src, &jac);
        const int es = sign_of(jac);
        ok = es != -jsign;
    }
    const double d = ok ? md2 : C.rho2 + 1.0;
    *dz2 = d;
    double b = 0.0;
    if (d <= C.rho2) b = C.uniform ? 1.0 : (C.lds ? ld_lookup_shared(C.lds, md2 * C.inv_rho2)
                                                  : ld_lookup(C.ld, md2 * C.inv_rho2));
    *bright = b;
}

__host__ __device__ inline long long table_slots(int cap)
{
    long long t = 1;
    while (t < 2ll * cap) t <<= 1;
    return t;
}

__device__ __forceinline__ int row_key(double y, double inv_incr) { return to_int_x86(y * inv_incr + kRowKeyOffset); }

// True when n repeated additions x0 + d, (x0 + d) + d, ... each add one and the
// same rounded step, which is then returned: x0 and x0 + n * step lie in one
// binade (same sign and exponent, the end strictly above the binade's lower
// bound) and the first two steps agree.  Inside a binade every sum is a
// multiple of its ulp u, and fl(x + d) = x + (d rounded to a multiple of u);
// only a d exactly halfway between multiples can alternate between two
// rounded steps, and then the steps are constant from the first pair of equal
// steps on.
__device__ __forceinline__ bool constant_run(double x0, double d, int n, double* step)
{
    if (x0 == 0.0) return false;
    const double x1 = x0 + d;
    const double s1 = x1 - x0;
    const double x2 = x1 + d;
    if (x2 - x1 != s1) return false;
    const double xe = x0 + static_cast<double>(n) * s1;
    int e0, e1;
    frexp(x0, &e0);
    const double me = frexp(xe, &e1);
    if (e0 != e1 || (x0 < 0.0) != (xe < 0.0) || xe == 0.0 || fabs(me) == 0.5) return false;
    *step = s1;
    return true;
}

// x0 after t reference additions of d: binade stretches in closed form (the
// longest stretch by bisection), the crossings one addition at a time.
__device__ __forceinline__ double advance(double x0, double d, int t)
{
    double x = x0;
    int k = t;
    for (int guard = 0; k > 0 && guard < 64; ++guard) {
        double s;
        if (constant_run(x, d, k, &s)) {
            return x + static_cast<double>(k) * s;
        }
        int lo = 0, hi = k;  // constant_run holds for lo steps (trivially for 0), fails for hi
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            double sm;
            if (constant_run(x, d, mid, &sm)) lo = mid;
            else hi = mid;
        }
        if (lo > 0) {
            double sl;
            constant_run(x, d, lo, &sl);
            x = x + static_cast<double>(lo) * sl;
            k -= lo;
        }
        x = x + d;
        --k;
    }
    for (; k > 0; --k) x = x + d;
    return x;
}

// Evaluates the chunk of cells starting at ix along dx into shared memory:
// cells [0, na).  With na < N the cells [na, N) hold a second segment, the
// scan of the row at sy from sx in the other direction (step -dx): after a
// left-scan chunk, the next row's first right-scan cells; after a row's first
// right-scan chunk, its left-scan cells (whose continue bits use want_cont2
// and thr2).  na is a multiple of 32, so each warp evaluates one segment.
template <int W>
__device__ void fill_chunk(Ctx& C, CartShared<W>& S, double ix, double iy, double dx, int jsign, bool want_cont,
                           double thr, int na, double sx, double sy, bool want_cont2 = false, double thr2 = 0.0)
{
    const int t = Grp<W>::rank();
    Grp<W>::sync();  // every thread is done with the previous chunk
    const bool first = t < na;
    const double x = first ? advance(ix, dx, t) : advance(sx, -dx, t - na);
    double d, b;
    eval_for_scan(C, x, first ? iy : sy, jsign, &d, &b);
    S.d[t] = d;
    S.b[t] = b;
    S.x[t] = x;
    const unsigned in = __ballot_sync(kFull, d <= C.rho2);
    const unsigned co = __ballot_sync(kFull, first ? (want_cont && x >= thr) : (want_cont2 && x >= thr2));
    if (lane_id() == 0) {
        S.in[t >> 5] = in;
        S.cont[t >> 5] = co;
    }
    C.evals += Grp<W>::N;
    Grp<W>::sync();
}

// First eventful chunk cell in [from, end): an outside cell while counting;
// otherwise an inside cell or one past the continue threshold; end if none.
template <int W>
__device__ __forceinline__ int first_event(const CartShared<W>& S, int from, int end, bool counting)
{
    const int fw = from >> 5;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        if (w < fw) continue;
        if ((w << 5) >= end) break;
        const unsigned lo = (w == fw) ? (kFull << (from & 31)) : kFull;
        const unsigned ev = counting ? (~S.in[w] & lo) : ((S.in[w] | ~S.cont[w]) & lo);
        if (ev) return (w << 5) + __ffs(ev) - 1;
    }
    return end;
}

// Sequential brightness sum of chunk cells [a, b) in order.  Every thread
// forms the same sum from broadcast reads, so no barrier is needed to share
// it (one thread summing while the others waited at two barriers measured
// about 1 % slower on a 200-epoch light curve).  The loads run a group of
// eight ahead of the additions, which stay in order, so the sum costs about
// one FP64 addition latency per cell; a group's cells past b load as +0.0,
// which leaves the sum unchanged (it starts at +0.0 and only grows).
template <int W>
__device__ __forceinline__ double chunk_sum(CartShared<W>& S, double acc, int a, int b)
{
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = (a + k < b) ? S.b[a + k] : 0.0;
    for (int j = a; j < b; j += 8) {
        double nv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) nv[k] = (j + 8 + k < b) ? S.b[j + 8 + k] : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) acc += v[k];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = nv[k];
    }
    return acc;
}

// cartesian_image_area_impl: one directional flood fill from `seed`
// (with stop_rows > 0, only until that many rows have completed).
//
// Every thread runs the same state machine on the same values, so the row
// bounds the scan needs again (the previous row's xmin and xmax, the current
// row's) are kept in registers instead of being read back from the scratch,
// which only rank 0 writes and which is read back only after the scan.  The
// row-key table slot of each row is fetched when the row starts, so its load
// overlaps the row's lens-map evaluations.
template <int W>
__device__ double image_area(Ctx& C, RowScratch& R, CartShared<W>& S, P2 seed, double dy, int& yi, int jsign,
                             int stop_rows = 0, bool have_pred = false, double pred_xmin = 0.0)
{
    constexpr int N = Grp<W>::N;
    double countx = 0.0, countall = 0.0, dz2 = 99999999.9;
    const double incr = fabs(dy);
    const double inv_incr = 1.0 / incr;
    double dx = incr;
    double ix = seed.x, iy = seed.y;
    double x0 = seed.x;
    int guard = 0;
    // Row bounds in registers (see above); the scan's first row follows the
    // predecessor row its caller prepared.  A row that ends with a count has
    // had both of its bounds set during its own scan, so the current row's
    // registers need no initial value.
    double prev_xmin = 0.0, cur_xmin = 0.0, cur_xmax = 0.0;
    rows_ensure<W>(R, yi);
    if (R.ovf) return countall;
    // The predecessor row's xmin: given by a caller that has just written it
    // (a gap repair), which saves reading it back.
    if (yi > 0) prev_xmin = have_pred ? pred_xmin : R.xmin[yi - 1];
    // Row-key table slot of the current row, fetched ahead.
    int key = row_key(iy, inv_incr);
    unsigned pre_h = key_hash(key, R.tmask);
    ulonglong2 pre = R.table[pre_h];
    // Chunk: cells [cidx, cend) from (chunk start, cy) along cdx; cidx is the
    // next one to consume.  On a block, a left-scan fill of a row whose right
    // scan has counted cells also evaluates the next row's first kSpecCells
    // right-scan cells, in chunk cells [kSpecAt, N): that row starts at
    // (cur_xmax - incr) + incr, one row up or down, and cur_xmax no longer
    // changes once the row has a count.  The next row takes those cells when
    // its start matches bit for bit (spec_x, spec_y), so every cell the scan
    // consumes has the value a fill at that position would give.  Likewise a
    // row's first right-scan fill (a scan's first row, a gap repair, or a
    // row whose right end moved past the next-row cells) evaluates
    // kFirstRight right-scan cells and, in chunk cells [kFirstRight, N), the
    // row's left-scan cells from (x0 - incr), which the left scan takes when
    // it starts there (lspec): a narrow row then needs one fill, not two.
    constexpr bool kSpec = W > 1;
    constexpr int kSpecCells = 32;
    constexpr int kSpecAt = N - kSpecCells;
    constexpr int kFirstRight = 32;
    bool have = false;
    int cidx = 0, cend = N;
    double cdx = 0.0, cy = 0.0;
    bool spec = false;
    double spec_x = 0.0, spec_y = 0.0;
    bool lspec = false, row_start = true;
    double lspec_x = 0.0, lspec_y = 0.0;
    for (;;) {
        if (!(have && cidx < cend && cdx == dx && cy == iy)) {
            if (kSpec && spec && dx == incr && spec_x == ix && spec_y == iy) {
                have = true;
                cidx = kSpecAt;
                cend = N;
                cdx = dx;
                cy = iy;
                spec = false;
            } else if (kSpec && lspec && dx == -incr && lspec_x == ix && lspec_y == iy) {
                have = true;
                cidx = kFirstRight;
                cend = N;
                cdx = dx;
                cy = iy;
                lspec = false;
            } else {
                if (C.budget > 0 && C.evals > C.budget) {
                    R.ovf = true;  // hand the point to the second pass
                    return countall;
                }
                const bool want_cont = dx != incr && yi != 0;
                const double thr = want_cont ? prev_xmin - dx : 0.0;
                const bool first_right = kSpec && dx == incr && row_start;
                const bool next_row = kSpec && dx != incr && countx != 0.0;
                int na = N;
                double nx = 0.0, ny = 0.0, thr2 = 0.0;
                bool want_cont2 = false;
                if (first_right) {
                    na = kFirstRight;
                    nx = x0 + (-incr);
                    ny = iy;
                    want_cont2 = yi != 0;
                    thr2 = want_cont2 ? prev_xmin - (-incr) : 0.0;
                } else if (next_row) {
                    na = kSpecAt;
                    nx = (cur_xmax - incr) + incr;
                    ny = iy + dy;
                }
                fill_chunk<W>(C, S, ix, iy, dx, jsign, want_cont, thr, na, nx, ny, want_cont2, thr2);
                have = true;
                cidx = 0;
                cend = na;
                cdx = dx;
                cy = iy;
                spec = next_row;
                spec_x = nx;
                spec_y = ny;
                lspec = first_right;
                lspec_x = nx;
                lspec_y = ny;
                row_start = false;
            }
        }
        // Bulk step: consume the run of cells that only accumulate (inside cells of
        // the right scan, or of the left scan once the row has a count) or only
        // step on (outside cells the left scan walks over before the row's first
        // inside cell, while abscissa >= xmin(previous row) + incr).  Needs every
        // inside cell to have brightness > 0, so "countx == 0" means "no inside
        // cell yet".
        if (C.bulk && guard + N + 2 < C.max_steps) {
            const bool counting = dx == incr || countx != 0.0;
            if (counting || yi != 0) {
                const int stop = first_event<W>(S, cidx, cend, counting);
                const int n = stop - cidx;
                if (n > 0) {
                    if (counting) {
                        if (C.uniform) countx += static_cast<double>(n);
                        else countx = chunk_sum<W>(S, countx, cidx, stop);
                        C.rays += n;
                    }
                    guard += n;
                    dz2 = S.d[stop - 1];
                    if (stop == cend) {
                        ix = S.x[cend - 1] + dx;
                        have = false;
                        continue;
                    }
                    ix = S.x[stop];
                    cidx = stop;
                }
            }
        }
        // Single-cell step: the reference's loop body (FSM:1919-2011).
        if (!(++guard < C.max_steps)) break;
        const double last = dz2;
        dz2 = S.d[cidx];
        const double b = S.b[cidx];
        ++cidx;
        rows_ensure<W>(R, yi);
        if (R.ovf) return countall;
        // Cells near the limb go on the refinement tape (FSM:1952-1961).
        if (C.tape && Grp<W>::rank() == 0 && fabs(dz2 - C.rho2) <= C.band)
            tape_add(C, ix, iy, dz2 <= C.rho2 ? b : 0.0);
        if (dz2 <= C.rho2) {
            if (dx == -incr && countx == 0.0) {
                cur_xmax = ix - dx;
                wset<W>(R.xmax, yi, cur_xmax);
            }
            countx += b;
            ++C.rays;
        } else if (dx == incr) {
            if (last <= C.rho2) {
                cur_xmax = ix;
                wset<W>(R.xmax, yi, ix);
            }
            dx = -incr;
            ix = x0;
            cur_xmin = ix + dx;
            wset<W>(R.xmin, yi, cur_xmin);
            have = false;
        } else {
            if (last <= C.rho2) {
                cur_xmin = ix;
                wset<W>(R.xmin, yi, ix);
            }
            if (yi != 0 && countx == 0.0) {
                rows_ensure<W>(R, yi - 1);
                if (ix >= prev_xmin - dx) {
                    ix += dx;
                    continue;
                }
            }
            countall += countx;
            wset<W>(R.ax, yi, countx);
            wset<W>(R.y, yi, iy);
            wset<W>(R.dys, yi, dy);
            if (countx == 0.0) {
                wset<W>(R.dys, yi, -dy);
                break;
            }
            // Same-row overlap with an earlier row of this seed's scans (FSM:1990-1999).
            unsigned slot;
            int e;
            if (pre.x != R.gen) {
                slot = pre_h;
                e = -1;
            } else if ((int)(pre.y >> 32) == key) {
                slot = pre_h;
                e = (int)(pre.y & 0xffffffffull) - 1;
            } else {
                e = key_lookup(R, key, &slot);
                if (slot == 0xffffffffu) {
                    R.ovf = true;
                    return countall;
                }
            }
            const int head = e;
            for (int hops = 0; e >= 0 && hops < R.cap; ++hops) {
                if (cur_xmin + incr < R.xmax[e] && cur_xmax - incr > R.xmin[e]) return countall - countx;
                e = R.next[e];
            }
            // The row's entry goes into the table.  Every thread of the group
            // must have finished this row's reads of the table first (a row
            // can end inside the cells evaluated ahead, with no other group
            // barrier in it): a thread that lagged would otherwise find the
            // row's own entry and take the row for an overlap with itself.
            // Every thread then stores the same entry, so each one's later
            // probes see all rows up to this one in its own program order
            // and stop on the same slots as every other thread's.
            Grp<W>::sync();
            R.table[slot] = make_ulonglong2(R.gen, ((unsigned long long)(unsigned)key << 32) |
                                                       (unsigned long long)(unsigned)(yi + 1));
            if (Grp<W>::rank() == 0) R.next[yi] = head;
            ++yi;
            // A split point's down unit needs only the up scan's first row.
            if (stop_rows > 0 && yi >= stop_rows) return countall;
            rows_ensure<W>(R, yi);
            if (R.ovf) return countall;
            dx = incr;
            x0 = cur_xmax;
            prev_xmin = cur_xmin;
            ix = x0 - dx;
            iy += dy;
            countx = 0.0;
            have = false;
            key = row_key(iy, inv_incr);
            pre_h = key_hash(key, R.tmask);
            pre = R.table[pre_h];
            row_start = true;
        }
        ix += dx;
    }
    return countall;
}

struct Diag {
    int seed_count, processed, fold, boundary_rows, gap_repairs, overlaps;
    double max_jump;
};

// high_magnification_floor_coefficient (FSM:1017-1063).
__device__ double floor_coefficient(const Diag& d, double mag, double rho)
{
    const double am = fabs(mag);
    if (rho >= 0.1 && (d.gap_repairs > 0 || d.max_jump > 50.0)) return 0.06;
    if (rho < 1.0e-2 && d.seed_count <= 5 && am <= 10.0 && d.gap_repairs > 0 && d.max_jump > 20.0) return 0.035;
    if (rho < 1.0e-2 && d.seed_count <= 5 && am <= 10.0 && d.max_jump > 1000.0) return 0.04;
    if (rho < 1.0e-2 && d.seed_count >= 16 && d.overlaps >= 8 && d.gap_repairs >= 100 && d.max_jump > 1000.0 &&
        am <= 50.0)
        return 0.035;
    if (rho < 1.0e-2 && am <= 300.0) return 0.02;
    if (rho < 1.0e-2 && am <= 1000.0) return 0.04;
    if (rho < 1.0e-2 && d.seed_count <= 5 && d.gap_repairs > 0 && d.max_jump > 20.0) return 0.04;
    if (am <= 80.0 || d.gap_repairs <= 1000) return 0.0;
    return rho >= 1.0e-2 ? 0.04 : 0.05;
}

// cartesian_area_error_indicator (FSM:1065-1106).
__device__ double area_error(const Diag& d, double rho, int source_bins, double c, double dd)
{
    const int bins = source_bins > 1 ? source_bins : 1;
    const double flux = source_flux(rho, c, dd);
    if (!isfinite(flux) || flux <= 0.0 || rho <= 0.0) return 0.0;
    const double gw = rho >= 2.0e-2 ? 0.005 : ((rho < 1.0e-2 && d.seed_count >= 16) ? 0.015 : 0.03);
    const double ow = rho >= 2.0e-2 ? 0.005 : 0.02;
    const double bw = rho >= 2.0e-2 ? 0.012 : 0.03;
    double u = bw * static_cast<double>(d.boundary_rows) + gw * static_cast<double>(d.gap_repairs) +
               ow * static_cast<double>(d.overlaps) + 0.02 * static_cast<double>(d.fold > 0 ? d.fold : 0) +
               0.002 * static_cast<double>(d.seed_count - 5 > 0 ? d.seed_count - 5 : 0);
    if (rho >= 1.0e-3 && d.seed_count >= 16 && d.overlaps >= 8) {
        const double iw = rho < 1.0e-2 ? 0.001 : 0.0005;
        u += iw * static_cast<double>(d.seed_count) * static_cast<double>(d.overlaps);
    }
    if (rho >= 1.0e-3 && d.max_jump > 10.0) {
        const double jw = rho >= 2.0e-2 ? 0.2 : 4.0;
        u += jw * log10(d.max_jump / 10.0);
    }
    const double cell = (rho / static_cast<double>(bins)) * (rho / static_cast<double>(bins));
    const double e = 1.25 * u * cell / flux;
    return isfinite(e) ? e : 0.0;
}

// One gap-repair scan (FSM:2576-2663): pre-set the virtual predecessor row,
// flood from `es` in direction `dy`, drop the rows again if nothing was found.
template <int W>
__device__ __forceinline__ void repair(Ctx& C, RowScratch& R, CartShared<W>& S, P2 es, double xmin_v, double xmax_v,
                                       double dy, int& yi, int js, double& areai, double& areabound)
{
    rows_ensure<W>(R, yi);
    if (R.ovf) return;
    wset<W>(R.xmin, yi, xmin_v);
    wset<W>(R.xmax, yi, xmax_v);
    wset<W>(R.dys, yi, dy);
    // The scan reads no field of the predecessor row but its xmin, which it
    // is given; the barrier after the scan publishes rank 0's writes.
    ++yi;
    const double area0 = image_area<W>(C, R, S, es, dy, yi, js, 0, true, xmin_v);
    Grp<W>::sync();  // rows written by rank 0 just before the scan ended
    areai += area0;
    areabound += area0;
    if (area0 <= 0.0) --yi;
}

// ----- adaptive local refinement (fixed_inverse_ray_binary, FSM:3074-3289) -----

struct RefCell {
    double cx, cy, size, area, coarse, err;
    int depth;
    int pad;
};

// cell_weight (FSM:3088-3095): brightness at a point, 0 outside the source.
__device__ __forceinline__ double ref_weight(const Ctx& C, double x, double y)
{
    const double md2 = mapped_dist2(C.m, x, y, C.src);
    if (md2 > C.rho2) return 0.0;
    return C.uniform ? 1.0 : ld_lookup(C.ld, md2 / C.rho2);
}

// estimate_local_cell_error (FSM:3100-3127).
__device__ double ref_error(const Ctx& C, const RefCell& c)
{
    const double half = 0.5 * c.size;
    const double xs[4] = {c.cx - half, c.cx + half, c.cx - half, c.cx + half};
    const double ys[4] = {c.cy - half, c.cy - half, c.cy + half, c.cy + half};
    double sum = 0.0, lo = dinf(), hi = 0.0;
    int nonzero = 0;
    for (int k = 0; k < 4; ++k) {
        const double wgt = ref_weight(C, xs[k], ys[k]);
        sum += wgt;
        lo = (wgt < lo) ? wgt : lo;
        hi = (hi < wgt) ? wgt : hi;
        if (wgt > 0.0) ++nonzero;
    }
    const double avg = 0.25 * sum;
    const double center = fabs(avg - c.coarse);
    const double variation = 0.5 * (hi - lo);
    const double boundary = (nonzero > 0 && nonzero < 4) ? 0.25 * hi : 0.0;
    double m = center;
    if (m < variation) m = variation;
    if (m < boundary) m = boundary;
    return c.area * m;
}

// The binary max-heap of std::priority_queue (ordered by err): push sifts the
// new cell up past smaller parents; pop moves the last cell into the root's
// place by walking the hole down to a leaf along the larger child (the right
// one on ties) and sifting it back up, so cells of equal error leave in the
// same order as from the reference's queue.
__device__ void heap_up(RefCell* H, int hole, int top, const RefCell& v)
{
    int parent = (hole - 1) / 2;
    while (hole > top && H[parent].err < v.err) {
        H[hole] = H[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    H[hole] = v;
}

__device__ void heap_push(RefCell* H, int& n, const RefCell& v)
{
    heap_up(H, n, 0, v);
    ++n;
}

__device__ RefCell heap_pop(RefCell* H, int& n)
{
    const RefCell top = H[0];
    if (n > 1) {
        const RefCell v = H[n - 1];
        H[n - 1] = H[0];
        const int len = n - 1;
        int hole = 0, second = 0;
        while (second < (len - 1) / 2) {
            second = 2 * (second + 1);
            if (H[second].err < H[second - 1].err) --second;
            H[hole] = H[second];
            hole = second;
        }
        if ((len & 1) == 0 && second == (len - 2) / 2) {
            second = 2 * (second + 1);
            H[hole] = H[second - 1];
            hole = second - 1;
        }
        heap_up(H, hole, 0, v);
    }
    --n;
    return top;
}

struct Refined {
    double A, err;
    int level;
    bool ovf;
};

// The refinement loop (FSM:3201-3280) over the tape, by one thread; the heap
// lives in `heap` (capacity `cap` cells).  `err0` is the scan's error
// estimate, `level0` the refinement level before the loop (1 after a
// topology retry).
__device__ Refined refine(const Ctx& C, const FsSettingsDev& st, double A, double err0, double scale, int active_bins,
                          int level0,
                          RefCell* heap, int cap)
{
    Refined out{A, err0, level0, false};
    const double safety =
        st.source_bins < 32 ? 8.0 : (C.rho >= 8.0e-3 ? 2.5 : (C.rho >= 3.0e-3 ? 1.8 : 1.25));
    auto guarded = [&](double mag) { return (st.tol + st.reltol * dmax_(fabs(mag), 1.0)) / safety; };
    int n = 0;
    double lerr = 0.0;
    for (int i = 0; i < C.tape_n; ++i) {
        RefCell c{C.tape[i].x, C.tape[i].y, C.step, 1.0, C.tape[i].w, 0.0, 0, 0};
        c.err = ref_error(C, c);
        lerr += c.err;
        if (n >= cap) {
            out.ovf = true;
            return out;
        }
        heap_push(heap, n, c);
    }
    double corr = 0.0;
    const int max_bins = active_bins > st.max_source_bins ? active_bins : st.max_source_bins;
    int max_depth = 0;
    for (int bins = active_bins > 1 ? active_bins : 1; bins < max_bins && max_depth < 8; bins *= 2) ++max_depth;
    const int max_splits = 4 * max_bins > 64 ? 4 * max_bins : 64;
    int splits = 0, level = level0;
    while (n > 0 && lerr > guarded(A + corr / scale) * scale && splits < max_splits) {
        RefCell parent = heap_pop(heap, n);
        if (parent.err <= 0.0 || parent.depth >= max_depth) break;
        int batch = 0;
        bool defer = false;
        while (batch < 1 && parent.depth < max_depth && lerr > guarded(A + corr / scale) * scale &&
               splits < max_splits) {
            defer = false;
            // split_cell (FSM:3128-3147).
            RefCell ch[4];
            const double size = 0.5 * parent.size;
            const double off = 0.25 * parent.size;
            const double cxs[4] = {parent.cx - off, parent.cx + off, parent.cx - off, parent.cx + off};
            const double cys[4] = {parent.cy - off, parent.cy - off, parent.cy + off, parent.cy + off};
            double contribution = 0.0, child_err = 0.0;
            int worst = 0;
            for (int k = 0; k < 4; ++k) {
                ch[k] = RefCell{cxs[k], cys[k], size, 0.25 * parent.area, ref_weight(C, cxs[k], cys[k]), 0.0,
                                parent.depth + 1, 0};
                ch[k].err = ref_error(C, ch[k]);
            }
            for (int k = 0; k < 4; ++k) {
                contribution += ch[k].area * ch[k].coarse;
                child_err += ch[k].err;
                if (ch[k].err > ch[worst].err) worst = k;
            }
            const RefCell wc = ch[worst];
            corr += contribution - parent.area * parent.coarse;
            lerr += child_err - parent.err;
            level = level > parent.depth + 1 ? level : parent.depth + 1;
            ++splits;
            ++batch;
            if (n + 4 > cap) {
                out.ovf = true;
                return out;
            }
            if (lerr <= guarded(A + corr / scale) * scale || wc.err <= 0.0 || wc.depth >= max_depth) {
                for (int k = 0; k < 4; ++k) heap_push(heap, n, ch[k]);
                defer = false;
                break;
            }
            for (int k = 0; k < 4; ++k)
                if (k != worst) heap_push(heap, n, ch[k]);
            parent = wc;
            defer = true;
        }
        if (defer) {
            if (n >= cap) {
                out.ovf = true;
                return out;
            }
            heap_push(heap, n, parent);
        }
    }
    if (level > 0) out.A = A + corr / scale;
    double e = safety * lerr / scale;
    if (level == 0 && st.ld_c == 0.0 && st.ld_d == 0.0) e = (e < err0) ? err0 : e;
    out.err = e;
    out.level = level;
    return out;
}

// The row scratch at `base` (cartesian_scratch_bytes(cap, seed_cap) bytes):
// five row arrays and the per-seed areas (doubles), the row-key table
// (16-byte entries), then the row chains and the per-seed flags (ints).
__device__ __forceinline__ RowScratch rows_at(char* base, int cap, int seed_cap, double** areaimage, int** flags)
{
    RowScratch R;
    R.xmin = reinterpret_cast<double*>(base);
    R.xmax = R.xmin + cap;
    R.ax = R.xmax + cap;
    R.y = R.ax + cap;
    R.dys = R.y + cap;
    double* ai = R.dys + cap;
    R.table = reinterpret_cast<ulonglong2*>((reinterpret_cast<uintptr_t>(ai + seed_cap) + 15) &
                                            ~static_cast<uintptr_t>(15));
    R.tmask = (unsigned)table_slots(cap) - 1u;
    R.next = reinterpret_cast<int*>(R.table + table_slots(cap));
    R.cap = cap;
    R.hw = 0;
    R.gen = 0;
    R.ovf = false;
    if (areaimage) *areaimage = ai;
    if (flags) *flags = R.next + cap + 2;  // per seed: bit0 overlapped (skip), bit1 subtracted
    return R;
}

// The units of a split early point: seed ii's up scan is unit 2 ii, its down
// scan unit 2 ii + 1, each with a SplitInfo naming its kSplitRowCap-row
// scratch area (slot) in the pool at `scratch`.
struct SplitUse {
    const SplitInfo* info;
    char* scratch;
    long long bytes;
    int seed_cap;
    const SeedInfo* seeds;  // the point's seeds after their gap repairs (kSplitSeeds)
};

__device__ __forceinline__ SplitInfo load_info(const SplitInfo* p)
{
    SplitInfo v;
    v.area = __ldcg(&p->area);
    v.rays = __ldcg(&p->rays);
    v.yi_final = __ldcg(&p->yi_final);
    v.pred = __ldcg(&p->pred);
    v.ok = __ldcg(&p->ok);
    v.slot = __ldcg(&p->slot);
    for (int i = 0; i < 3; ++i) v.row0[i] = __ldcg(&p->row0[i]);
    return v;
}

__device__ __forceinline__ bool same_bits(double a, double b)
{
    return __double_as_longlong(a) == __double_as_longlong(b);
}

// Seed ii's two directional scans taken from its units instead of run here:
// R receives the up scan's rows, the predecessor row the down scan starts
// from, then the down scan's rows, at the indices one scan of the seed
// gives them, and yi, areai and the cell count follow as after the two
// scans (the caller sets R.hw, yi, areai and the cells from the result).
// The two scans of one seed are independent: the down scan reads
// the first row's bounds (its unit scans that row itself and stops) and
// rows of its own row keys, and every down-scan row lies below every up-scan
// row, so when the down scan's first key is below the up scan's first key
// (keys grow with y) no key is shared.  The rows are not yet in the row-key
// table: fill_table enters them when a gap repair is about to read it, and
// n_up is the up scan's row count for that.  ok = false, with R untouched:
// a unit did not fit its rows, the keys could meet, or the merged rows would
// not fit R; the seed is then scanned here.
struct MergeOut {
    bool ok;
    int yi, n_up, hw;
    double areai;
    unsigned long long rays;
};

template <int W>
__device__ __noinline__ MergeOut merge_halves(RowScratch R, SplitUse sp, int ii, P2 seed, double incr)
{
    constexpr int N = Grp<W>::N;
    const int t = Grp<W>::rank();
    MergeOut m{false, 0, 0, 0, 0.0, 0ull};
    const SplitInfo U = load_info(sp.info + 2 * ii);
    const SplitInfo D = load_info(sp.info + 2 * ii + 1);
    if (!U.ok || !D.ok) return m;
    const double inv_incr = 1.0 / incr;
    if (!(row_key(seed.y + (-incr), inv_incr) < row_key(seed.y, inv_incr))) return m;
    const RowScratch UR = rows_at(sp.scratch + (long long)U.slot * sp.bytes, kSplitRowCap, sp.seed_cap, nullptr,
                                  nullptr);
    const RowScratch DR = rows_at(sp.scratch + (long long)D.slot * sp.bytes, kSplitRowCap, sp.seed_cap, nullptr,
                                  nullptr);
    const int nu = U.yi_final;
    if (D.pred != (nu > 0 ? 1 : 0)) return m;
    const double x0m = __ldcg(UR.xmin), x0M = __ldcg(UR.xmax), y0 = __ldcg(UR.y);
    if (!same_bits(D.row0[0], x0m) || !same_bits(D.row0[1], x0M) || !same_bits(D.row0[2], y0)) return m;
    const int total = nu + (D.yi_final - D.pred);
    if (total + 1 > R.cap) return m;
    for (int r = t; r <= total; r += N) {
        const bool up = r <= nu;
        const RowScratch& Q = up ? UR : DR;
        const int q = up ? r : D.pred + (r - nu);
        R.xmin[r] = __ldcg(Q.xmin + q);
        R.xmax[r] = __ldcg(Q.xmax + q);
        R.ax[r] = __ldcg(Q.ax + q);
        R.y[r] = __ldcg(Q.y + q);
        R.dys[r] = __ldcg(Q.dys + q);
    }
    Grp<W>::sync();
    // The predecessor row: the first row's bounds and y, direction down (its
    // ax stays what the up scan left at that index).
    if (t == 0) {
        R.xmin[nu] = x0m;
        R.xmax[nu] = x0M;
        R.y[nu] = y0;
        R.dys[nu] = -incr;
    }
    Grp<W>::sync();
    m.ok = true;
    m.yi = total;
    m.n_up = nu;
    m.hw = total + 1;
    m.areai = U.area;
    m.areai += D.area;
    m.rays = U.rays + D.rays;
    return m;
}

// Enters a merged seed's rows into the row-key table in row order, as its
// two scans would have: rows [0, n_up) and (n_up, yi) (the predecessor row
// and the down scan's last row never get an entry).  By rank 0, then a
// barrier; true (in every thread) when the table is full.
template <int W>
__device__ __noinline__ bool fill_table(RowScratch R, int n_up, int yi, double incr)
{
    bool full = false;
    if (Grp<W>::rank() == 0) {
        const double inv_incr = 1.0 / incr;
        for (int r = 0; r < yi; ++r) {
            if (r == n_up) continue;
            const int key = row_key(R.y[r], inv_incr);
            unsigned slot;
            const int e = key_lookup(R, key, &slot);
            if (slot == 0xffffffffu) {
                full = true;
                break;
            }
            R.next[r] = e;
            R.table[slot] = make_ulonglong2(R.gen, ((unsigned long long)(unsigned)key << 32) |
                                                       (unsigned long long)(unsigned)(r + 1));
        }
    }
    Grp<W>::sync();
    return Grp<W>::any(full);
}

// A seed whose split units and gap repairs are done: its rows [0, nyi]
// copied from the up half's area into R, and its results.  ok = false (R
// untouched) when the seed's block could not complete it.
struct SeedTake {
    bool ok;
    int nyi, repairs;
    double areai, max_jump;
    unsigned long long rays;
};

template <int W>
__device__ __noinline__ SeedTake take_seed(RowScratch R, SplitUse sp, int ii)
{
    constexpr int N = Grp<W>::N;
    const int t = Grp<W>::rank();
    SeedTake k{false, 0, 0, 0.0, 0.0, 0ull};
    const SeedInfo* p = sp.seeds + ii;
    if (__ldcg(&p->ok) != 1) return k;
    const int nyi = __ldcg(&p->nyi);
    if (nyi + 1 > R.cap) return k;
    const RowScratch UR = rows_at(sp.scratch + (long long)__ldcg(&sp.info[2 * ii].slot) * sp.bytes, kSplitRowCap,
                                  sp.seed_cap, nullptr, nullptr);
    for (int r = t; r <= nyi; r += N) {
        R.xmin[r] = __ldcg(UR.xmin + r);
        R.xmax[r] = __ldcg(UR.xmax + r);
        R.ax[r] = __ldcg(UR.ax + r);
        R.y[r] = __ldcg(UR.y + r);
        R.dys[r] = __ldcg(UR.dys + r);
    }
    Grp<W>::sync();
    k.ok = true;
    k.nyi = nyi;
    k.repairs = __ldcg(&p->repairs);
    k.areai = __ldcg(&p->areai);
    k.max_jump = __ldcg(&p->max_jump);
    k.rays = __ldcg(&p->rays);
    return k;
}

// The gap-repair walk of one seed's rows (FSM:2576-2663, the rows loop of
// inverse_ray_cartesian_binary_mag) after its two directional scans, which
// left yi rows and the area areai; n_up >= 0: the scans came from split units
// and their rows enter the row-key table before the first repair.  Returns
// the walk's final row count nyi (the rows the bookkeeping reads); the
// largest row jump and the repair count accumulate into max_jump and
// gap_repairs.
template <int W>
__device__ __forceinline__ int repair_walk(Ctx& C, RowScratch& R, CartShared<W>& S, int js, double incr, int& yi,
                                           double& areai, int n_up, double& max_jump, int& gap_repairs)
{
    constexpr int N = Grp<W>::N;
    const int t = Grp<W>::rank();
    auto table_ready = [&]() {
        if (n_up >= 0) {
            if (fill_table<W>(R, n_up, yi, incr)) R.ovf = true;
            n_up = -1;
        }
    };
    int nyi = yi;
    double areabound = 0.0;
    // The repairs of one row (FSM:2576-2663), in the reference's order.
    auto repair_row = [&](int row, double dxmax, double dxmin) {
        if (dxmax > 1.1 * incr) {
            ++gap_repairs;
            table_ready();
            repair<W>(C, R, S, P2{R.xmax[row + 1], R.y[row]}, R.xmax[row], R.xmax[row + 1], -R.dys[row], yi,
                      js, areai, areabound);
        }
        if (dxmin > 1.1 * incr) {
            ++gap_repairs;
            table_ready();
            repair<W>(C, R, S, P2{R.xmin[row + 1] - incr, R.y[row + 1]}, R.xmin[row], R.xmin[row + 1],
                      R.dys[row], yi, js, areai, areabound);
        }
        if (dxmin < -1.1 * incr) {
            ++gap_repairs;
            table_ready();
            repair<W>(C, R, S, P2{R.xmin[row] - incr, R.y[row]}, R.xmin[row + 1], R.xmin[row], -R.dys[row], yi,
                      js, areai, areabound);
        }
        if (dxmax < -1.1 * incr) {
            ++gap_repairs;
            table_ready();
            repair<W>(C, R, S, P2{R.xmax[row + 1] + incr, R.y[row + 1]}, R.xmax[row + 1], R.xmax[row],
                      R.dys[row], yi, js, areai, areabound);
        }
    };
    // The reference walks rows [0, nyi) one by one, and when its last row
    // has added rows with area it walks those too.  A repair only writes
    // rows from yi >= nyi on, so for every row but a walk's last one the
    // row and its successor are as the scans left them: the group reads
    // their conditions N rows at a time and runs the repairs they call
    // for in row order.  The last row, whose successor a repair may have
    // overwritten, is read after them, as the reference reads it.  The
    // largest row jump is a maximum, so its order does not matter.
    int lo = 0;
    while (lo < nyi && !R.ovf) {
        const int hi = nyi;
        rows_ensure<W>(R, hi);
        for (int base = lo; base < hi - 1 && !R.ovf; base += N) {
            const int row = base + t;
            bool ev = false;
            double jmp = 0.0;
            if (row < hi - 1 && R.ax[row + 1] > 0.0) {
                const double dxmax = R.xmax[row + 1] - R.xmax[row];
                const double dxmin = R.xmin[row + 1] - R.xmin[row];
                jmp = dmax_(fabs(dxmax), fabs(dxmin)) / incr;
                ev = dxmax > 1.1 * incr || dxmin > 1.1 * incr || dxmin < -1.1 * incr || dxmax < -1.1 * incr;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) jmp = dmax_(jmp, __shfl_xor_sync(kFull, jmp, o));
            const unsigned wb = __ballot_sync(kFull, ev);
            if (lane_id() == 0) {
                S.ev[Grp<W>::warp()] = wb;
                S.mx[Grp<W>::warp()] = jmp;
            }
            Grp<W>::sync();
            unsigned evw[W];
            double gm = 0.0;
#pragma unroll
            for (int w8 = 0; w8 < W; ++w8) {
                evw[w8] = S.ev[w8];
                gm = dmax_(gm, S.mx[w8]);
            }
            Grp<W>::sync();
            max_jump = dmax_(max_jump, gm);
#pragma unroll 1
            for (int w8 = 0; w8 < W && !R.ovf; ++w8) {
                unsigned m = evw[w8];
                while (m && !R.ovf) {
                    const int r = base + 32 * w8 + __ffs(m) - 1;
                    m &= m - 1u;
                    repair_row(r, R.xmax[r + 1] - R.xmax[r], R.xmin[r + 1] - R.xmin[r]);
                }
            }
        }
        if (!R.ovf) {
            const int row = hi - 1;
            rows_ensure<W>(R, row + 1);
            const double dxmax = R.xmax[row + 1] - R.xmax[row];
            const double dxmin = R.xmin[row + 1] - R.xmin[row];
            if (R.ax[row + 1] > 0.0) {
                max_jump = dmax_(max_jump, dmax_(fabs(dxmax), fabs(dxmin)) / incr);
                repair_row(row, dxmax, dxmin);
            }
        }
        if (areabound > 0.0 && yi > nyi) {
            lo = hi;
            nyi = yi;
        } else {
            break;
        }
    }
    return nyi;
}

// One scan of a point's lattice (inverse_ray_cartesian_binary_mag,
// FSM:2470-2768) at `source_bins` cells per source radius: the directional
// flood fills of every seed that no earlier seed's rows cover, their gap
// repairs and the overlap bookkeeping between seeds.  Leaves the summed
// brightness in `area` and the scan's diagnostics in `d`; returns true when
// the scan outgrew the group's scratch (rows or the row-key table).
template <int W>
__device__ bool scan_point(Ctx& C, RowScratch& R, CartShared<W>& S, const P2* seeds, int ns, double rho,
                           int source_bins, unsigned long long epoch, unsigned long long& local_gen,
                           double* areaimage, int* flags, Diag& d, double& area, const SplitUse* sp = nullptr)
{
    constexpr int N = Grp<W>::N;
    const int t = Grp<W>::rank();
    const double nbin = static_cast<double>(max(source_bins, 1));
    const double incr = rho / nbin;
    C.max_steps = max(100000, source_bins * source_bins * 2000);
    C.band = dmax_(4.0 * rho * incr, 4.0 * incr * incr);
    C.step = incr;
    C.tape_n = 0;
    const double margin = 0.5 * incr * 1.01;
    bool ovf = false;
    for (int i = t; i < ns; i += N) {
        areaimage[i] = 0.0;
        flags[i] = 0;
    }
    Grp<W>::sync();
    area = 0.0;
    for (int ii = 0; ii < ns && !ovf; ++ii) {
        if (flags[ii] & 1) continue;
        ++local_gen;
        R.gen = (epoch << 32) | (local_gen & 0xffffffffull);
        R.hw = 0;
        R.ovf = false;
        rows_ensure<W>(R, 1);
        const P2 seed = seeds[ii];
        if (C.f32) C.A = make_anchor32(C.m, seed.x, seed.y, C.src);
        double areai = 0.0;
        double dy = incr;
        int yi = 0;
        const double jseed = jacobian(C.m, seed.x, seed.y);
        const int js = (fabs(jseed) < 0.02) ? sign_of(jseed) : 0;
        ++d.processed;
        if (js != 0) ++d.fold;
        // A split point's first kSplitSeeds seeds come scanned and repaired
        // from their units (seed_finish); the others, and any seed its
        // block could not complete, are scanned here.
        int nyi = 0;
        SeedTake tk{false, 0, 0, 0.0, 0.0, 0ull};
        if (sp != nullptr && ii < kSplitSeeds) tk = take_seed<W>(R, *sp, ii);
        if (tk.ok) {
            nyi = tk.nyi;
            yi = tk.nyi;
            R.hw = tk.nyi + 1;
            areai = tk.areai;
            C.rays += tk.rays;
            d.max_jump = dmax_(d.max_jump, tk.max_jump);
            d.gap_repairs += tk.repairs;
        } else {
            wset<W>(R.xmin, 0, seed.x);
            wset<W>(R.xmax, 0, seed.x);
            Grp<W>::sync();
            areai = image_area<W>(C, R, S, seed, dy, yi, js);
            Grp<W>::sync();
            dy = -incr;
            rows_ensure<W>(R, yi);
            if (R.ovf) {
                ovf = true;
                break;
            }
            const P2 lower{R.xmax[0], seed.y + dy};
            {
                const double xm0 = R.xmin[0], xM0 = R.xmax[0], y0 = R.y[0];
                Grp<W>::sync();
                wset<W>(R.xmin, yi, xm0);
                wset<W>(R.xmax, yi, xM0);
                wset<W>(R.y, yi, y0);
                wset<W>(R.dys, yi, dy);
                Grp<W>::sync();
            }
            ++yi;
            areai += image_area<W>(C, R, S, lower, dy, yi, js);
            Grp<W>::sync();
            nyi = repair_walk<W>(C, R, S, js, incr, yi, areai, -1, d.max_jump, d.gap_repairs);
        }
        if (R.ovf) {
            ovf = true;
            break;
        }
        area += areai;
        if (t == 0) areaimage[ii] = areai;
        {
            int br = 0;
            for (int row = t; row < nyi; row += N) br += (R.ax[row] > 0.0) ? 1 : 0;
            br = warp_sum_i(br);
            if (W > 1) {
                if (lane_id() == 0) S.red[warp_in_block()] = br;
                __syncthreads();
                br = 0;
                for (int i = 0; i < W; ++i) br += S.red[i];
                __syncthreads();
            }
            d.boundary_rows += br;
        }
        // Overlap bookkeeping against every other seed (FSM:2681-2739).
        for (int oi = 0; oi < ns; ++oi) {
            if (oi == ii) continue;
            const P2 p = seeds[oi];
            if (js != 0) {
                if (sign_of(jacobian(C.m, p.x, p.y)) == -js) continue;
                if (rho >= 4.0e-3 && source_bins >= 35 && oi > ii && fabs(jseed) < 1.0e-3 &&
                    fabs(jacobian(C.m, p.x, p.y)) < 0.02)
                    continue;
            }
            bool hit = false;
            for (int r0 = 0; r0 < nyi; r0 += N) {
                const int row = r0 + t;
                bool h = false;
                if (row < nyi && R.ax[row] > 0.0) {
                    h = p.y >= R.y[row] - margin && p.y <= R.y[row] + margin &&
                        p.x >= R.xmin[row] - margin && p.x <= R.xmax[row] + margin;
                }
                if (Grp<W>::any(h)) {
                    hit = true;
                    break;
                }
            }
            if (hit) {
                ++d.overlaps;
                if (oi < ii) {
                    const int f = flags[oi];
                    if (!(f & 2)) {
                        area -= areaimage[oi];
                        Grp<W>::sync();
                        if (t == 0) flags[oi] = f | 2;
                    }
                } else {
                    if (t == 0) flags[oi] = flags[oi] | 1;
                }
                Grp<W>::sync();
            }
        }
        Grp<W>::sync();
    }
    return ovf;
}

// The list a kernel instance works through.
struct CartList {
    const int* slots;   // inverse-ray Cartesian slot of each entry (null: the identity)
    const int* count;
    int* next;          // dynamic work counter
};

// The per-point state of a scan (cartesian_body, run_unit): the point's lens
// map, source and limb-darkening table (copied to ld_smem, when given, once
// per table), and the scan limits.
template <int W>
__device__ void init_ctx(Ctx& C, const FsWork& w, const FsItem& item, const FsSettingsDev& st, TapeCell* tape,
                         double* ld_smem, int& ld_loaded)
{
    const int t = Grp<W>::rank();
    const double rho = item.rho;
    C.m = make_mapper(item.s, item.q);
    C.src = P2{item.x, item.y};
    C.rho = rho;
    C.rho2 = rho * rho;
    C.inv_rho2 = 1.0 / C.rho2;
    C.uniform = st.ld_c == 0.0 && st.ld_d == 0.0;
    // I(r^2) >= 1 - c - d on [0, 1] for c, d >= 0, so every counted cell adds > 0.
    C.bulk = C.uniform || (st.ld_c >= 0.0 && st.ld_d >= 0.0 && st.ld_c + st.ld_d < 1.0);
    C.ld = w.ld_tables + (long long)st.ld_table * (kLdTable + 1);
    C.lds = nullptr;
    if (ld_smem != nullptr && !C.uniform) {
        // A block scan keeps its point's table in shared memory: the
        // brightness lookup ends every cell's evaluation.
        if (ld_loaded != st.ld_table) {
            Grp<W>::sync();
            for (int i = t; i <= kLdTable; i += Grp<W>::N) ld_smem[i] = C.ld[i];
            Grp<W>::sync();
            ld_loaded = st.ld_table;
        }
        C.lds = ld_smem;
    }
    C.max_steps = max(100000, st.source_bins * st.source_bins * 2000);
    C.f32 = w.f32_rays != 0;
    // Adaptive local refinement records the scan's boundary cells, so
    // every cell goes through the reference's loop body (no bulk runs).
    const bool adaptive = tape && st.adaptive_source_bins != 0 && (st.tol > 0.0 || st.reltol > 0.0);
    C.tape = adaptive ? tape : nullptr;
    C.tape_max = max(64, st.max_source_bins);
    if (C.tape_max > kTapeMax) C.tape_max = kTapeMax;
    if (adaptive) C.bulk = false;
}

// One unit of a split early point (early point e, seed ii, half 0 up or 1
// down): the seed's directional scan at the point's source_bins into a row
// scratch area of its own, exactly as scan_point runs it (the down half
// first scans the up scan's first row itself, for the bounds it starts
// from, and counts only its own cells).  The result goes to the unit's
// SplitInfo; a missing point or seed, a pool with no area left, or a scan
// that outgrows the area's rows leaves ok = 0, and the finishing block scans
// that seed itself.
struct UnitArgs {
    int* slots_taken;
    int split_slots;
    SeedInfo* seed_info;
    const int* early_cart;
    const int* ir_cart;
    const FsItem* items;
    const FsOut* out;
    const FsSettingsDev* settings;
    const double* ld_tables;
    const P2* seeds;
    char* split_scratch;
    SplitInfo* split_info;
    long long split_bytes;
    int seed_cap;
    int f32_rays;
};

template <int W>
__device__ __noinline__ int run_unit(UnitArgs w, unsigned long long epoch, int e, int ii, int half, CartShared<W>& S,
                                     double* ld_smem, int ld_loaded)
{
    const int u = (e * kSplitSeeds + ii) * 2 + half;
    SplitInfo info{};
    const int k = w.early_cart[e];
    const int it = w.ir_cart[k];
    const FsItem item = w.items[it];
    const FsOut o = w.out[it];
    int slot = -1;
    if (o.status == kFsOk && ii < o.n_seeds && item.rho > 0.0) {
        if (Grp<W>::rank() == 0) {
            const int a = atomicAdd(w.slots_taken, 1);
            S.item = a < w.split_slots ? a : -1;
        }
        Grp<W>::sync();
        slot = S.item;
        Grp<W>::sync();
    }
    if (slot >= 0) {
        const FsSettingsDev st = w.settings[item.settings];
        Ctx C;
        C.rays = 0;
        C.evals = 0;
        C.budget = 0;
        FsWork lw{};
        lw.ld_tables = w.ld_tables;
        lw.f32_rays = w.f32_rays;
        init_ctx<W>(C, lw, item, st, nullptr, ld_smem, ld_loaded);
        RowScratch R = rows_at(w.split_scratch + (long long)slot * w.split_bytes, kSplitRowCap, w.seed_cap, nullptr,
                               nullptr);
        info.slot = slot;
        R.gen = (epoch << 32) | 1ull;
        const double incr = item.rho / static_cast<double>(max(st.source_bins, 1));
        C.band = dmax_(4.0 * item.rho * incr, 4.0 * incr * incr);
        C.step = incr;
        C.tape_n = 0;
        rows_ensure<W>(R, 1);
        const P2 seed = w.seeds[(long long)k * w.seed_cap + ii];
        if (C.f32) C.A = make_anchor32(C.m, seed.x, seed.y, C.src);
        const double jseed = jacobian(C.m, seed.x, seed.y);
        const int js = (fabs(jseed) < 0.02) ? sign_of(jseed) : 0;
        wset<W>(R.xmin, 0, seed.x);
        wset<W>(R.xmax, 0, seed.x);
        Grp<W>::sync();
        int yi = 0;
        if (half == 0) {
            info.area = image_area<W>(C, R, S, seed, incr, yi, js);
            Grp<W>::sync();
            rows_ensure<W>(R, yi);
            info.yi_final = yi;
            info.rays = C.rays;
        } else {
            image_area<W>(C, R, S, seed, incr, yi, js, 1);
            Grp<W>::sync();
            const unsigned long long rays0 = C.rays;
            rows_ensure<W>(R, yi);
            if (!R.ovf) {
                const double dy = -incr;
                const double xm0 = R.xmin[0], xM0 = R.xmax[0], y0 = R.y[0];
                info.row0[0] = xm0;
                info.row0[1] = xM0;
                info.row0[2] = y0;
                const P2 lower{xM0, seed.y + dy};
                Grp<W>::sync();
                wset<W>(R.xmin, yi, xm0);
                wset<W>(R.xmax, yi, xM0);
                wset<W>(R.y, yi, y0);
                wset<W>(R.dys, yi, dy);
                Grp<W>::sync();
                info.pred = yi;
                ++yi;
                info.area = image_area<W>(C, R, S, lower, dy, yi, js);
                Grp<W>::sync();
                rows_ensure<W>(R, yi);
                info.yi_final = yi;
                info.rays = C.rays - rays0;
            }
        }
        info.ok = R.ovf ? 0 : 1;
    }
    if (Grp<W>::rank() == 0) w.split_info[u] = info;
    return ld_loaded;
}

// The second block to complete one of seed ii's halves (early point e)
// finishes the seed: it merges the two halves in its own scratch R, runs the
// seed's gap repairs there (a seed's rows and repairs touch no other seed's),
// and leaves the rows [0, nyi] in the up half's area and the results in the
// seed's SeedInfo, for the block that finishes the point.  A missing seed, a
// merge that cannot be taken, an overflow, or rows past the area leave
// ok = 0 and that block scans the seed itself.  The row-key tags use the
// epoch with a per-seed generation above every generation of scan_point.
template <int W>
__device__ __noinline__ int seed_finish(UnitArgs w, unsigned long long epoch, int e, int ii, CartShared<W>& S,
                                        double* ld_smem, int ld_loaded, RowScratch R)
{
    constexpr int N = Grp<W>::N;
    const int t = Grp<W>::rank();
    SeedInfo out{};
    const int k = w.early_cart[e];
    const int it = w.ir_cart[k];
    const FsItem item = w.items[it];
    const FsOut o = w.out[it];
    if (o.status == kFsOk && ii < o.n_seeds && item.rho > 0.0) {
        const FsSettingsDev st = w.settings[item.settings];
        Ctx C;
        C.rays = 0;
        C.evals = 0;
        C.budget = 0;
        FsWork lw{};
        lw.ld_tables = w.ld_tables;
        lw.f32_rays = w.f32_rays;
        init_ctx<W>(C, lw, item, st, nullptr, ld_smem, ld_loaded);
        const double incr = item.rho / static_cast<double>(max(st.source_bins, 1));
        C.band = dmax_(4.0 * item.rho * incr, 4.0 * incr * incr);
        C.step = incr;
        C.tape_n = 0;
        R.gen = (epoch << 32) | (0x80000000ull + static_cast<unsigned long long>(e * kSplitSeeds + ii));
        R.hw = 0;
        R.ovf = false;
        rows_ensure<W>(R, 1);
        const P2 seed = w.seeds[(long long)k * w.seed_cap + ii];
        if (C.f32) C.A = make_anchor32(C.m, seed.x, seed.y, C.src);
        const double jseed = jacobian(C.m, seed.x, seed.y);
        const int js = (fabs(jseed) < 0.02) ? sign_of(jseed) : 0;
        const SplitUse sp{w.split_info + (long long)e * 2 * kSplitSeeds, w.split_scratch, w.split_bytes, w.seed_cap,
                          nullptr};
        const MergeOut mo = merge_halves<W>(R, sp, ii, seed, incr);
        if (mo.ok) {
            int yi = mo.yi;
            R.hw = mo.hw;
            double areai = mo.areai;
            C.rays += mo.rays;
            double mj = 0.0;
            int reps = 0;
            const int nyi = repair_walk<W>(C, R, S, js, incr, yi, areai, mo.n_up, mj, reps);
            Grp<W>::sync();
            if (!R.ovf && nyi + 1 <= kSplitRowCap) {
                const RowScratch UR = rows_at(w.split_scratch + (long long)__ldcg(&sp.info[2 * ii].slot) *
                                                                   w.split_bytes,
                                              kSplitRowCap, w.seed_cap, nullptr, nullptr);
                for (int r = t; r <= nyi; r += N) {
                    UR.xmin[r] = R.xmin[r];
                    UR.xmax[r] = R.xmax[r];
                    UR.ax[r] = R.ax[r];
                    UR.y[r] = R.y[r];
                    UR.dys[r] = R.dys[r];
                }
                out.areai = areai;
                out.max_jump = mj;
                out.rays = C.rays;
                out.nyi = nyi;
                out.repairs = reps;
                out.ok = 1;
            }
        }
    }
    Grp<W>::sync();
    if (t == 0) w.seed_info[e * kSplitSeeds + ii] = out;
    return ld_loaded;
}

// Work items: the list's points in order, each with the group's scratch at
// `base`.  The early pass with split points (split_info set) takes instead
// the units of its points, kSplitSeeds seeds by two halves each, in list
// order (largest first), and the block whose unit completes a point's last
// unit finishes that point from the units' rows: the units of a point run
// on several blocks at once, so its scans take the time of the longest half
// instead of the sum of all.
template <int W>
__device__ void cartesian_body(const FsWork& w, unsigned long long epoch, CartList L, char* base, CartShared<W>& S,
                               TapeCell* tape, double* ld_smem = nullptr)
{
    int ld_loaded = -1;  // the limb-darkening table now in ld_smem
    const int t = Grp<W>::rank();
    const int cap = w.row_cap;
    double* areaimage;
    int* flags;
    RowScratch R = rows_at(base, cap, w.seed_cap, &areaimage, &flags);
    unsigned long long local_gen = w.gen_base;
    const int n = *L.count;
    const bool split = w.early_pass && w.split_info != nullptr && L.slots != nullptr;
    const int n_split = split ? min(n, kEarlyMax) : 0;
    const int n_units = n_split * 2 * kSplitSeeds;
    const int n_work = split ? n_units + (n - n_split) : n;
    for (;;) {
        Grp<W>::sync();
        if (t == 0) S.item = atomicAdd(L.next, 1);
        Grp<W>::sync();
        const int idx = S.item;
        if (idx >= n_work) break;
        int k = idx;
        int e = idx;  // early pass: the point's list position
        SplitUse su{nullptr, nullptr, 0, 0};
        const SplitUse* use = nullptr;
        if (split) {
            if (idx < n_units) {
                e = idx / (2 * kSplitSeeds);
                const UnitArgs ua{w.ir_count + kSplitAlloc, w.split_slots, w.seed_info, w.early_cart, w.ir_cart, w.items, w.out, w.settings,
                                  w.ld_tables, w.seeds, w.split_scratch, w.split_info, w.split_bytes, w.seed_cap,
                                  w.f32_rays};
                const int ii = (idx >> 1) % kSplitSeeds;
                ld_loaded = run_unit<W>(ua, epoch, e, ii, idx & 1, S, ld_smem, ld_loaded);
                // The second of a seed's halves to complete finishes the seed,
                // and the last seed of a point to complete finishes the point.
                __threadfence();
                Grp<W>::sync();
                if (t == 0) S.item = atomicAdd(w.ir_count + kSeedCounter + e * kSplitSeeds + ii, 1);
                Grp<W>::sync();
                if (S.item != 1) continue;
                __threadfence();
                ld_loaded = seed_finish<W>(ua, epoch, e, ii, S, ld_smem, ld_loaded, R);
                __threadfence();
                Grp<W>::sync();
                if (t == 0) S.item = atomicAdd(w.ir_count + kSplitCounter + e, 1);
                Grp<W>::sync();
                if (S.item != kSplitSeeds - 1) continue;
                __threadfence();
                su = SplitUse{w.split_info + (long long)e * 2 * kSplitSeeds, w.split_scratch, w.split_bytes,
                              w.seed_cap, w.seed_info + (long long)e * kSplitSeeds};
                use = &su;
            } else {
                e = n_split + (idx - n_units);
            }
        }
        if (w.early_pass) k = L.slots[e];
        else if (L.slots) k = L.slots[k];
        if (W == 1 && !w.retry_pass && w.early_cart != nullptr) {
            // Points routed to the early block pass are not run here.
            const int ne = w.ir_count[5];
            bool routed = false;
            for (int e = 0; e < ne; ++e) routed |= w.early_cart[e] == k;
            if (routed) continue;
        }
        const int it = w.ir_cart[k];
        const long long t_item = clock64();
        const FsItem item = w.items[it];
        FsOut o = w.out[it];
        if (o.status != kFsOk) continue;
        const FsSettingsDev st = w.settings[item.settings];
        const P2* seeds = w.seeds + (long long)k * w.seed_cap;
        const int ns = o.n_seeds;
        const double rho = item.rho;
        double A = dnan();
        bool ovf = false;
        Ctx C;
        C.rays = 0;
        C.evals = 0;
        C.budget = (W == 1 && !w.retry_pass) ? (n <= w.few_points ? 1 : w.cell_budget) : 0;
        if (ns > 0 && rho > 0.0) {
            init_ctx<W>(C, w, item, st, tape, ld_smem, ld_loaded);
            // The scan, and the topology retry of fixed_inverse_ray_binary
            // (FSM:3168-3196): when needs_global_topology_retry (FSM:1108-1121)
            // holds, the same seeds are scanned again at
            // min(max_source_bins, max(50, 2 source_bins)) bins, and that scan's
            // magnification, diagnostics and tape replace the first one's
            // (refinement level 1).  A retry that is not finite leaves the first
            // scan's results, which a third scan at the original bins restores
            // (its tape included).
            const int retry_bins = min(st.max_source_bins, max(50, 2 * max(st.source_bins, 1)));
            int bins = st.source_bins;  // the settings' source_bins of the current scan
            int level0 = 0;
            double err = 0.0, scale = 1.0;
            for (int attempt = 0;; ++attempt) {
                Diag d{ns, 0, 0, 0, 0, 0, 0.0};
                double area = 0.0;
                ovf = scan_point<W>(C, R, S, seeds, ns, rho, bins, epoch, local_gen, areaimage, flags, d, area,
                                    attempt == 0 ? use : nullptr);
                if (ovf) break;
                const double nb = static_cast<double>(max(bins, 1));
                const double flux = source_flux(rho, st.ld_c, st.ld_d);
                const double sc = flux / (rho * rho) * nb * nb;
                const double a = area / sc;
                if (attempt == 1 && !isfinite(a)) {
                    bins = st.source_bins;
                    continue;
                }
                double e = area_error(d, rho, bins, st.ld_c, st.ld_d);
                const double fc = floor_coefficient(d, a, rho);
                if (fc > 0.0) e = dmax_(e, fabs(a) * (fc / nb));
                A = a;
                err = e;
                scale = sc;
                if (attempt == 1) level0 = 1;
                if (attempt == 0 && isfinite(a) && st.adaptive_source_bins != 0 && st.source_bins < 50 &&
                    st.max_source_bins > st.source_bins && rho < 1.0e-2 && d.seed_count >= 16 &&
                    d.overlaps >= 100 && d.gap_repairs >= 1000 && d.max_jump >= 1000.0 &&
                    retry_bins > st.source_bins) {
                    bins = retry_bins;
                    continue;
                }
                break;
            }
            if (t == 0) w.rays[it] = C.rays;
            if (!ovf) {
                o.err = isfinite(A) ? err : dnan();
                const double target = st.tol + st.reltol * dmax_(fabs(A), 1.0);
                o.converged = isfinite(A) && err <= 0.999 * target;
                if (t == 0 && w.levels) w.levels[it] = level0;
                if (C.tape && isfinite(A)) {
                    const int active_bins = max(bins, 1);
                    Refined rf{A, err, level0, false};
                    if (t == 0 && C.tape_n > 0) {
                        // The row arrays are free once the scans are done: they hold the heap.
                        rf = refine(C, st, A, err, scale, active_bins, level0, reinterpret_cast<RefCell*>(R.xmin),
                                    static_cast<int>((5ll * cap * sizeof(double)) / sizeof(RefCell)));
                    }
                    if (t == 0) {
                        if (rf.ovf) {
                            o.status = kFsRowOverflow;
                        } else {
                            A = rf.A;
                            o.err = rf.err;
                            const double tg = st.tol + st.reltol * dmax_(fabs(A), 1.0);
                            o.converged = rf.err <= 0.999 * tg && active_bins >= 32;
                            if (w.levels) w.levels[it] = rf.level;
                        }
                    }
                }
            }
        }
        if (ovf && !w.retry_pass) {
            // Too large for one warp, or for this pass's scratch: the second pass
            // runs it again on a whole block with the large scratch.
            if (t == 0) w.retry_cart[atomicAdd(&w.ir_count[2], 1)] = k;
            continue;
        }
        o.A = A;
        if (ovf) o.status = kFsRowOverflow;
        else if (o.status == kFsOk && !isfinite(A)) o.status = kFsNumerical;
        if (o.status != kFsOk && o.status != kFsNumerical) o.A = dnan();
        if (t == 0) {
            w.out[it] = o;
            if (w.cycles) w.cycles[it] += clock64() - t_item;
        }
    }
}

__global__ void __launch_bounds__(128, 2) cartesian_warp_kernel(FsWork w, unsigned long long epoch)
{
    __shared__ CartShared<1> sh[4];
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const CartList L{nullptr, w.ir_count + 0, w.next_item + 1};
    cartesian_body<1>(w, epoch, L, w.scratch + (long long)gw * w.scratch_per_warp, sh[warp_in_block()],
                      w.tape ? w.tape + (long long)gw * kTapeMax : nullptr);
}

// Dynamic shared memory of the block kernel: one limb-darkening table.
constexpr size_t kBlockLdBytes = (size_t)(kLdTable + 1) * sizeof(double);

__global__ void __launch_bounds__(32 * kBigWarps, 1) cartesian_block_kernel(FsWork w, unsigned long long epoch)
{
    __shared__ CartShared<kBigWarps> sh;
    extern __shared__ double ld_smem[];
    const CartList L{w.retry_cart, w.ir_count + 2, w.next_item + 3};
    cartesian_body<kBigWarps>(w, epoch, L, w.scratch + (long long)blockIdx.x * w.scratch_per_warp, sh,
                              w.tape ? w.tape + (long long)blockIdx.x * kTapeMax : nullptr, ld_smem);
}

// The early pass: blocks of kEarlyWarps warps, one per SM.  Its work is the
// split points' seed-half units, each a serial row scan whose speed is set
// by latency, not by the SM's issue rate.  The point's limb-darkening table
// in shared memory (160 KB) leaves room for one block per SM; blocks without
// it (two per SM, the entries evaluated where needed or read through L1) were
// measured no faster on the 4,096-point batch.
__global__ void __launch_bounds__(32 * kEarlyWarps, 1) cartesian_early_kernel(FsWork w, unsigned long long epoch)
{
    __shared__ CartShared<kEarlyWarps> sh;
    extern __shared__ double ld_smem[];
    const CartList L{w.early_cart, w.ir_count + 5, w.next_item + 6};
    cartesian_body<kEarlyWarps>(w, epoch, L, w.scratch + (long long)blockIdx.x * w.scratch_per_warp, sh, nullptr,
                                ld_smem);
}

} // namespace

size_t cartesian_scratch_bytes(int row_cap, int seed_cap)
{
    return ((size_t)row_cap * 5 + seed_cap + 2) * sizeof(double) + (size_t)table_slots(row_cap) * sizeof(ulonglong2) +
           ((size_t)row_cap + 2 + seed_cap) * sizeof(int) + 256;
}

// First pass: one warp per point (n_groups warps).  Second pass
// (w.retry_pass): one block of kBigWarps warps per point, n_groups blocks,
// each with its own scratch.  Early pass (w.early_pass): n_groups blocks of
// kEarlyWarps warps, each with its own scratch.
cudaError_t launch_cartesian(const FsWork& w, int n_groups, cudaStream_t stream, unsigned long long epoch)
{
    if (w.retry_pass) {
        // The shared-memory limit is a per-device attribute of each kernel, set
        // before its first launch on each device (setting it again is harmless).
        static std::atomic<unsigned long long> attr_set{0};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_set.load() & bit)) {
            e = cudaFuncSetAttribute(cartesian_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kBlockLdBytes));
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(cartesian_early_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kBlockLdBytes));
            if (e != cudaSuccess) return e;
            attr_set.fetch_or(bit);
        }
        if (w.early_pass)
            cartesian_early_kernel<<<n_groups, 32 * kEarlyWarps, kBlockLdBytes, stream>>>(w, epoch);
        else
            cartesian_block_kernel<<<n_groups, 32 * kBigWarps, kBlockLdBytes, stream>>>(w, epoch);
    } else {
        cartesian_warp_kernel<<<(n_groups + 3) / 4, 128, 0, stream>>>(w, epoch);
    }
    return cudaGetLastError();
}

} // namespace lcbi
