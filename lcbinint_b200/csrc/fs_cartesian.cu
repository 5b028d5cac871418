// Cartesian inverse-ray integration, one warp per evaluation
// (inverse_ray_cartesian_binary_mag, finite_source_magnifier.cpp:2470-2768,
// with the row-scan flood fill cartesian_image_area_impl, :1891-2014).
//
// The reference walks the image plane one cell at a time: each row runs right
// from the previous row's right edge, then left, with gap repairs and overlap
// bookkeeping that depend on the order of visits.  A warp reproduces that walk
// exactly: the lens map of the next 32 cells along the current scan direction
// is evaluated in parallel (lane l takes the cell l steps ahead, its abscissa
// built by the same l successive additions the reference performs), and the
// state machine consumes those results in order.  Row bookkeeping lives in a
// per-warp global scratch area with the reference's zero-on-growth semantics,
// and the same-row overlap test uses a direct-mapped table keyed by the
// reference's integer row key, so the magnification is bit-identical.
#include "lcbi_fs_kernels.h"
#include "lcbi_warp.cuh"

#include <cstdint>

namespace lcbi {

namespace {

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

__device__ __forceinline__ void rows_ensure(RowScratch& R, int i)
{
    if (i < R.hw) return;
    if (i >= R.cap) {
        R.ovf = true;
        return;
    }
    for (int r = R.hw + lane_id(); r <= i; r += 32) {
        R.xmin[r] = 0.0;
        R.xmax[r] = 0.0;
        R.ax[r] = 0.0;
        R.y[r] = 0.0;
        R.dys[r] = 0.0;
    }
    R.hw = i + 1;
    __syncwarp();
}

// Row values are written by lane 0; every lane keeps the same control flow.
__device__ __forceinline__ void wset(double* a, int i, double v)
{
    if (lane_id() == 0) a[i] = v;
}

struct Ctx {
    unsigned long long rays;  // inside cells consumed (identical in every lane)
    bool bulk;                // every inside cell has brightness > 0 (run consumption allowed)
    Mapper m;
    P2 src;
    double rho, rho2, inv_rho2;
    bool uniform;
    const double* ld;
    int max_steps;
};

// Lens map of one cell, as the reference evaluates it for the current scan.
__device__ __forceinline__ void eval_for_scan(const Ctx& C, double x, double y, int jsign, double* dz2, double* bright)
{
    double md2;
    bool ok = true;
    if (jsign == 0) {
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
    if (d <= C.rho2) b = C.uniform ? 1.0 : ld_lookup(C.ld, md2 * C.inv_rho2);
    *bright = b;
}

__host__ __device__ inline long long table_slots(int cap)
{
    long long t = 1;
    while (t < 2ll * cap) t <<= 1;
    return t;
}

__device__ __forceinline__ int row_key(double y, double inv_incr) { return to_int_x86(y * inv_incr + kRowKeyOffset); }

// cartesian_image_area_impl: one directional flood fill from `seed`.
__device__ double image_area(Ctx& C, RowScratch& R, P2 seed, double dy, int& yi, int jsign)
{
    const int lane = lane_id();
    double countx = 0.0, countall = 0.0, dz2 = 99999999.9;
    const double incr = fabs(dy);
    const double inv_incr = 1.0 / incr;
    double dx = incr;
    double ix = seed.x, iy = seed.y;
    double x0 = seed.x;
    int guard = 0;
    // Speculative chunk: lane l holds the cell l steps from (cx, cy) along cdx.
    bool have = false;
    int cidx = 0;
    double cdx = 0.0, cy = 0.0;
    double my_x = 0.0, my_d = 0.0, my_b = 0.0;
    for (;;) {
        if (!(have && cidx < 32 && cdx == dx && cy == iy)) {
            double x = ix;
            for (int t = 0; t < 31; ++t)
                if (t < lane) x = x + dx;
            my_x = x;
            eval_for_scan(C, x, iy, jsign, &my_d, &my_b);
            have = true;
            cidx = 0;
            cdx = dx;
            cy = iy;
        }
        // Bulk step: consume, in one go, the run of cells whose processing only
        // accumulates (inside cells once the row has a count, or inside cells of
        // the right scan) or only steps on (outside cells the left scan walks
        // over before the row's first inside cell).  The next "eventful" cell
        // goes through the single-cell step below, which is the reference's
        // loop body verbatim.  Needs every inside cell to have brightness > 0,
        // so that "countx == 0" means "no inside cell yet".
        if (C.bulk && guard + 34 < C.max_steps) {
            const unsigned rem = kFull << cidx;
            const unsigned ins = __ballot_sync(kFull, my_d <= C.rho2) & rem;
            unsigned ev;
            bool counting;
            if (dx == incr || countx != 0.0) {
                ev = rem & ~ins;
                counting = true;
            } else if (yi != 0) {
                const double thr = R.xmin[yi - 1] - dx;
                const unsigned cont = __ballot_sync(kFull, my_x >= thr) & rem;
                ev = rem & ~(~ins & cont);
                counting = false;
            } else {
                ev = rem;
                counting = false;
            }
            const int stop = ev ? __ffs(ev) - 1 : 32;
            const int n = stop - cidx;
            if (n > 0) {
                if (counting) {
                    if (C.uniform) {
                        countx += static_cast<double>(n);
                    } else {
                        for (int j = cidx; j < stop; ++j) countx += shfl_d(my_b, j);
                    }
                    C.rays += n;
                }
                guard += n;
                dz2 = shfl_d(my_d, stop - 1);
                const double xl = shfl_d(my_x, stop == 32 ? 31 : stop);
                if (stop == 32) {
                    ix = xl + dx;
                    have = false;
                    continue;
                }
                ix = xl;
                cidx = stop;
            }
        }
        if (!(++guard < C.max_steps)) break;
        const double last = dz2;
        dz2 = shfl_d(my_d, cidx);
        const double b = shfl_d(my_b, cidx);
        ++cidx;
        rows_ensure(R, yi);
        if (R.ovf) return countall;
        if (dz2 <= C.rho2) {
            if (dx == -incr && countx == 0.0) wset(R.xmax, yi, ix - dx);
            countx += b;
            ++C.rays;
        } else if (dx == incr) {
            if (last <= C.rho2) wset(R.xmax, yi, ix);
            dx = -incr;
            ix = x0;
            wset(R.xmin, yi, ix + dx);
            have = false;
        } else {
            if (last <= C.rho2) wset(R.xmin, yi, ix);
            __syncwarp();
            if (yi != 0 && countx == 0.0) {
                rows_ensure(R, yi - 1);
                if (ix >= R.xmin[yi - 1] - dx) {
                    ix += dx;
                    continue;
                }
            }
            countall += countx;
            wset(R.ax, yi, countx);
            wset(R.y, yi, iy);
            wset(R.dys, yi, dy);
            if (countx == 0.0) {
                wset(R.dys, yi, -dy);
                __syncwarp();
                break;
            }
            __syncwarp();
            // Same-row overlap with an earlier row of this seed's scans (FSM:1990-1999).
            const int key = row_key(iy, inv_incr);
            unsigned slot;
            int e = key_lookup(R, key, &slot);
            if (slot == 0xffffffffu) {
                R.ovf = true;
                return countall;
            }
            const int head = e;
            const double xmin_y = R.xmin[yi], xmax_y = R.xmax[yi];
            for (int hops = 0; e >= 0 && hops < R.cap; ++hops) {
                if (xmin_y + incr < R.xmax[e] && xmax_y - incr > R.xmin[e]) return countall - countx;
                e = R.next[e];
            }
            if (lane == 0) {
                R.next[yi] = head;
                R.table[slot] = make_ulonglong2(R.gen, ((unsigned long long)(unsigned)key << 32) |
                                                           (unsigned long long)(unsigned)(yi + 1));
            }
            ++yi;
            rows_ensure(R, yi);
            if (R.ovf) return countall;
            __syncwarp();
            dx = incr;
            x0 = R.xmax[yi - 1];
            ix = x0 - dx;
            iy += dy;
            countx = 0.0;
            have = false;
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
__device__ __forceinline__ void repair(Ctx& C, RowScratch& R, P2 es, double xmin_v, double xmax_v, double dy,
                                       int& yi, int js, double& areai, double& areabound)
{
    rows_ensure(R, yi);
    if (R.ovf) return;
    wset(R.xmin, yi, xmin_v);
    wset(R.xmax, yi, xmax_v);
    wset(R.dys, yi, dy);
    __syncwarp();
    ++yi;
    const double area0 = image_area(C, R, es, dy, yi, js);
    areai += area0;
    areabound += area0;
    if (area0 <= 0.0) --yi;
}

} // namespace

__global__ void __launch_bounds__(128) cartesian_kernel(FsWork w, unsigned long long epoch)
{
    const int lane = lane_id();
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    char* base = w.scratch + (long long)gw * w.scratch_per_warp;
    const int cap = w.row_cap;
    RowScratch R;
    R.xmin = reinterpret_cast<double*>(base);
    R.xmax = R.xmin + cap;
    R.ax = R.xmax + cap;
    R.y = R.ax + cap;
    R.dys = R.y + cap;
    // Layout, every array 8-byte aligned: five row arrays and the per-seed areas
    // (doubles), the row-key table (u64), then the int arrays.
    double* areaimage = R.dys + cap;
    R.table = reinterpret_cast<ulonglong2*>((reinterpret_cast<uintptr_t>(areaimage + w.seed_cap) + 15) &
                                            ~static_cast<uintptr_t>(15));
    R.tmask = (unsigned)table_slots(cap) - 1u;
    R.next = reinterpret_cast<int*>(R.table + table_slots(cap));
    int* flags = R.next + cap + 2;  // per seed: bit0 overlapped (skip), bit1 subtracted
    R.cap = cap;
    unsigned long long local_gen = 0;
    const int n = w.retry_pass ? w.ir_count[2] : w.ir_count[0];
    for (;;) {
        int k = 0;
        if (lane == 0) k = atomicAdd(&w.next_item[w.retry_pass ? 3 : 1], 1);
        k = shfl_i(k, 0);
        if (k >= n) break;
        if (w.retry_pass) k = w.retry_cart[k];
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
        if (ns > 0 && rho > 0.0) {
            Ctx C;
            C.rays = 0;
            C.m = make_mapper(item.s, item.q);
            C.src = P2{item.x, item.y};
            C.rho = rho;
            C.rho2 = rho * rho;
            C.inv_rho2 = 1.0 / C.rho2;
            C.uniform = st.ld_c == 0.0 && st.ld_d == 0.0;
            // I(r^2) >= 1 - c - d on [0, 1] for c, d >= 0, so every counted cell adds > 0.
            C.bulk = C.uniform || (st.ld_c >= 0.0 && st.ld_d >= 0.0 && st.ld_c + st.ld_d < 1.0);
            C.ld = w.ld_tables + (long long)st.ld_table * (kLdTable + 1);
            C.max_steps = max(100000, st.source_bins * st.source_bins * 2000);
            const double nbin = static_cast<double>(max(st.source_bins, 1));
            const double incr = rho / nbin;
            const double margin = 0.5 * incr * 1.01;
            Diag d{ns, 0, 0, 0, 0, 0, 0.0};
            for (int i = lane; i < ns; i += 32) {
                areaimage[i] = 0.0;
                flags[i] = 0;
            }
            __syncwarp();
            double area = 0.0;
            for (int ii = 0; ii < ns && !ovf; ++ii) {
                if (flags[ii] & 1) continue;
                ++local_gen;
                R.gen = (epoch << 32) | (local_gen & 0xffffffffull);
                R.hw = 0;
                R.ovf = false;
                rows_ensure(R, 1);
                const P2 seed = seeds[ii];
                double areai = 0.0;
                double dy = incr;
                int yi = 0;
                const double jseed = jacobian(C.m, seed.x, seed.y);
                const int js = (fabs(jseed) < 0.02) ? sign_of(jseed) : 0;
                ++d.processed;
                if (js != 0) ++d.fold;
                wset(R.xmin, 0, seed.x);
                wset(R.xmax, 0, seed.x);
                __syncwarp();
                areai = image_area(C, R, seed, dy, yi, js);
                dy = -incr;
                rows_ensure(R, yi);
                if (R.ovf) {
                    ovf = true;
                    break;
                }
                const P2 lower{R.xmax[0], seed.y + dy};
                {
                    const double xm0 = R.xmin[0], xM0 = R.xmax[0], y0 = R.y[0];
                    wset(R.xmin, yi, xm0);
                    wset(R.xmax, yi, xM0);
                    wset(R.y, yi, y0);
                    wset(R.dys, yi, dy);
                    __syncwarp();
                }
                ++yi;
                areai += image_area(C, R, lower, dy, yi, js);
                int nyi = yi;
                double areabound = 0.0;
                for (int row = 0; row < nyi && !R.ovf; ++row) {
                    rows_ensure(R, row + 1);
                    const double dxmax = R.xmax[row + 1] - R.xmax[row];
                    const double dxmin = R.xmin[row + 1] - R.xmin[row];
                    if (R.ax[row + 1] > 0.0) d.max_jump = dmax_(d.max_jump, dmax_(fabs(dxmax), fabs(dxmin)) / incr);
                    if (R.ax[row + 1] > 0.0) {
                        if (dxmax > 1.1 * incr) {
                            ++d.gap_repairs;
                            repair(C, R, P2{R.xmax[row + 1], R.y[row]}, R.xmax[row], R.xmax[row + 1], -R.dys[row], yi,
                                   js, areai, areabound);
                        }
                        if (dxmin > 1.1 * incr) {
                            ++d.gap_repairs;
                            repair(C, R, P2{R.xmin[row + 1] - incr, R.y[row + 1]}, R.xmin[row], R.xmin[row + 1],
                                   R.dys[row], yi, js, areai, areabound);
                        }
                        if (dxmin < -1.1 * incr) {
                            ++d.gap_repairs;
                            repair(C, R, P2{R.xmin[row] - incr, R.y[row]}, R.xmin[row + 1], R.xmin[row], -R.dys[row],
                                   yi, js, areai, areabound);
                        }
                        if (dxmax < -1.1 * incr) {
                            ++d.gap_repairs;
                            repair(C, R, P2{R.xmax[row + 1] + incr, R.y[row + 1]}, R.xmax[row + 1], R.xmax[row],
                                   R.dys[row], yi, js, areai, areabound);
                        }
                    }
                    if (row == nyi - 1 && areabound > 0.0 && yi > nyi) nyi = yi;
                }
                if (R.ovf) {
                    ovf = true;
                    break;
                }
                area += areai;
                if (lane == 0) areaimage[ii] = areai;
                for (int row = 0; row < nyi; ++row)
                    if (R.ax[row] > 0.0) ++d.boundary_rows;
                // Overlap bookkeeping against every other seed (FSM:2681-2739).
                for (int oi = 0; oi < ns; ++oi) {
                    if (oi == ii) continue;
                    const P2 p = seeds[oi];
                    if (js != 0) {
                        if (sign_of(jacobian(C.m, p.x, p.y)) == -js) continue;
                        if (rho >= 4.0e-3 && st.source_bins >= 35 && oi > ii && fabs(jseed) < 1.0e-3 &&
                            fabs(jacobian(C.m, p.x, p.y)) < 0.02)
                            continue;
                    }
                    bool hit = false;
                    for (int r0 = 0; r0 < nyi; r0 += 32) {
                        const int row = r0 + lane;
                        bool h = false;
                        if (row < nyi && R.ax[row] > 0.0) {
                            h = p.y >= R.y[row] - margin && p.y <= R.y[row] + margin &&
                                p.x >= R.xmin[row] - margin && p.x <= R.xmax[row] + margin;
                        }
                        if (__any_sync(kFull, h)) {
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
                                __syncwarp();
                                if (lane == 0) flags[oi] = f | 2;
                            }
                        } else {
                            if (lane == 0) flags[oi] = flags[oi] | 1;
                        }
                        __syncwarp();
                    }
                }
                __syncwarp();
            }
            if (lane == 0) w.rays[it] = C.rays;
            if (!ovf) {
                const double flux = source_flux(rho, st.ld_c, st.ld_d);
                const double scale = flux / (rho * rho) * nbin * nbin;
                A = area / scale;
                double err = area_error(d, rho, st.source_bins, st.ld_c, st.ld_d);
                const double fc = floor_coefficient(d, A, rho);
                if (fc > 0.0) err = dmax_(err, fabs(A) * (fc / static_cast<double>(max(st.source_bins, 1))));
                o.err = isfinite(A) ? err : dnan();
                const double target = st.tol + st.reltol * dmax_(fabs(A), 1.0);
                o.converged = isfinite(A) && err <= 0.999 * target;
            }
        }
        if (ovf && !w.retry_pass) {
            // Too many rows for this pass's scratch: run again with the large one.
            if (lane == 0) w.retry_cart[atomicAdd(&w.ir_count[2], 1)] = k;
            __syncwarp();
            continue;
        }
        o.A = A;
        if (ovf) o.status = kFsRowOverflow;
        else if (!isfinite(A)) o.status = kFsNumerical;
        if (lane == 0) {
            w.out[it] = o;
            if (w.cycles) w.cycles[it] += clock64() - t_item;
        }
        __syncwarp();
    }
}

size_t cartesian_scratch_bytes(int row_cap, int seed_cap)
{
    return ((size_t)row_cap * 5 + seed_cap + 2) * sizeof(double) + (size_t)table_slots(row_cap) * sizeof(ulonglong2) +
           ((size_t)row_cap + 2 + seed_cap) * sizeof(int) + 256;
}

cudaError_t launch_cartesian(const FsWork& w, int n_warps, cudaStream_t stream, unsigned long long epoch)
{
    const int blocks = (n_warps + 3) / 4;
    cartesian_kernel<<<blocks, 128, 0, stream>>>(w, epoch);
    return cudaGetLastError();
}

} // namespace lcbi
