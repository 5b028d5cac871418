// Adjoint of the finite-source magnification: dA/d(y1, y2, s, q, rho, c) per
// point, for the method the forward pass chose.  No reference counterpart (the
// reference has no gradient API; its users difference the forward).
//
// * Point source (method 0): A = sum over the physical images of 1/|J|.  The
//   images move with a parameter p by implicit differentiation of the lens
//   equation F(z, conj z; p) = y:  dz + kappa conj(dz) = w dp, w = y_p - F_p,
//   so dz = (w - kappa conj(w)) / J with kappa = dF/d(conj z) and
//   J = 1 - |kappa|^2; then dJ = -2 Re(conj(kappa) dkappa) and
//   d(1/|J|) = -sign(J) dJ / J^2.  The roots and the image selection are the
//   forward's, so A is the forward's value.
// * Hexadecapole (method 1): the derivative of its closed form
//   (finite_source_magnifier.cpp:792-847) through the 13 point-source
//   gradients it is built from (the ring samples move with y and rho).
// * Inverse ray (methods 2, 3): the derivative of the continuum magnification
//   the lattice sums approximate.  With U(R) the image-plane area of the
//   images of the disc of radius R about the source, linear limb darkening
//   I = 1 - c (1 - sqrt(1 - r^2)) gives
//       int_D I dx = (1 - c) U(rho) + c int_0^{pi/2} U(rho sin phi) sin phi dphi,
//   A = that / (pi rho^2 (1 - c/3)), so every derivative is a combination of
//   dU(R)/dp and dU/dR at a few radii (R = rho and 6 Gauss-Legendre nodes) --
//   contour integrals over the image boundaries |F(x) - y| = R, with no
//   interior singularity from the limb-darkening law.  A square image-plane
//   lattice (cell h = rho / grad_bins) is visited by the same tile-parallel
//   flood fill as the polar inverse ray, from the forward's seeds, over the
//   cells inside the outer contour; then every lattice square with a visited
//   corner is cut into two triangles, on
//   which the area below each level of the linear interpolant of |F(x) - y|
//   and its exact derivatives are formed (marching triangles).  The gradient
//   is thus the exact gradient of a piecewise-linear approximation of the
//   continuum magnification (slot 6 of the output), O(h^2) from it, with no
//   division by the lens map's point gradient, which vanishes where a contour
//   meets a critical curve.
//   Quadratic limb darkening, I = 1 - c (1 - mu) - d (1 - sqrt(mu)), adds
//   d int_0^1 U(rho sqrt(1 - u^4)) du, six more radii on a second contour
//   pass that points without a quadratic term skip.
#include "lcbi_fs_kernels.h"
#include "lcbi_ps.cuh"
#include "lcbi_warp.cuh"

#include <cstdint>

namespace lcbi {

namespace {

constexpr double kSqrtHalf = 0.70710678118654752440;
constexpr int kRadiiLin = 7;    // rho and 6 Gauss-Legendre nodes of phi in [0, pi/2]
constexpr int kRadiiQuad = 6;   // 6 Gauss-Legendre nodes of u in [0, 1]: the quadratic term
constexpr int kRadii = kRadiiLin + kRadiiQuad;
constexpr int kAcc = 6;         // U, dU/dy1, dU/dy2, dU/ds, dU/dq, dU/dR per radius
constexpr int kKeyBits = 25;
constexpr unsigned long long kKeyMask = (1ull << kKeyBits) - 1;
constexpr int kKeyOffset = 1 << 24;  // tile coordinates may be negative
constexpr int kMaxProbe = 4096;
constexpr unsigned kSpinLimit = 1u << 25;

// Gauss-Legendre nodes and weights on [-1, 1] (6 points).
__device__ __constant__ double kGLx[6] = {-0.9324695142031521, -0.6612093864662645, -0.2386191860831969,
                                          0.2386191860831969,  0.6612093864662645,  0.9324695142031521};
__device__ __constant__ double kGLw[6] = {0.1713244923791704, 0.3607615730481386, 0.4679139345726910,
                                          0.4679139345726910, 0.3607615730481386, 0.1713244923791704};

__device__ __forceinline__ dc cinv(dc a)
{
    const double d = a.re * a.re + a.im * a.im;
    return dc{a.re / d, -a.im / d};
}
__device__ __forceinline__ dc cconj(dc a) { return dc{a.re, -a.im}; }
__device__ __forceinline__ double cabs2(dc a) { return a.re * a.re + a.im * a.im; }

// Lens parameters in the lens frame (heavier mass m1 at a, lighter m2 at the
// origin) and their derivatives with respect to s and the core-convention q.
struct LensDeriv {
    double a, m1, m2, da_ds, dm1_dq, dm2_dq;
};

__device__ __forceinline__ LensDeriv lens_deriv(double separation, double mass_ratio)
{
    const double s = fabs(separation);
    const double q_in = fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    LensDeriv L;
    L.a = q_in < 1.0 ? -s : s;
    L.m1 = 1.0 / (1.0 + q);
    L.m2 = q * L.m1;
    const double sgn_s = separation < 0.0 ? -1.0 : 1.0;
    L.da_ds = (q_in < 1.0 ? -1.0 : 1.0) * sgn_s;
    const double dq = q_in < 1.0 ? 1.0 : -1.0 / (q_in * q_in);
    const double opq2 = (1.0 + q) * (1.0 + q);
    L.dm1_dq = -dq / opq2;
    L.dm2_dq = dq / opq2;
    return L;
}

struct PsGrad {
    double A, dy1, dy2, ds, dq;
};

// binary_mag0 and its gradient in (y1, y2, s, q_core).
__device__ PsGrad ps_grad(double separation, double mass_ratio, double y1, double y2)
{
    PsGrad r{0.0, 0.0, 0.0, 0.0, 0.0};
    if (separation == 0.0 || mass_ratio <= 0.0) return r;
    const BinaryGeom g = make_geom(separation, mass_ratio, y1, y2);
    dc roots[5];
    if (!solve_images(g, roots)) {
        r.A = r.dy1 = r.dy2 = r.ds = r.dq = dnan();
        return r;
    }
    const unsigned mask = physical_mask(g, roots);
    int cnt = 0;
    r.A = sum_inverse_jacobians(g, roots, mask, &cnt);
    const LensDeriv L = lens_deriv(separation, mass_ratio);
    for (int i = 0; i < 5; ++i) {
        if (!(mask & (1u << i))) continue;
        const dc zb = cconj(roots[i]);
        const dc i1 = cinv(dc{zb.re - L.a, zb.im});
        const dc i2 = cinv(zb);
        const dc i1s = cmul(i1, i1), i2s = cmul(i2, i2);
        const dc kap = cadd(cscale(L.m1, i1s), cscale(L.m2, i2s));
        const double J = 1.0 - cabs2(kap);
        const dc kap_zb = cscale(-2.0, cadd(cscale(L.m1, cmul(i1s, i1)), cscale(L.m2, cmul(i2s, i2))));
        const double sJ = J < 0.0 ? -1.0 : 1.0;
        const double inv_J2 = 1.0 / (J * J);
        // d(1/|J|) for a parameter with w = y_p - F_p and kappa_p.
        auto dterm = [&](dc w, dc kp) {
            const dc dz = cscale(1.0 / J, csub(w, cmul(kap, cconj(w))));
            const dc dk = cadd(cmul(kap_zb, cconj(dz)), kp);
            const double dJ = -2.0 * (kap.re * dk.re + kap.im * dk.im);
            return -sJ * dJ * inv_J2;
        };
        r.dy1 += dterm(dc{1.0, 0.0}, dc{0.0, 0.0});
        r.dy2 += dterm(dc{0.0, 1.0}, dc{0.0, 0.0});
        // F = z - m1/(conj z - a) - m2/conj z - a m1 (centre-of-mass frame).
        const dc F_a = dc{-L.m1 * i1s.re - L.m1, -L.m1 * i1s.im};
        const dc k_a = cscale(2.0 * L.m1, cmul(i1s, i1));
        r.ds += dterm(cscale(-L.da_ds, F_a), cscale(L.da_ds, k_a));
        const dc F_m1 = dc{-i1.re - L.a, -i1.im};
        const dc F_m2 = dc{-i2.re, -i2.im};
        const dc F_q = cadd(cscale(L.dm1_dq, F_m1), cscale(L.dm2_dq, F_m2));
        const dc k_q = cadd(cscale(L.dm1_dq, i1s), cscale(L.dm2_dq, i2s));
        r.dq += dterm(cscale(-1.0, F_q), k_q);
    }
    return r;
}

__device__ __forceinline__ void ring_dir(int k, double* cx, double* cy, double* f)
{
    // hexadecapole_binary sample order (FSM:807-820): for i in 0..3: +rho, +rho/2, diagonal.
    const double sineta[8] = {0.0, 1.0, 0.0, -1.0, kSqrtHalf, kSqrtHalf, -kSqrtHalf, -kSqrtHalf};
    const double coseta[8] = {1.0, 0.0, -1.0, 0.0, kSqrtHalf, -kSqrtHalf, -kSqrtHalf, kSqrtHalf};
    const int i = k / 3;
    const int j = k - 3 * i;
    const int e = j == 2 ? i + 4 : i;
    *cx = coseta[e];
    *cy = sineta[e];
    *f = j == 1 ? 0.5 : 1.0;
}

// Warp per point: gradients of the point-source and hexadecapole results.
__global__ void __launch_bounds__(128) grad_direct_kernel(FsWork w, double* grads)
{
    const int lane = lane_id();
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < w.n_items; it += nw) {
        const FsOut o = w.out[it];
        double* gout = grads + (long long)it * 8;
        if (o.method >= 2) continue;  // inverse ray: the tile pass
        const FsItem item = w.items[it];
        const FsSettingsDev st = w.settings[item.settings];
        double res[8] = {dnan(), dnan(), dnan(), dnan(), dnan(), dnan(), o.A, static_cast<double>(o.method)};
        if (o.status == kFsOk && o.method == 0) {
            if (lane == 0) {
                const PsGrad p = ps_grad(item.s, item.q, item.x, item.y);
                res[0] = p.dy1;
                res[1] = p.dy2;
                res[2] = p.ds;
                res[3] = p.dq;
                res[4] = 0.0;
                res[5] = 0.0;
            }
        } else if (o.status == kFsOk && o.method == 1) {
            const double rho = item.rho;
            PsGrad p{0.0, 0.0, 0.0, 0.0, 0.0};
            double drho = 0.0;
            if (lane < 12) {
                double cx, cy, f;
                ring_dir(lane, &cx, &cy, &f);
                double px, py;
                if (f == 0.5) {
                    px = item.x + 0.5 * rho * cx;
                    py = item.y + 0.5 * rho * cy;
                } else {
                    px = item.x + rho * cx;
                    py = item.y + rho * cy;
                }
                p = ps_grad(item.s, item.q, px, py);
                drho = f * (cx * p.dy1 + cy * p.dy2);
            } else if (lane == 12) {
                p = ps_grad(item.s, item.q, item.x, item.y);
                // The decision's centre value: the caller's exact one, else binary_mag0 itself.
                if ((item.flags & kItemPsExact) && !(item.flags & kItemPsOnDevice)) p.A = item.a_ps;
            }
            double v[6] = {p.A, p.dy1, p.dy2, p.ds, p.dq, drho};
            double a0[6], a1p[6], a2p[6], a1c[6];
            for (int c = 0; c < 6; ++c) {
                a0[c] = shfl_d(v[c], 12);
                a1p[c] = a2p[c] = a1c[c] = 0.0;
                for (int i = 0; i < 4; ++i) {
                    a1p[c] += shfl_d(v[c], 3 * i);
                    a2p[c] += shfl_d(v[c], 3 * i + 1);
                    a1c[c] += shfl_d(v[c], 3 * i + 2);
                }
                a1p[c] = a1p[c] / 4.0 - a0[c];
                a2p[c] = a2p[c] / 4.0 - a0[c];
                a1c[c] = a1c[c] / 4.0 - a0[c];
            }
            const double den = 15.0 - 5.0 * st.ld_c - 3.0 * st.ld_d;
            const double gm = ld_gamma(st.ld_c, st.ld_d), lm = ld_lambda(st.ld_c, st.ld_d);
            const double dg = den == 0.0 ? 0.0 : (10.0 * den + 50.0 * st.ld_c) / (den * den);
            const double dl = den == 0.0 ? 0.0 : 60.0 * st.ld_d / (den * den);
            const double F2 = 1.0 - 0.2 * gm - lm / 9.0;
            const double F4 = 1.0 - 11.0 * gm / 35.0 - 7.0 * lm / 39.0;
            // Component 0 is the value itself; 1..5 are y1, y2, s, q, rho.
            double out6[6];
            for (int c = 0; c < 6; ++c) {
                const double a2rho2 = (16.0 * a2p[c] - a1p[c]) / 3.0;
                const double a4rho4 = (a1p[c] + a1c[c]) / 2.0 - a2rho2;
                out6[c] = a0[c] + 0.5 * a2rho2 * F2 + a4rho4 / 3.0 * F4;
                if (c == 0) {
                    res[5] = 0.5 * a2rho2 * (-0.2 * dg - dl / 9.0) + a4rho4 / 3.0 * (-11.0 * dg / 35.0 - 7.0 * dl / 39.0);
                }
            }
            res[0] = out6[1];
            res[1] = out6[2];
            res[2] = out6[3];
            res[3] = out6[4];
            res[4] = out6[5];
        }
        if (lane == 0) {
            for (int c = 0; c < 8; ++c) gout[c] = res[c];
        }
    }
}

// ---------------------------------------------------------------- inverse ray

struct GradSlot {
    unsigned long long key;   // 0 empty; else 1 + (point << 50 | (ty + off) << 25 | (tx + off))
    int queued;
    int mready;
    unsigned m[32];           // band mask of each row (bit c: x cell 32 tx + c)
    unsigned v[32];
    unsigned p[32];
};

enum : int { kGActive = 0, kGDone = 1, kGOverflow = 2 };

struct GradItem {
    LensDeriv L;
    P2 src;
    double rho, c, d, h, tau;
    double R[kRadii];
    double acc[kRadii][kAcc];
    int state;
    int slot_item;  // item index in the chunk
};

struct GradCtl {
    unsigned long long head, tail;
    long long in_flight;
    int error;
    int pad;
};

struct GradCtx {
    GradItem* items;
    GradSlot* slots;
    unsigned* ring;
    GradCtl* ctl;
    unsigned long long mask;
    unsigned spin_limit;      // polls before a wait gives up
    int* timeouts;            // waits that gave up (null: not counted)
};

__device__ __forceinline__ unsigned long long gkey(int item, int ty, int tx)
{
    return 1ull + (((unsigned long long)item << (2 * kKeyBits)) |
                   ((unsigned long long)(unsigned)(ty + kKeyOffset) << kKeyBits) |
                   (unsigned long long)(unsigned)(tx + kKeyOffset));
}

__device__ long long gfind_or_insert(const GradCtx& G, unsigned long long key)
{
    unsigned long long h = (key * 0x9e3779b97f4a7c15ull) >> 20;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        h &= G.mask;
        GradSlot* s = G.slots + h;
        const unsigned long long k = __ldcg(&s->key);
        if (k == key) return (long long)h;
        if (k == 0) {
            const unsigned long long prev = atomicCAS(&s->key, 0ull, key);
            if (prev == 0 || prev == key) return (long long)h;
        }
        ++h;
    }
    return -1;
}

__device__ __forceinline__ void gpush(const GradCtx& G, unsigned slot)
{
    atomicAdd(reinterpret_cast<unsigned long long*>(&G.ctl->in_flight), 1ull);
    const unsigned long long pos = atomicAdd(&G.ctl->tail, 1ull);
    __threadfence();
    atomicExch(G.ring + (pos & G.mask), slot + 1u);
}

__device__ __forceinline__ bool tile_in_range(int ty, int tx)
{
    return ty > -kKeyOffset && ty < kKeyOffset && tx > -kKeyOffset && tx < kKeyOffset;
}

// One thread: OR entry bits into row `row` of tile (ty, tx) and queue it.
__device__ void gsend_row(const GradCtx& G, int item, int ty, int tx, int row, unsigned bits)
{
    if (!tile_in_range(ty, tx)) {
        atomicExch(&G.items[item].state, kGOverflow);
        return;
    }
    const long long s = gfind_or_insert(G, gkey(item, ty, tx));
    if (s < 0) {
        atomicExch(&G.items[item].state, kGOverflow);
        return;
    }
    GradSlot* T = G.slots + s;
    atomicOr(&T->p[row], bits);
    __threadfence();
    if (atomicExch(&T->queued, 1) == 0) gpush(G, (unsigned)s);
}

// Whole warp: lane j ORs `bits` into row j of tile (ty, tx).
__device__ void gsend_rows(const GradCtx& G, int item, int ty, int tx, unsigned bits)
{
    long long s = -1;
    if (lane_id() == 0) {
        if (tile_in_range(ty, tx)) s = gfind_or_insert(G, gkey(item, ty, tx));
        if (s < 0) atomicExch(&G.items[item].state, kGOverflow);
    }
    s = __shfl_sync(kFull, s, 0);
    if (s < 0) return;
    GradSlot* T = G.slots + s;
    if (bits) atomicOr(&T->p[lane_id()], bits);
    __threadfence();
    __syncwarp();
    if (lane_id() == 0 && atomicExch(&T->queued, 1) == 0) gpush(G, (unsigned)s);
}

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

// Lens map of the centre of cell (ix, iy): w = F - y, the stretch
// g = |grad |F - y|| and, when `full`, dG/dp (G = |F - y|^2) for y1, y2, s, q.
struct CellEval {
    double r, g;      // |w| and |grad |w||
    double dG[4];
};

__device__ __forceinline__ CellEval cell_eval(const GradItem& I, int ix, int iy, bool full)
{
    const double x = (static_cast<double>(ix) + 0.5) * I.h;
    const double y = (static_cast<double>(iy) + 0.5) * I.h;
    const dc zb{x, -y};
    const dc i1 = cinv(dc{zb.re - I.L.a, zb.im});
    const dc i2 = cinv(zb);
    const dc F{x - I.L.m1 * i1.re - I.L.m2 * i2.re - I.L.a * I.L.m1, y - I.L.m1 * i1.im - I.L.m2 * i2.im};
    const dc w{F.re - I.src.x, F.im - I.src.y};
    const dc i1s = cmul(i1, i1), i2s = cmul(i2, i2);
    const dc kap = cadd(cscale(I.L.m1, i1s), cscale(I.L.m2, i2s));
    CellEval e;
    e.r = sqrt(cabs2(w));
    const dc gv = cadd(w, cmul(cconj(w), kap));
    e.g = e.r > 0.0 ? sqrt(cabs2(gv)) / e.r : 1.0;
    if (full) {
        e.dG[0] = -2.0 * w.re;
        e.dG[1] = -2.0 * w.im;
        const dc F_a = dc{-I.L.m1 * i1s.re - I.L.m1, -I.L.m1 * i1s.im};
        e.dG[2] = 2.0 * I.L.da_ds * (w.re * F_a.re + w.im * F_a.im);
        const dc F_q{I.L.dm1_dq * (-i1.re - I.L.a) + I.L.dm2_dq * (-i2.re),
                     I.L.dm1_dq * (-i1.im) + I.L.dm2_dq * (-i2.im)};
        e.dG[3] = 2.0 * (w.re * F_q.re + w.im * F_q.im);
    }
    return e;
}

// Corner data of the contour pass: |w| and d|w|/dp = (dG/dp) / (2 |w|) for
// p = y1, y2, s, q.
struct Corner {
    double r, d[4];
};

__device__ __forceinline__ Corner corner_of(const CellEval& e)
{
    Corner c;
    c.r = e.r;
    const double inv = 1.0 / (2.0 * e.r);
    for (int a = 0; a < 4; ++a) c.d[a] = e.dG[a] * inv;
    return c;
}

// One lattice triangle against the level R, for the linear interpolant v of
// |w| - R over it: the area where v < 0, its derivatives in y1, y2, s, q
// (the level segment moves with normal speed -dv/|grad v|, which is exact for
// linear v and linear dv) and its derivative in R.  `upper` selects the
// triangle (0,0), (1,1), (0,1) of the unit square, else (0,0), (1,0), (1,1).
// acc: area, 4 parameter derivatives, dU/dR.
__device__ __forceinline__ void triangle(const Corner& A, const Corner& B, const Corner& C, bool upper, double R,
                                         double h, double* acc)
{
    const double va = A.r - R, vb = B.r - R, vc = C.r - R;
    const bool ia = va < 0.0, ib = vb < 0.0, ic = vc < 0.0;
    const int n_in = (int)ia + (int)ib + (int)ic;
    const double full = 0.5 * h * h;
    if (n_in == 3) {
        acc[0] += full;
        return;
    }
    if (n_in == 0) return;
    // Gradient of v in cells: lower (0,0),(1,0),(1,1); upper (0,0),(1,1),(0,1).
    const double gx = upper ? vb - vc : vb - va;
    const double gy = upper ? vc - va : vc - vb;
    const double gnorm = sqrt(gx * gx + gy * gy) / h;
    const P2 pa{0.0, 0.0};
    const P2 pb = upper ? P2{1.0, 1.0} : P2{1.0, 0.0};
    const P2 pc = upper ? P2{0.0, 1.0} : P2{1.0, 1.0};
    // Rotate so that the odd vertex (the one on its own side) comes first.
    const Corner *P = &A, *Q = &B, *S = &C;
    P2 pp = pa, pq = pb, ps = pc;
    double vp = va, vq = vb, vs = vc;
    const bool odd_in = n_in == 1;
    if ((ib == odd_in) && (ia != odd_in)) {
        P = &B; Q = &C; S = &A; pp = pb; pq = pc; ps = pa; vp = vb; vq = vc; vs = va;
    } else if ((ic == odd_in) && (ia != odd_in)) {
        P = &C; Q = &A; S = &B; pp = pc; pq = pa; ps = pb; vp = vc; vq = va; vs = vb;
    }
    const double tq = vp / (vp - vq);  // crossing on P-Q
    const double ts = vp / (vp - vs);  // crossing on P-S
    const double small = full * tq * ts;
    acc[0] += odd_in ? small : full - small;
    const P2 e1{pp.x + tq * (pq.x - pp.x), pp.y + tq * (pq.y - pp.y)};
    const P2 e2{pp.x + ts * (ps.x - pp.x), pp.y + ts * (ps.y - pp.y)};
    const double len = h * sqrt((e1.x - e2.x) * (e1.x - e2.x) + (e1.y - e2.y) * (e1.y - e2.y));
    const double w = len / gnorm;
    for (int a = 0; a < 4; ++a) {
        const double d1 = P->d[a] + tq * (Q->d[a] - P->d[a]);
        const double d2 = P->d[a] + ts * (S->d[a] - P->d[a]);
        acc[1 + a] -= 0.5 * (d1 + d2) * w;
    }
    acc[5] += w;
}

// One visit of one tile by one warp during the flood: band mask on the first
// visit, in-tile closure of the entry cells, new visited cells, exits.
__device__ void grad_tile(const GradCtx& G, unsigned slot)
{
    const int j = lane_id();
    GradSlot* T = G.slots + slot;
    const unsigned long long key = __ldcg(&T->key) - 1ull;
    const int item = static_cast<int>(key >> (2 * kKeyBits));
    const int ty = static_cast<int>((key >> kKeyBits) & kKeyMask) - kKeyOffset;
    const int tx = static_cast<int>(key & kKeyMask) - kKeyOffset;
    const GradItem& Ig = G.items[item];
    if (j == 0) atomicExch(&T->queued, 0);
    __syncwarp();
    __threadfence();
    const unsigned pend = atomicExch(&T->p[j], 0u);
    if (__ldcg(&G.items[item].state) != kGActive) return;
    GradItem I;
    I.L = Ig.L;
    I.src = Ig.src;
    I.rho = Ig.rho;
    I.c = Ig.c;
    I.h = Ig.h;
    I.tau = Ig.tau;
    const int iy = ty * 32 + j;
    int ready = 0;
    if (j == 0) ready = __ldcg(&T->mready);
    ready = __shfl_sync(kFull, ready, 0);
    unsigned M = 0;
    if (ready == 0) {
        for (int c = 0; c < 32; ++c) {
            const CellEval e = cell_eval(I, tx * 32 + c, iy, false);
            if (e.r <= I.rho) M |= 1u << c;
        }
        T->m[j] = M;
        __threadfence();
        __syncwarp();
        if (j == 0) atomicExch(&T->mready, 1);
    } else {
        M = __ldcg(&T->m[j]);
    }
    const unsigned S = pend & M;
    if (!__any_sync(kFull, S != 0u)) return;
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
    if (!__any_sync(kFull, nw != 0u)) return;
    // Exits to the four neighbouring tiles.
    if (__any_sync(kFull, (nw >> 31) != 0u)) gsend_rows(G, item, ty, tx + 1, (nw >> 31) ? 1u : 0u);
    if (__any_sync(kFull, (nw & 1u) != 0u)) gsend_rows(G, item, ty, tx - 1, (nw & 1u) ? 0x80000000u : 0u);
    if (j == 31 && nw) gsend_row(G, item, ty + 1, tx, 0, nw);
    if (j == 0 && nw) gsend_row(G, item, ty - 1, tx, 31, nw);
}

// Slot of `key`, or -1 when absent.
__device__ long long gfind(const GradCtx& G, unsigned long long key)
{
    unsigned long long h = (key * 0x9e3779b97f4a7c15ull) >> 20;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        h &= G.mask;
        const unsigned long long k = G.slots[h].key;
        if (k == key) return (long long)h;
        if (k == 0) return -1;
        ++h;
    }
    return -1;
}

// A lattice square belongs to the tile of its lower-left cell; squares that
// touch visited cells only through their right or upper corners may lie in
// tiles the flood never entered, so those tiles (left, below, below-left of
// each visited tile) are added to the table, unvisited, before the contour pass.
__global__ void __launch_bounds__(128) grad_phantom_kernel(GradCtx G)
{
    const int j = lane_id();
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long sl = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl <= (long long)G.mask;
         sl += nwarps) {
        const unsigned long long key = G.slots[sl].key;
        if (key == 0) continue;
        const unsigned V = G.slots[sl].v[j];
        if (!__any_sync(kFull, V != 0u)) continue;
        if (j < 3) {
            const unsigned long long k1 = key - 1ull;
            const int item = static_cast<int>(k1 >> (2 * kKeyBits));
            const int ty = static_cast<int>((k1 >> kKeyBits) & kKeyMask) - kKeyOffset;
            const int tx = static_cast<int>(k1 & kKeyMask) - kKeyOffset;
            const int dx = j == 1 ? 0 : -1;
            const int dy = j == 0 ? 0 : -1;
            if (!tile_in_range(ty + dy, tx + dx) || gfind_or_insert(G, gkey(item, ty + dy, tx + dx)) < 0)
                atomicExch(&G.items[item].state, kGOverflow);
        }
    }
}

// After the flood: every lattice square with a visited corner is split into
// two triangles and integrated against each radius (areas and their
// derivatives exact for the linear interpolant).  Warp per tile (the tile of
// the squares' lower-left cells); lane j owns row j and takes row j + 1 from
// lane j + 1 (lane 31 evaluates row 32).
template <int K0, int NK>
__global__ void __launch_bounds__(128) grad_contour_kernel(GradCtx G)
{
    const int j = lane_id();
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long sl = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl <= (long long)G.mask;
         sl += nwarps) {
        const GradSlot* T = G.slots + sl;
        const unsigned long long key = T->key;
        if (key == 0) continue;
        const unsigned long long k1 = key - 1ull;
        const int item = static_cast<int>(k1 >> (2 * kKeyBits));
        const int ty = static_cast<int>((k1 >> kKeyBits) & kKeyMask) - kKeyOffset;
        const int tx = static_cast<int>(k1 & kKeyMask) - kKeyOffset;
        if (G.items[item].state != kGActive) continue;
        if (K0 >= kRadiiLin && G.items[item].d == 0.0) continue;  // no quadratic term
        // Visited bits of the tile's cells and of the cells just right of and
        // above it (neighbouring tiles), as 33-bit rows.
        long long sr = -1, su = -1, sru = -1;
        if (j == 0) {
            sr = gfind(G, gkey(item, ty, tx + 1));
            su = gfind(G, gkey(item, ty + 1, tx));
            sru = gfind(G, gkey(item, ty + 1, tx + 1));
        }
        sr = __shfl_sync(kFull, sr, 0);
        su = __shfl_sync(kFull, su, 0);
        sru = __shfl_sync(kFull, sru, 0);
        unsigned long long row = T->v[j];
        if (sr >= 0) row |= (unsigned long long)(G.slots[sr].v[j] & 1u) << 32;
        unsigned long long above = __shfl_down_sync(kFull, row, 1);
        if (j == 31) {
            above = su >= 0 ? (unsigned long long)G.slots[su].v[0] : 0ull;
            if (sru >= 0) above |= (unsigned long long)(G.slots[sru].v[0] & 1u) << 32;
        }
        const unsigned V = static_cast<unsigned>((row | (row >> 1) | above | (above >> 1)) & 0xffffffffull);
        if (!__any_sync(kFull, V != 0u)) continue;
        const GradItem& Ig = G.items[item];
        GradItem I;
        I.L = Ig.L;
        I.src = Ig.src;
        I.rho = Ig.rho;
        I.c = Ig.c;
        I.h = Ig.h;
        I.tau = Ig.tau;
        double R[NK];
        for (int k = 0; k < NK; ++k) R[k] = Ig.R[K0 + k];
        double acc[NK][kAcc];
#pragma unroll
        for (int k = 0; k < NK; ++k)
#pragma unroll
            for (int a = 0; a < kAcc; ++a) acc[k][a] = 0.0;
        const int iy = ty * 32 + j;
        const int ix0 = tx * 32;
        // Column 0 of rows j and j + 1.
        Corner c00 = corner_of(cell_eval(I, ix0, iy, true));
        Corner c01;
        {
            Corner own32;
            if (j == 31) own32 = corner_of(cell_eval(I, ix0, iy + 1, true));
            c01.r = __shfl_down_sync(kFull, c00.r, 1);
            for (int a = 0; a < 4; ++a) c01.d[a] = __shfl_down_sync(kFull, c00.d[a], 1);
            if (j == 31) c01 = own32;
        }
        for (int c = 0; c < 32; ++c) {
            Corner c10 = corner_of(cell_eval(I, ix0 + c + 1, iy, true));
            Corner c11;
            Corner own32;
            if (j == 31) own32 = corner_of(cell_eval(I, ix0 + c + 1, iy + 1, true));
            c11.r = __shfl_down_sync(kFull, c10.r, 1);
            for (int a = 0; a < 4; ++a) c11.d[a] = __shfl_down_sync(kFull, c10.d[a], 1);
            if (j == 31) c11 = own32;
            if (V & (1u << c)) {
#pragma unroll
                for (int k = 0; k < NK; ++k) {
                    double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                    triangle(c00, c10, c11, false, R[k], I.h, t);
                    triangle(c00, c11, c01, true, R[k], I.h, t);
#pragma unroll
                    for (int a = 0; a < kAcc; ++a) acc[k][a] += t[a];
                }
            }
            c00 = c10;
            c01 = c11;
        }
#pragma unroll
        for (int k = 0; k < NK; ++k) {
#pragma unroll
            for (int a = 0; a < kAcc; ++a) {
                double v = acc[k][a];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
                if (j == ((k * kAcc + a) & 31) && v != 0.0) atomicAdd(&G.items[item].acc[K0 + k][a], v);
            }
        }
    }
}

__global__ void __launch_bounds__(128) grad_flood_kernel(GradCtx G)
{
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
                if (__ldcg(reinterpret_cast<const long long*>(&G.ctl->in_flight)) == 0 || __ldcg(&G.ctl->error)) {
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
        grad_tile(G, v - 1u);
        __syncwarp();
        __threadfence();
        if (lane_id() == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&G.ctl->in_flight), ~0ull);
    }
}

// Warp per inverse-ray slot: lattice, radii and the start cells (the cells of
// the forward's seeds).
__global__ void __launch_bounds__(128) grad_start_kernel(FsWork w, GradCtx G, int grad_bins)
{
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int n_cart = w.ir_count[0];
    const int n = n_cart + w.ir_count[1];
    if (k >= n) return;
    const int it = k < n_cart ? w.ir_cart[k] : w.ir_polar[k - n_cart];
    const FsItem item = w.items[it];
    const FsOut o = w.out[it];
    GradItem I{};
    I.state = kGDone;
    I.slot_item = it;
    if (o.status == kFsOk && o.n_seeds > 0 && (o.method == 2 || o.method == 3)) {
        const FsSettingsDev st = w.settings[item.settings];
        I.L = lens_deriv(item.s, item.q);
        I.src = P2{item.x, item.y};
        I.rho = item.rho;
        I.c = st.ld_c;
        I.d = st.ld_d;
        I.h = item.rho / static_cast<double>(grad_bins);
        I.tau = 2.0 * I.h;
        I.R[0] = item.rho;
        for (int q = 0; q < 6; ++q) I.R[1 + q] = item.rho * sin(0.25 * kPi * (kGLx[q] + 1.0));
        for (int q = 0; q < 6; ++q) {
            const double u = 0.5 * (kGLx[q] + 1.0);
            I.R[kRadiiLin + q] = item.rho * sqrt(1.0 - u * u * u * u);
        }
        I.state = item.rho > 0.0 ? kGActive : kGDone;
    }
    if (lane_id() == 0) G.items[k] = I;
    __syncwarp();
    __threadfence();
    if (I.state != kGActive || lane_id() != 0) return;
    const P2* seeds = w.seeds + (long long)k * w.seed_cap;
    for (int i = 0; i < o.n_seeds; ++i) {
        const double fx = floor(seeds[i].x / I.h), fy = floor(seeds[i].y / I.h);
        if (!(fabs(fx) < 1.0e9 && fabs(fy) < 1.0e9)) continue;
        const int ix = static_cast<int>(fx), iy = static_cast<int>(fy);
        const CellEval e = cell_eval(I, ix, iy, false);
        if (!(e.r <= I.rho)) continue;
        const int tx = ix >= 0 ? ix / 32 : -((-ix + 31) / 32);
        const int ty = iy >= 0 ? iy / 32 : -((-iy + 31) / 32);
        gsend_row(G, k, ty, tx, iy - 32 * ty, 1u << (ix - 32 * tx));
    }
}

// Thread per inverse-ray slot: the magnification's derivatives from the
// contour integrals.
__global__ void grad_finish_kernel(FsWork w, GradCtx G, double* grads)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = w.ir_count[0] + w.ir_count[1];
    if (k >= n) return;
    const GradItem I = G.items[k];
    double* gout = grads + (long long)I.slot_item * 8;
    const FsOut o = w.out[I.slot_item];
    double res[8] = {dnan(), dnan(), dnan(), dnan(), dnan(), dnan(), o.A, static_cast<double>(o.method)};
    if (I.state == kGActive && G.ctl->error == 0) {
        // Layer-cake form of the brightness integral: with I(t) the law at
        // t = r / rho, int_D I = I(1) U(rho) + int_0^1 (-I'(t)) U(rho t) dt.
        // The linear term, c t / sqrt(1 - t^2), takes t = sin(phi); the
        // quadratic one, (d t / 2)(1 - t^2)^(-3/4), takes u = (1 - t^2)^(1/4),
        // which makes it d int_0^1 U(rho sqrt(1 - u^4)) du.
        const double c = I.c, d = I.d;
        const double edge = 1.0 - c - d;
        double N = edge * I.acc[0][0];
        double dN[4], dNR = edge * I.acc[0][5], dNc = -I.acc[0][0];
        for (int a = 0; a < 4; ++a) dN[a] = edge * I.acc[0][1 + a];
        for (int q = 0; q < 6; ++q) {
            const double phi = 0.25 * kPi * (kGLx[q] + 1.0);
            const double wq = 0.25 * kPi * kGLw[q];
            const double sp = sin(phi);
            N += c * wq * I.acc[1 + q][0] * sp;
            dNc += wq * I.acc[1 + q][0] * sp;
            for (int a = 0; a < 4; ++a) dN[a] += c * wq * I.acc[1 + q][1 + a] * sp;
            dNR += c * wq * I.acc[1 + q][5] * sp * sp;
        }
        if (d != 0.0) {
            for (int q = 0; q < 6; ++q) {
                const double u = 0.5 * (kGLx[q] + 1.0);
                const double vq = 0.5 * kGLw[q];
                const double f = sqrt(1.0 - u * u * u * u);  // dR / drho
                const double* acc = I.acc[kRadiiLin + q];
                N += d * vq * acc[0];
                for (int a = 0; a < 4; ++a) dN[a] += d * vq * acc[1 + a];
                dNR += d * vq * acc[5] * f;
            }
        }
        const double Phi = kPi * I.rho * I.rho * (1.0 - c / 3.0 - d / 5.0);
        const double A = N / Phi;
        for (int a = 0; a < 4; ++a) res[a] = dN[a] / Phi;
        res[4] = dNR / Phi - 2.0 * A / I.rho;
        res[5] = dNc / Phi + A * (kPi * I.rho * I.rho / 3.0) / Phi;
        res[6] = A;
    }
    if (o.status != kFsOk || o.method < 2) return;
    for (int c = 0; c < 8; ++c) gout[c] = res[c];
}

} // namespace

size_t grad_tile_bytes(long long capacity, int max_items)
{
    return (size_t)capacity * sizeof(GradSlot) + (size_t)capacity * sizeof(unsigned) +
           (size_t)max_items * sizeof(GradItem) + sizeof(GradCtl) + 1024;
}

int grad_flood_blocks_per_sm()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, grad_flood_kernel, 128, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 2;
    }
    return nb;
}

// Gradients of every point of the chunk into grads (8 doubles per point:
// dA/d(y1, y2, s, q, rho, c), the value differentiated, the method).
cudaError_t launch_grad(const FsWork& w, void* area, long long capacity, int max_items, int flood_blocks,
                        int grad_bins, int sm_count, double* grads, cudaStream_t stream)
{
    const int blocks = sm_count * 4;
    grad_direct_kernel<<<blocks, 128, 0, stream>>>(w, grads);
    char* a = static_cast<char*>(area);
    GradCtx G;
    G.slots = reinterpret_cast<GradSlot*>(a);
    a += (size_t)capacity * sizeof(GradSlot);
    G.ring = reinterpret_cast<unsigned*>(a);
    a += (size_t)capacity * sizeof(unsigned);
    a = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(a) + 255) & ~uintptr_t(255));
    G.items = reinterpret_cast<GradItem*>(a);
    a += (size_t)max_items * sizeof(GradItem);
    a = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(a) + 255) & ~uintptr_t(255));
    G.ctl = reinterpret_cast<GradCtl*>(a);
    G.mask = (unsigned long long)capacity - 1ull;
    G.spin_limit = w.wait_limit ? w.wait_limit : kSpinLimit;
    G.timeouts = w.wait_timeouts;
    cudaError_t e = cudaMemsetAsync(area, 0, (size_t)capacity * (sizeof(GradSlot) + sizeof(unsigned)), stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(G.ctl, 0, sizeof(GradCtl), stream);
    if (e != cudaSuccess) return e;
    grad_start_kernel<<<(max_items * 32 + 127) / 128, 128, 0, stream>>>(w, G, grad_bins);
    grad_flood_kernel<<<flood_blocks, 128, 0, stream>>>(G);
    grad_phantom_kernel<<<sm_count * 8, 128, 0, stream>>>(G);
    grad_contour_kernel<0, kRadiiLin><<<sm_count * 8, 128, 0, stream>>>(G);
    grad_contour_kernel<kRadiiLin, kRadiiQuad><<<sm_count * 8, 128, 0, stream>>>(G);
    grad_finish_kernel<<<(max_items + 127) / 128, 128, 0, stream>>>(w, G, grads);
    return cudaGetLastError();
}

} // namespace lcbi
