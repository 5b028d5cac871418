// Calls the C++ entry points of include/lcbinint_b200.hpp the way code written
// against the reference's core calls PointSourceMagnifier and
// FiniteSourceMagnifier, and prints every result with %a (exact doubles) for
// tests/test_cpp_api.py to compare with the reference.
//
// Input lines (stdin):
//   ps  s q x y                            binary_mag0 / _with_derivatives
//   cand s q x y                           binary_image_candidates / binary_images
//   le  s q x y                            binary_lens_equation
//   fs  mode nbin c s q x y rho aps exact  FiniteSourceMagnifier::binary_mag
//   batch s q n x0 y0 dx                   binary_mag0_batch along a line
#include "lcbinint_b200.hpp"

#include <cstdio>
#include <cstring>
#include <vector>

namespace lm = lcbinint_b200::magnification;
using lcbinint_b200::SourcePosition;

int main()
{
    lm::PointSourceMagnifier pm;
    char op[16];
    while (std::scanf("%15s", op) == 1) {
        if (!std::strcmp(op, "ps")) {
            double s, q, x, y;
            if (std::scanf("%lf %lf %lf %lf", &s, &q, &x, &y) != 4) return 2;
            const auto r = pm.binary_mag0(s, q, {x, y});
            const auto d = pm.binary_mag0_with_derivatives_cached(s, q, {x, y});
            std::printf("ps %a %d %a %d %a\n", r.magnification, r.image_count, d.magnification, d.image_count,
                        d.derivative_error_indicator);
        } else if (!std::strcmp(op, "cand")) {
            double s, q, x, y;
            if (std::scanf("%lf %lf %lf %lf", &s, &q, &x, &y) != 4) return 2;
            const auto c = pm.binary_image_candidates(s, q, {x, y});
            const auto im = pm.binary_images(s, q, {x, y});
            std::printf("cand %zu %zu", c.size(), im.size());
            for (const auto& k : c)
                std::printf(" %a %a %a %a %d", k.position.x, k.position.y, k.jacobian_determinant, k.residual,
                            k.physical ? 1 : 0);
            std::printf("\n");
        } else if (!std::strcmp(op, "le")) {
            double s, q, x, y;
            if (std::scanf("%lf %lf %lf %lf", &s, &q, &x, &y) != 4) return 2;
            const SourcePosition p = pm.binary_lens_equation(s, q, {x, y});
            std::printf("le %a %a\n", p.x, p.y);
        } else if (!std::strcmp(op, "fs")) {
            int mode, nbin, exact;
            double c, s, q, x, y, rho, aps;
            if (std::scanf("%d %d %lf %lf %lf %lf %lf %lf %lf %d", &mode, &nbin, &c, &s, &q, &x, &y, &rho, &aps,
                           &exact) != 10)
                return 2;
            lm::FiniteSourceSettings st;
            st.finite_mode = mode;
            st.source_bins = nbin;
            st.limb_darkening_c = c;
            const lm::FiniteSourceMagnifier fm(st);
            const auto r = fm.binary_mag(s, q, {x, y}, rho, aps, nullptr, exact != 0);
            std::printf("fs %a %a %d %d %d\n", r.magnification, r.error_estimate, static_cast<int>(r.decision.method),
                        r.refinement_level, r.converged ? 1 : 0);
        } else if (!std::strcmp(op, "batch")) {
            double s, q, x0, y0, dx;
            int n;
            if (std::scanf("%lf %lf %d %lf %lf %lf", &s, &q, &n, &x0, &y0, &dx) != 6) return 2;
            std::vector<SourcePosition> src(n);
            for (int i = 0; i < n; ++i) src[i] = {x0 + dx * i, y0};
            std::vector<double> A(n);
            pm.binary_mag0_batch(s, q, src.data(), A.data(), A.size());
            std::printf("batch %d", n);
            for (double a : A) std::printf(" %a", a);
            std::printf("\n");
        } else {
            return 3;
        }
    }
    return 0;
}
