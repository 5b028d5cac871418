// C entry points of the CPU oracle library (oracle/_build/liblcbi_oracle.so).
// Test infrastructure only: loaded by tests/, __graft_entry__.smoke() and the
// CPU baseline arm of bench.py, never by the product.
#include "oracle_fs.h"
#include "oracle_ps.h"

#include <cmath>

extern "C" {

void orc_binary_mag0_many(int n, const double* s, const double* q, const double* x, const double* y,
                          double* A, int* nimg)
{
    for (int i = 0; i < n; ++i) {
        const auto r = oracle::binary_mag0(s[i], q[i], x[i], y[i]);
        A[i] = r.magnification;
        if (nimg) nimg[i] = r.image_count;
    }
}

void orc_binary_mag0_derivatives_many(int n, const double* s, const double* q, const double* x,
                                      const double* y, double* A, int* nimg, double* indicator)
{
    for (int i = 0; i < n; ++i) {
        const auto r = oracle::binary_mag0_derivatives(s[i], q[i], x[i], y[i], &indicator[i]);
        A[i] = r.magnification;
        nimg[i] = r.image_count;
    }
}

int orc_image_candidates(double s, double q, double x, double y, double* out)
{
    return oracle::binary_image_candidates(s, q, x, y, out);
}

void orc_roots(const double* coef, int degree, double* roots, int polish)
{
    oracle::cplx p[6], r[5];
    for (int i = 0; i <= degree; ++i) p[i] = {coef[2 * i], coef[2 * i + 1]};
    oracle::roots_gen(r, p, degree, polish != 0);
    for (int i = 0; i < degree; ++i) {
        roots[2 * i] = r[i].re;
        roots[2 * i + 1] = r[i].im;
    }
}

} // extern "C"
