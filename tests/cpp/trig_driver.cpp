// Host build of the device's correctly rounded sin/cos (lcbi_trig.cuh), for
// tests: sincos_cr over an array.  Compiled with -ffp-contract=off.
#include "lcbi_trig.cuh"

#include <cstdint>

extern "C" void trig_sincos_cr(int64_t n, const double* x, double* s, double* c)
{
    for (int64_t i = 0; i < n; ++i) lcbi::trig::sincos_cr(x[i], s + i, c + i);
}
