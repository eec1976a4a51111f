// Library-wide C ABI pieces: error text, version, FFT twiddle tables.
#include <cmath>
#include <cstdarg>
#include <cstdio>

#include "pt_common.cuh"
#include "pt_fft.cuh"

namespace {
thread_local char g_err[1024] = "";
}

namespace pt {
void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = '\0'; }
}  // namespace pt

void pt_make_twiddles(float2 *tw, int L)
{
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < L; ++m) {
        double a = two_pi * (double)m / (double)L;
        tw[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
}

extern "C" const char *pt_last_error(void) { return g_err; }
extern "C" const char *pt_version(void) { return "ptychotomo_b200 0.1.0 (sm_100a)"; }
