// Host build of the exact accumulator's arithmetic (tortoise_b200/csrc/
// tb_exact.cuh) for the CPU tests: conversions to and from the 192-bit
// fixed-point words and the carrying add, through a C ABI for ctypes.
#include "../tortoise_b200/csrc/tb_exact.cuh"

extern "C" {

// words[3] = v on the 2^-112 grid; returns 0 when v cannot be held
int fx_host_of(double v, unsigned long long* words) {
    tb::Fx x;
    const bool ok = tb::fx_of(v, x);
    words[0] = x.w0;
    words[1] = x.w1;
    words[2] = x.w2;
    return ok ? 1 : 0;
}

double fx_host_value(const unsigned long long* words) { return tb::fx_value(words[0], words[1], words[2]); }

// the clamp of out-of-range finite contributions
double fx_host_clamp() { return tb::FX_CLAMP; }

// acc[3] += the words of every v[i] in the given order; returns how many
// values could not be held
int fx_host_sum(const double* v, const long long* order, long long n, unsigned long long* acc) {
    int bad = 0;
    for (long long k = 0; k < n; ++k) {
        tb::Fx x;
        if (!tb::fx_of(v[order[k]], x)) { ++bad; continue; }
        tb::fx_add_plain(acc, x);
    }
    return bad;
}

}
