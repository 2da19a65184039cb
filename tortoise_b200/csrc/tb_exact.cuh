// tb_exact.cuh -- order-independent accumulation of FP64 sums (the library's
// deterministic mode, tb_options.deterministic).
//
// FP64 atomics add in whatever order the threads arrive, and every order
// rounds differently: two evaluations of the same collision operator differ
// in their last bits, and an adaptive integration amplifies that.  In the
// deterministic mode the collision, rate and VJP kernels add every per-tuple
// result into an exact fixed-point accumulator instead:
//
//   * a coefficient is a 192-bit two's-complement integer X in units of
//     2^-112 (three 64-bit words, least significant first): range +-2^79,
//     resolution 2^-112 (1.9e-34);
//   * a contribution v is rounded once to that grid (fx_of), then added with
//     64-bit integer atomics and explicit carries (fx_atomic_add).  Integer
//     addition modulo 2^192 is associative and commutative, and the carry out
//     of a word is decided by the running total alone, so any interleaving of
//     the adds leaves the same three words;
//   * the flush kernel rounds X back to FP64 once (fx_value, round to nearest
//     even) and clears the words.
//
// The result is therefore a function of the per-tuple values alone: not of
// the launch geometry, the warp or block a tuple lands in, the contraction
// schedule, or other launches running beside it.  Its accuracy is at least
// that of an FP64 sum: each contribution is off by at most 2^-113, the sum is
// exact, and only the final conversion rounds.
//
// A non-finite contribution cannot be represented: it sets the buffer's
// poison word, and the flush then writes NaN into every coefficient, which
// the integrator reports as TB_ERR_NONFINITE.  A finite contribution of
// magnitude 2^64 or more (a trial stage of a step far too large, on its way
// to rejection) is clamped to the largest double below 2^64 with its sign
// and sets the saturation word: the sum stays exact and deterministic, the
// coefficient stays huge (so the step's error norm rejects it, as it rejects
// the unclamped FP64 value), and the host paths that return an operator
// report the clamping as an error.
//
// The functions compile for the host too (the CPU tests exercise the
// conversions and the order independence through a host build).
#pragma once

#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define TB_HD __host__ __device__ __forceinline__
#else
#define TB_HD inline
#endif

namespace tb {

constexpr int FX_FRAC = 112;   // fraction bits: X = v * 2^112

struct Fx {
    unsigned long long w0, w1, w2;
};

TB_HD unsigned long long fx_bits(double v) {
#ifdef __CUDA_ARCH__
    return (unsigned long long)__double_as_longlong(v);
#else
    unsigned long long u;
    memcpy(&u, &v, sizeof(u));
    return u;
#endif
}

TB_HD double fx_from_bits(unsigned long long u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double v;
    memcpy(&v, &u, sizeof(v));
    return v;
#endif
}

TB_HD int fx_clz(unsigned long long x) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return x ? __builtin_clzll(x) : 64;
#endif
}

// unsigned 64-bit integer to FP64, rounded to nearest even
TB_HD double fx_u64_to_double(unsigned long long x) {
#ifdef __CUDA_ARCH__
    return __ull2double_rn(x);
#else
    return (double)x;
#endif
}

// X = v * 2^112 rounded to the nearest integer (halves away from zero), as
// three two's-complement words.  Returns false (and X = 0) when v is not
// finite or |v| >= 2^64.
TB_HD bool fx_of(double v, Fx& x) {
    const unsigned long long u = fx_bits(v);
    const int E = int((u >> 52) & 0x7ff);
    x.w0 = x.w1 = x.w2 = 0ull;
    if (E >= 1023 + 64) return false;   // |v| >= 2^64, Inf, NaN
    if (E == 0) return true;            // zero and subnormals lie below the grid
    const unsigned long long m = (u & 0xfffffffffffffull) | (1ull << 52);
    // v = m 2^(E - 1075), X = m 2^(E - 1075 + 112)
    const int sh = E - 1075 + FX_FRAC;
    if (sh < 0) {
        const int r = -sh;
        if (r < 64) x.w0 = (m + (1ull << (r - 1))) >> r;
    } else if (sh < 64) {
        x.w0 = m << sh;
        x.w1 = sh ? (m >> (64 - sh)) : 0ull;
    } else {   // 64 <= sh <= 123: the top bit stays below bit 176
        const int s = sh - 64;
        x.w1 = m << s;
        x.w2 = s ? (m >> (64 - s)) : 0ull;
    }
    if (u >> 63) {   // two's complement of the magnitude
        x.w0 = ~x.w0 + 1ull;
        const unsigned long long c0 = (x.w0 == 0ull) ? 1ull : 0ull;
        x.w1 = ~x.w1 + c0;
        const unsigned long long c1 = (c0 && x.w1 == 0ull) ? 1ull : 0ull;
        x.w2 = ~x.w2 + c1;
    }
    return true;
}

// X * 2^-112 as FP64, rounded to nearest even.
TB_HD double fx_value(unsigned long long w0, unsigned long long w1, unsigned long long w2) {
    const bool neg = (w2 >> 63) != 0ull;
    if (neg) {
        w0 = ~w0 + 1ull;
        const unsigned long long c0 = (w0 == 0ull) ? 1ull : 0ull;
        w1 = ~w1 + c0;
        const unsigned long long c1 = (c0 && w1 == 0ull) ? 1ull : 0ull;
        w2 = ~w2 + c1;
    }
    // magnitude M = w2 2^128 + w1 2^64 + w0 = hi 2^b + (rest below 2^b)
    unsigned long long hi, rest;
    int b;
    if (w2) {
        const int lz = fx_clz(w2);
        hi = lz ? ((w2 << lz) | (w1 >> (64 - lz))) : w2;
        rest = (lz ? (w1 << lz) : w1) | w0;
        b = 128 - lz;
    } else if (w1) {
        const int lz = fx_clz(w1);
        hi = lz ? ((w1 << lz) | (w0 >> (64 - lz))) : w1;
        rest = lz ? (w0 << lz) : w0;
        b = 64 - lz;
    } else {
        hi = w0;
        rest = 0ull;
        b = 0;
    }
    // hi has 64 significant bits whenever rest can be non-zero, so a sticky
    // bit in its bit 0 (below the rounding bit 10) rounds like the whole tail
    const double d = fx_u64_to_double(hi | (rest ? 1ull : 0ull));
    const double scale = fx_from_bits((unsigned long long)(1023 + b - FX_FRAC) << 52);   // 2^(b - 112), exact
    const double r = d * scale;
    return neg ? -r : r;
}

// p[0..2] += x (plain, one thread owns p).
TB_HD void fx_add_plain(unsigned long long* p, const Fx& x) {
    const unsigned long long s0 = p[0] + x.w0;
    const unsigned long long c0 = (s0 < x.w0) ? 1ull : 0ull;
    const unsigned long long t1 = x.w1 + c0;
    const unsigned long long c1a = (t1 < c0) ? 1ull : 0ull;
    const unsigned long long s1 = p[1] + t1;
    const unsigned long long c1 = c1a + ((s1 < t1) ? 1ull : 0ull);
    p[0] = s0;
    p[1] = s1;
    p[2] = p[2] + x.w2 + c1;
}

// The sink of a deterministic launch: w holds three words per FP64 slot of
// the accumulator it stands for (slot k at w + 3k); poison is the buffer's
// flag for values the grid cannot hold.  w == nullptr: FP64 atomics instead.
struct FxAcc {
    unsigned long long* w = nullptr;
    unsigned int* poison = nullptr;
    unsigned int* sat = nullptr;   // sticky: a contribution was clamped (null: poison instead)
};

// The largest double below 2^64: the clamp of out-of-range contributions.
constexpr double FX_CLAMP = 18446744073709549568.0;   // 2^64 - 2^11

#ifdef __CUDACC__
// p[0..2] += x with atomics, exact for any interleaving with other adds.
__device__ __forceinline__ void fx_atomic_add(unsigned long long* p, const Fx& x) {
    unsigned long long c = 0ull;
    if (x.w0) {
        const unsigned long long o = atomicAdd(p, x.w0);
        c = (o + x.w0 < o) ? 1ull : 0ull;
    }
    const unsigned long long a1 = x.w1 + c;
    unsigned long long c2 = (a1 < c) ? 1ull : 0ull;   // x.w1 + c wrapped to 0
    if (a1) {
        const unsigned long long o = atomicAdd(p + 1, a1);
        c2 += (o + a1 < o) ? 1ull : 0ull;
    }
    const unsigned long long a2 = x.w2 + c2;
    if (a2) atomicAdd(p + 2, a2);
}

__device__ __forceinline__ void fx_add(const FxAcc& a, int64_t slot, double v) {
    Fx x;
    if (!fx_of(v, x)) {
        if (!isfinite(v) || !a.sat) {
            atomicOr(a.poison, 1u);
            return;
        }
        atomicOr(a.sat, 1u);
        fx_of(v < 0.0 ? -FX_CLAMP : FX_CLAMP, x);
    }
    if (x.w0 | x.w1 | x.w2) fx_atomic_add(a.w + 3 * slot, x);
}

__device__ __forceinline__ void fx_add3(const FxAcc& a, int64_t slot, double v0, double v1, double v2) {
    fx_add(a, slot, v0);
    fx_add(a, slot + 1, v1);
    fx_add(a, slot + 2, v2);
}
#endif

}  // namespace tb
