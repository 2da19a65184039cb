// tb_mcpoint.cuh -- the Monte-Carlo quadrature of one tuple over the points
// inside the simplices, shared by the stored-list collision kernel
// (k_collision_mc, tb_collision.cu) and the streamed one (k_collision_stream,
// tb_stream.cu), so that both form every tuple's sums with the same
// operations in the same order.
#pragma once

#include "tb_geom.cuh"

namespace tb {

// The tuple's legs f as (f0, f1, f2) of its linear form t = f0 + f1 x + f2 y
// (the rate's leg: the constant unit form).
template <int L, bool RATE>
__device__ __forceinline__ void leg_values(const ChanDev& c, const InstDev& in, const double* __restrict__ f,
                                           const int (&e)[L], int rate_leg, double (&fv)[L][3]) {
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const double* fe = f + in.foff[l] + 3 * (int64_t)e[l];
#pragma unroll
        for (int j = 0; j < 3; ++j) fv[l][j] = (RATE && l == rate_leg) ? (j == 0 ? 1.0 : 0.0) : __ldg(fe + j);
    }
}

// s0 += sum over the set bits m of mk (increasing m) of the gain-plus-loss
// product at point m, sx[l] / sy[l] += its first moments per leg: TypeB's
// sums (IntegratorCore.hpp:338-357) without the terms whose Theta is 0.  The
// leg forms are A = fa t + fa0, B = fb t + fb0 of the leg's linear form t
// (LegDev: fa, fb = +-1, fa0, fb0 in {0, +-1}), so only f stays in registers.
template <int L, bool RATE>
__device__ __forceinline__ void inside_point_sums(const ChanDev& c, const AlphaMap<L>& am, const double* s_mc,
                                                  uint64_t mk0, const double (&fv)[L][3], int rate_leg, double& s0,
                                                  double (&sx)[L], double (&sy)[L]) {
    constexpr int R = 2 * (L - 2) + 1;
    // One point inside: the legs' points and the gain-plus-loss product (the
    // integrand without its Theta, which is 1 here).
    auto point = [&](int m, double (&px)[L], double (&py)[L]) -> double {
        const double* qv = s_mc + m * R;
        double al[3];
        alpha_fast<L>(am, qv, al);
#pragma unroll
        for (int l = 0; l < L - 2; ++l) { px[l] = qv[2 * l]; py[l] = qv[2 * l + 1]; }
        px[L - 2] = qv[R - 1]; py[L - 2] = al[0];
        px[L - 1] = al[1]; py[L - 1] = al[2];
        double pa = 1.0, pb = 1.0;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const double t = fma(fv[l][2], py[l], fma(fv[l][1], px[l], fv[l][0]));
            double fa = c.leg[l].fa, fa0 = c.leg[l].fa0, fb = c.leg[l].fb, fb0 = c.leg[l].fb0;
            if (RATE && l == rate_leg) {
                // scattering rate of this leg: constant in / out unit forms
                // (ScatteringChannel.cpp:562-564)
                const double d = c.leg[l].dir, st = c.leg[l].stat;
                fa = (l == 0 ? -1.0 : 1.0) * ((1. - d) * st + (1. + d));
                fb = (1. + d) * st + (1. - d);
                fa0 = 0.0;
                fb0 = 0.0;
            }
            pa *= fma(fa, t, fa0);
            pb *= fma(fb, t, fb0);
        }
        return pa + pb;
    };
    auto accumulate = [&](double common, const double (&px)[L], const double (&py)[L]) {
        s0 += common;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            sx[l] = fma(px[l], common, sx[l]);
            sy[l] = fma(py[l], common, sy[l]);
        }
    };
    for (uint64_t mk = mk0; mk; mk &= mk - 1) {
        double px[L], py[L];
        accumulate(point(__ffsll((long long)mk) - 1, px, py), px, py);
    }
}

}  // namespace tb
