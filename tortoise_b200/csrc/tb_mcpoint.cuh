// tb_mcpoint.cuh -- the Monte-Carlo quadrature of one tuple over the points
// inside the simplices, shared by the stored-list collision kernel
// (k_collision_mc, tb_collision.cu) and the streamed one (k_collision_stream,
// tb_stream.cu), so that both form every tuple's sums with the same
// operations in the same order.
#pragma once

#include "tb_geom.cuh"
#include "tb_kernels.cuh"

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
        // explicit products and sum: no contraction the compiler could choose
        // differently in another kernel
        double pa = 1.0, pb = 1.0;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const double t = fma(fv[l][2], py[l], fma(fv[l][1], px[l], fv[l][0]));
            double fa = c.leg[l].fa, fa0 = c.leg[l].fa0, fb = c.leg[l].fb, fb0 = c.leg[l].fb0;
            if (RATE && l == rate_leg) {
                // scattering rate of this leg: constant in / out unit forms
                // (ScatteringChannel.cpp:562-564)
                const double d = c.leg[l].dir, st = c.leg[l].stat;
                fa = (l == 0 ? -1.0 : 1.0) * __dadd_rn(__dmul_rn(1. - d, st), 1. + d);
                fb = __dadd_rn(__dmul_rn(1. + d, st), 1. - d);
                fa0 = 0.0;
                fb0 = 0.0;
            }
            pa = __dmul_rn(pa, fma(fa, t, fa0));
            pb = __dmul_rn(pb, fma(fb, t, fb0));
        }
        return __dadd_rn(pa, pb);
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

// Sum over the warp, then one add per warp into dst (exact into slot k of
// fx in the deterministic mode; the warp's own sum runs in a fixed order, so
// it depends only on which tuples share the warp).  All lanes call it.
__device__ __forceinline__ void block_atomic_sum(double v, double* dst, const FxAcc& fx, int k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) {
        if (fx.w) fx_add(fx, k, v);
        else atomicAdd(dst, v);
    }
}

// The loss / gain forms A, B of every leg (ScatteringChannel.cpp:633-641)
// and their slopes sa, sb with respect to the leg's coefficients of f.
template <int L>
__device__ __forceinline__ void leg_forms(const ChanDev& c, const InstDev& in, const double* f, const int (&e)[L],
                                          double (&A)[L][3], double (&B)[L][3], double (&sa)[L], double (&sb)[L]) {
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const double d = c.leg[l].dir, s = c.leg[l].stat;
        const double* fe = f + in.foff[l] + 3 * (int64_t)e[l];
        const double ka = (l == 0 ? -1.0 : 1.0) * 0.5;
        const double ca = (1. - d) * s + (1. + d);
        const double cb = (1. + d) * s + (1. - d);
        sa[l] = ka * ca;    // dA[l][j] / df_j
        sb[l] = 0.5 * cb;   // dB[l][j] / df_j
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double unit = (j == 0) ? 1.0 : 0.0;
            const double fj = __ldg(fe + j);
            A[l][j] = ka * ((1. - d) * unit + ca * fj);
            B[l][j] = 0.5 * ((1. + d) * unit + cb * fj);
        }
    }
}

// The transposed quadrature of one tuple for one instance (the VJP of
// TypeB's sums): gA[l][j], gB[l][j] = d/dA[l][j], d/dB[l][j] of
// sum_points (u-weighted test functions) x (prod A + prod B), and gamp = the
// sum itself, over the points with Theta = 1: every point (LIST false, the
// exact decision per point) or the set bits of mk0 in increasing order (LIST
// true).  Zeros when valid is false.
template <int L, bool LIST>
__device__ __forceinline__ void vjp_point_sums(const ChanDev& c, const InstDev& in, const double* __restrict__ f,
                                               const double* __restrict__ u, const int (&e)[L],
                                               const TupleGeom<L>& g, const double (&Ci)[3][3], const double* s_mc,
                                               uint64_t mk0, bool valid, double (&gA)[L][3], double (&gB)[L][3],
                                               double& gamp, double (&sa)[L], double (&sb)[L]) {
    constexpr int R = 2 * (L - 2) + 1;
    double A[L][3], B[L][3];
    leg_forms<L>(c, in, f, e, A, B, sa, sb);
    double ul[L][3];
#pragma unroll
    for (int l = 0; l < L; ++l)
#pragma unroll
        for (int j = 0; j < 3; ++j) ul[l][j] = c.leg[l].dir * __ldg(u + in.foff[l] + 3 * (int64_t)e[l] + j);
    gamp = 0.0;
#pragma unroll
    for (int l = 0; l < L; ++l)
#pragma unroll
        for (int j = 0; j < 3; ++j) { gA[l][j] = 0.0; gB[l][j] = 0.0; }
    if (!valid) return;
    uint64_t mk = mk0;
    for (int m = 0; LIST ? (mk != 0) : (m < c.nmc); ++m) {
        if (LIST) {
            m = __ffsll((long long)mk) - 1;
            mk &= mk - 1;
        }
        const double* qv = s_mc + m * R;
        double p[L][2];
        if (!mc_point_exact<L>(g, Ci, qv, p)) continue;
        // every product-sum as explicit fused multiply-adds or rounded
        // operations: the same bits in every kernel that runs this
        double av[L], bv[L];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            av[l] = __dadd_rn(fma(A[l][2], p[l][1], __dmul_rn(A[l][1], p[l][0])), A[l][0]);
            bv[l] = __dadd_rn(fma(B[l][2], p[l][1], __dmul_rn(B[l][1], p[l][0])), B[l][0]);
        }
        double om = 0.0;   // sum over legs of dir * (u . test functions)
#pragma unroll
        for (int l = 0; l < L; ++l) om = __dadd_rn(om, fma(ul[l][2], p[l][1], fma(ul[l][1], p[l][0], ul[l][0])));
        double pa = 1.0, pb = 1.0;
#pragma unroll
        for (int l = 0; l < L; ++l) { pa = __dmul_rn(pa, av[l]); pb = __dmul_rn(pb, bv[l]); }
        gamp = fma(om, __dadd_rn(pa, pb), gamp);
#pragma unroll
        for (int mm = 0; mm < L; ++mm) {
            double ra = om, rb = om;
#pragma unroll
            for (int l = 0; l < L; ++l)
                if (l != mm) { ra = __dmul_rn(ra, av[l]); rb = __dmul_rn(rb, bv[l]); }
            gA[mm][0] = __dadd_rn(gA[mm][0], ra);
            gA[mm][1] = fma(ra, p[mm][0], gA[mm][1]);
            gA[mm][2] = fma(ra, p[mm][1], gA[mm][2]);
            gB[mm][0] = __dadd_rn(gB[mm][0], rb);
            gB[mm][1] = fma(rb, p[mm][0], gB[mm][1]);
            gB[mm][2] = fma(rb, p[mm][1], gB[mm][2]);
        }
    }
}

}  // namespace tb
