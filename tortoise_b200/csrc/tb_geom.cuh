// tb_geom.cuh -- per-tuple delta-constraint geometry shared by the tuple
// enumeration and the collision kernels.
//
// For one tuple of L elements (one per leg) the energy/momentum delta
// delta(D K - N) of the reference is built from the P1 coefficients of
// kx, ky and E of each leg's element:
//   constructD / constructN   src/Physics/Scattering/ScatteringChannel.cpp:302-352
//   integrationInversionDeterminant  include/Physics/Scattering/IntegratorCore.hpp:153-155
// The constrained block DC is the last 3 columns of D (NDim+1 = 3).
#pragma once

#include "tb_common.cuh"

namespace tb {

// Explicitly rounded FP64 operations: never contracted into FMAs, so these
// expressions round exactly like the unfused C++ of the reference (and the
// oracle) whatever --fmad says.  Every quantity that feeds a discrete
// decision (determinant filter, simplex tests Theta) is computed with them.
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }

template <int L>
struct TupleGeom {
    double D[3][2 * L];
    double N[3];
    double det;       // det(DC), 3x3 cofactor expansion along row 0
};

template <int L>
__device__ __forceinline__ void tuple_geometry(const ChanDev& c, const int (&e)[L], int umk, TupleGeom<L>& g) {
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const double d = c.leg[l].dir;
        const double* kx = c.leg[l].kx + 3 * (int64_t)e[l];
        const double* ky = c.leg[l].ky + 3 * (int64_t)e[l];
        const double* en = c.leg[l].disp + 3 * (int64_t)e[l];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            g.D[0][2 * l + j] = d * __ldg(kx + 1 + j);
            g.D[1][2 * l + j] = d * __ldg(ky + 1 + j);
            g.D[2][2 * l + j] = d * __ldg(en + 1 + j);
        }
    }
    g.N[0] = 0.0; g.N[1] = 0.0; g.N[2] = 0.0;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const double d = c.leg[l].dir;
        g.N[0] = xs(g.N[0], xm(d, __ldg(c.leg[l].kx + 3 * (int64_t)e[l])));
        g.N[1] = xs(g.N[1], xm(d, __ldg(c.leg[l].ky + 3 * (int64_t)e[l])));
        g.N[2] = xs(g.N[2], xm(d, __ldg(c.leg[l].disp + 3 * (int64_t)e[l])));
    }
    const double u0 = c.umk[2 * umk], u1 = c.umk[2 * umk + 1];
#pragma unroll
    for (int dim = 0; dim < 2; ++dim) {
        g.N[dim] = xs(g.N[dim], xm(u0, c.gvec[dim]));
        g.N[dim] = xs(g.N[dim], xm(u1, c.gvec[2 + dim]));
    }
    const int c0 = 2 * L - 3;
    const double a00 = g.D[0][c0], a01 = g.D[0][c0 + 1], a02 = g.D[0][c0 + 2];
    const double a10 = g.D[1][c0], a11 = g.D[1][c0 + 1], a12 = g.D[1][c0 + 2];
    const double a20 = g.D[2][c0], a21 = g.D[2][c0 + 1], a22 = g.D[2][c0 + 2];
    g.det = xa(xs(xm(a00, xs(xm(a11, a22), xm(a12, a21))), xm(a01, xs(xm(a10, a22), xm(a12, a20)))),
               xm(a02, xs(xm(a10, a21), xm(a11, a20))));
}

// Inverse of DC by cofactors scaled with the reciprocal of the column-0
// cofactor expansion (the standard adjugate formula).
template <int L>
__device__ __forceinline__ void dc_inverse(const TupleGeom<L>& g, double Ci[3][3]) {
    const int c0 = 2 * L - 3;
    double a[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a[i][j] = g.D[i][c0 + j];
    double cof[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            cof[i][j] = xs(xm(a[i1][j1], a[i2][j2]), xm(a[i1][j2], a[i2][j1]));
        }
    const double det = xa(xa(xm(cof[0][0], a[0][0]), xm(cof[1][0], a[1][0])), xm(cof[2][0], a[2][0]));
    const double invdet = __ddiv_rn(1.0, det);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Ci[j][i] = xm(cof[i][j], invdet);
}

// alpha = -DC^-1 (DF q - N) in the reference's evaluation order, unfused.
template <int L>
__device__ __forceinline__ void exact_alpha(const TupleGeom<L>& g, const double (&Ci)[3][3], const double* q,
                                            double (&alpha)[3]) {
    constexpr int R = 2 * (L - 2) + 1;
    const double kp0 = q[R - 1];
    double r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        if (L >= 3) s = xa(s, xa(xm(g.D[i][0], q[0]), xm(g.D[i][1], q[1])));
        if (L >= 4) s = xa(s, xa(xm(g.D[i][2], q[2]), xm(g.D[i][3], q[3])));
        s = xa(s, xm(g.D[i][2 * (L - 2)], kp0));
        r[i] = xs(s, g.N[i]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) alpha[i] = -xa(xa(xm(Ci[i][0], r[0]), xm(Ci[i][1], r[1])), xm(Ci[i][2], r[2]));
}

// ThetapC * ThetaFC (IntegratorCore.hpp:318-320): both partially and fully
// constrained legs strictly inside the reference triangle.
__device__ __forceinline__ bool theta_of(double kp0, const double (&al)[3]) {
    const bool thp = (kp0 > 0.0) && (al[0] > 0.0) && (xa(kp0, al[0]) < 1.0);
    const bool thc = (al[1] > 0.0) && (al[2] > 0.0) && (xa(al[1], al[2]) < 1.0);
    return thp && thc;
}

// The affine map q -> alpha = G q + alpha0 (G = -DC^-1 DF, alpha0 = DC^-1 N)
// of one tuple, for the fast fused evaluation, with a rigorous rounding
// bound mg per coordinate: a point whose fast alpha lies farther than that
// from every simplex boundary gets the same Theta as the unfused reference
// order; the others are re-evaluated exactly (alpha_theta).
template <int L>
struct AlphaMap {
    static constexpr int R = 2 * (L - 2) + 1;
    double G[3][R], a0[3], mg[3];
};

// Every product-sum is written as explicit fused multiply-adds in a fixed
// order, so the map (and everything the quadrature computes from it) has the
// same bits in every kernel that builds it, whatever the compiler would
// contract on its own.
template <int L>
__device__ __forceinline__ void alpha_map(const TupleGeom<L>& g, const double (&Ci)[3][3], AlphaMap<L>& am) {
    constexpr int R = AlphaMap<L>::R;
    double rho[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double t = fabs(g.N[k]);
#pragma unroll
        for (int j = 0; j < R; ++j) t += fabs(g.D[k][j]);
        rho[k] = t;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        am.a0[r] = fma(Ci[r][2], g.N[2], fma(Ci[r][1], g.N[1], __dmul_rn(Ci[r][0], g.N[0])));
        double sg = 0.0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            am.G[r][j] = -fma(Ci[r][2], g.D[2][j], fma(Ci[r][1], g.D[1][j], __dmul_rn(Ci[r][0], g.D[0][j])));
            sg += fabs(am.G[r][j]);
        }
        const double sc = fma(fabs(Ci[r][2]), rho[2], fma(fabs(Ci[r][1]), rho[1], __dmul_rn(fabs(Ci[r][0]), rho[0])));
        am.mg[r] = 32.0 * 1.1102230246251565e-16 * (sc + fabs(am.a0[r]) + sg);
    }
}

// Fast constrained coordinates of point qv (fused multiply-adds).
template <int L>
__device__ __forceinline__ void alpha_fast(const AlphaMap<L>& am, const double* qv, double (&al)[3]) {
    constexpr int R = AlphaMap<L>::R;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double t = am.a0[r];
#pragma unroll
        for (int j = 0; j < R; ++j) t = fma(am.G[r][j], qv[j], t);
        al[r] = t;
    }
}

// Constrained coordinates and Theta of point qv with the reference's
// decisions: the fast value, re-evaluated in the exact order when it lies
// within the rounding bound of a simplex boundary.
template <int L>
__device__ __forceinline__ bool alpha_theta(const TupleGeom<L>& g, const double (&Ci)[3][3], const AlphaMap<L>& am,
                                            const double* qv, double (&al)[3]) {
    constexpr int R = AlphaMap<L>::R;
    alpha_fast<L>(am, qv, al);
    const double kp0 = qv[R - 1];
    const double tiny = 8.0 * 1.1102230246251565e-16;
    const bool near = (fabs(al[0]) <= am.mg[0]) || (fabs(al[1]) <= am.mg[1]) || (fabs(al[2]) <= am.mg[2]) ||
                      (fabs(kp0 + al[0] - 1.0) <= am.mg[0] + tiny * (2.0 + fabs(al[0]))) ||
                      (fabs(al[1] + al[2] - 1.0) <= am.mg[1] + am.mg[2] + tiny * (1.0 + fabs(al[1]) + fabs(al[2])));
    if (near) exact_alpha<L>(g, Ci, qv, al);
    return theta_of(kp0, al);
}

// The decision of alpha_theta for point qv without its coordinates: a point
// whose fused coordinates already violate a simplex test by more than the
// rounding bound is outside whatever the evaluation order (the exact value
// lies within the bound of the fused one), so it is decided after the fused
// map alone; every other point goes through alpha_theta.  Most points of a
// tuple that does not survive are decided that way.
template <int L>
__device__ __forceinline__ bool theta_decide(const TupleGeom<L>& g, const double (&Ci)[3][3], const AlphaMap<L>& am,
                                             const double* qv) {
    constexpr int R = AlphaMap<L>::R;
    double al[3];
    alpha_fast<L>(am, qv, al);
    const double kp0 = qv[R - 1];
    const double tiny = 8.0 * 1.1102230246251565e-16;
    const bool out = (al[0] < -am.mg[0]) || (al[1] < -am.mg[1]) || (al[2] < -am.mg[2]) ||
                     (kp0 + al[0] - 1.0 > am.mg[0] + tiny * (2.0 + fabs(al[0]))) ||
                     (al[1] + al[2] - 1.0 > am.mg[1] + am.mg[2] + tiny * (1.0 + fabs(al[1]) + fabs(al[2])));
    if (out) return false;
    return alpha_theta<L>(g, Ci, am, qv, al);
}

// Constrained coordinates of one MC point q (row of the MC table),
// IntegratorCore.hpp:298-320:  alpha = -DC^-1 (DF q - N).
// Returns the simplex tests ThetapC * ThetaFC (IntegratorCore.hpp:318-320);
// p receives the leg points in reference coordinates.
template <int L>
__device__ __forceinline__ bool mc_point_exact(const TupleGeom<L>& g, const double (&Ci)[3][3], const double* q,
                                               double (&p)[L][2]) {
    constexpr int R = 2 * (L - 2) + 1;
    const double kp0 = q[R - 1];
    double alpha[3];
    exact_alpha<L>(g, Ci, q, alpha);
#pragma unroll
    for (int l = 0; l < L - 2; ++l) { p[l][0] = q[2 * l]; p[l][1] = q[2 * l + 1]; }
    p[L - 2][0] = kp0;
    p[L - 2][1] = alpha[0];
    p[L - 1][0] = alpha[1];
    p[L - 1][1] = alpha[2];
    return theta_of(kp0, alpha);
}

}  // namespace tb
