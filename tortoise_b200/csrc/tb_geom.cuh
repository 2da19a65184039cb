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
        g.N[0] -= d * __ldg(c.leg[l].kx + 3 * (int64_t)e[l]);
        g.N[1] -= d * __ldg(c.leg[l].ky + 3 * (int64_t)e[l]);
        g.N[2] -= d * __ldg(c.leg[l].disp + 3 * (int64_t)e[l]);
    }
    const double u0 = c.umk[2 * umk], u1 = c.umk[2 * umk + 1];
#pragma unroll
    for (int dim = 0; dim < 2; ++dim) {
        g.N[dim] -= u0 * c.gvec[dim];
        g.N[dim] -= u1 * c.gvec[2 + dim];
    }
    const int c0 = 2 * L - 3;
    const double a00 = g.D[0][c0], a01 = g.D[0][c0 + 1], a02 = g.D[0][c0 + 2];
    const double a10 = g.D[1][c0], a11 = g.D[1][c0 + 1], a12 = g.D[1][c0 + 2];
    const double a20 = g.D[2][c0], a21 = g.D[2][c0 + 1], a22 = g.D[2][c0 + 2];
    g.det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
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
            cof[i][j] = a[i1][j1] * a[i2][j2] - a[i1][j2] * a[i2][j1];
        }
    const double det = (cof[0][0] * a[0][0] + cof[1][0] * a[1][0]) + cof[2][0] * a[2][0];
    const double invdet = 1.0 / det;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Ci[j][i] = cof[i][j] * invdet;
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
    double r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        if (L >= 3) s += g.D[i][0] * q[0] + g.D[i][1] * q[1];
        if (L >= 4) s += g.D[i][2] * q[2] + g.D[i][3] * q[3];
        s += g.D[i][2 * (L - 2)] * kp0;
        r[i] = s - g.N[i];
    }
    double alpha[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) alpha[i] = -(Ci[i][0] * r[0] + Ci[i][1] * r[1] + Ci[i][2] * r[2]);
#pragma unroll
    for (int l = 0; l < L - 2; ++l) { p[l][0] = q[2 * l]; p[l][1] = q[2 * l + 1]; }
    p[L - 2][0] = kp0;
    p[L - 2][1] = alpha[0];
    p[L - 1][0] = alpha[1];
    p[L - 1][1] = alpha[2];
    const bool thp = (kp0 > 0.0) && (alpha[0] > 0.0) && (kp0 + alpha[0] < 1.0);
    const bool thc = (alpha[1] > 0.0) && (alpha[2] > 0.0) && (alpha[1] + alpha[2] < 1.0);
    return thp && thc;
}

}  // namespace tb
