// tb_errnorm.cuh -- per-element integrands of Band::relativeError and a
// block reduction, shared by the integrator's error norm and the standalone
// error-norm entry points.
#pragma once

#include "tb_kernels.cuh"

namespace tb {

__device__ __forceinline__ void to_nodal(const double c[3], double n[3]) { n[0] = c[0]; n[1] = c[1] + c[0]; n[2] = c[2] + c[0]; }
__device__ __forceinline__ void to_lin(const double n[3], double c[3]) { c[0] = n[0]; c[1] = n[1] - n[0]; c[2] = n[2] - n[0]; }

__device__ __forceinline__ double gauss2_sq(const double c[3]) {
    const double a = TB_GP2_A, b = TB_GP2_B, w = TB_GW2;
    const double v0 = (c[1] * a + c[2] * a) + c[0];
    const double v1 = (c[1] * b + c[2] * a) + c[0];
    const double v2 = (c[1] * a + c[2] * b) + c[0];
    return ((v0 * v0) * w + (v1 * v1) * w) + (v2 * v2) * w;
}

// Per-element integrands of Band::relativeError with the reference's exact
// sequence of nodal <-> linear-form conversions (Function.cpp:75-109, 152-159).
__device__ __forceinline__ void elem_rel_err(const BandDev& b, const double* err, const double* p, double& rel,
                                             double& pen) {
    double np[3];
    to_nodal(p, np);
    double sc[3];
    double pe[3];
    if (b.stat == -1.0) {
        const double om[3] = {-(p[0] - 1.0), -p[1], -p[2]};
        double nom[3], fa[3], fb[3], la[3], lb[3], na[3], nb[3], mn[3], lm[3];
        to_nodal(om, nom);
#pragma unroll
        for (int k = 0; k < 3; ++k) { fa[k] = fabs(np[k]); fb[k] = fabs(nom[k]); }
        to_lin(fa, la); to_lin(fb, lb);
        to_nodal(la, na); to_nodal(lb, nb);
#pragma unroll
        for (int k = 0; k < 3; ++k) mn[k] = fmin(na[k], nb[k]);
        to_lin(mn, lm);
#pragma unroll
        for (int k = 0; k < 3; ++k) sc[k] = b.rel_tol * lm[k];
        sc[0] += b.abs_tol;
        if (b.penal != 0.0) {
            double m0[3], lm0[3], pm1[3] = {p[0] - 1.0, p[1], p[2]}, npm1[3], x1[3], lx1[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) m0[k] = fmin(np[k], 0.);
            to_lin(m0, lm0);
            to_nodal(pm1, npm1);
#pragma unroll
            for (int k = 0; k < 3; ++k) x1[k] = fmax(npm1[k], 0.);
            to_lin(x1, lx1);
#pragma unroll
            for (int k = 0; k < 3; ++k) pe[k] = -lm0[k] + lx1[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) sc[k] = b.rel_tol * p[k];
        sc[0] += b.abs_tol;
        if (b.penal != 0.0) {
            double m0[3], lm0[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) m0[k] = fmin(np[k], 0.);
            to_lin(m0, lm0);
#pragma unroll
            for (int k = 0; k < 3; ++k) pe[k] = -lm0[k];
        }
    }
    double nsc[3], ner[3], r[3];
    to_nodal(sc, nsc);
    to_nodal(err, ner);
#pragma unroll
    for (int k = 0; k < 3; ++k) ner[k] /= nsc[k];
    to_lin(ner, r);
    rel = gauss2_sq(r);
    pen = 0.0;
    if (b.penal != 0.0) {
        double npe[3], q[3];
        to_nodal(pe, npe);
#pragma unroll
        for (int k = 0; k < 3; ++k) npe[k] /= nsc[k];
        to_lin(npe, q);
        pen = gauss2_sq(q);
    }
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < NT / 32; ++i) s += sh[i];
    return s;
}

}  // namespace tb
