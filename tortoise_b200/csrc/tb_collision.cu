// tb_collision.cu -- collision operator, Monte-Carlo quadrature per tuple.
//
// One thread owns one tuple (grid-stride), which is the reference's
// singleScatteringPropagator (src/Physics/Scattering/ScatteringChannel.cpp:
// 618-650) with scatteringIntegrationTypeB (include/Physics/Scattering/
// IntegratorCore.hpp:260-357) inlined:
//   * geometry D, N, det DC, DC^-1 from the per-element P1 tables (L2/L1 hits)
//   * the affine map q -> alpha of the constrained coordinates is folded once
//     per tuple into alpha = alpha0 + G q  (G = -DC^-1 DF, alpha0 = DC^-1 N)
//   * the Monte-Carlo table lives in shared memory and is read as a broadcast
//   * gain-minus-loss products and the (1 + 2L) distinct output moments are
//     accumulated in FP64 registers
//   * the 3L results are scattered with FP64 atomics (RED) into the pre-M^-1
//     accumulator, which stays L2-resident.
// The kernel is FP64-FMA bound (about 55 FP64 operations per MC point for L=4).
#include "tb_dp45.cuh"
#include "tb_geom.cuh"
#include "tb_kernels.cuh"
#include "tb_scatter.cuh"

namespace tb {

// RATE: scattering-rate variant (rate_leg >= 0), a separate instantiation so
// that the propagate path keeps its register allocation.
template <int L, bool RATE>
__global__ void __launch_bounds__(256) k_collision_mc(ChanDev c, const InstDev* __restrict__ insts, int n_insts,
                                                      const int32_t* __restrict__ tup, int64_t stride, int64_t n,
                                                      const double* __restrict__ f, double* __restrict__ acc,
                                                      const DPCtl* __restrict__ ctl, int rate_leg) {
    extern __shared__ double s_mc[];
    constexpr int R = 2 * (L - 2) + 1;
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) s_mc[i] = c.mc[i];
    __syncthreads();
    const double inv_fact_nmc = c.fact * double(c.nmc);
    // warp-uniform loop: every lane of a warp shares `base`, so the warp
    // scatter below can reduce across lanes
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool valid = i < n;
        int e[L];
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = valid ? __ldg(tup + l * stride + i) : 0;
        const int u = valid ? __ldg(tup + L * stride + i) : 0;
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, u, g);
        if (!(fabs(g.det) >= c.min_det)) valid = false;   // also NaN-safe for padding lanes
        double Ci[3][3];
        dc_inverse<L>(g, Ci);
        // alpha = -Ci (DF q - N) = G q + alpha0 (fast path, FMA).  The
        // simplex tests must agree with the unfused reference evaluation,
        // so every point whose fast alpha lies within a rigorous rounding
        // bound of a test boundary is re-evaluated in the exact order.
        double G[3][R], a0[3], mg[3];
        {
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
                a0[r] = Ci[r][0] * g.N[0] + Ci[r][1] * g.N[1] + Ci[r][2] * g.N[2];
                double sg = 0.0;
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    G[r][j] = -(Ci[r][0] * g.D[0][j] + Ci[r][1] * g.D[1][j] + Ci[r][2] * g.D[2][j]);
                    sg += fabs(G[r][j]);
                }
                const double sc = fabs(Ci[r][0]) * rho[0] + fabs(Ci[r][1]) * rho[1] + fabs(Ci[r][2]) * rho[2];
                mg[r] = 32.0 * 1.1102230246251565e-16 * (sc + fabs(a0[r]) + sg);
            }
        }
        // functAmplitude of this tuple (fullAmplitude = amplitude * volumes * functAmplitude)
        const double tf = (c.tamp && valid) ? __ldg(c.tamp + i) : 1.0;
        for (int k = 0; k < n_insts; ++k) {
            const InstDev in = insts[k];
            if (in.amp_full == 0.0) continue;
            if (ctl && ctl[in.run].done) continue;
            if (!__any_sync(0xffffffffu, valid)) continue;
            const double ampt = in.amp_full * tf;
            // commonLinForm0 (A, direct) and commonLinForm1 (B, time reversed),
            // ScatteringChannel.cpp:633-641
            double A[L][3], B[L][3];
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const double d = c.leg[l].dir, s = c.leg[l].stat;
                const double* fe = f + in.foff[l] + 3 * (int64_t)e[l];
                const double ka = (l == 0 ? -1.0 : 1.0) * 0.5;
                const double ca = (1. - d) * s + (1. + d);
                const double cb = (1. + d) * s + (1. - d);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double unit = (j == 0) ? 1.0 : 0.0;
                    const double fj = __ldg(fe + j);
                    A[l][j] = ka * ((1. - d) * unit + ca * fj);
                    B[l][j] = 0.5 * ((1. + d) * unit + cb * fj);
                }
                if (RATE && l == rate_leg) {
                    // scattering rate of this leg: constant in / out unit forms
                    // (ScatteringChannel.cpp:562-564)
                    A[l][0] = (l == 0 ? -1.0 : 1.0) * ca; A[l][1] = 0.0; A[l][2] = 0.0;
                    B[l][0] = cb; B[l][1] = 0.0; B[l][2] = 0.0;
                }
            }
            double s0 = 0.0, sx[L], sy[L];
#pragma unroll
            for (int l = 0; l < L; ++l) { sx[l] = 0.0; sy[l] = 0.0; }
            for (int m = 0; m < c.nmc; ++m) {
                const double* q = s_mc + m * R;
                double qv[R];
#pragma unroll
                for (int j = 0; j < R; ++j) qv[j] = q[j];
                double al[3];
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    double t = a0[r];
#pragma unroll
                    for (int j = 0; j < R; ++j) t = fma(G[r][j], qv[j], t);
                    al[r] = t;
                }
                const double kp0 = qv[R - 1];
                const double tiny = 8.0 * 1.1102230246251565e-16;
                const bool near = (fabs(al[0]) <= mg[0]) || (fabs(al[1]) <= mg[1]) || (fabs(al[2]) <= mg[2]) ||
                                  (fabs(kp0 + al[0] - 1.0) <= mg[0] + tiny * (2.0 + fabs(al[0]))) ||
                                  (fabs(al[1] + al[2] - 1.0) <= mg[1] + mg[2] + tiny * (1.0 + fabs(al[1]) + fabs(al[2])));
                if (near) exact_alpha<L>(g, Ci, qv, al);
                const bool th = theta_of(kp0, al);
                double px[L], py[L];
#pragma unroll
                for (int l = 0; l < L - 2; ++l) { px[l] = qv[2 * l]; py[l] = qv[2 * l + 1]; }
                px[L - 2] = kp0; py[L - 2] = al[0];
                px[L - 1] = al[1]; py[L - 1] = al[2];
                double pa = 1.0, pb = 1.0;
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    pa *= (A[l][1] * px[l] + A[l][2] * py[l]) + A[l][0];
                    pb *= (B[l][1] * px[l] + B[l][2] * py[l]) + B[l][0];
                }
                const double common = (pa + pb) * (th ? 1.0 : 0.0);
                s0 += common;
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    sx[l] = fma(px[l], common, sx[l]);
                    sy[l] = fma(py[l], common, sy[l]);
                }
            }
            const double scale = valid ? 1.0 / (inv_fact_nmc * fabs(g.det)) : 0.0;
#pragma unroll
            for (int l = 0; l < L; ++l) {
                if (RATE && l != rate_leg) continue;   // uniform: the rate keeps one leg
                const double d = RATE ? -c.leg[l].dir : c.leg[l].dir;
                const int64_t key = in.foff[l] + 3 * (int64_t)e[l];
                if (l < L - 1) {
                    warp_scatter3(valid ? key : -1, acc + key, d * ((scale * s0) * ampt),
                                  d * ((scale * sx[l]) * ampt), d * ((scale * sy[l]) * ampt));
                } else if (valid) {
                    double* o = acc + key;
                    atomicAdd(o + 0, d * ((scale * s0) * ampt));
                    atomicAdd(o + 1, d * ((scale * sx[l]) * ampt));
                    atomicAdd(o + 2, d * ((scale * sy[l]) * ampt));
                }
            }
        }
    }
}

int launch_collision_mc(const ChanDev& c, const InstDev* insts, int n_insts, const int32_t* tup, int64_t stride,
                        int64_t n, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s, int grid_hint,
                        int rate_leg) {
    if (n <= 0 || n_insts <= 0) return TB_OK;
    const int threads = 256;
    int64_t blocks = (n + threads - 1) / threads;
    if (grid_hint > 0 && blocks > grid_hint) blocks = grid_hint;
    const size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
#define TB_MC_LAUNCH(LL)                                                                                           \
    if (rate_leg >= 0)                                                                                             \
        k_collision_mc<LL, true><<<unsigned(blocks), threads, smem, s>>>(c, insts, n_insts, tup, stride, n, f, acc, \
                                                                          ctl, rate_leg);                          \
    else                                                                                                           \
        k_collision_mc<LL, false><<<unsigned(blocks), threads, smem, s>>>(c, insts, n_insts, tup, stride, n, f,     \
                                                                           acc, ctl, -1);
    switch (c.L) {
        case 2: TB_MC_LAUNCH(2) break;
        case 3: TB_MC_LAUNCH(3) break;
        case 4: TB_MC_LAUNCH(4) break;
        default: set_error("nlegs must be 2..4"); return TB_ERR_ARG;
    }
#undef TB_MC_LAUNCH
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// ------------------------------------------------------------ inverse mass
__global__ void k_inverse_mass(ElemDev ed, const double* __restrict__ acc, double* __restrict__ out) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const double* a = acc + bd.off + 3 * (int64_t)e;
    double* o = out + bd.off + 3 * (int64_t)e;
    const double x = a[0], y = a[1], z = a[2];
#pragma unroll
    for (int j = 0; j < 3; ++j) o[j] = x * bd.mesh.Minv[0][j] + y * bd.mesh.Minv[1][j] + z * bd.mesh.Minv[2][j];
}

int launch_inverse_mass(const ElemDev& ed, const double* acc, double* out, cudaStream_t s) {
    k_inverse_mass<<<ed.nblk, 256, 0, s>>>(ed, acc, out);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

}  // namespace tb
