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
//     accumulator, which stays L2-resident; in the deterministic mode they
//     go to the exact fixed-point accumulator instead (tb_exact.cuh), one
//     lane at a time.
// The kernel is FP64-FMA bound (about 55 FP64 operations per MC point for L=4).
// LIST: the same quadrature over a ThetaList (tb_theta.cu): the tuples with at
// least one point inside the simplices, each visiting only those points (set
// bits of its mask, in increasing order), i.e. the dense sums without their
// terms that are the integrand times Theta = 0.
#include "tb_dp45.cuh"
#include "tb_geom.cuh"
#include "tb_kernels.cuh"
#include "tb_mcpoint.cuh"
#include "tb_scatter.cuh"

// Largest shared-memory accumulator (all instances' blocks) a launch uses;
// beyond it the results go straight to the global accumulator.
#ifndef TB_MC_SACC_MAX_BYTES
#define TB_MC_SACC_MAX_BYTES (160 * 1024)
#endif
// Resident blocks per SM the list kernels are compiled for: 2 caps them at
// 128 registers (16 warps per SM instead of 8 at 157 registers, a few bytes
// of spill); measured 3.63 against 5.50 ms on the 16x16 e-e channel.
#ifndef TB_MC_LIST_MIN_BLOCKS
#define TB_MC_LIST_MIN_BLOCKS 2
#endif
// With the shared-memory accumulator, legs below this index merge equal
// element keys across the warp before their atomics (the list is grouped by
// the leg-0 element); the others add directly.  Merging every leg measured
// faster than merging leg 0 only (3.63 against 4.24 ms, 16x16 e-e).
#ifndef TB_MC_SACC_SCAN_LEGS
#define TB_MC_SACC_SCAN_LEGS 4
#endif

namespace tb {

// One Monte-Carlo point of TypeB (IntegratorCore.hpp:338-357): the legs'
// points in reference coordinates (free legs from the table, the partially
// and fully constrained legs from alpha), the gain-plus-loss product times
// Theta, and its first moments per leg.
template <int L>
__device__ __forceinline__ void mc_point_accumulate(const double (&A)[L][3], const double (&B)[L][3],
                                                    const double* qv, const double (&al)[3], double th, double& s0,
                                                    double (&sx)[L], double (&sy)[L]) {
    constexpr int R = 2 * (L - 2) + 1;
    double px[L], py[L];
#pragma unroll
    for (int l = 0; l < L - 2; ++l) { px[l] = qv[2 * l]; py[l] = qv[2 * l + 1]; }
    px[L - 2] = qv[R - 1]; py[L - 2] = al[0];
    px[L - 1] = al[1]; py[L - 1] = al[2];
    double pa = 1.0, pb = 1.0;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        pa *= (A[l][1] * px[l] + A[l][2] * py[l]) + A[l][0];
        pb *= (B[l][1] * px[l] + B[l][2] * py[l]) + B[l][0];
    }
    const double common = (pa + pb) * th;
    s0 += common;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        sx[l] = fma(px[l], common, sx[l]);
        sy[l] = fma(py[l], common, sy[l]);
    }
}

// RATE: scattering-rate variant (rate_leg >= 0), a separate instantiation so
// that the propagate path keeps its register allocation.  LIST: tup is a
// ThetaList's ids (row stride n), mask / perm its masks and original indices.
// SACC: the block adds its results into a shared-memory copy of the legs'
// bands (one block of c.sinst doubles per instance) and adds that copy to
// acc once at the end.  Small meshes make the accumulator a few KB, so FP64
// atomics from every SM into it contend on a few L2 lines; in shared memory
// they stay on the SM.
template <int L, bool RATE, bool LIST, bool SACC>
__global__ void __launch_bounds__(256, LIST ? TB_MC_LIST_MIN_BLOCKS : 1) k_collision_mc(ChanDev c, const InstDev* __restrict__ insts, int n_insts,
                                                      const int32_t* __restrict__ tup, int64_t stride, int64_t n,
                                                      const uint64_t* __restrict__ mask, const int32_t* __restrict__ perm,
                                                      const double* __restrict__ f, double* __restrict__ acc,
                                                      const DPCtl* __restrict__ ctl, int rate_leg, FxAcc fx) {
    // Nothing to add when every instance is switched off or its run has
    // finished (the speculative DP45 attempts after the end of an
    // integration): leave before walking the tuples.  Uniform in the block.
    {
        bool any = false;
        for (int k = 0; k < n_insts && !any; ++k)
            any = insts[k].amp_full != 0.0 && !(ctl && ctl[insts[k].run].done);
        if (!any) return;
    }
    extern __shared__ double s_mc[];
    constexpr int R = 2 * (L - 2) + 1;
    double* s_acc = s_mc + c.nmc * R;   // SACC: [n_insts][c.sinst]
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) s_mc[i] = c.mc[i];
    if (SACC)
        for (int i = threadIdx.x; i < n_insts * c.sinst; i += blockDim.x) s_acc[i] = 0.0;
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
        AlphaMap<L> am;
        alpha_map<L>(g, Ci, am);
        const uint64_t mk0 = (LIST && valid) ? __ldg(reinterpret_cast<const unsigned long long*>(mask) + i) : 0ull;
        // functAmplitude of this tuple (fullAmplitude = amplitude * volumes * functAmplitude)
        const double tf = (c.tamp && valid) ? __ldg(c.tamp + (LIST ? int64_t(__ldg(perm + i)) : i)) : 1.0;
        for (int k = 0; k < n_insts; ++k) {
            const InstDev in = insts[k];
            if (in.amp_full == 0.0) continue;
            if (ctl && ctl[in.run].done) continue;
            if (!__any_sync(0xffffffffu, valid)) continue;
            const double ampt = in.amp_full * tf;
            double s0 = 0.0, sx[L], sy[L];
#pragma unroll
            for (int l = 0; l < L; ++l) { sx[l] = 0.0; sy[l] = 0.0; }
            if (LIST) {
                double fv[L][3];
                leg_values<L, RATE>(c, in, f, e, rate_leg, fv);
                inside_point_sums<L, RATE>(c, am, s_mc, mk0, fv, rate_leg, s0, sx, sy);
            } else {
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
                for (int m = 0; m < c.nmc; ++m) {
                    const double* qv = s_mc + m * R;
                    double al[3];
                    const bool th = alpha_theta<L>(g, Ci, am, qv, al);
                    mc_point_accumulate<L>(A, B, qv, al, th ? 1.0 : 0.0, s0, sx, sy);
                }
            }
            const double scale = valid ? 1.0 / (inv_fact_nmc * fabs(g.det)) : 0.0;
#pragma unroll
            for (int l = 0; l < L; ++l) {
                if (RATE && l != rate_leg) continue;   // uniform: the rate keeps one leg
                const double d = RATE ? -c.leg[l].dir : c.leg[l].dir;
                const int64_t key = SACC ? int64_t(k * c.sinst + c.sseg[l] + 3 * e[l]) : in.foff[l] + 3 * (int64_t)e[l];
                double* const dst = (SACC ? s_acc : acc) + key;
                if (!SACC && fx.w) {   // deterministic mode (never with SACC)
                    if (valid)
                        fx_add3(fx, key, d * ((scale * s0) * ampt), d * ((scale * sx[l]) * ampt),
                                d * ((scale * sy[l]) * ampt));
                } else if (l < L - 1 && (!SACC || l < TB_MC_SACC_SCAN_LEGS)) {
                    warp_scatter3(valid ? key : -1, dst, d * ((scale * s0) * ampt), d * ((scale * sx[l]) * ampt),
                                  d * ((scale * sy[l]) * ampt));
                } else if (valid) {
                    atomicAdd(dst + 0, d * ((scale * s0) * ampt));
                    atomicAdd(dst + 1, d * ((scale * sx[l]) * ampt));
                    atomicAdd(dst + 2, d * ((scale * sy[l]) * ampt));
                }
            }
        }
    }
    if (SACC) {
        __syncthreads();
        for (int i = threadIdx.x; i < n_insts * c.sinst; i += blockDim.x) {
            const double v = s_acc[i];
            if (v == 0.0) continue;   // adding zero changes nothing
            const int k = i / c.sinst, r = i - k * c.sinst;
            int sg = 0;
            while (sg + 1 < c.nseg && r >= c.seg_off[sg + 1]) ++sg;
            atomicAdd(acc + insts[k].foff[c.seg_leg[sg]] + (r - c.seg_off[sg]), v);
        }
    }
}

template <int L, bool RATE, bool LIST, bool SACC>
static int launch_mc(const ChanDev& c, const InstDev* insts, int n_insts, const int32_t* tup, int64_t stride,
                     int64_t n, const uint64_t* mask, const int32_t* perm, const double* f, double* acc,
                     const DPCtl* ctl, cudaStream_t s, int grid_hint, int rate_leg, const FxAcc& fx) {
    auto kern = k_collision_mc<L, RATE, LIST, SACC>;
    const int threads = 256;
    int64_t blocks = (n + threads - 1) / threads;
    size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
    if (SACC) {
        smem += sizeof(double) * size_t(n_insts) * size_t(c.sinst);
        // the shared-memory limit, set once on each device the kernel runs on
        static unsigned long long attr_devices = 0;
        int dev = 0, nsm = 148, per_sm = 1;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !((attr_devices >> dev) & 1ull)) {
            TB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(TB_MC_SACC_MAX_BYTES + sizeof(double) * 64 * 5)));
            if (dev >= 0 && dev < 64) attr_devices |= 1ull << dev;
        }
        // one wave of resident blocks: each block clears and flushes its copy once
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
        if (per_sm < 1) per_sm = 1;
        if (blocks > int64_t(nsm) * per_sm) blocks = int64_t(nsm) * per_sm;
    } else if (grid_hint > 0 && blocks > grid_hint) {
        blocks = grid_hint;
    }
    kern<<<unsigned(blocks), threads, smem, s>>>(c, insts, n_insts, tup, stride, n, mask, perm, f, acc, ctl,
                                                 RATE ? rate_leg : -1, fx);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

template <int L>
static int launch_mc_l(const ChanDev& c, const InstDev* insts, int n_insts, const int32_t* tup, int64_t stride,
                       int64_t n, const uint64_t* mask, const int32_t* perm, const double* f, double* acc,
                       const DPCtl* ctl, cudaStream_t s, int grid_hint, int rate_leg, const FxAcc& fx) {
    const bool list = mask != nullptr;
    // the shared-memory accumulator adds in FP64: not in the deterministic mode
    const bool sacc = list && !fx.w && c.sinst > 0 && c.nmc <= 64 &&
                      sizeof(double) * size_t(n_insts) * size_t(c.sinst) <= TB_MC_SACC_MAX_BYTES;
#define TB_MC_ARGS c, insts, n_insts, tup, stride, n, mask, perm, f, acc, ctl, s, grid_hint, rate_leg, fx
    if (rate_leg >= 0) {
        if (sacc) return launch_mc<L, true, true, true>(TB_MC_ARGS);
        if (list) return launch_mc<L, true, true, false>(TB_MC_ARGS);
        return launch_mc<L, true, false, false>(TB_MC_ARGS);
    }
    if (sacc) return launch_mc<L, false, true, true>(TB_MC_ARGS);
    if (list) return launch_mc<L, false, true, false>(TB_MC_ARGS);
    return launch_mc<L, false, false, false>(TB_MC_ARGS);
#undef TB_MC_ARGS
}

int launch_collision_mc(const ChanDev& c, const InstDev* insts, int n_insts, const int32_t* tup, int64_t stride,
                        int64_t n, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s, int grid_hint,
                        int rate_leg, const uint64_t* mask, const int32_t* perm, const FxAcc& fx) {
    if (n <= 0 || n_insts <= 0) return TB_OK;
    switch (c.L) {
        case 2: return launch_mc_l<2>(c, insts, n_insts, tup, stride, n, mask, perm, f, acc, ctl, s, grid_hint, rate_leg, fx);
        case 3: return launch_mc_l<3>(c, insts, n_insts, tup, stride, n, mask, perm, f, acc, ctl, s, grid_hint, rate_leg, fx);
        case 4: return launch_mc_l<4>(c, insts, n_insts, tup, stride, n, mask, perm, f, acc, ctl, s, grid_hint, rate_leg, fx);
        default: set_error("nlegs must be 2..4"); return TB_ERR_ARG;
    }
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

// ------------------------------------------------- exact accumulator flush
__global__ void __launch_bounds__(256) k_fx_flush(FxAcc fx, double* __restrict__ acc, int64_t n) {
    const bool poisoned = *fx.poison != 0u;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        unsigned long long* p = fx.w + 3 * i;
        const unsigned long long w0 = p[0], w1 = p[1], w2 = p[2];
        const bool nz = (w0 | w1 | w2) != 0ull;
        if (nz) { p[0] = 0ull; p[1] = 0ull; p[2] = 0ull; }
        if (poisoned) acc[i] = __longlong_as_double(0x7ff8000000000000ll);   // NaN
        else if (nz) acc[i] += fx_value(w0, w1, w2);
    }
}

int launch_fx_flush(const FxAcc& fx, double* acc, int64_t n, cudaStream_t s) {
    if (n <= 0 || !fx.w) return TB_OK;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_fx_flush<<<unsigned(blocks), 256, 0, s>>>(fx, acc, n);
    TB_CUDA(cudaGetLastError());
    // every thread has read the poison word once the kernel is done
    TB_CUDA(cudaMemsetAsync(fx.poison, 0, sizeof(unsigned int), s));
    return TB_OK;
}

}  // namespace tb
