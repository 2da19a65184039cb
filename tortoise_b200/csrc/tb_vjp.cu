// tb_vjp.cu -- vector-Jacobian products of the right-hand side
// F(f) = M^-1 (C(f) + V f)  (collision operator C, Vlasov drift V).
//
// No counterpart in the reference (it has no derivatives); these are the
// exact transposes of the forward kernels in tb_collision.cu, tb_tensor.cu,
// tb_drift.cu and of applyInverseMass:
//   u        = M^-T theta                      (per element)
//   grad_f  += C'(f)^T u  + V^T u
//   grad_amp[c] = <u, C_c(f)> / amplitude_c    (C_c is linear in its amplitude)
// Each leg factor of a tuple is affine in its element's 3 coefficients of f
// (ScatteringChannel.cpp:633-641), so the derivative of the product of L
// factors is the sum over legs of (other legs' factors) x (that leg's slope).
#include "tb_dp45.cuh"
#include "tb_geom.cuh"
#include "tb_mcpoint.cuh"
#include "tb_scatter.cuh"
#include "tb_tensor.cuh"
#include "tb_vjp.cuh"

namespace tb {

template <int L> struct VDim {
    static constexpr int K = (L == 2) ? 9 : (L == 3) ? 27 : 81;
    static constexpr int KM = K / 3;
    static constexpr int NMOM = K * (1 + L);
};


// ---------------------------------------------------------------- M^-T
__global__ void k_minv_t(ElemDev ed, const double* __restrict__ theta, double* __restrict__ u) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    const double t0 = theta[o], t1 = theta[o + 1], t2 = theta[o + 2];
#pragma unroll
    for (int i = 0; i < 3; ++i) u[o + i] = bd.mesh.Minv[i][0] * t0 + bd.mesh.Minv[i][1] * t1 + bd.mesh.Minv[i][2] * t2;
}

// Zero the constrained bands (the projection of MaterialStatus::applyConstraints).
__global__ void k_project(ElemDev ed, double* __restrict__ v) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    if (!bd.constrained) return;
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    v[o] = 0.0; v[o + 1] = 0.0; v[o + 2] = 0.0;
}

int launch_minv_t(const ElemDev& ed, const double* theta, double* u, cudaStream_t s) {
    k_minv_t<<<ed.nblk, 256, 0, s>>>(ed, theta, u);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

int launch_project(const ElemDev& ed, double* v, cudaStream_t s) {
    k_project<<<ed.nblk, 256, 0, s>>>(ed, v);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// --------------------------------------------- collision VJP, Monte-Carlo
// LIST: tup / stride / n describe a ThetaList (tb_theta.cuh) and every tuple
// visits only the set bits of its mask, the points whose Theta is 1.
template <int L, bool LIST>
__global__ void __launch_bounds__(128) k_vjp_mc(ChanDev c, const InstDev* __restrict__ insts, int n_insts,
                                                const int32_t* __restrict__ tup, int64_t stride, int64_t n,
                                                const uint64_t* __restrict__ mask, const int32_t* __restrict__ perm,
                                                const double* __restrict__ f, const double* __restrict__ u,
                                                double* __restrict__ grad_f, double* __restrict__ grad_amp, FxAcc fx,
                                                FxAcc fx_amp) {
    extern __shared__ double s_mc[];
    constexpr int R = 2 * (L - 2) + 1;
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) s_mc[i] = c.mc[i];
    __syncthreads();
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool valid = i < n;
        int e[L];
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = valid ? __ldg(tup + l * stride + i) : 0;
        const int uu = valid ? __ldg(tup + L * stride + i) : 0;
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, uu, g);
        if (!(fabs(g.det) >= c.min_det)) valid = false;
        double Ci[3][3];
        dc_inverse<L>(g, Ci);
        const double scale = valid ? 1.0 / (c.fact * double(c.nmc) * fabs(g.det)) : 0.0;
        // functAmplitude of the tuple
        const double tf = (c.tamp && valid) ? __ldg(c.tamp + (LIST ? int64_t(__ldg(perm + i)) : i)) : 1.0;
        const uint64_t mk0 = (LIST && valid) ? __ldg(reinterpret_cast<const unsigned long long*>(mask) + i) : 0ull;
        for (int k = 0; k < n_insts; ++k) {
            const InstDev in = insts[k];
            double gA[L][3], gB[L][3], gamp, sa[L], sb[L];
            vjp_point_sums<L, LIST>(c, in, f, u, e, g, Ci, s_mc, mk0, valid, gA, gB, gamp, sa, sb);
            if (valid) {
                const double sc = scale * (in.amp_full * tf);
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    const int64_t key = in.foff[l] + 3 * (int64_t)e[l];
                    double* o = grad_f + key;
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const double g = __dmul_rn(sc, fma(sb[l], gB[l][j], __dmul_rn(sa[l], gA[l][j])));
                        if (fx.w) fx_add(fx, key + j, g);
                        else atomicAdd(o + j, g);
                    }
                }
            }
            block_atomic_sum(valid ? scale * (c.amp_vol * tf) * gamp : 0.0, grad_amp + k, fx_amp, k);
        }
    }
}

// Gradient of  sum_J w[J] prod_l X[l][J_l]  with respect to every X[m][j]
// (g[m][j] = sum over J with J_m = j of w[J] prod_{l != m} X[l][J_l]) and the
// sum itself, by contracting w from the last leg backwards (suffixes S_m over
// legs 0..m) and multiplying prefixes P_m over legs 0..m-1: 81 FMAs per form
// for three legs instead of the 324 products of the term-by-term expansion.
// J is leg-0-most-significant, so the last leg is the fastest digit.
template <int L>
__device__ __forceinline__ void leg_grads(const double* __restrict__ w, const double (&X)[L][3], double (&g)[L][3],
                                          double& total) {
    constexpr int K = VDim<L>::K;
    double S[L][K];   // S[m]: 3^(m+1) values (S[L-1] = w)
    double P[L][K];   // P[m]: 3^m values
#pragma unroll
    for (int i = 0; i < K; ++i) S[L - 1][i] = w[i];
#pragma unroll
    for (int m = L - 2; m >= 0; --m) {
        int sz = 3;
#pragma unroll
        for (int q = 0; q < m; ++q) sz *= 3;
#pragma unroll
        for (int i = 0; i < sz; ++i)
            S[m][i] = S[m + 1][3 * i] * X[m + 1][0] + S[m + 1][3 * i + 1] * X[m + 1][1] + S[m + 1][3 * i + 2] * X[m + 1][2];
    }
    P[0][0] = 1.0;
#pragma unroll
    for (int m = 1; m < L; ++m) {
        int sz = 1;
#pragma unroll
        for (int q = 0; q < m - 1; ++q) sz *= 3;
#pragma unroll
        for (int i = 0; i < sz; ++i)
#pragma unroll
            for (int t = 0; t < 3; ++t) P[m][3 * i + t] = (m == 1) ? X[0][t] : P[m - 1][i] * X[m - 1][t];
    }
#pragma unroll
    for (int m = 0; m < L; ++m) {
        int sz = 1;
#pragma unroll
        for (int q = 0; q < m; ++q) sz *= 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
#pragma unroll
            for (int i = 0; i < sz; ++i) acc = fma(P[m][i], S[m][3 * i + j], acc);
            g[m][j] = acc;
        }
    }
    total = X[0][0] * S[0][0] + X[0][1] * S[0][1] + X[0][2] * S[0][2];
}

// --------------------------------------------- collision VJP, moment tensor
template <int L, int KIND>
__global__ void __launch_bounds__(128) k_vjp_tensor(ChanDev c, const InstDev* __restrict__ insts, int n_insts,
                                                    const void* __restrict__ mom, int TT, const int32_t* __restrict__ tup,
                                                    int64_t stride, int64_t n, const double* __restrict__ f,
                                                    const double* __restrict__ u, double* __restrict__ grad_f,
                                                    double* __restrict__ grad_amp, FxAcc fx, FxAcc fx_amp) {
    constexpr int K = VDim<L>::K, KM = VDim<L>::KM, NMOM = VDim<L>::NMOM;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool valid = i < n;
        int e[L];
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = valid ? __ldg(tup + l * stride + i) : 0;
        // moment j of tuple i: tile-major rows of TT tuples (FP64, FP32, or
        // the upper 40 / 48 bits of FP64 as a word row plus packed byte /
        // half-word rows)
        constexpr int NB = (KIND == TK_F40) ? (NMOM + 3) / 4 : (KIND == TK_F48) ? (NMOM + 1) / 2 : 0;
        constexpr int ROWB = (KIND == TK_F64) ? 8 : 4;
        const unsigned char* tb = static_cast<const unsigned char*>(mom) + (i / TT) * (int64_t)(NMOM + NB) * TT * ROWB;
        const int64_t pos = i % TT;
        auto M = [&](int j) -> double {
            if constexpr (KIND == TK_F64) {
                return reinterpret_cast<const double*>(tb)[(int64_t)j * TT + pos];
            } else if constexpr (KIND == TK_F32) {
                return double(reinterpret_cast<const float*>(tb)[(int64_t)j * TT + pos]);
            } else if constexpr (KIND == TK_F48) {
                const uint32_t* w = reinterpret_cast<const uint32_t*>(tb);
                const uint32_t lw = w[(int64_t)(NMOM + (j >> 1)) * TT + pos];
                return __hiloint2double(int(w[(int64_t)j * TT + pos]), int((j & 1) ? (lw & 0xffff0000u) : (lw << 16)));
            } else {
                const uint32_t* w = reinterpret_cast<const uint32_t*>(tb);
                const uint32_t lw = w[(int64_t)(NMOM + (j >> 2)) * TT + pos];
                return __hiloint2double(int(w[(int64_t)j * TT + pos]),
                                        int(__byte_perm(lw, 0u, 0x0444u | (uint32_t(j & 3) << 12))));
            }
        };
        for (int k = 0; k < n_insts; ++k) {
            const InstDev in = insts[k];
            double A[L][3], B[L][3], sa[L], sb[L];
            leg_forms<L>(c, in, f, e, A, B, sa, sb);
            // w[J] = sum_{lam, beta} dir_lam u[e_lam, beta] W[lam, beta][J]
            double w[K];
#pragma unroll
            for (int j = 0; j < K; ++j) w[j] = 0.0;
            if (valid) {
                double usum0 = 0.0;
#pragma unroll
                for (int lam = 0; lam < L; ++lam) usum0 += c.leg[lam].dir * __ldg(u + in.foff[lam] + 3 * (int64_t)e[lam]);
#pragma unroll
                for (int j = 0; j < K; ++j) w[j] = usum0 * M(j);
#pragma unroll
                for (int lam = 0; lam < L; ++lam) {
                    const double d = c.leg[lam].dir;
                    const double u1 = d * __ldg(u + in.foff[lam] + 3 * (int64_t)e[lam] + 1);
                    const double u2 = d * __ldg(u + in.foff[lam] + 3 * (int64_t)e[lam] + 2);
                    int sstep = 1;
#pragma unroll
                    for (int l = L - 1; l > lam; --l) sstep *= 3;
#pragma unroll
                    for (int km = 0; km < KM; ++km) {
                        const int hi = km / sstep, lo = km % sstep;
                        const int j0 = hi * 3 * sstep + lo, j1 = j0 + sstep, j2 = j0 + 2 * sstep;
                        const double qxx = M(K + (lam * 3 + 0) * KM + km);
                        const double qxy = M(K + (lam * 3 + 1) * KM + km);
                        const double qyy = M(K + (lam * 3 + 2) * KM + km);
                        const double s1 = M(j1);
                        const double s2 = M(j2);
                        w[j0] += u1 * s1 + u2 * s2;
                        w[j1] += u1 * qxx + u2 * qxy;
                        w[j2] += u1 * qxy + u2 * qyy;
                    }
                }
            }
            // d/dA[m][j] of sum_J w[J] prod_l A[l][J_l]; the same for B
            double gA[L][3], gB[L][3], ta, tb2;
            leg_grads<L>(w, A, gA, ta);
            leg_grads<L>(w, B, gB, tb2);
            const double gamp = ta + tb2;
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const int64_t key = in.foff[l] + 3 * (int64_t)e[l];
                const double g0 = in.amplitude * (sa[l] * gA[l][0] + sb[l] * gB[l][0]);
                const double g1 = in.amplitude * (sa[l] * gA[l][1] + sb[l] * gB[l][1]);
                const double g2 = in.amplitude * (sa[l] * gA[l][2] + sb[l] * gB[l][2]);
                if (fx.w) {   // deterministic mode: exact adds, lane by lane
                    if (valid) fx_add3(fx, key, g0, g1, g2);
                } else if (l < L - 1) {
                    warp_scatter3(valid ? key : -1, grad_f + (valid ? key : 0), g0, g1, g2);
                } else if (valid) {
                    atomicAdd(grad_f + key, g0);
                    atomicAdd(grad_f + key + 1, g1);
                    atomicAdd(grad_f + key + 2, g2);
                }
            }
            block_atomic_sum(valid ? gamp : 0.0, grad_amp + k, fx_amp, k);
        }
    }
}

int launch_collision_vjp(const ChanDev& c, const InstDev* insts, int n_insts, int layout, const MomentTensor& T,
                         const int32_t* tup, int64_t stride, int64_t n, const double* f, const double* u,
                         double* grad_f, double* grad_amp, cudaStream_t s, const uint64_t* mask,
                         const int32_t* perm, const FxAcc& fx, const FxAcc& fx_amp) {
    if (n <= 0 || n_insts <= 0) return TB_OK;
    const int threads = 128;
    int64_t blocks = (n + threads - 1) / threads;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (layout == TB_LAYOUT_MC64) {
        const size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
#define TB_VJP_MC(LL, LS) k_vjp_mc<LL, LS><<<unsigned(blocks), threads, smem, s>>>(c, insts, n_insts, tup, stride, n, \
                                                                                 mask, perm, f, u, grad_f, grad_amp, \
                                                                                 fx, fx_amp)
        const bool list = mask != nullptr;
        switch (c.L) {
            case 2: if (list) TB_VJP_MC(2, true); else TB_VJP_MC(2, false); break;
            case 3: if (list) TB_VJP_MC(3, true); else TB_VJP_MC(3, false); break;
            default: if (list) TB_VJP_MC(4, true); else TB_VJP_MC(4, false); break;
        }
#undef TB_VJP_MC
    } else {
        const int TT = tile_tuples(c.L, T.kind);
#define TB_VJP_T(LL, KK) k_vjp_tensor<LL, KK><<<unsigned(blocks), threads, 0, s>>>(c, insts, n_insts, T.d, TT, tup, \
                                                                                 stride, n, f, u, grad_f, grad_amp, \
                                                                                 fx, fx_amp)
        switch (c.L * 4 + T.kind) {
            case 8: TB_VJP_T(2, TK_F64); break;
            case 9: TB_VJP_T(2, TK_F32); break;
            case 10: TB_VJP_T(2, TK_F40); break;
            case 11: TB_VJP_T(2, TK_F48); break;
            case 12: TB_VJP_T(3, TK_F64); break;
            case 13: TB_VJP_T(3, TK_F32); break;
            case 14: TB_VJP_T(3, TK_F40); break;
            case 15: TB_VJP_T(3, TK_F48); break;
            case 16: TB_VJP_T(4, TK_F64); break;
            case 17: TB_VJP_T(4, TK_F32); break;
            case 18: TB_VJP_T(4, TK_F40); break;
            default: TB_VJP_T(4, TK_F48); break;
        }
#undef TB_VJP_T
    }
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// ---------------------------------------------------------- drift VJP
// Transpose of k_drift: the volume term couples an element to itself, the
// upwind surface term couples the element to the face neighbour it reads.
__device__ __forceinline__ int adj_el(int nx, int nt, int e, int face) {
    if (e & 1) {
        if (face == 0) return (e + 2 * nx - 1 + nt) % nt;
        if (face == 1) return e - 1;
        return ((e - 1) % (2 * nx) == 0) ? e + 2 * nx - 3 : e - 3;
    } else {
        if (face == 0) return ((e + 2) % (2 * nx) == 0) ? e - 2 * nx + 3 : e + 3;
        if (face == 1) return e + 1;
        return (e - 2 * nx + 1 + nt) % nt;
    }
}

__device__ __forceinline__ void normal_of(const MeshDev& m, int e, int face, double n[2]) {
    const double d00 = m.dG[0][0], d01 = m.dG[0][1], d10 = m.dG[1][0], d11 = m.dG[1][1];
    double v0, v1, sgn;
    if (e & 1) {
        if (face == 0) { v0 = d10; v1 = -d00; sgn = (v0 * d01 + v1 * d11 > 0.) ? 1. : -1.; }
        else if (face == 1) { v0 = d11 + d10; v1 = -d01 - d00; sgn = (v0 * d00 + v1 * d10 > 0.) ? 1. : -1.; }
        else { v0 = d11; v1 = -d01; sgn = (v0 * d00 + v1 * d10 > 0.) ? -1. : 1.; }
    } else {
        if (face == 0) { v0 = d11; v1 = -d01; sgn = (v0 * d00 + v1 * d10 > 0.) ? 1. : -1.; }
        else if (face == 1) { v0 = d11 + d10; v1 = -d01 - d00; sgn = (v0 * d00 + v1 * d10 > 0.) ? -1. : 1.; }
        else { v0 = d10; v1 = -d00; sgn = (v0 * d01 + v1 * d11 > 0.) ? -1. : 1.; }
    }
    const double nn = sqrt(v0 * v0 + v1 * v1);
    n[0] = v0 / nn * sgn;
    n[1] = v1 / nn * sgn;
}

__device__ __forceinline__ double area_of(const MeshDev& m, int e, int face) {
    const double d00 = m.dG[0][0], d01 = m.dG[0][1], d10 = m.dG[1][0], d11 = m.dG[1][1];
    const int ff = (e & 1) ? face : 2 - face;
    if (ff == 0) return sqrt(d00 * d00 + d10 * d10);
    if (ff == 1) return sqrt((d00 + d01) * (d00 + d01) + (d10 + d11) * (d10 + d11));
    return sqrt(d01 * d01 + d11 * d11);
}

__device__ __forceinline__ void side_pt(int side, int q, double& x, double& y) {
    const double g = q ? TB_GP1_1 : TB_GP1_0;
    if (side == 0) { x = 1. - g; y = g; }
    else if (side == 1) { x = 0.; y = g; }
    else { x = g; y = 0.; }
}

__global__ void __launch_bounds__(256) k_drift_vjp(ElemDev ed, const double* __restrict__ u, double* __restrict__ grad_f,
                                                   FxAcc fx) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const double vel0 = bd.vel[0], vel1 = bd.vel[1];
    if (vel0 == 0.0 && vel1 == 0.0) return;
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const MeshDev m = bd.mesh;
    const int nt = m.ne;
    const double* ub = u + bd.off;
    double* gb = grad_f + bd.off;
    const double ue[3] = {ub[3 * e], ub[3 * e + 1], ub[3 * e + 2]};
    // volume: out[e,b] += vol * (v0 dx_b + v1 dy_b) * sum_q w_q f_e(q)
    const int s = e / 2, par = e & 1;
    const double sx = double(s % m.nx), sy = double(s / m.nx);
    double vx[3], vy[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double ox = (k == 0) ? 0.0 : (par ? (k == 1 ? 0.0 : 1.0) : 1.0);
        const double oy = (k == 0) ? 0.0 : (par ? 1.0 : (k == 1 ? 0.0 : 1.0));
        const double px = sx + ox, py = sy + oy;
        vx[k] = m.rel_origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
        vy[k] = m.rel_origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
    }
    const double v0X = vx[0], v0Y = vy[0], v1X = vx[1], v1Y = vy[1], v2X = vx[2], v2Y = vy[2];
    const double denx = v0Y * (v1X - v2X) + v1Y * (v2X - v0X) + v2Y * (v0X - v1X);
    const double deny = v0X * (v1Y - v2Y) + v1X * (v2Y - v0Y) + v2X * (v0Y - v1Y);
    const double dx[3] = {0.0, (v0Y - v2Y) / denx, -(v0Y - v1Y) / denx};
    const double dy[3] = {0.0, (v0X - v2X) / deny, -(v0X - v1X) / deny};
    double coef = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) coef += ue[b] * (m.vol * vel0 * dx[b] + m.vol * vel1 * dy[b]);
    // d/dc_j of sum_q w f(q) with f(q) = c0 + c1 x_q + c2 y_q
    const double w = TB_GW2, ga = TB_GP2_A, gbb = TB_GP2_B;
    auto add = [&](int64_t el, int j, double v) {
        if (fx.w) fx_add(fx, bd.off + 3 * el + j, v);
        else atomicAdd(gb + 3 * el + j, v);
    };
    add(e, 0, coef * (3.0 * w));
    add(e, 1, coef * (w * (ga + gbb + ga)));
    add(e, 2, coef * (w * (ga + ga + gbb)));
    // surface: out[e,b] -= s * area * sum_q 0.5 phi_b(pt(side,q)) f_ei(pt(si,q))
#pragma unroll
    for (int side = 0; side < 3; ++side) {
        double n[2];
        normal_of(m, e, side, n);
        const double sv = vel0 * n[0] + vel1 * n[1];
        int ei, si;
        if (sv > 0.) { ei = e; si = side; }
        else { ei = adj_el(m.nx, nt, e, side); si = 2 - side; }
        const double area = area_of(m, e, side);
        double g3[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            double bx, by, xi, yi;
            side_pt(side, q, bx, by);
            side_pt(si, q, xi, yi);
            const double phiu = ue[0] + ue[1] * bx + ue[2] * by;
            const double wq = -sv * area * 0.5 * phiu;
            g3[0] += wq; g3[1] += wq * xi; g3[2] += wq * yi;
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) add(ei, j, g3[j]);
    }
}

int launch_drift_vjp(const ElemDev& ed, const double* u, double* grad_f, cudaStream_t s, const FxAcc& fx) {
    k_drift_vjp<<<ed.nblk, 256, 0, s>>>(ed, u, grad_f, fx);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

}  // namespace tb
