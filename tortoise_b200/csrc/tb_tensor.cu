// tb_tensor.cu -- the collision operator as a precomputed sparse tensor.
//
// The reference declares a precomputed scattering matrix (scatteringMatrix,
// precalculate(), propagatePrecalculatedSingle in include/Physics/Scattering/
// ScatteringChannel.hpp:90,129,176) but never implements it; every RHS
// evaluation re-runs the Monte-Carlo quadrature of scatteringIntegrationTypeB
// (IntegratorCore.hpp:260-357).  Because each leg's gain/loss factor is an
// affine function of its element's 3 P1 coefficients, the quadrature factors
// exactly into f-independent moments of the delta-constrained MC points:
//
//   result[lam][beta] = amp * sum_J W[lam,beta][J] * (prod_l a_{l,J_l} + prod_l b_{l,J_l})
//   W[lam,beta][J]    = norm * sum_m Theta_m phi_beta(p_lam,m) prod_l phi_{J_l}(p_l,m)
//
// with phi = (1, x, y) on the reference triangle.  Only 3^L (1+L) of the
// 3L*3^L entries of W are distinct:
//   S0[J]            (beta = 0, identical for every lam)           3^L
//   Q_lam[t][J_-lam] (t = xx, xy, yy: the degree-2 monomial of leg lam)   3L * 3^(L-1)
// which is 108 numbers per 3-leg tuple and 405 per 4-leg tuple.
//
// Storage is tile-major: a tile of TT tuples is one contiguous block
// [nmom][TT], so the contraction kernel streams whole tiles into shared memory
// with one 1-D bulk TMA copy (cp.async.bulk + mbarrier, double buffered) and
// each thread reads its tuple's moments bank-conflict free.  Three storage
// kinds:
//   TK_F64    FP64 moments;
//   TK_F32    FP32 moments (2^-24 relative rounding each), half the bytes;
//   TK_F40    the upper 40 bits of each FP64 moment (sign, exponent and 28
//             mantissa bits, rounded to nearest: 2^-29 relative), 5 bytes per
//             moment: a row of the upper 32-bit words, then rows that pack
//             the next byte of four consecutive moments into one word.  A
//             moment is rebuilt as an FP64 register pair (upper word, byte
//             << 24) with one byte permute: no conversion instruction.
//   TK_F48    the upper 48 bits (36 mantissa bits: 2^-37 relative), 6 bytes
//             per moment: the row of upper words, then rows that pack the
//             next 16 bits of two consecutive moments into one word.
// Products and accumulation are FP64 for every kind; the gain-minus-loss
// vector v = ka + kb is formed in FP64 from f.
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "tb_dp45.cuh"
#include "tb_geom.cuh"
#include "tb_scatter.cuh"
#include "tb_tensor.cuh"

namespace tb {

template <int L> struct TDim {
    static constexpr int K = (L == 2) ? 9 : (L == 3) ? 27 : 81;     // 3^L
    static constexpr int KM = K / 3;                                // 3^(L-1)
    static constexpr int NMOM = K * (1 + L);
};

template <int L, int KIND> struct TTile {
    // tuples per tile: keeps one stage at <= ~56 KB of shared memory
    static constexpr int TT = (L == 4)                                          ? 32
                              : (KIND == TK_F32)                                ? 128
                              : ((KIND == TK_F40 || KIND == TK_F48) && L == 2) ? 128
                                                                                : 64;
};

static int nmom_of(int L) { return (L == 2 ? 9 : L == 3 ? 27 : 81) * (1 + L); }

int tile_tuples(int L, int kind) {
    if (L == 4) return 32;
    if (kind == TK_F32 || ((kind == TK_F40 || kind == TK_F48) && L == 2)) return 128;
    return 64;
}

// bytes of one tuple's moments in a tile
static int64_t tuple_bytes(int L, int kind) {
    const int64_t nm = nmom_of(L);
    return kind == TK_F64 ? 8 * nm : kind == TK_F32 ? 4 * nm : kind == TK_F48 ? 4 * (nm + (nm + 1) / 2)
                                                                              : 4 * (nm + (nm + 3) / 4);
}

int64_t tensor_bytes(int L, int kind, int64_t n) {
    const int64_t TT = tile_tuples(L, kind);
    const int64_t ntiles = (n + TT - 1) / TT;
    return ntiles * TT * tuple_bytes(L, kind);
}

void MomentTensor::release() {
    if (d) cudaFree(d);
    if (fT) cudaFree(fT);
    if (accT) cudaFree(accT);
    if (accTx) cudaFree(accTx);
    d = nullptr;
    fT = accT = nullptr;
    accTx = nullptr;
    n = ntiles = 0;
    runs = np = runs_distinct = 0;
}

// ------------------------------------------------------------ precompute
// One warp per tuple; every lane recomputes the MC point (cheap) and owns a
// strided subset of the moments.
template <int L, int KIND>
__global__ void __launch_bounds__(256) k_build_moments(ChanDev c, const int32_t* __restrict__ tup, int64_t stride,
                                                       int64_t n, void* __restrict__ out, int TT) {
    extern __shared__ double s_mc[];
    constexpr int R = 2 * (L - 2) + 1;
    constexpr int K = TDim<L>::K, KM = TDim<L>::KM, NMOM = TDim<L>::NMOM;
    constexpr int PER = (NMOM + 31) / 32;
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) s_mc[i] = c.mc[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // decode the owned moments: factor selector per leg (0:1, 1:x, 2:y, 3:xx, 4:xy, 5:yy)
    int sel[PER][L];
    bool own[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int k = lane + 32 * q;
        own[q] = k < NMOM;
        int J[L];
        if (k < K) {
            int r = k;
#pragma unroll
            for (int l = L - 1; l >= 0; --l) { J[l] = r % 3; r /= 3; }
#pragma unroll
            for (int l = 0; l < L; ++l) sel[q][l] = J[l];
        } else {
            const int kk = own[q] ? k - K : 0;
            const int lam = kk / (3 * KM);
            const int rr = kk % (3 * KM);
            const int t = rr / KM;
            int jm = rr % KM;
#pragma unroll
            for (int l = L - 1; l >= 0; --l) {
                if (l == lam) continue;
                sel[q][l] = jm % 3;
                jm /= 3;
            }
#pragma unroll
            for (int l = 0; l < L; ++l)
                if (l == lam) sel[q][l] = 3 + t;
        }
    }
    for (int64_t i = warp; i < n; i += nwarps) {
        int e[L];
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = __ldg(tup + l * stride + i);
        const int u = __ldg(tup + L * stride + i);
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, u, g);
        double acc[PER];
#pragma unroll
        for (int q = 0; q < PER; ++q) acc[q] = 0.0;
        double norm = 0.0;
        if (fabs(g.det) >= c.min_det) {
            double Ci[3][3];
            dc_inverse<L>(g, Ci);
            for (int m = 0; m < c.nmc; ++m) {
                double qv[R];
#pragma unroll
                for (int j = 0; j < R; ++j) qv[j] = s_mc[m * R + j];
                // exact (unfused) evaluation: Theta decisions identical to the reference order
                double al[3];
                exact_alpha<L>(g, Ci, qv, al);
                const double kp0 = qv[R - 1];
                if (!theta_of(kp0, al)) continue;   // warp-uniform: every lane evaluates the same point
                double px[L], py[L];
#pragma unroll
                for (int l = 0; l < L - 2; ++l) { px[l] = qv[2 * l]; py[l] = qv[2 * l + 1]; }
                px[L - 2] = kp0; py[L - 2] = al[0];
                px[L - 1] = al[1]; py[L - 1] = al[2];
#pragma unroll
                for (int q = 0; q < PER; ++q) {
                    double v = 1.0;
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int s = sel[q][l];
                        const double f = (s == 0) ? 1.0 : (s == 1) ? px[l] : (s == 2) ? py[l]
                                       : (s == 3) ? px[l] * px[l] : (s == 4) ? px[l] * py[l] : py[l] * py[l];
                        v *= f;
                    }
                    acc[q] += v;
                }
            }
            norm = c.amp_vol / (c.fact * double(c.nmc) * fabs(g.det));
            if (c.tamp) norm *= __ldg(c.tamp + i);   // functAmplitude folded into the moments
        }
        const int64_t tile = i / TT, pos = i % TT;
        if (KIND == TK_F64) {
            double* base = static_cast<double*>(out) + tile * (int64_t)NMOM * TT + pos;
#pragma unroll
            for (int q = 0; q < PER; ++q)
                if (own[q]) base[(int64_t)(lane + 32 * q) * TT] = acc[q] * norm;
        } else if (KIND == TK_F32) {
            float* base = static_cast<float*>(out) + tile * (int64_t)NMOM * TT + pos;
#pragma unroll
            for (int q = 0; q < PER; ++q)
                if (own[q]) base[(int64_t)(lane + 32 * q) * TT] = float(acc[q] * norm);
        } else if (KIND == TK_F48) {
            // upper 48 bits of the FP64 pattern, rounded to nearest on bit 15
            constexpr int NH = (NMOM + 1) / 2;   // rows of packed 16-bit halves
            uint32_t* hi = static_cast<uint32_t*>(out) + tile * (int64_t)(NMOM + NH) * TT;
            uint16_t* lo = reinterpret_cast<uint16_t*>(hi + (int64_t)NMOM * TT);
#pragma unroll
            for (int q = 0; q < PER; ++q)
                if (own[q]) {
                    const int k = lane + 32 * q;
                    const unsigned long long b = (unsigned long long)__double_as_longlong(acc[q] * norm) + 0x8000ull;
                    hi[(int64_t)k * TT + pos] = uint32_t(b >> 32);
                    lo[2 * ((int64_t)(k >> 1) * TT + pos) + (k & 1)] = uint16_t(b >> 16);
                }
        } else {
            // upper 40 bits of the FP64 pattern, rounded to nearest on bit 23
            constexpr int NB = (NMOM + 3) / 4;   // rows of packed bytes
            uint32_t* hi = static_cast<uint32_t*>(out) + tile * (int64_t)(NMOM + NB) * TT;
            uint8_t* lo = reinterpret_cast<uint8_t*>(hi + (int64_t)NMOM * TT);
#pragma unroll
            for (int q = 0; q < PER; ++q)
                if (own[q]) {
                    const int k = lane + 32 * q;
                    const unsigned long long b = (unsigned long long)__double_as_longlong(acc[q] * norm) + 0x800000ull;
                    hi[(int64_t)k * TT + pos] = uint32_t(b >> 32);
                    lo[4 * ((int64_t)(k >> 2) * TT + pos) + (k & 3)] = uint8_t(b >> 24);
                }
        }
    }
}

// ------------------------------------------------------------ contraction
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx_arrive(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false when the spin limit is
// reached (the caller records an error and abandons the tile).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = (1 << 22)) {
    for (int it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Moment j of this thread's tuple in a staged tile, as FP64.
template <int KIND, int NMOM, int TT>
__device__ __forceinline__ double tile_moment(const unsigned char* __restrict__ tile, int tid, int j) {
    if constexpr (KIND == TK_F64) {
        return reinterpret_cast<const double*>(tile)[j * TT + tid];
    } else if constexpr (KIND == TK_F32) {
        return double(reinterpret_cast<const float*>(tile)[j * TT + tid]);
    } else if constexpr (KIND == TK_F48) {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(tile);
        const uint32_t hi = w[j * TT + tid];
        const uint32_t lw = w[(NMOM + (j >> 1)) * TT + tid];
        // half j % 2 of lw into the top half of the low word, zeros below
        const uint32_t lo = (j & 1) ? (lw & 0xffff0000u) : (lw << 16);
        return __hiloint2double(int(hi), int(lo));
    } else {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(tile);
        const uint32_t hi = w[j * TT + tid];
        const uint32_t lw = w[(NMOM + (j >> 2)) * TT + tid];
        // byte j % 4 of lw into the top byte of the low word, zeros below
        const uint32_t lo = __byte_perm(lw, 0u, 0x0444u | (uint32_t(j & 3) << 12));
        return __hiloint2double(int(hi), int(lo));
    }
}

// Contraction of one tuple (this thread's) for NI = 1 or 2 instances of
// the channel; every moment is read from shared memory once and used by all
// NI instances.  Results are scattered into acc (legs 0 .. L-2 through the
// warp-segmented reduction, so all 32 lanes must call this together).
template <int L, int KIND, int TT, int NI, bool RATE>
__device__ __forceinline__ void contract_tuple(const ChanDev& c, const InstDev (&in)[NI], const int (&e)[L], bool valid,
                                               const unsigned char* __restrict__ tile, int tid,
                                               const double* __restrict__ f, double* __restrict__ acc, int rate_leg,
                                               const FxAcc& fx) {
    constexpr int K = TDim<L>::K, KM = TDim<L>::KM, NMOM = TDim<L>::NMOM;
    auto M = [&](int j) { return tile_moment<KIND, NMOM, TT>(tile, tid, j); };
    // v = kron(A) + kron(B) per instance, leg 0 most significant; gain (B) /
    // loss (A) forms of ScatteringChannel.cpp:633-641
    double v[NI][K];
#pragma unroll
    for (int q = 0; q < NI; ++q) {
        double A[L][3], B[L][3];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const LegDev& lg = c.leg[l];
            const double* fe = f + in[q].foff[l] + 3 * (int64_t)e[l];
            const double f0 = __ldg(fe), f1 = __ldg(fe + 1), f2 = __ldg(fe + 2);
            A[l][0] = fma(lg.fa, f0, lg.fa0);
            A[l][1] = lg.fa * f1;
            A[l][2] = lg.fa * f2;
            B[l][0] = fma(lg.fb, f0, lg.fb0);
            B[l][1] = lg.fb * f1;
            B[l][2] = lg.fb * f2;
            if (RATE && l == rate_leg) {
                // scattering rate of this leg: constant in / out unit forms
                // (ScatteringChannel.cpp:562-564): (+-1) ca and cb, i.e. 2 fa, 2 fb
                A[l][0] = 2.0 * lg.fa; A[l][1] = 0.0; A[l][2] = 0.0;
                B[l][0] = 2.0 * lg.fb; B[l][1] = 0.0; B[l][2] = 0.0;
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            int r = j;
            double pa = 1.0, pb = 1.0;
#pragma unroll
            for (int l = L - 1; l >= 0; --l) {
                const int Jl = r % 3;
                r /= 3;
                pa *= A[l][Jl];
                pb *= B[l][Jl];
            }
            v[q][j] = pa + pb;
        }
    }
    // the constant mode as three interleaved FMA chains, summed (a + b) + c:
    // the same arithmetic as contract_run, so that every schedule gives each
    // tuple the same values
    double r0[NI];
#pragma unroll
    for (int q = 0; q < NI; ++q) {
        double ra = 0.0, rb = 0.0, rc = 0.0;
#pragma unroll
        for (int j = 0; j < K; j += 3) {
            ra = fma(M(j), v[q][j], ra);
            rb = fma(M(j + 1), v[q][j + 1], rb);
            rc = fma(M(j + 2), v[q][j + 2], rc);
        }
        r0[q] = (ra + rb) + rc;
    }
#pragma unroll
    for (int lam = 0; lam < L; ++lam) {
        if (RATE && lam != rate_leg) continue;   // uniform: the rate keeps one leg
        int sstep = 1;
#pragma unroll
        for (int l = L - 1; l > lam; --l) sstep *= 3;
        double r1[NI], r2[NI];
#pragma unroll
        for (int q = 0; q < NI; ++q) { r1[q] = 0.0; r2[q] = 0.0; }
#pragma unroll
        for (int km = 0; km < KM; ++km) {
            // J with J_lam = 0 whose other legs enumerate km in leg order
            const int hi = km / sstep, lo = km % sstep;
            const int j0 = hi * 3 * sstep + lo;
            const int j1 = j0 + sstep, j2 = j0 + 2 * sstep;
            const int qa = K + (lam * 3 + 0) * KM + km;
            const double qxx = M(qa), qxy = M(qa + KM), qyy = M(qa + 2 * KM);
            const double s1 = M(j1), s2 = M(j2);
#pragma unroll
            for (int q = 0; q < NI; ++q) {
                r1[q] = fma(s1, v[q][j0], r1[q]);
                r1[q] = fma(qxx, v[q][j1], r1[q]);
                r1[q] = fma(qxy, v[q][j2], r1[q]);
                r2[q] = fma(s2, v[q][j0], r2[q]);
                r2[q] = fma(qxy, v[q][j1], r2[q]);
                r2[q] = fma(qyy, v[q][j2], r2[q]);
            }
        }
        const double d = RATE ? -c.leg[lam].dir : c.leg[lam].dir;
#pragma unroll
        for (int q = 0; q < NI; ++q) {
            const double amp = in[q].amplitude;
            const int64_t key = in[q].foff[lam] + 3 * (int64_t)e[lam];
            if (fx.w) {   // deterministic mode: exact adds, lane by lane
                if (valid) fx_add3(fx, key, d * (r0[q] * amp), d * (r1[q] * amp), d * (r2[q] * amp));
            } else if (lam < L - 1) {
                warp_scatter3(valid ? key : -1, acc + key, d * (r0[q] * amp), d * (r1[q] * amp), d * (r2[q] * amp));
            } else if (valid) {
                double* o = acc + key;
                atomicAdd(o + 0, d * (r0[q] * amp));
                atomicAdd(o + 1, d * (r1[q] * amp));
                atomicAdd(o + 2, d * (r2[q] * amp));
            }
        }
    }
}

// bytes of one tuple's moments (compile-time twin of tuple_bytes)
template <int L, int KIND> struct TBytes {
    static constexpr int NM = TDim<L>::NMOM;
    static constexpr int B = KIND == TK_F64   ? 8 * NM
                             : KIND == TK_F32 ? 4 * NM
                             : KIND == TK_F48 ? 4 * (NM + (NM + 1) / 2)
                                              : 4 * (NM + (NM + 3) / 4);
};

// RATE: scattering-rate variant (rate_leg >= 0), a separate instantiation so
// that the propagate path keeps all its arrays in registers.
template <int L, int KIND, int TT, int STAGES, bool PAIR, bool RATE>
__global__ void __launch_bounds__(TT) k_collision_tensor(ChanDev c, const InstDev* __restrict__ insts, int n_insts,
                                                         const unsigned char* __restrict__ mom, int64_t ntiles,
                                                         const int32_t* __restrict__ tup, int64_t stride, int64_t n,
                                                         const double* __restrict__ f, double* __restrict__ acc,
                                                         const DPCtl* __restrict__ ctl, int* __restrict__ err_flag,
                                                         int rate_leg, FxAcc fx) {
    constexpr uint32_t TILE_BYTES = uint32_t(TBytes<L, KIND>::B) * TT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* stage_buf = smem_raw;
    __shared__ __align__(8) uint64_t bars[STAGES];
    {
        // every instance finished or switched off: nothing to stream
        bool any = false;
        for (int k = 0; k < n_insts; ++k) {
            const InstDev in = insts[k];
            any |= (in.amplitude != 0.0) && !(ctl && ctl[in.run].done);
        }
        if (!any) return;
    }
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            const int64_t tile = blockIdx.x + (int64_t)s * gridDim.x;
            if (tile < ntiles) {
                mbar_expect_tx_arrive(&bars[s], TILE_BYTES);
                bulk_g2s(stage_buf + (size_t)s * TILE_BYTES, mom + tile * (int64_t)TILE_BYTES, TILE_BYTES, &bars[s]);
            }
        }
    }
    for (int64_t it = 0;; ++it) {
        const int64_t tile = blockIdx.x + it * gridDim.x;
        if (tile >= ntiles) break;
        const int s = int(it % STAGES);
        const uint32_t parity = uint32_t((it / STAGES) & 1);
        if (!mbar_wait(&bars[s], parity, c.wait_polls)) {
            // record the failure, then give every copy still in flight a
            // bounded chance to land before the CTA releases its shared memory
            if (tid == 0) atomicExch(err_flag, 1);
            for (int k = 0; k < STAGES; ++k) {
                const int64_t itk = it + ((k - s + STAGES) % STAGES);
                if (blockIdx.x + itk * gridDim.x < ntiles) mbar_wait(&bars[k], uint32_t((itk / STAGES) & 1), 1 << 16);
            }
            return;
        }
        const unsigned char* sm = stage_buf + (size_t)s * TILE_BYTES;
        const int64_t i = tile * TT + tid;
        {
            // every lane runs the instance loop (padding lanes contribute zero
            // moments and no atomics) so that the warp scatter can reduce
            const bool valid = i < n;
            int e[L];
#pragma unroll
            for (int l = 0; l < L; ++l) e[l] = valid ? __ldg(tup + l * stride + i) : 0;
            // instances in pairs: each moment read from shared memory (and
            // widened to FP64) serves two runs' contractions
            auto active = [&](const InstDev& q) { return q.amplitude != 0.0 && !(ctl && ctl[q.run].done); };
            int k = 0;
            while (k < n_insts) {
                const InstDev a = insts[k];
                if (!active(a)) { ++k; continue; }
                int k2 = k + 1;
                while (k2 < n_insts && !active(insts[k2])) ++k2;
                if (PAIR && k2 < n_insts) {
                    const InstDev pair[2] = {a, insts[k2]};
                    contract_tuple<L, KIND, TT, 2, RATE>(c, pair, e, valid, sm, tid, f, acc, rate_leg, fx);
                    k = k2 + 1;
                } else {
                    const InstDev one[1] = {a};
                    contract_tuple<L, KIND, TT, 1, RATE>(c, one, e, valid, sm, tid, f, acc, rate_leg, fx);
                    k = PAIR ? k2 : k + 1;
                }
            }
        }
        __syncthreads();   // every thread is done with stage s
        if (tid == 0) {
            const int64_t next = tile + (int64_t)STAGES * gridDim.x;
            if (next < ntiles) {
                mbar_expect_tx_arrive(&bars[s], TILE_BYTES);
                bulk_g2s(stage_buf + (size_t)s * TILE_BYTES, mom + next * (int64_t)TILE_BYTES, TILE_BYTES, &bars[s]);
            }
        }
    }
}

// ------------------------------------------------- run-minor contraction
// For a group shared by many runs (a batched ensemble) the per-thread
// contraction above spends most of its instructions on per-tuple work that
// every instance repeats (moment loads and widening, tuple ids, scatter
// keys) and gathers each run's f from its own, distant slice of the state.
// Here one warp contracts one staged tuple for 32 runs at once, lane = run:
//   k_runs_gather     the legs' f of every instance into fT[leg][dof][np]
//                     (32x32 shared-memory transpose, coalesced both ways);
//   k_collision_runs  per tuple, the moments are read at one shared-memory
//                     address by all lanes (broadcast), the lanes' f rows and
//                     their reductions into accT are coalesced 256-byte rows;
//   k_runs_scatter    accT back into the state-layout accumulator, cleared.
// The arithmetic per instance is that of contract_tuple (NI = 1).
struct RunsDev {
    double* fT;
    double* accT;
    FxAcc accTx;   // deterministic mode: accT's exact twin (w null otherwise)
    int64_t loff[TB_MAX_LEGS];
    int64_t ndof[TB_MAX_LEGS];
    int np;
};

// a[l] for a kernel-parameter array without a local-memory copy of it
__device__ __forceinline__ int64_t leg_pick(const int64_t (&a)[TB_MAX_LEGS], int l) {
    return l == 0 ? a[0] : l == 1 ? a[1] : l == 2 ? a[2] : a[3];
}

constexpr int RUNS_THREADS = 256;
constexpr int RUNS_MIN = 8;           // smallest group given the buffers
constexpr int RUNS_DEFAULT_MIN = 16;  // untuned handles use the path from here
constexpr int RUNS_NP_MAX = 1024;     // s_amp: at most 8 KB of shared memory

__global__ void __launch_bounds__(256) k_runs_gather(const InstDev* __restrict__ insts, int n_insts, RunsDev R,
                                                     const double* __restrict__ f) {
    __shared__ double tile[32][33];
    const int l = blockIdx.z;
    const int64_t ndof = leg_pick(R.ndof, l), loff = leg_pick(R.loff, l);
    const int64_t d0 = int64_t(blockIdx.x) * 32;
    const int i0 = blockIdx.y * 32;
    if (d0 >= ndof) return;   // uniform in the block
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int i = i0 + k;
        const int64_t d = d0 + threadIdx.x;
        tile[k][threadIdx.x] = (i < n_insts && d < ndof) ? __ldg(f + insts[i].foff[l] + d) : 0.0;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int64_t d = d0 + k;
        if (d < ndof) R.fT[loff + d * R.np + i0 + threadIdx.x] = tile[threadIdx.x][k];
    }
}

// Every leg in turn through one block of 32 x 32 threads, so that a (dof,
// instance) pair stays with one thread for all legs; then, when the group's
// instances belong to distinct runs (DISTINCT), no two threads add into one
// coefficient and the adds need no atomics (two legs of one band are added by
// the same thread).  The block's instance offsets are staged in shared
// memory, so each add waits on one global load only.
template <bool DISTINCT>
__global__ void __launch_bounds__(1024) k_runs_scatter(const InstDev* __restrict__ insts, int n_insts, RunsDev R,
                                                       int nlegs, double* __restrict__ acc) {
    __shared__ double tile[32][33];
    __shared__ int64_t s_foff[TB_MAX_LEGS][32];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t d0 = int64_t(blockIdx.x) * 32;
    const int i0 = blockIdx.y * 32;
    if (ty < nlegs) s_foff[ty][tx] = (i0 + tx < n_insts) ? insts[i0 + tx].foff[ty] : 0;
    for (int l = 0; l < nlegs; ++l) {
        const int64_t ndof = leg_pick(R.ndof, l), loff = leg_pick(R.loff, l);
        if (d0 >= ndof) continue;   // uniform in the block
        {
            const int64_t d = d0 + ty;
            double v = 0.0;
            if (d < ndof) {
                double* p = R.accT + loff + d * R.np + i0 + tx;
                v = *p;
                *p = 0.0;
            }
            tile[ty][tx] = v;
        }
        __syncthreads();   // also publishes s_foff on the first leg
        {
            const int i = i0 + ty;
            const int64_t d = d0 + tx;
            if (i < n_insts && d < ndof) {
                const double v = tile[tx][ty];
                double* o = acc + s_foff[l][ty] + d;
                if (DISTINCT) *o += v;
                else if (v != 0.0) atomicAdd(o, v);
            }
        }
        __syncthreads();   // the tile is reused by the next leg
    }
}

// The deterministic mode's scatter: accTx (exact words) into the handle's
// exact accumulator fx, the same transpose as k_runs_scatter; the adds are
// integer adds, so neither their order nor DISTINCT changes the result.
template <bool DISTINCT>
__global__ void __launch_bounds__(1024) k_runs_scatter_exact(const InstDev* __restrict__ insts, int n_insts,
                                                             RunsDev R, int nlegs, FxAcc fx) {
    __shared__ Fx tile[32][33];
    __shared__ int64_t s_foff[TB_MAX_LEGS][32];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t d0 = int64_t(blockIdx.x) * 32;
    const int i0 = blockIdx.y * 32;
    if (ty < nlegs) s_foff[ty][tx] = (i0 + tx < n_insts) ? insts[i0 + tx].foff[ty] : 0;
    for (int l = 0; l < nlegs; ++l) {
        const int64_t ndof = leg_pick(R.ndof, l), loff = leg_pick(R.loff, l);
        if (d0 >= ndof) continue;   // uniform in the block
        {
            const int64_t d = d0 + ty;
            Fx v{0ull, 0ull, 0ull};
            if (d < ndof) {
                unsigned long long* p = R.accTx.w + 3 * (loff + d * R.np + i0 + tx);
                v.w0 = p[0];
                v.w1 = p[1];
                v.w2 = p[2];
                if (v.w0 | v.w1 | v.w2) { p[0] = 0ull; p[1] = 0ull; p[2] = 0ull; }
            }
            tile[ty][tx] = v;
        }
        __syncthreads();   // also publishes s_foff on the first leg
        {
            const int i = i0 + ty;
            const int64_t d = d0 + tx;
            if (i < n_insts && d < ndof) {
                const Fx v = tile[tx][ty];
                if (v.w0 | v.w1 | v.w2) {
                    unsigned long long* o = fx.w + 3 * (s_foff[l][ty] + d);
                    if (DISTINCT) fx_add_plain(o, v);
                    else fx_atomic_add(o, v);
                }
            }
        }
        __syncthreads();   // the tile is reused by the next leg
    }
}

// One tuple (staged at column t of the tile) for the instance of this lane.
// EXACT: the deterministic mode's adds into R.accTx (a separate
// instantiation, so that the FP64-atomic kernels keep their registers).
template <int L, int KIND, int TT, bool EXACT>
__device__ __forceinline__ void contract_run(const ChanDev& c, const RunsDev& R, const int (&e)[L], int t, int i,
                                             double amp, const unsigned char* __restrict__ tile) {
    constexpr int K = TDim<L>::K, KM = TDim<L>::KM, NMOM = TDim<L>::NMOM;
    auto M = [&](int j) { return tile_moment<KIND, NMOM, TT>(tile, t, j); };
    double v[K];
    {
        double A[L][3], B[L][3];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const LegDev& lg = c.leg[l];
            const double* fe = R.fT + R.loff[l] + int64_t(3 * e[l]) * R.np + i;
            const double f0 = __ldg(fe), f1 = __ldg(fe + R.np), f2 = __ldg(fe + 2 * R.np);
            A[l][0] = fma(lg.fa, f0, lg.fa0);
            A[l][1] = lg.fa * f1;
            A[l][2] = lg.fa * f2;
            B[l][0] = fma(lg.fb, f0, lg.fb0);
            B[l][1] = lg.fb * f1;
            B[l][2] = lg.fb * f2;
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            int r = j;
            double pa = 1.0, pb = 1.0;
#pragma unroll
            for (int l = L - 1; l >= 0; --l) {
                const int Jl = r % 3;
                r /= 3;
                pa *= A[l][Jl];
                pb *= B[l][Jl];
            }
            v[j] = pa + pb;
        }
    }
    // independent FMA chains: three partial sums for the constant mode and,
    // per km, the r1 / r2 rows of every leg together (the warp has few
    // siblings on its scheduler to hide FMA latency behind)
    double r0a = 0.0, r0b = 0.0, r0c = 0.0;
#pragma unroll
    for (int j = 0; j < K; j += 3) {
        r0a = fma(M(j), v[j], r0a);
        r0b = fma(M(j + 1), v[j + 1], r0b);
        r0c = fma(M(j + 2), v[j + 2], r0c);
    }
    const double r0 = (r0a + r0b) + r0c;
    double r1[L], r2[L];
#pragma unroll
    for (int lam = 0; lam < L; ++lam) { r1[lam] = 0.0; r2[lam] = 0.0; }
#pragma unroll
    for (int km = 0; km < KM; ++km) {
#pragma unroll
        for (int lam = 0; lam < L; ++lam) {
            int sstep = 1;
#pragma unroll
            for (int l = L - 1; l > lam; --l) sstep *= 3;
            const int hi = km / sstep, lo = km % sstep;
            const int j0 = hi * 3 * sstep + lo;
            const int j1 = j0 + sstep, j2 = j0 + 2 * sstep;
            const int qa = K + (lam * 3 + 0) * KM + km;
            const double qxx = M(qa), qxy = M(qa + KM), qyy = M(qa + 2 * KM);
            const double s1 = M(j1), s2 = M(j2);
            r1[lam] = fma(s1, v[j0], r1[lam]);
            r1[lam] = fma(qxx, v[j1], r1[lam]);
            r1[lam] = fma(qxy, v[j2], r1[lam]);
            r2[lam] = fma(s2, v[j0], r2[lam]);
            r2[lam] = fma(qxy, v[j1], r2[lam]);
            r2[lam] = fma(qyy, v[j2], r2[lam]);
        }
    }
    if (amp != 0.0) {
#pragma unroll
        for (int lam = 0; lam < L; ++lam) {
            const double da = c.leg[lam].dir * amp;   // d = +-1: d (r amp) == r (d amp)
            const int64_t slot = R.loff[lam] + int64_t(3 * e[lam]) * R.np + i;
            if (EXACT) {   // deterministic mode: exact adds
                fx_add(R.accTx, slot, r0 * da);
                fx_add(R.accTx, slot + R.np, r1[lam] * da);
                fx_add(R.accTx, slot + 2 * R.np, r2[lam] * da);
            } else {
                double* o = R.accT + slot;
                atomicAdd(o, r0 * da);
                atomicAdd(o + R.np, r1[lam] * da);
                atomicAdd(o + 2 * R.np, r2[lam] * da);
            }
        }
    }
}

// DEC (40-bit moments): the staged tile is widened once, cooperatively, into
// an FP64 copy that the contraction reads; the stage is refilled at once, so
// one stage already overlaps the next copy with the contraction.
// S runs per lane group: a warp takes 32 / S tuples at a time, each for S
// runs (S = 4, 8, 16, 32), so a group of n runs pads to a multiple of S
// rather than of 32; each
// instruction still serves 32 lanes, the moment reads hit 32 / S adjacent
// words and every f row / reduction stays whole 32-byte sectors (S >= 4).
template <int L, int KIND, int TT, int STAGES, int S, bool EXACT>
__global__ void __launch_bounds__(RUNS_THREADS) k_collision_runs(ChanDev c, const InstDev* __restrict__ insts,
                                                                 int n_insts, RunsDev R,
                                                                 const unsigned char* __restrict__ mom, int64_t ntiles,
                                                                 const int32_t* __restrict__ tup, int64_t stride,
                                                                 int64_t n, const DPCtl* __restrict__ ctl,
                                                                 int* __restrict__ err_flag) {
    constexpr uint32_t TILE_BYTES = uint32_t(TBytes<L, KIND>::B) * TT;
    constexpr int NMOM = TDim<L>::NMOM;
    constexpr bool DEC = KIND == TK_F40 || KIND == TK_F48;
    constexpr int KREAD = DEC ? TK_F64 : KIND;
    constexpr size_t DEC_BYTES = DEC ? sizeof(double) * NMOM * TT : 0;
    constexpr int NW = RUNS_THREADS / 32;
    static_assert(TT % NW == 0, "tile tuples must split evenly over the warps");
    constexpr int TPW = TT / NW;
    constexpr int G = 32 / S;   // tuples per warp step
    static_assert(TPW % G == 0, "a warp's tuples must split into steps of 32 / S");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* stage_buf = smem_raw;
    double* dec = reinterpret_cast<double*>(smem_raw + size_t(STAGES) * TILE_BYTES);
    double* s_amp = reinterpret_cast<double*>(smem_raw + size_t(STAGES) * TILE_BYTES + DEC_BYTES);
    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ int s_any;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_any = 0;
    __syncthreads();
    // amplitude of every lane's instance, 0 for padding, switched-off and
    // finished runs (those lanes compute along but emit nothing)
    for (int i = tid; i < R.np; i += RUNS_THREADS) {
        double a = 0.0;
        if (i < n_insts) {
            const InstDev in = insts[i];
            if (in.amplitude != 0.0 && !(ctl && ctl[in.run].done)) a = in.amplitude;
        }
        s_amp[i] = a;
        if (a != 0.0) s_any = 1;
    }
    __syncthreads();
    if (!s_any) return;   // uniform in the block
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            const int64_t tile = blockIdx.x + (int64_t)s * gridDim.x;
            if (tile < ntiles) {
                mbar_expect_tx_arrive(&bars[s], TILE_BYTES);
                bulk_g2s(stage_buf + (size_t)s * TILE_BYTES, mom + tile * (int64_t)TILE_BYTES, TILE_BYTES, &bars[s]);
            }
        }
    }
    const int nch = (n_insts + S - 1) / S;   // nch * S <= np (np: a multiple of 32)
    const int g = lane / S, sl = lane % S;
    for (int64_t it = 0;; ++it) {
        const int64_t tile = blockIdx.x + it * gridDim.x;
        if (tile >= ntiles) break;
        const int s = int(it % STAGES);
        const uint32_t parity = uint32_t((it / STAGES) & 1);
        if (!mbar_wait(&bars[s], parity, c.wait_polls)) {
            if (tid == 0) atomicExch(err_flag, 1);
            for (int k = 0; k < STAGES; ++k) {
                const int64_t itk = it + ((k - s + STAGES) % STAGES);
                if (blockIdx.x + itk * gridDim.x < ntiles) mbar_wait(&bars[k], uint32_t((itk / STAGES) & 1), 1 << 16);
            }
            return;
        }
        const unsigned char* sm = stage_buf + (size_t)s * TILE_BYTES;
        auto refill = [&]() {
            if (tid == 0) {
                const int64_t next = tile + (int64_t)STAGES * gridDim.x;
                if (next < ntiles) {
                    mbar_expect_tx_arrive(&bars[s], TILE_BYTES);
                    bulk_g2s(stage_buf + (size_t)s * TILE_BYTES, mom + next * (int64_t)TILE_BYTES, TILE_BYTES,
                             &bars[s]);
                }
            }
        };
        const unsigned char* rd = sm;
        if constexpr (DEC) {
            for (int k = tid; k < NMOM * TT; k += RUNS_THREADS)
                dec[k] = tile_moment<KIND, NMOM, TT>(sm, k % TT, k / TT);
            __syncthreads();   // dec complete, stage s consumed
            refill();
            rd = reinterpret_cast<const unsigned char*>(dec);
        }
        // warp w: tuples [w TPW, (w+1) TPW) of the tile, G at a time (lane
        // group g takes tuple tt + g), each for every chunk of S instances;
        // lanes past the list's end contract element 0 with amplitude 0
#pragma unroll 1
        for (int tt = 0; tt < TPW; tt += G) {
            if (tile * TT + warp * TPW + tt >= n) break;   // uniform in the warp
            const int t = warp * TPW + tt + g;
            const int64_t gi = tile * TT + t;
            const bool tv = gi < n;
            int e[L];
#pragma unroll
            for (int l = 0; l < L; ++l) e[l] = tv ? __ldg(tup + l * stride + gi) : 0;
#pragma unroll 1
            for (int ch = 0; ch < nch; ++ch) {
                const int i = ch * S + sl;
                const double amp = tv ? s_amp[i] : 0.0;
                if (__all_sync(0xffffffffu, amp == 0.0)) continue;
                contract_run<L, KREAD, TT, EXACT>(c, R, e, t, i, amp, rd);
            }
        }
        __syncthreads();   // every warp is done with stage s (and dec)
        if constexpr (!DEC) refill();
    }
}

// Fills T.d (allocated, sized for n tuples of this kind) with the moments.
template <int L, int KIND>
static int fill_t(const ChanDev& c, const int32_t* tup, int64_t stride, int64_t n, MomentTensor& T, cudaStream_t s) {
    constexpr int TT = TTile<L, KIND>::TT;
    TB_CUDA(cudaMemsetAsync(T.d, 0, size_t(tensor_bytes(L, KIND, n)), s));
    const size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
    int64_t blocks = (n * 32 + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_build_moments<L, KIND><<<unsigned(blocks), 256, smem, s>>>(c, tup, stride, n, T.d, TT);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

template <int L, int KIND>
static int build_t(const ChanDev& c, const int32_t* tup, int64_t stride, int64_t n, MomentTensor& T, cudaStream_t s) {
    constexpr int TT = TTile<L, KIND>::TT;
    const int64_t ntiles = (n + TT - 1) / TT;
    const size_t bytes = size_t(tensor_bytes(L, KIND, n));
    T.release();
    if (cudaMalloc(&T.d, bytes) != cudaSuccess) {
        T.d = nullptr;
        set_error("moment tensor allocation failed");
        return TB_ERR_OOM;
    }
    TB_CUDA(cudaMemsetAsync(T.d, 0, bytes, s));
    const size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
    int64_t blocks = (n * 32 + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_build_moments<L, KIND><<<unsigned(blocks), 256, smem, s>>>(c, tup, stride, n, T.d, TT);
    TB_CUDA(cudaGetLastError());
    T.n = n;
    T.ntiles = ntiles;
    T.nmom = TDim<L>::NMOM;
    T.kind = KIND;
    return TB_OK;
}

int refill_tensor(const ChanDev& c, const int32_t* tup, int64_t stride, int64_t n, MomentTensor& T, cudaStream_t s) {
    if (!T.d || T.n != n) { set_error("refill of a tensor that was not built for this list"); return TB_ERR_ARG; }
    switch (c.L * 4 + T.kind) {
        case 8: return fill_t<2, TK_F64>(c, tup, stride, n, T, s);
        case 9: return fill_t<2, TK_F32>(c, tup, stride, n, T, s);
        case 10: return fill_t<2, TK_F40>(c, tup, stride, n, T, s);
        case 11: return fill_t<2, TK_F48>(c, tup, stride, n, T, s);
        case 12: return fill_t<3, TK_F64>(c, tup, stride, n, T, s);
        case 13: return fill_t<3, TK_F32>(c, tup, stride, n, T, s);
        case 14: return fill_t<3, TK_F40>(c, tup, stride, n, T, s);
        case 15: return fill_t<3, TK_F48>(c, tup, stride, n, T, s);
        case 16: return fill_t<4, TK_F64>(c, tup, stride, n, T, s);
        case 17: return fill_t<4, TK_F32>(c, tup, stride, n, T, s);
        case 18: return fill_t<4, TK_F40>(c, tup, stride, n, T, s);
        case 19: return fill_t<4, TK_F48>(c, tup, stride, n, T, s);
    }
    set_error("nlegs must be 2..4");
    return TB_ERR_ARG;
}

int build_tensor(const ChanDev& c, const int32_t* tup, int64_t stride, int64_t n, int kind, MomentTensor& T,
                 cudaStream_t s) {
    switch (c.L * 4 + kind) {
        case 8: return build_t<2, TK_F64>(c, tup, stride, n, T, s);
        case 9: return build_t<2, TK_F32>(c, tup, stride, n, T, s);
        case 10: return build_t<2, TK_F40>(c, tup, stride, n, T, s);
        case 11: return build_t<2, TK_F48>(c, tup, stride, n, T, s);
        case 12: return build_t<3, TK_F64>(c, tup, stride, n, T, s);
        case 13: return build_t<3, TK_F32>(c, tup, stride, n, T, s);
        case 14: return build_t<3, TK_F40>(c, tup, stride, n, T, s);
        case 15: return build_t<3, TK_F48>(c, tup, stride, n, T, s);
        case 16: return build_t<4, TK_F64>(c, tup, stride, n, T, s);
        case 17: return build_t<4, TK_F32>(c, tup, stride, n, T, s);
        case 18: return build_t<4, TK_F40>(c, tup, stride, n, T, s);
        case 19: return build_t<4, TK_F48>(c, tup, stride, n, T, s);
    }
    set_error("nlegs must be 2..4");
    return TB_ERR_ARG;
}

// The kernels' large-shared-memory attribute, set once per device.
constexpr int TB_MAX_DEVICES = 64;

static int current_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

// The handle's bounded-wait flag (ChanDev::err_flag), which every
// contraction launch needs.
static int channel_err_flag(const ChanDev& c, int** flag) {
    if (!c.err_flag) { set_error("channel without its wait-timeout flag"); return TB_ERR_ARG; }
    *flag = c.err_flag;
    return TB_OK;
}

// Sets kern's dynamic shared-memory limit once on each device.
template <class K>
static int ensure_smem_attr(K kern, int bytes, unsigned long long& done_devices) {
    const int dev = current_device();
    if (dev >= 0 && dev < TB_MAX_DEVICES && (done_devices >> dev) & 1ull) return TB_OK;
    TB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (dev >= 0 && dev < TB_MAX_DEVICES) done_devices |= 1ull << dev;
    return TB_OK;
}

static RunsDev runs_dev(const ChanDev& c, const MomentTensor& T, const FxAcc& fx) {
    RunsDev R{};
    R.fT = T.fT;
    R.accT = T.accT;
    if (fx.w) {
        R.accTx.w = T.accTx;
        R.accTx.poison = fx.poison;
        R.accTx.sat = fx.sat;
    }
    R.np = T.np;
    for (int l = 0; l < TB_MAX_LEGS; ++l) {
        R.loff[l] = T.loff[l];
        R.ndof[l] = l < c.L ? 3 * int64_t(c.leg[l].ne) : 0;
    }
    return R;
}

// gather -> run-minor contraction -> scatter (three launches on s)
template <int L, int KIND, int STAGES, int S>
static int launch_runs(const ChanDev& c, const InstDev* insts, int n_insts, const MomentTensor& T, const int32_t* tup,
                       int64_t stride, int64_t n, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s,
                       const FxAcc& fx) {
    constexpr int TT = TTile<L, KIND>::TT;
    if (fx.w && !T.accTx) { set_error("run-minor contraction without its exact accumulator"); return TB_ERR_ARG; }
    const RunsDev R = runs_dev(c, T, fx);
    int64_t maxd = 0;
    for (int l = 0; l < L; ++l) maxd = std::max(maxd, R.ndof[l]);
    const dim3 tb(32, 8), tg(unsigned((maxd + 31) / 32), unsigned(T.np / 32), unsigned(L));
    k_runs_gather<<<tg, tb, 0, s>>>(insts, n_insts, R, f);
    TB_CUDA(cudaGetLastError());
    auto kern = fx.w ? k_collision_runs<L, KIND, TT, STAGES, S, true> : k_collision_runs<L, KIND, TT, STAGES, S, false>;
    const size_t fixed = size_t(STAGES) * TT * tuple_bytes(L, KIND) +
                         ((KIND == TK_F40 || KIND == TK_F48) ? sizeof(double) * TDim<L>::NMOM * TT : 0);
    const size_t smem = fixed + sizeof(double) * size_t(T.np);
    static unsigned long long attr_devices[2] = {0, 0};
    TB_TRY(ensure_smem_attr(kern, int(fixed + sizeof(double) * RUNS_NP_MAX), attr_devices[fx.w ? 1 : 0]));
    int* err_flag = nullptr;
    TB_TRY(channel_err_flag(c, &err_flag));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RUNS_THREADS, smem);
    if (per_sm < 1) per_sm = 1;
    int64_t grid = int64_t(nsm) * per_sm;
    if (grid > T.ntiles) grid = T.ntiles;
    if (grid >= 1) {
        kern<<<unsigned(grid), RUNS_THREADS, smem, s>>>(c, insts, n_insts, R, static_cast<const unsigned char*>(T.d),
                                                       T.ntiles, tup, stride, n, ctl, err_flag);
        TB_CUDA(cudaGetLastError());
    }
    const dim3 sg(tg.x, tg.y, 1), sb(32, 32);
    if (fx.w) {
        if (T.runs_distinct) k_runs_scatter_exact<true><<<sg, sb, 0, s>>>(insts, n_insts, R, L, fx);
        else k_runs_scatter_exact<false><<<sg, sb, 0, s>>>(insts, n_insts, R, L, fx);
    } else if (T.runs_distinct) {
        k_runs_scatter<true><<<sg, sb, 0, s>>>(insts, n_insts, R, L, acc);
    } else {
        k_runs_scatter<false><<<sg, sb, 0, s>>>(insts, n_insts, R, L, acc);
    }
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

int prepare_runs(const ChanDev& c, int n_insts, bool distinct_runs, MomentTensor& T, cudaStream_t s, bool exact) {
    if (c.L > 3 || n_insts < RUNS_MIN || T.fT || !T.d) return TB_OK;
    const int np = (n_insts + 31) & ~31;
    if (np > RUNS_NP_MAX) return TB_OK;
    int64_t tot = 0;
    for (int l = 0; l < c.L; ++l) {
        T.loff[l] = tot;
        tot += 3 * int64_t(c.leg[l].ne) * np;
    }
    const size_t bytes = sizeof(double) * size_t(tot);
    if (cudaMalloc(&T.fT, bytes) != cudaSuccess) {
        cudaGetLastError();
        T.fT = nullptr;
        return TB_OK;
    }
    if (cudaMalloc(&T.accT, bytes) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(T.fT);
        T.fT = nullptr;
        T.accT = nullptr;
        return TB_OK;
    }
    if (exact) {
        if (cudaMalloc(&T.accTx, 3 * bytes) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(T.fT);
            cudaFree(T.accT);
            T.fT = nullptr;
            T.accT = nullptr;
            T.accTx = nullptr;
            return TB_OK;
        }
        TB_CUDA(cudaMemsetAsync(T.accTx, 0, 3 * bytes, s));
    }
    TB_CUDA(cudaMemsetAsync(T.accT, 0, bytes, s));
    T.np = np;
    T.runs_distinct = distinct_runs ? 1 : 0;
    T.runs = n_insts >= RUNS_DEFAULT_MIN ? 8 : 0;
    return TB_OK;
}

template <int L, int KIND, int STAGES, bool PAIR, bool RATE = false>
static int launch_variant(const ChanDev& c, const InstDev* insts, int n_insts, const MomentTensor& T,
                          const int32_t* tup, int64_t stride, int64_t n, const double* f, double* acc,
                          const DPCtl* ctl, cudaStream_t s, int rate_leg, const FxAcc& fx) {
    constexpr int TT = TTile<L, KIND>::TT;
    auto kern = k_collision_tensor<L, KIND, TT, STAGES, PAIR, RATE>;
    const size_t smem = size_t(STAGES) * TT * tuple_bytes(L, KIND);
    static unsigned long long attr_devices = 0;
    TB_TRY(ensure_smem_attr(kern, int(smem), attr_devices));
    int* err_flag = nullptr;
    TB_TRY(channel_err_flag(c, &err_flag));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TT, smem);
    if (per_sm < 1) per_sm = 1;
    int64_t grid = int64_t(nsm) * per_sm;
    if (grid > T.ntiles) grid = T.ntiles;
    if (grid < 1) return TB_OK;
    kern<<<unsigned(grid), TT, smem, s>>>(c, insts, n_insts, static_cast<const unsigned char*>(T.d), T.ntiles, tup,
                                          stride, n, f, acc, ctl, err_flag, rate_leg, fx);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// The instance-pair path (one moment read for two runs) exists for L <= 3
// only (four-leg pairs would spill registers) and only matters where a group
// has several instances; it needs more registers than the single path.
template <int L, int KIND>
static int launch_t(const ChanDev& c, const InstDev* insts, int n_insts, const MomentTensor& T, const int32_t* tup,
                    int64_t stride, int64_t n, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s,
                    int rate_leg, const FxAcc& fx) {
#define TB_VARIANT(ST, PR, RT) \
    launch_variant<L, KIND, ST, PR, RT>(c, insts, n_insts, T, tup, stride, n, f, acc, ctl, s, rate_leg, fx)
    if (rate_leg >= 0)   // diagnostic operator: one fixed schedule
        return TB_VARIANT(2, false, true);
    if constexpr (L <= 3) {
        // the run-minor path needs its exact twin in the deterministic mode
        if (T.runs && T.fT && (!fx.w || T.accTx)) {
#define TB_RUNS(ST, SS) launch_runs<L, KIND, ST, SS>(c, insts, n_insts, T, tup, stride, n, f, acc, ctl, s, fx)
            if (T.stages == 1)
                return T.runs == 4 ? TB_RUNS(1, 4) : T.runs == 8 ? TB_RUNS(1, 8) : T.runs == 16 ? TB_RUNS(1, 16)
                                                                                 : TB_RUNS(1, 32);
            return T.runs == 4 ? TB_RUNS(2, 4) : T.runs == 8 ? TB_RUNS(2, 8) : T.runs == 16 ? TB_RUNS(2, 16)
                                                                             : TB_RUNS(2, 32);
#undef TB_RUNS
        }
    }
    const bool pair = (L <= 3) && n_insts > 1 && T.pair;
    if (T.stages == 1) return pair ? TB_VARIANT(1, (L <= 3), false) : TB_VARIANT(1, false, false);
    return pair ? TB_VARIANT(2, (L <= 3), false) : TB_VARIANT(2, false, false);
#undef TB_VARIANT
}

int launch_collision_tensor(const ChanDev& c, const InstDev* insts, int n_insts, const MomentTensor& T,
                            const int32_t* tup, int64_t stride, int64_t n, const double* f, double* acc,
                            const DPCtl* ctl, cudaStream_t s, int rate_leg, const FxAcc& fx) {
    if (n <= 0 || n_insts <= 0) return TB_OK;
#define TB_LT(LL, KK) launch_t<LL, KK>(c, insts, n_insts, T, tup, stride, n, f, acc, ctl, s, rate_leg, fx)
    switch (c.L * 4 + T.kind) {
        case 8: return TB_LT(2, TK_F64);
        case 9: return TB_LT(2, TK_F32);
        case 10: return TB_LT(2, TK_F40);
        case 11: return TB_LT(2, TK_F48);
        case 12: return TB_LT(3, TK_F64);
        case 13: return TB_LT(3, TK_F32);
        case 14: return TB_LT(3, TK_F40);
        case 15: return TB_LT(3, TK_F48);
        case 16: return TB_LT(4, TK_F64);
        case 17: return TB_LT(4, TK_F32);
        case 18: return TB_LT(4, TK_F40);
        case 19: return TB_LT(4, TK_F48);
    }
#undef TB_LT
    set_error("nlegs must be 2..4");
    return TB_ERR_ARG;
}

int tune_tensor(const ChanDev& c, const InstDev* insts, int n_insts, MomentTensor& T, const int32_t* tup,
                int64_t stride, int64_t n, const double* f, double* acc, cudaStream_t s) {
    if (n <= 0 || n_insts <= 0 || !T.d) return TB_OK;
    // tuple counts within a factor 2^(1/8) share a cache entry
    const int64_t bucket = int64_t(std::llround(std::log2(double(n)) * 8.0));
    const std::tuple<int, int, int64_t, int> key(c.L, T.kind, bucket, n_insts);
    static std::mutex mu;
    static std::map<std::tuple<int, int, int64_t, int>, std::tuple<int, int, int, double>> cache;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            T.stages = std::get<0>(it->second);
            T.pair = std::get<1>(it->second);
            T.runs = T.fT ? std::get<2>(it->second) : 0;
            T.tuned_seconds = std::get<3>(it->second);
            return TB_OK;
        }
    }
    cudaEvent_t e0, e1;
    TB_CUDA(cudaEventCreate(&e0));
    TB_CUDA(cudaEventCreate(&e1));
    double best = 1e300;
    int bs = T.stages, bp = T.pair, br = T.runs;
    const int pairs_max = (c.L <= 3 && n_insts > 1) ? 1 : 0;
    const int runs_max = T.fT ? 4 : 0;
    int rc = TB_OK;
    for (int st = 1; st <= 2 && rc == TB_OK; ++st)
        for (int pr = 0; pr <= 1 + runs_max && rc == TB_OK; ++pr) {
            // pr: 0 one instance per thread, 1 instance pairs, 2 / 3 / 4 / 5
            // run-minor with 32 / 8 / 4 / 16 runs per lane group
            if (pr == 1 && !pairs_max) continue;
            T.stages = st;
            T.pair = pr == 1;
            T.runs = pr == 2 ? 32 : pr == 3 ? 8 : pr == 4 ? 4 : pr == 5 ? 16 : 0;
            rc = launch_collision_tensor(c, insts, n_insts, T, tup, stride, n, f, acc, nullptr, s);   // warm-up
            if (rc != TB_OK) break;
            constexpr int REPS = 3;
            cudaEventRecord(e0, s);
            for (int r = 0; r < REPS && rc == TB_OK; ++r)
                rc = launch_collision_tensor(c, insts, n_insts, T, tup, stride, n, f, acc, nullptr, s);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) { rc = TB_ERR_CUDA; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double sec = 1e-3 * double(ms) / REPS;
            if (sec < best) { best = sec; bs = st; bp = T.pair; br = T.runs; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    T.stages = bs;
    T.pair = bp;
    T.runs = br;
    if (rc != TB_OK) return rc;
    T.tuned_seconds = best;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = std::make_tuple(bs, bp, br, best);
    return TB_OK;
}

int take_wait_timeout(int* flag, cudaStream_t s, int* value) {
    *value = 0;
    if (!flag) return TB_OK;
    TB_CUDA(cudaMemcpyAsync(value, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    TB_CUDA(cudaStreamSynchronize(s));
    if (*value) TB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    return TB_OK;
}

}  // namespace tb
