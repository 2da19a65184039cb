// tb_theta.cu -- which Monte-Carlo points of a tuple lie inside the
// simplices, decided once per handle, and the compacted tuple list the
// Monte-Carlo collision kernels walk.
//
// In scatteringIntegrationTypeB (include/Physics/Scattering/IntegratorCore.hpp:
// 298-357) a point contributes the integrand times ThetapC * ThetaFC
// (:318-320): both the partially and the fully constrained leg strictly
// inside the reference triangle.  That factor depends on the tuple's geometry
// and on the point only, never on f, and the table of points is fixed for
// the life of a handle.  So bit m of mask[i] records it for tuple i and point
// m (same decision procedure as the dense kernel: fast fused alpha, exact
// reference-order re-evaluation near a boundary), and the collision kernel
// evaluates the integrand only at set bits, in increasing m.  A skipped term
// is the integrand times 0, i.e. exactly zero for finite f, so the sums are
// those of the full quadrature.
//
// On the 16x16 one-band e-e channel about 5 % of the points are inside and
// 30 % of the tuples have none.  Tuples without a point are dropped; the
// others are stably sorted by (leg-0 element, descending point count): the
// 32 lanes of a warp then run nearly the same number of points (0.98 of the
// work is useful, against 0.26 in enumeration order), and lanes that share
// the leg-0 element still merge their scatter in the warp reduction.
#include <cub/cub.cuh>

#include <algorithm>

#include "tb_geom.cuh"
#include "tb_theta.cuh"

namespace tb {

void ThetaList::release() {
    if (ids) cudaFree(ids);
    if (mask) cudaFree(mask);
    if (perm) cudaFree(perm);
    ids = nullptr;
    mask = nullptr;
    perm = nullptr;
    n = 0;
    points = 0;
    built = false;
    use = false;
}

template <int L>
__global__ void __launch_bounds__(256) k_theta_mask(ChanDev c, const int32_t* __restrict__ tup, int64_t stride,
                                                    int64_t n, uint64_t* __restrict__ mask, uint32_t* __restrict__ key,
                                                    int32_t* __restrict__ idx, unsigned long long* counts) {
    extern __shared__ double s_mc[];
    constexpr int R = 2 * (L - 2) + 1;
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) s_mc[i] = c.mc[i];
    __syncthreads();
    unsigned long long kept = 0, pts = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int e[L];
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = __ldg(tup + l * stride + i);
        const int u = __ldg(tup + L * stride + i);
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, u, g);
        uint64_t mk = 0;
        if (fabs(g.det) >= c.min_det) {   // the kernels' validity test (false for NaN)
            double Ci[3][3];
            dc_inverse<L>(g, Ci);
            AlphaMap<L> am;
            alpha_map<L>(g, Ci, am);
            for (int m = 0; m < c.nmc; ++m) {
                double al[3];
                if (alpha_theta<L>(g, Ci, am, s_mc + m * R, al)) mk |= 1ull << m;
            }
        }
        const int pc = __popcll(mk);
        mask[i] = mk;
        idx[i] = int32_t(i);
        key[i] = mk ? ((uint32_t(e[0]) << 6) | uint32_t(64 - pc)) : 0xffffffffu;
        kept += mk ? 1 : 0;
        pts += pc;
    }
    for (int o = 16; o > 0; o >>= 1) {
        kept += __shfl_down_sync(0xffffffffu, kept, o);
        pts += __shfl_down_sync(0xffffffffu, pts, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counts + 0, kept);
        atomicAdd(counts + 1, pts);
    }
}

__global__ void k_theta_gather(const int32_t* __restrict__ tup, int64_t stride, int L,
                               const int32_t* __restrict__ order, const uint64_t* __restrict__ mask_in, int64_t nl,
                               int32_t* __restrict__ ids, uint64_t* __restrict__ mask_out, int32_t* __restrict__ perm) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nl; j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = order[j];
        for (int l = 0; l <= L; ++l) ids[l * nl + j] = tup[l * stride + s];
        mask_out[j] = mask_in[s];
        perm[j] = s;
    }
}

namespace {

// Temporaries of one build, freed on every return path.
struct Scratch {
    std::vector<void*> p;
    template <class T>
    T* get(size_t n) {
        void* q = nullptr;
        if (cudaMalloc(&q, n * sizeof(T) + 16) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        p.push_back(q);
        return static_cast<T*>(q);
    }
    ~Scratch() {
        for (void* q : p) cudaFree(q);
    }
};

}  // namespace

int build_theta_list(const ChanDev& c, const DeviceTuples& tup, ThetaList& out, cudaStream_t stream) {
    out.release();
    const int64_t n = tup.n;
    // one bit per point; sort keys hold the leg-0 element above 6 bits of
    // point count, below the 0xffffffff of tuples without a point (so the
    // element must fit 25 bits); cub sorts int-sized inputs
    if (n <= 0 || c.nmc < 1 || c.nmc > 64 || c.leg[0].ne >= (1 << 25) || n > int64_t(0x7fffffff)) return TB_OK;
    Scratch tmp;
    uint64_t* mask = tmp.get<uint64_t>(size_t(n));
    uint32_t* key[2] = {tmp.get<uint32_t>(size_t(n)), tmp.get<uint32_t>(size_t(n))};
    int32_t* idx[2] = {tmp.get<int32_t>(size_t(n)), tmp.get<int32_t>(size_t(n))};
    unsigned long long* counts = tmp.get<unsigned long long>(2);
    if (!mask || !key[0] || !key[1] || !idx[0] || !idx[1] || !counts) return TB_OK;   // no room: full quadrature
    TB_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), stream));
    const int threads = 256;
    const int64_t blocks = std::min<int64_t>((n + threads - 1) / threads, 148 * 16);
    const size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
    switch (c.L) {
        case 2: k_theta_mask<2><<<unsigned(blocks), threads, smem, stream>>>(c, tup.d, tup.cap, n, mask, key[0], idx[0], counts); break;
        case 3: k_theta_mask<3><<<unsigned(blocks), threads, smem, stream>>>(c, tup.d, tup.cap, n, mask, key[0], idx[0], counts); break;
        case 4: k_theta_mask<4><<<unsigned(blocks), threads, smem, stream>>>(c, tup.d, tup.cap, n, mask, key[0], idx[0], counts); break;
        default: set_error("nlegs must be 2..4"); return TB_ERR_ARG;
    }
    TB_CUDA(cudaGetLastError());
    cub::DoubleBuffer<uint32_t> kb(key[0], key[1]);
    cub::DoubleBuffer<int32_t> vb(idx[0], idx[1]);
    size_t tbytes = 0;
    TB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tbytes, kb, vb, int(n), 0, 32, stream));
    void* d_tmp = tmp.get<char>(tbytes);
    if (!d_tmp) return TB_OK;
    TB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tbytes, kb, vb, int(n), 0, 32, stream));   // stable
    unsigned long long h_counts[2] = {0, 0};
    TB_CUDA(cudaMemcpyAsync(h_counts, counts, sizeof(h_counts), cudaMemcpyDeviceToHost, stream));
    TB_CUDA(cudaStreamSynchronize(stream));
    const int64_t nl = int64_t(h_counts[0]);
    if (nl > 0) {
        if (cudaMalloc(&out.ids, sizeof(int32_t) * size_t(c.L + 1) * size_t(nl)) != cudaSuccess ||
            cudaMalloc(&out.mask, sizeof(uint64_t) * size_t(nl)) != cudaSuccess ||
            cudaMalloc(&out.perm, sizeof(int32_t) * size_t(nl)) != cudaSuccess) {
            cudaGetLastError();
            out.release();
            return TB_OK;
        }
        const int64_t gb = std::min<int64_t>((nl + threads - 1) / threads, 148 * 16);
        k_theta_gather<<<unsigned(gb), threads, 0, stream>>>(tup.d, tup.cap, c.L, vb.Current(), mask, nl, out.ids,
                                                             out.mask, out.perm);
        TB_CUDA(cudaGetLastError());
        TB_CUDA(cudaStreamSynchronize(stream));
    }
    out.n = nl;
    out.points = int64_t(h_counts[1]);
    out.built = true;
    out.use = true;
    return TB_OK;
}

}  // namespace tb
