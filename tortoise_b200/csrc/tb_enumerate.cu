// tb_enumerate.cu -- on-device tuple enumeration (the "precalculateIndices"
// step of the reference), compiled with --fmad=false so that every
// floating-point decision (box floors, energy window, determinant filter,
// survival threshold) rounds exactly like the reference's unfused C++.
//
// Reference loop structure (followed one-to-one):
//   deterministicIteration / nestedForSections / nestedForElements
//       include/Physics/Scattering/ScatteringChannel.hpp:205-255
//   survival test inside precalculateIndices
//       src/Physics/Scattering/ScatteringChannel.cpp:476-504
//   TrapezoidalSubset box arithmetic
//       src/Geometry/Structured/DirectSpace/MeshSubset.cpp:62-66, 82-87, 121-125, 169-194
//
// Design: the work items are (umklapp, section of legs 0..L-2, element choice
// of legs 0..L-2) flattened so that increasing item index is the reference's
// loop order; each item scans the element box of the last leg in increasing
// element id (which is the reference's MeshSubsetElementIterator order).  A
// count pass, an exclusive scan and a write pass then emit the surviving
// tuples in exactly the reference's order, deterministically, with no sort.
#include <cub/cub.cuh>

#include "tb_enumerate.cuh"
#include "tb_geom.cuh"

namespace tb {

struct EnumLeg {
    const double* minE;
    const double* maxE;
    int nx, ny;
    double origin[2];
    double dG[2][2];
    double invdG[2][2];
};

struct EnumArgs {
    ChanDev c;
    EnumLeg leg[TB_MAX_LEGS];
    int64_t nsec[TB_MAX_LEGS];   // sections of legs 0..L-2 (1 for unused)
    const double* mc_pre;        // [nmc*R] device
};

struct Box { double l[2], h[2]; };

__device__ __forceinline__ Box section_box(const EnumLeg& m, int sx, int sy) {
    Box b;
    const double lo0 = double(sx) + 0.00000001, lo1 = double(sy) + 0.00000001;
    const double hi0 = double(sx + 1) - 0.00000001, hi1 = double(sy + 1) - 0.00000001;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        b.l[i] = m.origin[i] + (m.dG[i][0] * lo0 + m.dG[i][1] * lo1);
        b.h[i] = m.origin[i] + (m.dG[i][0] * hi0 + m.dG[i][1] * hi1);
    }
    return b;
}

__device__ __forceinline__ Box box_scale(Box b, double s) {
    if (s >= 0.0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) { b.l[i] *= s; b.h[i] *= s; }
    } else {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const double t = b.l[i];
            b.l[i] = b.h[i] * s;
            b.h[i] = t * s;
        }
    }
    return b;
}

template <int L>
__global__ void __launch_bounds__(256) k_enumerate(EnumArgs a, int64_t item0, int64_t count, uint32_t* counts,
                                                   const uint32_t* offsets, int32_t* out, int64_t stride,
                                                   int64_t base, unsigned long long* diag) {
    extern __shared__ double s_mc[];
    const ChanDev& c = a.c;
    constexpr int R = 2 * (L - 2) + 1;
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) s_mc[i] = a.mc_pre[i];
    __syncthreads();
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n_pre = 0, n_det = 0, n_surv = 0;
    if (t < count) {
        const int64_t item = item0 + t;
        constexpr int C = 1 << (L - 1);
        const int comb = int(item % C);
        int64_t r = item / C;
        int sec[TB_MAX_LEGS] = {0, 0, 0, 0};
#pragma unroll
        for (int l = L - 2; l >= 0; --l) {
            sec[l] = int(r % a.nsec[l]);
            r /= a.nsec[l];
        }
        const int u = int(r);
        // box of the last leg: -dir[L-1] * (sum_l dir[l] * box_l + gVec * u)
        const double ux = c.umk[2 * u], uy = c.umk[2 * u + 1];
        const double gu0 = c.gvec[0] * ux + c.gvec[2] * uy;
        const double gu1 = c.gvec[1] * ux + c.gvec[3] * uy;
        Box acc;
#pragma unroll
        for (int l = 0; l < L - 1; ++l) {
            const EnumLeg& m = a.leg[l];
            Box b = box_scale(section_box(m, sec[l] % m.nx, sec[l] / m.nx), c.leg[l].dir);
            if (l == 0) acc = b;
            else {
#pragma unroll
                for (int i = 0; i < 2; ++i) { acc.l[i] += b.l[i]; acc.h[i] += b.h[i]; }
            }
        }
        acc.l[0] += gu0; acc.h[0] += gu0;
        acc.l[1] += gu1; acc.h[1] += gu1;
        acc = box_scale(acc, -c.leg[L - 1].dir);
        const EnumLeg& ml = a.leg[L - 1];
        int lo[2], hi[2];
        const int ns[2] = {ml.nx, ml.ny};
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const double tl = ml.invdG[i][0] * (acc.l[0] - ml.origin[0]) + ml.invdG[i][1] * (acc.l[1] - ml.origin[1]);
            const double th = ml.invdG[i][0] * (acc.h[0] - ml.origin[0]) + ml.invdG[i][1] * (acc.h[1] - ml.origin[1]);
            const int aa = int(floor(tl));
            const int bb = int(floor(th) + 1.0);
            lo[i] = min(max(aa, 0), ns[i]);
            hi[i] = min(max(bb, 0), ns[i]);
        }
        if (lo[0] != hi[0] && lo[1] != hi[1]) {
            int e[L];
            double mn[L], mx[L];
#pragma unroll
            for (int l = 0; l < L - 1; ++l) {
                const int bit = (comb >> (L - 2 - l)) & 1;
                e[l] = 2 * sec[l] + bit;
                const double emin = __ldg(a.leg[l].minE + e[l]), emax = __ldg(a.leg[l].maxE + e[l]);
                mn[l] = (c.leg[l].dir > 0) ? emin : -emax;
                mx[l] = (c.leg[l].dir > 0) ? emax : -emin;
            }
            const double sqrt2 = 1.4142135623730951;  // sqrt(2.0) correctly rounded
            double prodc = 1.0;
#pragma unroll
            for (int l = 0; l < L; ++l) prodc *= sqrt2;
            uint32_t local = 0;
            for (int sy = lo[1]; sy < hi[1]; ++sy)
                for (int sx = lo[0]; sx < hi[0]; ++sx)
                    for (int ie = 0; ie < 2; ++ie) {
                        const int el = 2 * (sx + sy * ml.nx) + ie;
                        e[L - 1] = el;
                        const double emin = __ldg(ml.minE + el), emax = __ldg(ml.maxE + el);
                        mn[L - 1] = (c.leg[L - 1].dir > 0) ? emin : -emax;
                        mx[L - 1] = (c.leg[L - 1].dir > 0) ? emax : -emin;
                        double minE = 0.0, maxE = 0.0;
#pragma unroll
                        for (int k = 0; k < L; ++k) { minE += mn[k]; maxE += mx[k]; }
                        if (!((minE <= 0.0) && (maxE >= 0.0))) continue;
                        ++n_pre;
                        TupleGeom<L> g;
                        tuple_geometry<L>(c, e, u, g);
                        if (!(fabs(g.det) >= c.min_det)) continue;
                        ++n_det;
                        double Ci[3][3];
                        dc_inverse<L>(g, Ci);
                        double sum = 0.0;
                        double p[L][2];
                        for (int m = 0; m < c.nmc; ++m) {
                            const bool th = mc_point_exact<L>(g, Ci, s_mc + m * R, p);
                            sum += th ? prodc : 0.0;
                        }
                        double res = (1.0 / (c.fact * double(c.nmc) * fabs(g.det))) * sum;
                        res *= c.amp_vol;
                        if (!(fabs(res) > c.threshold)) continue;
                        if (offsets) {
                            const int64_t pos = base + (int64_t)offsets[t] + local;
#pragma unroll
                            for (int l = 0; l < L; ++l) out[l * stride + pos] = e[l];
                            out[L * stride + pos] = u;
                        }
                        ++local;
                    }
            n_surv = local;
        }
        if (counts) counts[t] = n_surv;
    }
    if (diag && !offsets) {
        unsigned long long v0 = n_pre, v1 = n_det, v2 = n_surv;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0 += __shfl_down_sync(0xffffffffu, v0, o);
            v1 += __shfl_down_sync(0xffffffffu, v1, o);
            v2 += __shfl_down_sync(0xffffffffu, v2, o);
        }
        if ((threadIdx.x & 31) == 0 && (v0 | v1 | v2)) {
            atomicAdd(diag + 0, v0);
            atomicAdd(diag + 1, v1);
            atomicAdd(diag + 2, v2);
        }
    }
}

// Host driver: chunked count / scan / write.  Output is SoA with L+1 rows
// (L element-id rows, then the umklapp row) of length `cap`.
int enumerate_channel(const ChanDev& c, const HostMesh* meshes, const HostBand* bands, const int* leg_band,
                      const double* d_mc_pre, const double* const* d_minE, const double* const* d_maxE,
                      cudaStream_t stream, DeviceTuples& outT, int64_t diag[3]) {
    const int L = c.L;
    EnumArgs a;
    a.c = c;
    for (int l = 0; l < TB_MAX_LEGS; ++l) a.nsec[l] = 1;
    for (int l = 0; l < L; ++l) {
        const HostMesh& m = meshes[bands[leg_band[l]].mesh];
        EnumLeg& el = a.leg[l];
        el.minE = d_minE[l];
        el.maxE = d_maxE[l];
        el.nx = m.nx;
        el.ny = m.ny;
        for (int i = 0; i < 2; ++i) {
            el.origin[i] = m.origin[i];
            for (int j = 0; j < 2; ++j) { el.dG[i][j] = m.dG[i][j]; el.invdG[i][j] = m.invdG[i][j]; }
        }
        if (l < L - 1) a.nsec[l] = int64_t(m.nx) * m.ny;
    }
    a.mc_pre = d_mc_pre;
    int64_t total = c.n_umk;
    for (int l = 0; l < L - 1; ++l) total *= a.nsec[l];
    total *= (int64_t(1) << (L - 1));

    const int64_t CH = int64_t(1) << 24;
    const int64_t chunk = total < CH ? total : CH;
    uint32_t *d_counts = nullptr, *d_offsets = nullptr;
    unsigned long long* d_diag = nullptr;
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    int rc = TB_OK;
    auto fail = [&](int code, const char* what) {
        set_error(std::string("enumerate: ") + what);
        rc = code;
    };
    if (cudaMalloc(&d_counts, sizeof(uint32_t) * (chunk > 0 ? chunk : 1)) != cudaSuccess ||
        cudaMalloc(&d_offsets, sizeof(uint32_t) * (chunk > 0 ? chunk : 1)) != cudaSuccess ||
        cudaMalloc(&d_diag, sizeof(unsigned long long) * 3) != cudaSuccess) {
        fail(TB_ERR_OOM, "counts allocation failed");
    }
    if (rc == TB_OK) {
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_counts, d_offsets, int(chunk > 0 ? chunk : 1), stream);
        if (cudaMalloc(&d_tmp, tmp_bytes) != cudaSuccess) fail(TB_ERR_OOM, "scan scratch allocation failed");
    }
    if (rc == TB_OK) cudaMemsetAsync(d_diag, 0, sizeof(unsigned long long) * 3, stream);
    const size_t smem = sizeof(double) * size_t(c.nmc) * c.R;
    int64_t n = 0;
    if (outT.cap == 0 && rc == TB_OK) rc = outT.reserve(L, int64_t(1) << 20, stream);
    for (int64_t s = 0; s < total && rc == TB_OK; s += chunk) {
        const int64_t cnt = (total - s) < chunk ? (total - s) : chunk;
        const unsigned grid = unsigned((cnt + 255) / 256);
        switch (L) {
            case 2: k_enumerate<2><<<grid, 256, smem, stream>>>(a, s, cnt, d_counts, nullptr, nullptr, 0, 0, d_diag); break;
            case 3: k_enumerate<3><<<grid, 256, smem, stream>>>(a, s, cnt, d_counts, nullptr, nullptr, 0, 0, d_diag); break;
            default: k_enumerate<4><<<grid, 256, smem, stream>>>(a, s, cnt, d_counts, nullptr, nullptr, 0, 0, d_diag); break;
        }
        if (cudaGetLastError() != cudaSuccess) { fail(TB_ERR_CUDA, "count launch failed"); break; }
        cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_counts, d_offsets, int(cnt), stream);
        uint32_t last[2];
        cudaMemcpyAsync(&last[0], d_offsets + cnt - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(&last[1], d_counts + cnt - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
        if (cudaStreamSynchronize(stream) != cudaSuccess) { fail(TB_ERR_CUDA, "count pass failed"); break; }
        const uint64_t add = uint64_t(last[0]) + uint64_t(last[1]);
        if (add >= (uint64_t(1) << 31)) { fail(TB_ERR_CAPACITY, "more than 2^31 survivors in one chunk"); break; }
        if (add == 0) continue;
        if (n + int64_t(add) > outT.cap) {
            int64_t want = outT.cap;
            while (want < n + int64_t(add)) want *= 2;
            rc = outT.grow(L, want, n, stream);
            if (rc != TB_OK) break;
        }
        switch (L) {
            case 2: k_enumerate<2><<<grid, 256, smem, stream>>>(a, s, cnt, nullptr, d_offsets, outT.d, outT.cap, n, nullptr); break;
            case 3: k_enumerate<3><<<grid, 256, smem, stream>>>(a, s, cnt, nullptr, d_offsets, outT.d, outT.cap, n, nullptr); break;
            default: k_enumerate<4><<<grid, 256, smem, stream>>>(a, s, cnt, nullptr, d_offsets, outT.d, outT.cap, n, nullptr); break;
        }
        if (cudaGetLastError() != cudaSuccess) { fail(TB_ERR_CUDA, "write launch failed"); break; }
        n += int64_t(add);
    }
    if (rc == TB_OK) {
        unsigned long long h[3];
        cudaMemcpyAsync(h, d_diag, sizeof(h), cudaMemcpyDeviceToHost, stream);
        if (cudaStreamSynchronize(stream) != cudaSuccess) fail(TB_ERR_CUDA, "enumeration failed");
        diag[0] = int64_t(h[0]); diag[1] = int64_t(h[1]); diag[2] = int64_t(h[2]);
        outT.n = n;
    }
    cudaFree(d_counts);
    cudaFree(d_offsets);
    cudaFree(d_diag);
    cudaFree(d_tmp);
    return rc;
}

int DeviceTuples::reserve(int L, int64_t cap_, cudaStream_t stream) {
    release();
    if (cudaMalloc(&d, sizeof(int32_t) * size_t(L + 1) * size_t(cap_)) != cudaSuccess) {
        d = nullptr;
        set_error("tuple list allocation failed");
        return TB_ERR_OOM;
    }
    cap = cap_;
    n = 0;
    return TB_OK;
}

int DeviceTuples::grow(int L, int64_t cap_, int64_t keep, cudaStream_t stream) {
    int32_t* nd = nullptr;
    if (cudaMalloc(&nd, sizeof(int32_t) * size_t(L + 1) * size_t(cap_)) != cudaSuccess) {
        set_error("tuple list allocation failed while growing");
        return TB_ERR_OOM;
    }
    for (int r = 0; r <= L; ++r)
        if (keep > 0)
            cudaMemcpyAsync(nd + size_t(r) * cap_, d + size_t(r) * cap, sizeof(int32_t) * size_t(keep),
                            cudaMemcpyDeviceToDevice, stream);
    cudaStreamSynchronize(stream);
    cudaFree(d);
    d = nd;
    cap = cap_;
    return TB_OK;
}

void DeviceTuples::release() {
    if (d) cudaFree(d);
    d = nullptr;
    cap = 0;
    n = 0;
}

}  // namespace tb
