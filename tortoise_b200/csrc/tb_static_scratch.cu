// tb_static_scratch.cu -- the error norm of one band computed without any
// device allocation at call time.
//
// Who needs it: callers that cannot call cudaMalloc at the moment they need
// the norm.  Typical cases are a host application whose device memory is
// entirely reserved by its own pool allocator (a fresh cudaMalloc would fail
// or fragment the pool), and callers that must not risk the implicit device
// synchronisation a cudaMalloc / cudaFree can cause in the middle of their
// own asynchronous work.  They pass device buffers for the inputs and the
// result; the per-block partial sums live in a fixed array that the library
// declares at file scope.
//
// The array is `g_noalloc_scratch` below: TB_NOALLOC_SCRATCH_DOUBLES doubles
// (64 KiB) on every device that loads this library, held until the process
// exits.  Host code must not pass the array's name to a kernel (on the host it
// is only a stand-in, not a device address); the device address is obtained
// once per device with cudaGetSymbolAddress while that device is current, on
// the first call made on that device, and reused afterwards.  It belongs to
// the device's primary context: after a cudaDeviceReset the kept address is
// stale, so a process that resets a device must not call in again there.
//
// All calls share the one array, which keeps the last call's contents.  Every
// entry a call reads is written earlier in the same call, so nothing has to
// be cleared; but two calls whose kernels overlap on the GPU (different
// streams, or different host threads on the same device) race on it.
#include <mutex>

#include "tb_errnorm.cuh"

namespace tb {

#define TB_NOALLOC_SCRATCH_DOUBLES 8192
#define TB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double g_noalloc_scratch[TB_NOALLOC_SCRATCH_DOUBLES];

static double* g_noalloc_addr[TB_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device (set-up on the
// first call per device).
static int noalloc_scratch(double** out) {
    int dev = -1;
    TB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= TB_NOALLOC_MAX_DEVICES) {
        set_error("device ordinal beyond the scratch table of the no-allocation entry point");
        return TB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cudaGetSymbolAddress of the static scratch array failed: ") + cudaGetErrorString(e));
            return TB_ERR_CUDA;
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return TB_OK;
}

__global__ void __launch_bounds__(256) k_band_error_partials_static(BandDev bd, const double* __restrict__ err,
                                                                    const double* __restrict__ pop,
                                                                    double* __restrict__ part, int nblk) {
    __shared__ double sh[8];
    double r = 0.0, p = 0.0;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < bd.ne) elem_rel_err(bd, err + 3 * (int64_t)e, pop + 3 * (int64_t)e, r, p);
    const double rs = block_sum<256>(r, sh);
    const double ps = block_sum<256>(p, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = rs;
        part[nblk + blockIdx.x] = ps;
    }
}

__global__ void k_band_error_finish_static(BandDev bd, const double* __restrict__ part, int nblk,
                                           double* __restrict__ result) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sr = 0.0, sp = 0.0;
    for (int k = 0; k < nblk; ++k) {
        sr = __dadd_rn(sr, part[k]);
        sp = __dadd_rn(sp, part[nblk + k]);
    }
    const double ir = __dmul_rn(bd.mesh.vol, sr), ip = __dmul_rn(bd.mesh.vol, sp);
    *result = sqrt(__ddiv_rn(__dadd_rn(ir, __dmul_rn(bd.penal, ip)), __dmul_rn(double(bd.ne), bd.mesh.vol)));
}

}  // namespace tb

using namespace tb;

extern "C" int tb_band_relative_error_noalloc(const double* err, const double* pop, int64_t n_elements,
                                              double elem_volume, double statistics, double rel_tol, double abs_tol,
                                              double penalisation, double* result, void* stream) {
    if (!err || !pop || !result) { set_error("null argument"); return TB_ERR_ARG; }
    if (n_elements <= 0) { set_error("n_elements must be > 0"); return TB_ERR_ARG; }
    if (statistics != TB_FERMION && statistics != TB_BOSON) {
        set_error("statistics must be -1 (fermion) or +1 (boson)");
        return TB_ERR_ARG;
    }
    const int64_t nblk = (n_elements + 255) / 256;
    if (2 * nblk > TB_NOALLOC_SCRATCH_DOUBLES) {
        set_error("tb_band_relative_error_noalloc: " + std::to_string(n_elements) +
                  " elements exceed the static scratch limit of " +
                  std::to_string(int64_t(TB_NOALLOC_SCRATCH_DOUBLES / 2) * 256) + " elements");
        return TB_ERR_CAPACITY;
    }
    double* scratch = nullptr;
    TB_TRY(noalloc_scratch(&scratch));
    BandDev bd{};
    bd.ne = int(n_elements);
    bd.mesh.ne = int(n_elements);
    bd.mesh.vol = elem_volume;
    bd.stat = statistics;
    bd.rel_tol = rel_tol;
    bd.abs_tol = abs_tol;
    bd.penal = penalisation;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_band_error_partials_static<<<unsigned(nblk), 256, 0, s>>>(bd, err, pop, scratch, int(nblk));
    TB_CUDA(cudaGetLastError());
    k_band_error_finish_static<<<1, 32, 0, s>>>(bd, scratch, int(nblk), result);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}
