// tb_probe.cu -- the FP64 FMA throughput of the device, the roofline
// denominator of the FP64-bound kernels (the batched run-minor contraction,
// the Monte-Carlo quadrature).
//
// Every thread runs 8 independent FMA chains x <- x a + b in registers
// (a = 1 - 2^-20, b = 2^-20: the chains stay near 1, no overflow, no
// subnormals), enough independent work per warp to keep the FP64 pipe busy;
// the grid fills every SM with 8 blocks of 256 threads.  The rate is the FMA
// count over the CUDA-event time of the launch, after a warm-up launch.
#include "tb_common.cuh"

namespace tb {

constexpr int PROBE_CHAINS = 8;

__global__ void __launch_bounds__(256) k_dfma_rate(double* out, int iters, double a, double b) {
    double x[PROBE_CHAINS];
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k) x[k] = 1.0 + double(threadIdx.x + k) * 1e-6;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < PROBE_CHAINS; ++k) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k) s += x[k];
    if (s == -1.0) out[0] = s;   // never true: keeps the chains alive
}

}  // namespace tb

using namespace tb;

extern "C" int tb_fp64_fma_rate(int device, double* fma_per_second) {
    if (!fma_per_second) { set_error("null argument"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(device));
    int nsm = 0;
    TB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    cudaStream_t s = nullptr;
    TB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double* out = nullptr;
    int rc = TB_OK;
    const unsigned blocks = unsigned(nsm) * 8u;
    const int iters = 2048;
    const double a = 1.0 - 0x1p-20, b = 0x1p-20;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaMalloc(&out, sizeof(double)) != cudaSuccess) {
        set_error("probe set-up failed");
        rc = TB_ERR_CUDA;
    } else {
        k_dfma_rate<<<blocks, 256, 0, s>>>(out, iters / 8, a, b);   // warm-up (clocks, module load)
        cudaEventRecord(e0, s);
        k_dfma_rate<<<blocks, 256, 0, s>>>(out, iters, a, b);
        cudaEventRecord(e1, s);
        float ms = 0.f;
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || !(ms > 0.f)) {
            set_error("probe launch failed");
            rc = TB_ERR_CUDA;
        } else {
            *fma_per_second = double(blocks) * 256.0 * double(iters) * PROBE_CHAINS / (1e-3 * double(ms));
        }
    }
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    return rc;
}
