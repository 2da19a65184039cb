// tb_kernels.cuh -- launch wrappers of the element-wise and tuple kernels.
#pragma once

#include "tb_common.cuh"

namespace tb {

#define TB_MAX_BANDS 8

struct BandsDev {
    int nb;
    int64_t ndofs;
    BandDev b[TB_MAX_BANDS];
};

// Layout of the per-tuple moment tensor used by the precomputed-tensor
// contraction (see tb_tensor.cu).
enum TensorPrec { TENSOR_NONE = 0, TENSOR_F64 = 1, TENSOR_F32 = 2 };

// Collision contribution of one channel (before M^-1), added into acc:
// Monte-Carlo quadrature evaluated per tuple (scatteringIntegrationTypeB).
int launch_collision_mc(const ChanDev& c, double amp_full, const int32_t* tup, int64_t stride, int64_t n,
                        const double* f, double* acc, const int* done, cudaStream_t s, int grid_hint);

// Vlasov drift (volume minus upwind surface term, before M^-1) of every band
// with a nonzero drift velocity, added into acc.
int launch_drift(const BandsDev& bands, const double* f, double* acc, const int* done, cudaStream_t s);

// out = acc * M^-1 per element (Function::applyInverseMass).
int launch_inverse_mass(const BandsDev& bands, const double* acc, double* out, cudaStream_t s);

}  // namespace tb
