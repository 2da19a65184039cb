// tb_enumerate.cuh -- device tuple lists and the enumeration entry point.
#pragma once

#include "tb_common.cuh"

namespace tb {

// SoA tuple storage: rows 0..L-1 hold element ids of each leg, row L the
// umklapp column index; every row has length `cap`, the first `n` are valid.
struct DeviceTuples {
    int32_t* d = nullptr;
    int64_t cap = 0;
    int64_t n = 0;
    int reserve(int L, int64_t cap, cudaStream_t stream);
    int grow(int L, int64_t cap, int64_t keep, cudaStream_t stream);
    void release();
};

int enumerate_channel(const ChanDev& c, const HostMesh* meshes, const HostBand* bands, const int* leg_band,
                      const double* d_mc_pre, const double* const* d_minE, const double* const* d_maxE,
                      cudaStream_t stream, DeviceTuples& out, int64_t diag[3]);

}  // namespace tb
