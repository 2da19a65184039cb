// tb_theta.cuh -- simplex masks of the Monte-Carlo quadrature and the
// compacted tuple list the Monte-Carlo collision kernels walk.
#pragma once

#include "tb_common.cuh"
#include "tb_enumerate.cuh"

namespace tb {

// Tuples of one channel whose quadrature has at least one point inside the
// simplices, reordered for the kernel (see tb_theta.cu).  ids has the SoA
// layout of DeviceTuples (rows 0..L-1 element ids, row L umklapp index, row
// stride n); mask[i] bit m is ThetapC * ThetaFC of Monte-Carlo point m;
// perm[i] is the tuple's index in the channel's list (for per-tuple data
// such as functAmplitude).
struct ThetaList {
    int32_t* ids = nullptr;
    uint64_t* mask = nullptr;
    int32_t* perm = nullptr;
    int64_t n = 0;          // tuples in the list
    int64_t points = 0;     // set bits over the list (points inside)
    bool built = false;
    bool use = false;       // the collision kernels walk this list instead of the full one
    void release();
};

// Builds the list for the tuples tup[0, tup.n) of channel c (Monte-Carlo
// table c.mc, c.nmc <= 64).  On return out.built is false when the channel
// does not qualify (more than 64 points) or there was no room, and the full
// quadrature stays in use.
int build_theta_list(const ChanDev& c, const DeviceTuples& tup, ThetaList& out, cudaStream_t stream);

}  // namespace tb
