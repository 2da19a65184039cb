// tb_common.cuh -- shared device/host definitions of the tortoise_b200 library.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/tortoise_b200.h"

namespace tb {

// ----------------------------------------------------------------- errors
void set_error(const std::string& msg);
const char* get_error();

#define TB_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t _e = (call);                                                       \
        if (_e != cudaSuccess) {                                                       \
            ::tb::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));      \
            return TB_ERR_CUDA;                                                        \
        }                                                                              \
    } while (0)

// A named range on the NVTX timeline around a host-side phase of the library
// (handle creation and its steps, right-hand sides, integrations, adjoint
// sweeps), for Nsight tools (e.g. ncu --nvtx --nvtx-include "tb_rhs/").
// nvtx3 is header-only; with no tool attached a push / pop costs a few ns.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

#define TB_TRY(call)                      \
    do {                                  \
        int _rc = (call);                 \
        if (_rc != TB_OK) return _rc;     \
    } while (0)

// --------------------------------------------------------------- constants
// Order-2 Gauss rule on the reference triangle with the reference's 14-digit
// constants (GaussQuadratureConst.hpp:84-90) and on [0,1] (:60-61).
#define TB_GP2_A 0.16666666666667
#define TB_GP2_B 0.66666666666667
#define TB_GW2 0.33333333333333
#define TB_GP1_0 0.2113248654051871
#define TB_GP1_1 0.7886751345948129

// ------------------------------------------------------------ host mirrors
struct HostMesh {
    int nx, ny, ne;
    double origin[2];
    double dG[2][2];
    double invdG[2][2];
    double vol;
    double rel_origin[2];
    double M[3][3], Minv[3][3];
};

struct HostBand {
    int mesh, ne;
    int64_t off;
    double charge, stat, abs_tol, rel_tol, penal;
    int constrained;
    double vel[2];
    std::vector<double> disp, kx, ky, minE, maxE, cpop;
};

// ---------------------------------------------------- device-side records
// Everything a kernel needs about one leg of a channel.
struct LegDev {
    const double* disp;   // [ne*3]
    const double* kx;     // [ne*3]
    const double* ky;     // [ne*3]
    int64_t foff;         // band offset in the status vector
    double dir;           // +1 in, -1 out
    double stat;          // -1 fermion, +1 boson
    int ne;
    // The leg's loss / gain forms (ScatteringChannel.cpp:633-641),
    //   A_j = ka ((1 - d) [j = 0] + ca f_j),  B_j = 1/2 ((1 + d) [j = 0] + cb f_j),
    // as A_j = fa f_j + fa0 [j = 0], B_j = fb f_j + fb0 [j = 0]: ka = -1/2 on
    // leg 0 and 1/2 elsewhere, ca, cb = +-2, so every folded product is exact
    // and the forms round exactly as the unfolded ones.
    double fa, fa0, fb, fb0;
};

struct ChanDev {
    int L;
    int nmc;
    int R;                // MC table row length 2*(L-2)+1
    int n_umk;
    LegDev leg[TB_MAX_LEGS];
    double amp_vol;       // prod_l (elemVolume_l * 2) (constructAmplitude without amplitude)
    double fact;          // (NDim!)^(L-2) * (NDim-1)!
    double min_det;
    double threshold;
    double gvec[4];       // region gVec, column-major
    const double* umk;    // [n_umk*2] device
    const double* mc;     // [nmc*R] device
    // functAmplitude at the tuple's element barycentres, one factor per tuple
    // of the group's list (ScatteringChannel.cpp:399-415); null: 1
    const double* tamp = nullptr;
    // Shared-memory accumulation (Monte-Carlo kernels): one instance's block
    // holds the distinct bands of the legs as segments of 3 ne doubles each.
    int nseg = 0;
    int sinst = 0;                    // doubles per instance (all segments)
    int sseg[TB_MAX_LEGS] = {};       // per leg: offset of its band's segment
    int seg_off[TB_MAX_LEGS] = {};    // per segment: offset in the block
    int seg_leg[TB_MAX_LEGS] = {};    // per segment: a leg of that band (its foff)
    // Moment-tensor contractions: the handle's flag that a bounded wait for a
    // staged tile ran out (then TB_ERR_TIMEOUT), and that wait's poll limit
    // (tb_set_copy_wait_limit).
    int* err_flag = nullptr;
    int wait_polls = 1 << 22;
};

// Mesh data needed by the element-wise kernels.
struct MeshDev {
    int nx, ny, ne;
    double dG[2][2];
    double vol;
    double rel_origin[2];
    double Minv[3][3];
    double M[3][3];
};

// Element-wise per-band record (drift, inverse mass, error norm, constraints).
struct BandDev {
    MeshDev mesh;
    int64_t off;
    int ne;
    double stat, abs_tol, rel_tol, penal;
    int constrained;
    const double* cpop;   // device, [ne*3] or null
    int64_t coff;         // offset of the band in a slot of time-dependent constrained values (-1: none)
    double vel[2];
};

}  // namespace tb
