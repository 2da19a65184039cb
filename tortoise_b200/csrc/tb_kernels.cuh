// tb_kernels.cuh -- launch wrappers of the element-wise and tuple kernels.
#pragma once

#include "tb_common.cuh"
#include "tb_exact.cuh"

namespace tb {

struct DPCtl;

// One run's use of a shared channel: where its bands live in the global
// state and its coupling constant.  Runs with identical structure share the
// channel's tuple list (and moment tensor); each run is one instance.
struct InstDev {
    int64_t foff[TB_MAX_LEGS];  // band offsets of the run's legs in the state
    double amp_full;            // amplitude * prod_l (vol_l * 2)  (Monte-Carlo path)
    double amplitude;           // amplitude                     (moment-tensor path)
    int run;
    int pad;
};

// Element-wise work over every band of every run.  Blocks of 256 elements;
// block b belongs to band blk_band[b] and covers elements
// (b - blk_first[band]) * 256 + [0, 256).
struct ElemDev {
    const BandDev* bands;       // [nb]
    const int* band_run;        // [nb]
    const int* blk_band;        // [nblk]
    const int* blk_first;       // [nb + 1]
    int nb;
    int nblk;
    int64_t ndofs;
};

// Collision contribution of one channel for every instance in `insts`
// (before M^-1), added into acc.  ctl (per run, may be null) lets finished
// runs skip their work inside a batched integration.  rate_leg >= 0 computes
// instead the scattering rate of that leg (its forms replaced by the in / out
// unit forms, only its block kept, with the opposite sign).  mask / perm
// non-null: tup, stride, n describe a ThetaList (tb_theta.cuh) and only the
// points inside the simplices are evaluated.
// fx.w non-null (deterministic mode): the results go to the exact fixed-point
// accumulator fx (tb_exact.cuh) instead of acc.
int launch_collision_mc(const ChanDev& c, const InstDev* insts, int n_insts, const int32_t* tup, int64_t stride,
                        int64_t n, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s, int grid_hint,
                        int rate_leg = -1, const uint64_t* mask = nullptr, const int32_t* perm = nullptr,
                        const FxAcc& fx = FxAcc{});

// acc[i] += fx slot i for i < n (rounded once to FP64), then the slots are
// cleared; a poisoned buffer writes NaN into every acc[i] instead and the
// poison word is cleared too.
int launch_fx_flush(const FxAcc& fx, double* acc, int64_t n, cudaStream_t s);

// Vlasov drift (volume minus upwind surface term, before M^-1) of every band
// with a nonzero drift velocity, added into acc.
int launch_drift(const ElemDev& ed, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s);

// out = acc * M^-1 per element (Function::applyInverseMass).
int launch_inverse_mass(const ElemDev& ed, const double* acc, double* out, cudaStream_t s);

}  // namespace tb
