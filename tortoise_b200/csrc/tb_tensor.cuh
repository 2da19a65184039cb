// tb_tensor.cuh -- precomputed moment tensors of the collision operator.
#pragma once

#include "tb_kernels.cuh"

namespace tb {

// storage kinds of the moments (see tb_tensor.cu)
enum { TK_F64 = 0, TK_F32 = 1, TK_F40 = 2, TK_F48 = 3 };

struct MomentTensor {
    void* d = nullptr;        // moments, tile-major (see tb_tensor.cu)
    int64_t n = 0;            // tuples
    int64_t ntiles = 0;
    int nmom = 0;             // moments per tuple
    int kind = TK_F64;
    // contraction schedule (set by tune_tensor): bulk-copy pipeline stages,
    // and whether groups with several instances contract two per moment read
    int stages = 2;
    int pair = 1;
    double tuned_seconds = 0.0;   // best measured launch time (0: not tuned)
    // run-minor contraction for a group shared by many runs (k_collision_runs
    // in tb_tensor.cu): runs = the lane-group width (4, 8 or 32 runs per
    // tuple), 0 = off; the buffers come from prepare_runs
    int runs = 0;
    int np = 0;                   // instances rounded up to a multiple of 32
    int runs_distinct = 0;        // every instance belongs to another run
    double* fT = nullptr;         // [leg][3 ne_leg][np]: the legs' f, run-minor
    double* accT = nullptr;       // same shape; all zero between launches
    unsigned long long* accTx = nullptr;   // deterministic mode: accT's exact twin
                                           // (3 words per slot, tb_exact.cuh); zero between launches
    int64_t loff[4] = {0, 0, 0, 0};
    void release();
};

int64_t tensor_bytes(int L, int kind, int64_t n_tuples);
// tuples per tile of the tile-major moment layout
int tile_tuples(int L, int kind);
int build_tensor(const ChanDev& c, const int32_t* tup, int64_t stride, int64_t n, int kind, MomentTensor& T,
                 cudaStream_t s);
// Recomputes the moments of an existing tensor in place (same list, kind,
// schedule and run-minor buffers), e.g. after the channel's per-tuple
// amplitudes (ChanDev::tamp) changed.
int refill_tensor(const ChanDev& c, const int32_t* tup, int64_t stride, int64_t n, MomentTensor& T, cudaStream_t s);
// rate_leg >= 0: scattering rate of that leg instead (see launch_collision_mc);
// fx.w non-null: deterministic mode, the results go to fx instead of acc
int launch_collision_tensor(const ChanDev& c, const InstDev* insts, int n_insts, const MomentTensor& T,
                            const int32_t* tup, int64_t stride, int64_t n, const double* f, double* acc,
                            const DPCtl* ctl, cudaStream_t s, int rate_leg = -1, const FxAcc& fx = FxAcc{});

// Buffers of the run-minor contraction for a group of n_insts instances
// (legs <= 3, 8 <= n_insts <= 1024); sets runs = 8 from 16 instances on.
// exact: also the fixed-point twin of the accumulator (deterministic mode).
// Does nothing for other groups, or when the device memory is short.
int prepare_runs(const ChanDev& c, int n_insts, bool distinct_runs, MomentTensor& T, cudaStream_t s,
                 bool exact = false);

// Autotuner: times the contraction of one group for every schedule
// (stages 1 / 2, instance pairs off / on where several instances exist, the
// run-minor contraction where prepare_runs gave it buffers) on
// the device data and keeps the fastest in T.  f is any state of the handle's
// size; acc is scratch (left dirty).  A process-wide cache keyed by
// (legs, storage kind, tuple count, instance count) skips repeated timing.
int tune_tensor(const ChanDev& c, const InstDev* insts, int n_insts, MomentTensor& T, const int32_t* tup,
                int64_t stride, int64_t n, const double* f, double* acc, cudaStream_t s);

// *value = 1 when a bounded wait of a contraction kernel ran out since the
// last call (the handle's flag, ChanDev::err_flag; then TB_ERR_TIMEOUT), and
// the flag is cleared.  Waits for s (the stream the kernels ran on).
int take_wait_timeout(int* flag, cudaStream_t s, int* value);

}  // namespace tb
