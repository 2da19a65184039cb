// tb_dp45.cuh -- device state of the Dormand-Prince 5(4) integrator.
#pragma once

#include "tb_kernels.cuh"

namespace tb {

#define TB_MAX_DENSE_PER_STEP 64

// Controller state, resident in device memory; only the controller kernel
// writes the scalars, every other kernel reads dt / done / skip / acc_now.
struct DPCtl {
    double t, dt, tf, dense_step, dense_time, min_step, olderror, last_err;
    double step_t, step_dt;   // time and step size of the attempt just decided
    int rejected;       // previous attempt rejected (caps the next growth at 1)
    int done;           // integration finished or failed: later attempts no-op
    int skip;           // this attempt was a no-op (done was already set)
    int acc_now;        // this attempt was accepted
    int status;         // TB_OK / TB_ERR_DT_UNDERFLOW / TB_ERR_NONFINITE / TB_ERR_CAPACITY
    int n_now;          // dense outputs scheduled in this attempt
    long long attempts, accepted, rejected_n, rhs_evals;
    long long n_dense;  // dense outputs produced so far (may exceed capacity -> status)
    long long dense_cap;
    double dense_s[TB_MAX_DENSE_PER_STEP];
    double dense_t[TB_MAX_DENSE_PER_STEP];
    long long max_attempts;  // 0 = unbounded
};

struct DPBufs {
    double* y;       // current state
    double* tmp;     // stage input
    double* y5;      // 5th-order solution (stage-7 input)
    double* k[7];    // stages k1..k7
    double* acc;     // pre-M^-1 RHS accumulator (zero between evaluations)
    double* part;    // [2 * nb * nblk] error-norm partial sums
    int nblk;        // blocks of the element-wise kernels
    double* dense;   // [dense_cap * ndofs]
    double* dense_t; // [dense_cap]
    DPCtl* ctl;
};

// Stage kernel s (0..6) of one attempt:
//   s == 0:  tmp = enforce(y + a21 dt k1)
//   1..4  :  k_{s+1} = acc M^-1, acc = 0, tmp = enforce(y + sum_j a_{s+2,j} dt k_j)
//   5     :  k6 = acc M^-1, acc = 0, y5 = enforce(y + sum_j b_j dt k_j)
//   6     :  k7 = acc M^-1, acc = 0, err = y5 - enforce(y + sum_j bh_j dt k_j) and
//            the per-band error-norm partials.
int launch_stage(const BandsDev& bands, const DPBufs& B, int s, cudaStream_t st);
int launch_controller(const BandsDev& bands, const DPBufs& B, cudaStream_t st);
int launch_dense_commit(const BandsDev& bands, const DPBufs& B, cudaStream_t st);
// k1 = M^-1 acc, acc = 0 (first evaluation of an integration).
int launch_k1(const BandsDev& bands, const DPBufs& B, cudaStream_t st);
// dst = enforce(src)  (applyConstraints)
int launch_enforce(const BandsDev& bands, const double* src, double* dst, cudaStream_t st);
// Band::relativeError partial sums for arbitrary err/pop (diagnostics, tests).
int launch_error_norm(const BandsDev& bands, const double* err, const double* pop, double* part, int nblk,
                      cudaStream_t st);

}  // namespace tb
