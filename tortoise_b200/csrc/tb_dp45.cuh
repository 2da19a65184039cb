// tb_dp45.cuh -- device state of the Dormand-Prince 5(4) integrator.
#pragma once

#include "tb_kernels.cuh"

namespace tb {

#define TB_MAX_DENSE_PER_STEP 64
// dense outputs per step with time-dependent constraints (TB_ERR_CAPACITY beyond)
#define TB_TC_DENSE TB_TC_DENSE_PER_STEP
// slots of time-dependent constrained values per attempt: the stage times
// t + c2 dt, t + c3 dt, t + c4 dt, t + c5 dt, t + dt, then the dense times
#define TB_TC_SLOTS (5 + TB_TC_DENSE)

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
    long long last_dense_step;  // index (among accepted steps) of the step that made the last dense output
    double last_dense_s;        // its dense-output fraction s in (0, 1.0001]
    // time-dependent constraints (written by the host node before an attempt)
    int veto_pending;           // an accepted step left timeStepVetoer to the host
    int tc_ndense;              // dense times with constrained values in this attempt's slots
    double tc_dense_t[TB_TC_DENSE];
};

// Per-run layout inside the concatenated state of a batch.
struct RunDev {
    int band0, nbands;      // global band range of the run
    int blk0, blk1;         // element-block range of its bands
    int64_t dof_off, ndofs; // state slice
    int64_t dense_off;      // offset (doubles) of its dense-output block
    int64_t dense_t_off;    // offset of its dense-time block
};

struct DPBufs {
    double* y;       // current state (all runs)
    double* tmp;     // stage input
    double* y5;      // 5th-order solution (stage-7 input)
    double* k[7];    // stages k1..k7
    double* acc;     // pre-M^-1 RHS accumulator (zero between evaluations)
    double* part;    // [2 * nblk] error-norm partial sums per element block
    int nblk;
    int nruns;
    const RunDev* runs;   // [nruns]
    double* dense;   // per-run dense blocks [slot][ndofs_run]
    double* dense_t; // per-run dense times [slot]
    DPCtl* ctl;      // [nruns]
    // adjoint recording (single run; null in a plain integration):
    // step_log[2 n], step_log[2 n + 1] = t, dt of accepted step n;
    // ckpt[c] = y after accepted step c * ckpt_every (ckpt[0] = enforced y0)
    double* step_log;
    long long log_cap;
    double* ckpt;
    long long ckpt_every;
    long long ckpt_cap;
    // time-dependent constraints (tc = 1): the constrained bands' values at
    // the attempt's times, [TB_TC_SLOTS][cdofs] (BandDev::coff within a slot)
    const double* ctv;
    long long cdofs;
    int tc;
};

// Stage kernel s (0..6) of one attempt:
//   s == 0:  tmp = enforce(y + a21 dt k1)
//   1..4  :  k_{s+1} = acc M^-1, acc = 0, tmp = enforce(y + sum_j a_{s+2,j} dt k_j)
//   5     :  k6 = acc M^-1, acc = 0, y5 = enforce(y + sum_j b_j dt k_j)
//   6     :  k7 = acc M^-1, acc = 0, err = y5 - enforce(y + sum_j bh_j dt k_j) and
//            the per-band error-norm partials.
int launch_stage(const ElemDev& ed, const DPBufs& B, int s, cudaStream_t st);
int launch_controller(const ElemDev& ed, const DPBufs& B, cudaStream_t st);
int launch_dense_commit(const ElemDev& ed, const DPBufs& B, cudaStream_t st);
// k1 = M^-1 acc, acc = 0 (first evaluation of an integration).
int launch_k1(const ElemDev& ed, const DPBufs& B, cudaStream_t st);
// dst = enforce(src)  (applyConstraints); cv: one slot of time-dependent
// constrained values, or null for the bands' constant populations
int launch_enforce(const ElemDev& ed, const double* src, double* dst, cudaStream_t st, const double* cv = nullptr);
// Band::relativeError partial sums per element block for arbitrary err/pop:
// part[blk] (relative term), part[nblk + blk] (penalisation term).
int launch_error_norm(const ElemDev& ed, const double* err, const double* pop, double* part, cudaStream_t st);

}  // namespace tb
