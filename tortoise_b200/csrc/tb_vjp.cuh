// tb_vjp.cuh -- transposed (vector-Jacobian) kernels of the right-hand side.
#pragma once

#include "tb_tensor.cuh"

namespace tb {

// u = M^-T theta per element (transpose of launch_inverse_mass).
int launch_minv_t(const ElemDev& ed, const double* theta, double* u, cudaStream_t s);

// Zero the entries of constrained bands (transpose of the constraint
// projection; the constrained values themselves carry no derivative).
int launch_project(const ElemDev& ed, double* v, cudaStream_t s);

// grad_f += C'(f)^T u and grad_amp[k] += <u, dC/d amplitude_k> for every
// instance k of one channel group (u is the pre-M^-1 co-state).  In the
// deterministic mode (fx.w non-null) the grad_f terms go to fx and the
// grad_amp terms to fx_amp (slot k) instead, as exact fixed-point adds.
int launch_collision_vjp(const ChanDev& c, const InstDev* insts, int n_insts, int layout, const MomentTensor& T,
                         const int32_t* tup, int64_t stride, int64_t n, const double* f, const double* u,
                         double* grad_f, double* grad_amp, cudaStream_t s, const uint64_t* mask = nullptr,
                         const int32_t* perm = nullptr, const FxAcc& fx = FxAcc{}, const FxAcc& fx_amp = FxAcc{});

// grad_f += V^T u (Vlasov drift); fx.w non-null: into fx instead.
int launch_drift_vjp(const ElemDev& ed, const double* u, double* grad_f, cudaStream_t s, const FxAcc& fx = FxAcc{});

}  // namespace tb
