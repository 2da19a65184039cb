// tb_adjoint.cu -- discrete adjoint of the Dormand-Prince 5(4) integration.
//
// No counterpart in the reference.  The reference integrates with
// Algorithms::dormandPrince54 (include/Generics/Algorithms/
// DormandPrince54.hpp:479-665); this file differentiates exactly the map its
// accepted steps apply, with the step sizes frozen at the values the forward
// controller chose (the dependence of dt on f is not differentiated):
//
//   Y_1 = y_n,  Y_i = P(y_n + dt sum_{j<i} a_ij k_j) + c,  k_i = F(Y_i)
//   y_{n+1}     = P(y_n + dt sum_j b_j k_j) + c
//   f(t_obs)    = P(y_m + dt sum_j s bt_j(s) k_j) + c        (dense output)
//
// with P the projection that zeroes constrained bands and c their fixed
// populations (MaterialStatus::applyConstraints, MaterialStatus.cpp:198-206).
// The observable is J = <lambda_T, f(t_obs)> at the last dense output.
// Reverse sweep of one step, incoming co-state lam of y_{n+1}:
//   v = P lam;  lam <- v;  D_j = dt b_j v
//   for i = 6..1:  mu = F'(Y_i)^T D_i  (tb_vjp.cu),  g_amp += dF/damp^T D_i
//                  nu = (i > 1 ? P mu : mu);  lam += nu;  D_j += dt a_ij nu (j < i)
// Memory: the forward sweep stores y every `every` accepted steps
// (checkpoints) and the (t, dt) of each accepted step.  The reverse sweep
// walks the segments backwards; per segment it replays `every` steps from
// the checkpoint with the frozen dt, keeping the 6 stage inputs of each step
// (6 every + 1 states), then runs the reverse steps over them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tb_handle.cuh"
#include "tb_vjp.cuh"

namespace tb {

// Butcher tableau, DormandPrince54.hpp:502-511 (the same values as tb_dp45.cu)
static const double kA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1. / 5., 0, 0, 0, 0, 0},
    {3. / 40., 9. / 40., 0, 0, 0, 0},
    {44. / 45., -56. / 15., 32. / 9., 0, 0, 0},
    {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729., 0, 0},
    {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656., 0},
    {0, 0, 0, 0, 0, 0}};
static const double kB[6] = {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.};

// Dense-output weights bt_j(s), DormandPrince54.hpp:598-611 (bt_2 = 0).
static void dense_weights(double s, double bt[7]) {
    bt[0] = -(435. * s * s * s - 1184. * s * s + 1098. * s - 384.) / (384.);
    bt[1] = 0.0;
    bt[2] = 500. * s * (6. * s * s - 14. * s + 9.) / (1113.);
    bt[3] = -125. * s * (9. * s * s - 16. * s + 6.) / (192.);
    bt[4] = 729. * s * (35. * s * s - 64. * s + 26.) / (6784.);
    bt[5] = -11. * s * (3. * s - 2.) * (5. * s - 6.) / (84.);
    bt[6] = s * (s - 1.) * (5. * s - 3.) / (2.);
}

struct AdjointState {
    int64_t ndofs = 0;
    int every = 0;
    int64_t max_steps = 0;
    int64_t ckpt_cap = 0;
    double* ckpt = nullptr;    // [ckpt_cap][ndofs]
    double* log = nullptr;     // [2 max_steps] (t, dt) of accepted steps
    double* seg = nullptr;     // [6 every + 1][ndofs] stage inputs of one segment
    double* k[7] = {};         // stage derivatives (replay)
    double* D[6] = {};         // stage co-states
    double** dD = nullptr;     // device copy of the D pointers
    double* lam = nullptr;     // co-state of y
    double* lam_T = nullptr;   // observable weights (device copy)
    double* nud = nullptr;     // P lam_T
    double* u = nullptr;       // M^-T D_i
    double* g = nullptr;       // VJP accumulator
    double* ry = nullptr;      // replay: y, stage input, next y
    double* rtmp = nullptr;
    double* ry5 = nullptr;
    double* gamp = nullptr;    // [slots] amplitude gradients, group-major
    FxAcc gamp_fx{};           // deterministic mode: gamp's exact accumulator
    std::vector<int> gamp_off; // per group
    int n_slots = 0;
    // last forward sweep
    bool have_forward = false;
    int flags = 0;
    int64_t n_steps = 0;       // steps up to and including the observable's step
    int64_t attempts = 0;
    int64_t n_ckpt = 0;
    double dense_s = 1.0;
    double t_obs = 0.0;
    std::vector<double> step_dt;
    int64_t rhs_evals = 0;
    int64_t vjp_evals = 0;
    std::vector<void*> allocs;
};

static double* adj_alloc(AdjointState* A, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * (n ? n : 1)) != cudaSuccess) return nullptr;
    A->allocs.push_back(p);
    return static_cast<double*>(p);
}

void adjoint_release(tb_handle* h) {
    if (!h || !h->adj) return;
    for (void* p : h->adj->allocs) cudaFree(p);
    delete h->adj;
    h->adj = nullptr;
}

// Buffers independent of the step budget (replay tool, reverse sweep).
static int adj_base(tb_handle* h) {
    if (!h->adj) h->adj = new AdjointState();
    AdjointState* A = h->adj;
    if (A->lam) return TB_OK;
    const size_t n = size_t(h->ndofs);
    A->ndofs = h->ndofs;
    for (int i = 0; i < 7; ++i) A->k[i] = adj_alloc(A, n);
    for (int i = 0; i < 6; ++i) A->D[i] = adj_alloc(A, n);
    A->lam = adj_alloc(A, n);
    A->lam_T = adj_alloc(A, n);
    A->nud = adj_alloc(A, n);
    A->u = adj_alloc(A, n);
    A->g = adj_alloc(A, n);
    A->ry = adj_alloc(A, n);
    A->rtmp = adj_alloc(A, n);
    A->ry5 = adj_alloc(A, n);
    A->gamp_off.assign(h->groups.size() + 1, 0);
    for (size_t gi = 0; gi < h->groups.size(); ++gi)
        A->gamp_off[gi + 1] = A->gamp_off[gi] + int(h->groups[gi].insts.size());
    A->n_slots = A->gamp_off.back();
    A->gamp = adj_alloc(A, size_t(std::max(A->n_slots, 1)));
    if (h->opts.deterministic) {
        // 3 words per slot and the poison word, in double-sized units
        double* p3 = adj_alloc(A, size_t(3 * std::max(A->n_slots, 1) + 1));
        if (p3) {
            TB_CUDA(cudaMemset(p3, 0, sizeof(double) * size_t(3 * std::max(A->n_slots, 1) + 1)));
            A->gamp_fx.w = reinterpret_cast<unsigned long long*>(p3);
            A->gamp_fx.poison = reinterpret_cast<unsigned int*>(A->gamp_fx.w + 3 * std::max(A->n_slots, 1));
            A->gamp_fx.sat = h->fx.sat;   // one sticky flag per handle
        }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(double*) * 6) == cudaSuccess) {
        A->allocs.push_back(p);
        A->dD = static_cast<double**>(p);
    }
    bool ok = A->lam && A->lam_T && A->nud && A->u && A->g && A->ry && A->rtmp && A->ry5 && A->gamp && A->dD &&
              (!h->opts.deterministic || A->gamp_fx.w);
    for (int i = 0; i < 7; ++i) ok = ok && A->k[i];
    for (int i = 0; i < 6; ++i) ok = ok && A->D[i];
    if (!ok) {
        adjoint_release(h);
        set_error("adjoint allocation failed");
        return TB_ERR_OOM;
    }
    TB_CUDA(cudaMemset(A->g, 0, sizeof(double) * n));
    TB_CUDA(cudaMemcpy(A->dD, A->D, sizeof(double*) * 6, cudaMemcpyHostToDevice));
    return TB_OK;
}

// Step log, checkpoints and the segment store for a given budget.
static int adj_budget(tb_handle* h, int every, int64_t max_steps) {
    TB_TRY(adj_base(h));
    AdjointState* A = h->adj;
    const size_t n = size_t(h->ndofs);
    if (A->every != every || A->max_steps < max_steps) {
        auto drop = [&](double*& p) {
            if (!p) return;
            cudaFree(p);
            A->allocs.erase(std::remove(A->allocs.begin(), A->allocs.end(), (void*)p), A->allocs.end());
            p = nullptr;
        };
        drop(A->ckpt);
        drop(A->log);
        drop(A->seg);
        A->every = every;
        A->max_steps = max_steps;
        A->ckpt_cap = max_steps / every + 2;
        A->ckpt = adj_alloc(A, size_t(A->ckpt_cap) * n);
        A->log = adj_alloc(A, size_t(2 * max_steps));
        A->seg = adj_alloc(A, size_t(6 * every + 1) * n);
        if (!A->ckpt || !A->log || !A->seg) {
            set_error("adjoint checkpoint allocation failed");
            A->every = 0;
            A->max_steps = 0;
            return TB_ERR_OOM;
        }
    }
    return TB_OK;
}

// ------------------------------------------------------------ kernels
struct Combo {
    const double* y;
    const double* k[7];
    double c[7];
    int use[7];
};

// k_{j} = acc M^-1, acc = 0; out = P(y + sum_{use} c_j k_j) + c, in the
// summation order of the forward stage kernels (j ascending).
// kout is one of cb.k (the combination reads the value just written), so no
// pointer here is declared __restrict__.
__global__ void __launch_bounds__(256) k_replay_stage(ElemDev ed, double* acc, double* kout, Combo cb, double* out) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    {
        const double x = acc[o], y = acc[o + 1], z = acc[o + 2];
#pragma unroll
        for (int j = 0; j < 3; ++j) kout[o + j] = x * bd.mesh.Minv[0][j] + y * bd.mesh.Minv[1][j] + z * bd.mesh.Minv[2][j];
        acc[o] = 0.0; acc[o + 1] = 0.0; acc[o + 2] = 0.0;
    }
    if (!out) return;
    double v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double t = cb.y[o + c];
#pragma unroll
        for (int j = 0; j < 7; ++j)
            if (cb.use[j]) t = t + cb.c[j] * cb.k[j][o + c];
        v[c] = t;
    }
    if (bd.constrained) {
        const double* cp = bd.cpop + 3 * (int64_t)e;
        v[0] = cp[0]; v[1] = cp[1]; v[2] = cp[2];
    }
    out[o] = v[0]; out[o + 1] = v[1]; out[o + 2] = v[2];
}

__device__ __forceinline__ void minv_apply(const BandDev& bd, const double d[3], double u[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i) u[i] = bd.mesh.Minv[i][0] * d[0] + bd.mesh.Minv[i][1] * d[1] + bd.mesh.Minv[i][2] * d[2];
}

// nud = P lam_T;  u = M^-T (c7 nud)   (seed of the dense-output step)
__global__ void __launch_bounds__(256) k_adj_seed(ElemDev ed, const double* __restrict__ lamT, double* __restrict__ nud,
                                                  double c7, double* __restrict__ u) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    double v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = bd.constrained ? 0.0 : lamT[o + c];
    double d[3] = {c7 * v[0], c7 * v[1], c7 * v[2]}, w[3];
    minv_apply(bd, d, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) { nud[o + c] = v[c]; u[o + c] = w[c]; }
}

struct StepCoef {
    double cb[6];     // dt b_j
    double cd[6];     // s dt bt_j (dense step) or 0
    double ca[6];     // dt a_ij of the stage being accumulated
};

// Start of a reverse step: v = P lam_in, lam = v (+ nud), D_j = cb_j v (+ cd_j nud),
// g = 0, u = M^-T D_6.
// lam_in may be lam (in place) or g (dense step), so neither is __restrict__.
__global__ void __launch_bounds__(256) k_adj_init(ElemDev ed, const double* lam_in, const double* __restrict__ nud,
                                                  double* lam, double* const* __restrict__ Dp, StepCoef sc, double* g,
                                                  double* __restrict__ u) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    double v[3], nd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        v[c] = bd.constrained ? 0.0 : lam_in[o + c];
        nd[c] = nud ? nud[o + c] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        lam[o + c] = v[c] + nd[c];
        g[o + c] = 0.0;
    }
    double d6[3];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double dj = sc.cb[j] * v[c] + sc.cd[j] * nd[c];
            Dp[j][o + c] = dj;
            if (j == 5) d6[c] = dj;
        }
    }
    double w[3];
    minv_apply(bd, d6, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) u[o + c] = w[c];
}

// After the VJP of stage i (1-based, g = mu_i): nu = (i > 1 ? P g : g),
// lam += nu, D_j += ca_j nu (j < i), g = 0, u = M^-T D_{i-1}.
__global__ void __launch_bounds__(256) k_adj_accum(ElemDev ed, int i, double* __restrict__ g, double* __restrict__ lam,
                                                   double* const* __restrict__ Dp, StepCoef sc, double* __restrict__ u) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    double nu[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        nu[c] = (i > 1 && bd.constrained) ? 0.0 : g[o + c];
        g[o + c] = 0.0;
        lam[o + c] += nu[c];
    }
    if (i <= 1) return;
    double dn[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < i - 1; ++j) {
        double* Dj = Dp[j];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = Dj[o + c] + sc.ca[j] * nu[c];
            Dj[o + c] = v;
            if (j == i - 2) dn[c] = v;
        }
    }
    double w[3];
    minv_apply(bd, dn, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) u[o + c] = w[c];
}

// out = P v
__global__ void __launch_bounds__(256) k_adj_project_copy(ElemDev ed, const double* __restrict__ v, double* __restrict__ out) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[o + c] = bd.constrained ? 0.0 : v[o + c];
}

// ------------------------------------------------------------ host helpers
static int rhs_acc(tb_handle* h, const double* y, int flags) {
    return run_rhs_acc(h, y, h->d_acc, nullptr, flags & (TB_NO_DRIFT | TB_NO_COLLISIONS), -1);
}

static int replay_stage(tb_handle* h, double* kout, const Combo& cb, double* out) {
    k_replay_stage<<<h->ed.nblk, 256, 0, h->stream>>>(h->ed, h->d_acc, kout, cb, out);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// One frozen-dt step from Y[0] = y: writes stage inputs Y[1..5] (when
// Y is non-null) and the next state into y_next; k[0..5] hold the stage
// derivatives afterwards.  6 right-hand sides.
static int replay_step(tb_handle* h, double* const* k, const double* y, double* const* Y, double* tmp, double* y_next,
                       double dt, int flags) {
    const double* in = y;
    for (int s = 1; s <= 6; ++s) {
        TB_TRY(rhs_acc(h, in, flags));
        Combo cb{};
        cb.y = y;
        for (int j = 0; j < 7; ++j) cb.k[j] = k[j];
        double* out;
        if (s <= 5) {
            for (int j = 0; j < s; ++j) { cb.c[j] = kA[s][j] * dt; cb.use[j] = 1; }
            out = Y ? Y[s] : tmp;
        } else {
            for (int j = 0; j < 6; ++j) { cb.c[j] = dt * kB[j]; cb.use[j] = (j != 1); }
            out = y_next;
        }
        TB_TRY(replay_stage(h, k[s - 1], cb, out));
        in = out;
    }
    return TB_OK;
}

// mu (into A->g) = F'(Y)^T D with u = M^-T D already formed; amplitude
// gradients accumulate into A->gamp.
static int vjp_at(tb_handle* h, const double* Y, int flags) {
    AdjointState* A = h->adj;
    if (!(flags & TB_NO_COLLISIONS)) {
        for (size_t gi = 0; gi < h->groups.size(); ++gi) {
            GroupChan& G = h->groups[gi];
            if ((G.tup.n == 0 && !G.stream) || G.insts.empty()) continue;
            // deterministic mode: the group's amplitude slots in the exact accumulator
            FxAcc fa = A->gamp_fx;
            if (fa.w) fa.w += 3 * int64_t(A->gamp_off[gi]);
            if (G.stream) {   // tuples enumerated again, as in the forward evaluations
                TB_TRY(launch_vjp_stream(G.dev, G.sdev, G.item_begin, G.item_end, G.d_insts, int(G.insts.size()), Y,
                                         A->u, A->g, A->gamp + A->gamp_off[gi], h->stream, h->fx, fa));
                continue;
            }
            if (G.layout == TB_LAYOUT_MC64 && G.theta.use)   // the tuples and points inside the simplices only
                TB_TRY(launch_collision_vjp(G.dev, G.d_insts, int(G.insts.size()), G.layout, G.tensor, G.theta.ids,
                                            G.theta.n, G.theta.n, Y, A->u, A->g, A->gamp + A->gamp_off[gi], h->stream,
                                            G.theta.mask, G.theta.perm, h->fx, fa));
            else
                TB_TRY(launch_collision_vjp(G.dev, G.d_insts, int(G.insts.size()), G.layout, G.tensor, G.tup.d,
                                            G.tup.cap, G.tup.n, Y, A->u, A->g, A->gamp + A->gamp_off[gi], h->stream,
                                            nullptr, nullptr, h->fx, fa));
        }
        TB_TRY(launch_fx_flush(h->fx, A->g, h->ndofs, h->stream));   // deterministic mode
        TB_TRY(shard_allreduce(h, A->g, size_t(h->ndofs)));   // sharded: all ranks' partial VJPs
    }
    if (!(flags & TB_NO_DRIFT) && h->any_drift) {
        TB_TRY(launch_drift_vjp(h->ed, A->u, A->g, h->stream, h->fx));
        TB_TRY(launch_fx_flush(h->fx, A->g, h->ndofs, h->stream));
    }
    A->vjp_evals += 1;
    return TB_OK;
}

static int copy_gamp_out(tb_handle* h, double* grad_amp) {
    AdjointState* A = h->adj;
    TB_TRY(launch_fx_flush(A->gamp_fx, A->gamp, A->n_slots, h->stream));   // deterministic mode
    TB_TRY(shard_allreduce(h, A->gamp, size_t(A->n_slots)));   // sharded: all ranks' partial sums
    std::vector<double> slots(size_t(std::max(A->n_slots, 1)));
    TB_CUDA(cudaMemcpyAsync(slots.data(), A->gamp, sizeof(double) * size_t(A->n_slots), cudaMemcpyDeviceToHost,
                            h->stream));
    TB_TRY(stream_wait(h));
    for (size_t c = 0; c < h->insts.size(); ++c) {
        const ChanInst& I = h->insts[c];
        grad_amp[c] = slots[size_t(A->gamp_off[I.group] + I.slot)];
    }
    return TB_OK;
}

}  // namespace tb

using namespace tb;

extern "C" {

int tb_adjoint_rhs_vjp(tb_handle* h, const double* f, const double* theta, double* grad_f, double* grad_amp,
                       int flags) {
    if (!h || !f || !theta || !grad_f) { set_error("null argument"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(adj_base(h));
    AdjointState* A = h->adj;
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const double* df = f;
    const double* dth = theta;
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(A->ry, f, bytes, cudaMemcpyHostToDevice, h->stream));
        TB_CUDA(cudaMemcpyAsync(A->rtmp, theta, bytes, cudaMemcpyHostToDevice, h->stream));
        df = A->ry;
        dth = A->rtmp;
    }
    TB_CUDA(cudaMemsetAsync(A->g, 0, bytes, h->stream));
    TB_CUDA(cudaMemsetAsync(A->gamp, 0, sizeof(double) * size_t(std::max(A->n_slots, 1)), h->stream));
    if (A->gamp_fx.w)   // a sweep that failed half-way may have left words behind
        TB_CUDA(cudaMemsetAsync(A->gamp_fx.w, 0, sizeof(double) * size_t(3 * std::max(A->n_slots, 1) + 1), h->stream));
    TB_TRY(launch_minv_t(h->ed, dth, A->u, h->stream));
    TB_TRY(vjp_at(h, df, flags));
    if (flags & TB_PTR_HOST) TB_CUDA(cudaMemcpyAsync(grad_f, A->g, bytes, cudaMemcpyDeviceToHost, h->stream));
    else TB_CUDA(cudaMemcpyAsync(grad_f, A->g, bytes, cudaMemcpyDeviceToDevice, h->stream));
    TB_CUDA(cudaMemsetAsync(A->g, 0, bytes, h->stream));
    if (grad_amp) TB_TRY(copy_gamp_out(h, grad_amp));
    else TB_TRY(stream_wait(h));
    bool clamped = false;
    TB_TRY(fx_take_saturation(h, clamped));
    if (clamped) return fx_saturation_error();
    return TB_OK;
}

int tb_dp45_replay(tb_handle* h, const double* f0, const double* dts, int64_t n_steps, double dense_s, double* f_out,
                   int flags) {
    if (!h || !f0 || !dts || !f_out || n_steps < 1) { set_error("bad argument"); return TB_ERR_ARG; }
    if (!(dense_s > 0.0) || !(dense_s <= 1.0001)) { set_error("dense_s must lie in (0, 1.0001]"); return TB_ERR_ARG; }
    if (h->cfn) { set_error("the replay has no time-dependent constraints"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(adj_base(h));
    AdjointState* A = h->adj;
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    TB_CUDA(cudaMemcpyAsync(A->ry5, f0, bytes, (flags & TB_PTR_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            h->stream));
    TB_TRY(launch_enforce(h->ed, A->ry5, A->ry, h->stream));
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    for (int64_t n = 0; n < n_steps; ++n) {
        const double dt = dts[n];
        TB_TRY(replay_step(h, A->k, A->ry, nullptr, A->rtmp, A->ry5, dt, flags));
        if (n + 1 < n_steps) {
            std::swap(A->ry, A->ry5);
            continue;
        }
        // dense output of the last step: k7 = F(y_{n+1}), then the bt combination
        TB_TRY(rhs_acc(h, A->ry5, flags));
        double bt[7];
        dense_weights(dense_s, bt);
        Combo cb{};
        cb.y = A->ry;
        for (int j = 0; j < 7; ++j) {
            cb.k[j] = A->k[j];
            cb.c[j] = dense_s * dt * bt[j];
            cb.use[j] = (j != 1);
        }
        TB_TRY(replay_stage(h, A->k[6], cb, A->rtmp));
    }
    TB_CUDA(cudaMemcpyAsync(f_out, A->rtmp, bytes, (flags & TB_PTR_HOST) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                            h->stream));
    TB_TRY(stream_wait(h));
    return TB_OK;
}

int tb_adjoint_forward(tb_handle* h, const double* f0, double t0, double t1, double dense_step, int checkpoint_every,
                       int64_t max_steps, double* f_obs, tb_adjoint_stats* st, int flags) {
    NvtxRange range("tb_adjoint_forward");
    if (!h || !f0) { set_error("null argument"); return TB_ERR_ARG; }
    if (h->runs.size() != 1) { set_error("the adjoint integrates single-run handles"); return TB_ERR_ARG; }
    if (checkpoint_every < 1 || max_steps < 1) { set_error("checkpoint_every and max_steps must be >= 1"); return TB_ERR_ARG; }
    if (h->cfn) { set_error("the adjoint has no time-dependent constraints"); return TB_ERR_ARG; }
    if (!(t1 > t0) || !(dense_step > 0.0) || dense_step > (t1 - t0) * (1.0 + 1e-12)) {
        set_error("need t1 > t0 and 0 < dense_step <= t1 - t0");
        return TB_ERR_ARG;
    }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(adj_budget(h, checkpoint_every, max_steps));
    AdjointState* A = h->adj;
    A->have_forward = false;
    A->rhs_evals = 0;
    A->vjp_evals = 0;
    DPBufs hooks{};
    hooks.step_log = A->log;
    hooks.log_cap = max_steps;
    hooks.ckpt = A->ckpt;
    hooks.ckpt_every = checkpoint_every;
    hooks.ckpt_cap = A->ckpt_cap;
    const int64_t max_dense = int64_t(std::floor((t1 - t0) / dense_step + 1e-9)) + 2;
    const double a0 = t0, a1 = t1, ds = dense_step;
    TB_TRY(dp_begin(h, f0, &a0, &a1, &ds, max_dense, flags, &hooks));
    int64_t batch = 4;
    tb_dp45_stats s{};
    for (;;) {
        TB_TRY(tb_dp45_advance(h, batch));
        TB_TRY(tb_dp45_poll(h, &s));
        if (s.done) break;
        if (batch < 64) batch *= 2;
    }
    const DPCtl& c = h->h_ctl[0];
    A->attempts = c.attempts;
    A->rhs_evals = c.rhs_evals;
    if (c.status != TB_OK) {
        set_error(c.status == TB_ERR_CAPACITY ? "adjoint forward: max_steps or dense capacity exceeded"
                                              : "adjoint forward integration failed");
        return c.status;
    }
    if (c.n_dense < 1 || c.last_dense_step < 0) { set_error("no dense output was produced"); return TB_ERR_ARG; }
    A->n_steps = c.last_dense_step + 1;
    A->dense_s = c.last_dense_s;
    A->n_ckpt = c.accepted / checkpoint_every + 1;
    A->flags = flags & (TB_NO_DRIFT | TB_NO_COLLISIONS);
    std::vector<double> lg(size_t(2 * A->n_steps));
    TB_CUDA(cudaMemcpyAsync(lg.data(), A->log, sizeof(double) * lg.size(), cudaMemcpyDeviceToHost, h->stream));
    const int64_t last = std::min<int64_t>(c.n_dense, h->dense_cap_alloc) - 1;
    TB_CUDA(cudaMemcpyAsync(&A->t_obs, h->dp.dense_t + last, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (f_obs)
        TB_CUDA(cudaMemcpyAsync(f_obs, h->dp.dense + last * h->ndofs, sizeof(double) * size_t(h->ndofs),
                                (flags & TB_PTR_HOST) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, h->stream));
    TB_TRY(stream_wait(h));
    A->step_dt.resize(size_t(A->n_steps));
    for (int64_t n = 0; n < A->n_steps; ++n) A->step_dt[size_t(n)] = lg[size_t(2 * n + 1)];
    A->have_forward = true;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->t_obs = A->t_obs;
        st->dense_s = A->dense_s;
        st->steps = A->n_steps;
        st->attempts = A->attempts;
        st->checkpoints = A->n_ckpt;
        st->rhs_evals = A->rhs_evals;
        st->vjp_evals = 0;
        st->status = TB_OK;
        st->checkpoint_every = checkpoint_every;
    }
    return TB_OK;
}

int tb_adjoint_steps(tb_handle* h, double* dts, int64_t cap, int64_t* n_steps, double* dense_s) {
    if (!h || !h->adj || !h->adj->have_forward) { set_error("tb_adjoint_forward was not called"); return TB_ERR_ARG; }
    AdjointState* A = h->adj;
    if (n_steps) *n_steps = A->n_steps;
    if (dense_s) *dense_s = A->dense_s;
    if (dts)
        for (int64_t n = 0; n < std::min(cap, A->n_steps); ++n) dts[n] = A->step_dt[size_t(n)];
    return TB_OK;
}

int tb_adjoint_backward(tb_handle* h, const double* lambda_T, double* grad_f0, double* grad_amp, tb_adjoint_stats* st,
                        int flags) {
    NvtxRange range("tb_adjoint_backward");
    if (!h || !lambda_T) { set_error("null argument"); return TB_ERR_ARG; }
    if (!h->adj || !h->adj->have_forward) { set_error("tb_adjoint_forward was not called"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    AdjointState* A = h->adj;
    const int rflags = A->flags;
    const size_t n = size_t(h->ndofs);
    const size_t bytes = sizeof(double) * n;
    const int K = A->every;
    TB_CUDA(cudaMemcpyAsync(A->lam_T, lambda_T, bytes,
                            (flags & TB_PTR_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, h->stream));
    TB_CUDA(cudaMemsetAsync(A->g, 0, bytes, h->stream));
    TB_CUDA(cudaMemsetAsync(A->lam, 0, bytes, h->stream));
    TB_CUDA(cudaMemsetAsync(A->gamp, 0, sizeof(double) * size_t(std::max(A->n_slots, 1)), h->stream));
    if (A->gamp_fx.w)   // a sweep that failed half-way may have left words behind
        TB_CUDA(cudaMemsetAsync(A->gamp_fx.w, 0, sizeof(double) * size_t(3 * std::max(A->n_slots, 1) + 1), h->stream));
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    // the forward sweep's rejected trial stages may have clamped; the
    // backward sweep only replays accepted steps, where a clamp is an error
    if (h->fx.sat) TB_CUDA(cudaMemsetAsync(h->fx.sat, 0, sizeof(unsigned int), h->stream));
    double* const* dD = A->dD;
    const int64_t nd = A->n_steps - 1;   // the dense-output step
    int64_t rhs = 0;
    A->vjp_evals = 0;
    for (int64_t sg = nd / K; sg >= 0; --sg) {
        const int64_t n0 = sg * K, n1 = std::min<int64_t>(n0 + K, A->n_steps);
        // replay the segment from its checkpoint, keeping every stage input
        TB_CUDA(cudaMemcpyAsync(A->seg, A->ckpt + size_t(sg) * n, bytes, cudaMemcpyDeviceToDevice, h->stream));
        for (int64_t m = n0; m < n1; ++m) {
            double* base = A->seg + size_t(6 * (m - n0)) * n;
            double* Ys[6];
            for (int i = 0; i < 6; ++i) Ys[i] = base + size_t(i) * n;
            TB_TRY(replay_step(h, A->k, Ys[0], Ys, nullptr, base + 6 * n, A->step_dt[size_t(m)], rflags));
            rhs += 6;
        }
        for (int64_t m = n1 - 1; m >= n0; --m) {
            const double dt = A->step_dt[size_t(m)];
            const double* base = A->seg + size_t(6 * (m - n0)) * n;
            StepCoef sc{};
            for (int j = 0; j < 6; ++j) sc.cb[j] = dt * kB[j];
            if (m == nd) {
                double bt[7];
                dense_weights(A->dense_s, bt);
                for (int j = 0; j < 6; ++j) sc.cd[j] = A->dense_s * dt * bt[j];
                const double c7 = A->dense_s * dt * bt[6];
                k_adj_seed<<<h->ed.nblk, 256, 0, h->stream>>>(h->ed, A->lam_T, A->nud, c7, A->u);
                TB_CUDA(cudaGetLastError());
                // k7 = F(y_{m+1}) enters the dense output only
                TB_TRY(vjp_at(h, base + 6 * n, rflags));
                k_adj_init<<<h->ed.nblk, 256, 0, h->stream>>>(h->ed, A->g, A->nud, A->lam, dD, sc, A->g, A->u);
            } else {
                k_adj_init<<<h->ed.nblk, 256, 0, h->stream>>>(h->ed, A->lam, nullptr, A->lam, dD, sc, A->g, A->u);
            }
            TB_CUDA(cudaGetLastError());
            for (int i = 6; i >= 1; --i) {
                TB_TRY(vjp_at(h, base + size_t(i - 1) * n, rflags));
                for (int j = 0; j < 6; ++j) sc.ca[j] = (j < i - 1) ? kA[i - 1][j] * dt : 0.0;
                k_adj_accum<<<h->ed.nblk, 256, 0, h->stream>>>(h->ed, i, A->g, A->lam, dD, sc, A->u);
                TB_CUDA(cudaGetLastError());
            }
        }
    }
    // y_0 enters through P (the forward enforces it before the first stage)
    double* out = (flags & TB_PTR_HOST) ? A->rtmp : grad_f0;
    if (grad_f0) {
        k_adj_project_copy<<<h->ed.nblk, 256, 0, h->stream>>>(h->ed, A->lam, out);
        TB_CUDA(cudaGetLastError());
        if (flags & TB_PTR_HOST) TB_CUDA(cudaMemcpyAsync(grad_f0, out, bytes, cudaMemcpyDeviceToHost, h->stream));
    }
    if (grad_amp) TB_TRY(copy_gamp_out(h, grad_amp));
    TB_TRY(stream_wait(h));
    int tflag = 0;
    TB_TRY(take_wait_timeout(h->d_err, h->stream, &tflag));
    if (tflag) { set_error("moment-tensor copy wait ran out"); return TB_ERR_TIMEOUT; }
    bool clamped = false;
    TB_TRY(fx_take_saturation(h, clamped));
    if (clamped) return fx_saturation_error();
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->t_obs = A->t_obs;
        st->dense_s = A->dense_s;
        st->steps = A->n_steps;
        st->attempts = A->attempts;
        st->checkpoints = A->n_ckpt;
        st->rhs_evals = A->rhs_evals + rhs;
        st->vjp_evals = A->vjp_evals;
        st->status = TB_OK;
        st->checkpoint_every = K;
    }
    return TB_OK;
}

int tb_adjoint_integrate(tb_handle* h, const double* f0, double t0, double t1, double dense_step,
                         int checkpoint_every, int64_t max_steps, const double* lambda_T, double* f_obs,
                         double* grad_f0, double* grad_amp, tb_adjoint_stats* st, int flags) {
    TB_TRY(tb_adjoint_forward(h, f0, t0, t1, dense_step, checkpoint_every, max_steps, f_obs, st, flags));
    return tb_adjoint_backward(h, lambda_T, grad_f0, grad_amp, st, flags);
}

}  // extern "C"
