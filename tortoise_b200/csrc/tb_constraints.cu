// tb_constraints.cu -- time-dependent constrained populations (lasers,
// reservoirs that follow a prescribed history) inside the device integrator.
//
// The reference keeps a std::function<Function(Real)> per constrained band
// (Band::constrainedPopulation, include/Physics/Material/Band.hpp:70-74),
// calls it in every enforceValue of the Dormand-Prince step
// (MaterialStatus::applyConstraints(time), src/Physics/Status/
// MaterialStatus.cpp:198-206) and in MaterialTimeStatus::timeStepVetoer
// (src/Physics/Status/MaterialTimeStatus.cpp:60-100), which caps the step
// size at the start and after every accepted step (DormandPrince54.hpp:554,
// 638-640).  Here the function is a C callback and the attempt graph starts
// with
//   copy the controllers to pinned memory -> host node -> copy back
//   (controllers and the constrained values of the attempt)
// The host node applies the vetoer where an accepted step left it pending and
// evaluates the callback at the attempt's five enforce times (t + c2 dt,
// t + c3 dt, t + c4 dt, t + c5 dt, t + dt) and at the dense-output times the
// attempt can produce; the stage, dense-output and enforce kernels read those
// slots instead of the constant populations.  Every time is formed on the host
// in the reference's own expressions, so the callback sees the same arguments
// as the reference's std::function would.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "tb_handle.cuh"

namespace tb {

namespace {

constexpr double kC2 = 1. / 5., kC3 = 3. / 10., kC4 = 4. / 5., kC5 = 8. / 9.;   // DormandPrince54.hpp:503

// toNodalFromLinForm / toLinFormFromNodal of one P1 element
inline void to_nodal(const double* c, double n[3]) { n[0] = c[0]; n[1] = c[1] + c[0]; n[2] = c[2] + c[0]; }
inline void to_lin(const double n[3], double* c) { c[0] = n[0]; c[1] = n[1] - n[0]; c[2] = n[2] - n[0]; }

// fabs(Function): nodal absolute value, stored back in linear form
// (Function.cpp:75-80 with std::fabs)
void fn_fabs(const double* c, double* out, int64_t ne) {
    for (int64_t e = 0; e < ne; ++e) {
        double n[3];
        to_nodal(c + 3 * e, n);
        for (int k = 0; k < 3; ++k) n[k] = std::fabs(n[k]);
        to_lin(n, out + 3 * e);
    }
}

// One band's constrained population at time t into out (Ne*3).
bool band_population(tb_handle* h, int b, double t, double* out) {
    if (h->cfn) return h->cfn(h->cuser, int32_t(b), t, out) == 0;
    std::copy(h->bands[b].cpop.begin(), h->bands[b].cpop.end(), out);
    return true;
}

// Every constrained band of run r at time t into one slot.
bool run_slot(tb_handle* h, int r, double t, double* slot) {
    const RunInfo& ri = h->runs[r];
    for (int b = ri.band0; b < ri.band0 + ri.nbands; ++b)
        if (h->bands[b].constrained && !band_population(h, b, t, slot + h->coff[b])) return false;
    return true;
}

// MaterialTimeStatus::timeStepVetoer for run r and the six stage times of a
// step of size dt from t, with the reference's Function arithmetic: + - and
// scalar * on the linear-form coefficients, Function + scalar on c0, fabs and
// Function / Function through the nodal values, max() over the nodal values.
// Returns false when the callback failed.
bool veto(tb_handle* h, int r, double t, double dt, double dense, double* out_dt) {
    const double times[6] = {t, t + kC2 * dt, t + kC3 * dt, t + kC4 * dt, t + kC5 * dt, t + dt};
    const double accept_rel = 0.3;
    double critical = times[5];
    bool found = false;
    const RunInfo& ri = h->runs[r];
    for (int b = ri.band0; b < ri.band0 + ri.nbands && !found; ++b) {
        const HostBand& B = h->bands[b];
        if (!B.constrained) continue;
        const int64_t ne = B.ne, n = 3 * ne;
        std::vector<double> left(n), right(n), avg(n), acc(n), tmp(n), tmp2(n), mid(n);
        double tt = times[0] + dense;
        if (!band_population(h, b, times[0], left.data()) || !band_population(h, b, times[1], right.data()))
            return false;
        for (int i = 0; i < 5 && !found; ++i) {
            if (i != 0) {
                left.swap(right);
                if (!band_population(h, b, times[i + 1], right.data())) return false;
            }
            for (int64_t k = 0; k < n; ++k) avg[k] = 0.5 * (left[k] + right[k]);
            for (int64_t k = 0; k < n; ++k) tmp[k] = left[k] - right[k];
            fn_fabs(tmp.data(), tmp2.data(), ne);
            for (int64_t k = 0; k < n; ++k) acc[k] = (1. + accept_rel) * tmp2[k];
            for (int64_t e = 0; e < ne; ++e) acc[3 * e] += B.abs_tol;
            fn_fabs(avg.data(), tmp2.data(), ne);
            for (int64_t k = 0; k < n; ++k) acc[k] = acc[k] + B.rel_tol * tmp2[k];
            while (tt < times[i + 1]) {
                if (!band_population(h, b, tt, mid.data())) return false;
                for (int64_t k = 0; k < n; ++k) tmp[k] = mid[k] - avg[k];
                fn_fabs(tmp.data(), tmp2.data(), ne);
                double mx = -INFINITY;
                for (int64_t e = 0; e < ne; ++e) {
                    double a[3], q[3], d[3], lin[3];
                    to_nodal(tmp2.data() + 3 * e, a);
                    to_nodal(acc.data() + 3 * e, q);
                    for (int k = 0; k < 3; ++k) d[k] = a[k] / q[k];
                    to_lin(d, lin);
                    to_nodal(lin, d);
                    for (int k = 0; k < 3; ++k) mx = std::max(mx, d[k]);
                }
                if (mx > 1.) {
                    critical = tt;
                    found = true;
                    break;
                }
                tt += dense;
            }
        }
    }
    *out_dt = critical - times[0];
    return true;
}

// Host node at the head of every attempt (the controllers were copied to
// h_ctl_tc just before; the node's edits and the slots are copied back after).
void CUDART_CB pre_attempt(void* arg) {
    tb_handle* h = static_cast<tb_handle*>(arg);
    for (size_t r = 0; r < h->runs.size(); ++r) {
        DPCtl& c = h->h_ctl_tc[r];
        if (c.done) continue;
        bool ok = true;
        if (c.veto_pending) {
            double v = 0.0;
            ok = veto(h, int(r), c.t, c.dt, c.dense_step, &v);
            if (ok) c.dt = std::min(c.dt, v);
            c.veto_pending = 0;
        }
        const double t = c.t, dt = c.dt;
        const double ts[5] = {t + kC2 * dt, t + kC3 * dt, t + kC4 * dt, t + kC5 * dt, t + dt};
        for (int s = 0; s < 5 && ok; ++s) ok = run_slot(h, int(r), ts[s], h->h_ctv + s * h->cdofs);
        // the dense times this attempt can produce: the controller's window
        // (dtime <= t + 1.0001 dt, <= tf + 1e-4 dt) with margin
        int k = 0;
        double dtime = c.dense_time;
        while (ok && k < TB_TC_DENSE && dtime <= t + 1.001 * dt && dtime <= c.tf + .001 * dt) {
            c.tc_dense_t[k] = dtime;
            ok = run_slot(h, int(r), dtime, h->h_ctv + (5 + k) * h->cdofs);
            dtime += c.dense_step;
            ++k;
        }
        c.tc_ndense = k;
        if (!ok) {
            c.status = TB_ERR_ARG;
            c.done = 1;
        }
    }
}

}  // namespace

int tc_record_pre_attempt(tb_handle* h) {
    const size_t nr = h->runs.size();
    DPBufs& B = h->dp;
    TB_CUDA(cudaMemcpyAsync(h->h_ctl_tc, B.ctl, sizeof(DPCtl) * nr, cudaMemcpyDeviceToHost, h->stream));
    TB_CUDA(cudaLaunchHostFunc(h->stream, pre_attempt, h));
    TB_CUDA(cudaMemcpyAsync(B.ctl, h->h_ctl_tc, sizeof(DPCtl) * nr, cudaMemcpyHostToDevice, h->stream));
    TB_CUDA(cudaMemcpyAsync(h->d_ctv, h->h_ctv, sizeof(double) * size_t(TB_TC_SLOTS) * size_t(h->cdofs),
                            cudaMemcpyHostToDevice, h->stream));
    return TB_OK;
}

// Called by dp_begin with the controllers initialised in h->h_ctl: slot 0
// gets every run's values at t0 (enforceValue of k1), and every run's first
// dt is vetoed (DormandPrince54.hpp:551-554).
int tc_begin(tb_handle* h) {
    for (size_t r = 0; r < h->runs.size(); ++r) {
        DPCtl& c = h->h_ctl[r];
        if (!run_slot(h, int(r), c.t, h->h_ctv)) {
            set_error("constraint callback failed");
            return TB_ERR_ARG;
        }
        double v = 0.0;
        if (!veto(h, int(r), c.t, c.dt, c.dense_step, &v)) {
            set_error("constraint callback failed");
            return TB_ERR_ARG;
        }
        c.dt = std::min(c.dt, v);
        c.veto_pending = 0;
    }
    TB_CUDA(cudaMemcpyAsync(h->d_ctv, h->h_ctv, sizeof(double) * size_t(h->cdofs), cudaMemcpyHostToDevice,
                            h->stream));
    return TB_OK;
}

void tc_release(tb_handle* h) {
    if (h->d_ctv) cudaFree(h->d_ctv);
    if (h->h_ctv) cudaFreeHost(h->h_ctv);
    if (h->h_ctl_tc) cudaFreeHost(h->h_ctl_tc);
    h->d_ctv = nullptr;
    h->h_ctv = nullptr;
    h->h_ctl_tc = nullptr;
}

}  // namespace tb

using namespace tb;

extern "C" {

int tb_set_constraint_fn(tb_handle* h, tb_constraint_fn fn, void* user) {
    if (!h) { set_error("null handle"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(stream_wait(h));
    if (fn && h->cdofs == 0) { set_error("the description has no constrained band"); return TB_ERR_ARG; }
    if (fn && !h->d_ctv) {
        const size_t slots = sizeof(double) * size_t(TB_TC_SLOTS) * size_t(h->cdofs);
        if (cudaMalloc(&h->d_ctv, slots) != cudaSuccess || cudaMallocHost(&h->h_ctv, slots) != cudaSuccess ||
            cudaMallocHost(&h->h_ctl_tc, sizeof(DPCtl) * h->runs.size()) != cudaSuccess) {
            cudaGetLastError();
            tc_release(h);
            set_error("constraint slot allocation failed");
            return TB_ERR_OOM;
        }
        std::memset(h->h_ctv, 0, slots);
        std::memset(h->h_ctl_tc, 0, sizeof(DPCtl) * h->runs.size());
    }
    h->cfn = fn;
    h->cuser = user;
    // the attempt graph gains or loses its host node; DPBufs change with it
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    h->dp.tc = fn ? 1 : 0;
    h->dp.ctv = fn ? h->d_ctv : nullptr;
    h->dp.cdofs = h->cdofs;
    return TB_OK;
}

int tb_apply_constraints_at(tb_handle* h, double* f, double t, int flags) {
    if (!h || !f) { set_error("null argument"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const double* cv = nullptr;
    TB_TRY(stream_wait(h));
    if (h->cfn) {
        for (size_t r = 0; r < h->runs.size(); ++r)
            if (!run_slot(h, int(r), t, h->h_ctv)) { set_error("constraint callback failed"); return TB_ERR_ARG; }
        TB_CUDA(cudaMemcpyAsync(h->d_ctv, h->h_ctv, sizeof(double) * size_t(h->cdofs), cudaMemcpyHostToDevice,
                                h->stream));
        cv = h->d_ctv;
    }
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(h->d_f, f, bytes, cudaMemcpyHostToDevice, h->stream));
        TB_TRY(launch_enforce(h->ed, h->d_f, h->d_f, h->stream, cv));
        TB_CUDA(cudaMemcpyAsync(f, h->d_f, bytes, cudaMemcpyDeviceToHost, h->stream));
    } else {
        TB_TRY(launch_enforce(h->ed, f, f, h->stream, cv));
    }
    TB_TRY(stream_wait(h));
    return TB_OK;
}

}  // extern "C"
