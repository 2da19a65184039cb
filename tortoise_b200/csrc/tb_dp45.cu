// tb_dp45.cu -- fused Dormand-Prince 5(4) stage kernels, on-device error norm
// and step-size controller.
//
// Reference: Algorithms::dormandPrince54, third overload
// (include/Generics/Algorithms/DormandPrince54.hpp:479-665) as driven by
// MaterialTimeStatus::propagate (src/Physics/Status/MaterialTimeStatus.cpp:
// 102-137); error norm MaterialStatus::relativeError / Band::relativeError
// (src/Physics/Status/MaterialStatus.cpp:189-196, src/Physics/Material/
// Band.cpp:87-101); constraints MaterialStatus::applyConstraints
// (MaterialStatus.cpp:198-206).
//
// Each stage kernel fuses, per element: M^-1 of the freshly accumulated RHS,
// the reset of the accumulator, the Butcher combination of the next stage
// input and the constraint enforcement -- one pass over the state per RHS
// evaluation instead of the reference's chain of vector temporaries.  The
// last stage kernel also forms y4, err = y5 - y4 and per-block partial sums of
// the Gauss-2 error integrals; the single-thread controller kernel reduces
// them in a fixed order (deterministic), applies the PI controller and
// schedules dense output.  dt never leaves the device.
#include <math.h>

#include "tb_dp45.cuh"
#include "tb_errnorm.cuh"

namespace tb {

// Butcher tableau, DormandPrince54.hpp:502-511
__constant__ double c_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1. / 5., 0, 0, 0, 0, 0},
    {3. / 40., 9. / 40., 0, 0, 0, 0},
    {44. / 45., -56. / 15., 32. / 9., 0, 0, 0},
    {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729., 0, 0},
    {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656., 0},
    {0, 0, 0, 0, 0, 0}};
__constant__ double c_b[6] = {35. / 384., 0., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.};
__constant__ double c_bh[7] = {5179. / 57600., 0., 7571. / 16695., 393. / 640., -92097. / 339200., 187. / 2100.,
                               1. / 40.};

// enforceValue on one element: constrained bands take the slot of
// time-dependent values cv when given, else their constant population.
__device__ __forceinline__ void enforce3(const BandDev& bd, int e, double v[3], const double* cv = nullptr) {
    if (bd.constrained) {
        const double* cp = (cv ? cv + bd.coff : bd.cpop) + 3 * (int64_t)e;
        v[0] = cp[0]; v[1] = cp[1]; v[2] = cp[2];
    }
}

// Element-wise stage kernel (see tb_dp45.cuh for the meaning of s).  One
// block covers 256 elements of one band, so every block belongs to one run.
template <int S>
__global__ void __launch_bounds__(256) k_stage(ElemDev ed, DPBufs B) {
    __shared__ double sh[8];
    const int band = ed.blk_band[blockIdx.x];
    const DPCtl& ctl = B.ctl[ed.band_run[band]];
    if (ctl.done) return;
    const double dt = ctl.dt;
    const BandDev& bd = ed.bands[band];
    // slot of the enforce time: t + c_{S+2} dt for S <= 3, t + dt after
    const double* cv = B.tc ? B.ctv + (S <= 4 ? S : 4) * B.cdofs : nullptr;
    double srel = 0.0, spen = 0.0;
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e < bd.ne) {
        const int64_t o = bd.off + 3 * (int64_t)e;
        if (S >= 1) {
            // k_{S+1} = acc * M^-1, acc = 0
            const double x = B.acc[o], y = B.acc[o + 1], z = B.acc[o + 2];
            double* kk = B.k[S];
#pragma unroll
            for (int j = 0; j < 3; ++j) kk[o + j] = x * bd.mesh.Minv[0][j] + y * bd.mesh.Minv[1][j] + z * bd.mesh.Minv[2][j];
            B.acc[o] = 0.0; B.acc[o + 1] = 0.0; B.acc[o + 2] = 0.0;
        }
        double v[3];
        if (S <= 4) {
            // input of k_{S+2}: y + sum_{j<=S} (a_{S+1,j} dt) k_{j+1}
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double t = B.y[o + c];
#pragma unroll
                for (int j = 0; j <= S; ++j) t = t + (c_A[S + 1][j] * dt) * B.k[j][o + c];
                v[c] = t;
            }
            enforce3(bd, e, v, cv);
#pragma unroll
            for (int c = 0; c < 3; ++c) B.tmp[o + c] = v[c];
        } else if (S == 5) {
            // y5 = y + (dt b1) k1 + (dt b3) k3 + (dt b4) k4 + (dt b5) k5 + (dt b6) k6
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double t = B.y[o + c];
                t = t + (dt * c_b[0]) * B.k[0][o + c];
                t = t + (dt * c_b[2]) * B.k[2][o + c];
                t = t + (dt * c_b[3]) * B.k[3][o + c];
                t = t + (dt * c_b[4]) * B.k[4][o + c];
                t = t + (dt * c_b[5]) * B.k[5][o + c];
                v[c] = t;
            }
            enforce3(bd, e, v, cv);
#pragma unroll
            for (int c = 0; c < 3; ++c) B.y5[o + c] = v[c];
        } else {
            // y4 and the error
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double t = B.y[o + c];
                t = t + (dt * c_bh[0]) * B.k[0][o + c];
                t = t + (dt * c_bh[2]) * B.k[2][o + c];
                t = t + (dt * c_bh[3]) * B.k[3][o + c];
                t = t + (dt * c_bh[4]) * B.k[4][o + c];
                t = t + (dt * c_bh[5]) * B.k[5][o + c];
                t = t + (dt * c_bh[6]) * B.k[6][o + c];
                v[c] = t;
            }
            enforce3(bd, e, v, cv);
            double err[3], p5[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) { p5[c] = B.y5[o + c]; err[c] = p5[c] - v[c]; }
            elem_rel_err(bd, err, p5, srel, spen);
        }
    }
    if (S == 6) {
        const double r = block_sum<256>(srel, sh);
        const double p = block_sum<256>(spen, sh);
        if (threadIdx.x == 0) {
            B.part[blockIdx.x] = r;
            B.part[B.nblk + blockIdx.x] = p;
        }
    }
}

int launch_stage(const ElemDev& ed, const DPBufs& B, int s, cudaStream_t st) {
    switch (s) {
        case 0: k_stage<0><<<ed.nblk, 256, 0, st>>>(ed, B); break;
        case 1: k_stage<1><<<ed.nblk, 256, 0, st>>>(ed, B); break;
        case 2: k_stage<2><<<ed.nblk, 256, 0, st>>>(ed, B); break;
        case 3: k_stage<3><<<ed.nblk, 256, 0, st>>>(ed, B); break;
        case 4: k_stage<4><<<ed.nblk, 256, 0, st>>>(ed, B); break;
        case 5: k_stage<5><<<ed.nblk, 256, 0, st>>>(ed, B); break;
        default: k_stage<6><<<ed.nblk, 256, 0, st>>>(ed, B); break;
    }
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// Controller, one thread per run: DormandPrince54.hpp:580-661.
__global__ void k_controller(ElemDev ed, DPBufs B) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B.nruns) return;
    DPCtl* c = B.ctl + r;
    const RunDev& run = B.runs[r];
    if (c->done) { c->skip = 1; return; }
    c->skip = 0;
    c->attempts += 1;
    c->rhs_evals += 6;
    double errNorm = 0.0;
    bool nonfinite = false;
    for (int bi = run.band0; bi < run.band0 + run.nbands; ++bi) {
        const BandDev& bd = ed.bands[bi];
        double sr = 0.0, sp = 0.0;
        for (int k = ed.blk_first[bi]; k < ed.blk_first[bi + 1]; ++k) { sr += B.part[k]; sp += B.part[B.nblk + k]; }
        const double ir = bd.mesh.vol * sr, ip = bd.mesh.vol * sp;
        const double be = sqrt((ir + bd.penal * ip) / (double(bd.ne) * bd.mesh.vol));
        if (!isfinite(be)) nonfinite = true;
        if (be >= errNorm) errNorm = be;   // a NaN never replaces the running max
    }
    c->last_err = errNorm;
    const double minscale = 0.333333, maxscale = 3.0, safety = 0.98, alpha = 0.7 / 5., beta = 0.4 / 5.;
    c->n_now = 0;
    c->acc_now = 0;
    if (nonfinite) {
        c->status = TB_ERR_NONFINITE;
        c->done = 1;
        return;
    }
    double dt = c->dt, t = c->t;
    c->step_t = t;
    c->step_dt = dt;
    if (errNorm <= 1.) {
        c->acc_now = 1;
        int k = 0;
        double dtime = c->dense_time;
        while (dtime <= t + (1.0001) * dt && dtime <= c->tf + .0001 * dt) {
            if (k < TB_MAX_DENSE_PER_STEP) {
                c->dense_s[k] = (dtime - t) / dt;
                c->dense_t[k] = dtime;
            }
            ++k;
            dtime += c->dense_step;
        }
        if (k > TB_MAX_DENSE_PER_STEP) { c->status = TB_ERR_CAPACITY; k = TB_MAX_DENSE_PER_STEP; }
        if (B.tc && k > c->tc_ndense) c->status = TB_ERR_CAPACITY;   // a dense time without constrained values
        c->n_now = k;
        c->dense_time = dtime;
        if (k > 0) {
            c->last_dense_step = c->accepted;
            c->last_dense_s = c->dense_s[(k < TB_MAX_DENSE_PER_STEP ? k : TB_MAX_DENSE_PER_STEP) - 1];
        }
        if (B.step_log) {
            if (c->accepted < B.log_cap) {
                B.step_log[2 * c->accepted] = t;
                B.step_log[2 * c->accepted + 1] = dt;
            } else {
                c->status = TB_ERR_CAPACITY;
            }
            const long long na = c->accepted + 1;
            if (B.ckpt && na % B.ckpt_every == 0 && na / B.ckpt_every >= B.ckpt_cap) c->status = TB_ERR_CAPACITY;
        }
        t += dt;
        double scale;
        if (errNorm == 0.) scale = maxscale;
        else {
            scale = safety * pow(1. / errNorm, alpha) * pow(c->olderror, beta);
            scale = fmin(fmax(scale, minscale), maxscale);
        }
        if (c->rejected) dt *= fmin(1.0, scale);
        else dt *= scale;
        // timeStepVetoer: without time-dependent constraints it returns
        // (t + dt) - t; with them the host node applies it before the next attempt
        if (B.tc) c->veto_pending = 1;
        else dt = fmin(dt, (t + dt) - t);
        c->rejected = 0;
        c->olderror = errNorm;
        c->accepted += 1;
    } else {
        double scale = safety * pow(1. / errNorm, 1 / 5.);
        scale = fmin(fmax(scale, minscale), maxscale);
        dt *= scale;
        c->rejected = 1;
        c->rejected_n += 1;
        if (dt < c->min_step) { c->status = TB_ERR_DT_UNDERFLOW; c->done = 1; }
    }
    c->t = t;
    c->dt = dt;
    if (!(t < c->tf)) c->done = 1;
    if (c->status == TB_ERR_CAPACITY) c->done = 1;
    if (c->max_attempts > 0 && c->attempts >= c->max_attempts) c->done = 1;
}

int launch_controller(const ElemDev& ed, const DPBufs& B, cudaStream_t st) {
    k_controller<<<(B.nruns + 127) / 128, 128, 0, st>>>(ed, B);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

// Dense output (DormandPrince54.hpp:598-611) followed by the FSAL commit
// y <- y5, k1 <- k7 of an accepted attempt, per run.  The dense outputs use
// the pre-commit y and the attempt's own dt (step_dt).
__global__ void __launch_bounds__(256) k_dense_commit(ElemDev ed, DPBufs B) {
    const int band = ed.blk_band[blockIdx.x];
    const int r = ed.band_run[band];
    const DPCtl* c = B.ctl + r;
    if (c->skip || !c->acc_now) return;
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const RunDev& run = B.runs[r];
    const int64_t o = bd.off + 3 * (int64_t)e;
    const long long base = c->n_dense;
    const double dt = c->step_dt;
    for (int k = 0; k < c->n_now; ++k) {
        const long long slot = base + k;
        if (slot >= c->dense_cap) break;
        const double s = c->dense_s[k];
        const double bt1 = -(435. * s * s * s - 1184. * s * s + 1098. * s - 384.) / (384.);
        const double bt3 = 500. * s * (6. * s * s - 14. * s + 9.) / (1113.);
        const double bt4 = -125. * s * (9. * s * s - 16. * s + 6.) / (192.);
        const double bt5 = 729. * s * (35. * s * s - 64. * s + 26.) / (6784.);
        const double bt6 = -11. * s * (3. * s - 2.) * (5. * s - 6.) / (84.);
        const double bt7 = s * (s - 1.) * (5. * s - 3.) / (2.);
        double v[3];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
            double t = B.y[o + cc];
            t = t + (s * dt * bt1) * B.k[0][o + cc];
            t = t + (s * dt * bt3) * B.k[2][o + cc];
            t = t + (s * dt * bt4) * B.k[3][o + cc];
            t = t + (s * dt * bt5) * B.k[4][o + cc];
            t = t + (s * dt * bt6) * B.k[5][o + cc];
            t = t + (s * dt * bt7) * B.k[6][o + cc];
            v[cc] = t;
        }
        const double* cv = nullptr;
        if (B.tc) {
            // the slot the host filled for this dense time (the controller
            // flagged TB_ERR_CAPACITY if there is none)
            for (int m = 0; m < c->tc_ndense; ++m)
                if (c->tc_dense_t[m] == c->dense_t[k]) { cv = B.ctv + (5 + m) * B.cdofs; break; }
        }
        enforce3(bd, e, v, cv);
        double* out = B.dense + run.dense_off + slot * run.ndofs + (o - run.dof_off);
        out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
    }
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
        B.y[o + cc] = B.y5[o + cc];
        B.k[0][o + cc] = B.k[6][o + cc];
    }
    if (B.ckpt && c->accepted % B.ckpt_every == 0) {
        // c->accepted already counts this step
        const long long slot = c->accepted / B.ckpt_every;
        if (slot < B.ckpt_cap) {
            double* ck = B.ckpt + slot * run.ndofs + (o - run.dof_off);
            ck[0] = B.y5[o]; ck[1] = B.y5[o + 1]; ck[2] = B.y5[o + 2];
        }
    }
}

__global__ void k_dense_count(DPBufs B) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B.nruns) return;
    DPCtl* c = B.ctl + r;
    if (c->skip || !c->acc_now) return;
    const RunDev& run = B.runs[r];
    for (int k = 0; k < c->n_now; ++k) {
        const long long slot = c->n_dense + k;
        if (slot < c->dense_cap) B.dense_t[run.dense_t_off + slot] = c->dense_t[k];
    }
    c->n_dense += c->n_now;
    if (c->dense_cap > 0 && c->n_dense > c->dense_cap) { c->status = TB_ERR_CAPACITY; c->done = 1; }
}

int launch_dense_commit(const ElemDev& ed, const DPBufs& B, cudaStream_t st) {
    k_dense_commit<<<ed.nblk, 256, 0, st>>>(ed, B);
    TB_CUDA(cudaGetLastError());
    k_dense_count<<<(B.nruns + 127) / 128, 128, 0, st>>>(B);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

__global__ void k_first(ElemDev ed, DPBufs B) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    const double x = B.acc[o], y = B.acc[o + 1], z = B.acc[o + 2];
#pragma unroll
    for (int j = 0; j < 3; ++j) B.k[0][o + j] = x * bd.mesh.Minv[0][j] + y * bd.mesh.Minv[1][j] + z * bd.mesh.Minv[2][j];
    B.acc[o] = 0.0; B.acc[o + 1] = 0.0; B.acc[o + 2] = 0.0;
}

int launch_k1(const ElemDev& ed, const DPBufs& B, cudaStream_t st) {
    k_first<<<ed.nblk, 256, 0, st>>>(ed, B);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

__global__ void k_enforce(ElemDev ed, const double* src, double* dst, const double* cv) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const int64_t o = bd.off + 3 * (int64_t)e;
    double v[3] = {src[o], src[o + 1], src[o + 2]};
    enforce3(bd, e, v, cv);
    dst[o] = v[0]; dst[o + 1] = v[1]; dst[o + 2] = v[2];
}

int launch_enforce(const ElemDev& ed, const double* src, double* dst, cudaStream_t st, const double* cv) {
    k_enforce<<<ed.nblk, 256, 0, st>>>(ed, src, dst, cv);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

__global__ void __launch_bounds__(256) k_error_norm(ElemDev ed, const double* err, const double* pop, double* part) {
    __shared__ double sh[8];
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    double r = 0.0, p = 0.0;
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e < bd.ne) {
        const int64_t o = bd.off + 3 * (int64_t)e;
        elem_rel_err(bd, err + o, pop + o, r, p);
    }
    const double rs = block_sum<256>(r, sh);
    const double ps = block_sum<256>(p, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = rs;
        part[ed.nblk + blockIdx.x] = ps;
    }
}

int launch_error_norm(const ElemDev& ed, const double* err, const double* pop, double* part, cudaStream_t st) {
    k_error_norm<<<ed.nblk, 256, 0, st>>>(ed, err, pop, part);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

}  // namespace tb
