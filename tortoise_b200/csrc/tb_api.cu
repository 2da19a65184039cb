// tb_api.cu -- the C ABI: handle life cycle, host-side mesh/band tables,
// the RHS driver and the Dormand-Prince integration loop.
//
// The host-side tables reproduce what the reference computes in its
// constructors (Mesh<2>: src/Geometry/Structured/DirectSpace/Mesh.cpp:95-123,
// 319-347; Band<2>: src/Physics/Material/Band.cpp:45-64) so that every device
// kernel reads ready P1 coefficients of E, kx, ky per element.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "tb_dp45.cuh"
#include "tb_enumerate.cuh"
#include "tb_kernels.cuh"
#include "tb_tensor.cuh"

namespace tb {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const char* get_error() { return g_err.c_str(); }

static const double kGP2[3][2] = {{TB_GP2_A, TB_GP2_A}, {TB_GP2_B, TB_GP2_A}, {TB_GP2_A, TB_GP2_B}};
static const double kVert[2][3][2] = {{{0, 0}, {1, 0}, {1, 1}}, {{0, 0}, {0, 1}, {1, 1}}};

static HostMesh make_mesh(const tb_region& rg, const tb_mesh_desc& md) {
    HostMesh m;
    m.nx = md.nsplit[0];
    m.ny = md.nsplit[1];
    m.ne = 2 * m.nx * m.ny;
    const double G[2][2] = {{rg.gvec[0], rg.gvec[2]}, {rg.gvec[1], rg.gvec[3]}};
    for (int i = 0; i < 2; ++i) m.origin[i] = rg.origin[i] + (G[i][0] * md.rel_origin[0] + G[i][1] * md.rel_origin[1]);
    const double ns[2] = {double(m.nx), double(m.ny)};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) m.dG[i][j] = (G[i][j] * md.rel_size[j]) * (1.0 / ns[j]);
    const double det = m.dG[0][0] * m.dG[1][1] - m.dG[0][1] * m.dG[1][0];
    const double invdet = 1.0 / det;
    m.invdG[0][0] = m.dG[1][1] * invdet;  m.invdG[1][0] = -m.dG[1][0] * invdet;
    m.invdG[0][1] = -m.dG[0][1] * invdet; m.invdG[1][1] = m.dG[0][0] * invdet;
    m.vol = std::fabs(det / 2.0);
    m.rel_origin[0] = md.rel_origin[0];
    m.rel_origin[1] = md.rel_origin[1];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int q = 0; q < 3; ++q) {
                const double bi = (i == 0) ? 1.0 : kGP2[q][i - 1];
                const double bj = (j == 0) ? 1.0 : kGP2[q][j - 1];
                s += bi * bj * TB_GW2;
            }
            m.M[i][j] = m.vol * s;
        }
    // 3x3 inverse by cofactors
    double cof[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            cof[i][j] = m.M[i1][j1] * m.M[i2][j2] - m.M[i1][j2] * m.M[i2][j1];
        }
    const double d3 = (cof[0][0] * m.M[0][0] + cof[1][0] * m.M[1][0]) + cof[2][0] * m.M[2][0];
    const double inv3 = 1.0 / d3;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m.Minv[j][i] = cof[i][j] * inv3;
    return m;
}

static void vertex(const HostMesh& m, int e, int v, double out[2]) {
    const int s = e / 2, par = e % 2;
    const double sx = double(s % m.nx), sy = double(s / m.nx);
    const double px = sx + kVert[par][v][0], py = sy + kVert[par][v][1];
    out[0] = m.origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
    out[1] = m.origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
}

static std::vector<double> coord_function(const HostMesh& m, int dim) {
    std::vector<double> v(size_t(m.ne) * 3);
    for (int e = 0; e < m.ne; ++e) {
        double n[3];
        for (int k = 0; k < 3; ++k) {
            double p[2];
            vertex(m, e, k, p);
            n[k] = p[dim];
        }
        v[3 * e] = n[0];
        v[3 * e + 1] = n[1] - n[0];
        v[3 * e + 2] = n[2] - n[0];
    }
    return v;
}

struct Channel {
    ChanDev dev;
    int L = 0;
    int band[TB_MAX_LEGS] = {0, 0, 0, 0};
    double amplitude = 0.0;
    double amp_full = 0.0;        // amplitude * prod_l (vol_l * 2), in the reference's order
    double* d_umk = nullptr;
    double* d_mc = nullptr;
    double* d_mc_pre = nullptr;
    DeviceTuples tup;
    int64_t diag[3] = {0, 0, 0};
    int layout = TB_LAYOUT_MC64;
    MomentTensor tensor;
};

}  // namespace tb

using namespace tb;

namespace tb {
int choose_layouts(tb_handle* h);
int run_rhs_acc(tb_handle* h, const double* d_in, double* d_acc, const int* done, int flags, int only_channel);
}  // namespace tb

struct tb_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    tb_options opts{};
    std::vector<HostMesh> meshes;
    std::vector<HostBand> bands;
    std::vector<double*> dev_allocs;
    BandsDev bandsdev{};
    std::vector<Channel> chans;
    int64_t ndofs = 0;
    int nblk = 1;
    double* d_f = nullptr;
    double* d_out = nullptr;
    double* d_acc = nullptr;
    double* d_part = nullptr;
    // DP45
    DPBufs dp{};
    bool dp_ready = false;
    int64_t dense_cap_alloc = -1;
    cudaGraphExec_t graph = nullptr;
    int graph_flags = -1;
    DPCtl* h_ctl = nullptr;   // pinned host mirror
    int dp_flags = 0;
};

namespace {

double* dev_alloc(tb_handle* h, size_t n) {
    double* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * (n ? n : 1)) != cudaSuccess) return nullptr;
    h->dev_allocs.push_back(p);
    return p;
}

double* dev_upload(tb_handle* h, const std::vector<double>& v) {
    double* p = dev_alloc(h, v.size());
    if (p && !v.empty()) cudaMemcpy(p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice);
    return p;
}

int validate(const tb_problem_desc* d) {
    if (!d) { set_error("null problem description"); return TB_ERR_BAD_DESC; }
    if (d->n_bands <= 0 || d->n_bands > TB_MAX_BANDS) { set_error("n_bands must be 1..8"); return TB_ERR_BAD_DESC; }
    if (d->n_meshes <= 0) { set_error("n_meshes must be > 0"); return TB_ERR_BAD_DESC; }
    for (int i = 0; i < d->n_meshes; ++i)
        if (d->meshes[i].nsplit[0] <= 0 || d->meshes[i].nsplit[1] <= 0) {
            set_error("mesh nsplit must be > 0");
            return TB_ERR_BAD_DESC;
        }
    for (int b = 0; b < d->n_bands; ++b) {
        const tb_band_desc& bd = d->bands[b];
        if (bd.mesh < 0 || bd.mesh >= d->n_meshes) { set_error("band mesh index out of range"); return TB_ERR_BAD_DESC; }
        if (!bd.dispersion) { set_error("band without dispersion"); return TB_ERR_BAD_DESC; }
        if (bd.constrained && !bd.constrained_population) {
            set_error("constrained band without population");
            return TB_ERR_BAD_DESC;
        }
        if (bd.statistics != TB_FERMION && bd.statistics != TB_BOSON) {
            set_error("statistics must be -1 (fermion) or +1 (boson)");
            return TB_ERR_BAD_DESC;
        }
    }
    for (int c = 0; c < d->n_channels; ++c) {
        const tb_channel_desc& cd = d->channels[c];
        if (cd.nlegs < 2 || cd.nlegs > 4) { set_error("nlegs must be 2..4"); return TB_ERR_BAD_DESC; }
        for (int l = 0; l < cd.nlegs; ++l) {
            if (cd.band[l] < 0 || cd.band[l] >= d->n_bands) { set_error("leg band out of range"); return TB_ERR_BAD_DESC; }
            if (cd.dir[l] != 1 && cd.dir[l] != -1) { set_error("leg direction must be +1 or -1"); return TB_ERR_BAD_DESC; }
        }
        if (cd.n_mc <= 0 || !cd.mc_points) { set_error("channel without Monte-Carlo points"); return TB_ERR_BAD_DESC; }
        if (cd.n_umklapp <= 0 || !cd.umklapp) { set_error("channel without umklapp vectors"); return TB_ERR_BAD_DESC; }
        if (cd.n_tuples < 0 || (cd.n_tuples > 0 && (!cd.tuples || !cd.tuple_umklapp))) {
            set_error("bad caller-supplied tuple list");
            return TB_ERR_BAD_DESC;
        }
        for (int64_t i = 0; i < cd.n_tuples; ++i) {
            for (int l = 0; l < cd.nlegs; ++l) {
                const int e = cd.tuples[i * cd.nlegs + l];
                const tb_mesh_desc& md = d->meshes[d->bands[cd.band[l]].mesh];
                if (e < 0 || e >= 2 * md.nsplit[0] * md.nsplit[1]) {
                    set_error("tuple element id out of range");
                    return TB_ERR_BAD_DESC;
                }
            }
            if (cd.tuple_umklapp[i] < 0 || cd.tuple_umklapp[i] >= cd.n_umklapp) {
                set_error("tuple umklapp index out of range");
                return TB_ERR_BAD_DESC;
            }
        }
    }
    return TB_OK;
}

int build(tb_handle* h, const tb_problem_desc* d) {
    TB_TRY(validate(d));
    for (int i = 0; i < d->n_meshes; ++i) h->meshes.push_back(make_mesh(d->region, d->meshes[i]));
    int64_t off = 0;
    h->bandsdev.nb = d->n_bands;
    int maxne = 1;
    for (int b = 0; b < d->n_bands; ++b) {
        const tb_band_desc& bd = d->bands[b];
        const HostMesh& m = h->meshes[bd.mesh];
        HostBand B;
        B.mesh = bd.mesh;
        B.ne = m.ne;
        B.off = off;
        B.charge = bd.charge;
        B.stat = bd.statistics;
        B.abs_tol = bd.abs_tol;
        B.rel_tol = bd.rel_tol;
        B.penal = bd.penalisation;
        B.constrained = bd.constrained;
        B.vel[0] = bd.drift_velocity[0];
        B.vel[1] = bd.drift_velocity[1];
        B.disp.assign(bd.dispersion, bd.dispersion + size_t(m.ne) * 3);
        B.kx = coord_function(m, 0);
        B.ky = coord_function(m, 1);
        B.minE.resize(m.ne);
        B.maxE.resize(m.ne);
        for (int e = 0; e < m.ne; ++e) {
            const double n0 = B.disp[3 * e], n1 = B.disp[3 * e + 1] + n0, n2 = B.disp[3 * e + 2] + n0;
            B.minE[e] = std::min(n0, std::min(n1, n2));
            B.maxE[e] = std::max(n0, std::max(n1, n2));
        }
        if (B.constrained) B.cpop.assign(bd.constrained_population, bd.constrained_population + size_t(m.ne) * 3);
        off += int64_t(m.ne) * 3;
        maxne = std::max(maxne, m.ne);
        h->bands.push_back(std::move(B));
    }
    h->ndofs = off;
    h->nblk = (maxne + 255) / 256;
    h->bandsdev.ndofs = off;
    // device band tables
    std::vector<const double*> d_disp(d->n_bands), d_kx(d->n_bands), d_ky(d->n_bands), d_minE(d->n_bands),
        d_maxE(d->n_bands);
    for (int b = 0; b < d->n_bands; ++b) {
        HostBand& B = h->bands[b];
        d_disp[b] = dev_upload(h, B.disp);
        d_kx[b] = dev_upload(h, B.kx);
        d_ky[b] = dev_upload(h, B.ky);
        d_minE[b] = dev_upload(h, B.minE);
        d_maxE[b] = dev_upload(h, B.maxE);
        const double* d_cpop = B.constrained ? dev_upload(h, B.cpop) : nullptr;
        if (!d_disp[b] || !d_kx[b] || !d_ky[b] || !d_minE[b] || !d_maxE[b] || (B.constrained && !d_cpop)) {
            set_error("band table allocation failed");
            return TB_ERR_OOM;
        }
        BandDev& bd = h->bandsdev.b[b];
        const HostMesh& m = h->meshes[B.mesh];
        bd.mesh.nx = m.nx; bd.mesh.ny = m.ny; bd.mesh.ne = m.ne;
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) bd.mesh.dG[i][j] = m.dG[i][j];
        bd.mesh.vol = m.vol;
        bd.mesh.rel_origin[0] = m.rel_origin[0];
        bd.mesh.rel_origin[1] = m.rel_origin[1];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) { bd.mesh.Minv[i][j] = m.Minv[i][j]; bd.mesh.M[i][j] = m.M[i][j]; }
        bd.off = B.off;
        bd.ne = B.ne;
        bd.stat = B.stat;
        bd.abs_tol = B.abs_tol;
        bd.rel_tol = B.rel_tol;
        bd.penal = B.penal;
        bd.constrained = B.constrained;
        bd.cpop = d_cpop;
        bd.vel[0] = B.vel[0];
        bd.vel[1] = B.vel[1];
    }
    // state scratch
    h->d_f = dev_alloc(h, size_t(h->ndofs));
    h->d_out = dev_alloc(h, size_t(h->ndofs));
    h->d_acc = dev_alloc(h, size_t(h->ndofs));
    h->d_part = dev_alloc(h, size_t(2 * TB_MAX_BANDS * h->nblk + 8));
    if (!h->d_f || !h->d_out || !h->d_acc || !h->d_part) { set_error("state allocation failed"); return TB_ERR_OOM; }
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, sizeof(double) * size_t(h->ndofs), h->stream));
    // channels
    h->chans.resize(d->n_channels);
    for (int ci = 0; ci < d->n_channels; ++ci) {
        const tb_channel_desc& cd = d->channels[ci];
        Channel& C = h->chans[ci];
        C.L = cd.nlegs;
        C.amplitude = cd.amplitude;
        ChanDev& c = C.dev;
        c.L = cd.nlegs;
        c.nmc = cd.n_mc;
        c.R = 2 * (cd.nlegs - 2) + 1;
        c.n_umk = cd.n_umklapp;
        double av = 1.0;
        for (int l = 0; l < C.L; ++l) {
            C.band[l] = cd.band[l];
            const HostBand& B = h->bands[cd.band[l]];
            LegDev& lg = c.leg[l];
            lg.disp = d_disp[cd.band[l]];
            lg.kx = d_kx[cd.band[l]];
            lg.ky = d_ky[cd.band[l]];
            lg.foff = B.off;
            lg.dir = double(cd.dir[l]);
            lg.stat = B.stat;
            lg.ne = B.ne;
            av *= h->meshes[B.mesh].vol * 2.0;
        }
        c.amp_vol = av;
        double af = C.amplitude;
        for (int l = 0; l < C.L; ++l) af *= h->meshes[h->bands[cd.band[l]].mesh].vol * 2.0;
        C.amp_full = af;
        c.fact = 1.0;
        for (int i = 0; i < C.L - 2; ++i) c.fact *= 2.0;
        c.min_det = cd.min_det;
        c.threshold = cd.threshold;
        for (int i = 0; i < 4; ++i) c.gvec[i] = d->region.gvec[i];
        C.d_umk = dev_upload(h, std::vector<double>(cd.umklapp, cd.umklapp + 2 * size_t(cd.n_umklapp)));
        C.d_mc = dev_upload(h, std::vector<double>(cd.mc_points, cd.mc_points + size_t(cd.n_mc) * c.R));
        const double* pre = cd.mc_points_precalc ? cd.mc_points_precalc : cd.mc_points;
        C.d_mc_pre = dev_upload(h, std::vector<double>(pre, pre + size_t(cd.n_mc) * c.R));
        if (!C.d_umk || !C.d_mc || !C.d_mc_pre) { set_error("channel table allocation failed"); return TB_ERR_OOM; }
        c.umk = C.d_umk;
        c.mc = C.d_mc;
        if (cd.n_tuples > 0) {
            TB_TRY(C.tup.reserve(C.L, cd.n_tuples, h->stream));
            std::vector<int32_t> soa(size_t(C.L + 1) * size_t(cd.n_tuples));
            for (int64_t i = 0; i < cd.n_tuples; ++i) {
                for (int l = 0; l < C.L; ++l) soa[size_t(l) * cd.n_tuples + i] = cd.tuples[i * C.L + l];
                soa[size_t(C.L) * cd.n_tuples + i] = cd.tuple_umklapp[i];
            }
            TB_CUDA(cudaMemcpy(C.tup.d, soa.data(), sizeof(int32_t) * soa.size(), cudaMemcpyHostToDevice));
            C.tup.n = cd.n_tuples;
            C.diag[0] = C.diag[1] = C.diag[2] = -1;
        } else {
            int legband[TB_MAX_LEGS];
            const double* mins[TB_MAX_LEGS];
            const double* maxs[TB_MAX_LEGS];
            for (int l = 0; l < C.L; ++l) { legband[l] = cd.band[l]; mins[l] = d_minE[cd.band[l]]; maxs[l] = d_maxE[cd.band[l]]; }
            TB_TRY(enumerate_channel(c, h->meshes.data(), h->bands.data(), legband, C.d_mc_pre, mins, maxs, h->stream,
                                     C.tup, C.diag));
        }
    }
    // layouts (and moment tensors)
    TB_TRY(choose_layouts(h));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    return TB_OK;
}

}  // namespace

// The RHS accumulation (pre-M^-1) of the input state into acc (which must be zero).
namespace tb {
int run_rhs_acc(tb_handle* h, const double* d_in, double* d_acc, const int* done, int flags, int only_channel) {
    if (!(flags & TB_NO_COLLISIONS)) {
        for (size_t ci = 0; ci < h->chans.size(); ++ci) {
            if (only_channel >= 0 && int(ci) != only_channel) continue;
            Channel& C = h->chans[ci];
            if (C.amplitude == 0.0 || C.tup.n == 0) continue;
            if (C.layout == TB_LAYOUT_MC64) {
                TB_TRY(launch_collision_mc(C.dev, C.amp_full, C.tup.d, C.tup.cap, C.tup.n, d_in, d_acc, done,
                                           h->stream, 148 * 32));
            } else {
                TB_TRY(launch_collision_tensor(C.dev, C.amplitude, C.tensor, C.tup.d, C.tup.cap, C.tup.n, d_in, d_acc,
                                               done, h->stream));
            }
        }
    }
    if (!(flags & TB_NO_DRIFT) && only_channel < 0) TB_TRY(launch_drift(h->bandsdev, d_in, d_acc, done, h->stream));
    return TB_OK;
}

int choose_layouts(tb_handle* h) {
    // Budget for precomputed tensors
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    int64_t budget = h->opts.tensor_budget_bytes > 0 ? h->opts.tensor_budget_bytes : int64_t(double(freeb) * 0.6);
    for (auto& C : h->chans) {
        int want = h->opts.layout;
        if (want == TB_LAYOUT_AUTO) {
            // L = 3 and L = 2 tensors are cheaper per tuple than the Monte-Carlo
            // evaluation (HBM-bound contraction vs FP64-bound quadrature);
            // for L = 4 the 405-moment tensor costs more bytes than the
            // quadrature costs FP64 cycles on B200.
            if (C.L <= 3) want = h->opts.allow_fp32 ? TB_LAYOUT_T32 : TB_LAYOUT_T64;
            else want = TB_LAYOUT_MC64;
        }
        if (want == TB_LAYOUT_T32 || want == TB_LAYOUT_T64) {
            const int64_t bytes = tensor_bytes(C.L, want == TB_LAYOUT_T32, C.tup.n);
            if (C.tup.n == 0 || bytes > budget) want = TB_LAYOUT_MC64;
            else budget -= bytes;
        }
        C.layout = want;
        if (want != TB_LAYOUT_MC64) TB_TRY(build_tensor(C.dev, C.tup.d, C.tup.cap, C.tup.n, want == TB_LAYOUT_T32,
                                                        C.tensor, h->stream));
    }
    return TB_OK;
}
}  // namespace tb

// ---------------------------------------------------------------- DP45 glue
namespace {

int dp_alloc(tb_handle* h, int64_t max_dense) {
    if (!h->dp_ready) {
        DPBufs& B = h->dp;
        const size_t n = size_t(h->ndofs);
        B.y = dev_alloc(h, n);
        B.tmp = dev_alloc(h, n);
        B.y5 = dev_alloc(h, n);
        for (int i = 0; i < 7; ++i) B.k[i] = dev_alloc(h, n);
        B.acc = h->d_acc;
        B.part = dev_alloc(h, size_t(2 * TB_MAX_BANDS * h->nblk + 8));
        B.nblk = h->nblk;
        DPCtl* c = nullptr;
        if (cudaMalloc(&c, sizeof(DPCtl)) != cudaSuccess) { set_error("controller allocation failed"); return TB_ERR_OOM; }
        B.ctl = c;
        h->dev_allocs.push_back(reinterpret_cast<double*>(c));
        if (cudaMallocHost(&h->h_ctl, sizeof(DPCtl)) != cudaSuccess) { set_error("pinned allocation failed"); return TB_ERR_OOM; }
        for (int i = 0; i < 7; ++i)
            if (!B.k[i]) { set_error("stage allocation failed"); return TB_ERR_OOM; }
        if (!B.y || !B.tmp || !B.y5 || !B.part) { set_error("stage allocation failed"); return TB_ERR_OOM; }
        B.dense = nullptr;
        B.dense_t = nullptr;
        h->dp_ready = true;
    }
    if (max_dense > h->dense_cap_alloc) {
        // (re)allocate the dense buffers; invalidates the captured graph
        DPBufs& B = h->dp;
        if (B.dense) { cudaFree(B.dense); B.dense = nullptr; }
        if (B.dense_t) { cudaFree(B.dense_t); B.dense_t = nullptr; }
        const int64_t cap = std::max<int64_t>(max_dense, 1);
        if (cudaMalloc(&B.dense, sizeof(double) * size_t(cap) * size_t(h->ndofs)) != cudaSuccess ||
            cudaMalloc(&B.dense_t, sizeof(double) * size_t(cap)) != cudaSuccess) {
            set_error("dense output allocation failed");
            return TB_ERR_OOM;
        }
        h->dense_cap_alloc = cap;
        if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    }
    return TB_OK;
}

int record_attempt(tb_handle* h, int flags) {
    const DPBufs& B = h->dp;
    const int* done = &B.ctl->done;
    TB_TRY(launch_stage(h->bandsdev, B, 0, h->stream));
    for (int s = 1; s <= 5; ++s) {
        TB_TRY(run_rhs_acc(h, B.tmp, B.acc, done, flags, -1));
        TB_TRY(launch_stage(h->bandsdev, B, s, h->stream));
    }
    TB_TRY(run_rhs_acc(h, B.y5, B.acc, done, flags, -1));
    TB_TRY(launch_stage(h->bandsdev, B, 6, h->stream));
    TB_TRY(launch_controller(h->bandsdev, B, h->stream));
    TB_TRY(launch_dense_commit(h->bandsdev, B, h->stream));
    return TB_OK;
}

int ensure_graph(tb_handle* h, int flags) {
    if (h->graph && h->graph_flags == flags) return TB_OK;
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    cudaGraph_t g = nullptr;
    TB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = record_attempt(h, flags);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc != TB_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) { set_error(std::string("graph capture: ") + cudaGetErrorString(e)); return TB_ERR_CUDA; }
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { set_error(std::string("graph instantiate: ") + cudaGetErrorString(e)); return TB_ERR_CUDA; }
    h->graph_flags = flags;
    return TB_OK;
}

void fill_stats(const DPCtl& c, tb_dp45_stats* st) {
    if (!st) return;
    st->t = c.t;
    st->dt = c.dt;
    st->last_err = c.last_err;
    st->attempts = c.attempts;
    st->accepted = c.accepted;
    st->rejected = c.rejected_n;
    st->rhs_evals = c.rhs_evals;
    st->n_dense = c.n_dense;
    st->status = c.status;
    st->done = c.done;
}

}  // namespace

// ====================================================================== C API
extern "C" {

const char* tb_last_error(void) { return tb::get_error(); }

int tb_create(tb_handle** out, const tb_problem_desc* desc, const tb_options* opts) {
    if (!out) { set_error("null handle pointer"); return TB_ERR_ARG; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device available");
        return TB_ERR_NO_DEVICE;
    }
    std::unique_ptr<tb_handle> h(new tb_handle());
    if (opts) h->opts = *opts;
    else { h->opts.layout = TB_LAYOUT_AUTO; h->opts.allow_fp32 = 0; }
    h->device = h->opts.device;
    TB_CUDA(cudaSetDevice(h->device));
    TB_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    int rc = build(h.get(), desc);
    if (rc != TB_OK) { tb_destroy(h.release()); return rc; }
    *out = h.release();
    return TB_OK;
}

int tb_destroy(tb_handle* h) {
    if (!h) return TB_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    for (auto& C : h->chans) { C.tup.release(); C.tensor.release(); }
    for (double* p : h->dev_allocs) cudaFree(p);
    if (h->dp.dense) cudaFree(h->dp.dense);
    if (h->dp.dense_t) cudaFree(h->dp.dense_t);
    if (h->h_ctl) cudaFreeHost(h->h_ctl);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return TB_OK;
}

int64_t tb_num_dofs(const tb_handle* h) { return h ? h->ndofs : -1; }

int64_t tb_band_offset(const tb_handle* h, int band) {
    if (!h || band < 0 || band >= int(h->bands.size())) return -1;
    return h->bands[band].off;
}

int tb_num_channels(const tb_handle* h) { return h ? int(h->chans.size()) : -1; }

int tb_channel_info(const tb_handle* h, int ch, int64_t* n_tuples, int64_t* n_prefilter, int64_t* n_det,
                    int32_t* layout) {
    if (!h || ch < 0 || ch >= int(h->chans.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const Channel& C = h->chans[ch];
    if (n_tuples) *n_tuples = C.tup.n;
    if (n_prefilter) *n_prefilter = C.diag[0];
    if (n_det) *n_det = C.diag[1];
    if (layout) *layout = C.layout;
    return TB_OK;
}

int tb_get_tuples(const tb_handle* h, int ch, int32_t* ids, int32_t* umk) {
    if (!h || ch < 0 || ch >= int(h->chans.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const Channel& C = h->chans[ch];
    const int64_t n = C.tup.n;
    if (n == 0) return TB_OK;
    std::vector<int32_t> soa(size_t(C.L + 1) * size_t(n));
    cudaSetDevice(h->device);
    for (int r = 0; r <= C.L; ++r)
        TB_CUDA(cudaMemcpy(soa.data() + size_t(r) * n, C.tup.d + size_t(r) * C.tup.cap, sizeof(int32_t) * size_t(n),
                           cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) {
        if (ids)
            for (int l = 0; l < C.L; ++l) ids[i * C.L + l] = soa[size_t(l) * n + i];
        if (umk) umk[i] = soa[size_t(C.L) * n + i];
    }
    return TB_OK;
}

int tb_set_amplitude(tb_handle* h, int ch, double amplitude) {
    if (!h || ch < 0 || ch >= int(h->chans.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    Channel& C = h->chans[ch];
    C.amplitude = amplitude;
    double af = amplitude;
    for (int l = 0; l < C.L; ++l) af *= h->meshes[h->bands[C.band[l]].mesh].vol * 2.0;
    C.amp_full = af;
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }  // amplitudes are baked into the graph
    return TB_OK;
}

static int rhs_common(tb_handle* h, const double* f, double* out, int flags, int only_channel) {
    if (!h || !f || !out) { set_error("null argument"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const double* d_in = f;
    double* d_res = out;
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(h->d_f, f, bytes, cudaMemcpyHostToDevice, h->stream));
        d_in = h->d_f;
        d_res = h->d_out;
    }
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    TB_TRY(run_rhs_acc(h, d_in, h->d_acc, nullptr, flags, only_channel));
    TB_TRY(launch_inverse_mass(h->bandsdev, h->d_acc, d_res, h->stream));
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(out, h->d_out, bytes, cudaMemcpyDeviceToHost, h->stream));
        TB_CUDA(cudaStreamSynchronize(h->stream));
    }
    return TB_OK;
}

int tb_rhs(tb_handle* h, const double* f, double* dfdt, int flags) { return rhs_common(h, f, dfdt, flags, -1); }

int tb_channel_propagate(tb_handle* h, int ch, const double* f, double* out, int flags) {
    if (!h || ch < 0 || ch >= int(h->chans.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    return rhs_common(h, f, out, flags | TB_NO_DRIFT, ch);
}

int tb_relative_error(tb_handle* h, const double* err, const double* pop, double* result, int flags) {
    if (!h || !err || !pop || !result) { set_error("null argument"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const double *de = err, *dp = pop;
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(h->d_f, err, bytes, cudaMemcpyHostToDevice, h->stream));
        TB_CUDA(cudaMemcpyAsync(h->d_out, pop, bytes, cudaMemcpyHostToDevice, h->stream));
        de = h->d_f;
        dp = h->d_out;
    }
    TB_TRY(launch_error_norm(h->bandsdev, de, dp, h->d_part, h->nblk, h->stream));
    std::vector<double> part(size_t(2 * h->bandsdev.nb * h->nblk));
    TB_CUDA(cudaMemcpyAsync(part.data(), h->d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->stream));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    double errNorm = 0.0;
    for (int b = 0; b < h->bandsdev.nb; ++b) {
        const BandDev& bd = h->bandsdev.b[b];
        double sr = 0.0, sp = 0.0;
        for (int k = 0; k < h->nblk; ++k) { sr += part[size_t(2 * b) * h->nblk + k]; sp += part[size_t(2 * b + 1) * h->nblk + k]; }
        const double be = std::sqrt((bd.mesh.vol * sr + bd.penal * (bd.mesh.vol * sp)) / (double(bd.ne) * bd.mesh.vol));
        if (be >= errNorm) errNorm = be;
    }
    *result = errNorm;
    return TB_OK;
}

int tb_apply_constraints(tb_handle* h, double* f, int flags) {
    if (!h || !f) { set_error("null argument"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(h->d_f, f, bytes, cudaMemcpyHostToDevice, h->stream));
        TB_TRY(launch_enforce(h->bandsdev, h->d_f, h->d_f, h->stream));
        TB_CUDA(cudaMemcpyAsync(f, h->d_f, bytes, cudaMemcpyDeviceToHost, h->stream));
        TB_CUDA(cudaStreamSynchronize(h->stream));
    } else {
        TB_TRY(launch_enforce(h->bandsdev, f, f, h->stream));
    }
    return TB_OK;
}

int tb_dp45_begin(tb_handle* h, const double* f0, double t0, double t_final, double dense_step, int64_t max_dense,
                  int flags) {
    if (!h || !f0) { set_error("null argument"); return TB_ERR_ARG; }
    if (!(dense_step > 0.0)) { set_error("dense_step must be > 0"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(dp_alloc(h, max_dense));
    const int rflags = flags & (TB_NO_DRIFT | TB_NO_COLLISIONS);
    h->dp_flags = flags;
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    DPBufs& B = h->dp;
    TB_CUDA(cudaMemcpyAsync(B.y, f0, bytes, (flags & TB_PTR_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            h->stream));
    DPCtl c;
    std::memset(&c, 0, sizeof(c));
    c.t = t0;
    c.tf = t_final;
    c.dense_step = dense_step;
    c.dense_time = t0 + dense_step;
    c.min_step = dense_step / 10000.;
    c.olderror = 1.0;
    c.dt = dense_step;
    c.dt = std::min(c.dt, (c.t + c.dt) - c.t);   // timeStepVetoer with no time-dependent constraints
    c.dense_cap = max_dense;
    c.rhs_evals = 1;
    c.done = (t0 < t_final) ? 0 : 1;
    *h->h_ctl = c;
    TB_CUDA(cudaMemcpyAsync(B.ctl, h->h_ctl, sizeof(DPCtl), cudaMemcpyHostToDevice, h->stream));
    // k1 = timeOp(t0, enforceValue(t0, y0))
    TB_TRY(launch_enforce(h->bandsdev, B.y, B.tmp, h->stream));
    TB_CUDA(cudaMemsetAsync(B.acc, 0, bytes, h->stream));
    TB_TRY(run_rhs_acc(h, B.tmp, B.acc, nullptr, rflags, -1));
    TB_TRY(launch_k1(h->bandsdev, B, h->stream));
    TB_TRY(ensure_graph(h, rflags));
    return TB_OK;
}

int tb_dp45_advance(tb_handle* h, int64_t n_attempts) {
    if (!h || !h->graph) { set_error("tb_dp45_begin was not called"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    for (int64_t i = 0; i < n_attempts; ++i) TB_CUDA(cudaGraphLaunch(h->graph, h->stream));
    return TB_OK;
}

int tb_dp45_poll(tb_handle* h, tb_dp45_stats* st) {
    if (!h || !h->dp_ready) { set_error("tb_dp45_begin was not called"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_CUDA(cudaMemcpyAsync(h->h_ctl, h->dp.ctl, sizeof(DPCtl), cudaMemcpyDeviceToHost, h->stream));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    fill_stats(*h->h_ctl, st);
    int tflag = 0;
    TB_TRY(tensor_error_flag(&tflag));
    if (tflag && st) { st->status = TB_ERR_TIMEOUT; st->done = 1; }
    return TB_OK;
}

int tb_dp45_end(tb_handle* h, double* f_out, double* dense_out, double* dense_times, int64_t max_dense,
                tb_dp45_stats* st, int flags) {
    tb_dp45_stats s;
    TB_TRY(tb_dp45_poll(h, &s));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const cudaMemcpyKind kind = (flags & TB_PTR_HOST) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (f_out) TB_CUDA(cudaMemcpyAsync(f_out, h->dp.y, bytes, kind, h->stream));
    const int64_t nd = std::min<int64_t>(std::min<int64_t>(s.n_dense, max_dense), h->dense_cap_alloc);
    if (nd > 0 && dense_out) TB_CUDA(cudaMemcpyAsync(dense_out, h->dp.dense, bytes * size_t(nd), kind, h->stream));
    if (nd > 0 && dense_times) TB_CUDA(cudaMemcpyAsync(dense_times, h->dp.dense_t, sizeof(double) * size_t(nd), kind, h->stream));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    if (st) *st = s;
    return s.status;
}

int tb_dp45_integrate(tb_handle* h, double* f_inout, double t0, double t_final, double dense_step, double* dense_out,
                      double* dense_times, int64_t max_dense, tb_dp45_stats* st, int flags) {
    TB_TRY(tb_dp45_begin(h, f_inout, t0, t_final, dense_step, max_dense, flags));
    // speculative batches of attempts: attempts after the end are no-ops
    int64_t batch = 4;
    tb_dp45_stats s;
    for (;;) {
        TB_TRY(tb_dp45_advance(h, batch));
        TB_TRY(tb_dp45_poll(h, &s));
        if (s.done) break;
        if (batch < 64) batch *= 2;
    }
    return tb_dp45_end(h, f_inout, dense_out, dense_times, max_dense, st, flags);
}

int tb_synchronize(tb_handle* h) {
    if (!h) return TB_ERR_ARG;
    TB_CUDA(cudaStreamSynchronize(h->stream));
    return TB_OK;
}

void* tb_get_stream(tb_handle* h) { return h ? (void*)h->stream : nullptr; }

int tb_collision_accumulate(tb_handle* h, int ch, const double* f, double* acc) {
    if (!h || !f || !acc) { set_error("null argument"); return TB_ERR_ARG; }
    if (ch < -1 || ch >= int(h->chans.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    return run_rhs_acc(h, f, acc, nullptr, TB_NO_DRIFT, ch);
}

}  // extern "C"
