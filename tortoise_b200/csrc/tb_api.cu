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
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "tb_handle.cuh"

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

}  // namespace tb

using namespace tb;

namespace tb {
int choose_layouts(tb_handle* h);
int autotune(tb_handle* h);
}  // namespace tb

namespace tb {

double* dev_alloc(tb_handle* h, size_t n) {
    double* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * (n ? n : 1)) != cudaSuccess) return nullptr;
    h->dev_allocs.push_back(p);
    return p;
}

int fx_alloc(tb_handle* h, int64_t n, FxAcc& out) {
    void* p = nullptr;
    const size_t bytes = sizeof(unsigned long long) * size_t(3 * n + 1);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("exact accumulator allocation failed");
        return TB_ERR_OOM;
    }
    h->dev_raw.push_back(p);
    TB_CUDA(cudaMemset(p, 0, bytes));
    out.w = static_cast<unsigned long long*>(p);
    // the last word: the poison flag (cleared by every flush), then the
    // sticky saturation flag (cleared by the host when it reports it)
    out.poison = reinterpret_cast<unsigned int*>(out.w + 3 * n);
    out.sat = out.poison + 1;
    return TB_OK;
}

template <typename T>
T* dev_upload_raw(tb_handle* h, const T* src, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
    h->dev_raw.push_back(p);
    if (n) cudaMemcpy(p, src, sizeof(T) * n, cudaMemcpyHostToDevice);
    return static_cast<T*>(p);
}

double* dev_upload(tb_handle* h, const std::vector<double>& v) {
    double* p = dev_alloc(h, v.size());
    if (p && !v.empty()) cudaMemcpy(p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice);
    return p;
}

int validate(const tb_problem_desc* d) {
    if (!d) { set_error("null problem description"); return TB_ERR_BAD_DESC; }
    if (d->n_bands <= 0) { set_error("n_bands must be > 0"); return TB_ERR_BAD_DESC; }
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

// Bytes that decide the structure of a run: region, meshes, band dispersions
// and statistics, channel definitions, Monte-Carlo tables and supplied tuple
// lists.  Runs with equal keys share tuple lists and moment tensors;
// amplitudes, tolerances, constraints, drift and states may differ.
std::string structure_key(const tb_problem_desc* d) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    put(&d->region, sizeof(tb_region));
    put(&d->n_meshes, sizeof(int32_t));
    for (int i = 0; i < d->n_meshes; ++i) put(&d->meshes[i], sizeof(tb_mesh_desc));
    put(&d->n_bands, sizeof(int32_t));
    for (int b = 0; b < d->n_bands; ++b) {
        const tb_band_desc& bd = d->bands[b];
        put(&bd.mesh, sizeof(int32_t));
        put(&bd.statistics, sizeof(double));
        const tb_mesh_desc& md = d->meshes[bd.mesh];
        put(bd.dispersion, sizeof(double) * size_t(2 * md.nsplit[0] * md.nsplit[1]) * 3);
    }
    put(&d->n_channels, sizeof(int32_t));
    for (int c = 0; c < d->n_channels; ++c) {
        const tb_channel_desc& cd = d->channels[c];
        put(&cd.nlegs, sizeof(int32_t));
        put(cd.band, sizeof(cd.band));
        put(cd.dir, sizeof(cd.dir));
        put(&cd.n_mc, sizeof(int32_t));
        put(&cd.min_det, sizeof(double));
        put(&cd.threshold, sizeof(double));
        put(&cd.n_umklapp, sizeof(int32_t));
        put(cd.umklapp, sizeof(double) * 2 * size_t(cd.n_umklapp));
        const int R = 2 * (cd.nlegs - 2) + 1;
        put(cd.mc_points, sizeof(double) * size_t(cd.n_mc) * R);
        const double* pre = cd.mc_points_precalc ? cd.mc_points_precalc : cd.mc_points;
        put(pre, sizeof(double) * size_t(cd.n_mc) * R);
        put(&cd.n_tuples, sizeof(int64_t));
        if (cd.n_tuples > 0) {
            put(cd.tuples, sizeof(int32_t) * size_t(cd.n_tuples) * cd.nlegs);
            put(cd.tuple_umklapp, sizeof(int32_t) * size_t(cd.n_tuples));
        }
    }
    return k;
}

double amp_full_of(tb_handle* h, const ChanInst& ci, int L, double amplitude) {
    double af = amplitude;   // constructAmplitude order: amplitude * prod_l (vol_l * 2)
    for (int l = 0; l < L; ++l) af *= h->meshes[h->bands[ci.band[l]].mesh].vol * 2.0;
    return af;
}

int build_runs(tb_handle* h, const tb_problem_desc* const* descs, int nruns) {
    if (nruns <= 0) { set_error("at least one run is needed"); return TB_ERR_ARG; }
    for (int r = 0; r < nruns; ++r) TB_TRY(validate(descs[r]));
    std::vector<std::string> keys(nruns);
    std::vector<int> group_of_run(nruns, -1), group_first_run;
    int64_t off = 0;
    for (int r = 0; r < nruns; ++r) {
        const tb_problem_desc* d = descs[r];
        RunInfo ri;
        ri.band0 = int(h->bands.size());
        ri.nbands = d->n_bands;
        ri.dof_off = off;
        const int mesh0 = int(h->meshes.size());
        for (int i = 0; i < d->n_meshes; ++i) h->meshes.push_back(make_mesh(d->region, d->meshes[i]));
        for (int b = 0; b < d->n_bands; ++b) {
            const tb_band_desc& bd = d->bands[b];
            const HostMesh& m = h->meshes[mesh0 + bd.mesh];
            HostBand B;
            B.mesh = mesh0 + bd.mesh;
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
            if (B.constrained) B.cpop.assign(bd.constrained_population, bd.constrained_population + size_t(m.ne) * 3);
            off += int64_t(m.ne) * 3;
            h->bands.push_back(std::move(B));
        }
        ri.ndofs = off - ri.dof_off;
        ri.chan0 = int(h->insts.size());
        ri.nchans = d->n_channels;
        h->runs.push_back(ri);
        keys[r] = structure_key(d);
        for (int q = 0; q < int(group_first_run.size()); ++q)
            if (keys[group_first_run[q]] == keys[r]) { group_of_run[r] = q; break; }
        if (group_of_run[r] < 0) {
            group_of_run[r] = int(group_first_run.size());
            group_first_run.push_back(r);
        }
        for (int c = 0; c < d->n_channels; ++c) h->insts.emplace_back();
    }
    h->ndofs = off;
    // per-band device tables (every band its own; equal-structure runs read
    // their group's first-run tables inside the channel kernels)
    const int nb = int(h->bands.size());
    std::vector<const double*> d_disp(nb), d_kx(nb), d_ky(nb), d_minE(nb), d_maxE(nb);
    h->banddev.resize(nb);
    for (int b = 0; b < nb; ++b) {
        HostBand& B = h->bands[b];
        const HostMesh& m = h->meshes[B.mesh];
        const int r = int(std::upper_bound(h->runs.begin(), h->runs.end(), b,
                                           [](int x, const RunInfo& ri) { return x < ri.band0; }) - h->runs.begin()) - 1;
        const bool first_of_group = group_first_run[group_of_run[r]] == r;
        if (first_of_group) {
            B.kx = coord_function(m, 0);
            B.ky = coord_function(m, 1);
            B.minE.resize(m.ne);
            B.maxE.resize(m.ne);
            for (int e = 0; e < m.ne; ++e) {
                const double n0 = B.disp[3 * e], n1 = B.disp[3 * e + 1] + n0, n2 = B.disp[3 * e + 2] + n0;
                B.minE[e] = std::min(n0, std::min(n1, n2));
                B.maxE[e] = std::max(n0, std::max(n1, n2));
            }
            d_disp[b] = dev_upload(h, B.disp);
            d_kx[b] = dev_upload(h, B.kx);
            d_ky[b] = dev_upload(h, B.ky);
            d_minE[b] = dev_upload(h, B.minE);
            d_maxE[b] = dev_upload(h, B.maxE);
            if (!d_disp[b] || !d_kx[b] || !d_ky[b] || !d_minE[b] || !d_maxE[b]) {
                set_error("band table allocation failed");
                return TB_ERR_OOM;
            }
        }
        const double* d_cpop = B.constrained ? dev_upload(h, B.cpop) : nullptr;
        if (B.constrained && !d_cpop) { set_error("band table allocation failed"); return TB_ERR_OOM; }
        BandDev& bd = h->banddev[b];
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
        bd.coff = B.constrained ? h->cdofs : -1;
        h->coff.push_back(bd.coff);
        if (B.constrained) h->cdofs += 3 * int64_t(B.ne);
        bd.vel[0] = B.vel[0];
        bd.vel[1] = B.vel[1];
        if (B.vel[0] != 0.0 || B.vel[1] != 0.0) h->any_drift = true;
    }
    // element blocks
    std::vector<int> blk_first(nb + 1, 0), blk_band, band_run(nb);
    for (int b = 0; b < nb; ++b) {
        const int nblk = (h->bands[b].ne + 255) / 256;
        blk_first[b + 1] = blk_first[b] + nblk;
        for (int k = 0; k < nblk; ++k) blk_band.push_back(b);
    }
    for (int r = 0; r < nruns; ++r)
        for (int b = h->runs[r].band0; b < h->runs[r].band0 + h->runs[r].nbands; ++b) band_run[b] = r;
    h->ed.bands = dev_upload_raw(h, h->banddev.data(), h->banddev.size());
    h->ed.band_run = dev_upload_raw(h, band_run.data(), band_run.size());
    h->ed.blk_band = dev_upload_raw(h, blk_band.data(), blk_band.size());
    h->ed.blk_first = dev_upload_raw(h, blk_first.data(), blk_first.size());
    h->ed.nb = nb;
    h->ed.nblk = blk_first[nb];
    h->ed.ndofs = h->ndofs;
    if (!h->ed.bands || !h->ed.band_run || !h->ed.blk_band || !h->ed.blk_first) {
        set_error("element table allocation failed");
        return TB_ERR_OOM;
    }
    h->hruns.resize(nruns);
    for (int r = 0; r < nruns; ++r) {
        RunDev& rd = h->hruns[r];
        rd.band0 = h->runs[r].band0;
        rd.nbands = h->runs[r].nbands;
        rd.blk0 = blk_first[rd.band0];
        rd.blk1 = blk_first[rd.band0 + rd.nbands];
        rd.dof_off = h->runs[r].dof_off;
        rd.ndofs = h->runs[r].ndofs;
        rd.dense_off = 0;
        rd.dense_t_off = 0;
    }
    // state scratch
    h->d_f = dev_alloc(h, size_t(h->ndofs));
    h->d_out = dev_alloc(h, size_t(h->ndofs));
    h->d_acc = dev_alloc(h, size_t(h->ndofs));
    h->d_part = dev_alloc(h, size_t(2 * h->ed.nblk + 8));
    if (!h->d_f || !h->d_out || !h->d_acc || !h->d_part) { set_error("state allocation failed"); return TB_ERR_OOM; }
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, sizeof(double) * size_t(h->ndofs), h->stream));
    if (h->opts.deterministic) TB_TRY(fx_alloc(h, h->ndofs, h->fx));
    {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) { set_error("flag allocation failed"); return TB_ERR_OOM; }
        h->dev_raw.push_back(p);
        h->d_err = static_cast<int*>(p);
        TB_CUDA(cudaMemset(h->d_err, 0, sizeof(int)));
    }
    // channel groups and instances
    std::vector<int> group_chan0(group_first_run.size(), -1);
    for (int r = 0; r < nruns; ++r) {
        const tb_problem_desc* d = descs[r];
        const int g = group_of_run[r];
        const RunInfo& ri = h->runs[r];
        if (group_first_run[g] == r) {
            group_chan0[g] = int(h->groups.size());
            for (int ci = 0; ci < d->n_channels; ++ci) {
                const tb_channel_desc& cd = d->channels[ci];
                h->groups.emplace_back();
                GroupChan& G = h->groups.back();
                G.L = cd.nlegs;
                ChanDev& c = G.dev;
                c.L = cd.nlegs;
                c.nmc = cd.n_mc;
                c.R = 2 * (cd.nlegs - 2) + 1;
                c.n_umk = cd.n_umklapp;
                double av = 1.0;
                for (int l = 0; l < G.L; ++l) {
                    const int gb = ri.band0 + cd.band[l];
                    const HostBand& B = h->bands[gb];
                    LegDev& lg = c.leg[l];
                    lg.disp = d_disp[gb];
                    lg.kx = d_kx[gb];
                    lg.ky = d_ky[gb];
                    lg.foff = B.off;
                    lg.dir = double(cd.dir[l]);
                    lg.stat = B.stat;
                    lg.ne = B.ne;
                    {
                        const double d = lg.dir, st = lg.stat, ka = (l == 0 ? -1.0 : 1.0) * 0.5;
                        lg.fa = ka * ((1. - d) * st + (1. + d));
                        lg.fa0 = ka * (1. - d);
                        lg.fb = 0.5 * ((1. + d) * st + (1. - d));
                        lg.fb0 = 0.5 * (1. + d);
                    }
                    av *= h->meshes[B.mesh].vol * 2.0;
                }
                c.amp_vol = av;
                // segments of the shared-memory accumulator: the distinct
                // bands of the legs, in leg order
                c.nseg = 0;
                c.sinst = 0;
                for (int l = 0; l < G.L; ++l) {
                    int s = 0;
                    while (s < c.nseg && cd.band[c.seg_leg[s]] != cd.band[l]) ++s;
                    if (s == c.nseg) {
                        c.seg_leg[s] = l;
                        c.seg_off[s] = c.sinst;
                        c.sinst += 3 * c.leg[l].ne;
                        ++c.nseg;
                    }
                    c.sseg[l] = c.seg_off[s];
                }
                c.fact = 1.0;
                for (int i = 0; i < G.L - 2; ++i) c.fact *= 2.0;
                c.min_det = cd.min_det;
                c.threshold = cd.threshold;
                c.err_flag = h->d_err;
                for (int i = 0; i < 4; ++i) c.gvec[i] = d->region.gvec[i];
                G.d_umk = dev_upload(h, std::vector<double>(cd.umklapp, cd.umklapp + 2 * size_t(cd.n_umklapp)));
                G.d_mc = dev_upload(h, std::vector<double>(cd.mc_points, cd.mc_points + size_t(cd.n_mc) * c.R));
                const double* pre = cd.mc_points_precalc ? cd.mc_points_precalc : cd.mc_points;
                G.d_mc_pre = dev_upload(h, std::vector<double>(pre, pre + size_t(cd.n_mc) * c.R));
                if (!G.d_umk || !G.d_mc || !G.d_mc_pre) { set_error("channel table allocation failed"); return TB_ERR_OOM; }
                c.umk = G.d_umk;
                c.mc = G.d_mc;
                if (cd.n_tuples > 0) {
                    TB_TRY(G.tup.reserve(G.L, cd.n_tuples, h->stream));
                    std::vector<int32_t> soa(size_t(G.L + 1) * size_t(cd.n_tuples));
                    for (int64_t i = 0; i < cd.n_tuples; ++i) {
                        for (int l = 0; l < G.L; ++l) soa[size_t(l) * cd.n_tuples + i] = cd.tuples[i * G.L + l];
                        soa[size_t(G.L) * cd.n_tuples + i] = cd.tuple_umklapp[i];
                    }
                    TB_CUDA(cudaMemcpy(G.tup.d, soa.data(), sizeof(int32_t) * soa.size(), cudaMemcpyHostToDevice));
                    G.tup.n = cd.n_tuples;
                    G.diag[0] = G.diag[1] = G.diag[2] = -1;
                } else if (h->opts.stream_legs >= 2 && G.L >= h->opts.stream_legs) {
                    // no stored list: the walk of precalculateIndices runs in every evaluation
                    if (cd.n_mc > 64) { set_error("streamed channels take at most 64 Monte-Carlo points"); return TB_ERR_BAD_DESC; }
                    StreamDev& sd = G.sdev;
                    for (int l = 0; l < TB_MAX_LEGS; ++l) sd.nsec[l] = 1;
                    sd.n_items = c.n_umk;
                    for (int l = 0; l < G.L; ++l) {
                        const int b = ri.band0 + cd.band[l];
                        const HostMesh& m = h->meshes[h->bands[b].mesh];
                        WalkLeg& w = sd.leg[l];
                        w.minE = d_minE[b];
                        w.maxE = d_maxE[b];
                        w.nx = m.nx;
                        w.ny = m.ny;
                        for (int i = 0; i < 2; ++i) {
                            w.origin[i] = m.origin[i];
                            for (int j = 0; j < 2; ++j) { w.dG[i][j] = m.dG[i][j]; w.invdG[i][j] = m.invdG[i][j]; }
                        }
                        if (l < G.L - 1) {
                            sd.nsec[l] = int64_t(m.nx) * m.ny;
                            sd.n_items *= sd.nsec[l];
                        }
                    }
                    sd.n_items *= int64_t(1) << (G.L - 1);
                    sd.mc_pre = G.d_mc_pre;
                    void* p = nullptr;
                    if (cudaMalloc(&p, sizeof(unsigned long long) * 5) != cudaSuccess) {
                        set_error("count buffer allocation failed");
                        return TB_ERR_OOM;
                    }
                    h->dev_raw.push_back(p);
                    sd.counts = static_cast<unsigned long long*>(p);
                    TB_CUDA(cudaMemset(sd.counts, 0, sizeof(unsigned long long) * 5));
                    G.stream = true;
                    G.layout = TB_LAYOUT_STREAM;
                    G.item_begin = 0;
                    G.item_end = sd.n_items;
                    G.diag[0] = G.diag[1] = G.diag[2] = -1;
                } else {
                    int legband[TB_MAX_LEGS];
                    const double* mins[TB_MAX_LEGS];
                    const double* maxs[TB_MAX_LEGS];
                    for (int l = 0; l < G.L; ++l) {
                        legband[l] = ri.band0 + cd.band[l];
                        mins[l] = d_minE[legband[l]];
                        maxs[l] = d_maxE[legband[l]];
                    }
                    NvtxRange enum_range("tb_create: enumerate tuples");
                    TB_TRY(enumerate_channel(c, h->meshes.data(), h->bands.data(), legband, G.d_mc_pre, mins, maxs,
                                             h->stream, G.tup, G.diag));
                }
            }
        }
        for (int ci = 0; ci < d->n_channels; ++ci) {
            const tb_channel_desc& cd = d->channels[ci];
            const int id = ri.chan0 + ci;
            ChanInst& I = h->insts[id];
            I.group = group_chan0[g] + ci;
            I.run = r;
            for (int l = 0; l < cd.nlegs; ++l) I.band[l] = ri.band0 + cd.band[l];
            I.amplitude = cd.amplitude;
            I.dev.run = r;
            for (int l = 0; l < TB_MAX_LEGS; ++l) I.dev.foff[l] = (l < cd.nlegs) ? h->bands[I.band[l]].off : 0;
            I.dev.amplitude = cd.amplitude;
            I.dev.amp_full = amp_full_of(h, I, cd.nlegs, cd.amplitude);
            GroupChan& G = h->groups[I.group];
            I.slot = int(G.insts.size());
            G.insts.push_back(id);
        }
    }
    for (auto& G : h->groups) {
        std::vector<InstDev> v;
        for (int id : G.insts) v.push_back(h->insts[id].dev);
        G.d_insts = dev_upload_raw(h, v.data(), v.size());
        if (!G.d_insts) { set_error("instance table allocation failed"); return TB_ERR_OOM; }
    }
    for (auto& I : h->insts) {
        I.d_single = dev_upload_raw(h, &I.dev, 1);
        if (!I.d_single) { set_error("instance table allocation failed"); return TB_ERR_OOM; }
    }
    for (auto& G : h->groups) TB_TRY(shard_tuples(h, G));
    {
        NvtxRange r("tb_create: layouts and moment tensors");
        TB_TRY(choose_layouts(h));
    }
    {
        NvtxRange r("tb_create: points inside the simplices");
        for (auto& G : h->groups)
            if (G.layout == TB_LAYOUT_MC64) TB_TRY(build_theta_list(G.dev, G.tup, G.theta, h->stream));
    }
    if (h->opts.autotune) {
        NvtxRange r("tb_create: autotune");
        TB_TRY(autotune(h));
    }
    TB_CUDA(cudaStreamSynchronize(h->stream));
    return TB_OK;
}

}  // namespace tb

// The RHS accumulation (pre-M^-1) of the input state into acc (which must be zero).
namespace tb {
// The Monte-Carlo collision of group G: over its ThetaList when in use, else
// the full quadrature of every tuple.
static int launch_group_mc(tb_handle* h, GroupChan& G, const InstDev* insts, int n_insts, const double* d_in,
                           double* d_acc, const DPCtl* ctl, int rate_leg) {
    if (G.theta.use)
        return launch_collision_mc(G.dev, insts, n_insts, G.theta.ids, G.theta.n, G.theta.n, d_in, d_acc, ctl,
                                   h->stream, 148 * 32, rate_leg, G.theta.mask, G.theta.perm, h->fx);
    return launch_collision_mc(G.dev, insts, n_insts, G.tup.d, G.tup.cap, G.tup.n, d_in, d_acc, ctl, h->stream,
                               148 * 32, rate_leg, nullptr, nullptr, h->fx);
}

// A streamed group over this handle's work items.  Outside an integration
// (ctl == nullptr) the launch records its counts for tb_channel_info; the
// attempts of an integration leave them alone.
static int launch_group_stream(tb_handle* h, GroupChan& G, const InstDev* insts, int n_insts, const double* d_in,
                               double* d_acc, const DPCtl* ctl, int rate_leg) {
    StreamDev sd = G.sdev;
    if (ctl) sd.counts = nullptr;
    else TB_CUDA(cudaMemsetAsync(sd.counts, 0, sizeof(unsigned long long) * 5, h->stream));
    return launch_collision_stream(G.dev, sd, G.item_begin, G.item_end, insts, n_insts, d_in, d_acc, ctl, h->stream,
                                   rate_leg, h->fx);
}

int run_rhs_acc(tb_handle* h, const double* d_in, double* d_acc, const DPCtl* ctl, int flags, int only_inst) {
    if (!(flags & TB_NO_COLLISIONS)) {
        for (size_t gi = 0; gi < h->groups.size(); ++gi) {
            GroupChan& G = h->groups[gi];
            if (G.tup.n == 0 && !G.stream) continue;
            const InstDev* insts = G.d_insts;
            int n_insts = int(G.insts.size());
            if (only_inst >= 0) {
                if (h->insts[only_inst].group != int(gi)) continue;
                insts = h->insts[only_inst].d_single;
                n_insts = 1;
            } else {
                bool any = false;
                for (int id : G.insts) any |= h->insts[id].amplitude != 0.0;
                if (!any) continue;
            }
            if (G.stream) {
                TB_TRY(launch_group_stream(h, G, insts, n_insts, d_in, d_acc, ctl, -1));
            } else if (G.layout == TB_LAYOUT_MC64) {
                TB_TRY(launch_group_mc(h, G, insts, n_insts, d_in, d_acc, ctl, -1));
            } else {
                TB_TRY(launch_collision_tensor(G.dev, insts, n_insts, G.tensor, G.tup.d, G.tup.cap, G.tup.n, d_in,
                                               d_acc, ctl, h->stream, -1, h->fx));
            }
        }
        // deterministic mode: the exact sums, rounded once, into d_acc
        TB_TRY(launch_fx_flush(h->fx, d_acc, h->ndofs, h->stream));
        // sharded: the partial collision sums of all ranks, before the
        // (replicated) drift term
        TB_TRY(shard_allreduce(h, d_acc, size_t(h->ndofs)));
    }
    if (!(flags & TB_NO_DRIFT) && only_inst < 0 && h->any_drift) TB_TRY(launch_drift(h->ed, d_in, d_acc, ctl, h->stream));
    return TB_OK;
}

// Times every contraction schedule of every moment-tensor group on a
// representative state (all coefficients 0.25; the cost does not depend on
// the values) and keeps the fastest (tune_tensor).  The accumulator is
// cleared afterwards.
int autotune(tb_handle* h) {
    const size_t n = size_t(h->ndofs);
    std::vector<double> probe(n, 0.25);
    TB_CUDA(cudaMemcpyAsync(h->d_f, probe.data(), sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    for (auto& G : h->groups) {
        if (G.layout == TB_LAYOUT_MC64 || G.tup.n == 0) continue;
        TB_TRY(tune_tensor(G.dev, G.d_insts, int(G.insts.size()), G.tensor, G.tup.d, G.tup.cap, G.tup.n, h->d_f,
                           h->d_acc, h->stream));
    }
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, sizeof(double) * n, h->stream));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    return TB_OK;
}

int choose_layouts(tb_handle* h) {
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    int64_t budget = h->opts.tensor_budget_bytes > 0 ? h->opts.tensor_budget_bytes : int64_t(double(freeb) * 0.6);
    for (auto& G : h->groups) {
        if (G.stream) continue;   // TB_LAYOUT_STREAM, fixed at creation
        int want = h->opts.layout;
        if (want == TB_LAYOUT_AUTO) {
            // L = 3 and L = 2 tensors are cheaper per tuple than the Monte-Carlo
            // evaluation (HBM-bound contraction vs FP64-bound quadrature);
            // for L = 4 the 405-moment tensor costs more bytes than the
            // quadrature costs FP64 cycles on B200.
            // allow_fp32 = 1: FP32 moments; 2: 40-bit, 3: 48-bit (upper bits of FP64) moments
            if (G.L <= 3)
                want = h->opts.allow_fp32 == 1   ? TB_LAYOUT_T32
                       : h->opts.allow_fp32 == 2 ? TB_LAYOUT_T40
                       : h->opts.allow_fp32 == 3 ? TB_LAYOUT_T48
                                                 : TB_LAYOUT_T64;
            else want = TB_LAYOUT_MC64;
        }
        const int kind = (want == TB_LAYOUT_T32)   ? TK_F32
                         : (want == TB_LAYOUT_T40) ? TK_F40
                         : (want == TB_LAYOUT_T48) ? TK_F48
                                                   : TK_F64;
        if (want == TB_LAYOUT_T32 || want == TB_LAYOUT_T64 || want == TB_LAYOUT_T40 || want == TB_LAYOUT_T48) {
            const int64_t bytes = tensor_bytes(G.L, kind, G.tup.n);
            if (G.tup.n == 0 || bytes > budget) want = TB_LAYOUT_MC64;
            else budget -= bytes;
        }
        G.layout = want;
        if (want != TB_LAYOUT_MC64) {
            TB_TRY(build_tensor(G.dev, G.tup.d, G.tup.cap, G.tup.n, kind, G.tensor, h->stream));
            std::vector<int> runs_of;
            for (int id : G.insts) runs_of.push_back(h->insts[id].run);
            std::sort(runs_of.begin(), runs_of.end());
            const bool distinct = std::adjacent_find(runs_of.begin(), runs_of.end()) == runs_of.end();
            TB_TRY(prepare_runs(G.dev, int(G.insts.size()), distinct, G.tensor, h->stream,
                                h->opts.deterministic != 0));
        }
    }
    return TB_OK;
}
}  // namespace tb

// ---------------------------------------------------------------- DP45 glue
namespace tb {

int dp_alloc(tb_handle* h, int64_t max_dense) {
    const int nruns = int(h->runs.size());
    if (!h->dp_ready) {
        DPBufs& B = h->dp;
        const size_t n = size_t(h->ndofs);
        B.y = dev_alloc(h, n);
        B.tmp = dev_alloc(h, n);
        B.y5 = dev_alloc(h, n);
        for (int i = 0; i < 7; ++i) B.k[i] = dev_alloc(h, n);
        B.acc = h->d_acc;
        B.part = dev_alloc(h, size_t(2 * h->ed.nblk + 8));
        B.nblk = h->ed.nblk;
        B.nruns = nruns;
        DPCtl* c = nullptr;
        if (cudaMalloc(&c, sizeof(DPCtl) * nruns) != cudaSuccess) { set_error("controller allocation failed"); return TB_ERR_OOM; }
        B.ctl = c;
        h->dev_raw.push_back(c);
        if (cudaMallocHost(&h->h_ctl, sizeof(DPCtl) * nruns) != cudaSuccess) {
            set_error("pinned allocation failed");
            return TB_ERR_OOM;
        }
        for (int i = 0; i < 7; ++i)
            if (!B.k[i]) { set_error("stage allocation failed"); return TB_ERR_OOM; }
        if (!B.y || !B.tmp || !B.y5 || !B.part) { set_error("stage allocation failed"); return TB_ERR_OOM; }
        B.dense = nullptr;
        B.dense_t = nullptr;
        h->dp_ready = true;
    }
    if (max_dense > h->dense_cap_alloc || !h->d_runs) {
        // (re)allocate the dense buffers; invalidates the captured graph
        DPBufs& B = h->dp;
        if (B.dense) { cudaFree(B.dense); B.dense = nullptr; }
        if (B.dense_t) { cudaFree(B.dense_t); B.dense_t = nullptr; }
        const int64_t cap = std::max<int64_t>(max_dense, 1);
        int64_t doff = 0, toff = 0;
        for (int r = 0; r < nruns; ++r) {
            h->hruns[r].dense_off = doff;
            h->hruns[r].dense_t_off = toff;
            doff += cap * h->hruns[r].ndofs;
            toff += cap;
        }
        if (cudaMalloc(&B.dense, sizeof(double) * size_t(doff)) != cudaSuccess ||
            cudaMalloc(&B.dense_t, sizeof(double) * size_t(toff)) != cudaSuccess) {
            set_error("dense output allocation failed");
            return TB_ERR_OOM;
        }
        if (!h->d_runs) {
            h->d_runs = dev_upload_raw(h, h->hruns.data(), h->hruns.size());
            if (!h->d_runs) { set_error("run table allocation failed"); return TB_ERR_OOM; }
        } else {
            TB_CUDA(cudaMemcpy(h->d_runs, h->hruns.data(), sizeof(RunDev) * h->hruns.size(), cudaMemcpyHostToDevice));
        }
        B.runs = h->d_runs;
        h->dense_cap_alloc = cap;
        if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    }
    return TB_OK;
}

int record_attempt(tb_handle* h, int flags) {
    const DPBufs& B = h->dp;
    if (h->cfn) TB_TRY(tc_record_pre_attempt(h));   // veto + constrained values of this attempt
    TB_TRY(launch_stage(h->ed, B, 0, h->stream));
    for (int s = 1; s <= 5; ++s) {
        TB_TRY(run_rhs_acc(h, B.tmp, B.acc, B.ctl, flags, -1));
        TB_TRY(launch_stage(h->ed, B, s, h->stream));
    }
    TB_TRY(run_rhs_acc(h, B.y5, B.acc, B.ctl, flags, -1));
    TB_TRY(launch_stage(h->ed, B, 6, h->stream));
    TB_TRY(launch_controller(h->ed, B, h->stream));
    TB_TRY(launch_dense_commit(h->ed, B, h->stream));
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

// Deterministic mode: was a contribution clamped to the exact accumulator's
// range since the flag was last cleared?  Reading clears it.
int fx_take_saturation(tb_handle* h, bool& clamped) {
    clamped = false;
    if (!h->fx.sat) return TB_OK;
    unsigned int v = 0;
    TB_CUDA(cudaMemcpyAsync(&v, h->fx.sat, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    if (v) {
        clamped = true;
        TB_CUDA(cudaMemsetAsync(h->fx.sat, 0, sizeof(v), h->stream));
    }
    return TB_OK;
}

int fx_saturation_error() {
    set_error("deterministic mode: a contribution of magnitude 2^64 or more was clamped to the exact accumulator's "
              "range; the result is unreliable");
    return TB_ERR_NONFINITE;
}
}  // namespace tb

// ====================================================================== C API
extern "C" {

const char* tb_last_error(void) { return tb::get_error(); }

int tb_create_batch(tb_handle** out, const tb_problem_desc* const* runs, int n_runs, const tb_options* opts) {
    if (!out || !runs) { set_error("null argument"); return TB_ERR_ARG; }
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
    if (h->opts.layout < TB_LAYOUT_AUTO || h->opts.layout > TB_LAYOUT_T48 || h->opts.allow_fp32 < 0 ||
        h->opts.allow_fp32 > 3) {
        set_error("tb_options: layout must be 0..5 and allow_fp32 0..3");
        return TB_ERR_ARG;
    }
    if (h->opts.stream_legs != 0 && (h->opts.stream_legs < 2 || h->opts.stream_legs > TB_MAX_LEGS)) {
        set_error("tb_options: stream_legs must be 0 or 2..4");
        return TB_ERR_ARG;
    }
    if (h->opts.deterministic != 0 && h->opts.deterministic != 1) {
        set_error("tb_options: deterministic must be 0 or 1");
        return TB_ERR_ARG;
    }
    if (h->opts.shard_count < 0 || h->opts.shard_rank < 0 ||
        (h->opts.shard_rank > 0 && h->opts.shard_rank >= h->opts.shard_count)) {
        set_error("tb_options: need 0 <= shard_rank < shard_count (or both 0)");
        return TB_ERR_ARG;
    }
    h->device = h->opts.device;
    NvtxRange range("tb_create");
    TB_CUDA(cudaSetDevice(h->device));
    TB_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    int rc = build_runs(h.get(), runs, n_runs);
    if (rc != TB_OK) { tb_destroy(h.release()); return rc; }
    *out = h.release();
    return TB_OK;
}

int tb_create(tb_handle** out, const tb_problem_desc* desc, const tb_options* opts) {
    const tb_problem_desc* one[1] = {desc};
    return tb_create_batch(out, one, 1, opts);
}

int tb_destroy(tb_handle* h) {
    if (!h) return TB_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    shard_release(h);
    tc_release(h);
    adjoint_release(h);
    for (auto& G : h->groups) {
        G.tup.release();
        G.tensor.release();
        G.theta.release();
        if (G.d_tamp) cudaFree(G.d_tamp);
    }
    for (double* p : h->dev_allocs) cudaFree(p);
    for (void* p : h->dev_raw) cudaFree(p);
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

int tb_num_runs(const tb_handle* h) { return h ? int(h->runs.size()) : -1; }

int tb_run_info(const tb_handle* h, int run, int64_t* dof_offset, int64_t* ndofs, int32_t* first_band,
                int32_t* first_channel) {
    if (!h || run < 0 || run >= int(h->runs.size())) { set_error("run index out of range"); return TB_ERR_ARG; }
    const RunInfo& r = h->runs[run];
    if (dof_offset) *dof_offset = r.dof_off;
    if (ndofs) *ndofs = r.ndofs;
    if (first_band) *first_band = r.band0;
    if (first_channel) *first_channel = r.chan0;
    return TB_OK;
}

int tb_num_channels(const tb_handle* h) { return h ? int(h->insts.size()) : -1; }

int tb_channel_info(const tb_handle* h, int ch, int64_t* n_tuples, int64_t* n_prefilter, int64_t* n_det,
                    int32_t* layout) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const GroupChan& G = h->groups[h->insts[ch].group];
    if (G.stream) {
        // the counts of the last evaluation outside an integration (zeros before one)
        unsigned long long cnt[5] = {0, 0, 0, 0, 0};
        TB_CUDA(cudaSetDevice(h->device));
        TB_CUDA(cudaStreamSynchronize(h->stream));
        TB_CUDA(cudaMemcpy(cnt, G.sdev.counts, sizeof(cnt), cudaMemcpyDeviceToHost));
        if (n_tuples) *n_tuples = int64_t(cnt[2]);
        if (n_prefilter) *n_prefilter = int64_t(cnt[0]);
        if (n_det) *n_det = int64_t(cnt[1]);
        if (layout) *layout = G.layout;
        return TB_OK;
    }
    if (n_tuples) *n_tuples = G.tup.n;
    if (n_prefilter) *n_prefilter = G.diag[0];
    if (n_det) *n_det = G.diag[1];
    if (layout) *layout = G.layout;
    return TB_OK;
}

int tb_channel_points_inside(const tb_handle* h, int ch, int64_t* n_tuples, int64_t* n_points) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const GroupChan& G = h->groups[h->insts[ch].group];
    if (G.stream) {
        unsigned long long cnt[5] = {0, 0, 0, 0, 0};
        TB_CUDA(cudaSetDevice(h->device));
        TB_CUDA(cudaStreamSynchronize(h->stream));
        TB_CUDA(cudaMemcpy(cnt, G.sdev.counts, sizeof(cnt), cudaMemcpyDeviceToHost));
        if (n_tuples) *n_tuples = int64_t(cnt[4]);
        if (n_points) *n_points = int64_t(cnt[3]);
        return TB_OK;
    }
    const bool has = G.layout == TB_LAYOUT_MC64 && G.theta.built;
    if (n_tuples) *n_tuples = has ? G.theta.n : -1;
    if (n_points) *n_points = has ? G.theta.points : -1;
    return TB_OK;
}

int tb_channel_schedule(const tb_handle* h, int ch, int32_t* stages, int32_t* pair, double* seconds) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const GroupChan& G = h->groups[h->insts[ch].group];
    if (G.stream) {
        if (stages) *stages = 0;
        if (pair) *pair = 7;
        if (seconds) *seconds = 0.0;
        return TB_OK;
    }
    const bool tensor = G.layout != TB_LAYOUT_MC64;
    if (stages) *stages = tensor ? G.tensor.stages : 0;
    if (pair)
        *pair = !tensor                ? (G.theta.use ? 6 : 0)
                : G.tensor.runs == 32 ? 2
                : G.tensor.runs == 8  ? 3
                : G.tensor.runs == 4  ? 4
                : G.tensor.runs == 16 ? 5
                : (G.L <= 3 && G.insts.size() > 1) ? G.tensor.pair
                                                   : 0;
    if (seconds) *seconds = tensor ? G.tensor.tuned_seconds : 0.0;
    return TB_OK;
}

int tb_set_channel_schedule(tb_handle* h, int ch, int32_t stages, int32_t pair) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    GroupChan& G = h->groups[h->insts[ch].group];
    if (G.stream) {
        if (stages != 0 || pair != 7) { set_error("streamed channels have the one schedule stages 0, pair 7"); return TB_ERR_ARG; }
        return TB_OK;
    }
    if (G.layout == TB_LAYOUT_MC64) {
        if (stages != 0 || (pair != 0 && pair != 6)) {
            set_error("Monte-Carlo channels take stages 0 and pair 0 (every point) or 6 (points inside only)");
            return TB_ERR_ARG;
        }
        if (pair == 6 && !G.theta.built) {
            set_error("this channel has no list of points inside (more than 64 Monte-Carlo points)");
            return TB_ERR_ARG;
        }
        TB_CUDA(cudaSetDevice(h->device));
        TB_CUDA(cudaStreamSynchronize(h->stream));
        G.theta.use = pair == 6;
        if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
        return TB_OK;
    }
    if (stages < 1 || stages > 2 || pair < 0 || pair > 5) { set_error("stages must be 1..2 and pair 0..5"); return TB_ERR_ARG; }
    if (pair >= 2 && !G.tensor.fT) {
        set_error("the run-minor contraction needs a group of 8..1024 runs with at most 3 legs");
        return TB_ERR_ARG;
    }
    TB_CUDA(cudaSetDevice(h->device));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    G.tensor.stages = stages;
    G.tensor.pair = pair == 1 ? 1 : 0;
    G.tensor.runs = pair == 2 ? 32 : pair == 3 ? 8 : pair == 4 ? 4 : pair == 5 ? 16 : 0;
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // the captured launches change
    return TB_OK;
}

int tb_get_tuples(const tb_handle* h, int ch, int32_t* ids, int32_t* umk) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const GroupChan& G = h->groups[h->insts[ch].group];
    if (G.stream) { set_error("a streamed channel keeps no tuple list"); return TB_ERR_ARG; }
    const int64_t n = G.tup.n;
    if (n == 0) return TB_OK;
    std::vector<int32_t> soa(size_t(G.L + 1) * size_t(n));
    cudaSetDevice(h->device);
    for (int r = 0; r <= G.L; ++r)
        TB_CUDA(cudaMemcpy(soa.data() + size_t(r) * n, G.tup.d + size_t(r) * G.tup.cap, sizeof(int32_t) * size_t(n),
                           cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) {
        if (ids)
            for (int l = 0; l < G.L; ++l) ids[i * G.L + l] = soa[size_t(l) * n + i];
        if (umk) umk[i] = soa[size_t(G.L) * n + i];
    }
    return TB_OK;
}

// The reference's tuple cache (ScatteringChannel::precalculateIndices,
// ScatteringChannel.cpp:421-458 reading, 516-534 writing), native byte order:
//   int32 nSecSplits[L][2]  (each leg's mesh, x then y)
//   uint64 number of tuples
//   per tuple: int32 element id of every leg, int32 umklapp column
int tb_write_scatt_indices(const tb_handle* h, int ch, const char* path) {
    if (!h || !path || ch < 0 || ch >= int(h->insts.size())) { set_error("bad argument"); return TB_ERR_ARG; }
    if (h->opts.shard_count > 1) {
        set_error("a sharded handle holds only its part of the tuple list");
        return TB_ERR_ARG;
    }
    const ChanInst& I = h->insts[ch];
    const GroupChan& G = h->groups[I.group];
    if (G.stream) { set_error("a streamed channel keeps no tuple list"); return TB_ERR_ARG; }
    const int L = G.L;
    const int64_t n = G.tup.n;
    std::vector<int32_t> ids(size_t(std::max<int64_t>(n, 1)) * L), umk(size_t(std::max<int64_t>(n, 1)));
    TB_TRY(tb_get_tuples(h, ch, ids.data(), umk.data()));
    FILE* fp = std::fopen(path, "wb");
    if (!fp) { set_error(std::string("cannot open ") + path); return TB_ERR_ARG; }
    bool ok = true;
    for (int l = 0; l < L; ++l) {
        const HostMesh& m = h->meshes[h->bands[I.band[l]].mesh];
        const int32_t ns[2] = {m.nx, m.ny};
        ok = ok && std::fwrite(ns, sizeof(int32_t), 2, fp) == 2;
    }
    const uint64_t total = uint64_t(n);
    ok = ok && std::fwrite(&total, sizeof(uint64_t), 1, fp) == 1;
    std::vector<int32_t> rec(size_t(L + 1));
    for (int64_t i = 0; i < n && ok; ++i) {
        for (int l = 0; l < L; ++l) rec[size_t(l)] = ids[size_t(i) * L + l];
        rec[size_t(L)] = umk[size_t(i)];
        ok = std::fwrite(rec.data(), sizeof(int32_t), size_t(L + 1), fp) == size_t(L + 1);
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) { set_error(std::string("write failed: ") + path); return TB_ERR_ARG; }
    return TB_OK;
}

int tb_read_scatt_indices(const char* path, int nlegs, const int32_t* nsplit, int64_t* n_tuples, int32_t* ids,
                          int32_t* umk, int64_t capacity) {
    if (!path || !n_tuples || nlegs < 2 || nlegs > TB_MAX_LEGS) { set_error("bad argument"); return TB_ERR_ARG; }
    FILE* fp = std::fopen(path, "rb");
    if (!fp) { set_error(std::string("cannot open ") + path); return TB_ERR_ARG; }
    int rc = TB_OK;
    int32_t ns[2 * TB_MAX_LEGS];
    uint64_t total = 0;
    if (std::fread(ns, sizeof(int32_t), size_t(2 * nlegs), fp) != size_t(2 * nlegs) ||
        std::fread(&total, sizeof(uint64_t), 1, fp) != 1) {
        set_error("truncated tuple cache header");
        rc = TB_ERR_BAD_DESC;
    }
    if (rc == TB_OK && nsplit)
        for (int k = 0; k < 2 * nlegs; ++k)
            if (ns[k] != nsplit[k]) { set_error("tuple cache was written for other meshes"); rc = TB_ERR_BAD_DESC; }
    if (rc == TB_OK) {
        *n_tuples = int64_t(total);
        if (ids || umk) {
            if (int64_t(total) > capacity) { set_error("tuple cache larger than the buffers"); rc = TB_ERR_CAPACITY; }
            std::vector<int32_t> rec(size_t(nlegs + 1));
            for (uint64_t i = 0; i < total && rc == TB_OK; ++i) {
                if (std::fread(rec.data(), sizeof(int32_t), size_t(nlegs + 1), fp) != size_t(nlegs + 1)) {
                    set_error("truncated tuple cache");
                    rc = TB_ERR_BAD_DESC;
                    break;
                }
                if (ids)
                    for (int l = 0; l < nlegs; ++l) ids[i * nlegs + l] = rec[size_t(l)];
                if (umk) umk[i] = rec[size_t(nlegs)];
            }
        }
    }
    std::fclose(fp);
    return rc;
}

// Mesh<2>::elemCentre (Mesh.cpp:533-535): the point (0.333333333,
// 0.333333333) of the reference element mapped as Mesh<2>::operator()(elem,
// refCoord) does (Mesh.cpp:503-509): origin + dG (section + E refCoord), E the
// element's vertices 1 and 2 in its reference section.
static void elem_centre(const HostMesh& m, int e, double out[2]) {
    const double r = 0.333333333;
    const int s = e / 2, par = e % 2;
    const double sx = double(s % m.nx), sy = double(s / m.nx);
    const double px = sx + (kVert[par][1][0] * r + kVert[par][2][0] * r);
    const double py = sy + (kVert[par][1][1] * r + kVert[par][2][1] * r);
    out[0] = m.origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
    out[1] = m.origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
}

int tb_set_channel_amplitude_fn(tb_handle* h, int ch, tb_amplitude_fn fn, void* user) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(stream_wait(h));
    const ChanInst& I = h->insts[ch];
    GroupChan& G = h->groups[I.group];
    if (G.stream && fn) { set_error("a streamed channel takes no functAmplitude (no per-tuple table)"); return TB_ERR_ARG; }
    const int L = G.L;
    const int64_t n = G.tup.n;
    if (G.d_tamp) { cudaFree(G.d_tamp); G.d_tamp = nullptr; }
    G.dev.tamp = nullptr;
    if (fn && n > 0) {
        if (cudaMalloc(&G.d_tamp, sizeof(double) * size_t(n)) != cudaSuccess) {
            G.d_tamp = nullptr;
            set_error("amplitude table allocation failed");
            return TB_ERR_OOM;
        }
        const HostMesh* lm[TB_MAX_LEGS];
        for (int l = 0; l < L; ++l) lm[l] = &h->meshes[h->bands[I.band[l]].mesh];
        const int64_t chunk = int64_t(1) << 20;
        std::vector<int32_t> ids(size_t(L + 1) * size_t(std::min(n, chunk)));
        std::vector<double> bary(size_t(std::min(n, chunk)) * L * 2), fac(size_t(std::min(n, chunk)));
        for (int64_t a = 0; a < n; a += chunk) {
            const int64_t m = std::min(chunk, n - a);
            for (int l = 0; l < L; ++l)
                TB_CUDA(cudaMemcpy(ids.data() + size_t(l) * m, G.tup.d + size_t(l) * G.tup.cap + a,
                                   sizeof(int32_t) * size_t(m), cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < m; ++i)
                for (int l = 0; l < L; ++l) elem_centre(*lm[l], ids[size_t(l) * m + i], &bary[(size_t(i) * L + l) * 2]);
            if (fn(user, m, L, bary.data(), fac.data()) != 0) {
                cudaFree(G.d_tamp);
                G.d_tamp = nullptr;
                set_error("amplitude callback failed");
                return TB_ERR_ARG;
            }
            TB_CUDA(cudaMemcpy(G.d_tamp + a, fac.data(), sizeof(double) * size_t(m), cudaMemcpyHostToDevice));
        }
        G.dev.tamp = G.d_tamp;
    }
    if (G.layout != TB_LAYOUT_MC64 && G.tensor.d)
        TB_TRY(refill_tensor(G.dev, G.tup.d, G.tup.cap, G.tup.n, G.tensor, h->stream));
    TB_TRY(stream_wait(h));
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // kernels take the channel by value
    return TB_OK;
}

int tb_set_amplitude(tb_handle* h, int ch, double amplitude) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    ChanInst& I = h->insts[ch];
    GroupChan& G = h->groups[I.group];
    I.amplitude = amplitude;
    I.dev.amplitude = amplitude;
    I.dev.amp_full = amp_full_of(h, I, G.L, amplitude);
    // the kernels read instances from device memory, so a captured graph
    // sees the new value at its next launch
    TB_TRY(stream_wait(h));
    TB_CUDA(cudaMemcpy(G.d_insts + I.slot, &I.dev, sizeof(InstDev), cudaMemcpyHostToDevice));
    TB_CUDA(cudaMemcpy(I.d_single, &I.dev, sizeof(InstDev), cudaMemcpyHostToDevice));
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }  // channel skip set changes
    return TB_OK;
}

// TB_ERR_TIMEOUT when a contraction's bounded wait ran out since the last
// check (the kernels that gave up left their part of the sum out).
static int check_wait_timeout(tb_handle* h) {
    int tflag = 0;
    TB_TRY(take_wait_timeout(h->d_err, h->stream, &tflag));
    if (tflag) {
        set_error("a moment-tensor contraction gave up waiting for its staged tiles; the result is incomplete");
        return TB_ERR_TIMEOUT;
    }
    bool clamped = false;
    TB_TRY(tb::fx_take_saturation(h, clamped));
    if (clamped) return tb::fx_saturation_error();
    return TB_OK;
}

static int rhs_common(tb_handle* h, const double* f, double* out, int flags, int only_inst) {
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
    TB_TRY(run_rhs_acc(h, d_in, h->d_acc, nullptr, flags, only_inst));
    TB_TRY(launch_inverse_mass(h->ed, h->d_acc, d_res, h->stream));
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(out, h->d_out, bytes, cudaMemcpyDeviceToHost, h->stream));
        TB_TRY(stream_wait(h));
        TB_TRY(check_wait_timeout(h));
    }
    return TB_OK;
}

int tb_rhs(tb_handle* h, const double* f, double* dfdt, int flags) {
    NvtxRange range("tb_rhs");
    return rhs_common(h, f, dfdt, flags, -1);
}

int tb_scattering_rates(tb_handle* h, int ch, int leg, const double* f, double* rates, int flags) {
    NvtxRange range("tb_scattering_rates");
    if (!h || !f || !rates) { set_error("null argument"); return TB_ERR_ARG; }
    if (ch < -1 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    if (leg < -1 || leg >= TB_MAX_LEGS || (ch >= 0 && leg >= h->groups[h->insts[ch].group].L)) {
        set_error("leg index out of range");
        return TB_ERR_ARG;
    }
    TB_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const double* d_in = f;
    double* d_res = rates;
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(h->d_f, f, bytes, cudaMemcpyHostToDevice, h->stream));
        d_in = h->d_f;
        d_res = h->d_out;
    }
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    for (size_t gi = 0; gi < h->groups.size(); ++gi) {
        GroupChan& G = h->groups[gi];
        if (G.tup.n == 0 && !G.stream) continue;
        const InstDev* insts = G.d_insts;
        int n_insts = int(G.insts.size());
        if (ch >= 0) {
            if (h->insts[ch].group != int(gi)) continue;
            insts = h->insts[ch].d_single;
            n_insts = 1;
        }
        for (int l = 0; l < G.L; ++l) {
            if (leg >= 0 && l != leg) continue;
            if (G.stream)
                TB_TRY(launch_group_stream(h, G, insts, n_insts, d_in, h->d_acc, nullptr, l));
            else if (G.layout == TB_LAYOUT_MC64)
                TB_TRY(launch_group_mc(h, G, insts, n_insts, d_in, h->d_acc, nullptr, l));
            else
                TB_TRY(launch_collision_tensor(G.dev, insts, n_insts, G.tensor, G.tup.d, G.tup.cap, G.tup.n, d_in,
                                               h->d_acc, nullptr, h->stream, l, h->fx));
        }
    }
    TB_TRY(launch_fx_flush(h->fx, h->d_acc, h->ndofs, h->stream));
    TB_TRY(shard_allreduce(h, h->d_acc, size_t(h->ndofs)));
    TB_TRY(launch_inverse_mass(h->ed, h->d_acc, d_res, h->stream));
    TB_CUDA(cudaMemsetAsync(h->d_acc, 0, bytes, h->stream));
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(rates, h->d_out, bytes, cudaMemcpyDeviceToHost, h->stream));
        TB_TRY(stream_wait(h));
        TB_TRY(check_wait_timeout(h));
    }
    return TB_OK;
}

int tb_channel_propagate(tb_handle* h, int ch, const double* f, double* out, int flags) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
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
    TB_TRY(launch_error_norm(h->ed, de, dp, h->d_part, h->stream));
    const int nblk = h->ed.nblk;
    std::vector<double> part(size_t(2 * nblk));
    TB_CUDA(cudaMemcpyAsync(part.data(), h->d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->stream));
    TB_TRY(stream_wait(h));
    std::vector<int> first(h->bands.size() + 1, 0);
    for (size_t b = 0; b < h->bands.size(); ++b) first[b + 1] = first[b] + (h->bands[b].ne + 255) / 256;
    for (size_t r = 0; r < h->runs.size(); ++r) {
        double errNorm = 0.0;
        for (int b = h->runs[r].band0; b < h->runs[r].band0 + h->runs[r].nbands; ++b) {
            const BandDev& bd = h->banddev[b];
            double sr = 0.0, sp = 0.0;
            for (int k = first[b]; k < first[b + 1]; ++k) { sr += part[size_t(k)]; sp += part[size_t(nblk + k)]; }
            const double be =
                std::sqrt((bd.mesh.vol * sr + bd.penal * (bd.mesh.vol * sp)) / (double(bd.ne) * bd.mesh.vol));
            if (be >= errNorm) errNorm = be;
        }
        result[r] = errNorm;
    }
    return TB_OK;
}

int tb_apply_constraints(tb_handle* h, double* f, int flags) {
    if (!h || !f) { set_error("null argument"); return TB_ERR_ARG; }
    if (h->cfn) { set_error("the constraints depend on time: use tb_apply_constraints_at"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    if (flags & TB_PTR_HOST) {
        TB_CUDA(cudaMemcpyAsync(h->d_f, f, bytes, cudaMemcpyHostToDevice, h->stream));
        TB_TRY(launch_enforce(h->ed, h->d_f, h->d_f, h->stream));
        TB_CUDA(cudaMemcpyAsync(f, h->d_f, bytes, cudaMemcpyDeviceToHost, h->stream));
        TB_TRY(stream_wait(h));
    } else {
        TB_TRY(launch_enforce(h->ed, f, f, h->stream));
    }
    return TB_OK;
}

}  // extern "C"

namespace tb {

// Start a (batched) integration.  `hooks` carries the adjoint recording
// buffers (step log, checkpoints) or is null for a plain integration; the
// captured attempt graph holds the DPBufs by value, so a change of hooks
// re-captures it.
int dp_begin(tb_handle* h, const double* f0, const double* t0, const double* t_final, const double* dense_step,
             int64_t max_dense, int flags, const DPBufs* hooks) {
    if (!h || !f0 || !t0 || !t_final || !dense_step) { set_error("null argument"); return TB_ERR_ARG; }
    const int nruns = int(h->runs.size());
    for (int r = 0; r < nruns; ++r)
        if (!(dense_step[r] > 0.0)) { set_error("dense_step must be > 0"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(dp_alloc(h, max_dense));
    const int rflags = flags & (TB_NO_DRIFT | TB_NO_COLLISIONS);
    h->dp_flags = flags;
    h->wait_timed_out = false;
    // clamped contributions of trial stages are rejected by the step's own
    // error norm; the integration does not report them
    if (h->fx.sat) TB_CUDA(cudaMemsetAsync(h->fx.sat, 0, sizeof(unsigned int), h->stream));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    DPBufs& B = h->dp;
    {
        const DPBufs none{};
        const DPBufs& hk = hooks ? *hooks : none;
        if (B.step_log != hk.step_log || B.log_cap != hk.log_cap || B.ckpt != hk.ckpt ||
            B.ckpt_every != hk.ckpt_every || B.ckpt_cap != hk.ckpt_cap) {
            B.step_log = hk.step_log;
            B.log_cap = hk.log_cap;
            B.ckpt = hk.ckpt;
            B.ckpt_every = hk.ckpt_every;
            B.ckpt_cap = hk.ckpt_cap;
            if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
        }
    }
    TB_CUDA(cudaMemcpyAsync(B.y, f0, bytes, (flags & TB_PTR_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            h->stream));
    TB_TRY(stream_wait(h));   // the pinned mirror is rewritten below
    for (int r = 0; r < nruns; ++r) {
        DPCtl& c = h->h_ctl[r];
        std::memset(&c, 0, sizeof(c));
        c.t = t0[r];
        c.tf = t_final[r];
        c.dense_step = dense_step[r];
        c.dense_time = t0[r] + dense_step[r];
        c.min_step = dense_step[r] / 10000.;
        c.olderror = 1.0;
        c.dt = dense_step[r];
        // timeStepVetoer: with no time-dependent constraints it returns
        // (t + dt) - t; with them tc_begin applies it below
        if (!h->cfn) c.dt = std::min(c.dt, (c.t + c.dt) - c.t);
        c.dense_cap = max_dense;
        c.rhs_evals = 1;
        c.done = (t0[r] < t_final[r]) ? 0 : 1;
        c.last_dense_step = -1;
    }
    if (h->cfn) TB_TRY(tc_begin(h));   // values at t0 into slot 0, first dt vetoed
    TB_CUDA(cudaMemcpyAsync(B.ctl, h->h_ctl, sizeof(DPCtl) * nruns, cudaMemcpyHostToDevice, h->stream));
    // k1 = timeOp(t0, enforceValue(t0, y0))
    TB_TRY(launch_enforce(h->ed, B.y, B.tmp, h->stream, h->cfn ? h->d_ctv : nullptr));
    TB_CUDA(cudaMemsetAsync(B.acc, 0, bytes, h->stream));
    TB_TRY(run_rhs_acc(h, B.tmp, B.acc, nullptr, rflags, -1));
    TB_TRY(launch_k1(h->ed, B, h->stream));
    if (B.ckpt) TB_CUDA(cudaMemcpyAsync(B.ckpt, B.tmp, bytes, cudaMemcpyDeviceToDevice, h->stream));
    TB_TRY(ensure_graph(h, rflags));
    return TB_OK;
}

}  // namespace tb

extern "C" {

int tb_dp45_begin_batch(tb_handle* h, const double* f0, const double* t0, const double* t_final,
                        const double* dense_step, int64_t max_dense, int flags) {
    return dp_begin(h, f0, t0, t_final, dense_step, max_dense, flags, nullptr);
}

int tb_dp45_begin(tb_handle* h, const double* f0, double t0, double t_final, double dense_step, int64_t max_dense,
                  int flags) {
    if (!h) { set_error("null handle"); return TB_ERR_ARG; }
    const size_t nr = h->runs.size();
    std::vector<double> a(nr, t0), b(nr, t_final), c(nr, dense_step);
    return tb_dp45_begin_batch(h, f0, a.data(), b.data(), c.data(), max_dense, flags);
}

int tb_dp45_advance(tb_handle* h, int64_t n_attempts) {
    if (!h || !h->graph) { set_error("tb_dp45_begin was not called"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    for (int64_t i = 0; i < n_attempts; ++i) TB_CUDA(cudaGraphLaunch(h->graph, h->stream));
    return TB_OK;
}

static int poll_all(tb_handle* h) {
    if (!h || !h->dp_ready) { set_error("tb_dp45_begin was not called"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_CUDA(cudaMemcpyAsync(h->h_ctl, h->dp.ctl, sizeof(DPCtl) * h->runs.size(), cudaMemcpyDeviceToHost, h->stream));
    TB_TRY(stream_wait(h));
    int tflag = 0;
    TB_TRY(take_wait_timeout(h->d_err, h->stream, &tflag));
    if (tflag) h->wait_timed_out = true;   // sticky for this integration: its state is unreliable
    if (h->wait_timed_out)
        for (size_t r = 0; r < h->runs.size(); ++r) { h->h_ctl[r].status = TB_ERR_TIMEOUT; h->h_ctl[r].done = 1; }
    return TB_OK;
}

int tb_dp45_poll(tb_handle* h, tb_dp45_stats* st) {
    TB_TRY(poll_all(h));
    fill_stats(h->h_ctl[0], st);
    if (st) {
        int all_done = 1;
        for (size_t r = 0; r < h->runs.size(); ++r) all_done &= h->h_ctl[r].done ? 1 : 0;
        st->done = all_done;
    }
    return TB_OK;
}

int tb_dp45_run_stats(tb_handle* h, int run, tb_dp45_stats* st) {
    if (!h || !h->dp_ready || run < 0 || run >= int(h->runs.size())) { set_error("bad run index"); return TB_ERR_ARG; }
    fill_stats(h->h_ctl[run], st);
    return TB_OK;
}

int tb_dp45_end(tb_handle* h, double* f_out, double* dense_out, double* dense_times, int64_t max_dense,
                tb_dp45_stats* st, int flags) {
    tb_dp45_stats s;
    TB_TRY(tb_dp45_poll(h, &s));
    const size_t bytes = sizeof(double) * size_t(h->ndofs);
    const cudaMemcpyKind kind = (flags & TB_PTR_HOST) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (f_out) TB_CUDA(cudaMemcpyAsync(f_out, h->dp.y, bytes, kind, h->stream));
    // dense outputs: run r's block holds max_dense slots of its own ndofs
    int64_t uoff = 0, utoff = 0;
    for (size_t r = 0; r < h->runs.size(); ++r) {
        const RunDev& rd = h->hruns[r];
        const int64_t nd = std::min<int64_t>(std::min<int64_t>(h->h_ctl[r].n_dense, max_dense), h->dense_cap_alloc);
        if (nd > 0 && dense_out)
            TB_CUDA(cudaMemcpyAsync(dense_out + uoff, h->dp.dense + rd.dense_off, sizeof(double) * size_t(nd * rd.ndofs),
                                    kind, h->stream));
        if (nd > 0 && dense_times)
            TB_CUDA(cudaMemcpyAsync(dense_times + utoff, h->dp.dense_t + rd.dense_t_off, sizeof(double) * size_t(nd),
                                    kind, h->stream));
        uoff += max_dense * rd.ndofs;
        utoff += max_dense;
    }
    TB_TRY(stream_wait(h));
    if (h->fx.sat) TB_CUDA(cudaMemsetAsync(h->fx.sat, 0, sizeof(unsigned int), h->stream));
    if (st) *st = s;
    int worst = TB_OK;
    for (size_t r = 0; r < h->runs.size(); ++r)
        if (h->h_ctl[r].status != TB_OK) { worst = h->h_ctl[r].status; break; }
    return worst;
}

int tb_dp45_integrate(tb_handle* h, double* f_inout, double t0, double t_final, double dense_step, double* dense_out,
                      double* dense_times, int64_t max_dense, tb_dp45_stats* st, int flags) {
    NvtxRange range("tb_dp45_integrate");
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
    TB_TRY(stream_wait(h));
    TB_TRY(check_wait_timeout(h));
    return TB_OK;
}

int tb_set_copy_wait_limit(tb_handle* h, int64_t polls) {
    if (!h) { set_error("null handle"); return TB_ERR_ARG; }
    if (polls < 0 || polls > 0x7fffffff) { set_error("polls must lie in [0, 2^31 - 1]"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_TRY(stream_wait(h));
    for (auto& G : h->groups) G.dev.wait_polls = int(polls);
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // launches keep their arguments
    return TB_OK;
}

void* tb_get_stream(tb_handle* h) { return h ? (void*)h->stream : nullptr; }

int tb_collision_accumulate(tb_handle* h, int ch, const double* f, double* acc) {
    if (!h || !f || !acc) { set_error("null argument"); return TB_ERR_ARG; }
    if (ch < -1 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    TB_CUDA(cudaSetDevice(h->device));
    return run_rhs_acc(h, f, acc, nullptr, TB_NO_DRIFT, ch);
}

}  // extern "C"
