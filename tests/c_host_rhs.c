/*
 * c_host_rhs.c -- a plain C host of the library, as a TORTOISE shim calls it:
 * it builds tb_problem_desc from raw arrays, creates the handle, evaluates
 * the right-hand side and runs a Dormand-Prince integration, all through
 * include/tortoise_b200.h with host pointers.  Used by tests/test_gpu_c_host.py.
 *
 *   c_host_rhs <input> <output>
 *
 * input (native byte order, written by the test):
 *   double origin[2], gvec[4]; double rel_origin[2], rel_size[2]; int32 nsplit[2]
 *   int32 nbands; per band: double charge, statistics, abs_tol, rel_tol, vel[2];
 *                           int32 ne; double dispersion[3 ne]
 *   int32 nchannels; per channel: int32 L, band[L], dir[L]; double amplitude;
 *                           int32 n_mc; double min_det, threshold; int32 n_umk;
 *                           double umk[2 n_umk], mc[n_mc R], mc_pre[n_mc R]  (R = 2L - 3)
 *   int64 ndofs; double f[ndofs]; double t_final, dense_step; int64 max_dense
 * output: double rhs[ndofs]; int64 stats[4] (attempts, accepted, rejected,
 *         n_dense); double dense[max_dense][ndofs]; double y[ndofs]
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tortoise_b200.h"

static FILE* in;

static void rd(void* p, size_t sz, size_t n) {
    if (fread(p, sz, n, in) != n) {
        fprintf(stderr, "short input\n");
        exit(2);
    }
}

static double* rd_doubles(size_t n) {
    double* p = (double*)malloc(sizeof(double) * (n ? n : 1));
    rd(p, sizeof(double), n);
    return p;
}

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    in = fopen(argv[1], "rb");
    if (!in) return 2;
    tb_problem_desc d;
    memset(&d, 0, sizeof(d));
    rd(d.region.origin, sizeof(double), 2);
    rd(d.region.gvec, sizeof(double), 4);
    tb_mesh_desc mesh;
    rd(mesh.rel_origin, sizeof(double), 2);
    rd(mesh.rel_size, sizeof(double), 2);
    rd(mesh.nsplit, sizeof(int32_t), 2);
    d.n_meshes = 1;
    d.meshes = &mesh;
    rd(&d.n_bands, sizeof(int32_t), 1);
    tb_band_desc* bands = (tb_band_desc*)calloc((size_t)d.n_bands, sizeof(tb_band_desc));
    for (int b = 0; b < d.n_bands; ++b) {
        rd(&bands[b].charge, sizeof(double), 1);
        rd(&bands[b].statistics, sizeof(double), 1);
        rd(&bands[b].abs_tol, sizeof(double), 1);
        rd(&bands[b].rel_tol, sizeof(double), 1);
        rd(bands[b].drift_velocity, sizeof(double), 2);
        int32_t ne;
        rd(&ne, sizeof(int32_t), 1);
        bands[b].dispersion = rd_doubles((size_t)ne * 3);
        bands[b].mesh = 0;
    }
    d.bands = bands;
    rd(&d.n_channels, sizeof(int32_t), 1);
    tb_channel_desc* chans = (tb_channel_desc*)calloc((size_t)d.n_channels, sizeof(tb_channel_desc));
    for (int c = 0; c < d.n_channels; ++c) {
        tb_channel_desc* ch = &chans[c];
        rd(&ch->nlegs, sizeof(int32_t), 1);
        rd(ch->band, sizeof(int32_t), (size_t)ch->nlegs);
        rd(ch->dir, sizeof(int32_t), (size_t)ch->nlegs);
        rd(&ch->amplitude, sizeof(double), 1);
        rd(&ch->n_mc, sizeof(int32_t), 1);
        rd(&ch->min_det, sizeof(double), 1);
        rd(&ch->threshold, sizeof(double), 1);
        rd(&ch->n_umklapp, sizeof(int32_t), 1);
        const size_t R = (size_t)(2 * ch->nlegs - 3);
        ch->umklapp = rd_doubles((size_t)ch->n_umklapp * 2);
        ch->mc_points = rd_doubles((size_t)ch->n_mc * R);
        ch->mc_points_precalc = rd_doubles((size_t)ch->n_mc * R);
        ch->n_tuples = 0;   /* enumerate on the device */
    }
    d.channels = chans;
    int64_t ndofs;
    rd(&ndofs, sizeof(int64_t), 1);
    double* f = rd_doubles((size_t)ndofs);
    double t_final, dense_step;
    int64_t max_dense;
    rd(&t_final, sizeof(double), 1);
    rd(&dense_step, sizeof(double), 1);
    rd(&max_dense, sizeof(int64_t), 1);
    fclose(in);

    tb_options opts;
    memset(&opts, 0, sizeof(opts));
    opts.layout = TB_LAYOUT_AUTO;
    tb_handle* h = NULL;
    int rc = tb_create(&h, &d, &opts);
    if (rc != TB_OK) {
        fprintf(stderr, "tb_create: %d %s\n", rc, tb_last_error());
        return 1;
    }
    if (tb_num_dofs(h) != ndofs) {
        fprintf(stderr, "dof count %lld != %lld\n", (long long)tb_num_dofs(h), (long long)ndofs);
        return 1;
    }
    double* rhs = (double*)malloc(sizeof(double) * (size_t)ndofs);
    rc = tb_rhs(h, f, rhs, TB_PTR_HOST);
    if (rc != TB_OK) {
        fprintf(stderr, "tb_rhs: %d %s\n", rc, tb_last_error());
        return 1;
    }
    double* dense = (double*)calloc((size_t)(max_dense * ndofs), sizeof(double));
    double* times = (double*)calloc((size_t)max_dense, sizeof(double));
    tb_dp45_stats st;
    rc = tb_dp45_integrate(h, f, 0.0, t_final, dense_step, dense, times, max_dense, &st, TB_PTR_HOST);
    if (rc != TB_OK) {
        fprintf(stderr, "tb_dp45_integrate: %d %s\n", rc, tb_last_error());
        return 1;
    }
    FILE* out = fopen(argv[2], "wb");
    if (!out) return 2;
    fwrite(rhs, sizeof(double), (size_t)ndofs, out);
    const int64_t stats[4] = {st.attempts, st.accepted, st.rejected, st.n_dense};
    fwrite(stats, sizeof(int64_t), 4, out);
    fwrite(dense, sizeof(double), (size_t)(max_dense * ndofs), out);
    fwrite(f, sizeof(double), (size_t)ndofs, out);
    fclose(out);
    tb_destroy(h);
    return 0;
}
