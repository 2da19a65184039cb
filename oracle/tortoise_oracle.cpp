// tortoise_oracle.cpp -- CPU oracle for the TORTOISE collision operator and
// Dormand-Prince 5(4) time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is a plain C++17 restatement (no Eigen,
// no TBB) of the reference's FP64 CPU path.  It is linked by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker;
// the product (tortoise_b200/) never links, imports or calls it.
//
// Parity status: the reference as a whole cannot be compiled here (Eigen 3.4
// and oneTBB are absent) and ships no tests or golden vectors.  Its
// Dormand-Prince integrator needs neither: oracle/ref_dp54_harness.cpp builds
// it from the reference tree, and tests/test_oracle_ref_dp54.py requires the
// restated integrator below (dp54_core) to take the same steps and give
// bit-identical dense outputs on the same operators.  The collision operator,
// error norm and drift are pinned only by the physical identities the
// reference's algorithm obeys (tests/test_oracle.py: particle-number
// conservation per tuple, detailed balance at equilibrium, mass-matrix
// identities): "parity unpinned" against the reference binary for those.
//
// Every function cites the reference file:line it follows (paths relative to
// the TORTOISE project root).

#include "../include/tortoise_b200.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace oracle {

// ------------------------------------------------------------------ constants
// GaussQuadratureConst.hpp:84-90 -- order-2 triangle rule, 14-digit constants
// exactly as written in the reference.
static const double kGP2[3][2] = {{0.16666666666667, 0.16666666666667},
                                  {0.66666666666667, 0.16666666666667},
                                  {0.16666666666667, 0.66666666666667}};
static const double kGW2[3] = {0.33333333333333, 0.33333333333333, 0.33333333333333};
// GaussQuadratureConst.hpp:60-61 -- order-2 rule on [0,1].
static const double kGP1[2] = {0.2113248654051871, 0.7886751345948129};
static const double kGW1[2] = {0.5, 0.5};
// Mesh.cpp:48-84 (addNextElementVertex): section-relative vertices of the two
// reference elements; columns are vertices.
static const double kVert[2][3][2] = {{{0, 0}, {1, 0}, {1, 1}},
                                      {{0, 0}, {0, 1}, {1, 1}}};

// --------------------------------------------------------------------- mesh
struct Mesh {
    int nx = 0, ny = 0, ne = 0;
    double origin[2];     // absolute origin (Mesh.cpp:321)
    double gv[2][2];      // mesh gVec = region.gVec * diag(relSize)  [row][col]
    double dG[2][2];      // section sides, column j = gv column j / nsplit(j) (Mesh.cpp:335)
    double invdG[2][2];
    double vol;           // |det dG| / 2 (Mesh.cpp:337)
    double rel_origin[2]; // kept for calculate_verticesCoord (Mesh.cpp:222-241)
    double M[3][3], Minv[3][3];
};

static double det2(const double a[2][2]) { return a[0][0] * a[1][1] - a[0][1] * a[1][0]; }

static void inv2(const double a[2][2], double r[2][2]) {
    // cofactor inverse scaled by the reciprocal determinant
    const double invdet = 1.0 / det2(a);
    r[0][0] = a[1][1] * invdet;  r[1][0] = -a[1][0] * invdet;
    r[0][1] = -a[0][1] * invdet; r[1][1] = a[0][0] * invdet;
}

static double det3(const double a[3][3]) {
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1])
         - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
         + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}

// Cofactor inverse: det from the column-0 cofactor expansion, every
// cofactor scaled by its reciprocal.
static inline double cof3(const double a[3][3], int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return a[i1][j1] * a[i2][j2] - a[i1][j2] * a[i2][j1];
}

static void inv3(const double a[3][3], double r[3][3]) {
    const double c00 = cof3(a, 0, 0), c10 = cof3(a, 1, 0), c20 = cof3(a, 2, 0);
    const double det = (c00 * a[0][0] + c10 * a[1][0]) + c20 * a[2][0];
    const double invdet = 1.0 / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[j][i] = cof3(a, i, j) * invdet;
    r[0][0] = c00 * invdet; r[0][1] = c10 * invdet; r[0][2] = c20 * invdet;
}

// Mesh<2> constructor, Mesh.cpp:319-347; mass matrices Mesh.cpp:95-123.
static Mesh make_mesh(const tb_region& rg, const tb_mesh_desc& md) {
    Mesh m;
    m.nx = md.nsplit[0];
    m.ny = md.nsplit[1];
    if (m.nx <= 0 || m.ny <= 0) throw std::runtime_error("mesh nsplit must be > 0");
    m.ne = 2 * m.nx * m.ny;
    double G[2][2] = {{rg.gvec[0], rg.gvec[2]}, {rg.gvec[1], rg.gvec[3]}};
    for (int i = 0; i < 2; ++i)
        m.origin[i] = rg.origin[i] + (G[i][0] * md.rel_origin[0] + G[i][1] * md.rel_origin[1]);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) m.gv[i][j] = G[i][j] * md.rel_size[j];
    const double ns[2] = {double(m.nx), double(m.ny)};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) m.dG[i][j] = m.gv[i][j] * (1.0 / ns[j]);
    inv2(m.dG, m.invdG);
    m.vol = std::fabs(det2(m.dG) / 2.0);
    m.rel_origin[0] = md.rel_origin[0];
    m.rel_origin[1] = md.rel_origin[1];
    // basis functions of the linear-form representation: 1, r0, r1
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int q = 0; q < 3; ++q) {
                double bi = (i == 0) ? 1.0 : kGP2[q][i - 1];
                double bj = (j == 0) ? 1.0 : kGP2[q][j - 1];
                s += bi * bj * kGW2[q];
            }
            m.M[i][j] = m.vol * s;
        }
    inv3(m.M, m.Minv);
    return m;
}

// Mesh<2>::operator()(elementID, vertex), Mesh.cpp:488-494.
static void vertex(const Mesh& m, int e, int v, double out[2]) {
    int s = e / 2, par = e % 2;
    double sx = double(s % m.nx), sy = double(s / m.nx);
    double px = sx + kVert[par][v][0], py = sy + kVert[par][v][1];
    out[0] = m.origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
    out[1] = m.origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
}

// ----------------------------------------------------------------- Function
// Function(mesh, lambda): nodal samples then linear form (Function.cpp:60-68).
template <class F>
static std::vector<double> function_from(const Mesh& m, F f) {
    std::vector<double> v(size_t(m.ne) * 3);
    for (int e = 0; e < m.ne; ++e) {
        double n[3];
        for (int k = 0; k < 3; ++k) {
            double p[2];
            vertex(m, e, k, p);
            n[k] = f(p);
        }
        v[3 * e] = n[0];
        v[3 * e + 1] = n[1] - n[0];
        v[3 * e + 2] = n[2] - n[0];
    }
    return v;
}

// Function::applyInverseMass, Function.cpp:801-804 (row-vector times invMass).
static void apply_inverse_mass(const Mesh& m, double* v) {
    for (int e = 0; e < m.ne; ++e) {
        double a = v[3 * e], b = v[3 * e + 1], c = v[3 * e + 2];
        for (int j = 0; j < 3; ++j) v[3 * e + j] = a * m.Minv[0][j] + b * m.Minv[1][j] + c * m.Minv[2][j];
    }
}

// apply(linearForm, point), LinearForm.hpp:63-65.
static inline double lf_apply(const double* c, double x, double y) { return (c[1] * x + c[2] * y) + c[0]; }

// Function::integrate(rhs), Function.cpp:373-375 (Gauss order 2).
static double integrate2(const Mesh& m, const double* a, const double* b) {
    double s = 0.0;
    for (int e = 0; e < m.ne; ++e)
        for (int q = 0; q < 3; ++q)
            s += lf_apply(a + 3 * e, kGP2[q][0], kGP2[q][1]) * lf_apply(b + 3 * e, kGP2[q][0], kGP2[q][1]) * kGW2[q];
    return m.vol * s;
}

// toNodalFromLinForm / toLinFormFromNodal, Function.hpp:330-341.
static inline void to_nodal(const double* c, double n[3]) { n[0] = c[0]; n[1] = c[1] + c[0]; n[2] = c[2] + c[0]; }
static inline void to_lin(const double n[3], double* c) { c[0] = n[0]; c[1] = n[1] - n[0]; c[2] = n[2] - n[0]; }

// --------------------------------------------------------------------- band
struct Band {
    int mesh;
    double charge, statistics;
    std::vector<double> disp, kx, ky, minE, maxE;
    double abs_tol, rel_tol, penal;
    bool constrained;
    std::vector<double> cpop;
    double vel[2];
};

// -------------------------------------------------------------------- channel
struct Channel {
    int L;
    int band[4], dir[4];
    double amplitude;
    int nmc;
    double min_det, threshold;
    std::vector<double> umk;          // [n_umk*2]
    std::vector<double> mc, mc_pre;   // [nmc*R]
    std::vector<int32_t> tuples;      // [n*L]
    std::vector<int32_t> tumk;        // [n]
    std::vector<double> tamp;         // functAmplitude per tuple (empty: 1)
    int64_t n_prefilter = 0, n_det = 0;
};

// Time-dependent constrained populations (Band::constrainedPopulation, a
// std::function<Function(Real)> in the reference, Band.hpp:70-74): a callback
// filling band `band`'s Ne*3 linear-form coefficients at time t; 0 = success.
typedef int (*or_constraint_fn)(void* user, int32_t band, double t, double* population);

struct Problem {
    tb_region region;
    std::vector<Mesh> meshes;
    std::vector<Band> bands;
    std::vector<Channel> chans;
    std::vector<int64_t> off;  // band offsets into the status vector
    int64_t ndofs = 0;
    or_constraint_fn cfn = nullptr;   // null: the time-independent cpop of each band
    void* cuser = nullptr;
};

// -------------------------------------------------- delta-constrained geometry
// constructD / constructN, ScatteringChannel.cpp:302-352 (array overloads);
// integrationInversionDeterminant, IntegratorCore.hpp:153-155.
struct Geom {
    double D[3][8];
    double N[3];
    double DC[3][3];
    double det;
};

static void build_geom(const Problem& P, const Channel& c, const int32_t* e, int umk, Geom& g) {
    const int L = c.L;
    for (int l = 0; l < L; ++l) {
        const Band& b = P.bands[c.band[l]];
        const double d = double(c.dir[l]);
        for (int j = 0; j < 2; ++j) {
            g.D[0][2 * l + j] = d * b.kx[3 * size_t(e[l]) + 1 + j];
            g.D[1][2 * l + j] = d * b.ky[3 * size_t(e[l]) + 1 + j];
            g.D[2][2 * l + j] = d * b.disp[3 * size_t(e[l]) + 1 + j];
        }
    }
    g.N[0] = g.N[1] = g.N[2] = 0.0;
    for (int l = 0; l < L; ++l) {
        const Band& b = P.bands[c.band[l]];
        const double d = double(c.dir[l]);
        g.N[0] -= d * b.kx[3 * size_t(e[l])];
        g.N[1] -= d * b.ky[3 * size_t(e[l])];
        g.N[2] -= d * b.disp[3 * size_t(e[l])];
    }
    const double* u = &c.umk[2 * size_t(umk)];
    const double* G = P.region.gvec;  // column-major
    for (int dim = 0; dim < 2; ++dim)
        for (int du = 0; du < 2; ++du) g.N[dim] -= u[du] * G[2 * du + dim];
    const int c0 = 2 * L - 3;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) g.DC[i][j] = g.D[i][c0 + j];
    g.det = det3(g.DC);
}

// Per-MC-point constrained coordinates and simplex tests,
// IntegratorCore.hpp:276-320.  q = one row of the MC table.
struct MCPoint {
    double p[4][2];  // leg points in reference coordinates
    bool theta;
};

static inline void mc_point(int L, const Geom& g, const double DCinv[3][3], const double* q, MCPoint& mp) {
    const int R = 2 * (L - 2) + 1;
    const double kp0 = q[R - 1];
    double r[3];
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        if (L >= 3) s += g.D[i][0] * q[0] + g.D[i][1] * q[1];
        if (L >= 4) s += g.D[i][2] * q[2] + g.D[i][3] * q[3];
        s += g.D[i][2 * (L - 2)] * kp0;
        r[i] = s - g.N[i];
    }
    double alpha[3];
    for (int i = 0; i < 3; ++i) alpha[i] = -(DCinv[i][0] * r[0] + DCinv[i][1] * r[1] + DCinv[i][2] * r[2]);
    for (int l = 0; l < L - 2; ++l) { mp.p[l][0] = q[2 * l]; mp.p[l][1] = q[2 * l + 1]; }
    mp.p[L - 2][0] = kp0;
    mp.p[L - 2][1] = alpha[0];
    mp.p[L - 1][0] = alpha[1];
    mp.p[L - 1][1] = alpha[2];
    const bool thp = (kp0 > 0.0) && (alpha[0] > 0.0) && (kp0 + alpha[0] < 1.0);
    const bool thc = (alpha[1] > 0.0) && (alpha[2] > 0.0) && (alpha[1] + alpha[2] < 1.0);
    mp.theta = thp && thc;
}

static double factorial_norm(int L) {
    // (NDim!)^(L-2) * (NDim-1)! with NDim = 2 (IntegratorCore.hpp:342-353)
    double f = 1.0;
    for (int i = 0; i < L - 2; ++i) f *= 2.0;
    return f;
}

// constructAmplitude, ScatteringChannel.cpp:399-415 (functAmplitude == 1).
static double full_amplitude(const Problem& P, const Channel& c, double amplitude) {
    double a = amplitude;
    for (int l = 0; l < c.L; ++l) a *= P.meshes[P.bands[c.band[l]].mesh].vol * 2.0;
    return a;
}

// ---------------------------------------------------------- tuple enumeration
// TrapezoidalSubset arithmetic, MeshSubset.cpp:82-87 (conversion to a box with
// the 1e-8 shrink), :169-194 (+, scalar *), :62-66 / :121-125 (back to
// section coordinates).
struct Box { double l[2], h[2]; };

static Box section_box(const Mesh& m, int sx, int sy) {
    Box b;
    const double lo[2] = {double(sx) + 0.00000001, double(sy) + 0.00000001};
    const double hi[2] = {double(sx + 1) - 0.00000001, double(sy + 1) - 0.00000001};
    for (int i = 0; i < 2; ++i) {
        b.l[i] = m.origin[i] + (m.dG[i][0] * lo[0] + m.dG[i][1] * lo[1]);
        b.h[i] = m.origin[i] + (m.dG[i][0] * hi[0] + m.dG[i][1] * hi[1]);
    }
    return b;
}

static Box box_scale(Box b, double s) {
    if (s >= 0.0) {
        for (int i = 0; i < 2; ++i) { b.l[i] *= s; b.h[i] *= s; }
    } else {
        for (int i = 0; i < 2; ++i) { std::swap(b.l[i], b.h[i]); b.l[i] *= s; b.h[i] *= s; }
    }
    return b;
}

static void box_to_sections(const Mesh& m, const Box& b, int lo[2], int hi[2]) {
    const int ns[2] = {m.nx, m.ny};
    for (int i = 0; i < 2; ++i) {
        double tl = m.invdG[i][0] * (b.l[0] - m.origin[0]) + m.invdG[i][1] * (b.l[1] - m.origin[1]);
        double th = m.invdG[i][0] * (b.h[0] - m.origin[0]) + m.invdG[i][1] * (b.h[1] - m.origin[1]);
        int a = int(std::floor(tl));
        int c = int(std::floor(th) + 1.0);
        lo[i] = std::min(std::max(a, 0), ns[i]);
        hi[i] = std::min(std::max(c, 0), ns[i]);
    }
}

// Survival test of precalculateIndices, ScatteringChannel.cpp:476-504:
// |det DC| >= minimumDeterminant and |TypeC(0,0) * fullAmplitude| > threshold,
// where TypeC with the constant modal form (sqrt 2 per leg,
// Function.hpp:384-388) reduces to fullAmp * sqrt2^L * hits / (norm*NMC*|det|).
static int tuple_survives(const Problem& P, const Channel& c, const int32_t* e, int umk, bool& det_ok) {
    Geom g;
    build_geom(P, c, e, umk, g);
    det_ok = std::fabs(g.det) >= c.min_det;
    if (!det_ok) return 0;
    double DCinv[3][3];
    inv3(g.DC, DCinv);
    const int R = 2 * (c.L - 2) + 1;
    const double s2 = std::sqrt(2.0);
    double prodc = 1.0;
    for (int l = 0; l < c.L; ++l) prodc *= s2;
    double sum = 0.0;
    MCPoint mp;
    for (int m = 0; m < c.nmc; ++m) {
        mc_point(c.L, g, DCinv, &c.mc_pre[size_t(m) * R], mp);
        sum += mp.theta ? prodc : 0.0;
    }
    double res = (1.0 / (factorial_norm(c.L) * double(c.nmc) * std::fabs(g.det))) * sum;
    res *= full_amplitude(P, c, 1.0);
    return std::fabs(res) > c.threshold ? 1 : 0;
}

struct EnumPart {
    std::vector<int32_t> tuples, tumk;
    int64_t n_pre = 0, n_det = 0;
};

static void enumerate_range(const Problem& P, const Channel& c, int u, int s0_begin, int s0_end, EnumPart& out) {
    const int L = c.L;
    const Mesh* ms[4];
    const Band* bs[4];
    for (int l = 0; l < L; ++l) { bs[l] = &P.bands[c.band[l]]; ms[l] = &P.meshes[bs[l]->mesh]; }
    const double* G = P.region.gvec;
    int sec[3] = {0, 0, 0};
    int nsec[3] = {1, 1, 1};
    for (int l = 0; l < L - 1; ++l) nsec[l] = ms[l]->nx * ms[l]->ny;
    int32_t e[4];
    const double ux = c.umk[2 * u], uy = c.umk[2 * u + 1];
    const double gu[2] = {G[0] * ux + G[2] * uy, G[1] * ux + G[3] * uy};
    for (sec[0] = s0_begin; sec[0] < s0_end; ++sec[0])
    for (sec[1] = 0; sec[1] < nsec[1]; ++sec[1])
    for (sec[2] = 0; sec[2] < nsec[2]; ++sec[2]) {
        // box of the last leg: -dir[L-1] * (sum_l dir[l]*box_l + gVec*umklapp)
        Box acc{};
        for (int l = 0; l < L - 1; ++l) {
            Box b = box_scale(section_box(*ms[l], sec[l] % ms[l]->nx, sec[l] / ms[l]->nx), double(c.dir[l]));
            if (l == 0) acc = b;
            else for (int i = 0; i < 2; ++i) { acc.l[i] += b.l[i]; acc.h[i] += b.h[i]; }
        }
        for (int i = 0; i < 2; ++i) { acc.l[i] += gu[i]; acc.h[i] += gu[i]; }
        acc = box_scale(acc, -double(c.dir[L - 1]));
        int lo[2], hi[2];
        box_to_sections(*ms[L - 1], acc, lo, hi);
        if (!(lo[0] != hi[0] && lo[1] != hi[1])) continue;
        const int ncomb = 1 << (L - 1);
        for (int comb = 0; comb < ncomb; ++comb) {
            // element of leg l within its section: bit (L-2-l) of comb
            double minE = 0.0, maxE = 0.0;
            double mn[4], mx[4];
            for (int l = 0; l < L - 1; ++l) {
                int i = (comb >> (L - 2 - l)) & 1;
                e[l] = 2 * sec[l] + i;
                mn[l] = (c.dir[l] > 0) ? bs[l]->minE[e[l]] : -bs[l]->maxE[e[l]];
                mx[l] = (c.dir[l] > 0) ? bs[l]->maxE[e[l]] : -bs[l]->minE[e[l]];
            }
            const Mesh& ml = *ms[L - 1];
            for (int sy = lo[1]; sy < hi[1]; ++sy)
                for (int sx = lo[0]; sx < hi[0]; ++sx)
                    for (int i = 0; i < 2; ++i) {
                        e[L - 1] = 2 * (sx + sy * ml.nx) + i;
                        const int l = L - 1;
                        mn[l] = (c.dir[l] > 0) ? bs[l]->minE[e[l]] : -bs[l]->maxE[e[l]];
                        mx[l] = (c.dir[l] > 0) ? bs[l]->maxE[e[l]] : -bs[l]->minE[e[l]];
                        minE = 0.0; maxE = 0.0;
                        for (int k = 0; k < L; ++k) { minE += mn[k]; maxE += mx[k]; }
                        if (!((minE <= 0.0) && (maxE >= 0.0))) continue;
                        ++out.n_pre;
                        bool det_ok;
                        if (tuple_survives(P, c, e, u, det_ok)) {
                            for (int k = 0; k < L; ++k) out.tuples.push_back(e[k]);
                            out.tumk.push_back(u);
                        }
                        if (det_ok) ++out.n_det;
                    }
        }
    }
}

// The same loops indexed by work item: item = (((u nsec0 + s0) nsec1 + s1)
// nsec2 + s2) 2^(L-1) + comb, i.e. the position of (umklapp, sections of
// legs 0..L-2, element choice of those legs) in the reference's loop order
// (comb innermost, because the element loops of legs 0..L-2 run inside the
// section loops; ScatteringChannel.hpp:216-255).  Enumerates items
// [item0, item1) in order: a contiguous piece of the full list.
static void enumerate_items(const Problem& P, const Channel& c, int64_t item0, int64_t item1, EnumPart& out) {
    const int L = c.L;
    const Mesh* ms[4];
    const Band* bs[4];
    for (int l = 0; l < L; ++l) { bs[l] = &P.bands[c.band[l]]; ms[l] = &P.meshes[bs[l]->mesh]; }
    const double* G = P.region.gvec;
    int64_t nsec[3] = {1, 1, 1};
    for (int l = 0; l < L - 1; ++l) nsec[l] = int64_t(ms[l]->nx) * ms[l]->ny;
    const int ncomb = 1 << (L - 1);
    int32_t e[4];
    for (int64_t item = item0; item < item1; ++item) {
        const int comb = int(item % ncomb);
        int64_t r = item / ncomb;
        int sec[3] = {0, 0, 0};
        for (int l = L - 2; l >= 0; --l) { sec[l] = int(r % nsec[l]); r /= nsec[l]; }
        const int u = int(r);
        const double ux = c.umk[2 * u], uy = c.umk[2 * u + 1];
        const double gu[2] = {G[0] * ux + G[2] * uy, G[1] * ux + G[3] * uy};
        Box acc{};
        for (int l = 0; l < L - 1; ++l) {
            Box b = box_scale(section_box(*ms[l], sec[l] % ms[l]->nx, sec[l] / ms[l]->nx), double(c.dir[l]));
            if (l == 0) acc = b;
            else for (int i = 0; i < 2; ++i) { acc.l[i] += b.l[i]; acc.h[i] += b.h[i]; }
        }
        for (int i = 0; i < 2; ++i) { acc.l[i] += gu[i]; acc.h[i] += gu[i]; }
        acc = box_scale(acc, -double(c.dir[L - 1]));
        int lo[2], hi[2];
        box_to_sections(*ms[L - 1], acc, lo, hi);
        if (!(lo[0] != hi[0] && lo[1] != hi[1])) continue;
        double mn[4], mx[4];
        for (int l = 0; l < L - 1; ++l) {
            const int i = (comb >> (L - 2 - l)) & 1;
            e[l] = 2 * sec[l] + i;
            mn[l] = (c.dir[l] > 0) ? bs[l]->minE[e[l]] : -bs[l]->maxE[e[l]];
            mx[l] = (c.dir[l] > 0) ? bs[l]->maxE[e[l]] : -bs[l]->minE[e[l]];
        }
        const Mesh& ml = *ms[L - 1];
        for (int sy = lo[1]; sy < hi[1]; ++sy)
            for (int sx = lo[0]; sx < hi[0]; ++sx)
                for (int i = 0; i < 2; ++i) {
                    e[L - 1] = 2 * (sx + sy * ml.nx) + i;
                    const int l = L - 1;
                    mn[l] = (c.dir[l] > 0) ? bs[l]->minE[e[l]] : -bs[l]->maxE[e[l]];
                    mx[l] = (c.dir[l] > 0) ? bs[l]->maxE[e[l]] : -bs[l]->minE[e[l]];
                    double minE = 0.0, maxE = 0.0;
                    for (int k = 0; k < L; ++k) { minE += mn[k]; maxE += mx[k]; }
                    if (!((minE <= 0.0) && (maxE >= 0.0))) continue;
                    ++out.n_pre;
                    bool det_ok;
                    if (tuple_survives(P, c, e, u, det_ok)) {
                        for (int k = 0; k < L; ++k) out.tuples.push_back(e[k]);
                        out.tumk.push_back(u);
                    }
                    if (det_ok) ++out.n_det;
                }
    }
}

// deterministicIteration / nestedForSections / nestedForElements,
// ScatteringChannel.hpp:205-255, driven by precalculateIndices
// (ScatteringChannel.cpp:461-507).  Tuples are produced in the reference's
// loop order: umklapp, sections of legs 0..L-2, elements of legs 0..L-1.
// The outermost section loop is split into contiguous ranges over threads and
// the per-range lists are concatenated in order.
static void enumerate(const Problem& P, Channel& c, int nthreads) {
    const int nU = int(c.umk.size() / 2);
    c.tuples.clear();
    c.tumk.clear();
    c.n_prefilter = 0;
    c.n_det = 0;
    const Mesh& m0 = P.meshes[P.bands[c.band[0]].mesh];
    const int ns0 = m0.nx * m0.ny;
    nthreads = std::max(1, std::min(nthreads, ns0));
    for (int u = 0; u < nU; ++u) {
        std::vector<EnumPart> parts(nthreads);
        std::vector<std::thread> th;
        auto work = [&](int t) {
            enumerate_range(P, c, u, int(int64_t(ns0) * t / nthreads), int(int64_t(ns0) * (t + 1) / nthreads), parts[t]);
        };
        for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
        work(0);
        for (auto& x : th) x.join();
        for (auto& p : parts) {
            c.tuples.insert(c.tuples.end(), p.tuples.begin(), p.tuples.end());
            c.tumk.insert(c.tumk.end(), p.tumk.begin(), p.tumk.end());
            c.n_prefilter += p.n_pre;
            c.n_det += p.n_det;
        }
    }
}

// ----------------------------------------------------------------- propagate
// singleScatteringPropagator (array overload), ScatteringChannel.cpp:618-650,
// with scatteringIntegrationTypeB, IntegratorCore.hpp:260-357.
// which < 0: singleScatteringPropagator (ScatteringChannel.cpp:618-650).
// which = leg: singleScatteringRate (ScatteringChannel.cpp:544-581): the forms
// of that leg become the constant in / out unit forms and only its block is
// kept, subtracted with the leg's direction.
static void single_propagator(const Problem& P, const Channel& c, const double* f, const int32_t* e, int umk,
                              double* out, int which = -1, double funct_amp = 1.0) {
    const int L = c.L;
    Geom g;
    build_geom(P, c, e, umk, g);
    if (std::fabs(g.det) < c.min_det) return;
    double DCinv[3][3];
    inv3(g.DC, DCinv);
    // commonLinForm0 / commonLinForm1, ScatteringChannel.cpp:633-641
    double A[4][3], B[4][3];
    for (int l = 0; l < L; ++l) {
        const Band& b = P.bands[c.band[l]];
        const double d = double(c.dir[l]), s = b.statistics;
        const double* fe = f + P.off[c.band[l]] + 3 * size_t(e[l]);
        const double ka = (l == 0 ? -1.0 : 1.0) * 0.5;
        const double ca = (1. - d) * s + (1. + d);
        const double cb = (1. + d) * s + (1. - d);
        for (int j = 0; j < 3; ++j) {
            const double unit = (j == 0) ? 1.0 : 0.0;
            if (l == which) {   // ScatteringChannel.cpp:562-564
                A[l][j] = (l == 0 ? -1.0 : 1.0) * ca * unit;
                B[l][j] = cb * unit;
            } else {
                A[l][j] = ka * ((1. - d) * unit + ca * fe[j]);
                B[l][j] = 0.5 * ((1. + d) * unit + cb * fe[j]);
            }
        }
    }
    const int R = 2 * (L - 2) + 1;
    double acc[4][3] = {};
    MCPoint mp;
    for (int m = 0; m < c.nmc; ++m) {
        mc_point(L, g, DCinv, &c.mc[size_t(m) * R], mp);
        double pa = 1.0, pb = 1.0;
        for (int l = 0; l < L; ++l) {
            pa *= lf_apply(A[l], mp.p[l][0], mp.p[l][1]);
            pb *= lf_apply(B[l], mp.p[l][0], mp.p[l][1]);
        }
        const double common = (pa + pb) * (mp.theta ? 1.0 : 0.0);
        for (int l = 0; l < L; ++l) {
            acc[l][0] += common;
            acc[l][1] += mp.p[l][0] * common;
            acc[l][2] += mp.p[l][1] * common;
        }
    }
    const double scale = 1.0 / (factorial_norm(L) * double(c.nmc) * std::fabs(g.det));
    const double amp = full_amplitude(P, c, c.amplitude) * funct_amp;
    for (int l = 0; l < L; ++l) {
        if (which >= 0 && l != which) continue;
        double* o = out + P.off[c.band[l]] + 3 * size_t(e[l]);
        const double d = double(c.dir[l]);
        for (int j = 0; j < 3; ++j) {
            if (which >= 0) o[j] -= d * ((scale * acc[l][j]) * amp);
            else o[j] += d * ((scale * acc[l][j]) * amp);
        }
    }
}

// ScatteringChannel::propagate, ScatteringChannel.cpp:651-670: parallel
// reduction over tuple ranges with one private accumulator per task
// (TBB parallel_reduce there, std::thread here), then applyInverseMass.
static void channel_propagate_range(const Problem& P, const Channel& c, const double* f, double* out,
                                    int64_t t0, int64_t t1, int nthreads, bool inverse_mass, int which = -1) {
    const int64_t n = t1 - t0;
    nthreads = std::max(1, std::min<int>(nthreads, int(std::max<int64_t>(1, n / 64))));
    std::vector<std::vector<double>> part(nthreads, std::vector<double>(size_t(P.ndofs), 0.0));
    auto work = [&](int t) {
        int64_t a = t0 + n * t / nthreads, b = t0 + n * (t + 1) / nthreads;
        for (int64_t i = a; i < b; ++i)
            single_propagator(P, c, f, &c.tuples[size_t(i) * c.L], c.tumk[size_t(i)], part[t].data(), which,
                              c.tamp.empty() ? 1.0 : c.tamp[size_t(i)]);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    std::vector<double> tot(size_t(P.ndofs), 0.0);
    for (int t = 0; t < nthreads; ++t)
        for (int64_t i = 0; i < P.ndofs; ++i) tot[i] += part[t][i];
    if (inverse_mass)
        for (size_t b = 0; b < P.bands.size(); ++b) apply_inverse_mass(P.meshes[P.bands[b].mesh], tot.data() + P.off[b]);
    for (int64_t i = 0; i < P.ndofs; ++i) out[i] += tot[i];
}

// Vlasov<2>::vlasovFlux = (volumeFlux - surfaceFlux) * M^-1,
// include/Physics/Transport/Vlasov.hpp:69-118, with Mesh<2> adjacency, normals
// and face areas from Mesh.cpp:573-660 and the basis derivatives of
// Mesh.cpp:147-163 evaluated on calculate_verticesCoord (Mesh.cpp:222-241).
static int adjacent_element(const Mesh& m, int e, int face) {
    const int nx = m.nx, nt = 2 * m.nx * m.ny;
    if (e % 2) {
        switch (face) {
            case 0: return (e + 2 * nx - 1 + nt) % nt;
            case 1: return e - 1;
            default: return ((e - 1) % (2 * nx) == 0) ? e + 2 * nx - 3 : e - 3;
        }
    } else {
        switch (face) {
            case 0: return ((e + 2) % (2 * nx) == 0) ? e - 2 * nx + 3 : e + 3;
            case 1: return e + 1;
            default: return (e - 2 * nx + 1 + nt) % nt;
        }
    }
}

static void face_normal(const Mesh& m, int e, int face, double n[2]) {
    const double (&d)[2][2] = m.dG;
    double v[2];
    double sgn;
    auto norm = [](const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1]); };
    auto dotc = [&](const double* a, int col) { return a[0] * d[0][col] + a[1] * d[1][col]; };
    if (e % 2) {
        switch (face) {
            case 0: v[0] = d[1][0]; v[1] = -d[0][0]; sgn = (dotc(v, 1) > 0.) ? 1. : -1.; break;
            case 1: v[0] = d[1][1] + d[1][0]; v[1] = -d[0][1] - d[0][0];
                    sgn = ((v[0] * d[0][0] + v[1] * d[1][0]) > 0.) ? 1. : -1.; break;
            default: v[0] = d[1][1]; v[1] = -d[0][1]; sgn = (dotc(v, 0) > 0.) ? -1. : 1.; break;
        }
    } else {
        switch (face) {
            case 0: v[0] = d[1][1]; v[1] = -d[0][1]; sgn = (dotc(v, 0) > 0.) ? 1. : -1.; break;
            case 1: v[0] = d[1][1] + d[1][0]; v[1] = -d[0][1] - d[0][0];
                    sgn = ((v[0] * d[0][0] + v[1] * d[1][0]) > 0.) ? -1. : 1.; break;
            default: v[0] = d[1][0]; v[1] = -d[0][0]; sgn = (dotc(v, 1) > 0.) ? -1. : 1.; break;
        }
    }
    const double nn = norm(v);
    n[0] = v[0] / nn * sgn;
    n[1] = v[1] / nn * sgn;
}

static double face_area(const Mesh& m, int e, int face) {
    const double (&d)[2][2] = m.dG;
    auto nc = [&](double x, double y) { return std::sqrt(x * x + y * y); };
    if (e % 2) {
        switch (face) {
            case 0: return nc(d[0][0], d[1][0]);
            case 1: return nc(d[0][0] + d[0][1], d[1][0] + d[1][1]);
            default: return nc(d[0][1], d[1][1]);
        }
    } else {
        switch (face) {
            case 0: return nc(d[0][1], d[1][1]);
            case 1: return nc(d[0][0] + d[0][1], d[1][0] + d[1][1]);
            default: return nc(d[0][0], d[1][0]);
        }
    }
}

// gaussPointsSide<2,2>, Vlasov.hpp:49-62.
static void side_point(int side, int q, double& x, double& y) {
    const double g = kGP1[q];
    switch (side) {
        case 0: x = 1. - g; y = g; break;
        case 1: x = 0.; y = g; break;
        default: x = g; y = 0.; break;
    }
}

// basisFuncDerivLF0thOrd for one element, Mesh.cpp:147-163 on the vertex
// table of calculate_verticesCoord<2> (which adds the *relative* origin).
static void basis_derivs(const Mesh& m, int e, double dx[3], double dy[3]) {
    double vx[3], vy[3];
    int s = e / 2, par = e % 2;
    double sx = double(s % m.nx), sy = double(s / m.nx);
    for (int k = 0; k < 3; ++k) {
        double px = sx + kVert[par][k][0], py = sy + kVert[par][k][1];
        vx[k] = m.rel_origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
        vy[k] = m.rel_origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
    }
    const double v0X = vx[0], v0Y = vy[0], v1X = vx[1], v1Y = vy[1], v2X = vx[2], v2Y = vy[2];
    dx[0] = 0.0;
    dx[1] = (v0Y - v2Y) / (v0Y * (v1X - v2X) + v1Y * (v2X - v0X) + v2Y * (v0X - v1X));
    dx[2] = -(v0Y - v1Y) / (v0Y * (v1X - v2X) + v1Y * (v2X - v0X) + v2Y * (v0X - v1X));
    dy[0] = 0.0;
    dy[1] = (v0X - v2X) / (v0X * (v1Y - v2Y) + v1X * (v2Y - v0Y) + v2X * (v0Y - v1Y));
    dy[2] = -(v0X - v1X) / (v0X * (v1Y - v2Y) + v1X * (v2Y - v0Y) + v2X * (v0Y - v1Y));
}

static void vlasov_flux(const Mesh& m, const double* f, const double vel[2], double* out) {
    std::vector<double> vol(size_t(m.ne) * 3, 0.0), sur(size_t(m.ne) * 3, 0.0);
    // volumeFlux, Vlasov.hpp:78-92
    for (int dim = 0; dim < 2; ++dim) {
        for (int e = 0; e < m.ne; ++e) {
            double gi = 0.0;
            for (int q = 0; q < 3; ++q) gi += lf_apply(f + 3 * e, kGP2[q][0], kGP2[q][1]) * kGW2[q];
            double dx[3], dy[3];
            basis_derivs(m, e, dx, dy);
            for (int b = 0; b < 3; ++b) {
                const double part = (dim == 0 ? dx[b] : dy[b]) * gi;
                vol[3 * e + b] += m.vol * vel[dim] * part;
            }
        }
    }
    // surfaceFlux, Vlasov.hpp:94-118
    for (int e = 0; e < m.ne; ++e)
        for (int b = 0; b < 3; ++b)
            for (int side = 0; side < 3; ++side) {
                double n[2];
                face_normal(m, e, side, n);
                const double s = vel[0] * n[0] + vel[1] * n[1];
                int ei, si;
                if (s > 0.) { ei = e; si = side; }
                else { ei = adjacent_element(m, e, side); si = 2 - side; }
                double acc = 0.0;
                for (int q = 0; q < 2; ++q) {
                    double x, y, xi, yi;
                    side_point(side, q, x, y);
                    side_point(si, q, xi, yi);
                    const double basis[3] = {0, 0, 0};
                    double bc[3] = {basis[0], basis[1], basis[2]};
                    bc[b] = 1.0;
                    acc += lf_apply(bc, x, y) * lf_apply(f + 3 * size_t(ei), xi, yi) * kGW1[q];
                }
                sur[3 * e + b] += s * acc * face_area(m, e, side);
            }
    std::vector<double> r(size_t(m.ne) * 3);
    for (size_t i = 0; i < r.size(); ++i) r[i] = vol[i] - sur[i];
    apply_inverse_mass(m, r.data());
    for (size_t i = 0; i < r.size(); ++i) out[i] += r[i];
}

// ---------------------------------------------------------------- RHS / error
// MaterialStatus::propagate, MaterialStatus.cpp:146-161 (channels with
// amplitude != 0), plus the Vlasov drift of every band with nonzero velocity.
static void rhs(const Problem& P, const double* f, double* out, int nthreads, bool drift) {
    std::fill(out, out + P.ndofs, 0.0);
    for (const Channel& c : P.chans) {
        if (c.amplitude == 0.) continue;
        channel_propagate_range(P, c, f, out, 0, int64_t(c.tumk.size()), nthreads, true);
    }
    if (drift)
        for (size_t b = 0; b < P.bands.size(); ++b) {
            const Band& bd = P.bands[b];
            if (bd.vel[0] == 0.0 && bd.vel[1] == 0.0) continue;
            vlasov_flux(P.meshes[bd.mesh], f + P.off[b], bd.vel, out + P.off[b]);
        }
}

// Band::relativeError, src/Physics/Material/Band.cpp:87-101, with the nodal
// min/max/fabs/division of Function.cpp:152-159 and Function.hpp:315-320.
static double band_relative_error(const Mesh& m, const Band& b, const double* err, const double* pop) {
    const int ne = m.ne;
    std::vector<double> scale(size_t(ne) * 3), rel(size_t(ne) * 3), pen(size_t(ne) * 3);
    for (int e = 0; e < ne; ++e) {
        const double* p = pop + 3 * e;
        double np[3];
        to_nodal(p, np);
        double sc[3];
        if (b.statistics == -1) {
            // 1 - population: AsymmetricMathFieldSpace operator-(Real, T) = -(T - r)
            double om[3] = {-(p[0] - 1.0), -p[1], -p[2]};
            double nom[3];
            to_nodal(om, nom);
            double fa[3], fb[3], mn[3];
            for (int k = 0; k < 3; ++k) { fa[k] = std::fabs(np[k]); fb[k] = std::fabs(nom[k]); }
            double la[3], lb[3];
            to_lin(fa, la);
            to_lin(fb, lb);
            double na[3], nb[3];
            to_nodal(la, na);
            to_nodal(lb, nb);
            for (int k = 0; k < 3; ++k) mn[k] = std::min(na[k], nb[k]);
            double lm[3];
            to_lin(mn, lm);
            for (int k = 0; k < 3; ++k) sc[k] = b.rel_tol * lm[k];
            sc[0] += b.abs_tol;
            // penalisation: (-min(pop,0) + max(pop-1,0)) / scale
            double m0[3], lm0[3];
            for (int k = 0; k < 3; ++k) m0[k] = std::min(np[k], 0.);
            to_lin(m0, lm0);
            double pm1[3] = {p[0] - 1.0, p[1], p[2]}, npm1[3], x1[3], lx1[3];
            to_nodal(pm1, npm1);
            for (int k = 0; k < 3; ++k) x1[k] = std::max(npm1[k], 0.);
            to_lin(x1, lx1);
            double pe[3];
            for (int k = 0; k < 3; ++k) pe[k] = -lm0[k] + lx1[k];
            double npe[3], nsc[3];
            to_nodal(pe, npe);
            to_nodal(sc, nsc);
            for (int k = 0; k < 3; ++k) npe[k] /= nsc[k];
            to_lin(npe, &pen[3 * e]);
        } else {
            for (int k = 0; k < 3; ++k) sc[k] = b.rel_tol * p[k];
            sc[0] += b.abs_tol;
            double m0[3], lm0[3];
            for (int k = 0; k < 3; ++k) m0[k] = std::min(np[k], 0.);
            to_lin(m0, lm0);
            double pe[3] = {-lm0[0], -lm0[1], -lm0[2]};
            double npe[3], nsc[3];
            to_nodal(pe, npe);
            to_nodal(sc, nsc);
            for (int k = 0; k < 3; ++k) npe[k] /= nsc[k];
            to_lin(npe, &pen[3 * e]);
        }
        double ner[3], nsc[3];
        to_nodal(err + 3 * e, ner);
        to_nodal(sc, nsc);
        for (int k = 0; k < 3; ++k) ner[k] /= nsc[k];
        to_lin(ner, &rel[3 * e]);
    }
    const double ir = integrate2(m, rel.data(), rel.data());
    const double ip = integrate2(m, pen.data(), pen.data());
    return std::sqrt((ir + b.penal * ip) / (double(ne) * m.vol));
}

// MaterialStatus::relativeError, MaterialStatus.cpp:189-196 (max over bands,
// a NaN band error never replaces the running maximum).
static double relative_error(const Problem& P, const double* err, const double* pop) {
    double error = 0.0;
    for (size_t b = 0; b < P.bands.size(); ++b) {
        const Band& bd = P.bands[b];
        double ne = band_relative_error(P.meshes[bd.mesh], bd, err + P.off[b], pop + P.off[b]);
        if (ne >= error) error = ne;
    }
    return error;
}

// MaterialStatus::applyConstraints, MaterialStatus.cpp:198-206 (time-independent
// constrained populations).
static void apply_constraints(const Problem& P, double* f) {
    for (size_t b = 0; b < P.bands.size(); ++b)
        if (P.bands[b].constrained)
            std::copy(P.bands[b].cpop.begin(), P.bands[b].cpop.end(), f + P.off[b]);
}

// MaterialStatus::applyConstraints(time): every constrained band takes
// constrainedPopulation(t) -- the callback when one is set.
static void apply_constraints_at(const Problem& P, double t, double* f) {
    if (!P.cfn) { apply_constraints(P, f); return; }
    for (size_t b = 0; b < P.bands.size(); ++b)
        if (P.bands[b].constrained && P.cfn(P.cuser, int32_t(b), t, f + P.off[b]) != 0)
            throw std::runtime_error("constraint callback failed");
}

// Function<2> element-wise operations as the reference evaluates them
// (Function.cpp:75-80, 152-159, 172-175, 338-341): + - and scalar * act on
// the linear-form coefficients, Function + scalar on c0 only, fabs and
// Function / Function go to the nodal values and back, max() is the largest
// nodal value.
static void fn_fabs(const double* c, double* out, int64_t ne) {
    for (int64_t e = 0; e < ne; ++e) {
        double n[3];
        to_nodal(c + 3 * e, n);
        for (int k = 0; k < 3; ++k) n[k] = std::fabs(n[k]);
        to_lin(n, out + 3 * e);
    }
}

// MaterialTimeStatus::timeStepVetoer, MaterialTimeStatus.cpp:60-100: the
// largest step from times[0] such that every constrained band stays, at the
// dense-step probes inside each stage interval, within 1.3 |left - right| +
// atol + rtol |average| of the interval's average (nodally).
static double veto_step(const Problem& P, const double* times, int ntimes, double dense) {
    double critical = times[ntimes - 1];
    bool found = false;
    for (size_t b = 0; b < P.bands.size() && !found; ++b) {
        const Band& bd = P.bands[b];
        if (!bd.constrained) continue;
        const int64_t ne = P.meshes[bd.mesh].ne, n = 3 * ne;
        std::vector<double> left(n), right(n), avg(n), acc(n), tmp(n), tmp2(n), mid(n);
        auto pop = [&](double t, double* out) {
            if (P.cfn) {
                if (P.cfn(P.cuser, int32_t(b), t, out) != 0) throw std::runtime_error("constraint callback failed");
            } else {
                std::copy(bd.cpop.begin(), bd.cpop.end(), out);
            }
        };
        double tt = times[0] + dense;
        pop(times[0], left.data());
        pop(times[1], right.data());
        for (int i = 0; i < ntimes - 1 && !found; ++i) {
            if (i != 0) {
                left.swap(right);
                pop(times[i + 1], right.data());
            }
            for (int64_t k = 0; k < n; ++k) avg[k] = 0.5 * (left[k] + right[k]);
            // (1 + 0.3) fabs(left - right) + atol + rtol fabs(avg)
            for (int64_t k = 0; k < n; ++k) tmp[k] = left[k] - right[k];
            fn_fabs(tmp.data(), tmp2.data(), ne);
            for (int64_t k = 0; k < n; ++k) acc[k] = (1. + 0.3) * tmp2[k];
            for (int64_t e = 0; e < ne; ++e) acc[3 * e] += bd.abs_tol;
            fn_fabs(avg.data(), tmp2.data(), ne);
            for (int64_t k = 0; k < n; ++k) acc[k] = acc[k] + bd.rel_tol * tmp2[k];
            while (tt < times[i + 1]) {
                pop(tt, mid.data());
                for (int64_t k = 0; k < n; ++k) tmp[k] = mid[k] - avg[k];
                fn_fabs(tmp.data(), tmp2.data(), ne);
                double mx = -INFINITY;
                for (int64_t e = 0; e < ne; ++e) {
                    double a[3], q[3], r[3], lin[3];
                    to_nodal(tmp2.data() + 3 * e, a);
                    to_nodal(acc.data() + 3 * e, q);
                    for (int k = 0; k < 3; ++k) r[k] = a[k] / q[k];
                    to_lin(r, lin);   // the quotient is stored in linear form ...
                    to_nodal(lin, r); // ... and max() reads it back nodally
                    for (int k = 0; k < 3; ++k) mx = std::max(mx, r[k]);
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
    return critical - times[0];
}

// --------------------------------------------------------------------- DP54
// Algorithms::dormandPrince54 (3rd overload), DormandPrince54.hpp:479-665,
// driven as MaterialTimeStatus::propagate does (MaterialTimeStatus.cpp:102-137).
// With only time-independent constraints MaterialTimeStatus::timeStepVetoer
// (MaterialTimeStatus.cpp:60-100) returns timesToTest.back()-timesToTest[0].
struct DPStats {
    int64_t attempts = 0, accepted = 0, rejected = 0, rhs_evals = 0;
    double t = 0.0, dt = 0.0, last_err = 0.0;
    int failed = 0;
};

// enforce_fn(t, v) is enforceValue at time t; veto_fn(times[6]) the
// timeStepVetoer (applied at the start and after every accepted step).
template <class RHS, class ENF, class NORM, class VETO>
static int dp54_core(int64_t n, double* y_io, double t0, double tf, double dense, double* dense_out,
                     double* dense_t, int max_dense, int* n_dense, int64_t max_attempts, DPStats& st, RHS rhs_fn,
                     ENF enforce_fn, NORM norm_fn, VETO veto_fn) {
    const double c2 = 1. / 5., c3 = 3. / 10., c4 = 4. / 5., c5 = 8. / 9.;
    const double a21 = 1. / 5., a31 = 3. / 40., a32 = 9. / 40., a41 = 44. / 45., a42 = -56. / 15., a43 = 32. / 9.,
                 a51 = 19372. / 6561., a52 = -25360. / 2187., a53 = 64448. / 6561., a54 = -212. / 729.,
                 a61 = 9017. / 3168., a62 = -355. / 33., a63 = 46732. / 5247., a64 = 49. / 176.,
                 a65 = -5103. / 18656.;
    const double b1 = 35. / 384., b3 = 500. / 1113., b4 = 125. / 192., b5 = -2187. / 6784., b6 = 11. / 84.;
    const double bh1 = 5179. / 57600., bh3 = 7571. / 16695., bh4 = 393. / 640., bh5 = -92097. / 339200.,
                 bh6 = 187. / 2100., bh7 = 1. / 40.;
    std::vector<double> y(y_io, y_io + n), k1(n), k2(n), k3(n), k4(n), k5(n), k6(n), k7(n), y5(n), err(n), tmp(n),
        tmp2(n);
    double t = t0, dt = dense, denseTime = t0 + dense;
    const double minStep = dense / 10000.;
    bool notfailed = true, rejected = false;
    const double minscale = 0.333333, maxscale = 3.0, safety = 0.98, alpha = 0.7 / 5., beta = 0.4 / 5.;
    double olderror = 1.0;
    *n_dense = 0;
    auto f_rhs = [&](const double* in, double* out) { rhs_fn(in, out); ++st.rhs_evals; };
    auto enforce = [&](double tt, double* v) { enforce_fn(tt, v); };
    auto veto = [&]() {
        const double times[6] = {t, t + c2 * dt, t + c3 * dt, t + c4 * dt, t + c5 * dt, t + dt};
        dt = std::min(dt, veto_fn(times));
    };
    // k1 = timeOp(t, enforceValue(t, y))
    std::copy(y.begin(), y.end(), tmp.begin());
    enforce(t, tmp.data());
    f_rhs(tmp.data(), k1.data());
    veto();
    // Expression templates of the reference evaluate currentY + (a*dt)*k1 + ...
    // left to right; the same order is used here.
    while (t < tf && notfailed) {
        if (max_attempts > 0 && st.attempts >= max_attempts) break;
        ++st.attempts;
        for (int64_t i = 0; i < n; ++i) tmp[i] = y[i] + (a21 * dt) * k1[i];
        enforce(t + c2 * dt, tmp.data()); f_rhs(tmp.data(), k2.data());
        for (int64_t i = 0; i < n; ++i) tmp[i] = y[i] + (a31 * dt) * k1[i] + (a32 * dt) * k2[i];
        enforce(t + c3 * dt, tmp.data()); f_rhs(tmp.data(), k3.data());
        for (int64_t i = 0; i < n; ++i) tmp[i] = y[i] + (a41 * dt) * k1[i] + (a42 * dt) * k2[i] + (a43 * dt) * k3[i];
        enforce(t + c4 * dt, tmp.data()); f_rhs(tmp.data(), k4.data());
        for (int64_t i = 0; i < n; ++i)
            tmp[i] = y[i] + (a51 * dt) * k1[i] + (a52 * dt) * k2[i] + (a53 * dt) * k3[i] + (a54 * dt) * k4[i];
        enforce(t + c5 * dt, tmp.data()); f_rhs(tmp.data(), k5.data());
        for (int64_t i = 0; i < n; ++i)
            tmp[i] = y[i] + (a61 * dt) * k1[i] + (a62 * dt) * k2[i] + (a63 * dt) * k3[i] + (a64 * dt) * k4[i] +
                     (a65 * dt) * k5[i];
        enforce(t + dt, tmp.data()); f_rhs(tmp.data(), k6.data());
        for (int64_t i = 0; i < n; ++i)
            y5[i] = y[i] + (dt * b1) * k1[i] + (dt * b3) * k3[i] + (dt * b4) * k4[i] + (dt * b5) * k5[i] +
                    (dt * b6) * k6[i];
        enforce(t + dt, y5.data());
        f_rhs(y5.data(), k7.data());
        for (int64_t i = 0; i < n; ++i)
            tmp2[i] = y[i] + (dt * bh1) * k1[i] + (dt * bh3) * k3[i] + (dt * bh4) * k4[i] + (dt * bh5) * k5[i] +
                      (dt * bh6) * k6[i] + (dt * bh7) * k7[i];
        enforce(t + dt, tmp2.data());
        for (int64_t i = 0; i < n; ++i) err[i] = y5[i] - tmp2[i];
        const double errNorm = norm_fn(err.data(), y5.data());
        st.last_err = errNorm;
        if (errNorm <= 1.) {
            while (denseTime <= t + (1.0001) * dt && denseTime <= tf + .0001 * dt) {
                const double s = (denseTime - t) / dt;
                const double bt1 = -(435. * s * s * s - 1184. * s * s + 1098. * s - 384.) / (384.);
                const double bt3 = 500. * s * (6. * s * s - 14. * s + 9.) / (1113.);
                const double bt4 = -125. * s * (9. * s * s - 16. * s + 6.) / (192.);
                const double bt5 = 729. * s * (35. * s * s - 64. * s + 26.) / (6784.);
                const double bt6 = -11. * s * (3. * s - 2.) * (5. * s - 6.) / (84.);
                const double bt7 = s * (s - 1.) * (5. * s - 3.) / (2.);
                if (*n_dense < max_dense) {
                    double* o = dense_out + size_t(*n_dense) * n;
                    for (int64_t i = 0; i < n; ++i)
                        o[i] = y[i] + (s * dt * bt1) * k1[i] + (s * dt * bt3) * k3[i] + (s * dt * bt4) * k4[i] +
                               (s * dt * bt5) * k5[i] + (s * dt * bt6) * k6[i] + (s * dt * bt7) * k7[i];
                    enforce(denseTime, o);
                    dense_t[*n_dense] = denseTime;
                }
                ++*n_dense;
                denseTime += dense;
            }
            y.swap(y5);
            t += dt;
            k1.swap(k7);
            double scale;
            if (errNorm == 0.) scale = maxscale;
            else {
                scale = safety * std::pow(1. / errNorm, alpha) * std::pow(olderror, beta);
                scale = std::min(std::max(scale, minscale), maxscale);
            }
            if (rejected) dt *= std::min(1.0, scale);
            else dt *= scale;
            veto();
            rejected = false;
            olderror = errNorm;
            ++st.accepted;
        } else {
            double scale = safety * std::pow(1. / errNorm, 1 / 5.);
            scale = std::min(std::max(scale, minscale), maxscale);
            dt *= scale;
            rejected = true;
            ++st.rejected;
            if (dt < minStep) notfailed = false;
        }
    }
    std::copy(y.begin(), y.end(), y_io);
    st.t = t;
    st.dt = dt;
    st.failed = notfailed ? 0 : 1;
    return notfailed ? 0 : TB_ERR_DT_UNDERFLOW;
}

// Fixed-step replay of accepted Dormand-Prince steps: the step arithmetic of
// dp54_core above with the step sizes given, then the dense output at
// fraction dense_s of the last step (DormandPrince54.hpp:598-611).  The
// reference has no such entry point; it is the map whose derivative the
// library's discrete adjoint computes (step sizes frozen).
template <class RHS, class ENF>
static void dp54_replay_core(int64_t n, const double* y0, const double* dts, int64_t n_steps, double s,
                             double* out, RHS f_rhs, ENF enforce) {
    const double a21 = 1. / 5., a31 = 3. / 40., a32 = 9. / 40., a41 = 44. / 45., a42 = -56. / 15., a43 = 32. / 9.,
                 a51 = 19372. / 6561., a52 = -25360. / 2187., a53 = 64448. / 6561., a54 = -212. / 729.,
                 a61 = 9017. / 3168., a62 = -355. / 33., a63 = 46732. / 5247., a64 = 49. / 176.,
                 a65 = -5103. / 18656.;
    const double b1 = 35. / 384., b3 = 500. / 1113., b4 = 125. / 192., b5 = -2187. / 6784., b6 = 11. / 84.;
    std::vector<double> y(y0, y0 + n), k1(n), k2(n), k3(n), k4(n), k5(n), k6(n), k7(n), y5(n), tmp(n);
    enforce(y.data());
    f_rhs(y.data(), k1.data());
    for (int64_t st = 0; st < n_steps; ++st) {
        const double dt = dts[st];
        for (int64_t i = 0; i < n; ++i) tmp[i] = y[i] + (a21 * dt) * k1[i];
        enforce(tmp.data()); f_rhs(tmp.data(), k2.data());
        for (int64_t i = 0; i < n; ++i) tmp[i] = y[i] + (a31 * dt) * k1[i] + (a32 * dt) * k2[i];
        enforce(tmp.data()); f_rhs(tmp.data(), k3.data());
        for (int64_t i = 0; i < n; ++i) tmp[i] = y[i] + (a41 * dt) * k1[i] + (a42 * dt) * k2[i] + (a43 * dt) * k3[i];
        enforce(tmp.data()); f_rhs(tmp.data(), k4.data());
        for (int64_t i = 0; i < n; ++i)
            tmp[i] = y[i] + (a51 * dt) * k1[i] + (a52 * dt) * k2[i] + (a53 * dt) * k3[i] + (a54 * dt) * k4[i];
        enforce(tmp.data()); f_rhs(tmp.data(), k5.data());
        for (int64_t i = 0; i < n; ++i)
            tmp[i] = y[i] + (a61 * dt) * k1[i] + (a62 * dt) * k2[i] + (a63 * dt) * k3[i] + (a64 * dt) * k4[i] +
                     (a65 * dt) * k5[i];
        enforce(tmp.data()); f_rhs(tmp.data(), k6.data());
        for (int64_t i = 0; i < n; ++i)
            y5[i] = y[i] + (dt * b1) * k1[i] + (dt * b3) * k3[i] + (dt * b4) * k4[i] + (dt * b5) * k5[i] +
                    (dt * b6) * k6[i];
        enforce(y5.data());
        f_rhs(y5.data(), k7.data());
        if (st + 1 == n_steps) {
            const double bt1 = -(435. * s * s * s - 1184. * s * s + 1098. * s - 384.) / (384.);
            const double bt3 = 500. * s * (6. * s * s - 14. * s + 9.) / (1113.);
            const double bt4 = -125. * s * (9. * s * s - 16. * s + 6.) / (192.);
            const double bt5 = 729. * s * (35. * s * s - 64. * s + 26.) / (6784.);
            const double bt6 = -11. * s * (3. * s - 2.) * (5. * s - 6.) / (84.);
            const double bt7 = s * (s - 1.) * (5. * s - 3.) / (2.);
            for (int64_t i = 0; i < n; ++i)
                out[i] = y[i] + (s * dt * bt1) * k1[i] + (s * dt * bt3) * k3[i] + (s * dt * bt4) * k4[i] +
                         (s * dt * bt5) * k5[i] + (s * dt * bt6) * k6[i] + (s * dt * bt7) * k7[i];
            enforce(out);
        }
        y.swap(y5);
        k1.swap(k7);
    }
}

static int dp54(const Problem& P, double* y_io, double t0, double tf, double dense, double* dense_out,
                double* dense_t, int max_dense, int* n_dense, int nthreads, bool drift, int64_t max_attempts,
                DPStats& st) {
    return dp54_core(
        P.ndofs, y_io, t0, tf, dense, dense_out, dense_t, max_dense, n_dense, max_attempts, st,
        [&](const double* in, double* out) { rhs(P, in, out, nthreads, drift); },
        [&](double t, double* v) { apply_constraints_at(P, t, v); },
        [&](const double* err, const double* y5) { return relative_error(P, err, y5); },
        [&](const double* times) { return veto_step(P, times, 6, dense); });
}

// ------------------------------------------------------------ construction
static Problem build(const tb_problem_desc* d, bool enumerate_tuples, int nthreads) {
    Problem P;
    P.region = d->region;
    for (int i = 0; i < d->n_meshes; ++i) P.meshes.push_back(make_mesh(d->region, d->meshes[i]));
    int64_t off = 0;
    for (int b = 0; b < d->n_bands; ++b) {
        const tb_band_desc& bd = d->bands[b];
        if (bd.mesh < 0 || bd.mesh >= d->n_meshes) throw std::runtime_error("band mesh index out of range");
        const Mesh& m = P.meshes[bd.mesh];
        Band B;
        B.mesh = bd.mesh;
        B.charge = bd.charge;
        B.statistics = bd.statistics;
        B.disp.assign(bd.dispersion, bd.dispersion + size_t(m.ne) * 3);
        B.kx = function_from(m, [](const double* p) { return p[0]; });
        B.ky = function_from(m, [](const double* p) { return p[1]; });
        B.minE.resize(m.ne);
        B.maxE.resize(m.ne);
        for (int e = 0; e < m.ne; ++e) {  // Band.cpp:58-64 / Function.cpp:308-336
            double n[3];
            to_nodal(&B.disp[3 * e], n);
            B.minE[e] = std::min(n[0], std::min(n[1], n[2]));
            B.maxE[e] = std::max(n[0], std::max(n[1], n[2]));
        }
        B.abs_tol = bd.abs_tol;
        B.rel_tol = bd.rel_tol;
        B.penal = bd.penalisation;
        B.constrained = bd.constrained != 0;
        if (B.constrained) {
            if (!bd.constrained_population) throw std::runtime_error("constrained band without population");
            B.cpop.assign(bd.constrained_population, bd.constrained_population + size_t(m.ne) * 3);
        }
        B.vel[0] = bd.drift_velocity[0];
        B.vel[1] = bd.drift_velocity[1];
        P.bands.push_back(std::move(B));
        P.off.push_back(off);
        off += int64_t(m.ne) * 3;
    }
    P.ndofs = off;
    for (int ci = 0; ci < d->n_channels; ++ci) {
        const tb_channel_desc& cd = d->channels[ci];
        Channel c;
        c.L = cd.nlegs;
        if (c.L < 2 || c.L > 4) throw std::runtime_error("nlegs must be 2..4");
        for (int l = 0; l < c.L; ++l) {
            c.band[l] = cd.band[l];
            c.dir[l] = cd.dir[l];
            if (c.band[l] < 0 || c.band[l] >= d->n_bands) throw std::runtime_error("leg band out of range");
        }
        c.amplitude = cd.amplitude;
        c.nmc = cd.n_mc;
        c.min_det = cd.min_det;
        c.threshold = cd.threshold;
        c.umk.assign(cd.umklapp, cd.umklapp + 2 * size_t(cd.n_umklapp));
        const int R = 2 * (c.L - 2) + 1;
        c.mc.assign(cd.mc_points, cd.mc_points + size_t(c.nmc) * R);
        const double* pre = cd.mc_points_precalc ? cd.mc_points_precalc : cd.mc_points;
        c.mc_pre.assign(pre, pre + size_t(c.nmc) * R);
        if (cd.n_tuples > 0) {
            c.tuples.assign(cd.tuples, cd.tuples + size_t(cd.n_tuples) * c.L);
            c.tumk.assign(cd.tuple_umklapp, cd.tuple_umklapp + size_t(cd.n_tuples));
        } else if (enumerate_tuples) {
            enumerate(P, c, nthreads);
        }
        P.chans.push_back(std::move(c));
    }
    return P;
}

}  // namespace oracle

// ======================================================================= C API
using namespace oracle;

static thread_local std::string g_err;

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

void* or_create(const tb_problem_desc* desc, int enumerate_tuples, int nthreads) {
    try {
        return new Problem(build(desc, enumerate_tuples != 0, nthreads));
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return nullptr;
    }
}

void or_destroy(void* h) { delete static_cast<Problem*>(h); }

int64_t or_num_dofs(void* h) { return static_cast<Problem*>(h)->ndofs; }

int64_t or_band_offset(void* h, int b) { return static_cast<Problem*>(h)->off[b]; }

int64_t or_num_tuples(void* h, int ch) { return int64_t(static_cast<Problem*>(h)->chans[ch].tumk.size()); }

void or_enum_counts(void* h, int ch, int64_t* prefilter, int64_t* det_ok) {
    const Channel& c = static_cast<Problem*>(h)->chans[ch];
    *prefilter = c.n_prefilter;
    *det_ok = c.n_det;
}

void or_get_tuples(void* h, int ch, int32_t* ids, int32_t* umk) {
    const Channel& c = static_cast<Problem*>(h)->chans[ch];
    std::copy(c.tuples.begin(), c.tuples.end(), ids);
    std::copy(c.tumk.begin(), c.tumk.end(), umk);
}

// Replace a channel's tuple list (fixtures, sharding tests).
void or_set_tuples(void* h, int ch, int64_t n, const int32_t* ids, const int32_t* umk) {
    Channel& c = static_cast<Problem*>(h)->chans[ch];
    c.tuples.assign(ids, ids + size_t(n) * c.L);
    c.tumk.assign(umk, umk + size_t(n));
    static_cast<Problem*>(h)->chans[size_t(ch)].tamp.clear();   // the factors follow the list
}

// Channel ch's tuple list becomes the tuples of work items [item0, item1)
// (enumerate_items), over nthreads contiguous item ranges concatenated in
// order; the prefilter and determinant counts are those of the range.
void or_enumerate_items(void* h, int ch, int64_t item0, int64_t item1, int nthreads) {
    Problem& P = *static_cast<Problem*>(h);
    Channel& c = P.chans[size_t(ch)];
    nthreads = int(std::max<int64_t>(1, std::min<int64_t>(nthreads, item1 - item0)));
    std::vector<EnumPart> parts(static_cast<size_t>(nthreads));
    std::vector<std::thread> th;
    auto work = [&](int t) {
        const int64_t a = item0 + (item1 - item0) * t / nthreads, b = item0 + (item1 - item0) * (t + 1) / nthreads;
        enumerate_items(P, c, a, b, parts[size_t(t)]);
    };
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    c.tuples.clear();
    c.tumk.clear();
    c.tamp.clear();
    c.n_prefilter = 0;
    c.n_det = 0;
    for (auto& q : parts) {
        c.tuples.insert(c.tuples.end(), q.tuples.begin(), q.tuples.end());
        c.tumk.insert(c.tumk.end(), q.tumk.begin(), q.tumk.end());
        c.n_prefilter += q.n_pre;
        c.n_det += q.n_det;
    }
}

void or_set_amplitude(void* h, int ch, double a) { static_cast<Problem*>(h)->chans[ch].amplitude = a; }

// ScatteringChannel::propagate restricted to tuples [t0,t1) (out += ...).
// Tuples of a channel's list with at least one Monte-Carlo point whose
// ThetapC * ThetaFC is 1 (IntegratorCore.hpp:318-320) and the number of such
// (tuple, point) pairs: the terms of TypeB that are not the integrand times 0.
// per_tuple (optional, one int32 per tuple of the list): that tuple's count.
void or_points_inside(void* h, int ch, int64_t* n_tuples, int64_t* n_points, int32_t* per_tuple) {
    const Problem& P = *static_cast<Problem*>(h);
    const Channel& c = P.chans[ch];
    const int L = c.L, R = 2 * (L - 2) + 1;
    int64_t nt = 0, np = 0;
    for (size_t i = 0; i < c.tumk.size(); ++i) {
        if (per_tuple) per_tuple[i] = 0;
        Geom g;
        build_geom(P, c, &c.tuples[i * size_t(L)], c.tumk[i], g);
        if (std::fabs(g.det) < c.min_det) continue;
        double DCinv[3][3];
        inv3(g.DC, DCinv);
        MCPoint mp;
        int64_t k = 0;
        for (int m = 0; m < c.nmc; ++m) {
            mc_point(L, g, DCinv, &c.mc[size_t(m) * R], mp);
            k += mp.theta ? 1 : 0;
        }
        nt += k > 0 ? 1 : 0;
        np += k;
        if (per_tuple) per_tuple[i] = int32_t(k);
    }
    *n_tuples = nt;
    *n_points = np;
}

void or_channel_propagate(void* h, int ch, const double* f, double* out, int64_t t0, int64_t t1, int nthreads,
                          int inverse_mass) {
    Problem& P = *static_cast<Problem*>(h);
    const Channel& c = P.chans[ch];
    if (t1 < 0 || t1 > int64_t(c.tumk.size())) t1 = int64_t(c.tumk.size());
    channel_propagate_range(P, c, f, out, t0, t1, nthreads, inverse_mass != 0);
}

void or_rhs(void* h, const double* f, double* out, int nthreads, int drift) {
    rhs(*static_cast<Problem*>(h), f, out, nthreads, drift != 0);
}

void or_vlasov(void* h, int band, const double* fband, double* out) {
    Problem& P = *static_cast<Problem*>(h);
    const Band& b = P.bands[band];
    vlasov_flux(P.meshes[b.mesh], fband, b.vel, out);
}

double or_relative_error(void* h, const double* err, const double* pop) {
    return relative_error(*static_cast<Problem*>(h), err, pop);
}

double or_band_relative_error(void* h, int band, const double* err, const double* pop) {
    Problem& P = *static_cast<Problem*>(h);
    const Band& b = P.bands[band];
    return band_relative_error(P.meshes[b.mesh], b, err, pop);
}

double or_integrate(void* h, int band, const double* a, const double* b) {
    Problem& P = *static_cast<Problem*>(h);
    return integrate2(P.meshes[P.bands[band].mesh], a, b);
}

void or_apply_inverse_mass(void* h, int band, double* v) {
    Problem& P = *static_cast<Problem*>(h);
    apply_inverse_mass(P.meshes[P.bands[band].mesh], v);
}

void or_mass_matrix(void* h, int mesh, double* M, double* Minv) {
    const Mesh& m = static_cast<Problem*>(h)->meshes[mesh];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { M[3 * i + j] = m.M[i][j]; Minv[3 * i + j] = m.Minv[i][j]; }
}

void or_apply_constraints(void* h, double* f) { apply_constraints(*static_cast<Problem*>(h), f); }

// Time-dependent constrained populations for every constrained band (null:
// back to the time-independent ones).
void or_set_constraint_fn(void* h, or_constraint_fn fn, void* user) {
    Problem& P = *static_cast<Problem*>(h);
    P.cfn = fn;
    P.cuser = user;
}

int or_apply_constraints_at(void* h, double* f, double t) {
    try {
        apply_constraints_at(*static_cast<Problem*>(h), t, f);
    } catch (const std::exception& e) {
        g_err = e.what();
        return TB_ERR_ARG;
    }
    return TB_OK;
}

// ScatteringChannel::functAmplitude at the element barycentres of every tuple
// of channel ch (constructAmplitude, ScatteringChannel.cpp:399-415; Mesh<2>::
// elemCentre, Mesh.cpp:533-535 through Mesh<2>::operator(), Mesh.cpp:503-509),
// computed for the channel's current tuple list; fn = null: 1.
typedef int (*or_amplitude_fn)(void* user, int64_t n, int32_t nlegs, const double* barycentres, double* out);
int or_set_channel_amplitude_fn(void* h, int ch, or_amplitude_fn fn, void* user) {
    Problem& P = *static_cast<Problem*>(h);
    Channel& c = P.chans[size_t(ch)];
    c.tamp.clear();
    if (!fn) return TB_OK;
    const int64_t n = int64_t(c.tumk.size());
    std::vector<double> bary(size_t(n) * c.L * 2);
    const double r = 0.333333333;
    for (int64_t i = 0; i < n; ++i)
        for (int l = 0; l < c.L; ++l) {
            const Mesh& m = P.meshes[P.bands[c.band[l]].mesh];
            const int e = c.tuples[size_t(i) * c.L + l];
            const int sec = e / 2, par = e % 2;
            const double sx = double(sec % m.nx), sy = double(sec / m.nx);
            const double px = sx + (kVert[par][1][0] * r + kVert[par][2][0] * r);
            const double py = sy + (kVert[par][1][1] * r + kVert[par][2][1] * r);
            double* o = &bary[(size_t(i) * c.L + l) * 2];
            o[0] = m.origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
            o[1] = m.origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
        }
    c.tamp.resize(size_t(n));
    if (n > 0 && fn(user, n, c.L, bary.data(), c.tamp.data()) != 0) {
        c.tamp.clear();
        g_err = "amplitude callback failed";
        return TB_ERR_ARG;
    }
    return TB_OK;
}

// The time-step veto of MaterialTimeStatus::timeStepVetoer for the six stage
// times of a step of size dt from t (a check of the restatement).
double or_veto_step(void* h, double t, double dt, double dense) {
    const double c2 = 1. / 5., c3 = 3. / 10., c4 = 4. / 5., c5 = 8. / 9.;
    const double times[6] = {t, t + c2 * dt, t + c3 * dt, t + c4 * dt, t + c5 * dt, t + dt};
    return veto_step(*static_cast<Problem*>(h), times, 6, dense);
}

// The order-2 Gauss rules the oracle integrates with (kGP2 / kGW2 on the
// reference triangle, kGP1 on [0, 1]): points as (x, y) pairs, weights.
void or_gauss_constants(double* tri_points, double* tri_weights, double* int_points) {
    for (int q = 0; q < 3; ++q) {
        tri_points[2 * q] = kGP2[q][0];
        tri_points[2 * q + 1] = kGP2[q][1];
        tri_weights[q] = kGW2[q];
    }
    int_points[0] = kGP1[0];
    int_points[1] = kGP1[1];
}

// MaterialTimeStatus::timeStepVetoer(timesToTest, denseStep)
// (MaterialTimeStatus.cpp:60-100) on the caller's times.
double or_veto_times(void* h, const double* times, int ntimes, double dense) {
    try {
        return veto_step(*static_cast<Problem*>(h), times, ntimes, dense);
    } catch (const std::exception& e) {
        g_err = e.what();
        return NAN;
    }
}

// stats: [attempts, accepted, rejected, rhs_evals] and dstats: [t, dt, last_err]
int or_dp45(void* h, double* y, double t0, double tf, double dense, double* dense_out, double* dense_t,
            int max_dense, int* n_dense, int nthreads, int drift, int64_t max_attempts, int64_t* stats,
            double* dstats) {
    DPStats st;
    int rc;
    try {
        rc = dp54(*static_cast<Problem*>(h), y, t0, tf, dense, dense_out, dense_t, max_dense, n_dense, nthreads,
                  drift != 0, max_attempts, st);
    } catch (const std::exception& e) {
        g_err = e.what();
        return TB_ERR_ARG;
    }
    stats[0] = st.attempts; stats[1] = st.accepted; stats[2] = st.rejected; stats[3] = st.rhs_evals;
    dstats[0] = st.t; dstats[1] = st.dt; dstats[2] = st.last_err;
    return rc;
}

// ScatteringChannel::scatteringRates(status, which) (ScatteringChannel.cpp:582-603)
// summed over the legs of one channel (ch >= 0, which < 0), one leg (which >=
// 0) or, with ch < 0, every channel with a nonzero amplitude and every leg
// (MaterialStatus::scatteringRates, MaterialStatus.cpp:170-187).  Each leg's
// rate lands in its own band; out (the whole state) is overwritten, M^-1
// applied.
void or_scattering_rates(void* h, int ch, int which, const double* f, double* out, int nthreads) {
    const Problem& P = *static_cast<Problem*>(h);
    std::fill(out, out + P.ndofs, 0.0);
    for (size_t ci = 0; ci < P.chans.size(); ++ci) {
        const Channel& c = P.chans[ci];
        if (ch >= 0 && int(ci) != ch) continue;
        if (ch < 0 && c.amplitude == 0.0) continue;
        for (int l = 0; l < c.L; ++l) {
            if (which >= 0 && l != which) continue;
            channel_propagate_range(P, c, f, out, 0, int64_t(c.tumk.size()), nthreads, true, l);
        }
    }
}

void or_dp45_replay(void* h, const double* y0, const double* dts, int64_t n_steps, double dense_s, double* out,
                    int nthreads, int drift) {
    const Problem& P = *static_cast<Problem*>(h);
    dp54_replay_core(
        P.ndofs, y0, dts, n_steps, dense_s, out,
        [&](const double* in, double* o) { rhs(P, in, o, nthreads, drift != 0); },
        [&](double* v) { apply_constraints(P, v); });
}

// The scalar example of the reference's DP54 documentation
// (DormandPrince54.hpp:80-106): y' = cos(t) through a time-dependent timeOp,
// error form 1e13*err^2.  timeOp is the only time-dependent piece, so the stage
// times c_i are threaded through a small wrapper.
int or_dp45_scalar_example(double t0, double y0, double tf, double dense, double* dense_out, double* dense_t,
                           int max_dense, int* n_dense, int64_t* stats) {
    DPStats st;
    double y = y0;
    // stage times: the integrator evaluates timeOp at t + c_i dt; the
    // autonomous core does not carry time, so the state is augmented with t.
    double ya[2] = {y0, t0};
    std::vector<double> dense2(size_t(max_dense) * 2);
    int rc = dp54_core(
        2, ya, t0, tf, dense, dense2.data(), dense_t, max_dense, n_dense, 0, st,
        [&](const double* in, double* out) { out[0] = std::cos(in[1]); out[1] = 1.0; },
        [&](double, double*) {},
        [&](const double* err, const double*) { return 10000000000000. * err[0] * err[0]; },
        [&](const double* times) { return times[5] - times[0]; });
    for (int i = 0; i < std::min(*n_dense, max_dense); ++i) dense_out[i] = dense2[2 * size_t(i)];
    stats[0] = st.attempts; stats[1] = st.accepted; stats[2] = st.rejected; stats[3] = st.rhs_evals;
    (void)y;
    return rc;
}

}  // extern "C"
