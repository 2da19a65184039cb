// tb_stream.cu -- the Monte-Carlo collision operator with its tuples
// enumerated on the fly, for channels whose tuple list does not fit in
// device memory (four-leg electron-electron channels on fine meshes: about
// 2e9 surviving tuples at 32x32, 3e10 at 64x64).
//
// Every evaluation walks the reference's candidate space again and keeps
// nothing between evaluations:
//   * work items (umklapp, sections of legs 0..L-2, element choice in those
//     sections) and, per item, the element box of the last leg: the nested
//     loops of nestedForSections / nestedForElements (include/Physics/
//     Scattering/ScatteringChannel.hpp:205-255) with the TrapezoidalSubset
//     box arithmetic (src/Geometry/Structured/DirectSpace/MeshSubset.cpp);
//   * the energy window, the determinant filter and the survival test of
//     precalculateIndices (src/Physics/Scattering/ScatteringChannel.cpp:
//     476-504) on the survival table;
//   * for the survivors, which points of the quadrature table lie inside the
//     simplices, and TypeB's sums over those points only
//     (include/Physics/Scattering/IntegratorCore.hpp:260-357).
// Every decision uses the same explicitly rounded operations as the stored
// enumeration (k_enumerate, compiled unfused) and the mask builder
// (k_theta_mask), and the sums use the stored-list kernel's code
// (tb_mcpoint.cuh), so a streamed evaluation adds the same per-tuple values
// as the stored-list path.
//
// Work distribution: a warp walks runs of consecutive work items, 32 at a
// time (one per lane); the lanes step through their boxes in lock step and
// push the candidates that pass the energy window into a per-warp queue in
// shared memory.  Three stages drain the queues, each on 32 entries at a
// time, one per lane: determinant filter and domain test (queue 0 -> 1), the
// survival test (queue 1 -> 2), then the points inside, the sums and the
// scatter for the surviving tuples.  So every stage runs on full warps
// whatever the box sizes and the pass rate of the stage before.
#include "tb_dp45.cuh"
#include "tb_mcpoint.cuh"
#include "tb_scatter.cuh"
#include "tb_stream.cuh"

namespace tb {

// 4 warps per block, 3 blocks per SM: the register cap of 168 per thread
// spills a little, but 12 resident warps per SM instead of 8 hide more of the
// FP64 latency (a 16x16 e-e evaluation: 306 ms against 387 ms with blocks of
// 8 warps at 221 registers, one block per SM)
constexpr int ST_WARPS = 4;    // warps per block
constexpr int ST_QUEUE = 64;   // candidate slots per warp (31 left over + 32 pushed at most)
constexpr int ST_SPAN = 16;    // steps of 32 consecutive items per run of a warp

struct WBox {
    double l[2], h[2];
};

// One section's box, shrunk by 1e-8 section units (MeshSubset.cpp:62-66),
// in absolute coordinates.
__device__ __forceinline__ WBox walk_section_box(const WalkLeg& m, int sx, int sy) {
    WBox b;
    const double lo0 = xa(double(sx), 0.00000001), lo1 = xa(double(sy), 0.00000001);
    const double hi0 = xs(double(sx + 1), 0.00000001), hi1 = xs(double(sy + 1), 0.00000001);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        b.l[i] = xa(m.origin[i], xa(xm(m.dG[i][0], lo0), xm(m.dG[i][1], lo1)));
        b.h[i] = xa(m.origin[i], xa(xm(m.dG[i][0], hi0), xm(m.dG[i][1], hi1)));
    }
    return b;
}

__device__ __forceinline__ WBox walk_box_scale(WBox b, double s) {
    if (s >= 0.0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) { b.l[i] = xm(b.l[i], s); b.h[i] = xm(b.h[i], s); }
    } else {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const double t = b.l[i];
            b.l[i] = xm(b.h[i], s);
            b.h[i] = xm(t, s);
        }
    }
    return b;
}

// A lane's place in the work-item numbering, as digits (least significant
// first): the element choice, then for legs L-2 .. 0 the section's x and y,
// then the umklapp column.  A warp walks runs of consecutive items, so most
// steps change the last digits only: the box sums of the legs in front
// (legs 0..L-3) and their energies are kept from the previous item.
template <int L>
struct WalkPos {
    int comb, u;
    int sx[TB_MAX_LEGS], sy[TB_MAX_LEGS];
};

template <int L>
__device__ __forceinline__ void walk_decode(const StreamDev& sd, int64_t item, WalkPos<L>& p) {
    constexpr int C = 1 << (L - 1);
    p.comb = int(item % C);
    int64_t r = item / C;
#pragma unroll
    for (int l = L - 2; l >= 0; --l) {
        const int sec = int(r % sd.nsec[l]);
        r /= sd.nsec[l];
        p.sx[l] = sec % sd.leg[l].nx;
        p.sy[l] = sec / sd.leg[l].nx;
    }
    p.u = int(r);
}

// p += 32 items.  Returns true when a digit of legs 0..L-3 or the umklapp
// column changed (the kept box sums are stale).
template <int L>
__device__ __forceinline__ bool walk_advance(const StreamDev& sd, WalkPos<L>& p) {
    constexpr int C = 1 << (L - 1);
    int carry = 32 / C;
    bool front = false;
#pragma unroll
    for (int l = L - 2; l >= 0; --l) {
        if (carry) {
            if (l < L - 2) front = true;
            int x = p.sx[l] + carry;
            carry = 0;
            if (x >= sd.leg[l].nx) { carry = x / sd.leg[l].nx; x -= carry * sd.leg[l].nx; }
            int y = p.sy[l] + carry;
            carry = 0;
            if (y >= sd.leg[l].ny) { carry = y / sd.leg[l].ny; y -= carry * sd.leg[l].ny; }
            p.sx[l] = x;
            p.sy[l] = y;
        }
    }
    if (carry) { p.u += carry; front = true; }
    return front;
}

// What the legs in front contribute to an item: their box sum (legs 0..L-3),
// the umklapp shift and the energy-window partial sums of legs 0..L-3.
struct WalkFront {
    WBox box;
    double gu[2];
    double mn, mx;
};

// The item at p: elements of legs 0..L-2, the last leg's section range
// [lo, hi) and the energy-window sums of legs 0..L-2 (pmn, pmx; the last
// leg's term is added per candidate).  The decoding and box arithmetic of
// k_enumerate, term for term and in the same order (the kept front sums are
// its partial sums); fr is refreshed when ok is false.
template <int L>
__device__ __forceinline__ void walk_at(const ChanDev& c, const StreamDev& sd, const WalkPos<L>& p, WalkFront& fr,
                                        bool& ok, int (&e)[L], int (&lo)[2], int (&hi)[2], double& pmn,
                                        double& pmx) {
#pragma unroll
    for (int l = 0; l < L - 1; ++l) e[l] = 2 * (p.sy[l] * sd.leg[l].nx + p.sx[l]) + ((p.comb >> (L - 2 - l)) & 1);
    if (!ok) {
        const double ux = c.umk[2 * p.u], uy = c.umk[2 * p.u + 1];
        fr.gu[0] = xa(xm(c.gvec[0], ux), xm(c.gvec[2], uy));
        fr.gu[1] = xa(xm(c.gvec[1], ux), xm(c.gvec[3], uy));
        fr.mn = 0.0;
        fr.mx = 0.0;
#pragma unroll
        for (int l = 0; l < L - 2; ++l) {
            const WBox b = walk_box_scale(walk_section_box(sd.leg[l], p.sx[l], p.sy[l]), c.leg[l].dir);
            if (l == 0) fr.box = b;
            else {
#pragma unroll
                for (int i = 0; i < 2; ++i) { fr.box.l[i] = xa(fr.box.l[i], b.l[i]); fr.box.h[i] = xa(fr.box.h[i], b.h[i]); }
            }
            const double emin = __ldg(sd.leg[l].minE + e[l]), emax = __ldg(sd.leg[l].maxE + e[l]);
            fr.mn += (c.leg[l].dir > 0) ? emin : -emax;
            fr.mx += (c.leg[l].dir > 0) ? emax : -emin;
        }
        ok = true;
    }
    constexpr int K = L - 2;   // the leg whose section changes from item to item
    WBox acc = walk_box_scale(walk_section_box(sd.leg[K], p.sx[K], p.sy[K]), c.leg[K].dir);
    if (K > 0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) { acc.l[i] = xa(fr.box.l[i], acc.l[i]); acc.h[i] = xa(fr.box.h[i], acc.h[i]); }
    }
    acc.l[0] = xa(acc.l[0], fr.gu[0]); acc.h[0] = xa(acc.h[0], fr.gu[0]);
    acc.l[1] = xa(acc.l[1], fr.gu[1]); acc.h[1] = xa(acc.h[1], fr.gu[1]);
    acc = walk_box_scale(acc, -c.leg[L - 1].dir);
    const WalkLeg& ml = sd.leg[L - 1];
    const int ns[2] = {ml.nx, ml.ny};
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const double tl = xa(xm(ml.invdG[i][0], xs(acc.l[0], ml.origin[0])), xm(ml.invdG[i][1], xs(acc.l[1], ml.origin[1])));
        const double th = xa(xm(ml.invdG[i][0], xs(acc.h[0], ml.origin[0])), xm(ml.invdG[i][1], xs(acc.h[1], ml.origin[1])));
        const int aa = int(floor(tl));
        const int bb = int(xa(floor(th), 1.0));
        lo[i] = min(max(aa, 0), ns[i]);
        hi[i] = min(max(bb, 0), ns[i]);
    }
    pmn = fr.mn;
    pmx = fr.mx;
    if (lo[0] != hi[0] && lo[1] != hi[1]) {
        const double emin = __ldg(sd.leg[K].minE + e[K]), emax = __ldg(sd.leg[K].maxE + e[K]);
        pmn += (c.leg[K].dir > 0) ? emin : -emax;
        pmx += (c.leg[K].dir > 0) ? emax : -emin;
    }
}

// True when no point of the Monte-Carlo domain -- every free leg's point in
// its reference triangle, the partially constrained leg's coordinate in
// [0, 1] -- can pass the simplex tests ThetapC * ThetaFC
// (IntegratorCore.hpp:318-320), whatever the order the constrained
// coordinates are evaluated in: over the whole domain one of al0, al1, al2
// stays below 0, or kp0 + al0 or al1 + al2 stays above 1, by more than four
// times the rounding bound am.mg (which already covers the distance between
// the fused map and the reference-order evaluation).  Then neither table has
// a point inside: the survival sum is 0 and the tuple does not survive.
template <int L>
__device__ __forceinline__ bool domain_excludes(const AlphaMap<L>& am) {
    constexpr int R = AlphaMap<L>::R;
    const double eps = 2.220446049250313e-16;
    double hi[3];
    double plo = am.a0[0];                 // min of kp0 + al0
    double slo = am.a0[1] + am.a0[2];      // min of al1 + al2
#pragma unroll
    for (int r = 0; r < 3; ++r) hi[r] = am.a0[r];
#pragma unroll
    for (int b = 0; b < L - 2; ++b) {      // free legs: vertices (0,0), (1,0), (0,1)
#pragma unroll
        for (int r = 0; r < 3; ++r) hi[r] += fmax(0.0, fmax(am.G[r][2 * b], am.G[r][2 * b + 1]));
        plo += fmin(0.0, fmin(am.G[0][2 * b], am.G[0][2 * b + 1]));
        slo += fmin(0.0, fmin(am.G[1][2 * b] + am.G[2][2 * b], am.G[1][2 * b + 1] + am.G[2][2 * b + 1]));
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) hi[r] += fmax(0.0, am.G[r][R - 1]);   // kp0 in [0, 1]
    plo += fmin(0.0, am.G[0][R - 1] + 1.0);
    slo += fmin(0.0, am.G[1][R - 1] + am.G[2][R - 1]);
    const double m0 = 4.0 * am.mg[0], m1 = 4.0 * am.mg[1], m2 = 4.0 * am.mg[2];
    if (hi[0] < -m0 || hi[1] < -m1 || hi[2] < -m2) return true;
    if (plo - m0 > 1.0 + 8.0 * eps * (1.0 + fabs(plo))) return true;
    if (slo - (m1 + m2) > 1.0 + 8.0 * eps * (1.0 + fabs(slo))) return true;
    return false;
}

// Per-tuple thresholds of a cheaper "clearly outside" test than
// theta_decide's: T[0] for kp0 + al0, T[1] for al1 + al2.  Over the whole
// Monte-Carlo domain (every coordinate of q in [0, 1]) the fused
// coordinates obey |al_r| <= B_r = |a0_r| + sum_j |G_rj| (up to a factor
// 1 + 1e-15, covered by the 1.000001 below), so theta_decide's per-point
// bounds mg0 + tiny (2 + |al0|) and mg1 + mg2 + tiny (1 + |al1| + |al2|) are
// at most X = mg0 + tiny (2 + B0) and Y = mg1 + mg2 + tiny (1 + B1 + B2).
// A point with fl(kp0 + al0) > fl(1 + 4 X) has fl(fl(kp0 + al0) - 1) > 3.8 X
// (X >= 2 tiny, so the roundings of 1 + 4 X and of the difference cost less
// than 0.2 X), above theta_decide's computed bound: theta_decide also calls
// it outside.  Likewise for al1 + al2 against fl(1 + 4 Y).  The faster test
// therefore only sends a few more points to the exact evaluation, and every
// decision stays the reference-order one.
template <int L>
__device__ __forceinline__ void outside_thresholds(const AlphaMap<L>& am, double (&T)[2]) {
    constexpr int R = AlphaMap<L>::R;
    const double tiny = 8.0 * 1.1102230246251565e-16;
    double B[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double t = fabs(am.a0[r]);
#pragma unroll
        for (int j = 0; j < R; ++j) t += fabs(am.G[r][j]);
        B[r] = 1.000001 * t;
    }
    const double X = am.mg[0] + tiny * (2.0 + B[0]);
    const double Y = (am.mg[1] + am.mg[2]) + tiny * ((1.0 + B[1]) + B[2]);
    T[0] = 1.0 + 4.0 * X;
    T[1] = 1.0 + 4.0 * Y;
}

// theta_decide with the per-tuple thresholds above: the same decision.
template <int L>
__device__ __forceinline__ bool theta_decide_t(const TupleGeom<L>& g, const double (&Ci)[3][3], const AlphaMap<L>& am,
                                               const double (&T)[2], const double* qv) {
    constexpr int R = AlphaMap<L>::R;
    double al[3];
    alpha_fast<L>(am, qv, al);
    const double kp0 = qv[R - 1];
    const bool out = (al[0] < -am.mg[0]) || (al[1] < -am.mg[1]) || (al[2] < -am.mg[2]) ||
                     (__dadd_rn(kp0, al[0]) > T[0]) || (__dadd_rn(al[1], al[2]) > T[1]);
    if (out) return false;
    return alpha_theta<L>(g, Ci, am, qv, al);
}

#ifndef TB_STREAM_MIN_BLOCKS
#define TB_STREAM_MIN_BLOCKS 3
#endif

// MODE: ST_PROPAGATE (the collision terms), ST_RATE (rate_leg's scattering
// rate) or ST_VJP (acc = grad_f += the transposed terms for the co-state co,
// grad_amp[k] += <co, dC/d amplitude_k>; the stored-list VJP's arithmetic).
enum { ST_PROPAGATE = 0, ST_RATE = 1, ST_VJP = 2 };

template <int L, int MODE>
__global__ void __launch_bounds__(ST_WARPS * 32, TB_STREAM_MIN_BLOCKS)
    k_collision_stream(ChanDev c, StreamDev sd, int64_t it0, int64_t it1, const InstDev* __restrict__ insts,
                       int n_insts, const double* __restrict__ f, double* __restrict__ acc,
                       const DPCtl* __restrict__ ctl, int rate_leg, FxAcc fx, const double* __restrict__ co,
                       double* __restrict__ grad_amp, FxAcc fx_amp) {
    constexpr bool RATE = MODE == ST_RATE;
    {
        // every instance off or its run finished: nothing to add
        bool any = false;
        for (int k = 0; k < n_insts && !any; ++k)
            any = insts[k].amp_full != 0.0 && !(ctl && ctl[insts[k].run].done);
        if (!any) return;
    }
    constexpr int R = 2 * (L - 2) + 1;
    extern __shared__ double s_tab[];   // [nmc R] quadrature table, then [nmc R] survival table
    // per-warp candidate queues: [0] inside the energy window, [1] past the
    // determinant filter and the domain test, [2] surviving tuples
    __shared__ int32_t s_q[3][ST_WARPS][L + 1][ST_QUEUE];
    double* s_mc = s_tab;
    double* s_pre = s_tab + c.nmc * R;
    for (int i = threadIdx.x; i < c.nmc * R; i += blockDim.x) {
        s_mc[i] = c.mc[i];
        s_pre[i] = sd.mc_pre[i];
    }
    __syncthreads();
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double sqrt2 = 1.4142135623730951;   // sqrt(2.0), correctly rounded
    double prodc = 1.0;
#pragma unroll
    for (int l = 0; l < L; ++l) prodc *= sqrt2;
    // s_cnt[k]: prodc added k times to 0.0, in sequence
    __shared__ double s_cnt[65];
    if (threadIdx.x == 0) {
        double t = 0.0;
        s_cnt[0] = t;
        for (int k = 1; k <= 64; ++k) s_cnt[k] = (t += prodc);
    }
    __syncthreads();
    const double inv_fact_nmc = c.fact * double(c.nmc);
    unsigned long long n_pre = 0, n_det = 0, n_surv = 0, n_pts = 0, n_tin = 0;

    int q2n = 0;   // candidates in queue 1 (warp-uniform)
    int q3n = 0;   // surviving tuples in queue 2 (warp-uniform)

    // Stage 1 for `take` candidates of queue 0 from slot `first` on, one per
    // lane: the determinant filter, then the domain test; the candidates that
    // may have a point inside go to queue 1.  Cheap next to stage 2 (about
    // 150 operations against 2 x NMC simplex tests), and most candidates of
    // the energy window end here.
    auto stage1 = [&](int first, int take) {
        const bool valid = lane < take;
        int e[L];
        int u = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = valid ? s_q[0][warp][l][first + lane] : 0;
        if (valid) u = s_q[0][warp][L][first + lane];
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, u, g);
        bool ok = valid && (fabs(g.det) >= c.min_det);
        n_pre += valid ? 1 : 0;
        n_det += ok ? 1 : 0;
        if (ok && c.threshold >= 0.0) {
            double Ci[3][3];
            dc_inverse<L>(g, Ci);
            AlphaMap<L> am;
            alpha_map<L>(g, Ci, am);
            ok = !domain_excludes<L>(am);
        }
        const unsigned bal = __ballot_sync(full, ok);
        if (ok) {
            const int pos = q2n + __popc(bal & ((1u << lane) - 1u));
#pragma unroll
            for (int l = 0; l <= L; ++l) s_q[1][warp][l][pos] = l < L ? e[l] : u;
        }
        q2n += __popc(bal);
        __syncwarp();
    };

    // Stage 2 for `take` candidates of queue 1 from slot `first` on, one per
    // lane: the survival test; the surviving tuples go to queue 2.
    auto survive = [&](int first, int take) {
        const bool valid = lane < take;
        int e[L];
        int u = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = valid ? s_q[1][warp][l][first + lane] : 0;
        if (valid) u = s_q[1][warp][L][first + lane];
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, u, g);
        const double adet = fabs(g.det);
        bool ok = valid && (adet >= c.min_det);
        double Ci[3][3];
        dc_inverse<L>(g, Ci);
        AlphaMap<L> am;
        alpha_map<L>(g, Ci, am);
        // survival test of precalculateIndices on the survival table: the
        // count of k_enumerate's, with each point's simplex decision taken
        // the way k_theta_mask takes it (the fused map, re-evaluated in the
        // reference's order near a face: the same decisions, at a fraction of
        // the cost of evaluating every point in that order)
        // (the reference adds prodc for every point inside: the sum of cnt
        // such terms is s_cnt[cnt], the same additions in the same order)
        double T[2];
        outside_thresholds<L>(am, T);
        int cnt = 0;
        for (int m = 0; m < c.nmc; ++m) cnt += theta_decide_t<L>(g, Ci, am, T, s_pre + m * R) ? 1 : 0;
        double res = (1.0 / (c.fact * double(c.nmc) * adet)) * s_cnt[cnt];
        res *= c.amp_vol;
        ok = ok && (fabs(res) > c.threshold);
        n_surv += ok ? 1 : 0;
        const unsigned bal = __ballot_sync(full, ok);
        if (ok) {
            const int pos = q3n + __popc(bal & ((1u << lane) - 1u));
#pragma unroll
            for (int l = 0; l <= L; ++l) s_q[2][warp][l][pos] = l < L ? e[l] : u;
        }
        q3n += __popc(bal);
        __syncwarp();
    };

    // Stage 3 for `take` surviving tuples of queue 2 from slot `first` on,
    // one per lane: the points inside, the sums, the scatter.  (The survivors
    // are a fifth of the candidates that reach stage 2; gathered into full
    // warps, the quadrature runs on every lane.)
    auto evaluate = [&](int first, int take) {
        const bool valid = lane < take;
        int e[L];
        int u = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) e[l] = valid ? s_q[2][warp][l][first + lane] : 0;
        if (valid) u = s_q[2][warp][L][first + lane];
        TupleGeom<L> g;
        tuple_geometry<L>(c, e, u, g);
        const double adet = fabs(g.det);
        double Ci[3][3];
        dc_inverse<L>(g, Ci);
        AlphaMap<L> am;
        alpha_map<L>(g, Ci, am);
        // the points inside the simplices on the quadrature table (k_theta_mask's)
        uint64_t mk = 0;
        if (valid) {
            double T[2];
            outside_thresholds<L>(am, T);
            for (int m = 0; m < c.nmc; ++m)
                if (theta_decide_t<L>(g, Ci, am, T, s_mc + m * R)) mk |= 1ull << m;
        }
        n_pts += __popcll(mk);
        n_tin += mk ? 1 : 0;
        if (!__any_sync(full, mk != 0ull)) return;
        const bool live = mk != 0ull;
        if (MODE == ST_VJP) {
            // k_vjp_mc's terms for the tuples of the list (tf = 1: no functAmplitude)
            const double scale = live ? 1.0 / (c.fact * double(c.nmc) * fabs(g.det)) : 0.0;
            for (int k = 0; k < n_insts; ++k) {
                const InstDev in = insts[k];
                double gA[L][3], gB[L][3], gamp, sa[L], sb[L];
                vjp_point_sums<L, true>(c, in, f, co, e, g, Ci, s_mc, mk, live, gA, gB, gamp, sa, sb);
                if (live) {
                    const double sc = scale * (in.amp_full * 1.0);
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int64_t key = in.foff[l] + 3 * (int64_t)e[l];
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            const double gv = __dmul_rn(sc, fma(sb[l], gB[l][j], __dmul_rn(sa[l], gA[l][j])));
                            if (fx.w) fx_add(fx, key + j, gv);
                            else atomicAdd(acc + key + j, gv);
                        }
                    }
                }
                block_atomic_sum(live ? scale * (c.amp_vol * 1.0) * gamp : 0.0, grad_amp + k, fx_amp, k);
            }
            return;
        }
        const double scale = live ? 1.0 / (inv_fact_nmc * adet) : 0.0;
        for (int k = 0; k < n_insts; ++k) {
            const InstDev in = insts[k];
            if (in.amp_full == 0.0) continue;
            if (ctl && ctl[in.run].done) continue;
            const double ampt = in.amp_full;
            double s0 = 0.0, sx[L], sy[L];
#pragma unroll
            for (int l = 0; l < L; ++l) { sx[l] = 0.0; sy[l] = 0.0; }
            if (live) {
                double fv[L][3];
                leg_values<L, RATE>(c, in, f, e, rate_leg, fv);
                inside_point_sums<L, RATE>(c, am, s_mc, mk, fv, rate_leg, s0, sx, sy);
            }
#pragma unroll
            for (int l = 0; l < L; ++l) {
                if (RATE && l != rate_leg) continue;   // uniform: the rate keeps one leg
                const double d = RATE ? -c.leg[l].dir : c.leg[l].dir;
                const int64_t key = in.foff[l] + 3 * (int64_t)e[l];
                const double v0 = d * ((scale * s0) * ampt), v1 = d * ((scale * sx[l]) * ampt),
                             v2 = d * ((scale * sy[l]) * ampt);
                if (fx.w) {
                    if (live) fx_add3(fx, key, v0, v1, v2);
                } else if (l < L - 1) {
                    warp_scatter3(live ? key : -1, acc + key, v0, v1, v2);
                } else if (live) {
                    atomicAdd(acc + key + 0, v0);
                    atomicAdd(acc + key + 1, v1);
                    atomicAdd(acc + key + 2, v2);
                }
            }
        }
    };

    int qn = 0;   // queued candidates (warp-uniform)
    // Each warp takes runs of ST_SPAN x 32 consecutive items, interleaved
    // over the grid; the lanes hold consecutive items and step by 32.
    const int64_t n_warps = int64_t(gridDim.x) * ST_WARPS;
    const int64_t run = int64_t(ST_SPAN) * 32;
    const WalkLeg& ml = sd.leg[L - 1];
    for (int64_t rb = it0 + (int64_t(blockIdx.x) * ST_WARPS + warp) * run; rb < it1; rb += n_warps * run) {
        WalkPos<L> p;
        walk_decode<L>(sd, rb + lane, p);
        WalkFront fr;
        bool front_ok = false;
        for (int st = 0; st < ST_SPAN; ++st) {
            const int64_t base = rb + int64_t(st) * 32;
            if (base >= it1) break;
            const int64_t item = base + lane;
            int e[L];
            int lo[2] = {0, 0}, hi[2] = {0, 0};
            double pmn = 0.0, pmx = 0.0;   // energy window of legs 0..L-2, summed in leg order
            int ncand = 0;
            if (item < it1) {
                walk_at<L>(c, sd, p, fr, front_ok, e, lo, hi, pmn, pmx);
                if (lo[0] != hi[0] && lo[1] != hi[1]) ncand = 2 * (hi[0] - lo[0]) * (hi[1] - lo[1]);
            }
            const int u = p.u;
            const int maxc = __reduce_max_sync(full, unsigned(ncand));
            // candidate k of the box: element 2 (cx + cy nx) + ie with
            // cx = lo0 + (k / 2) % nbx, cy = lo1 + (k / 2) / nbx, ie = k % 2
            int cx = lo[0], cy = lo[1], ie = 0;
            for (int k = 0; k < maxc; ++k) {
                bool pass = false;
                int el = 0;
                if (k < ncand) {
                    el = 2 * (cx + cy * ml.nx) + ie;
                    const double emin = __ldg(ml.minE + el), emax = __ldg(ml.maxE + el);
                    const double minE = pmn + ((c.leg[L - 1].dir > 0) ? emin : -emax);
                    const double maxE = pmx + ((c.leg[L - 1].dir > 0) ? emax : -emin);
                    pass = (minE <= 0.0) && (maxE >= 0.0);
                }
                if (ie) {
                    ie = 0;
                    if (++cx == hi[0]) { cx = lo[0]; ++cy; }
                } else {
                    ie = 1;
                }
                const unsigned bal = __ballot_sync(full, pass);
                if (pass) {
                    const int pos = qn + __popc(bal & ((1u << lane) - 1u));
#pragma unroll
                    for (int l = 0; l < L - 1; ++l) s_q[0][warp][l][pos] = e[l];
                    s_q[0][warp][L - 1][pos] = el;
                    s_q[0][warp][L][pos] = u;
                }
                qn += __popc(bal);
                __syncwarp();
                if (qn >= 32) {
                    stage1(qn - 32, 32);
                    qn -= 32;
                    if (q2n >= 32) {
                        survive(q2n - 32, 32);
                        q2n -= 32;
                        if (q3n >= 32) {
                            evaluate(q3n - 32, 32);
                            q3n -= 32;
                        }
                    }
                    __syncwarp();   // the slots are reused
                }
            }
            if (walk_advance<L>(sd, p)) front_ok = false;
        }
    }
    // the queues' remainders, survivors first once queue 1 is empty
    if (qn > 0) stage1(0, qn);
    for (;;) {
        if (q3n >= 32 || (q2n == 0 && q3n > 0)) {
            const int t = min(q3n, 32);
            evaluate(q3n - t, t);
            q3n -= t;
        } else if (q2n > 0) {
            const int t = min(q2n, 32);
            survive(q2n - t, t);
            q2n -= t;
        } else {
            break;
        }
        __syncwarp();
    }
    if (sd.counts) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_pre += __shfl_down_sync(full, n_pre, o);
            n_det += __shfl_down_sync(full, n_det, o);
            n_surv += __shfl_down_sync(full, n_surv, o);
            n_pts += __shfl_down_sync(full, n_pts, o);
            n_tin += __shfl_down_sync(full, n_tin, o);
        }
        if (lane == 0 && (n_pre | n_det | n_surv | n_pts | n_tin)) {
            atomicAdd(sd.counts + 0, n_pre);
            atomicAdd(sd.counts + 1, n_det);
            atomicAdd(sd.counts + 2, n_surv);
            atomicAdd(sd.counts + 3, n_pts);
            atomicAdd(sd.counts + 4, n_tin);
        }
    }
}

template <int L, int MODE>
static int launch_stream(const ChanDev& c, const StreamDev& sd, int64_t it0, int64_t it1, const InstDev* insts,
                         int n_insts, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s, int rate_leg,
                         const FxAcc& fx, const double* co = nullptr, double* grad_amp = nullptr,
                         const FxAcc& fx_amp = FxAcc{}) {
    auto kern = k_collision_stream<L, MODE>;
    const int threads = ST_WARPS * 32;
    const size_t smem = 2 * sizeof(double) * size_t(c.nmc) * c.R;
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (per_sm < 1) per_sm = 1;
    const int64_t batches = (it1 - it0 + ST_SPAN * 32 - 1) / (ST_SPAN * 32);
    int64_t blocks = (batches + ST_WARPS - 1) / ST_WARPS;
    // several waves of resident blocks: the work per item varies a lot
    const int64_t cap = int64_t(nsm) * per_sm * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) return TB_OK;
    kern<<<unsigned(blocks), threads, smem, s>>>(c, sd, it0, it1, insts, n_insts, f, acc, ctl,
                                                 MODE == ST_RATE ? rate_leg : -1, fx, co, grad_amp, fx_amp);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

int launch_collision_stream(const ChanDev& c, const StreamDev& sd, int64_t item_begin, int64_t item_end,
                            const InstDev* insts, int n_insts, const double* f, double* acc, const DPCtl* ctl,
                            cudaStream_t s, int rate_leg, const FxAcc& fx) {
    if (item_end <= item_begin || n_insts <= 0) return TB_OK;
    if (c.nmc > 64) { set_error("streamed channels take at most 64 Monte-Carlo points"); return TB_ERR_ARG; }
#define TB_ST(LL)                                                                                             \
    (rate_leg >= 0                                                                                            \
         ? launch_stream<LL, ST_RATE>(c, sd, item_begin, item_end, insts, n_insts, f, acc, ctl, s, rate_leg, fx) \
         : launch_stream<LL, ST_PROPAGATE>(c, sd, item_begin, item_end, insts, n_insts, f, acc, ctl, s, -1, fx))
    switch (c.L) {
        case 2: return TB_ST(2);
        case 3: return TB_ST(3);
        case 4: return TB_ST(4);
    }
#undef TB_ST
    set_error("nlegs must be 2..4");
    return TB_ERR_ARG;
}

int launch_vjp_stream(const ChanDev& c, const StreamDev& sd, int64_t item_begin, int64_t item_end,
                      const InstDev* insts, int n_insts, const double* f, const double* u, double* grad_f,
                      double* grad_amp, cudaStream_t s, const FxAcc& fx, const FxAcc& fx_amp) {
    if (item_end <= item_begin || n_insts <= 0) return TB_OK;
    if (c.nmc > 64) { set_error("streamed channels take at most 64 Monte-Carlo points"); return TB_ERR_ARG; }
    StreamDev q = sd;
    q.counts = nullptr;
#define TB_SV(LL) launch_stream<LL, ST_VJP>(c, q, item_begin, item_end, insts, n_insts, f, grad_f, nullptr, s, -1, \
                                            fx, u, grad_amp, fx_amp)
    switch (c.L) {
        case 2: return TB_SV(2);
        case 3: return TB_SV(3);
        case 4: return TB_SV(4);
    }
#undef TB_SV
    set_error("nlegs must be 2..4");
    return TB_ERR_ARG;
}

}  // namespace tb
