// tb_stream.cuh -- the Monte-Carlo collision operator over tuples enumerated
// on the fly (no stored tuple list).
#pragma once

#include "tb_kernels.cuh"

namespace tb {

// One leg's mesh as the candidate walk needs it.
struct WalkLeg {
    const double* minE;   // [ne] per-element energy range (Band.cpp:45-56 P1 vertices)
    const double* maxE;
    int nx, ny;
    double origin[2];
    double dG[2][2];
    double invdG[2][2];
};

// The candidate walk of one channel: the work items of the reference's
// nested loops (umklapp, sections of legs 0..L-2, element choice within
// those sections), ScatteringChannel.hpp:205-255, in the reference's order.
struct StreamDev {
    WalkLeg leg[TB_MAX_LEGS];
    int64_t nsec[TB_MAX_LEGS];   // sections of legs 0..L-2 (1 for the others)
    int64_t n_items;             // n_umk * prod nsec * 2^(L-1)
    const double* mc_pre;        // survival-test table (precalculateIndices)
    // per evaluation (cleared before each launch): candidates inside the
    // energy window, with a valid determinant, surviving tuples, points
    // inside the simplices, tuples with such points (unsigned long long[5])
    unsigned long long* counts;
};

// acc (or fx) += the collision terms of channel c over work items
// [item_begin, item_end): every surviving tuple of those items, the same
// tuples and the same per-tuple sums as the stored-list path over the points
// inside the simplices.  rate_leg >= 0: that leg's scattering rate.
int launch_collision_stream(const ChanDev& c, const StreamDev& sd, int64_t item_begin, int64_t item_end,
                            const InstDev* insts, int n_insts, const double* f, double* acc, const DPCtl* ctl,
                            cudaStream_t s, int rate_leg, const FxAcc& fx);

// The transposed operator over the same work items: grad_f += C'(f)^T u
// (or into fx) and grad_amp[k] += <u, dC/d amplitude_k> (or fx_amp slot k)
// for every instance k -- the stored-list VJP's per-tuple terms.
int launch_vjp_stream(const ChanDev& c, const StreamDev& sd, int64_t item_begin, int64_t item_end,
                      const InstDev* insts, int n_insts, const double* f, const double* u, double* grad_f,
                      double* grad_amp, cudaStream_t s, const FxAcc& fx, const FxAcc& fx_amp);

}  // namespace tb
