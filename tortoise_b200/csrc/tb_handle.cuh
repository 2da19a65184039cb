// tb_handle.cuh -- the library handle and the host-side helpers shared by
// the C ABI (tb_api.cu) and the adjoint driver (tb_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "tb_dp45.cuh"
#include "tb_enumerate.cuh"
#include "tb_kernels.cuh"
#include "tb_stream.cuh"
#include "tb_tensor.cuh"
#include "tb_theta.cuh"

namespace tb {

// A channel structure shared by every run of the same structure: the tuple
// list, the moment tensor and the Monte-Carlo tables exist once.
struct GroupChan {
    ChanDev dev;                  // table pointers of the group's first run
    int L = 0;
    double* d_umk = nullptr;
    double* d_mc = nullptr;
    double* d_mc_pre = nullptr;
    DeviceTuples tup;             // this handle's part of the list (all of it unless sharded)
    double* d_tamp = nullptr;     // functAmplitude per tuple of tup (dev.tamp), or null
    int64_t shard_begin = 0;      // index of tup's first tuple in the full list
    int64_t n_total = 0;          // length of the full list
    int64_t diag[3] = {0, 0, 0};
    int layout = TB_LAYOUT_MC64;
    MomentTensor tensor;
    ThetaList theta;              // Monte-Carlo layout: tuples with points inside the simplices, and which
    // streamed channel (TB_LAYOUT_STREAM): the candidate walk and this
    // handle's part [item_begin, item_end) of its work items; counts of the
    // last evaluation (prefilter, determinant, survivors, points inside,
    // tuples with points inside) in sdev.counts
    bool stream = false;
    StreamDev sdev{};
    int64_t item_begin = 0, item_end = 0;
    std::vector<int> insts;       // channel instances using it (run order)
    InstDev* d_insts = nullptr;   // [insts.size()]
};

// One run's channel (the unit tb_channel_info / tb_set_amplitude address).
struct ChanInst {
    int group = 0;
    int run = 0;
    int band[TB_MAX_LEGS] = {0, 0, 0, 0};   // global band ids
    double amplitude = 0.0;
    InstDev dev{};
    InstDev* d_single = nullptr;  // this instance alone (single-channel calls)
    int slot = 0;                 // position inside the group's d_insts
};

struct RunInfo {
    int band0 = 0, nbands = 0;
    int64_t dof_off = 0, ndofs = 0;
    int chan0 = 0, nchans = 0;
};

struct AdjointState;

}  // namespace tb

struct tb_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    tb_options opts{};
    std::vector<tb::HostMesh> meshes;
    std::vector<tb::HostBand> bands;
    std::vector<tb::BandDev> banddev;
    std::vector<double*> dev_allocs;
    std::vector<void*> dev_raw;
    std::vector<tb::RunInfo> runs;
    std::vector<tb::GroupChan> groups;
    std::vector<tb::ChanInst> insts;
    tb::ElemDev ed{};
    bool any_drift = false;
    int64_t ndofs = 0;
    double* d_f = nullptr;
    double* d_out = nullptr;
    double* d_acc = nullptr;
    double* d_part = nullptr;
    // deterministic mode: the exact accumulator behind d_acc (3 words per
    // dof and a poison word; w == nullptr otherwise)
    tb::FxAcc fx{};
    // set by a contraction kernel whose bounded wait for a staged tile ran
    // out; read and cleared by the synchronising calls (TB_ERR_TIMEOUT)
    int* d_err = nullptr;
    bool wait_timed_out = false;   // the current integration met a timed-out wait
    // DP45
    tb::DPBufs dp{};
    bool dp_ready = false;
    int64_t dense_cap_alloc = -1;
    tb::RunDev* d_runs = nullptr;
    std::vector<tb::RunDev> hruns;
    cudaGraphExec_t graph = nullptr;
    int graph_flags = -1;
    tb::DPCtl* h_ctl = nullptr;   // pinned host mirror [nruns]
    int dp_flags = 0;
    // adjoint (tb_adjoint.cu)
    tb::AdjointState* adj = nullptr;
    // tuple sharding (tb_shard.cu): ncclComm_t once connected
    void* comm = nullptr;
    double comm_timeout = 60.0;
    bool comm_failed = false;
    // time-dependent constraints (tb_constraints.cu)
    tb_constraint_fn cfn = nullptr;
    void* cuser = nullptr;
    int64_t cdofs = 0;                 // constrained dofs of all runs (one slot)
    std::vector<int64_t> coff;         // per band: offset in a slot, -1 unconstrained
    double* d_ctv = nullptr;           // device slots [TB_TC_SLOTS][cdofs]
    double* h_ctv = nullptr;           // pinned host copy the host node fills
    tb::DPCtl* h_ctl_tc = nullptr;     // pinned controllers the host node reads and edits
};


namespace tb {

double* dev_alloc(tb_handle* h, size_t n);
int run_rhs_acc(tb_handle* h, const double* d_in, double* d_acc, const DPCtl* ctl, int flags, int only_inst);
int dp_alloc(tb_handle* h, int64_t max_dense);
int ensure_graph(tb_handle* h, int flags);
int dp_begin(tb_handle* h, const double* f0, const double* t0, const double* t_final, const double* dense_step,
             int64_t max_dense, int flags, const DPBufs* hooks);
void adjoint_release(tb_handle* h);

// A zeroed exact accumulator of n slots (3 words each) plus its poison word,
// owned by the handle (deterministic mode).
int fx_alloc(tb_handle* h, int64_t n, FxAcc& out);
// deterministic mode's clamp flag: read (and clear) it; the error it reports
int fx_take_saturation(tb_handle* h, bool& clamped);
int fx_saturation_error();

// tb_shard.cu
int64_t shard_begin(int64_t n, int rank, int n_ranks);
int shard_tuples(tb_handle* h, GroupChan& G);          // keep this rank's part of G's tuple list
int shard_allreduce(tb_handle* h, double* buf, size_t n);   // in-place sum over the ranks (no-op unconnected)
int stream_wait(tb_handle* h);                         // stream sync, bounded when connected
void shard_release(tb_handle* h);

// tb_constraints.cu
int tc_record_pre_attempt(tb_handle* h);   // the host node + copies at the head of the attempt graph
int tc_begin(tb_handle* h);                // t0 values into slot 0, initial veto of every run's dt
void tc_release(tb_handle* h);

}  // namespace tb
