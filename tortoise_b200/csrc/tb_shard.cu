// tb_shard.cu -- one run's tuples split over several processes (one GPU
// each): the partition rule, the NCCL communicator and the bounded waits on
// a connected handle.
//
// The reference splits the tuples of ScatteringChannel<2,L>::propagate over
// host threads with a TBB reduce (src/Physics/Scattering/ScatteringChannel.cpp:
// 651-670: each task sums singleScatteringPropagator over its range into a
// private MaterialStatus, the partial statuses are added).  Here each GPU
// keeps a contiguous part of every tuple list for the lifetime of the handle,
// accumulates its partial collision term into the handle's accumulator and
// one in-place sum all-reduce over NVLink makes every rank's accumulator the
// full one.  Drift, M^-1 and the whole integrator stay replicated.
//
// NCCL is opened with dlopen on first use, so that the library loads (and
// unsharded handles run) on hosts without it; in a process that already
// loaded libnccl.so.2 (PyTorch) the same library is used.  The communicator
// is non-blocking: every NCCL call and every wait on the handle's stream is
// polled against the handle's deadline, and a wait that runs out aborts the
// communicator (ncclCommAbort also stops NCCL kernels still in flight) instead
// of leaving the process blocked on a rank that is gone.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "tb_handle.cuh"

namespace tb {

namespace {

struct NcclApi {
    bool tried = false;
    void* so = nullptr;
    std::string why;
    ncclResult_t (*getUniqueId)(ncclUniqueId*) = nullptr;
    ncclResult_t (*commInitRankConfig)(ncclComm_t*, int, ncclUniqueId, int, ncclConfig_t*) = nullptr;
    ncclResult_t (*commGetAsyncError)(ncclComm_t, ncclResult_t*) = nullptr;
    ncclResult_t (*allReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*commFinalize)(ncclComm_t) = nullptr;
    ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*commAbort)(ncclComm_t) = nullptr;
    const char* (*getErrorString)(ncclResult_t) = nullptr;
};

std::mutex g_nccl_mu;
NcclApi g_nccl;

template <class F>
bool bind(void* so, const char* name, F& fn) {
    fn = reinterpret_cast<F>(dlsym(so, name));
    return fn != nullptr;
}

const NcclApi* nccl() {
    std::lock_guard<std::mutex> lk(g_nccl_mu);
    NcclApi& A = g_nccl;
    if (A.tried) return A.so ? &A : nullptr;
    A.tried = true;
    const char* names[] = {"libnccl.so.2", "libnccl.so"};
    for (const char* n : names)
        if ((A.so = dlopen(n, RTLD_NOW | RTLD_GLOBAL)) != nullptr) break;
    if (!A.so) {
        const char* e = dlerror();
        A.why = std::string("cannot load libnccl.so.2: ") + (e ? e : "not found");
        return nullptr;
    }
    bool ok = bind(A.so, "ncclGetUniqueId", A.getUniqueId) && bind(A.so, "ncclCommInitRankConfig", A.commInitRankConfig) &&
              bind(A.so, "ncclCommGetAsyncError", A.commGetAsyncError) && bind(A.so, "ncclAllReduce", A.allReduce) &&
              bind(A.so, "ncclCommFinalize", A.commFinalize) && bind(A.so, "ncclCommDestroy", A.commDestroy) &&
              bind(A.so, "ncclCommAbort", A.commAbort) && bind(A.so, "ncclGetErrorString", A.getErrorString);
    if (!ok) {
        A.why = "libnccl.so.2 lacks a required symbol (NCCL >= 2.14 is needed)";
        dlclose(A.so);
        A.so = nullptr;
        return nullptr;
    }
    return &A;
}

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

// Marks the handle's communicator as failed after aborting it.
int comm_fail(tb_handle* h, int code, const std::string& msg) {
    const NcclApi* A = nccl();
    if (h->comm && A) A->commAbort(static_cast<ncclComm_t>(h->comm));
    h->comm = nullptr;
    h->comm_failed = true;
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // holds the aborted collective
    set_error(msg);
    return code;
}

// Polls the communicator until its pending operation is no longer in
// progress, within the handle's deadline.
int comm_settle(tb_handle* h, const char* what) {
    const NcclApi* A = nccl();
    ncclComm_t c = static_cast<ncclComm_t>(h->comm);
    const auto t0 = Clock::now();
    for (;;) {
        ncclResult_t st = ncclSuccess;
        const ncclResult_t q = A->commGetAsyncError(c, &st);
        if (q != ncclSuccess) return comm_fail(h, TB_ERR_CUDA, std::string(what) + ": " + A->getErrorString(q));
        if (st == ncclSuccess) return TB_OK;
        if (st != ncclInProgress) return comm_fail(h, TB_ERR_CUDA, std::string(what) + ": " + A->getErrorString(st));
        if (seconds_since(t0) > h->comm_timeout)
            return comm_fail(h, TB_ERR_TIMEOUT, std::string(what) + ": no progress within the shard timeout");
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

}  // namespace

int64_t shard_begin(int64_t n, int rank, int n_ranks) {
    if (rank <= 0) return 0;
    if (rank >= n_ranks) return n;
    const int64_t tile = 128;
    const int64_t tiles = (n + tile - 1) / tile;
    // tiles * rank / n_ranks without overflow for any n that fits device memory
    const int64_t t = int64_t((__int128)tiles * rank / n_ranks);
    return std::min(n, t * tile);
}

int shard_tuples(tb_handle* h, GroupChan& G) {
    const int R = h->opts.shard_count;
    const int r = h->opts.shard_rank;
    if (G.stream) {
        // a streamed channel splits its work items the same way
        G.n_total = G.sdev.n_items;
        G.item_begin = R <= 1 ? 0 : shard_begin(G.sdev.n_items, r, R);
        G.item_end = R <= 1 ? G.sdev.n_items : shard_begin(G.sdev.n_items, r + 1, R);
        G.shard_begin = G.item_begin;
        return TB_OK;
    }
    G.n_total = G.tup.n;
    G.shard_begin = 0;
    if (R <= 1) return TB_OK;
    const int64_t b = shard_begin(G.tup.n, r, R), e = shard_begin(G.tup.n, r + 1, R);
    const int64_t cnt = e - b;
    DeviceTuples part;
    TB_TRY(part.reserve(G.L, std::max<int64_t>(cnt, 1), h->stream));
    for (int l = 0; l <= G.L && cnt > 0; ++l)
        TB_CUDA(cudaMemcpyAsync(part.d + size_t(l) * size_t(part.cap), G.tup.d + size_t(l) * size_t(G.tup.cap) + size_t(b),
                                sizeof(int32_t) * size_t(cnt), cudaMemcpyDeviceToDevice, h->stream));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    G.tup.release();
    G.tup = part;
    G.tup.n = cnt;
    G.shard_begin = b;
    return TB_OK;
}

int shard_allreduce(tb_handle* h, double* buf, size_t n) {
    if (h->comm_failed) { set_error("the shard communicator was aborted; create new handles"); return TB_ERR_CUDA; }
    if (!h->comm || n == 0) return TB_OK;   // unconnected: partial sums
    const NcclApi* A = nccl();
    const ncclResult_t q = A->allReduce(buf, buf, n, ncclDouble, ncclSum, static_cast<ncclComm_t>(h->comm), h->stream);
    if (q != ncclSuccess && q != ncclInProgress)
        return comm_fail(h, TB_ERR_CUDA, std::string("ncclAllReduce: ") + A->getErrorString(q));
    return comm_settle(h, "ncclAllReduce");
}

int stream_wait(tb_handle* h) {
    if (!h->comm) {
        TB_CUDA(cudaStreamSynchronize(h->stream));
        return TB_OK;
    }
    const NcclApi* A = nccl();
    const auto t0 = Clock::now();
    for (;;) {
        const cudaError_t e = cudaStreamQuery(h->stream);
        if (e == cudaSuccess) return TB_OK;
        if (e != cudaErrorNotReady) {
            set_error(std::string("stream: ") + cudaGetErrorString(e));
            return TB_ERR_CUDA;
        }
        ncclResult_t st = ncclSuccess;
        A->commGetAsyncError(static_cast<ncclComm_t>(h->comm), &st);
        if (st != ncclSuccess && st != ncclInProgress)
            return comm_fail(h, TB_ERR_CUDA, std::string("shard communicator: ") + A->getErrorString(st));
        if (seconds_since(t0) > h->comm_timeout) {
            comm_fail(h, TB_ERR_TIMEOUT, "shard wait ran out (a rank stopped or diverged); communicator aborted");
            // the abort ends the NCCL kernels; let the stream drain, bounded
            const auto t1 = Clock::now();
            while (cudaStreamQuery(h->stream) == cudaErrorNotReady && seconds_since(t1) < h->comm_timeout)
                std::this_thread::sleep_for(std::chrono::microseconds(200));
            set_error("shard wait ran out (a rank stopped or diverged); communicator aborted");
            return TB_ERR_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

void shard_release(tb_handle* h) {
    if (!h->comm) return;
    const NcclApi* A = nccl();
    ncclComm_t c = static_cast<ncclComm_t>(h->comm);
    h->comm = nullptr;
    // finalize flushes outstanding work; bounded like every other wait
    const ncclResult_t q = A->commFinalize(c);
    bool clean = q == ncclSuccess || q == ncclInProgress;
    const auto t0 = Clock::now();
    while (clean) {
        ncclResult_t st = ncclSuccess;
        A->commGetAsyncError(c, &st);
        if (st == ncclSuccess) break;
        if (st != ncclInProgress || seconds_since(t0) > h->comm_timeout) { clean = false; break; }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    if (clean) A->commDestroy(c);
    else A->commAbort(c);
}

}  // namespace tb

using namespace tb;

extern "C" {

int tb_shard_range(int64_t n_tuples, int rank, int n_ranks, int64_t* begin, int64_t* end) {
    if (n_tuples < 0 || n_ranks < 1 || rank < 0 || rank >= n_ranks || !begin || !end) {
        set_error("tb_shard_range: need n_tuples >= 0 and 0 <= rank < n_ranks");
        return TB_ERR_ARG;
    }
    *begin = shard_begin(n_tuples, rank, n_ranks);
    *end = shard_begin(n_tuples, rank + 1, n_ranks);
    return TB_OK;
}

int tb_shard_unique_id(void* id) {
    if (!id) { set_error("null argument"); return TB_ERR_ARG; }
    const NcclApi* A = nccl();
    if (!A) { set_error(g_nccl.why); return TB_ERR_NO_DEVICE; }
    static_assert(sizeof(ncclUniqueId) == TB_SHARD_ID_BYTES, "NCCL unique id size");
    ncclUniqueId u;
    const ncclResult_t q = A->getUniqueId(&u);
    if (q != ncclSuccess) { set_error(std::string("ncclGetUniqueId: ") + A->getErrorString(q)); return TB_ERR_CUDA; }
    std::memcpy(id, &u, sizeof(u));
    return TB_OK;
}

int tb_shard_connect(tb_handle* h, const void* id, double timeout_s) {
    if (!h || !id) { set_error("null argument"); return TB_ERR_ARG; }
    if (h->comm || h->comm_failed) { set_error("the handle is already connected"); return TB_ERR_ARG; }
    if (!(timeout_s > 0.0)) { set_error("timeout_s must be > 0"); return TB_ERR_ARG; }
    const NcclApi* A = nccl();
    if (!A) { set_error(g_nccl.why); return TB_ERR_NO_DEVICE; }
    TB_CUDA(cudaSetDevice(h->device));
    TB_CUDA(cudaStreamSynchronize(h->stream));
    h->comm_timeout = timeout_s;
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
    cfg.blocking = 0;
    ncclComm_t c = nullptr;
    const int n_ranks = std::max(h->opts.shard_count, 1);
    const ncclResult_t q = A->commInitRankConfig(&c, n_ranks, u, h->opts.shard_rank, &cfg);
    if (q != ncclSuccess && q != ncclInProgress) {
        if (c) A->commAbort(c);
        set_error(std::string("ncclCommInitRankConfig: ") + A->getErrorString(q));
        return TB_ERR_CUDA;
    }
    h->comm = c;
    TB_TRY(comm_settle(h, "ncclCommInitRankConfig"));
    // One all-reduce of the (zero) accumulator outside any stream capture:
    // NCCL sets up its connections for this message size here, not inside
    // the DP45 graph capture.
    TB_TRY(shard_allreduce(h, h->d_acc, size_t(h->ndofs)));
    TB_TRY(stream_wait(h));
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // re-capture with the collective
    return TB_OK;
}

int tb_shard_info(const tb_handle* h, int ch, int64_t* begin, int64_t* n_total) {
    if (!h || ch < 0 || ch >= int(h->insts.size())) { set_error("channel index out of range"); return TB_ERR_ARG; }
    const GroupChan& G = h->groups[h->insts[ch].group];
    if (begin) *begin = G.shard_begin;
    if (n_total) *n_total = G.n_total;
    return TB_OK;
}

}  // extern "C"
