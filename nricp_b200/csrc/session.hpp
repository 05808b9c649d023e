// Host orchestration of one batch of wraps on one device stream.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/nricp_b200.h"
#include "common.cuh"
#include "kernels.cuh"

namespace nricp_b200 {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct TimeoutError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CapacityError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t status, const char* what);

struct Wrap;

class Batch {
public:
    Batch();
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    // Host preparation of one more wrap (validation, graph, layouts).
    void add(const NricpSolveDesc& desc);
    // The same for many wraps, prepared in parallel on the host's cores;
    // the first invalid wrap (in order) raises.
    void add_all(const NricpSolveDesc* descs, int count);
    // Device arenas, uploads, hierarchies; after this the batch can tick.
    void upload_all(LbvhExport* lbvh_out = nullptr);
    // Back to the start of every wrap's schedule, inputs kept resident
    // (device work only: state reset and the targets' hierarchies rebuilt).
    void reset();
    // One tick for every wrap (eager launches, optional kernel timers).
    void tick(KernelTimers* timers = nullptr);
    // Ticks (as a replayed CUDA graph) until every wrap is done.
    void run(int max_ticks = 1 << 20);
    // Eager ticks with per-tick kernel timing of the dominant kernels.
    void run_timed(KernelTimers* timers, std::vector<float>* query_ms, std::vector<float>* pcg_ms,
                   std::vector<float>* assemble_ms, int max_ticks = 1 << 20);
    // Per-tick records of wrap 0 from the last run_timed.
    struct TickRecord {
        int phase, level, pcg_iterations, pad;
        float query_ms, pcg_ms, assemble_ms, tick_ms;
    };
    const std::vector<TickRecord>& tick_records() const { return records_; }
    // Device time of reset() + run() on the batch's stream (CUDA events).
    double timed_step();
    // Sizes and work counters of one level (kLevelSizeEntries ints).
    static constexpr int kLevelSizeEntries = 15;
    void level_sizes(int i, int level, int* sizes) const;
    // Cluster size of the solve launch.  > 0: that size for every wrap; 0:
    // each wrap its own latency cluster (about 128 nodes per CTA), one launch
    // per size class, the classes in parallel; -s: the same classes halved s
    // times.  Every choice gives bit-identical results.
    void set_pcg_cluster(int cluster);
    int default_pcg_cluster() const;
    void pull_controls();
    bool all_done() const;
    void finish();

    int size() const { return static_cast<int>(wraps_.size()); }
    const WrapControl& control(int i) const;
    // The current system of wrap `i` and the state it was assembled at.
    void inspect(int i, NricpInspect* out);
    void result(int i, NricpResult* out);
    // Every wrap's result: downloads in turn, then the host work in parallel.
    void results(NricpResult* outs);
    void current_vertices(int i, double* out);
    int finest_nodes(int i) const;
    int levels(int i) const;
    int vertices(int i) const;
    long ticks() const { return ticks_; }
    long launches() const { return launches_; }
    const TickShape& shape() const { return shape_; }
    cudaStream_t stream() const { return stream_; }
    const WrapDev* device_wrap(int i) const;

private:
    std::vector<double> evaluate_host(int i, const std::vector<double>& rot,
                                      const std::vector<double>& trans, int level) const;

    std::vector<std::unique_ptr<Wrap>> wraps_;
    cudaStream_t stream_ = nullptr;
    WrapDev* dev_wraps_ = nullptr;
    WrapControl* dev_controls_ = nullptr;
    // Start states and target hierarchies are built on kBuildStreams side
    // streams, each with its own hierarchy scratch (sized for the largest
    // target), forked from and joined back into stream_.
    static constexpr int kBuildStreams = 4;
    void reset_all(const char* staging, const std::vector<size_t>* offset, LbvhExport* lbvh_out);
    cudaStream_t build_streams_[kBuildStreams] = {};
    cudaEvent_t build_fork_ = nullptr, build_done_[kBuildStreams] = {};
    void* build_scratch_[kBuildStreams] = {};
    cudaMemPool_t pool_ = nullptr;  // the arenas' and the scratch's (batch_pool)
    int* query_counter_ = nullptr;  // the query queues' heads (vertices, long walks)
    cudaStream_t side_stream_ = nullptr;  // the tick's refresh branch
    cudaEvent_t side_fork_ = nullptr, side_join_ = nullptr;
    int* pcg_index_ = nullptr;      // wraps ordered by solve class (device)
    cudaStream_t pcg_streams_[5] = {};
    cudaEvent_t pcg_join_[5] = {};
    cudaEvent_t pcg_fork_ = nullptr;
    WrapControl* host_controls_ = nullptr;
    TickShape shape_{};
    cudaGraphExec_t graph_exec_ = nullptr;
    // Solve launch fields of `shape` for the cluster setting `cluster` (as
    // set_pcg_cluster takes it), its class lists in `index` (device, made
    // here when needed); `cls` (if given) receives each wrap's cluster size.
    void solve_shape(int cluster, TickShape& shape, int*& index, std::vector<int>* cls);
    cudaGraphExec_t capture(const TickShape& shape);
    // The batch's tail.  With halved classes, once the wraps still running
    // would fit on the SMs in one round at one halving less, their ticks run
    // with that shape: few wraps left, each gets more CTAs.  Results do not
    // depend on the cluster size.
    bool tail_due() const;
    TickShape tail_shape_{};
    int* tail_index_ = nullptr;
    std::vector<int> tail_cls_;
    bool tail_ready_ = false, tail_on_ = false;
    cudaGraphExec_t tail_graph_ = nullptr;
    int sms_ = 148;
    std::vector<TickRecord> records_;
    long ticks_ = 0;
    long launches_ = 0;
};

extern thread_local std::string g_last_error;
struct TransferCounters {
    unsigned long long h2d = 0, d2h = 0;
};
extern thread_local TransferCounters g_transfers;

// Continuous batching on one device: resident wrap slots advanced by the
// same launches; requests prepared on host threads, admitted by memory
// budget as slots free up, retired when done (see nricp_server_* ).
class Server {
public:
    explicit Server(const NricpServerConfig& config);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;
    long submit(const NricpSolveDesc& desc);
    int poll(long id, double* latency_seconds);
    // The request's time in each phase so far, in seconds: host preparation
    // (graph, layouts), loading (waiting for memory, uploads, hierarchy),
    // waiting for a slot, on the device, composing the result.
    void phases(long id, double seconds[5]);
    bool wait(long id, double timeout_seconds);
    void result(long id, NricpResult* out);
    NricpServerStats stats();
    // Statistics of several servers as one (latency percentiles over all of
    // their requests; peak residency is the sum of the peaks).
    static NricpServerStats merged_stats(const std::vector<Server*>& servers);

    struct Impl;

private:
    std::unique_ptr<Impl> impl_;
};

}  // namespace nricp_b200
