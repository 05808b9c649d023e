// Host orchestration of the device schedule and the C-ABI (include/nricp_b200.h).
//
// A Batch owns one or more wraps: their device arenas, the WrapDev
// descriptors the kernels index by blockIdx.y, and one stream.  Running a
// batch means replaying the tick (captured once as a CUDA graph) until every
// wrap's device-side schedule reaches Done; the host only polls a pinned copy
// of the schedule scalars every few ticks.  A session is a batch of one that
// the caller advances one tick at a time.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/nricp_b200.h"
#include "common.cuh"
#include "host.hpp"
#include "graph_build.hpp"
#include "kernels.cuh"
#include "session.hpp"
#include "staging.hpp"

namespace nricp_b200 {

thread_local std::string g_last_error;
thread_local TransferCounters g_transfers;

void check(cudaError_t status, const char* what) {
    if (status != cudaSuccess)
        throw CudaError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(status));
}

namespace {

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One device allocation carved into aligned sub-arrays.
class Arena {
public:
    size_t reserve(size_t bytes) {
        const size_t at = size_;
        size_ += (bytes + 255) & ~size_t(255);
        return at;
    }
    void allocate() {
        if (size_ == 0) size_ = 256;
        check(cudaMalloc(&base_, size_), "cudaMalloc(wrap arena)");
    }
    // Stream-ordered, from `pool`: neither this nor release_async waits for
    // the device.
    void allocate(cudaMemPool_t pool, cudaStream_t stream) {
        if (size_ == 0) size_ = 256;
        check(cudaMallocFromPoolAsync(&base_, size_, pool, stream), "cudaMallocFromPoolAsync(wrap arena)");
    }
    void release_async(cudaStream_t stream) {
        if (base_) check(cudaFreeAsync(base_, stream), "cudaFreeAsync(wrap arena)");
        base_ = nullptr;
    }
    template <typename T>
    T* at(size_t offset) const { return reinterpret_cast<T*>(static_cast<char*>(base_) + offset); }
    size_t size() const { return size_; }
    void* base() const { return base_; }
    void release() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
    }

private:
    void* base_ = nullptr;
    size_t size_ = 0;
};

// Slack of the FP32 box pruning in the closest-point walk, relative to the
// target's diagonal: far above the rounding of FP32 boxes and queries.
constexpr double kRankWindow = 4e-6;

// The bounding-box diagonal of the normalised target, from the caller's
// points: normalisation ((p - center) * scale, scale > 0) is monotone in each
// coordinate, so the normalised box's corners are the normalised corners.
double normalized_diagonal(const double* p, size_t n, const double center[3], double scale) {
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = i ? std::min(lo[k], p[i * 3 + k]) : p[k];
            hi[k] = i ? std::max(hi[k], p[i * 3 + k]) : p[k];
        }
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = (hi[k] - center[k]) * scale - (lo[k] - center[k]) * scale;
    return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

template <typename T>
void upload(T* dst, const std::vector<T>& src, cudaStream_t stream) {
    if (!src.empty()) {
        check(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, stream),
              "upload");
        g_transfers.h2d += sizeof(T) * src.size();
    }
}

// Where a wrap's inputs go: straight to the device (a copy each, in stream
// order), or into a host staging area laid out like the arena's input
// prefix, which the caller then copies in one piece.
struct InputSink {
    cudaStream_t stream = nullptr;
    char* staging = nullptr;       // host image of the arena's input prefix
    const char* arena = nullptr;   // the arena's device base
    template <typename T>
    void put(T* dst, const std::vector<T>& src) const {
        if (src.empty()) return;
        if (staging) {
            std::memcpy(staging + (reinterpret_cast<const char*>(dst) - arena), src.data(), sizeof(T) * src.size());
        } else {
            upload(dst, src, stream);
        }
    }
};

// Device memory of batches: a stream-ordered pool per device that keeps up
// to 8 GB between batches, so that repeated batches allocate and free their
// arenas without waiting for the device.
cudaMemPool_t batch_pool(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
    uint64_t keep = 8ull << 30;
    check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool");
    pools[device] = pool;
    return pool;
}


}  // namespace

// ---------------------------------------------------------------------------
// Wrap: one template/target pair, prepared on the host, resident on the device
// ---------------------------------------------------------------------------
struct Wrap {
    NricpSolveDesc desc{};
    std::vector<NricpLevelSettings> level_settings;
    std::vector<double> template_in, target_in, landmark_targets_in;
    std::vector<int32_t> template_faces, target_faces, landmark_indices;
    std::vector<uint8_t> mask;
    TemplateGraph graph;
    std::vector<LevelLayout> layouts;
    int V = 0, T = 0, Vt = 0, F = 0, L = 0, levels = 0;
    int max_nodes = 0, max_edges = 0, max_pairs = 0, max_offdiag = 0;
    double setup_seconds = 0.0, solve_started = 0.0, solve_seconds = 0.0;
    Arena arena;
    WrapDev dev{};        // host copy of the descriptor
    WrapControl* control = nullptr;  // device
    WrapControl initial_control{};   // pinned-free host copy used by reset
    double* identity_rot = nullptr;  // device (in the arena): identity rotations
    LevelRecord* initial_records = nullptr;  // and the level records a run starts from
    size_t input_bytes = 0;          // the arena's prefix that holds the inputs
    bool target_ingested = false;    // the device has normalised the target and its normals
    ~Wrap() { arena.release(); }
};

namespace {

// Copies the caller's arrays: the wrap must not depend on them afterwards
// (the reference's session copies its inputs too, session.cu:593-596).
void copy_inputs(Wrap& w, const NricpSolveDesc& d) {
    w.desc = d;
    w.V = d.template_vertex_count;
    w.T = d.template_face_count;
    w.Vt = d.target_vertex_count;
    w.F = d.target_face_count;
    w.L = d.landmark_count > 0 ? d.landmark_count : 0;
    w.template_in.assign(d.template_points, d.template_points + (size_t)w.V * 3);
    w.target_in.assign(d.target_points, d.target_points + (size_t)w.Vt * 3);
    w.template_faces.assign(d.template_faces, d.template_faces + (size_t)w.T * 3);
    w.target_faces.assign(d.target_faces, d.target_faces + (size_t)w.F * 3);
    if (d.mask) {
        w.mask.resize(w.V);
        for (int i = 0; i < w.V; ++i) w.mask[i] = d.mask[i] ? 1 : 0;
    }
    if (w.L > 0) {
        w.landmark_indices.assign(d.landmark_indices, d.landmark_indices + w.L);
        w.landmark_targets_in.assign(d.landmark_targets, d.landmark_targets + (size_t)w.L * 3);
    }
    if (d.level_setting_count > 0) {
        w.level_settings.assign(d.levels, d.levels + d.level_setting_count);
    } else {
        NricpLevelSettings s;
        nricp_default_level(&s);
        w.level_settings.push_back(s);
    }
    w.desc.levels = w.level_settings.data();
    w.desc.level_setting_count = static_cast<int>(w.level_settings.size());
    w.desc.template_points = w.template_in.data();
    w.desc.target_points = w.target_in.data();
    w.desc.template_faces = w.template_faces.data();
    w.desc.target_faces = w.target_faces.data();
    w.desc.mask = w.mask.empty() ? nullptr : w.mask.data();
    w.desc.landmark_indices = w.L ? w.landmark_indices.data() : nullptr;
    w.desc.landmark_targets = w.L ? w.landmark_targets_in.data() : nullptr;
    w.desc.landmark_count = w.L;
}

void check_graph_capacity(const Wrap& w) {
    const NricpSolveDesc& d = w.desc;
    const int finest = level_node_count(std::max(1, d.graph_levels) - 1, d.nodes_initial, d.growth, w.V);
    if (finest > pcg_max_nodes())
        throw CapacityError("the finest graph level has " + std::to_string(finest) +
                            " nodes; the device solve supports at most " +
                            std::to_string(pcg_max_nodes()));
}

GraphRequest graph_request(const Wrap& w) {
    const NricpSolveDesc& d = w.desc;
    return GraphRequest{w.template_in.data(), w.V, d.graph_levels, d.nodes_initial, d.growth,
                        d.max_nodes_per_vertex > 0 ? d.max_nodes_per_vertex : 4,
                        d.edge_neighbours > 0 ? d.edge_neighbours : 4};
}

// The size envelope of a wrap whose layouts are built.
void envelope(Wrap& w) {
    for (const LevelLayout& L : w.layouts) {
        w.max_nodes = std::max(w.max_nodes, L.node_count);
        w.max_edges = std::max(w.max_edges, L.edge_count);
        w.max_pairs = std::max(w.max_pairs, L.pair_count);
        w.max_offdiag = std::max(w.max_offdiag, static_cast<int>(L.offdiag_nodes.size() / 2));
    }
}

// The level layouts and size envelope of a wrap whose graph is built.
void finish_host(Wrap& w) {
    w.levels = static_cast<int>(w.graph.levels.size());
    w.layouts.clear();
    for (int l = 0; l < w.levels; ++l) w.layouts.push_back(build_layout(w.graph, l, w.V));
    envelope(w);
}

// The host build: graph (bit-identical to the reference's) and layouts.
void prepare_host(Wrap& w) {
    check_graph_capacity(w);
    const GraphRequest r = graph_request(w);
    w.graph = build_template_graph(r.points, r.count, r.levels, r.nodes_initial, r.growth, r.max_nodes,
                                   r.edge_neighbours);
    finish_host(w);
}

size_t bytes_of_layout(const LevelLayout& L) {
    return 256 * 27 + sizeof(double) * (L.rest.size() + L.bind_weights.size() + L.transfer_weights.size()) +
           sizeof(int32_t) * (L.bind_nodes.size() + L.bind_counts.size() + L.gather_begin.size() +
                              L.gather_entry.size() + L.node_edge_begin.size() +
                              L.node_edge_list.size() + L.edges.size() + L.pair_nodes.size() +
                              L.pair_begin.size() + L.pair_entry.size() + L.row_begin.size() +
                              L.row_entry.size() + L.offdiag_nodes.size() + L.offdiag_slots.size() +
                              L.edge_block.size() +
                              L.transfer_nodes.size() +
                              L.transfer_counts.size());
}

// Lays out, allocates and fills the wrap's device arena: the inputs first
// (template, target, level layouts, start state: the prefix of
// w.input_bytes), then the hierarchy and the solver's state and scratch.
// `control` is this wrap's slot in the batch's control array.  With
// `staging`, the inputs are written there at their arena offsets and the
// caller copies the prefix; otherwise each is copied on `stream`.  The
// target's hierarchy is reset_device's.
size_t prepare_device(Wrap& w, WrapControl* control, cudaStream_t stream, bool plan_only = false,
                      cudaMemPool_t pool = nullptr, char* staging = nullptr) {
    const NricpSolveDesc& d = w.desc;
    const int V = w.V, N = std::max(1, w.max_nodes), B = std::max(1, w.max_offdiag);
    Arena& a = w.arena;
    // template and target
    const size_t o_tpl = a.reserve(sizeof(double) * 3 * V);
    const size_t o_tpl_faces = a.reserve(sizeof(int32_t) * 3 * w.T);
    std::vector<int32_t> vf_begin, vf_list;
    vertex_faces(w.template_faces.data(), w.T, V, vf_begin, vf_list);
    const size_t o_vf_begin = a.reserve(sizeof(int32_t) * vf_begin.size());
    const size_t o_vf_list = a.reserve(sizeof(int32_t) * std::max<size_t>(1, vf_list.size()));
    const size_t o_mask = a.reserve(w.mask.empty() ? 0 : V);
    const size_t o_lm_target = a.reserve(sizeof(double) * 3 * V);
    const size_t o_lm_flag = a.reserve(V);
    const size_t o_lm_vertices = a.reserve(sizeof(int32_t) * std::max(1, w.L));
    const size_t o_tgt = a.reserve(sizeof(double) * 3 * w.Vt);
    const size_t o_tgt_normals = a.reserve(sizeof(double) * 3 * w.Vt);
    const size_t o_tgt_faces = a.reserve(sizeof(int32_t) * 3 * w.F);
    // levels
    std::vector<size_t> level_base(w.levels);
    for (int l = 0; l < w.levels; ++l) level_base[l] = a.reserve(bytes_of_layout(w.layouts[l]));
    const size_t o_identity = a.reserve(sizeof(double) * 9 * N);
    const size_t o_init_records = a.reserve(sizeof(LevelRecord) * w.levels);
    w.input_bytes = a.size();
    // the target's hierarchy
    const size_t o_bvh_nodes = a.reserve(sizeof(float4) * 4 * std::max(1, w.F - 1));
    const size_t o_bvh_leaves = a.reserve(sizeof(float4) * kLeafFloat4s * w.F);
    // state and scratch
    size_t o_rot[2], o_trans[2], o_diag[2], o_rhs[2], o_off[2];
    for (int i = 0; i < 2; ++i) {
        o_rot[i] = a.reserve(sizeof(double) * 9 * N);
        o_trans[i] = a.reserve(sizeof(double) * 3 * N);
        o_diag[i] = a.reserve(sizeof(float) * 36 * N);
        o_rhs[i] = a.reserve(sizeof(float) * 6 * N);
        o_off[i] = a.reserve(sizeof(float) * 36 * 2 * B);
    }
    const size_t o_rot32 = a.reserve(sizeof(float) * 9 * N);
    const size_t o_deformed = a.reserve(sizeof(double) * 3 * V);
    const size_t o_deformed32 = a.reserve(sizeof(float4) * V);
    const size_t o_qn = a.reserve(sizeof(double) * 3 * V);
    const size_t o_cp = a.reserve(sizeof(double) * 3 * V);
    const size_t o_cn = a.reserve(sizeof(double) * 3 * V);
    const size_t o_cd = a.reserve(sizeof(double) * V);
    const size_t o_ct = a.reserve(sizeof(int32_t) * V);
    const size_t o_ll = a.reserve(sizeof(int32_t) * 2 * kLongCap);
    const size_t o_lc = a.reserve(sizeof(int32_t) * 2);
    const size_t o_lf = a.reserve(2 * static_cast<size_t>(V));
    const size_t o_cc = a.reserve(V);
    const size_t o_rb = a.reserve(sizeof(double) * V);
    const size_t o_r0 = a.reserve(sizeof(float4) * V);
    const size_t o_r1 = a.reserve(sizeof(float4) * V);
    const size_t o_r2 = a.reserve(sizeof(float4) * V);
    const size_t o_off32 = a.reserve(sizeof(float4) * kMaxSlots * V);
    const size_t o_factor = a.reserve(sizeof(float) * 36 * N);
    const size_t o_delta = a.reserve(sizeof(double) * 6 * N);
    const size_t o_x = a.reserve(sizeof(double) * 6 * N);
    const size_t o_r = a.reserve(sizeof(double) * 6 * N);
    const size_t o_p = a.reserve(sizeof(float) * 6 * N);
    const size_t o_ap = a.reserve(sizeof(float) * 6 * N);
    const size_t o_s = a.reserve(sizeof(float) * 6 * N);
    const size_t o_u = a.reserve(sizeof(float) * 6 * N);
    const int vblocks = (V + 255) / 256;
    const size_t o_part = a.reserve(sizeof(double) * kPartialStride * std::max(1, vblocks));
    const size_t o_epart = a.reserve(sizeof(double) * std::max(1, w.max_edges));
    const size_t o_npart = a.reserve(sizeof(double) * N);
    const size_t o_records = a.reserve(sizeof(LevelRecord) * w.levels);
    const size_t o_lstats = a.reserve(sizeof(CorrStats) * w.levels);
    const size_t o_fstats = a.reserve(sizeof(CorrStats));
    if (plan_only) {  // the arena's size only, nothing allocated
        const size_t bytes = a.size();
        a = Arena();
        return bytes;
    }
    if (pool) {
        a.allocate(pool, stream);
    } else {
        a.allocate();
    }
    const InputSink in{stream, staging, a.at<char>(0)};
    {
        // the state every run starts from: identity rotations, empty records
        std::vector<double> rot(static_cast<size_t>(N) * 9, 0.0);
        for (int n = 0; n < N; ++n) rot[n * 9] = rot[n * 9 + 4] = rot[n * 9 + 8] = 1.0;
        std::vector<LevelRecord> records(w.levels);
        std::memset(records.data(), 0, sizeof(LevelRecord) * records.size());
        for (int l = 0; l < w.levels; ++l) {
            records[l].level = l;
            records[l].nodes = w.layouts[l].node_count;
        }
        w.identity_rot = a.at<double>(o_identity);
        w.initial_records = a.at<LevelRecord>(o_init_records);
        in.put(w.identity_rot, rot);
        in.put(w.initial_records, records);
    }

    // ---- fill the descriptor ----
    WrapDev& D = w.dev;
    std::memset(&D, 0, sizeof D);
    D.V = V; D.T = w.T; D.Vt = w.Vt; D.F = w.F; D.L = w.L;
    D.max_nodes = w.max_nodes; D.max_offdiag = w.max_offdiag; D.max_pairs = w.max_pairs;
    D.max_edges = w.max_edges; D.energy_blocks = vblocks;
    const double units = w.graph.scale;
    for (int l = 0; l < kMaxLevels; ++l) {
        const NricpLevelSettings& s =
            w.level_settings[std::min<size_t>(l, w.level_settings.size() - 1)];
        D.weights[l][0] = s.point_to_point; D.weights[l][1] = s.point_to_plane;
        D.weights[l][2] = s.smoothness; D.weights[l][3] = s.anchor; D.weights[l][4] = s.landmark;
        D.robust_kernel[l] = s.robust_kernel;
        D.robust_threshold[l] = s.robust_threshold > 0.0 ? s.robust_threshold * units : s.robust_threshold;
        D.max_outer[l] = std::max(1, s.max_outer_iterations);
        D.max_inner[l] = std::max(1, s.max_inner_iterations);
        D.outer_tol[l] = s.outer_tolerance;
        D.inner_tol[l] = s.inner_tolerance;
    }
    D.distance_threshold = d.distance_threshold * units;  // bindings.cpp:631-639
    D.min_normal_cosine = d.min_normal_cosine;
    D.min_slope = d.min_slope;
    D.initial_damping = d.initial_damping;
    D.damping_decrease = d.damping_decrease;
    D.damping_increase = d.damping_increase;
    D.max_attempts = std::max(1, d.max_damping_attempts);
    D.diagonal_damping = d.diagonal_damping ? 1 : 0;
    D.pcg_max_iterations = std::max(1, d.pcg_max_iterations);
    D.pcg_tolerance = d.pcg_tolerance;

    // the template normalised with its own frame (written straight into the
    // staging area when there is one); the target goes up in the caller's
    // units and is normalised on the device, with its normals (ingest_target)
    std::vector<double> tpl_v;
    double* tpl;
    if (staging) {
        tpl = reinterpret_cast<double*>(staging + o_tpl);
        std::memcpy(staging + o_tgt, w.target_in.data(), sizeof(double) * 3 * w.Vt);
    } else {
        tpl_v.resize(static_cast<size_t>(V) * 3);
        tpl = tpl_v.data();
    }
    normalized_into(w.template_in.data(), V, w.graph.center, w.graph.scale, tpl);
    std::vector<double> lm_target(static_cast<size_t>(V) * 3, 0.0);
    std::vector<uint8_t> lm_flag(V, 0);
    for (int i = 0; i < w.L; ++i) {
        const int v = w.landmark_indices[i];
        lm_flag[v] = 1;
        for (int k = 0; k < 3; ++k)
            lm_target[v * 3 + k] = (w.landmark_targets_in[i * 3 + k] - w.graph.center[k]) * w.graph.scale;
    }
    D.tpl = a.at<double>(o_tpl);
    D.tpl_faces = a.at<int32_t>(o_tpl_faces);
    D.vf_begin = a.at<int32_t>(o_vf_begin);
    D.vf_faces = a.at<int32_t>(o_vf_list);
    D.mask = w.mask.empty() ? nullptr : a.at<uint8_t>(o_mask);
    D.lm_target = a.at<double>(o_lm_target);
    D.lm_flag = a.at<uint8_t>(o_lm_flag);
    D.lm_vertices = a.at<int32_t>(o_lm_vertices);
    D.tgt_points = a.at<double>(o_tgt);
    D.tgt_normals = a.at<double>(o_tgt_normals);
    D.tgt_faces = a.at<int32_t>(o_tgt_faces);
    D.bvh_nodes = a.at<float4>(o_bvh_nodes);
    D.bvh_leaves = a.at<float4>(o_bvh_leaves);
    D.rank_window = static_cast<float>(kRankWindow * normalized_diagonal(w.target_in.data(), w.Vt,
                                                                         w.graph.center, w.graph.scale));
    if (!staging) in.put(const_cast<double*>(D.tpl), tpl_v);
    in.put(const_cast<int32_t*>(D.tpl_faces), w.template_faces);
    in.put(const_cast<int32_t*>(D.vf_begin), vf_begin);
    in.put(const_cast<int32_t*>(D.vf_faces), vf_list);
    if (D.mask) in.put(const_cast<uint8_t*>(D.mask), w.mask);
    in.put(const_cast<double*>(D.lm_target), lm_target);
    in.put(const_cast<uint8_t*>(D.lm_flag), lm_flag);
    in.put(const_cast<int32_t*>(D.lm_vertices), w.landmark_indices);
    if (!staging) in.put(const_cast<double*>(D.tgt_points), w.target_in);
    in.put(const_cast<int32_t*>(D.tgt_faces), w.target_faces);

    for (int l = 0; l < w.levels; ++l) {
        const LevelLayout& L = w.layouts[l];
        LevelDev& G = D.levels[l];
        char* base = a.at<char>(level_base[l]);
        auto put = [&](const auto& vec) {
            using T = typename std::decay_t<decltype(vec)>::value_type;
            T* p = reinterpret_cast<T*>(base);
            base += (sizeof(T) * vec.size() + 255) & ~size_t(255);
            in.put(p, vec);
            return p;
        };
        G.node_count = L.node_count;
        G.edge_count = L.edge_count;
        G.pair_count = L.pair_count;
        G.offdiag_count = static_cast<int>(L.offdiag_nodes.size() / 2);
        G.rest = put(L.rest);
        G.bind_nodes = put(L.bind_nodes);
        G.bind_weights = put(L.bind_weights);
        G.bind_counts = put(L.bind_counts);
        G.gather_begin = put(L.gather_begin);
        G.gather_entry = put(L.gather_entry);
        G.node_edge_begin = put(L.node_edge_begin);
        G.node_edge_list = put(L.node_edge_list);
        G.edges = put(L.edges);
        G.pair_nodes = put(L.pair_nodes);
        G.pair_begin = put(L.pair_begin);
        G.pair_entry = put(L.pair_entry);
        G.row_begin = put(L.row_begin);
        G.row_entry = put(L.row_entry);
        G.offdiag_nodes = put(L.offdiag_nodes);
        G.offdiag_slots = put(L.offdiag_slots);
        G.edge_block = put(L.edge_block);
        G.row_entries = static_cast<int>(L.row_entry.size() / 2);
        G.transfer_nodes = put(L.transfer_nodes);
        G.transfer_weights = put(L.transfer_weights);
        G.transfer_counts = put(L.transfer_counts);
    }
    for (int i = 0; i < 2; ++i) {
        D.rot[i] = a.at<double>(o_rot[i]);
        D.trans[i] = a.at<double>(o_trans[i]);
        D.diag[i] = a.at<float>(o_diag[i]);
        D.rhs[i] = a.at<float>(o_rhs[i]);
        D.offdiag[i] = a.at<float>(o_off[i]);
    }
    D.rot32 = a.at<float>(o_rot32);
    D.deformed = a.at<double>(o_deformed);
    D.deformed32 = a.at<float4>(o_deformed32);
    D.qnormals = a.at<double>(o_qn);
    D.corr_point = a.at<double>(o_cp);
    D.corr_normal = a.at<double>(o_cn);
    D.corr_distance = a.at<double>(o_cd);
    D.corr_triangle = a.at<int32_t>(o_ct);
    D.long_list = a.at<int32_t>(o_ll);
    D.long_count = a.at<int32_t>(o_lc);
    D.long_flag = a.at<uint8_t>(o_lf);
    D.corr_code = a.at<uint8_t>(o_cc);
    D.robust = a.at<double>(o_rb);
    D.residual32 = a.at<float4>(o_r0);
    D.resid_aux32 = a.at<float4>(o_r1);
    D.lm_resid32 = a.at<float4>(o_r2);
    D.offsets32 = a.at<float4>(o_off32);
    D.factor = a.at<float>(o_factor);
    D.delta = a.at<double>(o_delta);
    D.pcg_x = a.at<double>(o_x);
    D.pcg_r = a.at<double>(o_r);
    D.pcg_p = a.at<float>(o_p);
    D.pcg_ap = a.at<float>(o_ap);
    D.pcg_s = a.at<float>(o_s);
    D.pcg_u = a.at<float>(o_u);
    D.partials = a.at<double>(o_part);
    D.edge_partials = a.at<double>(o_epart);
    D.node_partials = a.at<double>(o_npart);
    D.records = a.at<LevelRecord>(o_records);
    D.level_stats = a.at<CorrStats>(o_lstats);
    D.final_stats = a.at<CorrStats>(o_fstats);
    D.control = control;
    w.control = control;
    return a.size();
}

// Puts a wrap back at the start of its schedule: identity transforms, no
// previous correspondences, and a freshly built hierarchy of its target.  Runs
// on the device only (the inputs are already resident).
void reset_device(Wrap& w, cudaStream_t stream, void* lbvh_scratch, LbvhExport* lbvh_out) {
    WrapDev& D = w.dev;
    const int V = w.V, N = std::max(1, w.max_nodes);
    check(cudaMemcpyAsync(D.rot[0], w.identity_rot, sizeof(double) * 9 * N, cudaMemcpyDeviceToDevice, stream),
          "init rot");
    check(cudaMemsetAsync(D.trans[0], 0, sizeof(double) * 3 * N, stream), "init trans");
    check(cudaMemsetAsync(D.corr_triangle, 0xff, sizeof(int32_t) * V, stream), "init corr");
    check(cudaMemsetAsync(D.long_count, 0, sizeof(int32_t) * 2, stream), "init long walks");
    check(cudaMemsetAsync(D.long_flag, 0, 2 * static_cast<size_t>(V), stream), "init long walks");
    check(cudaMemsetAsync(D.corr_code, 0, V, stream), "init code");
    check(cudaMemcpyAsync(D.records, w.initial_records, sizeof(LevelRecord) * w.levels,
                          cudaMemcpyDeviceToDevice, stream), "init records");
    check(cudaMemsetAsync(D.level_stats, 0, sizeof(CorrStats) * w.levels, stream), "init stats");
    check(cudaMemsetAsync(D.final_stats, 0, sizeof(CorrStats), stream), "init stats");
    WrapControl& c = w.initial_control;
    std::memset(&c, 0, sizeof c);
    c.phase = kPhaseRefresh;
    c.route = w.desc.route;
    c.level = 0;
    c.level_count = w.levels;
    c.damping = w.desc.initial_damping;
    check(cudaMemcpyAsync(w.control, &c, sizeof c, cudaMemcpyHostToDevice, stream), "init control");

    // the target in the normalised frame and its normals, once after its
    // upload; then its hierarchy.  The batch's build scratch (sized for its
    // largest target) is reused by every wrap's build in stream order.
    if (!w.target_ingested) {
        ingest_target(const_cast<double*>(D.tgt_points), w.Vt, D.tgt_faces, w.F, w.graph.center,
                      w.graph.scale, const_cast<double*>(D.tgt_normals), lbvh_scratch, stream);
        check(cudaGetLastError(), "target ingestion");
        w.target_ingested = true;
    }
    const uint32_t root = lbvh_build(D.tgt_points, D.tgt_faces, w.F, lbvh_scratch,
                                     const_cast<float4*>(D.bvh_nodes), const_cast<float4*>(D.bvh_leaves),
                                     stream, lbvh_out);
    check(cudaGetLastError(), "lbvh build");
    D.bvh_root = static_cast<int>(root);
}

// Build scratch of one wrap's target structures (its ingestion, then its
// hierarchy, in stream order).
size_t build_scratch_bytes(const Wrap& w) {
    return std::max(lbvh_scratch_bytes(w.F), ingest_scratch_bytes(w.Vt, w.F));
}

// Kernels one hierarchy build launches (lbvh_build): centroids, two bound
// passes, Morton codes, 8 radix passes of 3 kernels, Karras, refit, 2 packs.
int lbvh_build_launches(int n) { return 4 + 8 * 3 + (n > 1 ? 1 : 0) + 1 + (n > 1 ? 2 : 1); }

// Kernels the target structures of a wrap launch per reset: the hierarchy.
int target_build_launches(const Wrap& w) { return lbvh_build_launches(w.F); }

}  // namespace

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------
Batch::Batch() {
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
}

Batch::~Batch() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (tail_graph_) cudaGraphExecDestroy(tail_graph_);
    if (tail_index_) cudaFree(tail_index_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (pool_) {  // back to the pool in stream order, without a device-wide wait
        for (auto& w : wraps_) w->arena.release_async(stream_);
        for (int k = 0; k < kBuildStreams; ++k)
            if (build_scratch_[k]) cudaFreeAsync(build_scratch_[k], stream_);
    }
    for (int k = 0; k < kBuildStreams; ++k) {
        if (build_streams_[k]) cudaStreamDestroy(build_streams_[k]);
        if (build_done_[k]) cudaEventDestroy(build_done_[k]);
    }
    if (build_fork_) cudaEventDestroy(build_fork_);
    wraps_.clear();
    if (query_counter_) cudaFree(query_counter_);
    if (side_stream_) cudaStreamDestroy(side_stream_);
    if (side_fork_) cudaEventDestroy(side_fork_);
    if (side_join_) cudaEventDestroy(side_join_);
    if (dev_wraps_) cudaFree(dev_wraps_);
    if (dev_controls_) cudaFree(dev_controls_);
    if (pcg_index_) cudaFree(pcg_index_);
    for (int g = 0; g < 5; ++g) {
        if (pcg_streams_[g]) cudaStreamDestroy(pcg_streams_[g]);
        if (pcg_join_[g]) cudaEventDestroy(pcg_join_[g]);
    }
    if (pcg_fork_) cudaEventDestroy(pcg_fork_);
    if (host_controls_) cudaFreeHost(host_controls_);
    if (stream_) cudaStreamDestroy(stream_);
}


void Batch::add(const NricpSolveDesc& desc) { add_all(&desc, 1); }

void Batch::add_all(const NricpSolveDesc* descs, int count) {
    // Inputs copied and checked on the host's cores (one wrap per thread),
    // every template graph built in one device pass (bit-identical to the
    // host build), then the level layouts on the host's cores again.
    std::vector<std::unique_ptr<Wrap>> prepared(count);
    std::vector<int> kind(count, 0);
    std::vector<std::string> message(count);
    auto guarded_step = [&](int i, auto&& step) {
        try {
            step();
        } catch (const InvalidArgument& e) {
            kind[i] = 1;
            message[i] = e.what();
        } catch (const CapacityError& e) {
            kind[i] = 2;
            message[i] = e.what();
        } catch (const std::bad_alloc&) {
            kind[i] = 3;
        } catch (const std::exception& e) {
            kind[i] = 4;
            message[i] = e.what();
        }
    };
    auto raise_first = [&] {
        for (int i = 0; i < count; ++i) {
            if (kind[i] == 1) throw InvalidArgument(message[i]);
            if (kind[i] == 2) throw CapacityError(message[i]);
            if (kind[i] == 3) throw std::bad_alloc();
            if (kind[i] == 4) throw std::runtime_error(message[i]);
        }
    };
    const double t0 = now_seconds();
#pragma omp parallel for schedule(dynamic, 1) if (count > 1)
    for (int i = 0; i < count; ++i)
        guarded_step(i, [&] {
            NricpSolveDesc d = descs[i];
            validate_settings(d);
            auto w = std::make_unique<Wrap>();
            copy_inputs(*w, d);
            check_graph_capacity(*w);
            prepared[i] = std::move(w);
        });
    raise_first();
    bool device = true;
    for (const auto& w : prepared) device = device && device_graph_supported(graph_request(*w).edge_neighbours);
    if (device) {
        std::vector<GraphRequest> requests;
        for (const auto& w : prepared) requests.push_back(graph_request(*w));
        std::vector<TemplateGraph> graphs = device_template_graphs(requests, stream_);
        for (int i = 0; i < count; ++i) prepared[i]->graph = std::move(graphs[i]);
    }
    if (device) {
        // the layouts: one task per (wrap, level), the largest first
        std::vector<std::pair<int, int>> tasks;
        for (int i = 0; i < count; ++i) {
            Wrap& w = *prepared[i];
            w.levels = static_cast<int>(w.graph.levels.size());
            w.layouts.assign(w.levels, LevelLayout{});
            for (int l = 0; l < w.levels; ++l) tasks.emplace_back(i, l);
        }
        auto work = [&](const std::pair<int, int>& t) {
            return static_cast<long>(prepared[t.first]->V) * (t.second + 1);
        };
        std::stable_sort(tasks.begin(), tasks.end(), [&](const auto& x, const auto& y) { return work(x) > work(y); });
        std::vector<std::string> failure(tasks.size());
#pragma omp parallel for schedule(dynamic, 1) if (tasks.size() > 1)
        for (long k = 0; k < static_cast<long>(tasks.size()); ++k) {
            Wrap& w = *prepared[tasks[k].first];
            try {
                w.layouts[tasks[k].second] = build_layout(w.graph, tasks[k].second, w.V);
            } catch (const std::exception& e) {
                failure[k] = e.what();
            }
        }
        for (size_t k = 0; k < tasks.size(); ++k)
            if (!failure[k].empty()) throw std::runtime_error(failure[k]);
        for (auto& w : prepared) {
            envelope(*w);
            // the layouts hold all the solve needs; the graph's per-vertex
            // bindings (about 100 bytes per vertex and level) go now
            std::vector<GraphLevel>().swap(w->graph.levels);
        }
    } else {
#pragma omp parallel for schedule(dynamic, 1) if (count > 1)
        for (int i = 0; i < count; ++i) guarded_step(i, [&] { prepare_host(*prepared[i]); });
        raise_first();
    }
    const double spent = (now_seconds() - t0) / std::max(1, count);
    for (auto& w : prepared) {
        w->setup_seconds = spent;
        wraps_.push_back(std::move(w));
    }
}

void Batch::upload_all(LbvhExport* lbvh_out) {
    const int W = static_cast<int>(wraps_.size());
    const double t0 = now_seconds();
    int device = 0;
    check(cudaGetDevice(&device), "device");
    pool_ = batch_pool(device);
    check(cudaMalloc(&dev_controls_, sizeof(WrapControl) * W), "cudaMalloc(controls)");
    check(cudaMallocHost(&host_controls_, sizeof(WrapControl) * W), "cudaMallocHost(controls)");
    size_t scratch_bytes = 0;
    for (const auto& w : wraps_) scratch_bytes = std::max(scratch_bytes, build_scratch_bytes(*w));
    for (int k = 0; k < kBuildStreams; ++k) {
        check(cudaMallocFromPoolAsync(&build_scratch_[k], scratch_bytes, pool_, stream_),
              "cudaMallocFromPoolAsync(scratch)");
        check(cudaStreamCreateWithFlags(&build_streams_[k], cudaStreamNonBlocking), "stream");
        check(cudaEventCreateWithFlags(&build_done_[k], cudaEventDisableTiming), "event");
    }
    check(cudaEventCreateWithFlags(&build_fork_, cudaEventDisableTiming), "event");
    // every wrap's input prefix, staged side by side in page-locked memory
    // on the host's cores, then one copy per wrap
    std::vector<size_t> offset(W + 1, 0);
#pragma omp parallel for schedule(dynamic, 1) if (W > 1)
    for (int i = 0; i < W; ++i) prepare_device(*wraps_[i], nullptr, nullptr, true);
    for (int i = 0; i < W; ++i) offset[i + 1] = offset[i] + ((wraps_[i]->input_bytes + 255) & ~size_t(255));
    StagingLease staging(offset[W]);
    std::vector<std::string> failure(W);
#pragma omp parallel for schedule(dynamic, 1) if (W > 1)
    for (int i = 0; i < W; ++i) {
        try {
            check(cudaSetDevice(device), "cudaSetDevice");  // this host thread's current device
            prepare_device(*wraps_[i], dev_controls_ + i, stream_, false, pool_, staging.data() + offset[i]);
        } catch (const std::exception& e) {
            failure[i] = e.what();
        }
    }
    for (int i = 0; i < W; ++i)
        if (!failure[i].empty()) throw std::runtime_error(failure[i]);
    shape_ = TickShape{};
    shape_.wraps = W;
    check(cudaMalloc(&query_counter_, 2 * sizeof(int)), "cudaMalloc(query queues)");
    shape_.query_counter = query_counter_;
    if (!side_stream_) {
        check(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking), "stream");
        check(cudaEventCreateWithFlags(&side_fork_, cudaEventDisableTiming), "event");
        check(cudaEventCreateWithFlags(&side_join_, cudaEventDisableTiming), "event");
    }
    shape_.side_stream = side_stream_;
    shape_.side_fork = side_fork_;
    shape_.side_join = side_join_;
    reset_all(staging.data(), &offset, lbvh_out);
    for (int i = 0; i < W; ++i) {
        Wrap& w = *wraps_[i];
        g_transfers.h2d += w.input_bytes;
        shape_.max_vertices = std::max(shape_.max_vertices, w.V);
        shape_.max_nodes = std::max(shape_.max_nodes, w.max_nodes);
        shape_.max_edges = std::max(shape_.max_edges, w.max_edges);
        shape_.max_pairs = std::max(shape_.max_pairs, w.max_pairs);
        if (w.desc.route == NRICP_ROUTE_C) shape_.route_c = 1;
    }
    set_pcg_cluster(default_pcg_cluster());
    check(cudaMalloc(&dev_wraps_, sizeof(WrapDev) * W), "cudaMalloc(wraps)");
    std::vector<WrapDev> host(W);
    for (int i = 0; i < W; ++i) host[i] = wraps_[i]->dev;
    check(cudaMemcpyAsync(dev_wraps_, host.data(), sizeof(WrapDev) * W, cudaMemcpyHostToDevice, stream_),
          "upload wraps");
    check(cudaStreamSynchronize(stream_), "prepare");  // the staging lease ends after this
    const double t = now_seconds();
    for (auto& w : wraps_) {
        w->setup_seconds += (t - t0) / std::max(1, W);
        w->solve_started = t;
    }
}

void Batch::reset_all(const char* staging, const std::vector<size_t>* offset, LbvhExport* lbvh_out) {
    check(cudaEventRecord(build_fork_, stream_), "event");
    for (int k = 0; k < kBuildStreams; ++k) check(cudaStreamWaitEvent(build_streams_[k], build_fork_, 0), "wait");
    for (size_t i = 0; i < wraps_.size(); ++i) {
        Wrap& w = *wraps_[i];
        const int k = static_cast<int>(i % kBuildStreams);
        if (staging)
            check(cudaMemcpyAsync(w.arena.base(), staging + (*offset)[i], w.input_bytes, cudaMemcpyHostToDevice,
                                  build_streams_[k]), "upload inputs");
        reset_device(w, build_streams_[k], build_scratch_[k], i == 0 ? lbvh_out : nullptr);
    }
    for (int k = 0; k < kBuildStreams; ++k) {
        check(cudaEventRecord(build_done_[k], build_streams_[k]), "event");
        check(cudaStreamWaitEvent(stream_, build_done_[k], 0), "wait");
    }
}

void Batch::reset() {
    check(cudaStreamSynchronize(stream_), "reset");
    reset_all(nullptr, nullptr, nullptr);
    for (auto& w : wraps_) w->solve_seconds = 0.0;
    ticks_ = 0;
    launches_ = 0;
    const double t = now_seconds();
    for (auto& w : wraps_) w->solve_started = t;
}

void Batch::tick(KernelTimers* timers) {
    const TickShape& shape = tail_on_ ? tail_shape_ : shape_;
    launch_tick(dev_wraps_, shape, stream_, timers);
    check(cudaGetLastError(), "tick launch");
    ticks_ += 1;
    launches_ += tick_kernel_launches(shape, timers && timers->active);
}

void Batch::pull_controls() {
    check(cudaMemcpyAsync(host_controls_, dev_controls_, sizeof(WrapControl) * wraps_.size(),
                          cudaMemcpyDeviceToHost, stream_), "pull controls");
    check(cudaStreamSynchronize(stream_), "tick");
}

bool Batch::all_done() const {
    for (size_t i = 0; i < wraps_.size(); ++i)
        if (host_controls_[i].phase != kPhaseDone) return false;
    return true;
}

// Per-wrap latency classes, halved until every class launch together needs
// at most three CTAs per SM (-s for nricp_batch_tune).  On the 64 uneven
// wraps of the benchmark that is one halving: the classes' CTAs then run in
// under three rounds of the SMs, while a second halving lengthens every
// solve iteration more than it saves.
int Batch::default_pcg_cluster() const {
    int device = 0, sms = 148;
    check(cudaGetDevice(&device), "device");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device");
    for (int shift = 0; shift < 4; ++shift) {
        long ctas = 0;
        for (const auto& w : wraps_) ctas += std::max(1, pcg_latency_cluster(w->max_nodes) >> shift);
        if (ctas <= 3L * sms) return -shift;
    }
    return -4;
}

void Batch::set_pcg_cluster(int cluster) {
    int device = 0;
    check(cudaGetDevice(&device), "device");
    check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device), "device");
    pcg_cluster_size(shape_.max_nodes, static_cast<int>(wraps_.size()), sms_);  // enables the launch attributes
    for (cudaGraphExec_t* g : {&graph_exec_, &tail_graph_})
        if (*g) {
            cudaGraphExecDestroy(*g);
            *g = nullptr;
        }
    tail_ready_ = tail_on_ = false;
    solve_shape(cluster, shape_, pcg_index_, nullptr);
    if (cluster < 0) {  // halved classes: halved once less for the tail
        tail_shape_ = shape_;
        solve_shape(cluster + 1, tail_shape_, tail_index_, &tail_cls_);
        tail_ready_ = true;
    }
}

void Batch::solve_shape(int cluster, TickShape& shape, int*& index, std::vector<int>* cls_out) {
    const int W = static_cast<int>(wraps_.size());
    std::vector<int> nodes(W);
    for (int i = 0; i < W; ++i) nodes[i] = wraps_[i]->max_nodes;
    shape.pcg_groups = 0;
    if (cluster > 0) {
        if (cluster > 16 || (cluster & (cluster - 1)) != 0)
            throw InvalidArgument("the solve's cluster size is a power of two from 1 to 16");
        shape.pcg_cluster = cluster;
        shape.pcg_shared_bytes = pcg_shared_bytes(nodes.data(), W, cluster);
        if (cls_out) cls_out->assign(W, cluster);
        return;
    }
    if (cluster < -4) throw InvalidArgument("the solve's class shift is 0 to 4");
    // one class per wrap: its own latency cluster, halved `shift` times
    const int shift = -cluster;
    std::vector<int> cls(W);
    for (int i = 0; i < W; ++i) cls[i] = std::max(1, pcg_latency_cluster(nodes[i]) >> shift);
    if (cls_out) *cls_out = cls;
    std::vector<int> sizes;
    for (int c = 16; c >= 1; c /= 2)
        if (std::count(cls.begin(), cls.end(), c) > 0) sizes.push_back(c);
    if (sizes.size() == 1) {
        shape.pcg_cluster = sizes[0];
        shape.pcg_shared_bytes = pcg_shared_bytes(nodes.data(), W, sizes[0]);
        return;
    }
    if (!index) check(cudaMalloc(&index, sizeof(int) * W), "cudaMalloc(solve groups)");
    std::vector<int> order;
    for (size_t g = 0; g < sizes.size(); ++g) {
        const int first = static_cast<int>(order.size());
        std::vector<int> members;
        for (int i = 0; i < W; ++i)
            if (cls[i] == sizes[g]) members.push_back(i);
        std::vector<int> member_nodes;
        for (int i : members) member_nodes.push_back(nodes[i]);
        order.insert(order.end(), members.begin(), members.end());
        shape.pcg_group_cluster[g] = sizes[g];
        shape.pcg_group_count[g] = static_cast<int>(members.size());
        shape.pcg_group_shared[g] = pcg_shared_bytes(member_nodes.data(), (int)members.size(), sizes[g]);
        shape.pcg_group_index[g] = index + first;
        if (g > 0 && !pcg_streams_[g]) {
            check(cudaStreamCreateWithFlags(&pcg_streams_[g], cudaStreamNonBlocking), "stream");
            check(cudaEventCreateWithFlags(&pcg_join_[g], cudaEventDisableTiming), "event");
        }
        shape.pcg_streams[g] = pcg_streams_[g];
        shape.pcg_join[g] = pcg_join_[g];
    }
    if (!pcg_fork_) check(cudaEventCreateWithFlags(&pcg_fork_, cudaEventDisableTiming), "event");
    shape.pcg_fork = pcg_fork_;
    check(cudaMemcpy(index, order.data(), sizeof(int) * W, cudaMemcpyHostToDevice), "solve groups");
    shape.pcg_groups = static_cast<int>(sizes.size());
    shape.pcg_cluster = sizes[0];
    shape.pcg_shared_bytes = shape.pcg_group_shared[0];
}

bool Batch::tail_due() const {
    long ctas = 0;
    for (size_t i = 0; i < wraps_.size(); ++i)
        if (host_controls_[i].phase != kPhaseDone) ctas += tail_cls_[i];
    return ctas <= sms_;
}

cudaGraphExec_t Batch::capture(const TickShape& shape) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
    launch_tick(dev_wraps_, shape, stream_, nullptr);
    check(cudaStreamEndCapture(stream_, &graph), "capture end");
    check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    return exec;
}

void Batch::run(int max_ticks) {
    if (!graph_exec_) graph_exec_ = capture(shape_);
    pull_controls();
    tail_on_ = false;
    int chunk = 4;
    while (!all_done()) {
        if (ticks_ >= max_ticks) throw StateError("the schedule did not finish within the tick limit");
        if (!tail_on_ && tail_ready_ && tail_due()) {
            tail_on_ = true;
            if (!tail_graph_) tail_graph_ = capture(tail_shape_);
        }
        for (int i = 0; i < chunk; ++i) {
            check(cudaGraphLaunch(tail_on_ ? tail_graph_ : graph_exec_, stream_), "graph launch");
            ticks_ += 1;
            launches_ += tick_kernel_launches(tail_on_ ? tail_shape_ : shape_);
        }
        pull_controls();
        chunk = std::min(chunk * 2, 16);
    }
    tail_on_ = false;
    finish();
}

void Batch::run_timed(KernelTimers* timers, std::vector<float>* query_ms, std::vector<float>* pcg_ms,
                      std::vector<float>* assemble_ms, int max_ticks) {
    records_.clear();
    cudaEvent_t tick_begin, tick_end;
    check(cudaEventCreate(&tick_begin), "event");
    check(cudaEventCreate(&tick_end), "event");
    pull_controls();
    tail_on_ = false;
    while (!all_done()) {
        if (ticks_ >= max_ticks) throw StateError("the schedule did not finish within the tick limit");
        if (!tail_on_ && tail_ready_ && tail_due()) tail_on_ = true;
        TickRecord r{};
        r.phase = host_controls_[0].phase;
        r.level = host_controls_[0].level;
        check(cudaEventRecord(tick_begin, stream_), "event");
        tick(timers);
        check(cudaEventRecord(tick_end, stream_), "event");
        pull_controls();
        r.pcg_iterations = r.phase == kPhaseSolve ? host_controls_[0].pcg_iterations : 0;
        cudaEventElapsedTime(&r.query_ms, timers->query_begin, timers->query_end);
        cudaEventElapsedTime(&r.pcg_ms, timers->pcg_begin, timers->pcg_end);
        cudaEventElapsedTime(&r.assemble_ms, timers->assemble_begin, timers->assemble_end);
        cudaEventElapsedTime(&r.tick_ms, tick_begin, tick_end);
        query_ms->push_back(r.query_ms);
        pcg_ms->push_back(r.pcg_ms);
        assemble_ms->push_back(r.assemble_ms);
        records_.push_back(r);
    }
    cudaEventDestroy(tick_begin);
    cudaEventDestroy(tick_end);
    tail_on_ = false;
    finish();
}

double Batch::timed_step() {
    cudaEvent_t begin, end;
    check(cudaEventCreate(&begin), "event");
    check(cudaEventCreate(&end), "event");
    check(cudaStreamSynchronize(stream_), "step");
    check(cudaEventRecord(begin, stream_), "event");
    reset_all(nullptr, nullptr, nullptr);
    ticks_ = 0;
    launches_ = 0;
    for (auto& w : wraps_) launches_ += target_build_launches(*w);
    run();
    check(cudaEventRecord(end, stream_), "event");
    check(cudaEventSynchronize(end), "step");
    float ms = 0.0f;
    check(cudaEventElapsedTime(&ms, begin, end), "event");
    cudaEventDestroy(begin);
    cudaEventDestroy(end);
    return ms;
}

void Batch::level_sizes(int i, int level, int* sizes) const {
    const Wrap& w = *wraps_[i];
    const LevelLayout& L = w.layouts[level];
    sizes[0] = L.node_count;
    sizes[1] = L.edge_count;
    sizes[2] = L.pair_count;
    sizes[3] = static_cast<int>(L.gather_entry.size());
    sizes[4] = static_cast<int>(L.pair_entry.size());
    sizes[5] = w.V;
    sizes[6] = w.F;
    sizes[7] = w.Vt;
    sizes[8] = w.T;
    sizes[9] = w.levels;
    // the work the last run did in this level
    LevelRecord r{};
    check(cudaMemcpy(&r, w.dev.records + level, sizeof r, cudaMemcpyDeviceToHost), "level record");
    sizes[10] = r.solves;
    sizes[11] = r.pcg_iterations;
    sizes[12] = r.queries;
    sizes[13] = r.assemblies;
    sizes[14] = static_cast<int>(L.offdiag_nodes.size() / 2);
    static_assert(kLevelSizeEntries == 15, "entries written above");
}

void Batch::finish() {
    const double t = now_seconds();
    for (size_t i = 0; i < wraps_.size(); ++i) {
        if (host_controls_[i].error)
            throw StateError("a closest-point traversal exceeded its stack; the hierarchy is too deep");
        if (wraps_[i]->solve_seconds == 0.0) wraps_[i]->solve_seconds = t - wraps_[i]->solve_started;
    }
}

const WrapControl& Batch::control(int i) const { return host_controls_[i]; }

void Batch::inspect(int i, NricpInspect* out) {
    pull_controls();
    const Wrap& w = *wraps_[i];
    const WrapControl& c = host_controls_[i];
    const int level = std::min(c.level, w.levels - 1);
    const LevelLayout& L = w.layouts[level];
    const int N = L.node_count, V = w.V;
    const int K = static_cast<int>(L.offdiag_nodes.size() / 2);
    out->level = level;
    out->node_count = N;
    out->phase = c.phase;
    out->off_count = K;
    for (int k = 0; k < kEnergyKinds; ++k) out->energies[k] = c.energy_parts[k];
    if (out->off_capacity < K) throw InvalidArgument("off-diagonal capacity too small");
    const WrapDev& D = w.dev;
    auto get = [this](void* dst, const void* src, size_t bytes) {  // a null output is skipped
        if (dst) check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_), "inspect");
    };
    get(out->rotations, D.rot[c.state], sizeof(double) * 9 * N);
    get(out->translations, D.trans[c.state], sizeof(double) * 3 * N);
    get(out->corr_points, D.corr_point, sizeof(double) * 3 * V);
    get(out->corr_normals, D.corr_normal, sizeof(double) * 3 * V);
    get(out->corr_robust, D.robust, sizeof(double) * V);
    get(out->corr_codes, D.corr_code, V);
    get(out->diag, D.diag[c.system], sizeof(float) * 36 * N);
    get(out->rhs, D.rhs[c.system], sizeof(float) * 6 * N);
    get(out->delta, D.delta, sizeof(double) * 6 * N);
    get(out->corr_distances, D.corr_distance, sizeof(double) * V);
    get(out->target_points, D.tgt_points, sizeof(double) * 3 * w.Vt);
    get(out->target_normals, D.tgt_normals, sizeof(double) * 3 * w.Vt);
    out->damping = c.damping;
    out->pcg_ok = c.pcg_ok;
    out->pcg_iterations = c.pcg_iterations;
    out->pcg_residual = c.pcg_residual;
    std::vector<float> rows(out->off_nodes && out->off_blocks ? L.row_entry.size() / 2 * 36 : 0);
    if (!rows.empty()) get(rows.data(), D.offdiag[c.system], sizeof(float) * rows.size());
    check(cudaStreamSynchronize(stream_), "inspect");
    for (int k = 0; k < K && !rows.empty(); ++k) {
        out->off_nodes[k * 2] = L.offdiag_nodes[k * 2];
        out->off_nodes[k * 2 + 1] = L.offdiag_nodes[k * 2 + 1];
        const float* block = rows.data() + static_cast<size_t>(L.offdiag_slots[k * 2]) * 36;
        std::copy(block, block + 36, out->off_blocks + static_cast<size_t>(k) * 36);
    }
}

namespace {

// v' = sum w (R (v - g) + g + t), then back to the caller's units
// (mesh.cpp:189-193).
std::vector<double> evaluate_host(const Wrap& w, const std::vector<double>& rot,
                                  const std::vector<double>& trans, int level) {
    const LevelLayout& L = w.layouts[level];
    const std::vector<double> tpl = normalized(w.template_in.data(), w.V, w.graph.center, w.graph.scale);
    std::vector<double> out(static_cast<size_t>(w.V) * 3);
    for (int v = 0; v < w.V; ++v) {
        double s[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < L.bind_counts[v]; ++k) {
            const int j = L.bind_nodes[v * NRICP_MAX_SLOTS + k];
            const double wt = L.bind_weights[v * NRICP_MAX_SLOTS + k];
            const double* g = &L.rest[j * 3];
            const double* R = &rot[j * 9];
            const double p[3] = {tpl[v * 3] - g[0], tpl[v * 3 + 1] - g[1], tpl[v * 3 + 2] - g[2]};
            for (int r = 0; r < 3; ++r) {
                const double a = R[r * 3] * p[0] + R[r * 3 + 1] * p[1] + R[r * 3 + 2] * p[2];
                s[r] = s[r] + ((a + g[r]) + trans[j * 3 + r]) * wt;
            }
        }
        for (int r = 0; r < 3; ++r) out[v * 3 + r] = s[r] / w.graph.scale + w.graph.center[r];
    }
    return out;
}

// What a finished (or paused) wrap's result needs from the device.
struct WrapDownload {
    WrapControl control{};
    std::vector<double> rot, trans;
    std::vector<LevelRecord> records;
    std::vector<CorrStats> lstats;
    CorrStats fstats{};
};

WrapDownload download_result(const Wrap& w, const WrapControl& c, cudaStream_t stream) {
    WrapDownload d;
    d.control = c;
    const int level = std::min(c.level, w.levels - 1);
    const int N = w.layouts[level].node_count;
    d.rot.resize(static_cast<size_t>(N) * 9);
    d.trans.resize(static_cast<size_t>(N) * 3);
    d.records.resize(w.levels);
    d.lstats.resize(w.levels);
    check(cudaMemcpyAsync(d.rot.data(), w.dev.rot[c.state], sizeof(double) * d.rot.size(),
                          cudaMemcpyDeviceToHost, stream), "download rot");
    check(cudaMemcpyAsync(d.trans.data(), w.dev.trans[c.state], sizeof(double) * d.trans.size(),
                          cudaMemcpyDeviceToHost, stream), "download trans");
    check(cudaMemcpyAsync(d.records.data(), w.dev.records, sizeof(LevelRecord) * w.levels,
                          cudaMemcpyDeviceToHost, stream), "download records");
    check(cudaMemcpyAsync(d.lstats.data(), w.dev.level_stats, sizeof(CorrStats) * w.levels,
                          cudaMemcpyDeviceToHost, stream), "download stats");
    check(cudaMemcpyAsync(&d.fstats, w.dev.final_stats, sizeof(CorrStats), cudaMemcpyDeviceToHost,
                          stream), "download stats");
    check(cudaStreamSynchronize(stream), "download");
    g_transfers.d2h += sizeof(double) * (d.rot.size() + d.trans.size()) +
                       sizeof(LevelRecord) * d.records.size() +
                       sizeof(CorrStats) * (d.lstats.size() + 1) + sizeof(WrapControl);
    return d;
}

// Result of one wrap in the caller's units (route_result_to_dict,
// src/python/bindings.cpp:674-710), from its downloaded state; host only.
void compose_result(const Wrap& w, const WrapDownload& d, NricpResult* out) {
    const WrapControl& c = d.control;
    const int level = std::min(c.level, w.levels - 1);
    const int N = w.layouts[level].node_count;
    const std::vector<double> vertices = evaluate_host(w, d.rot, d.trans, level);
    if (out->vertices) std::memcpy(out->vertices, vertices.data(), sizeof(double) * vertices.size());
    if (out->rotations) std::memcpy(out->rotations, d.rot.data(), sizeof(double) * d.rot.size());
    if (out->translations) std::memcpy(out->translations, d.trans.data(), sizeof(double) * d.trans.size());
    if (out->node_positions)
        std::memcpy(out->node_positions, w.layouts[level].rest.data(), sizeof(double) * 3 * N);
    if (out->level_nodes)
        for (int l = 0; l < w.levels; ++l) out->level_nodes[l] = w.layouts[l].node_count;
    // The report: levels run so far, the final correspondence statistics
    // (route_a.cpp:40-63) and the accepted energy's five parts.
    std::vector<LevelView> views;
    const int shown = c.phase == kPhaseDone || c.phase == kPhaseFinal ? w.levels : c.level + 1;
    for (int l = 0; l < shown && l < w.levels; ++l) {
        const LevelRecord& r = d.records[l];
        views.push_back({l, r.nodes, r.outer_iterations, r.inner_iterations, r.converged,
                         r.energy_start, r.energy_end, r.correspondence_mean});
    }
    const CorrStats& s = c.phase == kPhaseDone ? d.fstats : d.lstats[std::max(0, c.level - 1)];
    const StatsView stats{s.total, s.accepted, s.rejected_distance, s.rejected_normal,
                          s.rejected_slope, s.rejected_masked, s.mean, s.p95, s.max};
    const std::string json = report_json(c.route == 0 ? "route_b" : "route_c", "float",
                                         c.energy_parts, stats, views, w.desc, w.graph.scale,
                                         w.setup_seconds, w.solve_seconds);
    out->report_length = json.size();
    if (out->report_json && out->report_capacity > 0) {
        const size_t n = std::min(json.size(), out->report_capacity - 1);
        std::memcpy(out->report_json, json.data(), n);
        out->report_json[n] = 0;
    }
}

void write_result(const Wrap& w, const WrapControl& c, cudaStream_t stream, NricpResult* out) {
    compose_result(w, download_result(w, c, stream), out);
}

}  // namespace

void Batch::result(int i, NricpResult* out) { write_result(*wraps_[i], host_controls_[i], stream_, out); }

void Batch::results(NricpResult* outs) {
    const int W = static_cast<int>(wraps_.size());
    std::vector<WrapDownload> downloads;
    downloads.reserve(W);
    for (int i = 0; i < W; ++i) downloads.push_back(download_result(*wraps_[i], host_controls_[i], stream_));
    // vertices in FP64 and the reports, on the host's cores
    std::vector<std::string> failure(W);
#pragma omp parallel for schedule(dynamic, 1) if (W > 1)
    for (int i = 0; i < W; ++i) {
        try {
            compose_result(*wraps_[i], downloads[i], &outs[i]);
        } catch (const std::exception& e) {
            failure[i] = e.what();
        }
    }
    for (int i = 0; i < W; ++i)
        if (!failure[i].empty()) throw std::runtime_error(failure[i]);
}

std::vector<double> Batch::evaluate_host(int i, const std::vector<double>& rot,
                                         const std::vector<double>& trans, int level) const {
    return nricp_b200::evaluate_host(*wraps_[i], rot, trans, level);
}

int Batch::finest_nodes(int i) const { return wraps_[i]->layouts.back().node_count; }
int Batch::levels(int i) const { return wraps_[i]->levels; }
int Batch::vertices(int i) const { return wraps_[i]->V; }

void Batch::current_vertices(int i, double* out) {
    pull_controls();
    const WrapControl& c = host_controls_[i];
    Wrap& w = *wraps_[i];
    const int level = std::min(c.level, w.levels - 1);
    // a level whose warm start has not run yet still holds the previous one
    const int shown = c.phase == kPhaseTransfer ? level - 1 : level;
    const int N = w.layouts[shown].node_count;
    std::vector<double> rot(static_cast<size_t>(N) * 9), trans(static_cast<size_t>(N) * 3);
    check(cudaMemcpyAsync(rot.data(), w.dev.rot[c.state], sizeof(double) * rot.size(),
                          cudaMemcpyDeviceToHost, stream_), "download rot");
    check(cudaMemcpyAsync(trans.data(), w.dev.trans[c.state], sizeof(double) * trans.size(),
                          cudaMemcpyDeviceToHost, stream_), "download trans");
    check(cudaStreamSynchronize(stream_), "download");
    const std::vector<double> v = evaluate_host(i, rot, trans, shown);
    std::memcpy(out, v.data(), sizeof(double) * v.size());
}

const WrapDev* Batch::device_wrap(int i) const { return dev_wraps_ + i; }


// ---------------------------------------------------------------------------
// Server: continuous batching
// ---------------------------------------------------------------------------
namespace {

// A template's graph and level layouts, shared by every request that wraps
// the same template with the same graph settings.
struct TemplateEntry {
    TemplateGraph graph;
    std::vector<LevelLayout> layouts;
    int levels = 0, max_nodes = 0, max_edges = 0, max_pairs = 0, max_offdiag = 0;
};

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < bytes; ++i) h = (h ^ p[i]) * 1099511628211ull;
    return h;
}

uint64_t template_key(const Wrap& w) {
    const NricpSolveDesc& d = w.desc;
    const int settings[5] = {d.graph_levels, d.nodes_initial, d.growth, d.max_nodes_per_vertex,
                             d.edge_neighbours};
    uint64_t h = 14695981039346656037ull;
    h = fnv1a(w.template_in.data(), sizeof(double) * w.template_in.size(), h);
    h = fnv1a(w.template_faces.data(), sizeof(int32_t) * w.template_faces.size(), h);
    return fnv1a(settings, sizeof settings, h);
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t k = static_cast<size_t>(std::ceil(q * v.size()));
    return v[std::min(v.size() - 1, k > 0 ? k - 1 : 0)];
}

}  // namespace

struct Server::Impl {
    struct Request {
        long id = 0;
        std::unique_ptr<Wrap> wrap;
        int state = NRICP_REQUEST_WAITING;
        bool invalid = false;
        std::string error;
        // submit, graph and layouts built, loader done (uploads and hierarchy
        // enqueued), placed in a slot, finished on the device, result ready
        double t_submit = 0.0, t_prepared = 0.0, t_loaded = 0.0, t_admit = 0.0, t_retired = 0.0,
               t_done = 0.0;
        size_t bytes = 0;
        cudaEvent_t loaded = nullptr;  // the wrap's uploads and hierarchy are on the device
        std::unique_ptr<WrapDownload> download;  // a finished wrap's state, for the finisher
        std::vector<double> vertices, rotations, translations, nodes;
        std::vector<int32_t> level_nodes;
        std::string report;
    };
    using RequestPtr = std::shared_ptr<Request>;
    // A retired wrap whose arena is freed once `after` (recorded on the tick
    // stream after its last use) has passed.
    struct Dead {
        Arena arena;
        size_t bytes = 0;
        cudaEvent_t after = nullptr;
    };

    NricpServerConfig cfg{};
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;       // ticks, placement, results
    static constexpr int kLoaders = 4;
    cudaStream_t load_streams[kLoaders] = {};  // allocation, uploads, hierarchy builds, frees
    cudaMemPool_t pool = nullptr;
    WrapDev* dev_wraps = nullptr;
    WrapControl* dev_controls = nullptr;
    WrapControl* host_controls = nullptr;
    WrapControl* staging_controls = nullptr;  // where each loader's reset writes its wrap's control
    std::vector<WrapDev> host_wraps;
    std::vector<RequestPtr> slot_req;    // the running request of each slot, or null
    std::vector<int> slot_nodes;
    int slots_used = 0;
    size_t resident = 0, peak = 0;
    void* lbvh_scratch[kLoaders] = {};   // each loader's, on its stream, from the pool
    size_t lbvh_bytes[kLoaders] = {};
    TickShape shape{};                   // size envelope of every wrap placed so far
    std::map<int, cudaGraphExec_t> graphs;  // one tick graph per running-wrap count

    // Per-class solve launches: class g (cluster size class_top >> g) reads
    // its slots from row g of class_index, -1 past its members; the rows are
    // rewritten whenever the running set changes.
    int class_top = 0, class_count = 0;  // 0 classes: one uniform launch
    int* class_index = nullptr;          // class_count x max_slots, device
    std::vector<int> class_rows;         // what class_index holds now
    cudaStream_t class_streams[5] = {};
    cudaEvent_t class_fork = nullptr, class_join[5] = {};

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<long, RequestPtr> requests;
    std::deque<RequestPtr> prep_queue, ready, loaded;
    std::deque<Dead> graveyard;
    std::deque<RequestPtr> finishing;
    long next_id = 1;
    int running = 0, loading = 0;
    bool stop = false;
    std::vector<std::thread> preppers;
    std::thread pump_thread, finisher_thread;
    std::vector<std::thread> loader_threads;
    std::mutex cache_mu;
    std::map<uint64_t, std::shared_ptr<const TemplateEntry>> cache;

    long submitted = 0, completed = 0, failed = 0, ticks = 0, launches = 0, captures = 0;
    double busy_seconds = 0.0;
    cudaEvent_t tick_begin = nullptr, tick_end = nullptr;
    int* query_counter = nullptr;        // the query queues' heads (vertices, long walks)
    std::vector<double> latencies, queue_waits;
    double first_submit = -1.0, last_done = 0.0;

    void prepare_cached(Wrap& w) {
        const uint64_t key = template_key(w);
        std::shared_ptr<const TemplateEntry> entry;
        {
            std::lock_guard<std::mutex> lk(cache_mu);
            auto it = cache.find(key);
            if (it != cache.end()) entry = it->second;
        }
        if (!entry) {
            prepare_host(w);
            auto fresh = std::make_shared<TemplateEntry>();
            fresh->graph = w.graph;
            fresh->layouts = w.layouts;
            fresh->levels = w.levels;
            fresh->max_nodes = w.max_nodes;
            fresh->max_edges = w.max_edges;
            fresh->max_pairs = w.max_pairs;
            fresh->max_offdiag = w.max_offdiag;
            std::lock_guard<std::mutex> lk(cache_mu);
            cache.emplace(key, std::move(fresh));
            return;
        }
        w.graph = entry->graph;
        w.layouts = entry->layouts;
        w.levels = entry->levels;
        w.max_nodes = entry->max_nodes;
        w.max_edges = entry->max_edges;
        w.max_pairs = entry->max_pairs;
        w.max_offdiag = entry->max_offdiag;
    }

    void fail(const RequestPtr& r, const std::string& why, bool invalid) {
        // caller holds `mu`
        r->state = NRICP_REQUEST_FAILED;
        r->error = why;
        r->invalid = invalid;
        failed += 1;
        cv_done.notify_all();
    }

    // Host threads: graph and layouts (cached per template), arena size.
    void prep_loop() {
        while (true) {
            RequestPtr r;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !prep_queue.empty(); });
                if (stop) return;
                r = prep_queue.front();
                prep_queue.pop_front();
            }
            std::string why;
            bool invalid = false;
            try {
                prepare_cached(*r->wrap);
                r->bytes = prepare_device(*r->wrap, nullptr, nullptr, true);
            } catch (const InvalidArgument& e) {
                why = e.what();
                invalid = true;
            } catch (const std::exception& e) {
                why = e.what();
            }
            std::lock_guard<std::mutex> lk(mu);
            r->t_prepared = now_seconds();
            if (why.empty()) {
                ready.push_back(r);
            } else {
                fail(r, why, invalid);
            }
            cv_work.notify_all();
        }
    }

    bool can_load() const {
        // caller holds `mu`; never more wraps on the device than slots
        return !ready.empty() && running + loading + static_cast<int>(loaded.size()) < cfg.max_slots;
    }

    // Loader threads, each on its own stream: arenas from the pool, uploads,
    // the target's hierarchy and the start state, in budget order; and the
    // frees of retired arenas.  Nothing here waits for the tick stream.
    void loader_loop(int k) {
        cudaSetDevice(device);
        cudaStream_t load_stream = load_streams[k];
        while (true) {
            RequestPtr r;
            std::deque<Dead> dead;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    return stop || !graveyard.empty() ||
                           (can_load() && resident + ready.front()->bytes <= cfg.memory_budget_bytes) ||
                           (!ready.empty() && ready.front()->bytes > cfg.memory_budget_bytes);
                });
                if (stop) return;
                dead.swap(graveyard);
                while (!ready.empty() && ready.front()->bytes > cfg.memory_budget_bytes) {
                    RequestPtr big = ready.front();
                    ready.pop_front();
                    fail(big, "the wrap needs " + std::to_string(big->bytes) +
                                  " device bytes, more than the server's budget of " +
                                  std::to_string(cfg.memory_budget_bytes), false);
                }
                if (can_load() && resident + ready.front()->bytes <= cfg.memory_budget_bytes) {
                    r = ready.front();
                    ready.pop_front();
                    resident += r->bytes;
                    peak = std::max(peak, resident);
                    loading += 1;
                }
            }
            size_t freed = 0;
            for (Dead& d : dead) {
                cudaStreamWaitEvent(load_stream, d.after, 0);
                d.arena.release_async(load_stream);
                cudaEventDestroy(d.after);
                freed += d.bytes;
            }
            if (freed) {
                std::lock_guard<std::mutex> lk(mu);
                resident -= freed;
                cv_work.notify_all();
            }
            if (!r) continue;
            std::string why;
            try {
                Wrap& w = *r->wrap;
                prepare_device(w, staging_controls + k, load_stream, false, pool);
                const size_t need = build_scratch_bytes(w);
                if (need > lbvh_bytes[k]) {
                    if (lbvh_scratch[k]) check(cudaFreeAsync(lbvh_scratch[k], load_stream), "scratch");
                    lbvh_scratch[k] = nullptr;
                    check(cudaMallocFromPoolAsync(&lbvh_scratch[k], need, pool, load_stream), "scratch");
                    lbvh_bytes[k] = need;
                }
                reset_device(w, load_stream, lbvh_scratch[k], nullptr);
                check(cudaEventCreateWithFlags(&r->loaded, cudaEventDisableTiming), "event");
                check(cudaEventRecord(r->loaded, load_stream), "event");
            } catch (const std::exception& e) {
                why = e.what();
            }
            std::lock_guard<std::mutex> lk(mu);
            loading -= 1;
            r->t_loaded = now_seconds();
            if (why.empty()) {
                loaded.push_back(r);
            } else {
                resident -= r->bytes;
                if (r->wrap) r->wrap.reset();
                fail(r, why, false);
            }
            cv_work.notify_all();
        }
    }

    void grow_shape(const Wrap& w) {
        const TickShape before = shape;
        shape.max_vertices = std::max(shape.max_vertices, w.V);
        shape.max_nodes = std::max(shape.max_nodes, w.max_nodes);
        shape.max_edges = std::max(shape.max_edges, w.max_edges);
        shape.max_pairs = std::max(shape.max_pairs, w.max_pairs);
        if (w.desc.route == NRICP_ROUTE_C) shape.route_c = 1;
        if (std::memcmp(&before, &shape, sizeof shape) != 0) {
            for (auto& [count, g] : graphs) cudaGraphExecDestroy(g);
            graphs.clear();
        }
    }

    // The tick over the first `count` slots (the running wraps are kept in
    // slots 0 .. count-1), captured once per count and size envelope.
    cudaGraphExec_t graph_for(int count) {
        auto it = graphs.find(count);
        if (it != graphs.end()) return it->second;
        TickShape t = shape;
        t.wraps = count;
        t.pcg_groups = 0;
        pcg_cluster_size(t.max_nodes, count, sms);  // enables the launch attributes
        if (class_count == 0) {
            t.pcg_cluster = cfg.pcg_cluster;
            std::vector<int> nodes(count, t.max_nodes);  // any wrap may take any slot
            t.pcg_shared_bytes = pcg_shared_bytes(nodes.data(), count, t.pcg_cluster);
        } else {
            // every class launch covers `count` entries; a class's shared
            // memory is what its largest possible member would use
            for (int g = 0; g < class_count; ++g) {
                const int cluster = class_top >> g;
                const int nodes = std::min(t.max_nodes, class_node_bound(cluster));
                t.pcg_group_cluster[g] = cluster;
                t.pcg_group_count[g] = count;
                t.pcg_group_shared[g] = pcg_shared_bytes(&nodes, 1, cluster);
                t.pcg_group_index[g] = class_index + static_cast<size_t>(g) * cfg.max_slots;
                t.pcg_streams[g] = class_streams[g];
                t.pcg_join[g] = class_join[g];
            }
            t.pcg_fork = class_fork;
            t.pcg_groups = class_count;
            t.pcg_cluster = class_top;
            t.pcg_shared_bytes = t.pcg_group_shared[0];
        }
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
        launch_tick(dev_wraps, t, stream, nullptr);
        check(cudaStreamEndCapture(stream, &g), "capture end");
        check(cudaGraphInstantiate(&exec, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        captures += 1;
        launches_per_tick[count] = tick_kernel_launches(t);
        graphs[count] = exec;
        return exec;
    }
    std::map<int, int> launches_per_tick;

    // A wrap's class is its latency cluster halved `shift` times: a fixed
    // shift (pcg_cluster < 0), or by load (0) -- none while the running
    // wraps' latency clusters fit three CTAs per SM, else one.
    int max_shift() const { return cfg.pcg_cluster < 0 ? -cfg.pcg_cluster : 1; }
    int shift_for(int count) const {
        if (cfg.pcg_cluster < 0) return -cfg.pcg_cluster;
        long ctas = 0;
        for (int i = 0; i < count; ++i) ctas += pcg_latency_cluster(slot_nodes[i]);
        return ctas <= 3L * sms ? 0 : 1;
    }
    static int class_of(int nodes, int shift) { return std::max(1, pcg_latency_cluster(nodes) >> shift); }
    // The most nodes a wrap of class `cluster` can have: its latency cluster
    // is at most cluster << max_shift, which covers up to 128 nodes per CTA
    // below 16.
    int class_node_bound(int cluster) const {
        const int latency = cluster << max_shift();
        return latency >= 16 ? pcg_max_nodes() : latency * 128;
    }

    // Rewrites the class rows for the running wraps in slots 0 .. count-1
    // (tick stream order: the next tick reads them).
    void upload_classes(int count) {
        if (class_count == 0) return;
        std::vector<int> rows(static_cast<size_t>(class_count) * cfg.max_slots, -1);
        std::vector<int> fill(class_count, 0);
        const int shift = shift_for(count);
        for (int i = 0; i < count; ++i) {
            int g = 0;
            while ((class_top >> g) > class_of(slot_nodes[i], shift)) ++g;
            rows[static_cast<size_t>(g) * cfg.max_slots + fill[g]++] = i;
        }
        if (rows == class_rows) return;
        class_rows = rows;
        check(cudaMemcpyAsync(class_index, class_rows.data(), sizeof(int) * class_rows.size(),
                              cudaMemcpyHostToDevice, stream), "solve classes");
    }

    // Moves the running wrap of slot `from` into the free slot `to`: its
    // control block (device to device) and its descriptor.
    void move_slot(int from, int to) {
        RequestPtr r = slot_req[from];
        Wrap& w = *r->wrap;
        check(cudaMemcpyAsync(dev_controls + to, dev_controls + from, sizeof(WrapControl),
                              cudaMemcpyDeviceToDevice, stream), "move control");
        w.control = dev_controls + to;
        w.dev.control = w.control;
        host_wraps[to] = w.dev;
        check(cudaMemcpyAsync(dev_wraps + to, &host_wraps[to], sizeof(WrapDev), cudaMemcpyHostToDevice,
                              stream), "move descriptor");
        host_controls[to] = host_controls[from];
        slot_req[to] = r;
        slot_req[from] = nullptr;
    }

    // Downloads a finished wrap's result buffers (tick thread); the host
    // work -- vertices in FP64, the report -- is the finisher's.
    void retire(int slot, const RequestPtr& r) {
        r->wrap->solve_seconds = now_seconds() - r->t_admit;
        r->download = std::make_unique<WrapDownload>(download_result(*r->wrap, host_controls[slot], stream));
    }

    void compose(const RequestPtr& r) {
        Wrap& w = *r->wrap;
        const int N = w.layouts.back().node_count;
        r->vertices.assign(static_cast<size_t>(w.V) * 3, 0.0);
        r->rotations.assign(static_cast<size_t>(N) * 9, 0.0);
        r->translations.assign(static_cast<size_t>(N) * 3, 0.0);
        r->nodes.assign(static_cast<size_t>(N) * 3, 0.0);
        r->level_nodes.assign(w.levels, 0);
        std::vector<char> report(1 << 20);
        NricpResult out{r->vertices.data(), r->rotations.data(), r->translations.data(),
                        r->nodes.data(), r->level_nodes.data(), report.data(), report.size(), 0};
        compose_result(w, *r->download, &out);
        r->report.assign(report.data(), std::min(out.report_length, report.size() - 1));
    }

    void finish_loop() {
        while (true) {
            RequestPtr r;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !finishing.empty(); });
                if (stop) return;
                r = finishing.front();
                finishing.pop_front();
            }
            std::string why;
            try {
                compose(r);
            } catch (const std::exception& e) {
                why = e.what();
            }
            r->download.reset();
            r->wrap.reset();  // host side; the arena went back to the pool at retirement
            std::lock_guard<std::mutex> lk(mu);
            if (!why.empty()) {
                fail(r, why, false);
                continue;
            }
            r->state = NRICP_REQUEST_DONE;
            r->t_done = now_seconds();
            latencies.push_back(r->t_done - r->t_submit);
            last_done = std::max(last_done, r->t_done);
            completed += 1;
            cv_done.notify_all();
        }
    }

    // Hands a retired wrap's arena to the loader.  A finished wrap's tick
    // kernels read only its control block (its slot's entry in dev_controls,
    // which stays), so the arena can go as soon as the tick stream passes
    // this point.
    void bury(const RequestPtr& r) {
        Dead d;
        d.bytes = r->bytes;
        d.arena = r->wrap->arena;  // the device arena leaves; the host side stays for the finisher
        r->wrap->arena = Arena();
        check(cudaEventCreateWithFlags(&d.after, cudaEventDisableTiming), "event");
        check(cudaEventRecord(d.after, stream), "event");
        std::lock_guard<std::mutex> lk(mu);
        graveyard.push_back(std::move(d));
        cv_work.notify_all();
    }

    // The tick thread: places loaded wraps into free slots, launches ticks,
    // retires finished wraps.
    void pump_loop() {
        cudaSetDevice(device);
        const int per_poll = cfg.ticks_per_poll > 0 ? cfg.ticks_per_poll : 8;
        while (true) {
            std::vector<std::pair<int, RequestPtr>> placing;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || running > 0 || !loaded.empty(); });
                if (stop) return;
                while (!loaded.empty() && running < cfg.max_slots) {
                    RequestPtr r = loaded.front();
                    if (running > 0 && cudaEventQuery(r->loaded) == cudaErrorNotReady) break;
                    const int slot = running;  // running wraps stay in slots 0 .. running-1
                    loaded.pop_front();
                    slot_req[slot] = r;
                    slots_used = std::max(slots_used, slot + 1);
                    r->state = NRICP_REQUEST_RUNNING;
                    r->t_admit = now_seconds();
                    queue_waits.push_back(r->t_admit - r->t_submit);
                    running += 1;
                    placing.emplace_back(slot, r);
                }
            }
            int count = 0;
            try {
                for (auto& [slot, r] : placing) {
                    Wrap& w = *r->wrap;
                    check(cudaStreamWaitEvent(stream, r->loaded, 0), "wait loaded");
                    cudaEventDestroy(r->loaded);
                    r->loaded = nullptr;
                    w.control = dev_controls + slot;
                    w.dev.control = w.control;
                    host_wraps[slot] = w.dev;
                    check(cudaMemcpyAsync(dev_controls + slot, &w.initial_control, sizeof(WrapControl),
                                          cudaMemcpyHostToDevice, stream), "slot control");
                    check(cudaMemcpyAsync(dev_wraps + slot, &host_wraps[slot], sizeof(WrapDev),
                                          cudaMemcpyHostToDevice, stream), "slot descriptor");
                    slot_nodes[slot] = w.max_nodes;
                    grow_shape(w);
                }
                count = running_snapshot();
                upload_classes(count);
                cudaGraphExec_t g = graph_for(count);
                check(cudaEventRecord(tick_begin, stream), "event");
                for (int i = 0; i < per_poll; ++i) check(cudaGraphLaunch(g, stream), "graph launch");
                check(cudaEventRecord(tick_end, stream), "event");
                check(cudaMemcpyAsync(host_controls, dev_controls, sizeof(WrapControl) * count,
                                      cudaMemcpyDeviceToHost, stream), "pull controls");
                check(cudaStreamSynchronize(stream), "tick");
            } catch (const std::exception& e) {
                // the device failed under every running request
                std::lock_guard<std::mutex> lk(mu);
                for (int i = 0; i < slots_used; ++i)
                    if (slot_req[i]) {
                        fail(slot_req[i], e.what(), false);
                        slot_req[i] = nullptr;
                    }
                running = 0;
                stop = true;
                cv_work.notify_all();
                return;
            }
            float tick_ms = 0.0f;
            cudaEventElapsedTime(&tick_ms, tick_begin, tick_end);
            ticks += per_poll;
            launches += (long)per_poll * launches_per_tick[count];
            busy_seconds += 1e-3 * tick_ms;
            std::vector<int> holes;
            for (int i = 0; i < count; ++i) {
                RequestPtr r = slot_req[i];
                if (!r || host_controls[i].phase != kPhaseDone) continue;
                holes.push_back(i);
                std::string why;
                if (host_controls[i].error) {
                    why = "a closest-point traversal exceeded its stack; the hierarchy is too deep";
                } else {
                    try {
                        retire(i, r);
                    } catch (const std::exception& e) {
                        why = e.what();
                    }
                }
                bury(r);
                std::lock_guard<std::mutex> lk(mu);
                r->t_retired = now_seconds();
                slot_req[i] = nullptr;
                running -= 1;
                if (!why.empty()) {
                    r->wrap.reset();
                    fail(r, why, false);
                    continue;
                }
                finishing.push_back(r);
                cv_work.notify_all();
            }
            // keep the running wraps in slots 0 .. running-1: the last running
            // wraps fill the holes the retired ones left
            try {
                int last = count - 1;
                for (int hole : holes) {
                    while (last > hole && !slot_req[last]) --last;
                    if (last <= hole) break;
                    move_slot(last, hole);
                    --last;
                }
            } catch (const std::exception& e) {
                std::lock_guard<std::mutex> lk(mu);
                for (int i = 0; i < slots_used; ++i)
                    if (slot_req[i]) {
                        fail(slot_req[i], e.what(), false);
                        slot_req[i] = nullptr;
                    }
                running = 0;
                stop = true;
                cv_work.notify_all();
                return;
            }
        }
    }

    int running_snapshot() {
        std::lock_guard<std::mutex> lk(mu);
        return running;
    }
};

Server::Server(const NricpServerConfig& config) : impl_(std::make_unique<Impl>()) {
    Impl& m = *impl_;
    m.cfg = config;
    if (m.cfg.max_slots <= 0 || m.cfg.max_slots > 1024)
        throw InvalidArgument("max_slots is " + std::to_string(m.cfg.max_slots) + "; it must be 1 to 1024");
    if (m.cfg.pcg_cluster > 0 && (m.cfg.pcg_cluster > 16 || (m.cfg.pcg_cluster & (m.cfg.pcg_cluster - 1)) != 0))
        throw InvalidArgument("the solve's cluster size is a power of two from 1 to 16");
    if (m.cfg.pcg_cluster < -4) throw InvalidArgument("the solve's class shift is 0 to 4");
    check(cudaGetDevice(&m.device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&m.sms, cudaDevAttrMultiProcessorCount, m.device), "device");
    if (m.cfg.memory_budget_bytes == 0) {
        size_t free_bytes = 0, total = 0;
        check(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
        m.cfg.memory_budget_bytes = free_bytes / 10 * 9;
    }
    check(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int k = 0; k < Impl::kLoaders; ++k)
        check(cudaStreamCreateWithFlags(&m.load_streams[k], cudaStreamNonBlocking), "cudaStreamCreate");
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = m.device;
        check(cudaMemPoolCreate(&m.pool, &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;  // keep freed arenas for the next requests
        check(cudaMemPoolSetAttribute(m.pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool");
    }
    check(cudaMalloc(&m.staging_controls, sizeof(WrapControl) * Impl::kLoaders), "cudaMalloc(staging control)");
    check(cudaEventCreate(&m.tick_begin), "event");
    check(cudaMalloc(&m.query_counter, 2 * sizeof(int)), "cudaMalloc(query queues)");
    m.shape.query_counter = m.query_counter;
    check(cudaStreamCreateWithFlags(&m.shape.side_stream, cudaStreamNonBlocking), "stream");
    check(cudaEventCreateWithFlags(&m.shape.side_fork, cudaEventDisableTiming), "event");
    check(cudaEventCreateWithFlags(&m.shape.side_join, cudaEventDisableTiming), "event");
    check(cudaEventCreate(&m.tick_end), "event");
    if (m.cfg.pcg_cluster <= 0) {
        m.class_top = m.cfg.pcg_cluster < 0 ? std::max(1, 16 >> m.max_shift()) : 16;
        for (int c = m.class_top; c >= 1; c /= 2) m.class_count += 1;
        check(cudaMalloc(&m.class_index, sizeof(int) * m.class_count * m.cfg.max_slots), "cudaMalloc(classes)");
        check(cudaMemset(m.class_index, 0xff, sizeof(int) * m.class_count * m.cfg.max_slots), "classes");
        m.class_rows.assign(static_cast<size_t>(m.class_count) * m.cfg.max_slots, -1);
        for (int g = 1; g < m.class_count; ++g) {
            check(cudaStreamCreateWithFlags(&m.class_streams[g], cudaStreamNonBlocking), "stream");
            check(cudaEventCreateWithFlags(&m.class_join[g], cudaEventDisableTiming), "event");
        }
        check(cudaEventCreateWithFlags(&m.class_fork, cudaEventDisableTiming), "event");
    }
    check(cudaMalloc(&m.dev_wraps, sizeof(WrapDev) * m.cfg.max_slots), "cudaMalloc(slots)");
    check(cudaMalloc(&m.dev_controls, sizeof(WrapControl) * m.cfg.max_slots), "cudaMalloc(controls)");
    check(cudaMallocHost(&m.host_controls, sizeof(WrapControl) * m.cfg.max_slots), "cudaMallocHost(controls)");
    m.host_wraps.assign(m.cfg.max_slots, WrapDev{});
    m.slot_req.assign(m.cfg.max_slots, nullptr);
    m.slot_nodes.assign(m.cfg.max_slots, 0);
    int threads = m.cfg.prep_threads;
    if (threads <= 0) threads = std::max(1, static_cast<int>(std::thread::hardware_concurrency()) / 2);
    for (int i = 0; i < threads; ++i) m.preppers.emplace_back([&m] { m.prep_loop(); });
    for (int k = 0; k < Impl::kLoaders; ++k) m.loader_threads.emplace_back([&m, k] { m.loader_loop(k); });
    m.finisher_thread = std::thread([&m] { m.finish_loop(); });
    m.pump_thread = std::thread([&m] { m.pump_loop(); });
}

Server::~Server() {
    Impl& m = *impl_;
    {
        std::lock_guard<std::mutex> lk(m.mu);
        m.stop = true;
    }
    m.cv_work.notify_all();
    m.cv_done.notify_all();
    for (auto& t : m.preppers) t.join();
    if (m.pump_thread.joinable()) m.pump_thread.join();
    for (auto& t : m.loader_threads) t.join();
    if (m.finisher_thread.joinable()) m.finisher_thread.join();
    m.finishing.clear();
    cudaSetDevice(m.device);
    cudaStreamSynchronize(m.stream);
    for (int k = 0; k < Impl::kLoaders; ++k) cudaStreamSynchronize(m.load_streams[k]);
    for (auto& [count, g] : m.graphs) cudaGraphExecDestroy(g);
    for (auto& r : m.loaded)
        if (r->loaded) cudaEventDestroy(r->loaded);
    for (auto& d : m.graveyard) cudaEventDestroy(d.after);
    m.graveyard.clear();
    m.slot_req.clear();
    m.requests.clear();
    m.ready.clear();
    m.loaded.clear();
    m.prep_queue.clear();
    for (int k = 0; k < Impl::kLoaders; ++k)
        if (m.lbvh_scratch[k]) cudaFree(m.lbvh_scratch[k]);
    if (m.staging_controls) cudaFree(m.staging_controls);
    if (m.class_index) cudaFree(m.class_index);
    for (int g = 1; g < 5; ++g) {
        if (m.class_streams[g]) cudaStreamDestroy(m.class_streams[g]);
        if (m.class_join[g]) cudaEventDestroy(m.class_join[g]);
    }
    if (m.class_fork) cudaEventDestroy(m.class_fork);
    if (m.tick_begin) cudaEventDestroy(m.tick_begin);
    if (m.query_counter) cudaFree(m.query_counter);
    if (m.shape.side_stream) cudaStreamDestroy(m.shape.side_stream);
    if (m.shape.side_fork) cudaEventDestroy(m.shape.side_fork);
    if (m.shape.side_join) cudaEventDestroy(m.shape.side_join);
    if (m.tick_end) cudaEventDestroy(m.tick_end);
    if (m.dev_wraps) cudaFree(m.dev_wraps);
    if (m.dev_controls) cudaFree(m.dev_controls);
    if (m.host_controls) cudaFreeHost(m.host_controls);
    cudaStreamDestroy(m.stream);
    for (int k = 0; k < Impl::kLoaders; ++k) cudaStreamDestroy(m.load_streams[k]);
    if (m.pool) cudaMemPoolDestroy(m.pool);
}

long Server::submit(const NricpSolveDesc& desc) {
    Impl& m = *impl_;
    validate_settings(desc);
    auto r = std::make_shared<Impl::Request>();
    r->wrap = std::make_unique<Wrap>();
    copy_inputs(*r->wrap, desc);
    std::lock_guard<std::mutex> lk(m.mu);
    if (m.stop) throw StateError("the server has stopped");
    r->id = m.next_id++;
    r->t_submit = now_seconds();
    if (m.first_submit < 0.0) m.first_submit = r->t_submit;
    m.requests[r->id] = r;
    m.prep_queue.push_back(r);
    m.submitted += 1;
    m.cv_work.notify_all();
    return r->id;
}

int Server::poll(long id, double* latency_seconds) {
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lk(m.mu);
    auto it = m.requests.find(id);
    if (it == m.requests.end()) throw InvalidArgument("unknown request " + std::to_string(id));
    const auto& r = it->second;
    if (latency_seconds)
        *latency_seconds = r->state == NRICP_REQUEST_DONE ? r->t_done - r->t_submit : 0.0;
    return r->state;
}

void Server::phases(long id, double seconds[5]) {
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lk(m.mu);
    auto it = m.requests.find(id);
    if (it == m.requests.end()) throw InvalidArgument("unknown request " + std::to_string(id));
    const auto& r = it->second;
    const double t[6] = {r->t_submit, r->t_prepared, r->t_loaded, r->t_admit, r->t_retired, r->t_done};
    for (int k = 0; k < 5; ++k) seconds[k] = t[k + 1] > 0.0 && t[k] > 0.0 ? t[k + 1] - t[k] : 0.0;
}

bool Server::wait(long id, double timeout_seconds) {
    Impl& m = *impl_;
    std::unique_lock<std::mutex> lk(m.mu);
    auto it = m.requests.find(id);
    if (it == m.requests.end()) throw InvalidArgument("unknown request " + std::to_string(id));
    const auto r = it->second;
    auto finished = [&] {
        return r->state == NRICP_REQUEST_DONE || r->state == NRICP_REQUEST_FAILED || m.stop;
    };
    if (timeout_seconds <= 0.0) {
        m.cv_done.wait(lk, finished);
        return true;
    }
    return m.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), finished);
}

void Server::result(long id, NricpResult* out) {
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lk(m.mu);
    auto it = m.requests.find(id);
    if (it == m.requests.end()) throw InvalidArgument("unknown request " + std::to_string(id));
    const auto r = it->second;
    if (r->state == NRICP_REQUEST_FAILED) {
        m.requests.erase(it);
        if (r->invalid) throw InvalidArgument(r->error);
        throw StateError(r->error);
    }
    if (r->state != NRICP_REQUEST_DONE) throw StateError("request " + std::to_string(id) + " is not done");
    if (out->vertices) std::memcpy(out->vertices, r->vertices.data(), sizeof(double) * r->vertices.size());
    if (out->rotations) std::memcpy(out->rotations, r->rotations.data(), sizeof(double) * r->rotations.size());
    if (out->translations)
        std::memcpy(out->translations, r->translations.data(), sizeof(double) * r->translations.size());
    if (out->node_positions) std::memcpy(out->node_positions, r->nodes.data(), sizeof(double) * r->nodes.size());
    if (out->level_nodes)
        std::memcpy(out->level_nodes, r->level_nodes.data(), sizeof(int32_t) * r->level_nodes.size());
    out->report_length = r->report.size();
    if (out->report_json && out->report_capacity > 0) {
        const size_t n = std::min(r->report.size(), out->report_capacity - 1);
        std::memcpy(out->report_json, r->report.data(), n);
        out->report_json[n] = 0;
    }
    g_transfers.d2h += sizeof(double) * (r->vertices.size() + r->rotations.size() + r->translations.size());
    m.requests.erase(it);
}

NricpServerStats Server::merged_stats(const std::vector<Server*>& servers) {
    if (servers.size() == 1) return servers[0]->stats();
    NricpServerStats s{};
    std::vector<double> latencies, queue_waits;
    double first = -1.0, last = 0.0;
    for (Server* server : servers) {
        Impl& m = *server->impl_;
        std::lock_guard<std::mutex> lk(m.mu);
        s.submitted += m.submitted;
        s.completed += m.completed;
        s.failed += m.failed;
        s.running += m.running;
        s.waiting += static_cast<long>(m.prep_queue.size() + m.ready.size() + m.loaded.size()) + m.loading;
        latencies.insert(latencies.end(), m.latencies.begin(), m.latencies.end());
        queue_waits.insert(queue_waits.end(), m.queue_waits.begin(), m.queue_waits.end());
        if (m.first_submit >= 0.0) first = first < 0.0 ? m.first_submit : std::min(first, m.first_submit);
        last = std::max(last, m.last_done);
        s.ticks += m.ticks;
        s.launches += m.launches;
        s.captures += m.captures;
        s.busy_seconds += m.busy_seconds;
        s.resident_bytes += m.resident;
        s.peak_resident_bytes += m.peak;
        s.slots_used += m.slots_used;
    }
    s.latency_p50_ms = 1000.0 * percentile(latencies, 0.50);
    s.latency_p99_ms = 1000.0 * percentile(latencies, 0.99);
    double sum = 0.0;
    for (double x : latencies) sum += x;
    s.latency_mean_ms = latencies.empty() ? 0.0 : 1000.0 * sum / latencies.size();
    s.queue_p50_ms = 1000.0 * percentile(queue_waits, 0.50);
    const double span = last - first;
    s.wraps_per_second = first >= 0.0 && span > 0.0 ? s.completed / span : 0.0;
    return s;
}

NricpServerStats Server::stats() {
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lk(m.mu);
    NricpServerStats s{};
    s.submitted = m.submitted;
    s.completed = m.completed;
    s.failed = m.failed;
    s.running = m.running;
    s.waiting = static_cast<long>(m.prep_queue.size() + m.ready.size() + m.loaded.size()) + m.loading;
    s.latency_p50_ms = 1000.0 * percentile(m.latencies, 0.50);
    s.latency_p99_ms = 1000.0 * percentile(m.latencies, 0.99);
    double sum = 0.0;
    for (double x : m.latencies) sum += x;
    s.latency_mean_ms = m.latencies.empty() ? 0.0 : 1000.0 * sum / m.latencies.size();
    s.queue_p50_ms = 1000.0 * percentile(m.queue_waits, 0.50);
    const double span = m.last_done - m.first_submit;
    s.wraps_per_second = span > 0.0 ? m.completed / span : 0.0;
    s.ticks = m.ticks;
    s.launches = m.launches;
    s.captures = m.captures;
    s.busy_seconds = m.busy_seconds;
    s.resident_bytes = m.resident;
    s.peak_resident_bytes = m.peak;
    s.slots_used = m.slots_used;
    return s;
}

}  // namespace nricp_b200
