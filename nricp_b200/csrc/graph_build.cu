// The template graphs of many wraps at once on the device: farthest-point
// seeds, the nearest-node bindings of every vertex and the k-NN node edges of
// every level (src/core/graph.cpp:41-76, src/core/sampling.cpp:17-143).
//
// Every value is the host build's to the bit: the same FP64 operations in the
// same order, each rounded on its own (no contraction), and the same tie
// rules -- the first maximum for the seeds, (squared distance, index) for the
// bindings, (distance, index) for the edges.  Only the scan orders differ,
// and none of the rules depends on them.
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "graph_build.hpp"
#include "session.hpp"
#include "staging.hpp"

namespace nricp_b200 {

namespace cg = cooperative_groups;

namespace {

constexpr int kFpsThreads = 1024;
constexpr int kBindThreads = 128;
constexpr int kTile = 512;            // nodes staged in shared memory per pass
constexpr int kMaxEdgeNeighbours = 16;

__device__ inline double sq_rn(const double* a, const double* b) {  // sampling.cpp:17-19
    const double x = __dsub_rn(a[0], b[0]), y = __dsub_rn(a[1], b[1]), z = __dsub_rn(a[2], b[2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// (value, index) with the larger value winning and the lower index breaking ties.
__device__ inline void arg_max(double& v, int& i, double ov, int oi) {
    if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
}

// One block per template (templates[blockIdx.x]): seeds[0] = 0, then
// repeatedly the point farthest from all seeds so far (sampling.cpp:47-88).
__global__ void __launch_bounds__(kFpsThreads) k_fps(const double* __restrict__ points,
                                                     const long* __restrict__ point_offset,
                                                     const int* __restrict__ point_count,
                                                     const int* __restrict__ seed_count,
                                                     const long* __restrict__ seed_offset,
                                                     const int* __restrict__ templates,
                                                     double* __restrict__ nearest_all,
                                                     int* __restrict__ seeds_all) {
    const int t = templates[blockIdx.x];
    const int n = point_count[t];
    const int count = min(seed_count[t], n);
    if (n <= 0 || count <= 0) return;
    const double* p = points + point_offset[t] * 3;
    double* nearest = nearest_all + point_offset[t];
    int* seeds = seeds_all + seed_offset[t];
    __shared__ double red_v[kFpsThreads / 32];
    __shared__ int red_i[kFpsThreads / 32];
    __shared__ int chosen_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto block_arg_max = [&](double v, int i) {
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int oi = __shfl_xor_sync(0xffffffffu, i, o);
            arg_max(v, i, ov, oi);
        }
        if (lane == 0) { red_v[warp] = v; red_i[warp] = i; }
        __syncthreads();
        if (warp == 0) {
            v = lane < kFpsThreads / 32 ? red_v[lane] : -1.0;
            i = lane < kFpsThreads / 32 ? red_i[lane] : 0x7fffffff;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oi = __shfl_xor_sync(0xffffffffu, i, o);
                arg_max(v, i, ov, oi);
            }
            if (lane == 0) chosen_s = i;
        }
        __syncthreads();
        return chosen_s;
    };
    if (threadIdx.x == 0) seeds[0] = 0;
    double c[3] = {p[0], p[1], p[2]};
    double bv = -1.0;
    int bi = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += kFpsThreads) {
        const double d = sq_rn(p + (long)i * 3, c);
        nearest[i] = d;
        arg_max(bv, bi, d, i);
    }
    int best = block_arg_max(bv, bi);
    for (int k = 1; k < count; ++k) {
        if (threadIdx.x == 0) seeds[k] = best;
        c[0] = p[(long)best * 3];
        c[1] = p[(long)best * 3 + 1];
        c[2] = p[(long)best * 3 + 2];
        bv = -1.0;
        bi = 0x7fffffff;
        for (int i = threadIdx.x; i < n; i += kFpsThreads) {
            const double d = sq_rn(p + (long)i * 3, c);
            const double m = nearest[i] < d ? nearest[i] : d;
            nearest[i] = m;
            arg_max(bv, bi, m, i);
        }
        best = block_arg_max(bv, bi);
    }
}

// The same seeds from one thread-block cluster per template
// (templates[blockIdx.y]), for templates of at most kFpsClusterPoints
// points: the points are split in contiguous chunks over the cluster's CTAs,
// and every thread keeps up to four points and their distances to the
// nearest seed in registers.  Per seed: the thread's, the warp's and the
// CTA's farthest point, then every CTA writes its candidate into every CTA's
// shared slots (distributed shared memory, two sets used in turn), one
// cluster barrier, and every CTA takes the same winner in rank order.  The
// arithmetic and the tie rule (the larger distance, then the lower index) are
// k_fps's, so the winner and the seeds are the same for any split.
constexpr int kFpsClusterThreads = 1024;
constexpr int kFpsPerThread = 4;
constexpr int kFpsClusterPoints = 16 * kFpsClusterThreads * kFpsPerThread;  // 65,536

struct FpsCandidate {
    double v, x, y, z;
    int i, pad;
};

__device__ inline void better(FpsCandidate& a, const FpsCandidate& b) {
    if (b.v > a.v || (b.v == a.v && b.i < a.i)) a = b;
}

__device__ inline FpsCandidate shuffle(const FpsCandidate& c, int lane_mask) {
    FpsCandidate o;
    o.v = __shfl_xor_sync(0xffffffffu, c.v, lane_mask);
    o.x = __shfl_xor_sync(0xffffffffu, c.x, lane_mask);
    o.y = __shfl_xor_sync(0xffffffffu, c.y, lane_mask);
    o.z = __shfl_xor_sync(0xffffffffu, c.z, lane_mask);
    o.i = __shfl_xor_sync(0xffffffffu, c.i, lane_mask);
    o.pad = 0;
    return o;
}

__global__ void __launch_bounds__(kFpsClusterThreads) k_fps_cluster(const double* __restrict__ points,
                                                                   const long* __restrict__ point_offset,
                                                                   const int* __restrict__ point_count,
                                                                   const int* __restrict__ seed_count,
                                                                   const long* __restrict__ seed_offset,
                                                                   const int* __restrict__ templates,
                                                                   int* __restrict__ seeds_all) {
    cg::cluster_group cluster = cg::this_cluster();
    const int t = templates[blockIdx.y];
    const int n = point_count[t];
    const int count = min(seed_count[t], n);
    if (n <= 0 || count <= 0) return;  // the same for the whole cluster
    const int rank = (int)cluster.block_rank(), ranks = (int)cluster.num_blocks();
    const int chunk = (n + ranks - 1) / ranks;  // <= kFpsClusterThreads * kFpsPerThread
    const int c0 = rank * chunk, c1 = min(n, c0 + chunk);
    const double* p = points + point_offset[t] * 3;
    int* seeds = seeds_all + seed_offset[t];
    __shared__ FpsCandidate slots[2][16];
    __shared__ FpsCandidate warp_best[kFpsClusterThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double px[kFpsPerThread], py[kFpsPerThread], pz[kFpsPerThread], near[kFpsPerThread];
    int idx[kFpsPerThread];
    for (int k = 0; k < kFpsPerThread; ++k) {
        const int i = c0 + threadIdx.x + k * kFpsClusterThreads;
        idx[k] = i < c1 ? i : -1;
        px[k] = py[k] = pz[k] = near[k] = 0.0;
        if (idx[k] >= 0) {
            px[k] = p[(long)i * 3];
            py[k] = p[(long)i * 3 + 1];
            pz[k] = p[(long)i * 3 + 2];
        }
    }
    if (rank == 0 && threadIdx.x == 0) seeds[0] = 0;
    double c[3] = {p[0], p[1], p[2]};
    for (int s = 0;; ++s) {
        FpsCandidate best{-1.0, 0.0, 0.0, 0.0, INT_MAX, 0};
        for (int k = 0; k < kFpsPerThread; ++k) {
            if (idx[k] < 0) continue;
            const double q[3] = {px[k], py[k], pz[k]};
            const double d = sq_rn(q, c);
            const double m = s == 0 ? d : (near[k] < d ? near[k] : d);
            near[k] = m;
            better(best, FpsCandidate{m, px[k], py[k], pz[k], idx[k], 0});
        }
        if (s + 1 >= count) break;
        for (int o = 16; o > 0; o >>= 1) better(best, shuffle(best, o));
        if (lane == 0) warp_best[warp] = best;
        __syncthreads();
        if (warp == 0) {
            best = warp_best[lane];  // 32 warps
            for (int o = 16; o > 0; o >>= 1) better(best, shuffle(best, o));
            if (lane < ranks) *cluster.map_shared_rank(&slots[s & 1][rank], lane) = best;
        }
        cluster.sync();
        FpsCandidate win = slots[s & 1][0];
        for (int r = 1; r < ranks; ++r) better(win, slots[s & 1][r]);
        if (rank == 0 && threadIdx.x == 0) seeds[s + 1] = win.i;
        c[0] = win.x;
        c[1] = win.y;
        c[2] = win.z;
    }
    // no CTA leaves while another may still write into its shared memory
    cluster.sync();
}

// (sq, idx) kept sorted ascending, at most `capacity` entries, entries offered
// in increasing index (sampling.cpp:23-42).
__device__ inline void keep(double* sq, int* idx, int& held, int capacity, double value, int entry) {
    if (held == capacity && !(value < sq[capacity - 1] || (value == sq[capacity - 1] && entry < idx[capacity - 1])))
        return;
    int at = held < capacity ? held++ : capacity - 1;
    while (at > 0 && (sq[at - 1] > value || (sq[at - 1] == value && idx[at - 1] > entry))) {
        sq[at] = sq[at - 1];
        idx[at] = idx[at - 1];
        --at;
    }
    sq[at] = value;
    idx[at] = entry;
}

// Thread per (template, vertex) for one level: its `support` nearest nodes
// and weights (1 - d / d_max)^2, normalised (sampling.cpp:90-143).
__global__ void __launch_bounds__(kBindThreads) k_bind(const double* __restrict__ points,
                                                       const long* __restrict__ point_offset,
                                                       const int* __restrict__ point_count,
                                                       const int* __restrict__ seeds_all,
                                                       const long* __restrict__ seed_offset,
                                                       const int* __restrict__ level_nodes,
                                                       const int* __restrict__ support_of,
                                                       const long* __restrict__ bind_offset,
                                                       int* __restrict__ bind_nodes,
                                                       double* __restrict__ bind_weights) {
    const int t = blockIdx.y;
    const int n = point_count[t], nc = level_nodes[t];
    if (nc <= 0 || (long)blockIdx.x * kBindThreads >= n) return;
    const int v = blockIdx.x * kBindThreads + threadIdx.x;
    const double* p = points + point_offset[t] * 3;
    const int* seeds = seeds_all + seed_offset[t];
    const int support = support_of[t];
    __shared__ double tile[kTile * 3];
    double sq[NRICP_MAX_SLOTS];
    int idx[NRICP_MAX_SLOTS];
    int held = 0;
    double q[3] = {0.0, 0.0, 0.0};
    if (v < n) { q[0] = p[(long)v * 3]; q[1] = p[(long)v * 3 + 1]; q[2] = p[(long)v * 3 + 2]; }
    for (int base = 0; base < nc; base += kTile) {
        const int m = min(kTile, nc - base);
        __syncthreads();
        for (int j = threadIdx.x; j < m * 3; j += kBindThreads) {
            const int node = base + j / 3;
            tile[j] = p[(long)seeds[node] * 3 + j % 3];
        }
        __syncthreads();
        if (v < n)
            for (int j = 0; j < m; ++j) keep(sq, idx, held, support, sq_rn(q, tile + j * 3), base + j);
    }
    if (v >= n) return;
    const long at = bind_offset[t] + (long)v * NRICP_MAX_SLOTS;
    const double dmax = __dsqrt_rn(sq[support - 1]);
    double w[NRICP_MAX_SLOTS];
    double total = 0.0;
    for (int s = 0; s < support; ++s) {
        const double distance = __dsqrt_rn(sq[s]);
        const double ratio = dmax > 0.0 ? __ddiv_rn(distance, dmax) : 0.0;
        const double falloff = __dsub_rn(1.0, ratio);
        w[s] = __dmul_rn(falloff, falloff);
        total = __dadd_rn(total, w[s]);
    }
    for (int s = 0; s < NRICP_MAX_SLOTS; ++s) {
        bind_nodes[at + s] = s < support ? idx[s] : -1;
        bind_weights[at + s] =
            s < support ? (total > 0.0 ? __ddiv_rn(w[s], total) : __ddiv_rn(1.0, (double)support)) : 0.0;
    }
}

// Thread per (template, node) for one level: the `taken` nearest other nodes
// by (distance, index) (graph.cpp:11-39).
__global__ void __launch_bounds__(kBindThreads) k_neighbours(const double* __restrict__ points,
                                                             const long* __restrict__ point_offset,
                                                             const int* __restrict__ seeds_all,
                                                             const long* __restrict__ seed_offset,
                                                             const int* __restrict__ level_nodes,
                                                             const int* __restrict__ taken_of,
                                                             const long* __restrict__ edge_offset,
                                                             int* __restrict__ neighbours) {
    const int t = blockIdx.y;
    const int nc = level_nodes[t];
    if ((long)blockIdx.x * kBindThreads >= nc) return;
    const int i = blockIdx.x * kBindThreads + threadIdx.x;
    const double* p = points + point_offset[t] * 3;
    const int* seeds = seeds_all + seed_offset[t];
    const int taken = taken_of[t];
    __shared__ double tile[kTile * 3];
    double dist[kMaxEdgeNeighbours];
    int idx[kMaxEdgeNeighbours];
    int held = 0;
    double q[3] = {0.0, 0.0, 0.0};
    if (i < nc) {
        const long s = seeds[i];
        q[0] = p[s * 3]; q[1] = p[s * 3 + 1]; q[2] = p[s * 3 + 2];
    }
    for (int base = 0; base < nc; base += kTile) {
        const int m = min(kTile, nc - base);
        __syncthreads();
        for (int j = threadIdx.x; j < m * 3; j += kBindThreads) tile[j] = p[(long)seeds[base + j / 3] * 3 + j % 3];
        __syncthreads();
        if (i < nc && taken > 0)
            for (int j = 0; j < m; ++j) {
                const int o = base + j;
                if (o == i) continue;
                const double x = __dsub_rn(q[0], tile[j * 3]), y = __dsub_rn(q[1], tile[j * 3 + 1]),
                             z = __dsub_rn(q[2], tile[j * 3 + 2]);
                const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
                keep(dist, idx, held, taken, d, o);
            }
    }
    if (i >= nc) return;
    for (int k = 0; k < taken; ++k) neighbours[edge_offset[t] + (long)i * taken + k] = idx[k];
}

int blocks(long n, int threads) { return static_cast<int>((n + threads - 1) / threads); }

template <typename T>
T* to_device(const std::vector<T>& v, std::vector<void*>& owned, cudaStream_t stream) {
    T* d = nullptr;
    check(cudaMalloc(&d, sizeof(T) * std::max<size_t>(1, v.size())), "cudaMalloc(graph build)");
    owned.push_back(d);
    if (!v.empty())
        check(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream), "upload");
    return d;
}

}  // namespace

bool device_graph_supported(int edge_neighbours) { return edge_neighbours <= kMaxEdgeNeighbours; }

std::vector<TemplateGraph> device_template_graphs(const std::vector<GraphRequest>& requests,
                                                  cudaStream_t stream) {
    const int W = static_cast<int>(requests.size());
    std::vector<TemplateGraph> out(W);
    if (W == 0) return out;
    // host: normalisation (mesh.cpp:174-187) and the sizes of every level
    std::vector<double> points;
    std::vector<long> point_offset(W), seed_offset(W);
    std::vector<int> point_count(W), seed_count(W);
    std::vector<std::vector<int>> level_sizes(W);
    long total_points = 0, total_seeds = 0;
    int max_levels = 0, max_points = 0;
    for (int t = 0; t < W; ++t) {
        const GraphRequest& r = requests[t];
        point_offset[t] = total_points;
        point_count[t] = r.count;
        total_points += r.count;
        const int levels = std::max(1, r.levels);
        int most = 0;
        for (int l = 0; l < levels; ++l) {
            level_sizes[t].push_back(level_node_count(l, r.nodes_initial, r.growth, r.count));
            most = std::max(most, level_sizes[t].back());
        }
        most = std::min(most, r.count);
        seed_offset[t] = total_seeds;
        seed_count[t] = most;
        total_seeds += most;
        max_levels = std::max(max_levels, levels);
        max_points = std::max(max_points, r.count);
    }
    // every template normalised on its own host thread, into its place
    points.resize(static_cast<size_t>(total_points) * 3);
#pragma omp parallel for schedule(dynamic, 1) if (W > 1)
    for (int t = 0; t < W; ++t) {
        const GraphRequest& r = requests[t];
        TemplateGraph& g = out[t];
        compute_normalization(r.points, r.count, g.center, &g.scale);
        const std::vector<double> norm = normalized(r.points, r.count, g.center, g.scale);
        std::copy(norm.begin(), norm.end(), points.begin() + point_offset[t] * 3);
    }
    std::vector<void*> owned;
    double* d_points = to_device(points, owned, stream);
    long* d_point_offset = to_device(point_offset, owned, stream);
    int* d_point_count = to_device(point_count, owned, stream);
    int* d_seed_count = to_device(seed_count, owned, stream);
    long* d_seed_offset = to_device(seed_offset, owned, stream);
    double* d_nearest = nullptr;
    int* d_seeds = nullptr;
    check(cudaMalloc(&d_nearest, sizeof(double) * std::max<long>(1, total_points)), "cudaMalloc(graph build)");
    owned.push_back(d_nearest);
    check(cudaMalloc(&d_seeds, sizeof(int) * std::max<long>(1, total_seeds)), "cudaMalloc(graph build)");
    owned.push_back(d_seeds);
    // every level's sizes, on the host
    struct LevelPlan {
        std::vector<int> nodes, support, taken;
        std::vector<long> eoff;
        long edge_total = 0;
        int max_nodes = 0;
    };
    std::vector<LevelPlan> plan(max_levels);
    long all_edges = 0;
    std::vector<long> edge_base(max_levels + 1, 0);
    for (int l = 0; l < max_levels; ++l) {
        LevelPlan& p = plan[l];
        p.nodes.assign(W, 0);
        p.support.assign(W, 1);
        p.taken.assign(W, 0);
        p.eoff.assign(W, 0);
        for (int t = 0; t < W; ++t) {
            const GraphRequest& r = requests[t];
            if (l >= static_cast<int>(level_sizes[t].size())) continue;
            p.nodes[t] = std::min(level_sizes[t][l], seed_count[t]);
            p.support[t] = std::max(1, std::min({r.max_nodes, p.nodes[t], NRICP_MAX_SLOTS}));
            p.taken[t] = p.nodes[t] > 1 && r.edge_neighbours > 0 ? std::min(r.edge_neighbours, p.nodes[t] - 1) : 0;
            p.eoff[t] = p.edge_total;
            p.edge_total += static_cast<long>(p.nodes[t]) * p.taken[t];
            p.max_nodes = std::max(p.max_nodes, p.nodes[t]);
        }
        edge_base[l + 1] = edge_base[l] + std::max<long>(1, p.edge_total);
        all_edges = edge_base[l + 1];
    }

    // the downloads land in page-locked memory: seeds, then per level the
    // bindings' nodes and weights, then every level's neighbour lists
    const long bind_entries = std::max<long>(1, total_points * NRICP_MAX_SLOTS);
    const size_t seed_bytes = (sizeof(int) * std::max<long>(1, total_seeds) + 255) & ~size_t(255);
    const size_t level_bytes = (sizeof(int32_t) + sizeof(double)) * bind_entries;
    StagingLease lease(seed_bytes + level_bytes * max_levels + sizeof(int) * all_edges);
    int* seeds = reinterpret_cast<int*>(lease.data());
    auto host_nodes = [&](int l) {
        return reinterpret_cast<int32_t*>(lease.data() + seed_bytes + level_bytes * l);
    };
    auto host_weights = [&](int l) {
        return reinterpret_cast<double*>(lease.data() + seed_bytes + level_bytes * l + sizeof(int32_t) * bind_entries);
    };
    int* host_neigh = reinterpret_cast<int*>(lease.data() + seed_bytes + level_bytes * max_levels);

    // seeds: a cluster of 1-16 CTAs per template (4,096 points per CTA), one
    // launch per cluster size; a single block for templates beyond 65,536
    // points.  The launches touch different templates, so each runs on a
    // stream of its own, beside the others.
    {
        std::vector<std::vector<int>> by_size(5);
        std::vector<int> single;
        for (int t = 0; t < W; ++t) {
            if (point_count[t] > kFpsClusterPoints) {
                single.push_back(t);
                continue;
            }
            int g = 0;
            while ((1 << g) * kFpsClusterThreads * kFpsPerThread < point_count[t]) ++g;
            by_size[g].push_back(t);
        }
        static const bool enabled = [] {
            cudaFuncSetAttribute(k_fps_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            return true;
        }();
        (void)enabled;
        const int* d_group[5] = {};
        for (int g = 0; g < 5; ++g)
            if (!by_size[g].empty()) d_group[g] = to_device(by_size[g], owned, stream);
        const int* d_single = single.empty() ? nullptr : to_device(single, owned, stream);
        cudaStream_t lanes[6] = {};
        cudaEvent_t fork = nullptr, join[6] = {};
        check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
        check(cudaEventRecord(fork, stream), "event");
        for (int k = 0; k < 6; ++k) {
            check(cudaStreamCreateWithFlags(&lanes[k], cudaStreamNonBlocking), "stream");
            check(cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming), "event");
            check(cudaStreamWaitEvent(lanes[k], fork, 0), "wait");
        }
        for (int g = 0; g < 5; ++g) {
            if (by_size[g].empty()) continue;
            const int* d_templates = d_group[g];
            cudaLaunchConfig_t config = {};
            config.gridDim = dim3(1 << g, static_cast<unsigned>(by_size[g].size()));
            config.blockDim = dim3(kFpsClusterThreads);
            config.stream = lanes[g];
            cudaLaunchAttribute attribute[1];
            attribute[0].id = cudaLaunchAttributeClusterDimension;
            attribute[0].val.clusterDim.x = 1 << g;
            attribute[0].val.clusterDim.y = 1;
            attribute[0].val.clusterDim.z = 1;
            config.attrs = attribute;
            config.numAttrs = 1;
            check(cudaLaunchKernelEx(&config, k_fps_cluster, (const double*)d_points, (const long*)d_point_offset,
                                     (const int*)d_point_count, (const int*)d_seed_count,
                                     (const long*)d_seed_offset, d_templates, d_seeds),
                  "farthest-point seeds");
        }
        if (!single.empty()) {
            k_fps<<<static_cast<int>(single.size()), kFpsThreads, 0, lanes[5]>>>(
                d_points, d_point_offset, d_point_count, d_seed_count, d_seed_offset, d_single, d_nearest,
                d_seeds);
        }
        for (int k = 0; k < 6; ++k) {
            check(cudaEventRecord(join[k], lanes[k]), "event");
            check(cudaStreamWaitEvent(stream, join[k], 0), "wait");
        }
        for (int k = 0; k < 6; ++k) {
            cudaStreamDestroy(lanes[k]);  // released once its work is done
            cudaEventDestroy(join[k]);
        }
        cudaEventDestroy(fork);
    }
    check(cudaGetLastError(), "farthest-point seeds");
    check(cudaMemcpyAsync(seeds, d_seeds, sizeof(int) * std::max<long>(1, total_seeds), cudaMemcpyDeviceToHost,
                          stream), "download seeds");

    // per level: bindings and neighbour lists of every template in one launch each
    int32_t* d_bind_nodes = nullptr;
    double* d_bind_weights = nullptr;
    int* d_neigh = nullptr;
    check(cudaMalloc(&d_bind_nodes, sizeof(int32_t) * bind_entries * max_levels), "cudaMalloc(graph build)");
    owned.push_back(d_bind_nodes);
    check(cudaMalloc(&d_bind_weights, sizeof(double) * bind_entries * max_levels), "cudaMalloc(graph build)");
    owned.push_back(d_bind_weights);
    check(cudaMalloc(&d_neigh, sizeof(int) * all_edges), "cudaMalloc(graph build)");
    owned.push_back(d_neigh);
    std::vector<long> bind_offset(W);
    for (int t = 0; t < W; ++t) bind_offset[t] = point_offset[t] * NRICP_MAX_SLOTS;
    long* d_bind_offset = to_device(bind_offset, owned, stream);
    for (int l = 0; l < max_levels; ++l) {
        const LevelPlan& p = plan[l];
        int* d_nodes = to_device(p.nodes, owned, stream);
        int* d_support = to_device(p.support, owned, stream);
        int* d_taken = to_device(p.taken, owned, stream);
        long* d_eoff = to_device(p.eoff, owned, stream);
        int32_t* level_nodes = d_bind_nodes + bind_entries * l;
        double* level_weights = d_bind_weights + bind_entries * l;
        int* level_neigh = d_neigh + edge_base[l];
        k_bind<<<dim3(blocks(max_points, kBindThreads), W), kBindThreads, 0, stream>>>(
            d_points, d_point_offset, d_point_count, d_seeds, d_seed_offset, d_nodes, d_support,
            d_bind_offset, level_nodes, level_weights);
        check(cudaGetLastError(), "bindings");
        if (p.max_nodes > 0)
            k_neighbours<<<dim3(blocks(p.max_nodes, kBindThreads), W), kBindThreads, 0, stream>>>(
                d_points, d_point_offset, d_seeds, d_seed_offset, d_nodes, d_taken, d_eoff, level_neigh);
        check(cudaGetLastError(), "node edges");
        check(cudaMemcpyAsync(host_nodes(l), level_nodes, sizeof(int32_t) * bind_entries, cudaMemcpyDeviceToHost,
                              stream), "download bindings");
        check(cudaMemcpyAsync(host_weights(l), level_weights, sizeof(double) * bind_entries, cudaMemcpyDeviceToHost,
                              stream), "download bindings");
        if (p.edge_total > 0)
            check(cudaMemcpyAsync(host_neigh + edge_base[l], level_neigh, sizeof(int) * p.edge_total,
                                  cudaMemcpyDeviceToHost, stream), "download edges");
    }
    check(cudaStreamSynchronize(stream), "graph build");
    for (void* p : owned) cudaFree(p);

    // host: the graphs in the host build's form, one template per thread
#pragma omp parallel for schedule(dynamic, 1) if (W > 1)
    for (int t = 0; t < W; ++t) {
        TemplateGraph& g = out[t];
        const int levels = static_cast<int>(level_sizes[t].size());
        for (int l = 0; l < levels; ++l) {
            GraphLevel level;
            const int n = std::min(level_sizes[t][l], seed_count[t]);
            level.template_index.assign(seeds + seed_offset[t], seeds + seed_offset[t] + n);
            level.rest.resize(static_cast<size_t>(n) * 3);
            for (int i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k)
                    level.rest[i * 3 + k] = points[(point_offset[t] + level.template_index[i]) * 3 + k];
            level.bindings.resize(point_count[t]);
            const int32_t* nodes = host_nodes(l);
            const double* weights = host_weights(l);
            for (int v = 0; v < point_count[t]; ++v) {
                Binding& b = level.bindings[v];
                const long at = (point_offset[t] + v) * NRICP_MAX_SLOTS;
                for (int s = 0; s < NRICP_MAX_SLOTS; ++s) {
                    b.nodes[s] = nodes[at + s];
                    b.weights[s] = weights[at + s];
                }
                b.count = plan[l].support[t];
            }
            const int taken = plan[l].taken[t];
            const int* neigh = host_neigh + edge_base[l] + plan[l].eoff[t];
            std::vector<std::pair<int, int>> pairs;
            pairs.reserve(static_cast<size_t>(n) * taken);
            for (int i = 0; i < n; ++i)
                for (int k = 0; k < taken; ++k) {
                    const int o = neigh[static_cast<long>(i) * taken + k];
                    pairs.emplace_back(std::min(i, o), std::max(i, o));
                }
            std::sort(pairs.begin(), pairs.end());
            pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
            level.edges.reserve(pairs.size() * 2);
            for (auto& p : pairs) {
                level.edges.push_back(p.first);
                level.edges.push_back(p.second);
            }
            g.levels.push_back(std::move(level));
        }
    }
    return out;
}

}  // namespace nricp_b200
