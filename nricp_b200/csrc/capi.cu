// The C-ABI of include/nricp_b200.h: status codes, thread-local error
// messages, caller-allocated outputs.  Every entry point catches and converts;
// nothing throws across the boundary.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/nricp_b200.h"
#include "common.cuh"
#include "host.hpp"
#include "kernels.cuh"
#include "graph_build.hpp"
#include "session.hpp"

using namespace nricp_b200;

struct NricpSession {
    Batch batch;
};
struct NricpBatch {
    Batch batch;
};

namespace {

template <typename F>
int guarded(F&& body) {
    try {
        body();
        return NRICP_OK;
    } catch (const InvalidArgument& e) {
        g_last_error = e.what();
        return NRICP_ERR_INVALID;
    } catch (const TimeoutError& e) {
        g_last_error = e.what();
        return NRICP_ERR_TIMEOUT;
    } catch (const CapacityError& e) {
        g_last_error = e.what();
        return NRICP_ERR_CAPACITY;
    } catch (const StateError& e) {
        g_last_error = e.what();
        return NRICP_ERR_STATE;
    } catch (const CudaError& e) {
        g_last_error = e.what();
        return NRICP_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        g_last_error = "out of host memory";
        return NRICP_ERR_CAPACITY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return NRICP_ERR_CUDA;
    }
}

void require_device() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        throw CudaError("no CUDA device is available; the wrapping path has no CPU fallback");
    }
}

void fill_progress(const WrapControl& c, NricpProgress* p) {
    p->level = c.level;
    p->outer = c.outer;
    p->inner = c.inner;
    p->finished = c.phase == kPhaseDone;
    p->level_converged = 0;
    p->energy = c.energy;
    p->correspondence_mean = c.last_corr_mean;
}

}  // namespace

extern "C" {

void nricp_default_level(NricpLevelSettings* s) {
    s->point_to_point = 1.0;
    s->point_to_plane = 1.0;
    s->smoothness = 1.0;
    s->anchor = 0.0;
    s->landmark = 1.0;
    s->robust_kernel = NRICP_ROBUST_HUBER;
    s->robust_threshold = 0.0;
    s->max_outer_iterations = 10;
    s->max_inner_iterations = 10;
    s->outer_tolerance = 1e-3;
    s->inner_tolerance = 1e-4;
}

void nricp_default_desc(NricpSolveDesc* d) {
    std::memset(d, 0, sizeof *d);
    d->distance_threshold = std::numeric_limits<double>::infinity();
    d->min_normal_cosine = -1.0;
    d->min_slope = 0.0;
    d->initial_damping = 1e-3;
    d->damping_decrease = 0.3;
    d->damping_increase = 4.0;
    d->max_damping_attempts = 6;
    d->diagonal_damping = 1;
    d->graph_levels = 4;
    d->nodes_initial = 100;
    d->growth = 2;
    d->pcg_tolerance = 1e-5;
    d->pcg_max_iterations = 60;
    d->max_nodes_per_vertex = 4;
    d->edge_neighbours = 4;
    d->route = NRICP_ROUTE_B;
}

const char* nricp_last_error(void) { return g_last_error.c_str(); }

int nricp_transfer_counters(unsigned long long* h2d, unsigned long long* d2h, int reset) {
    *h2d = g_transfers.h2d;
    *d2h = g_transfers.d2h;
    if (reset) g_transfers = TransferCounters{};
    return NRICP_OK;
}

int nricp_device_info(int* available, char* description, size_t capacity) {
    return guarded([&] {
        int count = 0;
        const bool ok = cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
        if (!ok) cudaGetLastError();
        *available = ok ? 1 : 0;
        std::string text = "no CUDA device";
        if (ok) {
            cudaDeviceProp p{};
            int device = 0;
            cudaGetDevice(&device);
            if (cudaGetDeviceProperties(&p, device) == cudaSuccess)
                text = std::string(p.name) + " (cc " + std::to_string(p.major) + "." +
                       std::to_string(p.minor) + ", " + std::to_string(p.multiProcessorCount) + " SMs)";
        }
        if (description && capacity) {
            std::strncpy(description, text.c_str(), capacity - 1);
            description[capacity - 1] = 0;
        }
    });
}

int nricp_plan(const NricpSolveDesc* desc, int32_t* level_nodes, int capacity, int* level_count) {
    return guarded([&] {
        const int levels = desc->graph_levels > 1 ? desc->graph_levels : 1;
        *level_count = levels;
        for (int l = 0; l < levels && l < capacity; ++l)
            level_nodes[l] = level_node_count(l, desc->nodes_initial, desc->growth,
                                              desc->template_vertex_count);
    });
}

// ---- sessions ----------------------------------------------------------------

int nricp_session_create(const NricpSolveDesc* desc, NricpSession** out) {
    *out = nullptr;
    return guarded([&] {
        validate_settings(*desc);
        require_device();
        auto session = std::make_unique<NricpSession>();
        session->batch.add(*desc);
        session->batch.upload_all();
        *out = session.release();
    });
}

int nricp_session_step(NricpSession* s, NricpProgress* progress) {
    return guarded([&] {
        s->batch.pull_controls();
        if (!s->batch.all_done()) {
            s->batch.tick();
            s->batch.pull_controls();
            if (s->batch.all_done()) s->batch.finish();
        }
        if (progress) fill_progress(s->batch.control(0), progress);
    });
}

int nricp_session_run(NricpSession* s) {
    return guarded([&] { s->batch.run(); });
}

int nricp_session_finished(NricpSession* s, int* finished) {
    return guarded([&] {
        s->batch.pull_controls();
        *finished = s->batch.all_done() ? 1 : 0;
    });
}

int nricp_session_vertices(NricpSession* s, double* out) {
    return guarded([&] { s->batch.current_vertices(0, out); });
}

int nricp_session_result(NricpSession* s, NricpResult* out) {
    return guarded([&] {
        s->batch.pull_controls();
        s->batch.result(0, out);
    });
}

int nricp_session_ticks(NricpSession* s, long* ticks, long* launches) {
    return guarded([&] {
        *ticks = s->batch.ticks();
        *launches = s->batch.launches();
    });
}

int nricp_session_inspect(NricpSession* s, NricpInspect* out) {
    return guarded([&] { s->batch.inspect(0, out); });
}

void nricp_session_destroy(NricpSession* s) { delete s; }

// ---- one-call solves -------------------------------------------------------

int nricp_solve(const NricpSolveDesc* desc, NricpResult* out) {
    return guarded([&] {
        validate_settings(*desc);
        require_device();
        Batch batch;
        batch.add(*desc);
        batch.upload_all();
        batch.run();
        batch.result(0, out);
    });
}

// ---- batches ---------------------------------------------------------------

int nricp_batch_create(const NricpSolveDesc* descs, int count, NricpBatch** out) {
    *out = nullptr;
    return guarded([&] {
        if (count <= 0) throw InvalidArgument("a batch needs at least one wrap");
        require_device();
        auto b = std::make_unique<NricpBatch>();
        b->batch.add_all(descs, count);
        b->batch.upload_all();
        *out = b.release();
    });
}

int nricp_batch_reset(NricpBatch* b) { return guarded([&] { b->batch.reset(); }); }

int nricp_batch_run(NricpBatch* b) { return guarded([&] { b->batch.run(); }); }

int nricp_batch_result(NricpBatch* b, int index, NricpResult* out) {
    return guarded([&] {
        if (index < 0 || index >= b->batch.size()) throw InvalidArgument("wrap index out of range");
        b->batch.result(index, out);
    });
}

int nricp_batch_counters(NricpBatch* b, long* ticks, long* launches) {
    return guarded([&] {
        *ticks = b->batch.ticks();
        *launches = b->batch.launches();
    });
}

int nricp_batch_profile(NricpBatch* b, double* query_ms, double* pcg_ms, double* assemble_ms,
                        long* ticks) {
    return guarded([&] {
        KernelTimers t{};
        t.active = true;
        check(cudaEventCreate(&t.query_begin), "event");
        check(cudaEventCreate(&t.query_end), "event");
        check(cudaEventCreate(&t.pcg_begin), "event");
        check(cudaEventCreate(&t.pcg_end), "event");
        check(cudaEventCreate(&t.assemble_begin), "event");
        check(cudaEventCreate(&t.assemble_end), "event");
        std::vector<float> q, p, a;
        b->batch.reset();
        b->batch.run_timed(&t, &q, &p, &a);
        double sq = 0, sp = 0, sa = 0;
        for (float v : q) sq += v;
        for (float v : p) sp += v;
        for (float v : a) sa += v;
        *query_ms = sq;
        *pcg_ms = sp;
        *assemble_ms = sa;
        *ticks = static_cast<long>(q.size());
        cudaEventDestroy(t.query_begin); cudaEventDestroy(t.query_end);
        cudaEventDestroy(t.pcg_begin); cudaEventDestroy(t.pcg_end);
        cudaEventDestroy(t.assemble_begin); cudaEventDestroy(t.assemble_end);
    });
}

int nricp_batch_step(NricpBatch* b, double* device_ms) {
    return guarded([&] { *device_ms = b->batch.timed_step(); });
}

int nricp_batch_tune(NricpBatch* b, int pcg_cluster, int* cluster_out) {
    return guarded([&] {
        b->batch.set_pcg_cluster(pcg_cluster);
        if (cluster_out) *cluster_out = b->batch.shape().pcg_cluster;
    });
}

int nricp_batch_tick_records(NricpBatch* b, NricpTickRecord* out, int capacity, int* count) {
    return guarded([&] {
        const auto& records = b->batch.tick_records();
        *count = static_cast<int>(records.size());
        for (int i = 0; i < *count && i < capacity; ++i) {
            out[i].phase = records[i].phase;
            out[i].level = records[i].level;
            out[i].pcg_iterations = records[i].pcg_iterations;
            out[i].query_ms = records[i].query_ms;
            out[i].pcg_ms = records[i].pcg_ms;
            out[i].assemble_ms = records[i].assemble_ms;
            out[i].tick_ms = records[i].tick_ms;
        }
    });
}

int nricp_batch_level_sizes(NricpBatch* b, int index, int level, int32_t* sizes) {
    return guarded([&] {
        if (index < 0 || index >= b->batch.size()) throw InvalidArgument("wrap index out of range");
        if (level < 0 || level >= b->batch.levels(index)) throw InvalidArgument("level out of range");
        int v[Batch::kLevelSizeEntries];
        b->batch.level_sizes(index, level, v);
        for (int i = 0; i < Batch::kLevelSizeEntries; ++i) sizes[i] = v[i];
    });
}

void nricp_batch_destroy(NricpBatch* b) { delete b; }

int nricp_batch_solve(const NricpSolveDesc* descs, int count, NricpResult* results) {
    return guarded([&] {
        if (count <= 0) throw InvalidArgument("a batch needs at least one wrap");
        require_device();
        Batch batch;
        batch.add_all(descs, count);
        batch.upload_all();
        batch.run();
        batch.results(results);
    });
}

// ---- components ----------------------------------------------------------------

int nricp_template_graph_level(const double* points, int count, int levels, int nodes_initial,
                               int growth, int max_nodes, int edge_neighbours, int level,
                               double* center, double* scale, int32_t* template_indices,
                               double* node_positions, int32_t* bind_nodes, double* bind_weights,
                               int32_t* bind_counts, int32_t* edges, int edge_capacity,
                               int* edge_count, int use_device) {
    return guarded([&] {
        if (count <= 0) throw InvalidArgument("invalid mesh: mesh has no vertices");
        if (max_nodes > NRICP_MAX_SLOTS) throw InvalidArgument("max_nodes_per_vertex exceeds 8");
        TemplateGraph g;
        if (use_device && device_graph_supported(edge_neighbours)) {
            require_device();
            cudaStream_t stream;
            check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
            try {
                g = std::move(device_template_graphs(
                    {GraphRequest{points, count, levels, nodes_initial, growth, max_nodes, edge_neighbours}},
                    stream)[0]);
            } catch (...) {
                cudaStreamDestroy(stream);
                throw;
            }
            cudaStreamDestroy(stream);
        } else {
            g = build_template_graph(points, count, levels, nodes_initial, growth, max_nodes,
                                     edge_neighbours);
        }
        if (level < 0 || level >= static_cast<int>(g.levels.size()))
            throw InvalidArgument("level out of range");
        const GraphLevel& L = g.levels[level];
        for (int k = 0; k < 3; ++k) center[k] = g.center[k];
        *scale = g.scale;
        const int N = L.node_count();
        std::memcpy(template_indices, L.template_index.data(), sizeof(int32_t) * N);
        std::memcpy(node_positions, L.rest.data(), sizeof(double) * 3 * N);
        for (int v = 0; v < count; ++v) {
            for (int s = 0; s < NRICP_MAX_SLOTS; ++s) {
                bind_nodes[v * NRICP_MAX_SLOTS + s] = L.bindings[v].nodes[s];
                bind_weights[v * NRICP_MAX_SLOTS + s] = L.bindings[v].weights[s];
            }
            bind_counts[v] = L.bindings[v].count;
        }
        const int E = static_cast<int>(L.edges.size() / 2);
        *edge_count = E;
        if (E > edge_capacity) throw InvalidArgument("edge buffer too small");
        std::memcpy(edges, L.edges.data(), sizeof(int32_t) * 2 * E);
    });
}

int nricp_farthest_point_seeds(const double* points, int point_count, int count, int first_index,
                               int32_t* out, int* written) {
    return guarded([&] {
        if (point_count < 0) throw InvalidArgument("points must have shape (n, 3)");
        const std::vector<double> p(points, points + static_cast<size_t>(point_count) * 3);
        const std::vector<int> seeds = farthest_point_seeds(p, count, first_index);
        for (size_t i = 0; i < seeds.size(); ++i) out[i] = seeds[i];
        *written = static_cast<int>(seeds.size());
    });
}

int nricp_bind_vertices(const double* points, int point_count, const double* nodes, int node_count,
                        int max_nodes, int32_t* out_nodes, double* out_weights, int32_t* out_counts) {
    return guarded([&] {
        if (point_count < 0 || node_count < 0) throw InvalidArgument("points and nodes must have shape (n, 3)");
        if (max_nodes > NRICP_MAX_SLOTS) throw InvalidArgument("max_nodes_per_vertex exceeds 8");
        const std::vector<double> p(points, points + static_cast<size_t>(point_count) * 3);
        const std::vector<double> q(nodes, nodes + static_cast<size_t>(node_count) * 3);
        const std::vector<Binding> b = bind_vertices(p, q, max_nodes, NRICP_MAX_SLOTS);
        for (int v = 0; v < point_count; ++v) {
            for (int s = 0; s < NRICP_MAX_SLOTS; ++s) {
                out_nodes[static_cast<size_t>(v) * NRICP_MAX_SLOTS + s] = b[v].nodes[s];
                out_weights[static_cast<size_t>(v) * NRICP_MAX_SLOTS + s] = b[v].weights[s];
            }
            out_counts[v] = b[v].count;
        }
    });
}

int nricp_vertex_normals(const double* points, int point_count, const int32_t* faces, int face_count,
                         double* out) {
    return guarded([&] {
        if (point_count < 0 || face_count < 0) throw InvalidArgument("points and faces must have shape (n, 3)");
        for (long i = 0; i < static_cast<long>(face_count) * 3; ++i)
            if (faces[i] < 0 || faces[i] >= point_count)
                throw InvalidArgument("face " + std::to_string(i / 3) + " references a missing vertex");
        vertex_normals_into(points, point_count, faces, face_count, out);
    });
}

int nricp_fit_rigid(const double* source_points, const double* target_points, const double* weights,
                    int count, double* rotation, double* translation) {
    return guarded([&] {
        if (count < 0) throw InvalidArgument("fit_rigid expects (n, 3) point pairs and (n,) weights");
        require_device();
        const size_t n = static_cast<size_t>(count);
        const size_t bytes = sizeof(double) * (7 * std::max<size_t>(1, n) + 12);
        char* base = nullptr;
        check(cudaMalloc(&base, bytes), "cudaMalloc(rigid fit)");
        std::unique_ptr<char, void (*)(char*)> guard(base, [](char* p) { cudaFree(p); });
        double* src = reinterpret_cast<double*>(base);
        double* dst = src + 3 * std::max<size_t>(1, n);
        double* w = dst + 3 * std::max<size_t>(1, n);
        double* out = w + std::max<size_t>(1, n);
        cudaStream_t stream;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> stream_guard(stream, [](cudaStream_t s) {
            cudaStreamDestroy(s);
        });
        if (n > 0) {
            check(cudaMemcpyAsync(src, source_points, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, stream), "upload");
            check(cudaMemcpyAsync(dst, target_points, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, stream), "upload");
            check(cudaMemcpyAsync(w, weights, sizeof(double) * n, cudaMemcpyHostToDevice, stream), "upload");
        }
        launch_fit_rigid(src, dst, w, count, out, stream);
        check(cudaGetLastError(), "rigid fit");
        double host[12];
        check(cudaMemcpyAsync(host, out, sizeof host, cudaMemcpyDeviceToHost, stream), "download");
        check(cudaStreamSynchronize(stream), "rigid fit");
        std::memcpy(rotation, host, sizeof(double) * 9);
        std::memcpy(translation, host + 9, sizeof(double) * 3);
    });
}

int nricp_closest_points(const double* target_points, int vertex_count, const int32_t* faces,
                         int face_count, const double* queries, int query_count,
                         double* out_points, double* out_normals, double* out_distances,
                         int32_t* out_triangles) {
    return guarded([&] {
        validate_mesh(target_points, vertex_count, faces, face_count, "target");
        require_device();
        cudaStream_t stream;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        const std::vector<double> pts(target_points, target_points + (size_t)vertex_count * 3);
        const std::vector<double> normals = vertex_normals(pts, faces, face_count);
        size_t bytes = 0;
        auto reserve = [&bytes](size_t n) { size_t at = bytes; bytes += (n + 255) & ~size_t(255); return at; };
        const size_t o_p = reserve(sizeof(double) * pts.size());
        const size_t o_n = reserve(sizeof(double) * normals.size());
        const size_t o_f = reserve(sizeof(int32_t) * 3 * face_count);
        const size_t o_nodes = reserve(sizeof(float4) * 4 * std::max(1, face_count - 1));
        const size_t o_leaves = reserve(sizeof(float4) * kLeafFloat4s * face_count);
        const size_t o_q = reserve(sizeof(double) * 3 * std::max(1, query_count));
        const size_t o_op = reserve(sizeof(double) * 3 * std::max(1, query_count));
        const size_t o_on = reserve(sizeof(double) * 3 * std::max(1, query_count));
        const size_t o_od = reserve(sizeof(double) * std::max(1, query_count));
        const size_t o_ot = reserve(sizeof(int32_t) * std::max(1, query_count));
        const size_t o_flag = reserve(sizeof(int));
        const size_t o_wrap = reserve(sizeof(WrapDev));
        const size_t o_scratch = reserve(lbvh_scratch_bytes(face_count));
        char* base = nullptr;
        check(cudaMalloc(&base, bytes), "cudaMalloc(closest points)");
        std::unique_ptr<char, void (*)(char*)> guard(base, [](char* p) { cudaFree(p); });
        WrapDev w;
        std::memset(&w, 0, sizeof w);
        w.Vt = vertex_count;
        w.F = face_count;
        w.tgt_points = reinterpret_cast<double*>(base + o_p);
        w.tgt_normals = reinterpret_cast<double*>(base + o_n);
        w.tgt_faces = reinterpret_cast<int32_t*>(base + o_f);
        w.bvh_nodes = reinterpret_cast<float4*>(base + o_nodes);
        w.bvh_leaves = reinterpret_cast<float4*>(base + o_leaves);
        {
            double lo[3], hi[3];
            for (int k = 0; k < 3; ++k) lo[k] = hi[k] = pts[k];
            for (int i = 0; i < vertex_count; ++i)
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::min(lo[k], pts[i * 3 + k]);
                    hi[k] = std::max(hi[k], pts[i * 3 + k]);
                }
            const double d = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                       (hi[2] - lo[2]) * (hi[2] - lo[2]));
            w.rank_window = static_cast<float>(4e-6 * d);
        }
        check(cudaMemcpyAsync(base + o_p, pts.data(), sizeof(double) * pts.size(), cudaMemcpyHostToDevice, stream), "upload");
        check(cudaMemcpyAsync(base + o_n, normals.data(), sizeof(double) * normals.size(), cudaMemcpyHostToDevice, stream), "upload");
        check(cudaMemcpyAsync(base + o_f, faces, sizeof(int32_t) * 3 * face_count, cudaMemcpyHostToDevice, stream), "upload");
        if (query_count > 0)
            check(cudaMemcpyAsync(base + o_q, queries, sizeof(double) * 3 * query_count, cudaMemcpyHostToDevice, stream), "upload");
        check(cudaMemsetAsync(base + o_flag, 0, sizeof(int), stream), "flag");
        w.bvh_root = static_cast<int>(lbvh_build(w.tgt_points, w.tgt_faces, face_count, base + o_scratch,
                                                 const_cast<float4*>(w.bvh_nodes),
                                                 const_cast<float4*>(w.bvh_leaves), stream, nullptr));
        check(cudaMemcpyAsync(base + o_wrap, &w, sizeof w, cudaMemcpyHostToDevice, stream), "upload");
        if (query_count > 0) {
            launch_closest_points(reinterpret_cast<WrapDev*>(base + o_wrap),
                                  reinterpret_cast<double*>(base + o_q), query_count,
                                  reinterpret_cast<double*>(base + o_op),
                                  reinterpret_cast<double*>(base + o_on),
                                  reinterpret_cast<double*>(base + o_od),
                                  reinterpret_cast<int32_t*>(base + o_ot),
                                  reinterpret_cast<int*>(base + o_flag), stream);
            check(cudaGetLastError(), "closest points");
            check(cudaMemcpyAsync(out_points, base + o_op, sizeof(double) * 3 * query_count, cudaMemcpyDeviceToHost, stream), "download");
            check(cudaMemcpyAsync(out_normals, base + o_on, sizeof(double) * 3 * query_count, cudaMemcpyDeviceToHost, stream), "download");
            check(cudaMemcpyAsync(out_distances, base + o_od, sizeof(double) * query_count, cudaMemcpyDeviceToHost, stream), "download");
            check(cudaMemcpyAsync(out_triangles, base + o_ot, sizeof(int32_t) * query_count, cudaMemcpyDeviceToHost, stream), "download");
        }
        int flag = 0;
        check(cudaMemcpyAsync(&flag, base + o_flag, sizeof(int), cudaMemcpyDeviceToHost, stream), "download");
        check(cudaStreamSynchronize(stream), "closest points");
        cudaStreamDestroy(stream);
        if (flag) throw StateError("a closest-point traversal exceeded its stack");
    });
}

int nricp_lbvh_export(const double* target_points, int vertex_count, const int32_t* faces,
                      int face_count, uint32_t* codes, uint32_t* order, int32_t* left,
                      int32_t* right, float* bounds) {
    return guarded([&] {
        validate_mesh(target_points, vertex_count, faces, face_count, "target");
        require_device();
        cudaStream_t stream;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        char* base = nullptr;
        size_t bytes = 0;
        auto reserve = [&bytes](size_t n) { size_t at = bytes; bytes += (n + 255) & ~size_t(255); return at; };
        const size_t o_p = reserve(sizeof(double) * 3 * vertex_count);
        const size_t o_f = reserve(sizeof(int32_t) * 3 * face_count);
        const size_t o_nodes = reserve(sizeof(float4) * 4 * std::max(1, face_count - 1));
        const size_t o_leaves = reserve(sizeof(float4) * kLeafFloat4s * face_count);
        const size_t o_scratch = reserve(lbvh_scratch_bytes(face_count));
        check(cudaMalloc(&base, bytes), "cudaMalloc(lbvh)");
        std::unique_ptr<char, void (*)(char*)> guard(base, [](char* p) { cudaFree(p); });
        check(cudaMemcpyAsync(base + o_p, target_points, sizeof(double) * 3 * vertex_count, cudaMemcpyHostToDevice, stream), "upload");
        check(cudaMemcpyAsync(base + o_f, faces, sizeof(int32_t) * 3 * face_count, cudaMemcpyHostToDevice, stream), "upload");
        LbvhExport out{codes, order, left, right, bounds};
        lbvh_build(reinterpret_cast<double*>(base + o_p), reinterpret_cast<int32_t*>(base + o_f),
                   face_count, base + o_scratch, reinterpret_cast<float4*>(base + o_nodes),
                   reinterpret_cast<float4*>(base + o_leaves), stream, &out);
        check(cudaGetLastError(), "lbvh build");
        check(cudaStreamSynchronize(stream), "lbvh build");
        cudaStreamDestroy(stream);
    });
}


// ---- serving -------------------------------------------------------------

// One or two lanes: a lane is a Server (own slots, stream, ticks and memory
// pool).  Every tick of a lane runs in lockstep, so a request whose target
// has a million triangles would slow every smaller request sharing its
// ticks; large requests therefore get a lane of their own, whose ticks run
// beside the other lane's on the device.  Request ids are the composite's.
struct NricpServer {
    std::vector<std::unique_ptr<Server>> lanes;  // [0] regular, [1] large (if any)
    int large_faces = 0;
    std::mutex mu;
    std::map<long, std::pair<int, long>> ids;  // id -> (lane, the lane's id)
    long next_id = 1;

    std::pair<int, long> find(long id) {
        std::lock_guard<std::mutex> lk(mu);
        auto it = ids.find(id);
        if (it == ids.end()) throw InvalidArgument("unknown request id " + std::to_string(id));
        return it->second;
    }
};

void nricp_server_default_config(NricpServerConfig* c) {
    c->memory_budget_bytes = 0;
    c->max_slots = 64;
    c->prep_threads = 0;
    c->pcg_cluster = 0;
    c->ticks_per_poll = 8;
    c->large_face_threshold = 1000000;
    c->large_slots = 8;
}

int nricp_server_create(const NricpServerConfig* config, NricpServer** out) {
    *out = nullptr;
    return guarded([&] {
        require_device();
        NricpServerConfig c;
        nricp_server_default_config(&c);
        if (config) c = *config;
        if (c.large_face_threshold < 0) throw InvalidArgument("large_face_threshold must be >= 0");
        auto s = std::make_unique<NricpServer>();
        if (c.large_face_threshold == 0) {
            s->lanes.push_back(std::make_unique<Server>(c));
        } else {
            if (c.large_slots <= 0 || c.large_slots > 1024)
                throw InvalidArgument("large_slots is " + std::to_string(c.large_slots) + "; it must be 1 to 1024");
            size_t budget = c.memory_budget_bytes;
            if (budget == 0) {
                size_t free_bytes = 0, total = 0;
                check(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
                budget = free_bytes / 10 * 9;
            }
            const int cores = static_cast<int>(std::thread::hardware_concurrency());
            NricpServerConfig regular = c, large = c;
            regular.memory_budget_bytes = budget - budget / 3;
            large.memory_budget_bytes = budget / 3;
            large.max_slots = c.large_slots;
            if (c.prep_threads <= 0) {
                regular.prep_threads = std::max(1, cores / 2 - std::max(1, cores / 8));
                large.prep_threads = std::max(1, cores / 8);
            }
            s->lanes.push_back(std::make_unique<Server>(regular));
            s->lanes.push_back(std::make_unique<Server>(large));
            s->large_faces = c.large_face_threshold;
        }
        *out = s.release();
    });
}

int nricp_server_submit(NricpServer* s, const NricpSolveDesc* desc, long* id) {
    return guarded([&] {
        const int lane = s->lanes.size() > 1 && desc && desc->target_face_count >= s->large_faces ? 1 : 0;
        const long inner = s->lanes[lane]->submit(*desc);
        std::lock_guard<std::mutex> lk(s->mu);
        *id = s->next_id++;
        s->ids[*id] = {lane, inner};
    });
}

int nricp_server_poll(NricpServer* s, long id, int* status, double* latency_seconds) {
    return guarded([&] {
        const auto [lane, inner] = s->find(id);
        *status = s->lanes[lane]->poll(inner, latency_seconds);
    });
}

int nricp_server_phases(NricpServer* s, long id, double* seconds) {
    return guarded([&] {
        const auto [lane, inner] = s->find(id);
        s->lanes[lane]->phases(inner, seconds);
    });
}

int nricp_server_wait(NricpServer* s, long id, double timeout_seconds) {
    return guarded([&] {
        const auto [lane, inner] = s->find(id);
        if (!s->lanes[lane]->wait(inner, timeout_seconds))
            throw TimeoutError("request " + std::to_string(id) + " did not finish in time");
    });
}

int nricp_server_result(NricpServer* s, long id, NricpResult* out) {
    return guarded([&] {
        const auto [lane, inner] = s->find(id);
        double latency = 0.0;
        const int state = s->lanes[lane]->poll(inner, &latency);
        auto forget = [&] {
            std::lock_guard<std::mutex> lk(s->mu);
            s->ids.erase(id);
        };
        try {
            s->lanes[lane]->result(inner, out);
        } catch (...) {
            if (state == NRICP_REQUEST_FAILED) forget();  // the lane has forgotten it too
            throw;
        }
        forget();
    });
}

int nricp_server_stats(NricpServer* s, NricpServerStats* out) {
    return guarded([&] {
        std::vector<Server*> lanes;
        for (auto& lane : s->lanes) lanes.push_back(lane.get());
        *out = Server::merged_stats(lanes);
    });
}

void nricp_server_destroy(NricpServer* s) { delete s; }

}  // extern "C"
