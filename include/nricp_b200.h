/*
 * nricp_b200 -- C-ABI of the B200-native non-rigid ICP wrapping path.
 *
 * The reference ships its solve routes only as the pybind11 module `nricp_dp`
 * (src/python/bindings.cpp:714); it has no C ABI.  Every entry point below is
 * what that module's route B / route C surface binds, flattened to plain
 * pointers and sizes so that a cgo / JNI / ctypes / pybind11 caller can bind it
 * directly.  Each declaration names the reference interface it replaces.
 *
 * Conventions
 *   - Every function returns an int status (NRICP_OK on success).  The message
 *     of the last failure on the calling thread is nricp_last_error().
 *   - Outputs are caller-allocated.  Sizes are known up front from
 *     nricp_plan() (node counts per level) and the input sizes.
 *   - Points are double precision, row-major (n, 3); faces are int32 (m, 3).
 *   - Distances (distance_threshold, robust_threshold) are in the caller's
 *     units, exactly as the reference's route functions take them
 *     (src/python/bindings.cpp:631-639).
 */
#ifndef NRICP_B200_H
#define NRICP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  INVALID maps to the reference's py::value_error /
 * std::invalid_argument (ValueError), CUDA and DEVICE to std::runtime_error
 * (RuntimeError), see src/cuda/cuda_error.h:14-19 and
 * src/python/bindings.cpp:557-570. */
enum {
    NRICP_OK = 0,
    NRICP_ERR_INVALID = 1,   /* caller error: shapes, indices, settings */
    NRICP_ERR_CUDA = 2,      /* a CUDA call failed */
    NRICP_ERR_NO_DEVICE = 3, /* no usable sm_100 device */
    NRICP_ERR_CAPACITY = 4,  /* output buffer too small / budget exceeded */
    NRICP_ERR_STATE = 5,     /* call not valid in the object's current state */
    NRICP_ERR_TIMEOUT = 6    /* a bounded device wait gave up */
};

/* Maximum binding support per vertex.  The reference hard-codes 4
 * (src/core/sampling.h:17); the BASELINE configs ask for 6 and 8. */
#define NRICP_MAX_SLOTS 8

/* Robust kernels, src/energy/robust.h:9-13. */
enum { NRICP_ROBUST_NONE = 0, NRICP_ROBUST_HUBER = 1, NRICP_ROBUST_GEMAN_MCCLURE = 2 };

/* Device routes, src/cuda/gpu_solver.cuh:19-26. */
enum { NRICP_ROUTE_B = 0, NRICP_ROUTE_C = 1 };

/* One level of the coarse-to-fine schedule: LevelSettings,
 * src/solver/route_a.h:17-25, parsed from the level dict at
 * src/python/bindings.cpp:181-196 (same defaults). */
typedef struct NricpLevelSettings {
    double point_to_point;   /* 1.0 */
    double point_to_plane;   /* 1.0 */
    double smoothness;       /* 1.0 */
    double anchor;           /* 0.0 */
    double landmark;         /* 1.0 */
    int robust_kernel;       /* NRICP_ROBUST_HUBER */
    double robust_threshold; /* 0.0 (caller units; 0 disables reweighting) */
    int max_outer_iterations;  /* 10 */
    int max_inner_iterations;  /* 10 */
    double outer_tolerance;    /* 1e-3 */
    double inner_tolerance;    /* 1e-4 */
} NricpLevelSettings;

/* Everything one wrap needs: the arguments of solve_route_b/solve_route_c
 * (src/python/bindings.cpp:1426-1481), same meaning and defaults, plus the
 * extensions the BASELINE configs need (k > 4 bindings, k-NN edges). */
typedef struct NricpSolveDesc {
    const double* template_points; /* (template_vertex_count, 3) */
    int template_vertex_count;
    const int32_t* template_faces; /* (template_face_count, 3) */
    int template_face_count;
    const double* target_points;   /* (target_vertex_count, 3) */
    int target_vertex_count;
    const int32_t* target_faces;   /* (target_face_count, 3) */
    int target_face_count;
    const NricpLevelSettings* levels; /* one per level; last reused */
    int level_setting_count;
    const uint8_t* mask;            /* (template_vertex_count,) or NULL */
    const int32_t* landmark_indices; /* (landmark_count,) or NULL */
    const double* landmark_targets;  /* (landmark_count, 3) or NULL */
    int landmark_count;
    double distance_threshold;  /* +inf */
    double min_normal_cosine;   /* -1 */
    double min_slope;           /* 0 */
    double initial_damping;     /* 1e-3 */
    double damping_decrease;    /* 0.3 */
    double damping_increase;    /* 4 */
    int max_damping_attempts;   /* 6 */
    int diagonal_damping;       /* 1 */
    int graph_levels;           /* 4 */
    int nodes_initial;          /* 100 */
    int growth;                 /* 2 */
    double pcg_tolerance;       /* 1e-5 */
    int pcg_max_iterations;     /* 60 */
    /* extensions (0 selects the reference default of 4 for both) */
    int max_nodes_per_vertex;   /* binding support k, <= NRICP_MAX_SLOTS */
    int edge_neighbours;        /* k-NN graph edges */
    int route;                  /* NRICP_ROUTE_B or NRICP_ROUTE_C */
} NricpSolveDesc;

/* Fills `desc` with the reference's defaults; pointers and counts zeroed. */
void nricp_default_desc(NricpSolveDesc* desc);
void nricp_default_level(NricpLevelSettings* level);

/* The result dict of route_result_to_dict (src/python/bindings.cpp:674-710),
 * caller-allocated.  Sizes: vertices template_vertex_count*3; rotations,
 * translations and node_positions use the finest level's node count from
 * nricp_plan(); level_nodes holds one entry per level.  report_json receives
 * the run report (src/core/report.cpp:46-105 format), NUL-terminated;
 * report_length is set to the full length even when it was truncated. */
typedef struct NricpResult {
    double* vertices;
    double* rotations;
    double* translations;
    double* node_positions;
    int32_t* level_nodes;
    char* report_json;
    size_t report_capacity;
    size_t report_length;
} NricpResult;

/* Per-step progress, WrapProgress (src/cuda/gpu_solver.cuh:60-68). */
typedef struct NricpProgress {
    int level;
    int outer;
    int inner;
    int finished;
    int level_converged;
    double energy;
    double correspondence_mean;
} NricpProgress;

/* ---- identity and devices --------------------------------------------- */

/* Message of the last failing call on this thread (the text the reference
 * raises as ValueError / RuntimeError). */
const char* nricp_last_error(void);

/* Bytes this thread has copied host->device and device->host through the
 * library since the last reset (no reference counterpart; for accounting). */
int nricp_transfer_counters(unsigned long long* h2d, unsigned long long* d2h, int reset);

/* device_info(), src/python/bindings.cpp:1614-1622. */
int nricp_device_info(int* available, char* description, size_t capacity);

/* Node count per level for a descriptor (src/core/graph.cpp:52-57): sizes the
 * caller's result buffers.  `level_count` receives the number of levels. */
int nricp_plan(const NricpSolveDesc* desc, int32_t* level_nodes, int capacity,
               int* level_count);

/* ---- the route functions ------------------------------------------------ */

/* solve_route_b / solve_route_c (src/python/bindings.cpp:1422-1492 ->
 * src/cuda/gpu_solver.cu:14-39): one wrap, start to finish, on the current
 * device.  desc->route selects the route. */
int nricp_solve(const NricpSolveDesc* desc, NricpResult* out);

/* ---- the session (RouteBSession, bindings.cpp:1510-1612) ---------------- */

typedef struct NricpSession NricpSession;

/* RouteBSession(...) constructor (bindings.cpp:1513-1561): validates,
 * prepares the template graph, uploads, builds the target hierarchy. */
int nricp_session_create(const NricpSolveDesc* desc, NricpSession** out);
/* .step() (bindings.cpp:1562-1580): advances the schedule by one unit of
 * work -- a correspondence refresh or one damped solve attempt. */
int nricp_session_step(NricpSession* session, NricpProgress* progress);
/* Steps until finished, without host round trips between steps. */
int nricp_session_run(NricpSession* session);
/* .finished() (bindings.cpp:1581-1582). */
int nricp_session_finished(NricpSession* session, int* finished);
/* .vertices() (bindings.cpp:1583-1592): the current fit, caller units,
 * template_vertex_count x 3. */
int nricp_session_vertices(NricpSession* session, double* out);
/* .result() (bindings.cpp:1600-1611): the solve_route_b payload for the state
 * reached so far; .report() is result->report_json. */
int nricp_session_result(NricpSession* session, NricpResult* out);
/* Schedule ticks run and kernels launched so far. */
int nricp_session_ticks(NricpSession* session, long* ticks, long* launches);
/* No reference counterpart.  A session's current linear system and the state
 * it was assembled at, for checking the assembly against an FP64 restatement
 * of the reference's fused_system (bindings.cpp:1328-1360, the same system
 * as (J^T J, -J^T r)).  Call it when the session's phase is a solve
 * attempt right after a refresh: the system is then the one assembled at
 * the accepted state with the correspondences of that state.  All arrays are
 * caller-allocated: rotations (nodes x 9), translations (nodes x 3),
 * correspondence points and normals (template vertices x 3, normalised
 * frame), robust weights (V), rejection codes (V), diagonal blocks
 * (nodes x 36), right-hand side (nodes x 6), and for every off-diagonal block
 * its node pair (a < b) and its (a, b) block (capacity x 2 and capacity x 36).
 * Blocks appear once per smoothness edge and once per node pair that shares
 * a vertex, so one pair may appear twice; their sum is the system's block.
 * Also the damping of the next attempt and the last converged solve's
 * increment (nodes x 6), the correspondences' distances, the last solve's
 * outcome, and the target as the device holds it.  A NULL output pointer is
 * skipped. */
typedef struct NricpInspect {
    int level, node_count, phase, off_count;     /* out */
    int off_capacity;                            /* in */
    double energies[5];                          /* out: accepted energy parts */
    double* rotations;
    double* translations;
    double* corr_points;
    double* corr_normals;
    double* corr_robust;
    uint8_t* corr_codes;
    float* diag;
    float* rhs;
    int32_t* off_nodes;
    float* off_blocks;
    double damping;                              /* out: the next attempt's damping */
    double* delta;                               /* nodes x 6: the last converged solve's increment */
    double* corr_distances;                      /* V (may be NULL): the correspondences' distances */
    int pcg_ok, pcg_iterations;                  /* out: the last solve's outcome and iterations */
    double pcg_residual;                         /* out: its |r| / |b| when it stopped */
    double* target_points;                       /* Vt x 3 (may be NULL): the target, normalised */
    double* target_normals;                      /* Vt x 3 (may be NULL): its vertex normals */
} NricpInspect;
int nricp_session_inspect(NricpSession* session, NricpInspect* out);

void nricp_session_destroy(NricpSession* session);

/* ---- batches: many uneven wraps advanced by the same launches ----------- */

typedef struct NricpBatch NricpBatch;

/* No reference counterpart (the reference solves one wrap per call,
 * src/cuda/gpu_solver.cu:14-39): prepares and uploads `count` wraps. */
int nricp_batch_create(const NricpSolveDesc* descs, int count, NricpBatch** out);
/* Puts every wrap back at the start of its schedule, inputs kept resident. */
int nricp_batch_reset(NricpBatch* batch);
/* Runs every wrap to completion in one stream of shared launches. */
int nricp_batch_run(NricpBatch* batch);
int nricp_batch_result(NricpBatch* batch, int index, NricpResult* out);
int nricp_batch_counters(NricpBatch* batch, long* ticks, long* launches);
/* Re-runs the batch with CUDA events around the closest-point query, the
 * linear solve and the assembly of every tick; totals in milliseconds. */
int nricp_batch_profile(NricpBatch* batch, double* query_ms, double* pcg_ms,
                        double* assemble_ms, long* ticks);
/* Device time (CUDA events on the batch's stream) of one full pass: every
 * wrap reset to the start of its schedule (hierarchies rebuilt) and run to
 * completion.  Inputs stay resident in device memory. */
int nricp_batch_step(NricpBatch* batch, double* device_ms);

/* No reference counterpart.  Cluster size of the batch's linear solve: a
 * power of two from 1 to 16 gives every wrap that many CTAs in one launch;
 * 0 gives each wrap its own size (about 128 nodes per CTA), one launch per
 * size class, the classes running side by side; -s (s = 1..4) halves those
 * per-wrap sizes s times.  A new batch starts at the smallest s whose classes
 * need at most three CTAs per SM.  Every choice gives bit-identical results;
 * it trades one wrap's latency against the batch's throughput.
 * *cluster_out (may be NULL) receives the largest size in effect. */
int nricp_batch_tune(NricpBatch* batch, int pcg_cluster, int* cluster_out);
/* Per-tick records of wrap 0 from the last nricp_batch_profile. */
typedef struct NricpTickRecord {
    int phase;          /* 0 transfer, 1 refresh, 2 solve, 3 final */
    int level;
    int pcg_iterations; /* of this tick's solve */
    int pad;
    float query_ms, pcg_ms, assemble_ms, tick_ms;
} NricpTickRecord;
int nricp_batch_tick_records(NricpBatch* batch, NricpTickRecord* out, int capacity,
                             int* count);
/* Sizes of one level of one wrap (15 entries): nodes, smoothness edges,
 * node-pair groups, (vertex, slot) entries, pair entries, template vertices,
 * target triangles, target vertices, template triangles, level count; then
 * the work the last run did in the level: solves, PCG iterations,
 * closest-point queries (passes over the template), assemblies; last, the
 * system's off-diagonal blocks (one per node pair it couples). */
int nricp_batch_level_sizes(NricpBatch* batch, int index, int level, int32_t* sizes);
void nricp_batch_destroy(NricpBatch* batch);
/* One call: create, run, results, destroy. */
int nricp_batch_solve(const NricpSolveDesc* descs, int count, NricpResult* results);

/* ---- components ---------------------------------------------------------- */

/* ---- serving: continuous batching (no reference counterpart) ----------
 * The reference solves one wrap per call.  A server keeps a set of resident
 * wrap slots on one device and advances every running wrap by the same
 * launches, tick by tick; requests that arrive while others run are
 * prepared on host threads (graph and level layouts, cached per template),
 * admitted into a free slot as soon as one is free and the device-memory
 * budget allows, and retired -- result downloaded -- when their schedule
 * ends.  A wrap's result does not depend on what else shares its launches:
 * it is bit-identical to the same wrap solved alone. */
typedef struct NricpServer NricpServer;
typedef struct NricpServerConfig {
    size_t memory_budget_bytes;  /* device bytes resident wraps may hold; 0: 90 % of free memory */
    int max_slots;               /* wraps resident at once (1..1024) */
    int prep_threads;            /* host threads preparing requests; 0: half the cores */
    int pcg_cluster;             /* solve cluster: > 0 one size (a power of two up to 16) for every
                                    slot; 0 (the default) per-wrap latency classes, halved once
                                    when the running wraps would need more than three CTAs per
                                    SM; -s (1..4) latency classes always halved s times */
    int ticks_per_poll;          /* ticks launched between looks at the wraps' progress */
    int large_face_threshold;    /* requests whose target has at least this many triangles run
                                    in a lane of their own, with its own slots, stream and
                                    ticks, so that they do not slow the others' ticks; 0: one
                                    lane for all (default 1,000,000) */
    int large_slots;             /* slots of the large lane (default 8); it gets a third of the
                                    memory budget */
} NricpServerConfig;
typedef struct NricpServerStats {
    long submitted, completed, failed, waiting, running;
    double latency_p50_ms, latency_p99_ms, latency_mean_ms;  /* submit -> result ready */
    double queue_p50_ms;                                     /* submit -> admitted */
    double wraps_per_second;     /* completed / (last completion - first submission) */
    long ticks, launches, captures;
    double busy_seconds;         /* device time of the tick launches */
    size_t resident_bytes, peak_resident_bytes;
    int slots_used;
} NricpServerStats;
/* Request status from nricp_server_poll. */
enum { NRICP_REQUEST_WAITING = 0, NRICP_REQUEST_RUNNING = 1, NRICP_REQUEST_DONE = 2,
       NRICP_REQUEST_FAILED = 3 };

void nricp_server_default_config(NricpServerConfig* config);
int nricp_server_create(const NricpServerConfig* config, NricpServer** out);
/* Copies the inputs and validates them (NRICP_ERR_INVALID with the
 * reference's messages); the request then runs in the background. */
int nricp_server_submit(NricpServer* server, const NricpSolveDesc* desc, long* id);
/* Status of a request and, once done, its latency (submit to result ready). */
int nricp_server_poll(NricpServer* server, long id, int* status, double* latency_seconds);
/* No reference counterpart.  Where a request's latency went, in seconds, so
 * far: seconds[0] host preparation (graph, level layouts), [1] loading
 * (waiting for memory, uploads, target hierarchy), [2] waiting for a slot,
 * [3] on the device, [4] composing the result; a phase not reached yet is 0.
 * Valid until nricp_server_result takes the request. */
int nricp_server_phases(NricpServer* server, long id, double* seconds);
/* Blocks until the request is done or failed, or `timeout_seconds` pass
 * (NRICP_ERR_TIMEOUT). */
int nricp_server_wait(NricpServer* server, long id, double timeout_seconds);
/* Copies a done request's result (sizes as nricp_solve's) and forgets it; a
 * failed request returns its error. */
int nricp_server_result(NricpServer* server, long id, NricpResult* out);
int nricp_server_stats(NricpServer* server, NricpServerStats* out);
/* Stops the server; requests still running are abandoned. */
void nricp_server_destroy(NricpServer* server);

/* build_template_graph(...) (bindings.cpp:886-925), one level: the
 * normalisation, the sampled nodes, the bindings (stride NRICP_MAX_SLOTS) and
 * the k-NN edges of `level`.  `use_device` (the reference's own flag) builds
 * it on the GPU, bit-identical to the host build. */
int nricp_template_graph_level(const double* points, int count, int levels,
                               int nodes_initial, int growth, int max_nodes,
                               int edge_neighbours, int level, double* center,
                               double* scale, int32_t* template_indices,
                               double* node_positions, int32_t* bind_nodes,
                               double* bind_weights, int32_t* bind_counts,
                               int32_t* edges, int edge_capacity, int* edge_count,
                               int use_device);

/* farthest_point_seeds(points, count, first_index) (bindings.cpp:796-804,
 * src/core/sampling.cpp:47-88): deterministic farthest-point sampling, ties
 * to the lower index; first_index is clamped into range.  Writes
 * min(count, point_count) indices (none when either is <= 0) and their
 * number to *written.  Host code, the graph build's own. */
int nricp_farthest_point_seeds(const double* points, int point_count, int count, int first_index,
                               int32_t* out, int* written);
/* bind_vertices(points, nodes, max_nodes) (bindings.cpp:806-815,
 * sampling.cpp:90-143): each point's nearest max_nodes (1..8) nodes with the
 * reference's distance-ratio weights.  out_nodes / out_weights: point_count x
 * NRICP_MAX_SLOTS (-1 / 0 past the count); out_counts: point_count. */
int nricp_bind_vertices(const double* points, int point_count, const double* nodes, int node_count,
                        int max_nodes, int32_t* out_nodes, double* out_weights, int32_t* out_counts);
/* vertex_normals(points, faces) (bindings.cpp:1014-1024, mesh.cpp:71-88):
 * area-weighted vertex normals, zero where a vertex has no area. */
int nricp_vertex_normals(const double* points, int point_count, const int32_t* faces, int face_count,
                         double* out);

/* fit_rigid(source_points, target_points, weights) (bindings.cpp:857-883,
 * src/core/deformation.cpp:86-139), on the device: the weighted rigid
 * transform (reflections excluded) that best maps `count` source points onto
 * their targets; weights below zero count as zero.  rotation: 9 doubles,
 * row-major; translation: 3.  With no points or no positive weight, the
 * identity and zero, as the reference.  Host pointers. */
int nricp_fit_rigid(const double* source_points, const double* target_points, const double* weights,
                    int count, double* rotation, double* translation);

/* closest_points(...) (bindings.cpp:1004-1044 -> src/cuda/lbvh.cu:439-533):
 * nearest target point, interpolated normal, distance and triangle per query,
 * through the device hierarchy. */
int nricp_closest_points(const double* target_points, int vertex_count,
                         const int32_t* faces, int face_count, const double* queries,
                         int query_count, double* out_points, double* out_normals,
                         double* out_distances, int32_t* out_triangles);

/* The hierarchy's canonical arrays (src/cuda/lbvh.cu:553-668): sorted 30-bit
 * Morton codes, the sort permutation, and each internal node's Karras
 * children (child < face_count: leaf; else face_count + internal index). */
int nricp_lbvh_export(const double* target_points, int vertex_count,
                      const int32_t* faces, int face_count, uint32_t* codes,
                      uint32_t* order, int32_t* left, int32_t* right, float* bounds);

/* nricp_lbvh_export with DEVICE buffers and no device allocation; it has no
 * counterpart in the reference.  For callers that cannot allocate GPU memory
 * (inside another framework's pool or allocator hooks, with a fixed arena, or
 * with allocations audited after start-up): every intermediate lives in one
 * static 8 MiB device array, so at most 262,144 faces (more returns
 * NRICP_ERR_CAPACITY).  `target_points` (V x 3), `faces` (F x 3), `codes`,
 * `order` (F), `left`, `right` (F - 1) and `bounds` (6) are device pointers;
 * the work runs on `stream` (a cudaStream_t, NULL for the default stream).
 * Every call synchronises `stream` (it reads back the face-index check before
 * the build) and returns once the build has finished.  The array is reserved
 * when the library's device code loads on a device, which under lazy module
 * loading is the first call there: a caller that audits allocations after
 * start-up makes one call per device during start-up, before any stream
 * capture.  Every call looks up the array's address with the caller's device
 * current.  All calls share the array: calls whose work overlaps on the GPU
 * race. */
int nricp_lbvh_export_static(const double* target_points, int vertex_count,
                             const int32_t* faces, int face_count, uint32_t* codes,
                             uint32_t* order, int32_t* left, int32_t* right,
                             float* bounds, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NRICP_B200_H */
