// Launch entry points of the device kernels, shared by the host orchestration.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace nricp_b200 {

struct LbvhExport {
    uint32_t* codes;
    uint32_t* order;
    int32_t* left;
    int32_t* right;
    float* bounds;
};

size_t lbvh_scratch_bytes(int triangle_count);
uint32_t lbvh_build(const double* points, const int32_t* faces, int triangle_count,
                    void* scratch, float4* nodes, float4* leaves, cudaStream_t stream,
                    LbvhExport* out);
// The target's ingestion on the device, once after its upload in the caller's
// units: its points normalised in place ((p - center) * scale) and its
// area-weighted vertex normals, both bit-identical to the host's.
size_t ingest_scratch_bytes(int vertex_count, int face_count);
void ingest_target(double* points, int vertex_count, const int32_t* faces, int face_count,
                   const double center[3], double scale, double* normals, void* scratch,
                   cudaStream_t stream);
int ingest_launches(int vertex_count, int face_count);

// The closest-point query of every querying wrap: with `counter` (two device
// ints), over a grid that fits on the device at once, the wraps' listed long
// walks a warp each, then a queue of the other vertices a thread each;
// without, a thread per vertex in a block row per wrap.
void launch_query(const WrapDev* wraps, int wrap_count, int max_vertices, cudaStream_t stream,
                  int* counter = nullptr);
void launch_closest_points(const WrapDev* wrap, const double* queries, int count, double* points,
                           double* normals, double* distances, int32_t* triangles, int* overflow,
                           cudaStream_t stream);

// Launch shape of one tick, sized for the largest wrap of the batch.
struct TickShape {
    int wraps;
    int max_vertices;
    int max_nodes;
    int max_edges;
    int max_pairs;
    int route_c;         // some wrap solves by route C (else its Horn-fit kernels are not launched)
    int energy_blocks;   // vertex-pass blocks per wrap (partials written)
    int edge_blocks;
    int node_blocks;
    int pcg_cluster;       // CTAs per wrap in the cluster solve (any value gives the same result)
    int pcg_shared_bytes;  // dynamic shared memory of the solve launch
    // The solve may instead be split into launches by cluster class, each over
    // a list of wraps (device array), run as parallel branches of the tick.
    int pcg_groups;                      // 0: one launch over every wrap
    int pcg_group_cluster[5];
    int pcg_group_count[5];
    int pcg_group_shared[5];
    const int* pcg_group_index[5];       // device: wrap indices of the group
    cudaStream_t pcg_streams[5];         // branch streams (index 0 unused)
    cudaEvent_t pcg_fork, pcg_join[5];
    int* query_counter;                  // device: the query queues' heads, 2 ints (null: no queue)
    // The refresh chain's branch (null: one chain on the tick's stream).
    cudaStream_t side_stream;
    cudaEvent_t side_fork, side_join;
};

// Device timing hooks for the dominant kernels (CUDA events on the launching
// stream); null when not profiling.
struct KernelTimers {
    cudaEvent_t query_begin, query_end;
    cudaEvent_t pcg_begin, pcg_end;
    cudaEvent_t assemble_begin, assemble_end;
    bool active;
};

void launch_tick(const WrapDev* wraps, const TickShape& shape, cudaStream_t stream,
                 KernelTimers* timers);
// Kernels one tick launches (a timed tick runs its branches one after the
// other, with one assembly).
int tick_kernel_launches(const TickShape& shape, bool timed = false);
int pcg_latency_cluster(int nodes);
int pcg_cluster_size(int max_nodes, int wraps, int sm_count);
int pcg_shared_bytes(const int* max_nodes, int wraps, int cluster);
int pcg_max_nodes();
// The weighted rigid fit of n point pairs (device arrays); out = R (row-major
// 3x3), t.
void launch_fit_rigid(const double* src, const double* dst, const double* weights, int n, double* out,
                      cudaStream_t stream);
void launch_evaluate_state(const WrapDev* wraps, const TickShape& shape, cudaStream_t stream);

}  // namespace nricp_b200
