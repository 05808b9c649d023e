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
void launch_query(const WrapDev* wraps, int wrap_count, int max_vertices, cudaStream_t stream);
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
    int energy_blocks;   // vertex-pass blocks per wrap (partials written)
    int edge_blocks;
    int node_blocks;
    int pcg_cluster;     // CTAs per wrap in the cluster solve
    int pcg_shared_bytes;  // direction staged in shared memory
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
int tick_kernel_launches(const TickShape& shape);
int pcg_cluster_size(int max_nodes);
int pcg_shared_bytes(int max_nodes);
void launch_evaluate_state(const WrapDev* wraps, const TickShape& shape, cudaStream_t stream);

}  // namespace nricp_b200
