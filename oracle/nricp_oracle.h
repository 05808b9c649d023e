/*
 * CPU oracle for the nricp wrapping path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's FP64 route A (src/solver/route_a.cpp
 * and everything under src/core, src/geometry, src/energy, src/solver), of the
 * device route C's global/local schedule (src/cuda/local_global.cu,
 * src/cuda/session.cu) in FP64, and of the FP32 Morton/Karras LBVH build
 * (src/cuda/lbvh.cu).  Each function cites the reference lines it follows.
 *
 * Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library, and only as the checker: the product path never calls it.
 */
#ifndef NRICP_ORACLE_H
#define NRICP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/nricp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Routes the oracle can run. */
enum { ORACLE_ROUTE_A = 0, ORACLE_ROUTE_C = 1 };

/* Node count per level for a descriptor (graph.cpp:52-57). Returns levels. */
int oracle_plan(const NricpSolveDesc* desc, int32_t* level_nodes, int capacity);

/* Whole wrap, FP64.  Returns 0 or an NRICP_ERR_* code; message via
 * oracle_last_error(). */
int oracle_solve(const NricpSolveDesc* desc, int route, NricpResult* out);
const char* oracle_last_error(void);

/* Template graph pieces (src/core/mesh.cpp:174-193, sampling.cpp, graph.cpp). */
void oracle_normalization(const double* points, int count, double center[3],
                          double* scale);
int oracle_farthest_point_seeds(const double* points, int count, int seeds,
                                int first_index, int32_t* out);
void oracle_bind_vertices(const double* vertices, int vertex_count,
                          const double* nodes, int node_count, int max_nodes,
                          int32_t* out_nodes, double* out_weights,
                          int32_t* out_counts); /* out arrays stride 8 */
int oracle_node_edges(const double* nodes, int node_count, int neighbours,
                      int32_t* out_edges, int capacity);
void oracle_vertex_normals(const double* points, int point_count,
                           const int32_t* faces, int face_count, double* out);

/* Closest points, FP64.  `brute` selects an exhaustive scan instead of the
 * median-split hierarchy (closest_point.cpp:143-258). */
void oracle_closest_points(const double* points, int point_count,
                           const int32_t* faces, int face_count,
                           const double* queries, int query_count, int brute,
                           double* out_points, double* out_normals,
                           double* out_distances, int32_t* out_triangles);

/* FP32 LBVH build restated from src/cuda/lbvh.cu:33-352: sorted Morton codes,
 * the sort permutation, and the Karras children of every internal node
 * (child < count: leaf index; otherwise count + internal index). */
void oracle_lbvh_build(const float* points, int point_count,
                       const int32_t* faces, int face_count,
                       uint32_t* out_codes, uint32_t* out_order,
                       int32_t* out_left, int32_t* out_right, float out_bounds[6]);

/* The reduced system at a given state (fused_assembly.cpp:159-291), FP64.
 * Off-diagonal blocks come back sorted by (a, b), a < b; capacity in blocks. */
typedef struct OracleSystemInputs {
    const double* template_points; int vertex_count;
    const int32_t* binding_nodes;   /* stride 8 */
    const double* binding_weights;  /* stride 8 */
    const int32_t* binding_counts;
    const double* node_positions; int node_count;
    const double* rotations;        /* node_count * 9 */
    const double* translations;     /* node_count * 3 */
    const double* corr_points; const double* corr_normals;
    const double* corr_robust; const uint8_t* corr_accepted;
    const int32_t* edges; int edge_count;
    const int32_t* landmark_indices; const double* landmark_targets;
    int landmark_count;
    const uint8_t* mask;
    double weights[5]; /* p2p, plane, smoothness, anchor, landmark */
} OracleSystemInputs;

int oracle_fused_system(const OracleSystemInputs* in, double* diagonal,
                        double* rhs, int32_t* off_a, int32_t* off_b,
                        double* off_blocks, int capacity, int* off_count,
                        double energies[5]);

/* Damped block-sparse solve (normal_equations.cpp:81-96 + a block Cholesky in
 * place of Eigen's SimplicialLDLT, direct_solve.cpp:10-64). */
int oracle_solve_direct(int node_count, const double* diagonal, int off_count,
                        const int32_t* off_a, const int32_t* off_b,
                        const double* off_blocks, const double* rhs,
                        double damping, int diagonal_scaling, double* delta);

/* Correspondence statistics (correspondence.cpp:59-94) over per-vertex
 * outcome codes (0 accepted, 1 distance, 2 normal, 3 slope, 4 masked) and
 * distances: counts[6] = total, accepted, rejected by distance, normal,
 * slope, masked; stats[3] = mean, p95, max of the accepted distances. */
void oracle_summarize(int count, const uint8_t* codes, const double* distances,
                      int32_t counts[6], double stats[3]);

/* Horn's closed-form rotation from a 3x3 correlation (local_global.cu:53-157),
 * FP64 Jacobi on the 4x4. */
void oracle_horn_rotation(const double correlation[9], double rotation[9]);

#ifdef __cplusplus
}
#endif

#endif
