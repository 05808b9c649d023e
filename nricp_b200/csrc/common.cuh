// Device-side vocabulary of the B200 wrapping path: small vector algebra, the
// per-wrap device descriptor every kernel indexes by blockIdx.y, and the
// constants of the schedule.
//
// Precision split (the one the design asks for): the node state (R, t), the
// deformed template, the correspondences, the energies and the accept/reject
// test are FP64; the Gauss-Newton blocks, the right-hand side and the PCG
// matvec are FP32, with FP64 dot products and residual norms; the closest-point
// traversal runs on FP32 boxes and triangles and re-evaluates its winner in
// FP64.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nricp_b200 {

constexpr int kMaxSlots = 8;        // binding support (the reference caps at 4)
constexpr int kMaxLevels = 16;
constexpr int kEnergyKinds = 5;     // p2p, plane, smoothness, anchor, landmark
constexpr int kStackDepth = 64;     // LBVH traversal stack
constexpr int kLongCap = 2048;      // long walks a wrap lists for its next query's warps
constexpr int kPartialStride = 8;   // doubles per energy partial record

// Device phases of one wrap.  They mirror the reference session's
// BeginLevel / Refresh / InnerStep / CloseOuter / EndLevel
// (src/cuda/session.cu:504-542); CloseOuter folds into the decision kernel.
enum Phase : int {
    kPhaseTransfer = 0,  // warm-start the level from the previous one
    kPhaseRefresh = 1,   // correspondences + system at the accepted state
    kPhaseSolve = 2,     // one damped solve attempt + candidate system
    kPhaseFinal = 3,     // final correspondences for the report
    kPhaseDone = 4,
};

// Per-level, template-only layout (computed once on the host, uploaded once).
struct LevelDev {
    int node_count;
    int edge_count;        // smoothness edges (a < b)
    int pair_count;        // node-pair groups sharing a vertex (a < b)
    int offdiag_count;     // blocks: pair_count, then the edges whose pair shares no vertex
    const double* rest;            // node rest positions, N x 3
    const int32_t* bind_nodes;     // V x kMaxSlots, -1 padded, usable slots only
    const double* bind_weights;    // V x kMaxSlots
    const int32_t* bind_counts;    // V
    // node -> (vertex, slot) gather, CSR
    const int32_t* gather_begin;   // N + 1
    const int32_t* gather_entry;   // vertex * kMaxSlots + slot
    // node -> incident smoothness edges, CSR (edge index; sign by endpoint)
    const int32_t* node_edge_begin;
    const int32_t* node_edge_list;
    const int32_t* edges;          // edge_count x 2
    // pair groups: (a, b) and their (vertex, slot_a, slot_b) entries
    const int32_t* pair_nodes;     // pair_count x 2
    const int32_t* pair_begin;     // pair_count + 1
    const int32_t* pair_entry;     // vertex * 64 + slot_a * 8 + slot_b
    // off-diagonal row lists for the matvec: for each node, the blocks that
    // touch it; entry = block * 2 + (1 if the node is the block's b side)
    const int32_t* row_begin;      // N + 1
    const int32_t* row_entry;      // pairs: (block * 2 + side, other node)
    const int32_t* offdiag_nodes;  // offdiag_count x 2 (pair groups first, then edge-only pairs)
    const int32_t* edge_block;     // edge_count: the block edge e adds to (< pair_count) or owns
    const int32_t* offdiag_slots;  // offdiag_count x 2: row-entry slots of B (a) and B^T (b)
    int row_entries;               // 2 x offdiag_count
    // warm start from the previous level (level > 0): 4 source nodes + weights
    const int32_t* transfer_nodes;   // N x 4
    const double* transfer_weights;  // N x 4
    const int32_t* transfer_counts;  // N
};

// Per-level report record, LevelView (src/core/report.h:37-46).
struct LevelRecord {
    int level, nodes, outer_iterations, inner_iterations, converged, pad;
    double energy_start, energy_end, correspondence_mean;
    // work done in the level (measurement, not part of the report)
    int solves, pcg_iterations, queries, assemblies;
};

// Correspondence statistics, CorrespondenceCounts (correspondence.h:52-67).
struct CorrStats {
    int total, accepted, rejected_distance, rejected_normal, rejected_slope, rejected_masked;
    double mean, p95, max;
};

// The schedule's scalars for one wrap.  Written by the decision kernel only.
struct WrapControl {
    int phase;
    int route;            // 0 = B (Gauss-Newton), 1 = C (global/local)
    int level;
    int level_count;
    int outer;            // completed outer iterations in this level
    int inner;            // accepted inner steps in this outer iteration
    int attempt;          // damping attempt within this inner step
    int state;            // which of the two state buffers is accepted
    int system;           // which of the two system buffers is current
    int stats_pending;    // level-end statistics to take before the next query
    int final_stats;      // the next statistics pass is the final report's
    int pcg_ok;           // outcome of this tick's solve
    int pcg_iterations;
    int error;            // sticky device error (traversal overflow, ...)
    int steps;            // ticks that did work for this wrap
    int tick_phase;       // the phase at the start of the current tick
    int long_cur;         // the list of long walks the next query reads (0 / 1)
    double damping;
    double energy;              // accepted energy with the current correspondences
    double energy_parts[kEnergyKinds];
    double candidate_energy;
    double candidate_parts[kEnergyKinds];
    double previous_level_energy;
    double pcg_residual;
    double last_corr_mean;
};

// Everything one wrap's kernels need.  One of these per wrap in device memory;
// kernels index the array by blockIdx.y.
struct WrapDev {
    // sizes
    int V, T, Vt, F, L;
    int max_nodes, max_offdiag, max_pairs, max_edges;
    int energy_blocks;    // partial records written by the vertex pass
    // settings (per level where they vary)
    double weights[kMaxLevels][kEnergyKinds];
    int robust_kernel[kMaxLevels];
    double robust_threshold[kMaxLevels];    // normalised units
    int max_outer[kMaxLevels];
    int max_inner[kMaxLevels];
    double outer_tol[kMaxLevels];
    double inner_tol[kMaxLevels];
    double distance_threshold;              // normalised units
    double min_normal_cosine;
    double min_slope;
    double initial_damping, damping_decrease, damping_increase;
    int max_attempts;
    int diagonal_damping;
    int pcg_max_iterations;
    double pcg_tolerance;
    // template (normalised frame)
    const double* tpl;            // V x 3
    const int32_t* tpl_faces;     // T x 3
    const int32_t* vf_begin;      // V + 1: vertex -> incident faces, ascending
    const int32_t* vf_faces;
    const uint8_t* mask;          // V or null
    const double* lm_target;      // V x 3 (per-vertex landmark target)
    const uint8_t* lm_flag;       // V
    const int32_t* lm_vertices;   // L, in landmark order
    // target (normalised frame) and its hierarchy
    const double* tgt_points;     // Vt x 3
    const double* tgt_normals;    // Vt x 3 area-weighted, normalised
    const int32_t* tgt_faces;     // F x 3
    const float4* bvh_nodes;      // (F - 1) x 4 : child boxes + children
    const float4* bvh_leaves;     // F x kLeafFloat4s: FP64 corners + triangle id, sorted
    int bvh_root;                 // encoded child (leaf flag in bit 31)
    float rank_window;            // FP32 box-pruning slack (distance, normalised units)
    // levels
    LevelDev levels[kMaxLevels];
    // state: two buffers, `control.state` selects the accepted one
    double* rot[2];               // N x 9
    double* trans[2];             // N x 3
    float* rot32;                 // N x 9: FP32 copy of the state being evaluated
    double* deformed;             // V x 3
    float4* deformed32;           // V
    double* qnormals;             // V x 3 deformed-template normals
    // correspondences
    double* corr_point;           // V x 3
    double* corr_normal;          // V x 3
    double* corr_distance;        // V
    int32_t* corr_triangle;       // V (previous winner seeds the next search)
    // Vertices whose last walk was long, for the next query to give a warp
    // each: two lists (the one the query reads, long_cur, and the one it
    // fills), their counts and a flag per vertex and list.
    int32_t* long_list;           // 2 x kLongCap
    int32_t* long_count;          // 2
    uint8_t* long_flag;           // 2 x V
    uint8_t* corr_code;           // V rejection code
    double* robust;               // V
    float4* residual32;           // V: (o.x, o.y, o.z, plane value scale) per vertex
    float4* resid_aux32;          // V: (n.x, n.y, n.z, p2p scale)
    float4* lm_resid32;           // V: landmark offset (xyz), w
    float4* offsets32;            // V x kMaxSlots: each binding's node-local offset R (p - g), FP32,
                                  // for the tick's assembly (xyz, unused)
    // systems: two buffers, `control.system` selects the current one
    float* diag[2];               // N x 36
    float* rhs[2];                // N x 6
    float* offdiag[2];            // 2 x max_offdiag x 36, in row-entry order:
                                  // slot j holds the block of row list entry j
                                  // (B for the a side, B^T for the b side)
    // solve scratch
    float* factor;                // N x 36: inverse of the damped diagonal block
    double* delta;                // N x 6
    double* pcg_x;                // N x 6
    double* pcg_r;                // N x 6
    float* pcg_p;                 // N x 6: direction p
    float* pcg_ap;                // N x 6: w = A u
    float* pcg_s;                 // N x 6: s = A p (by recurrence)
    float* pcg_u;                 // N x 6: u = M^-1 r, every node
    // reductions
    double* partials;             // energy_blocks x kPartialStride
    double* edge_partials;        // edges: each edge's smoothness energy (the decision kernel sums them)
    double* node_partials;        // N: each node's anchor energy (the decision kernel sums them)
    int* counts;                  // stats scratch
    // report
    LevelRecord* records;         // level_count
    CorrStats* level_stats;       // level_count
    CorrStats* final_stats;       // 1
    WrapControl* control;
};

// ---------------------------------------------------------------------------
// small vector algebra
// ---------------------------------------------------------------------------

struct D3 { double x, y, z; };
struct F3 { float x, y, z; };

__host__ __device__ inline D3 d3(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline D3 load_d3(const double* p, long i) { return {p[i * 3], p[i * 3 + 1], p[i * 3 + 2]}; }
__device__ inline void store_d3(double* p, long i, D3 v) {
    p[i * 3] = v.x; p[i * 3 + 1] = v.y; p[i * 3 + 2] = v.z;
}
__device__ inline D3 mul3(const double* m, D3 v) {
    return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
            m[6] * v.x + m[7] * v.y + m[8] * v.z};
}

__host__ __device__ inline F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline F3 cross(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline F3 mul3f(const float* m, F3 v) {
    return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
            m[6] * v.x + m[7] * v.y + m[8] * v.z};
}

// Leaf / internal child encoding of the traversal hierarchy.
constexpr uint32_t kLeafBit = 0x80000000u;
// A hierarchy leaf: the triangle's three FP64 corners and its index, 80 bytes.
constexpr int kLeafFloat4s = 5;

}  // namespace nricp_b200
