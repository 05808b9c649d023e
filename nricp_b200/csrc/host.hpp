// Host-side preparation of a wrap: validation, normalisation, the template
// graph, the per-level layouts the kernels walk, and the run report.  All
// FP64; the graph and the report follow the reference bit for bit.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nricp_b200.h"

namespace nricp_b200 {

struct InvalidArgument : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};

struct Binding {
    int nodes[NRICP_MAX_SLOTS];
    double weights[NRICP_MAX_SLOTS];
    int count;
};

// One level of the template graph (src/core/graph.h:19-27).
struct GraphLevel {
    std::vector<double> rest;          // N x 3
    std::vector<int> template_index;   // N
    std::vector<Binding> bindings;     // V (reference semantics, zero weights kept)
    std::vector<int32_t> edges;        // E x 2, sorted unique (a < b)
    int node_count() const { return static_cast<int>(template_index.size()); }
};

struct TemplateGraph {
    double center[3];
    double scale;
    std::vector<GraphLevel> levels;
};

// Per-level layout in the form the device kernels read (kernels' LevelDev).
struct LevelLayout {
    int node_count = 0, edge_count = 0, pair_count = 0;
    std::vector<double> rest;
    std::vector<int32_t> bind_nodes;     // V x 8, usable slots only, -1 padded
    std::vector<double> bind_weights;    // V x 8
    std::vector<int32_t> bind_counts;    // V
    std::vector<int32_t> gather_begin, gather_entry;
    std::vector<int32_t> node_edge_begin, node_edge_list, edges;
    std::vector<int32_t> pair_nodes, pair_begin, pair_entry;
    std::vector<int32_t> row_begin, row_entry, offdiag_nodes, offdiag_slots;
    // the off-diagonal block that holds smoothness edge e: a node pair's own
    // block when the pair shares a vertex (< pair_count), else one of its own
    std::vector<int32_t> edge_block;
    std::vector<int32_t> transfer_nodes, transfer_counts;
    std::vector<double> transfer_weights;
};

// Validation with the reference's messages (mesh.cpp:90-116,
// constraints.cpp:8-58); throws InvalidArgument.
void validate_mesh(const double* points, int count, const int32_t* faces, int face_count,
                   const char* what);
void validate_settings(const NricpSolveDesc& desc);

void compute_normalization(const double* points, int count, double center[3], double* scale);
// The same two, written into caller memory (count x 3 doubles).
void normalized_into(const double* points, int count, const double center[3], double scale, double* out);
void vertex_normals_into(const double* points, int count, const int32_t* faces, int face_count, double* out);
std::vector<double> normalized(const double* points, int count, const double center[3],
                               double scale);
std::vector<double> vertex_normals(const std::vector<double>& points, const int32_t* faces,
                                   int face_count);

// Graph construction (src/core/sampling.cpp, src/core/graph.cpp).
std::vector<int> farthest_point_seeds(const std::vector<double>& points, int count,
                                      int first_index);
std::vector<Binding> bind_vertices(const std::vector<double>& vertices,
                                   const std::vector<double>& nodes, int max_nodes,
                                   int slot_cap);
std::vector<int32_t> node_edges(const std::vector<double>& nodes, int neighbours);
int level_node_count(int level, int nodes_initial, int growth, int vertex_count);
TemplateGraph build_template_graph(const double* points, int count, int levels,
                                   int nodes_initial, int growth, int max_nodes,
                                   int edge_neighbours);

LevelLayout build_layout(const TemplateGraph& graph, int level, int vertex_count);

// Template vertex -> incident faces (ascending face index), CSR.
void vertex_faces(const int32_t* faces, int face_count, int vertex_count,
                  std::vector<int32_t>& begin, std::vector<int32_t>& list);

struct LevelView {
    int level, nodes, outer_iterations, inner_iterations, converged;
    double energy_start, energy_end, correspondence_mean;
};
struct StatsView {
    int total, accepted, rejected_distance, rejected_normal, rejected_slope, rejected_masked;
    double mean, p95, max;
};

// RunReport JSON, src/core/report.cpp:46-105.
std::string report_json(const char* route, const char* precision, const double energy[5],
                        const StatsView& stats, const std::vector<LevelView>& levels,
                        const NricpSolveDesc& desc, double units, double setup_seconds,
                        double solve_seconds);

}  // namespace nricp_b200
