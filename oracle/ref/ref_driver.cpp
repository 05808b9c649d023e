// C-ABI driver over the reference's own route A -- TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the reference's sources (oracle/build.py) into
// oracle/_ref/libnricp_ref.so.  It reproduces what the reference's pybind11
// layer does around solve_route_a -- prepare_solve (src/python/bindings.cpp:
// 584-672) and route_result_to_dict (674-710) -- with plain pointers instead
// of numpy arrays, and exposes the graph / closest-point / assembly pieces the
// parity tests pin.  Signatures match oracle/nricp_oracle.h.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "core/constraints.h"
#include "core/deformation.h"
#include "core/graph.h"
#include "core/mesh.h"
#include "core/report.h"
#include "core/sampling.h"
#include "energy/energy.h"
#include "energy/robust.h"
#include "geometry/closest_point.h"
#include "solver/correspondence.h"
#include "solver/fused_assembly.h"
#include "solver/route_a.h"
#ifdef NRICP_REF_GPU
#include "cuda/gpu_solver.cuh"
#endif

#include "nricp_oracle.h"

namespace {

thread_local std::string g_error;

std::vector<nricp::Vec3> points_of(const double* p, int n) {
    std::vector<nricp::Vec3> out(static_cast<std::size_t>(n));
    for (int i = 0; i < n; ++i) out[i] = {p[i * 3], p[i * 3 + 1], p[i * 3 + 2]};
    return out;
}

std::vector<nricp::Int3> faces_of(const int32_t* f, int n) {
    std::vector<nricp::Int3> out(static_cast<std::size_t>(n));
    for (int i = 0; i < n; ++i) out[i] = {f[i * 3], f[i * 3 + 1], f[i * 3 + 2]};
    return out;
}

void raise_if_invalid(const nricp::ValidationIssues& issues, const char* what) {
    if (issues.ok) return;
    std::string message(what);
    message += ": ";
    for (std::size_t i = 0; i < issues.problems.size(); ++i) {
        if (i > 0) message += "; ";
        message += issues.problems[i];
    }
    throw std::invalid_argument(message);
}

}  // namespace

namespace {

// prepare_solve (src/python/bindings.cpp:584-672) around one of the
// reference's route functions, and route_result_to_dict's outputs.
template <typename Route>
int solve_with(const NricpSolveDesc* desc, NricpResult* out, Route route) {
    try {
        nricp::Mesh template_mesh{points_of(desc->template_points, desc->template_vertex_count),
                                  faces_of(desc->template_faces, desc->template_face_count)};
        raise_if_invalid(nricp::validate(template_mesh), "invalid template mesh");
        nricp::Mesh target_mesh{points_of(desc->target_points, desc->target_vertex_count),
                                faces_of(desc->target_faces, desc->target_face_count)};
        raise_if_invalid(nricp::validate(target_mesh), "invalid target mesh");
        nricp::GraphSettings graph_settings;
        graph_settings.levels = desc->graph_levels;
        graph_settings.nodes_initial = desc->nodes_initial;
        graph_settings.node_growth = desc->growth;
        const nricp::TemplateGraph graph =
            nricp::build_template_graph(template_mesh, graph_settings);
        nricp::Mesh normalized_template = template_mesh;
        nricp::apply_normalization(normalized_template, graph.normalization);
        nricp::Mesh normalized_target = target_mesh;
        nricp::apply_normalization(normalized_target, graph.normalization);
        nricp::RouteSettings settings;
        for (int i = 0; i < desc->level_setting_count; ++i) {
            const NricpLevelSettings& in = desc->levels[i];
            nricp::LevelSettings level;
            level.weights.point_to_point = in.point_to_point;
            level.weights.point_to_plane = in.point_to_plane;
            level.weights.smoothness = in.smoothness;
            level.weights.anchor = in.anchor;
            level.weights.landmark = in.landmark;
            level.robust_kernel = static_cast<nricp::RobustKernel>(in.robust_kernel);
            level.robust_threshold = in.robust_threshold;
            level.max_outer_iterations = in.max_outer_iterations;
            level.max_inner_iterations = in.max_inner_iterations;
            level.outer_tolerance = in.outer_tolerance;
            level.inner_tolerance = in.inner_tolerance;
            settings.levels.push_back(level);
        }
        const double units = graph.normalization.scale;
        settings.correspondence.distance_threshold = desc->distance_threshold * units;
        settings.correspondence.min_normal_cosine = desc->min_normal_cosine;
        settings.correspondence.min_slope = desc->min_slope;
        for (nricp::LevelSettings& level : settings.levels) {
            if (level.robust_threshold > 0.0) level.robust_threshold *= units;
        }
        settings.initial_damping = desc->initial_damping;
        settings.damping_decrease = desc->damping_decrease;
        settings.damping_increase = desc->damping_increase;
        settings.max_damping_attempts = desc->max_damping_attempts;
        settings.diagonal_damping = desc->diagonal_damping != 0;
        nricp::VertexMask mask;
        if (desc->mask) {
            mask.active.assign(desc->mask, desc->mask + desc->template_vertex_count);
            for (auto& value : mask.active) value = value ? 1 : 0;
            raise_if_invalid(nricp::validate_mask(mask, desc->template_vertex_count),
                             "invalid mask");
        }
        std::vector<nricp::Landmark> landmarks(static_cast<std::size_t>(desc->landmark_count));
        for (int i = 0; i < desc->landmark_count; ++i) {
            const nricp::Vec3 target{desc->landmark_targets[i * 3],
                                     desc->landmark_targets[i * 3 + 1],
                                     desc->landmark_targets[i * 3 + 2]};
            landmarks[i] = {desc->landmark_indices[i],
                            (target - graph.normalization.center) * graph.normalization.scale};
        }
        raise_if_invalid(nricp::validate_landmarks(
                             landmarks, static_cast<int>(normalized_template.vertices.size())),
                         "invalid landmarks");
        settings.pcg_tolerance = static_cast<float>(desc->pcg_tolerance);
        settings.pcg_max_iterations = desc->pcg_max_iterations;
        const nricp::RouteResult solved =
            route(normalized_template, normalized_target, graph, settings,
                  mask.active.empty() ? nullptr : &mask, landmarks);

        nricp::Mesh restored;
        restored.vertices = solved.vertices;
        nricp::undo_normalization(restored, graph.normalization);
        for (std::size_t i = 0; i < restored.vertices.size() && out->vertices; ++i) {
            out->vertices[i * 3] = restored.vertices[i].x;
            out->vertices[i * 3 + 1] = restored.vertices[i].y;
            out->vertices[i * 3 + 2] = restored.vertices[i].z;
        }
        for (std::size_t n = 0; n < solved.deformation.nodes.size(); ++n) {
            if (out->rotations)
                std::memcpy(out->rotations + n * 9, solved.deformation.nodes[n].rotation.m,
                            sizeof(double) * 9);
            if (out->translations) {
                out->translations[n * 3] = solved.deformation.nodes[n].translation.x;
                out->translations[n * 3 + 1] = solved.deformation.nodes[n].translation.y;
                out->translations[n * 3 + 2] = solved.deformation.nodes[n].translation.z;
            }
            if (out->node_positions) {
                out->node_positions[n * 3] = solved.deformation.node_rest_positions[n].x;
                out->node_positions[n * 3 + 1] = solved.deformation.node_rest_positions[n].y;
                out->node_positions[n * 3 + 2] = solved.deformation.node_rest_positions[n].z;
            }
        }
        if (out->level_nodes)
            for (std::size_t l = 0; l < graph.levels.size(); ++l)
                out->level_nodes[l] = graph.levels[l].node_count();
        const std::string json = nricp::to_json(solved.report);
        out->report_length = json.size();
        if (out->report_json && out->report_capacity > 0) {
            const std::size_t n = std::min(json.size(), out->report_capacity - 1);
            std::memcpy(out->report_json, json.data(), n);
            out->report_json[n] = 0;
        }
        return 0;
    } catch (const std::invalid_argument& error) {
        g_error = error.what();
        return NRICP_ERR_INVALID;
    } catch (const std::exception& error) {
        g_error = error.what();
        return NRICP_ERR_CUDA;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_solve_route_a(const NricpSolveDesc* desc, NricpResult* out) {
    return solve_with(desc, out, [](const nricp::Mesh& tpl, const nricp::Mesh& tgt, const nricp::TemplateGraph& graph,
                                    const nricp::RouteSettings& settings, const nricp::VertexMask* mask,
                                    const std::vector<nricp::Landmark>& landmarks) {
        const nricp::TargetQueries queries(tgt);
        return nricp::solve_route_a(tpl, queries, graph, settings, mask, landmarks);
    });
}

#ifdef NRICP_REF_GPU
// The reference's own GPU route B (src/cuda/gpu_solver.cu), in the GPU build
// of this driver only.
int ref_solve_route_b(const NricpSolveDesc* desc, NricpResult* out) {
    return solve_with(desc, out, [](const nricp::Mesh& tpl, const nricp::Mesh& tgt, const nricp::TemplateGraph& graph,
                                    const nricp::RouteSettings& settings, const nricp::VertexMask* mask,
                                    const std::vector<nricp::Landmark>& landmarks) {
        return nricp::solve_route_b(tpl, tgt, graph, settings, mask, landmarks);
    });
}

// The reference's own GPU route C (src/cuda/gpu_solver.cu, local_global.cu):
// the anchor for the FP64 route-C restatement, which has no CPU counterpart.
int ref_solve_route_c(const NricpSolveDesc* desc, NricpResult* out) {
    return solve_with(desc, out, [](const nricp::Mesh& tpl, const nricp::Mesh& tgt, const nricp::TemplateGraph& graph,
                                    const nricp::RouteSettings& settings, const nricp::VertexMask* mask,
                                    const std::vector<nricp::Landmark>& landmarks) {
        return nricp::solve_route_c(tpl, tgt, graph, settings, mask, landmarks);
    });
}
#endif

int ref_farthest_point_seeds(const double* points, int count, int seeds, int first,
                             int32_t* out) {
    const std::vector<int> result =
        nricp::farthest_point_seeds(points_of(points, count), seeds, first);
    for (std::size_t i = 0; i < result.size(); ++i) out[i] = result[i];
    return static_cast<int>(result.size());
}

void ref_bind_vertices(const double* vertices, int vertex_count, const double* nodes,
                       int node_count, int max_nodes, int32_t* out_nodes, double* out_weights,
                       int32_t* out_counts) {
    const auto bindings = nricp::bind_vertices(points_of(vertices, vertex_count),
                                               points_of(nodes, node_count), max_nodes);
    for (int v = 0; v < vertex_count; ++v) {
        for (int s = 0; s < NRICP_MAX_SLOTS; ++s) {
            out_nodes[v * NRICP_MAX_SLOTS + s] =
                s < nricp::VertexBinding::kMaxNodes ? bindings[v].nodes[s] : -1;
            out_weights[v * NRICP_MAX_SLOTS + s] =
                s < nricp::VertexBinding::kMaxNodes ? bindings[v].weights[s] : 0.0;
        }
        out_counts[v] = bindings[v].count;
    }
}

int ref_node_edges(const double* nodes, int node_count, int neighbours, int32_t* out,
                   int capacity) {
    const auto edges = nricp::build_node_edges(points_of(nodes, node_count), neighbours);
    if (static_cast<int>(edges.size()) > capacity) return -1;
    for (std::size_t i = 0; i < edges.size(); ++i) {
        out[i * 2] = edges[i].a;
        out[i * 2 + 1] = edges[i].b;
    }
    return static_cast<int>(edges.size());
}

void ref_vertex_normals(const double* points, int point_count, const int32_t* faces,
                        int face_count, double* out) {
    const nricp::Mesh mesh{points_of(points, point_count), faces_of(faces, face_count)};
    const auto normals = nricp::vertex_normals(mesh);
    for (std::size_t i = 0; i < normals.size(); ++i) {
        out[i * 3] = normals[i].x;
        out[i * 3 + 1] = normals[i].y;
        out[i * 3 + 2] = normals[i].z;
    }
}

// One level of the reference's own template graph (src/core/graph.cpp:43-76):
// normalisation, FPS prefix, frozen bindings and 4-NN edges.
int ref_template_graph_level(const double* points, int count, int levels, int nodes_initial,
                             int growth, int max_nodes, int level, double center[3],
                             double* scale, int32_t* node_indices, double* node_positions,
                             int32_t* binding_nodes, double* binding_weights,
                             int32_t* binding_counts, int32_t* edges, int edge_capacity,
                             int* node_count, int* edge_count) {
    nricp::Mesh mesh;
    mesh.vertices = points_of(points, count);
    nricp::GraphSettings settings;
    settings.levels = levels;
    settings.nodes_initial = nodes_initial;
    settings.node_growth = growth;
    settings.max_nodes_per_vertex = max_nodes;
    const nricp::TemplateGraph graph = nricp::build_template_graph(mesh, settings);
    if (level < 0 || level >= static_cast<int>(graph.levels.size())) return -1;
    const nricp::GraphLevel& g = graph.levels[static_cast<std::size_t>(level)];
    center[0] = graph.normalization.center.x;
    center[1] = graph.normalization.center.y;
    center[2] = graph.normalization.center.z;
    *scale = graph.normalization.scale;
    *node_count = g.node_count();
    for (int i = 0; i < g.node_count(); ++i) {
        node_indices[i] = g.node_template_indices[i];
        node_positions[i * 3] = g.node_rest_positions[i].x;
        node_positions[i * 3 + 1] = g.node_rest_positions[i].y;
        node_positions[i * 3 + 2] = g.node_rest_positions[i].z;
    }
    for (int v = 0; v < count; ++v) {
        for (int s = 0; s < NRICP_MAX_SLOTS; ++s) {
            const bool real = s < nricp::VertexBinding::kMaxNodes;
            binding_nodes[v * NRICP_MAX_SLOTS + s] = real ? g.bindings[v].nodes[s] : -1;
            binding_weights[v * NRICP_MAX_SLOTS + s] = real ? g.bindings[v].weights[s] : 0.0;
        }
        binding_counts[v] = g.bindings[v].count;
    }
    if (static_cast<int>(g.edges.size()) > edge_capacity) return -2;
    *edge_count = static_cast<int>(g.edges.size());
    for (std::size_t i = 0; i < g.edges.size(); ++i) {
        edges[i * 2] = g.edges[i].a;
        edges[i * 2 + 1] = g.edges[i].b;
    }
    return 0;
}

void ref_normalization(const double* points, int count, double center[3], double* scale) {
    nricp::Mesh mesh;
    mesh.vertices = points_of(points, count);
    const auto n = nricp::compute_normalization(mesh);
    center[0] = n.center.x;
    center[1] = n.center.y;
    center[2] = n.center.z;
    *scale = n.scale;
}

void ref_closest_points(const double* points, int point_count, const int32_t* faces,
                        int face_count, const double* queries, int query_count, int /*brute*/,
                        double* out_points, double* out_normals, double* out_distances,
                        int32_t* out_triangles) {
    const nricp::Mesh mesh{points_of(points, point_count), faces_of(faces, face_count)};
    const nricp::TargetQueries target(mesh);
    for (int q = 0; q < query_count; ++q) {
        const auto r = target.query({queries[q * 3], queries[q * 3 + 1], queries[q * 3 + 2]});
        out_points[q * 3] = r.point.x;
        out_points[q * 3 + 1] = r.point.y;
        out_points[q * 3 + 2] = r.point.z;
        out_normals[q * 3] = r.normal.x;
        out_normals[q * 3 + 1] = r.normal.y;
        out_normals[q * 3 + 2] = r.normal.z;
        out_distances[q] = r.distance;
        out_triangles[q] = r.triangle;
    }
}

int ref_fused_system(const OracleSystemInputs* in, double* diagonal, double* rhs,
                     int32_t* off_a, int32_t* off_b, double* off_blocks, int capacity,
                     int* off_count, double energies[5]) {
    nricp::EnergyInputs inputs;
    inputs.template_points = points_of(in->template_points, in->vertex_count);
    inputs.bindings.resize(static_cast<std::size_t>(in->vertex_count));
    for (int v = 0; v < in->vertex_count; ++v) {
        nricp::VertexBinding& b = inputs.bindings[v];
        b.count = std::min(in->binding_counts[v], nricp::VertexBinding::kMaxNodes);
        for (int s = 0; s < nricp::VertexBinding::kMaxNodes; ++s) {
            b.nodes[s] = in->binding_nodes[v * NRICP_MAX_SLOTS + s];
            b.weights[s] = in->binding_weights[v * NRICP_MAX_SLOTS + s];
        }
    }
    inputs.node_positions = points_of(in->node_positions, in->node_count);
    inputs.correspondences.resize(static_cast<std::size_t>(in->vertex_count));
    for (int v = 0; v < in->vertex_count; ++v) {
        inputs.correspondences[v] = {
            {in->corr_points[v * 3], in->corr_points[v * 3 + 1], in->corr_points[v * 3 + 2]},
            {in->corr_normals[v * 3], in->corr_normals[v * 3 + 1], in->corr_normals[v * 3 + 2]},
            in->corr_robust[v],
            in->corr_accepted[v] != 0};
    }
    for (int e = 0; e < in->edge_count; ++e)
        inputs.smoothness_edges.push_back({in->edges[e * 2], in->edges[e * 2 + 1]});
    for (int l = 0; l < in->landmark_count; ++l)
        inputs.landmarks.push_back({in->landmark_indices[l],
                                    {in->landmark_targets[l * 3], in->landmark_targets[l * 3 + 1],
                                     in->landmark_targets[l * 3 + 2]}});
    nricp::VertexMask mask;
    if (in->mask) {
        mask.active.assign(in->mask, in->mask + in->vertex_count);
        inputs.mask = &mask;
    }
    nricp::Deformation deformation = nricp::identity_deformation(inputs.node_positions);
    for (int n = 0; n < in->node_count; ++n) {
        std::memcpy(deformation.nodes[n].rotation.m, in->rotations + n * 9, sizeof(double) * 9);
        deformation.nodes[n].translation = {in->translations[n * 3], in->translations[n * 3 + 1],
                                            in->translations[n * 3 + 2]};
    }
    nricp::EnergyWeights weights;
    weights.point_to_point = in->weights[0];
    weights.point_to_plane = in->weights[1];
    weights.smoothness = in->weights[2];
    weights.anchor = in->weights[3];
    weights.landmark = in->weights[4];
    const nricp::FusedSystem fused = nricp::assemble_and_energy(inputs, deformation, weights);
    for (int n = 0; n < in->node_count; ++n) {
        std::memcpy(diagonal + n * 36, fused.system.diagonal[n].m, sizeof(double) * 36);
        for (int r = 0; r < 6; ++r) rhs[n * 6 + r] = fused.system.rhs[n * 6 + r];
    }
    energies[0] = fused.energies.point_to_point;
    energies[1] = fused.energies.point_to_plane;
    energies[2] = fused.energies.smoothness;
    energies[3] = fused.energies.anchor;
    energies[4] = fused.energies.landmark;
    *off_count = static_cast<int>(fused.system.off_diagonal.size());
    if (*off_count > capacity) return NRICP_ERR_CAPACITY;
    for (int i = 0; i < *off_count; ++i) {
        off_a[i] = fused.system.off_diagonal[i].a;
        off_b[i] = fused.system.off_diagonal[i].b;
        std::memcpy(off_blocks + i * 36, fused.system.off_diagonal[i].value.m, sizeof(double) * 36);
    }
    return 0;
}

}  // extern "C"

namespace {

nricp::Deformation deformation_of(int node_count, const double* rotations, const double* translations,
                                  const double* node_positions) {
    nricp::Deformation deformation;
    deformation.nodes.resize(static_cast<std::size_t>(node_count));
    deformation.node_rest_positions.resize(static_cast<std::size_t>(node_count));
    for (int n = 0; n < node_count; ++n) {
        std::memcpy(deformation.nodes[n].rotation.m, rotations + n * 9, sizeof(double) * 9);
        deformation.nodes[n].translation = {translations[n * 3], translations[n * 3 + 1],
                                            translations[n * 3 + 2]};
        if (node_positions != nullptr) {
            deformation.node_rest_positions[n] = {node_positions[n * 3], node_positions[n * 3 + 1],
                                                  node_positions[n * 3 + 2]};
        }
    }
    return deformation;
}

void store_deformation(const nricp::Deformation& deformation, double* rotations, double* translations) {
    for (std::size_t n = 0; n < deformation.nodes.size(); ++n) {
        std::memcpy(rotations + n * 9, deformation.nodes[n].rotation.m, sizeof(double) * 9);
        translations[n * 3] = deformation.nodes[n].translation.x;
        translations[n * 3 + 1] = deformation.nodes[n].translation.y;
        translations[n * 3 + 2] = deformation.nodes[n].translation.z;
    }
}

}  // namespace

extern "C" {

// ---- the deformation pieces of the Python module, one reference call each
// (src/python/bindings.cpp:817-856, 1026-1092).  Rotations are n x 9 row-major
// doubles, bindings n x 4 with a count per vertex.

void ref_retract(int node_count, double* rotations, double* translations, const double* delta) {
    nricp::Deformation deformation = deformation_of(node_count, rotations, translations, nullptr);
    nricp::retract(deformation, std::vector<double>(delta, delta + node_count * 6));
    store_deformation(deformation, rotations, translations);
}

void ref_tangent_difference(int node_count, const double* rotations_from, const double* translations_from,
                            const double* rotations_to, const double* translations_to, double* out) {
    const std::vector<double> delta = nricp::tangent_difference(
        deformation_of(node_count, rotations_from, translations_from, nullptr),
        deformation_of(node_count, rotations_to, translations_to, nullptr));
    std::memcpy(out, delta.data(), sizeof(double) * delta.size());
}

void ref_evaluate_deformation(const double* points, int point_count, const int32_t* binding_nodes,
                              const double* binding_weights, const int32_t* binding_counts,
                              int node_count, const double* rotations, const double* translations,
                              const double* node_positions, double* out) {
    std::vector<nricp::VertexBinding> bindings(static_cast<std::size_t>(point_count));
    for (int v = 0; v < point_count; ++v) {
        bindings[v].count = binding_counts[v];
        for (int s = 0; s < nricp::VertexBinding::kMaxNodes; ++s) {
            bindings[v].nodes[s] = binding_nodes[v * 4 + s];
            bindings[v].weights[s] = binding_weights[v * 4 + s];
        }
    }
    const auto result = nricp::evaluate(points_of(points, point_count), bindings,
                                        deformation_of(node_count, rotations, translations,
                                                       node_positions));
    for (int v = 0; v < point_count; ++v) {
        out[v * 3] = result[v].x;
        out[v * 3 + 1] = result[v].y;
        out[v * 3 + 2] = result[v].z;
    }
}

void ref_transfer_level(int from_count, const double* from_nodes, const double* rotations,
                        const double* translations, int to_count, const double* to_nodes, int max_nodes,
                        double* out_rotations, double* out_translations) {
    const nricp::Deformation transferred = nricp::transfer_level(
        points_of(from_nodes, from_count), deformation_of(from_count, rotations, translations, from_nodes),
        points_of(to_nodes, to_count), max_nodes);
    store_deformation(transferred, out_rotations, out_translations);
}

// mesh.cpp:118-173 through the Python binding's steps (bindings.cpp:762-778);
// returns the kept vertex count, faces in out_faces[0..out_counts[3]).
int ref_clean_mesh(const double* points, int point_count, const int32_t* faces, int face_count,
                   double* out_points, int32_t* out_faces, int* out_counts) {
    nricp::Mesh mesh{points_of(points, point_count), faces_of(faces, face_count)};
    const nricp::CleanReport report = nricp::clean(mesh);
    for (std::size_t i = 0; i < mesh.vertices.size(); ++i) {
        out_points[i * 3] = mesh.vertices[i].x;
        out_points[i * 3 + 1] = mesh.vertices[i].y;
        out_points[i * 3 + 2] = mesh.vertices[i].z;
    }
    for (std::size_t i = 0; i < mesh.faces.size(); ++i) {
        out_faces[i * 3] = mesh.faces[i].v0;
        out_faces[i * 3 + 1] = mesh.faces[i].v1;
        out_faces[i * 3 + 2] = mesh.faces[i].v2;
    }
    out_counts[0] = report.duplicate_faces;
    out_counts[1] = report.degenerate_faces;
    out_counts[2] = report.isolated_vertices;
    out_counts[3] = static_cast<int>(mesh.faces.size());
    return static_cast<int>(mesh.vertices.size());
}

// The reference's filtered correspondences (bindings.cpp:1187-1251) on its
// own FP64 closest points; counts: the six integers, then mean, p95, max.
void ref_find_correspondences(const double* target_points, int point_count, const int32_t* faces,
                              int face_count, const double* queries, int query_count,
                              const double* query_normals, int normal_count, double distance_threshold,
                              double min_normal_cosine, double min_slope, const uint8_t* mask,
                              int mask_count, double* out_points, double* out_normals,
                              double* out_distances, int32_t* out_triangles, int32_t* out_rejection,
                              int32_t* out_counts, double* out_stats) {
    const nricp::Mesh target{points_of(target_points, point_count), faces_of(faces, face_count)};
    nricp::VertexMask vertex_mask;
    vertex_mask.active.assign(mask, mask + mask_count);
    nricp::CorrespondenceSettings settings;
    settings.distance_threshold = distance_threshold;
    settings.min_normal_cosine = min_normal_cosine;
    settings.min_slope = min_slope;
    const nricp::TargetQueries queries_of(target);
    const nricp::CorrespondenceSet set = nricp::find_correspondences(
        queries_of, points_of(queries, query_count), points_of(query_normals, normal_count), settings,
        vertex_mask.active.empty() ? nullptr : &vertex_mask);
    for (int i = 0; i < query_count; ++i) {
        const nricp::Correspondence& c = set.items[i];
        out_points[i * 3] = c.point.x;
        out_points[i * 3 + 1] = c.point.y;
        out_points[i * 3 + 2] = c.point.z;
        out_normals[i * 3] = c.normal.x;
        out_normals[i * 3 + 1] = c.normal.y;
        out_normals[i * 3 + 2] = c.normal.z;
        out_distances[i] = c.distance;
        out_triangles[i] = c.triangle;
        out_rejection[i] = static_cast<int32_t>(c.rejection);
    }
    const auto& k = set.counts;
    const int32_t ints[6] = {k.total, k.accepted, k.rejected_distance, k.rejected_normal, k.rejected_slope,
                             k.rejected_masked};
    std::memcpy(out_counts, ints, sizeof ints);
    out_stats[0] = k.distance_mean;
    out_stats[1] = k.distance_p95;
    out_stats[2] = k.distance_max;
}

void ref_robust_weights(const char* kernel, const double* squared_residuals, int count,
                        double threshold, double* out) {
    const nricp::RobustKernel selected = nricp::robust_kernel_from_string(kernel);
    for (int i = 0; i < count; ++i) out[i] = nricp::robust_weight(selected, squared_residuals[i], threshold);
}

}  // extern "C"
