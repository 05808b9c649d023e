// Template graphs of many wraps built on the device, bit-identical to the
// host build (host.hpp: build_template_graph).
#pragma once

#include <vector>

#include <cuda_runtime.h>

#include "host.hpp"

namespace nricp_b200 {

struct GraphRequest {
    const double* points;  // template vertices, caller units, count x 3
    int count;
    int levels, nodes_initial, growth, max_nodes, edge_neighbours;
};

// Whether the device build handles this many edge neighbours (else build on the host).
bool device_graph_supported(int edge_neighbours);

// One graph per request, in order; runs on `stream` and returns when done.
std::vector<TemplateGraph> device_template_graphs(const std::vector<GraphRequest>& requests,
                                                  cudaStream_t stream);

}  // namespace nricp_b200
