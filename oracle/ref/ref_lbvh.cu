// The reference's own LBVH build, read back -- TEST INFRASTRUCTURE ONLY.
//
// Compiled with nvcc beside the reference's src/cuda sources into
// oracle/_ref/libnricp_ref_gpu.so (oracle/build.py, build_reference_gpu).  It
// runs nricp::gpu::Lbvh::build (src/cuda/lbvh.cu:553-668) and copies out the
// arrays the hierarchy keeps: the sorted 30-bit Morton codes, the sort
// permutation and the Karras children of every internal node, so that a test
// can compare them bit for bit with this library's hierarchy.
//
// Those arrays are private members of Lbvh.  The access rules do not apply to
// the names in an explicit instantiation ([temp.explicit]), so the Expose
// template below, instantiated once per member, hands out a pointer to each
// member without any change to the reference's sources.
#include <cstdint>
#include <exception>
#include <string>
#include <vector>

#include <thrust/copy.h>
#include <thrust/device_vector.h>

#include "core/mesh.h"
#include "cuda/lbvh.cuh"

namespace {

using nricp::gpu::Lbvh;
using nricp::gpu::LbvhNode;

template <typename Tag, typename Tag::type Member>
struct Expose {
    friend typename Tag::type member_of(Tag) { return Member; }
};

struct CodesTag {
    using type = thrust::device_vector<unsigned int> Lbvh::*;
    friend type member_of(CodesTag);
};
struct OrderTag {
    using type = thrust::device_vector<unsigned int> Lbvh::*;
    friend type member_of(OrderTag);
};
struct NodesTag {
    using type = thrust::device_vector<LbvhNode> Lbvh::*;
    friend type member_of(NodesTag);
};

template struct Expose<CodesTag, &Lbvh::codes_>;
template struct Expose<OrderTag, &Lbvh::order_>;
template struct Expose<NodesTag, &Lbvh::nodes_>;

thread_local std::string g_lbvh_error;

}  // namespace

extern "C" {

const char* ref_lbvh_last_error(void) { return g_lbvh_error.c_str(); }

// Builds the reference's hierarchy over (points, faces) on the default stream
// and writes codes[F], order[F] and, for each internal node i < F - 1, its
// children in the reference's numbering minus one: a child below F is the
// leaf at that sorted position, F + j is internal node j.  Returns 0, or -1
// with ref_lbvh_last_error() set.
int ref_lbvh_build(const double* points, int vertex_count, const int32_t* faces, int face_count,
                   uint32_t* codes, uint32_t* order, int32_t* left, int32_t* right) {
    try {
        nricp::Mesh mesh;
        mesh.vertices.resize(static_cast<std::size_t>(vertex_count));
        for (int i = 0; i < vertex_count; ++i)
            mesh.vertices[i] = {points[i * 3], points[i * 3 + 1], points[i * 3 + 2]};
        mesh.faces.resize(static_cast<std::size_t>(face_count));
        for (int i = 0; i < face_count; ++i)
            mesh.faces[i] = {faces[i * 3], faces[i * 3 + 1], faces[i * 3 + 2]};
        Lbvh lbvh;
        lbvh.build(mesh, 0);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("hierarchy build failed");
        const auto& c = lbvh.*member_of(CodesTag{});
        const auto& o = lbvh.*member_of(OrderTag{});
        const auto& n = lbvh.*member_of(NodesTag{});
        thrust::copy(c.begin(), c.end(), codes);
        thrust::copy(o.begin(), o.end(), order);
        std::vector<LbvhNode> nodes(n.size());
        thrust::copy(n.begin(), n.end(), nodes.begin());
        for (int i = 0; i + 1 < face_count; ++i) {
            left[i] = nodes[static_cast<std::size_t>(face_count + i)].left - 1;
            right[i] = nodes[static_cast<std::size_t>(face_count + i)].right - 1;
        }
        return 0;
    } catch (const std::exception& e) {
        g_lbvh_error = e.what();
        return -1;
    }
}

}  // extern "C"
