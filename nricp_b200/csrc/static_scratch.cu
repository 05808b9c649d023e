// The hierarchy export for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code running inside another
// framework's memory pool or allocator hooks, plugins handed a fixed device
// arena, or a process whose allocations are made once at start-up and audited
// thereafter.  This entry point serves them.  Its inputs and outputs are the
// caller's own device buffers; every intermediate the build needs lives in
// one statically sized device array, defined below, so the call allocates
// nothing (no cudaMalloc, no cudaFree, no allocating library routine).
//
// Limit: 262,144 triangles.  The array is 8 MiB per device.  It is reserved
// when this library's device code is loaded on that device -- with lazy module
// loading (the CUDA 12 default) that is the first call on the device, not the
// library's load -- and held until the process exits.  A caller that audits
// allocations after start-up should therefore make one call per device during
// start-up, before any stream capture.  Every call looks up the array's device
// address (cudaGetSymbolAddress, with the caller's device current), so the
// address stays right after the device's context is recreated.  Every call
// also synchronises the caller's stream before it returns: it reads back the
// face-index check before the build starts.  All calls share the array: it
// keeps the previous call's contents (the build clears what must start at
// zero), and two calls whose work overlaps on the GPU -- from two host
// threads, or on two streams -- race on it.
#include <cstdint>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/nricp_b200.h"
#include "session.hpp"

namespace nricp_b200 {

size_t lbvh_export_scratch_bytes(int n);
bool lbvh_export_to_device(const double* points, int vertex_count, const int32_t* faces, int n,
                           void* scratch, uint32_t* codes, uint32_t* order, int32_t* left,
                           int32_t* right, float* bounds, cudaStream_t stream);

namespace {

constexpr int kStaticTriangles = 262144;
// the export's intermediates for kStaticTriangles triangles (7.04 MiB), rounded up
constexpr size_t kStaticScratchBytes = 8u * 1024u * 1024u;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// The array's device address on the current device.  In host code the
// array's name is only a stand-in for it, so it is looked up on every call:
// once the module is loaded this allocates nothing, and it never returns an
// address from a context that has since been torn down.
void* scratch_address() {
    void* address = nullptr;
    check(cudaGetSymbolAddress(&address, g_static_scratch), "cudaGetSymbolAddress");
    if (address == nullptr) throw CudaError("cudaGetSymbolAddress returned no address");
    return address;
}

}  // namespace

}  // namespace nricp_b200

using namespace nricp_b200;

extern "C" int nricp_lbvh_export_static(const double* points, int vertex_count,
                                        const int32_t* faces, int face_count, uint32_t* codes,
                                        uint32_t* order, int32_t* left, int32_t* right,
                                        float* bounds, void* stream) {
    try {
        if (face_count <= 0 || vertex_count <= 0) {
            g_last_error = "invalid target mesh: the hierarchy needs at least one face and one vertex";
            return NRICP_ERR_INVALID;
        }
        if (face_count > kStaticTriangles ||
            lbvh_export_scratch_bytes(face_count) > kStaticScratchBytes) {
            g_last_error = "face_count " + std::to_string(face_count) +
                           " exceeds the static scratch's limit of " +
                           std::to_string(kStaticTriangles) +
                           " triangles; use nricp_lbvh_export for larger meshes";
            return NRICP_ERR_CAPACITY;
        }
        void* scratch = scratch_address();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (!lbvh_export_to_device(points, vertex_count, faces, face_count, scratch, codes, order,
                                   left, right, bounds, s)) {
            g_last_error = "invalid target mesh: a face index is out of range";
            return NRICP_ERR_INVALID;
        }
        check(cudaGetLastError(), "hierarchy export");
        check(cudaStreamSynchronize(s), "hierarchy export");
        return NRICP_OK;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return NRICP_ERR_CUDA;
    }
}
