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
// Limit: 262,144 triangles.  The array is 8 MiB on every GPU that loads this
// library, held until the process exits.  The first call on each device looks
// up the array's device address (cudaGetSymbolAddress, with that device
// current); make that first call before any stream capture.  All calls share
// the array: it keeps the previous call's contents (the build clears what
// must start at zero), and two calls whose work overlaps on the GPU -- from
// two host threads, or on two streams -- race on it.
#include <cstdint>
#include <cstring>
#include <mutex>
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

// The array's device address, resolved once per device with that device
// current.  (In host code the array's name is only a stand-in for it.)
constexpr int kMaxDevices = 64;
std::mutex g_resolve_mutex;
void* g_scratch_address[kMaxDevices] = {};

void* scratch_address() {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices) throw CudaError("device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_resolve_mutex);
    if (g_scratch_address[device] == nullptr) {
        void* address = nullptr;
        check(cudaGetSymbolAddress(&address, g_static_scratch), "cudaGetSymbolAddress");
        g_scratch_address[device] = address;
    }
    return g_scratch_address[device];
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
