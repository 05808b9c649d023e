// The target's Morton-code LBVH: build and closest-point query.
//
// Build (once per target, all on the device): FP32 triangle centroids and
// scene bounds, 30-bit Morton codes with the reference's quantisation
// (src/cuda/lbvh.cu:146-168), a stable LSD radix sort of (code, index) written
// here (4-bit digits, per-tile ranking in shared memory), Karras' split search
// with index tie-breaking (lbvh.cu:177-245), and a bottom-up box fit with the
// fence + arrival-counter protocol (no waiting: the second child to arrive
// merges).  The hierarchy is then packed for traversal with each child's box
// stored in its parent (64 B per internal node = one L2 line pair), so a
// visit costs one 64-byte load instead of three dependent ones.
//
// Query (thread per template vertex): the previous correspondence's triangle
// seeds the search radius, the traversal prunes FP32 boxes with a fixed-depth
// stack whose overflow is reported (never silently pruned), and every
// triangle it reaches is measured with the reference's FP64 closest-point
// routine (src/geometry/closest_point.cpp:24-121), so the winner, its point,
// normal and distance are those of an FP64 brute-force scan.
#include "common.cuh"
#include "kernels.cuh"

namespace nricp_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kSortItems = 8;                       // keys per thread per tile
constexpr int kSortTile = kThreads * kSortItems;    // 2048 keys
constexpr int kRadixBits = 4;
constexpr int kRadix = 1 << kRadixBits;             // 16 bins

__device__ inline uint32_t expand_bits(uint32_t v) {  // lbvh.cu:132-139
    v &= 0x000003ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// FP32 copies of the target corners, triangle centroids ((a+b+c)/3 with each
// operation rounded on its own, as lbvh.cu:44-45 evaluates it).
__global__ void k_centroids(const double* __restrict__ points, const int32_t* __restrict__ faces,
                            int count, float* __restrict__ centroids) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int32_t* f = faces + (long)t * 3;
    for (int k = 0; k < 3; ++k) {
        const float a = __double2float_rn(points[(long)f[0] * 3 + k]);
        const float b = __double2float_rn(points[(long)f[1] * 3 + k]);
        const float c = __double2float_rn(points[(long)f[2] * 3 + k]);
        centroids[(long)t * 3 + k] = __fdiv_rn(__fadd_rn(__fadd_rn(a, b), c), 3.0f);
    }
}

// Scene bounds of the centroids: per-block partials, then one block folds
// them.  min/max are exact, so the order does not matter.
__global__ void k_bounds_partial(const float* __restrict__ centroids, int count,
                                 float* __restrict__ partial) {
    __shared__ float lo[3][kThreads], hi[3][kThreads];
    float l[3] = {3.4e38f, 3.4e38f, 3.4e38f}, h[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) {
            l[k] = fminf(l[k], centroids[(long)i * 3 + k]);
            h[k] = fmaxf(h[k], centroids[(long)i * 3 + k]);
        }
    for (int k = 0; k < 3; ++k) { lo[k][threadIdx.x] = l[k]; hi[k][threadIdx.x] = h[k]; }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 3; ++k) {
                lo[k][threadIdx.x] = fminf(lo[k][threadIdx.x], lo[k][threadIdx.x + s]);
                hi[k][threadIdx.x] = fmaxf(hi[k][threadIdx.x], hi[k][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; ++k) {
            partial[blockIdx.x * 6 + k] = lo[k][0];
            partial[blockIdx.x * 6 + 3 + k] = hi[k][0];
        }
}

__global__ void k_bounds_final(const float* __restrict__ partial, int blocks,
                               float* __restrict__ bounds) {
    if (threadIdx.x != 0) return;
    float l[3] = {3.4e38f, 3.4e38f, 3.4e38f}, h[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int b = 0; b < blocks; ++b)
        for (int k = 0; k < 3; ++k) {
            l[k] = fminf(l[k], partial[b * 6 + k]);
            h[k] = fmaxf(h[k], partial[b * 6 + 3 + k]);
        }
    for (int k = 0; k < 3; ++k) { bounds[k] = l[k]; bounds[3 + k] = h[k]; }
}

__global__ void k_morton(const float* __restrict__ centroids, int count,
                         const float* __restrict__ bounds, uint32_t* __restrict__ codes,
                         uint32_t* __restrict__ order) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
        const float extent = __fsub_rn(bounds[3 + k], bounds[k]);
        const float scale = extent > 1e-10f ? __fdiv_rn(1023.0f, extent) : 0.0f;
        const float v = __fmul_rn(__fsub_rn(centroids[(long)t * 3 + k], bounds[k]), scale);
        q[k] = (uint32_t)fminf(1023.0f, fmaxf(0.0f, v));
    }
    codes[t] = (expand_bits(q[2]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[0]);
    order[t] = (uint32_t)t;
}

// ---- stable LSD radix sort of (key, value), 4-bit digits --------------------

__global__ void k_radix_histogram(const uint32_t* __restrict__ keys, int count, int shift,
                                  uint32_t* __restrict__ counts, int tiles) {
    __shared__ uint32_t bins[kRadix];
    if (threadIdx.x < kRadix) bins[threadIdx.x] = 0;
    __syncthreads();
    const long base = (long)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        const long at = base + i;
        if (at < count) atomicAdd(&bins[(keys[at] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kRadix) counts[threadIdx.x * tiles + blockIdx.x] = bins[threadIdx.x];
}

// Exclusive scan of the digit-major count matrix in one block.
__global__ void k_radix_scan(uint32_t* __restrict__ counts, int total) {
    __shared__ uint32_t sums[1024];
    const int per = (total + blockDim.x - 1) / blockDim.x;
    const int begin = threadIdx.x * per;
    uint32_t local = 0;
    for (int i = begin; i < begin + per && i < total; ++i) local += counts[i];
    sums[threadIdx.x] = local;
    __syncthreads();
    for (int s = 1; s < blockDim.x; s <<= 1) {
        const uint32_t v = threadIdx.x >= s ? sums[threadIdx.x - s] : 0;
        __syncthreads();
        sums[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t running = threadIdx.x == 0 ? 0 : sums[threadIdx.x - 1];
    for (int i = begin; i < begin + per && i < total; ++i) {
        const uint32_t c = counts[i];
        counts[i] = running;
        running += c;
    }
}

// Each thread owns kSortItems consecutive keys of the tile, so ranking by
// (digit, thread, position) preserves the input order within a digit.
__global__ void k_radix_scatter(const uint32_t* __restrict__ keys_in,
                                const uint32_t* __restrict__ values_in, int count, int shift,
                                const uint32_t* __restrict__ offsets, int tiles,
                                uint32_t* __restrict__ keys_out,
                                uint32_t* __restrict__ values_out) {
    __shared__ uint32_t grid_counts[kRadix * kThreads];  // [digit][thread]
    __shared__ uint32_t partial[kThreads];
    const long base = (long)blockIdx.x * kSortTile + (long)threadIdx.x * kSortItems;
    uint32_t k[kSortItems], v[kSortItems];
    int digit[kSortItems];
    uint32_t mine[kRadix];
    for (int d = 0; d < kRadix; ++d) mine[d] = 0;
    for (int i = 0; i < kSortItems; ++i) {
        const long at = base + i;
        digit[i] = -1;
        if (at < count) {
            k[i] = keys_in[at];
            v[i] = values_in[at];
            digit[i] = (k[i] >> shift) & (kRadix - 1);
            mine[digit[i]]++;
        }
    }
    for (int d = 0; d < kRadix; ++d) grid_counts[d * kThreads + threadIdx.x] = mine[d];
    __syncthreads();
    // exclusive scan of the [digit][thread] matrix: each thread sums a run of
    // kRadix consecutive entries, a block scan of the runs, then write-back.
    uint32_t run = 0;
    for (int i = 0; i < kRadix; ++i) run += grid_counts[threadIdx.x * kRadix + i];
    partial[threadIdx.x] = run;
    __syncthreads();
    for (int s = 1; s < kThreads; s <<= 1) {
        const uint32_t add = threadIdx.x >= s ? partial[threadIdx.x - s] : 0;
        __syncthreads();
        partial[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t running = threadIdx.x == 0 ? 0 : partial[threadIdx.x - 1];
    for (int i = 0; i < kRadix; ++i) {
        const uint32_t c = grid_counts[threadIdx.x * kRadix + i];
        grid_counts[threadIdx.x * kRadix + i] = running;
        running += c;
    }
    __syncthreads();
    uint32_t local[kRadix];
    for (int d = 0; d < kRadix; ++d)
        local[d] = grid_counts[d * kThreads + threadIdx.x] - grid_counts[d * kThreads] +
                   offsets[d * tiles + blockIdx.x];
    for (int i = 0; i < kSortItems; ++i) {
        if (digit[i] < 0) continue;
        const uint32_t at = local[digit[i]]++;
        keys_out[at] = k[i];
        values_out[at] = v[i];
    }
}

// ---- Karras build --------------------------------------------------------

__device__ inline int lcp(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz((uint32_t)(i ^ j));
    return __clz(a ^ b);
}

// Internal node i covers a range and splits it (lbvh.cu:190-245).  Children
// are written in the reference's numbering: a leaf is its sorted position
// (< n), an internal node is n + index.
__global__ void k_karras(const uint32_t* __restrict__ codes, int n, int32_t* __restrict__ left,
                         int32_t* __restrict__ right, int32_t* __restrict__ parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int pp = lcp(codes, n, i, i - 1);
    const int pn = lcp(codes, n, i, i + 1);
    const int dir = pn > pp ? 1 : -1;
    const int pmin = pp < pn ? pp : pn;
    int span = 2;
    while (lcp(codes, n, i, i + span * dir) > pmin) span *= 2;
    int last = 0;
    for (int step = span / 2; step >= 1; step /= 2)
        if (lcp(codes, n, i, i + (last + step) * dir) > pmin) last += step;
    const int j = i + last * dir;
    const int rl = i < j ? i : j, rr = i < j ? j : i;
    const int np = lcp(codes, n, rl, rr);
    int offset = 0, step = rr - rl;
    do {
        step = (step + 1) / 2;
        if (lcp(codes, n, rl, rl + offset + step) > np) offset += step;
    } while (step > 1);
    const int split = rl + offset;
    const int lc = rl == split ? rl : n + split;
    const int rc = split + 1 == rr ? rr : n + split + 1;
    left[i] = lc;
    right[i] = rc;
    parent[lc] = n + i;
    parent[rc] = n + i;
}

struct Box { float lo[3], hi[3]; };

// Leaf boxes from the FP32 corners, then the bottom-up merge: the fence makes
// a child's box visible before its arrival is counted, and only the second
// arrival at a parent carries on -- nothing ever waits.
__global__ void k_refit(const double* __restrict__ points, const int32_t* __restrict__ faces,
                        const uint32_t* __restrict__ order, int n,
                        const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                        const int32_t* __restrict__ parent, uint32_t* __restrict__ arrivals,
                        float* __restrict__ boxes) {
    const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    const int32_t* f = faces + (long)order[leaf] * 3;
    Box b;
    for (int k = 0; k < 3; ++k) {
        const float x = __double2float_rn(points[(long)f[0] * 3 + k]);
        const float y = __double2float_rn(points[(long)f[1] * 3 + k]);
        const float z = __double2float_rn(points[(long)f[2] * 3 + k]);
        b.lo[k] = fminf(x, fminf(y, z));
        b.hi[k] = fmaxf(x, fmaxf(y, z));
    }
    for (int k = 0; k < 3; ++k) {
        boxes[(long)leaf * 6 + k] = b.lo[k];
        boxes[(long)leaf * 6 + 3 + k] = b.hi[k];
    }
    int node = leaf;
    for (int depth = 0; depth < 2 * n + 2; ++depth) {
        const int p = parent[node];
        if (p < 0) return;
        __threadfence();
        if (atomicAdd(&arrivals[p - n], 1u) != 1u) return;
        __threadfence();
        const int l = left[p - n], r = right[p - n];
        for (int k = 0; k < 3; ++k) {
            const float a = __ldcg(&boxes[(long)l * 6 + k]);
            const float c = __ldcg(&boxes[(long)r * 6 + k]);
            boxes[(long)p * 6 + k] = fminf(a, c);
            const float a2 = __ldcg(&boxes[(long)l * 6 + 3 + k]);
            const float c2 = __ldcg(&boxes[(long)r * 6 + 3 + k]);
            boxes[(long)p * 6 + 3 + k] = fmaxf(a2, c2);
        }
        node = p;
    }
}


__device__ inline uint32_t encode_child(int child, int n) {
    return child < n ? (kLeafBit | (uint32_t)child) : (uint32_t)(child - n);
}

// Traversal layout: internal node i = 4 float4 = (left box lo, left hi.x),
// (left hi.yz, right lo.xy), (right lo.z, right hi), (children, unused).
__global__ void k_pack_nodes(const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                             const float* __restrict__ boxes, int n, float4* __restrict__ nodes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int l = left[i], r = right[i];
    const float* bl = boxes + (long)l * 6;
    const float* br = boxes + (long)r * 6;
    nodes[(long)i * 4 + 0] = make_float4(bl[0], bl[1], bl[2], bl[3]);
    nodes[(long)i * 4 + 1] = make_float4(bl[4], bl[5], br[0], br[1]);
    nodes[(long)i * 4 + 2] = make_float4(br[2], br[3], br[4], br[5]);
    nodes[(long)i * 4 + 3] = make_float4(__uint_as_float(encode_child(l, n)),
                                         __uint_as_float(encode_child(r, n)), 0.0f, 0.0f);
}

__global__ void k_pack_leaves(const double* __restrict__ points, const int32_t* __restrict__ faces,
                              const uint32_t* __restrict__ order, int n,
                              float4* __restrict__ leaves) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int tri = (int)order[i];
    const int32_t* f = faces + (long)tri * 3;
    double c[9];
    for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) c[k * 3 + a] = points[(long)f[k] * 3 + a];
    double2* l = reinterpret_cast<double2*>(leaves) + (long)i * kLeafFloat4s;
    l[0] = make_double2(c[0], c[1]);
    l[1] = make_double2(c[2], c[3]);
    l[2] = make_double2(c[4], c[5]);
    l[3] = make_double2(c[6], c[7]);
    l[4] = make_double2(c[8], __longlong_as_double((long long)tri));
}

int blocks_for(long n, int threads = kThreads) { return (int)((n + threads - 1) / threads); }

}  // namespace

size_t lbvh_scratch_bytes(int n) {
    // the carve sequence of lbvh_build, each piece rounded up to 256 bytes
    const size_t tiles = (size_t)((n + kSortTile - 1) / kSortTile);
    const size_t pieces[] = {
        sizeof(float) * 3 * (size_t)n,                 // centroids
        sizeof(float) * 6 * 1024,                      // bound partials
        64,                                            // bounds
        sizeof(uint32_t) * (size_t)n, sizeof(uint32_t) * (size_t)n,  // keys x2
        sizeof(uint32_t) * (size_t)n, sizeof(uint32_t) * (size_t)n,  // values x2
        sizeof(uint32_t) * kRadix * (tiles + 1),       // digit counts
        sizeof(int32_t) * (size_t)n, sizeof(int32_t) * (size_t)n,    // left, right
        sizeof(int32_t) * 2 * (size_t)n,               // parent
        sizeof(uint32_t) * (size_t)n,                  // arrivals
        sizeof(float) * 6 * 2 * (size_t)n,             // boxes
    };
    size_t total = 0;
    for (size_t bytes : pieces) total += (bytes + 255) & ~size_t(255);
    return total + 256;
}

// Builds the hierarchy over `n` target triangles into `nodes` ((n-1) x 4
// float4) and `leaves` (n x kLeafFloat4s float4) using `scratch`; optionally exports the
// canonical arrays (sorted codes, permutation, Karras children) for parity
// tests.  Returns the encoded root.
uint32_t lbvh_build(const double* points, const int32_t* faces, int n, void* scratch,
                    float4* nodes, float4* leaves, cudaStream_t stream, LbvhExport* out) {
    char* base = static_cast<char*>(scratch);
    auto carve = [&base](size_t bytes) {
        char* p = base;
        base += (bytes + 255) & ~size_t(255);
        return p;
    };
    float* centroids = reinterpret_cast<float*>(carve(sizeof(float) * 3 * n));
    float* bound_partial = reinterpret_cast<float*>(carve(sizeof(float) * 6 * 1024));
    float* bounds = reinterpret_cast<float*>(carve(64));
    uint32_t* keys[2] = {reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n)),
                         reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n))};
    uint32_t* values[2] = {reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n)),
                           reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n))};
    const int tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* counts = reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * kRadix * (tiles + 1)));
    int32_t* left = reinterpret_cast<int32_t*>(carve(sizeof(int32_t) * n));
    int32_t* right = reinterpret_cast<int32_t*>(carve(sizeof(int32_t) * n));
    int32_t* parent = reinterpret_cast<int32_t*>(carve(sizeof(int32_t) * 2 * n));
    uint32_t* arrivals = reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n));
    float* boxes = reinterpret_cast<float*>(carve(sizeof(float) * 6 * 2 * n));

    k_centroids<<<blocks_for(n), kThreads, 0, stream>>>(points, faces, n, centroids);
    const int bound_blocks = blocks_for(n) < 1024 ? blocks_for(n) : 1024;
    k_bounds_partial<<<bound_blocks, kThreads, 0, stream>>>(centroids, n, bound_partial);
    k_bounds_final<<<1, 32, 0, stream>>>(bound_partial, bound_blocks, bounds);
    k_morton<<<blocks_for(n), kThreads, 0, stream>>>(centroids, n, bounds, keys[0], values[0]);
    int cur = 0;
    for (int shift = 0; shift < 32; shift += kRadixBits) {
        k_radix_histogram<<<tiles, kThreads, 0, stream>>>(keys[cur], n, shift, counts, tiles);
        k_radix_scan<<<1, 1024, 0, stream>>>(counts, kRadix * tiles);
        k_radix_scatter<<<tiles, kThreads, 0, stream>>>(keys[cur], values[cur], n, shift, counts,
                                                        tiles, keys[1 - cur], values[1 - cur]);
        cur = 1 - cur;
    }
    const uint32_t* codes = keys[cur];
    const uint32_t* order = values[cur];
    cudaMemsetAsync(parent, 0xff, sizeof(int32_t) * 2 * n, stream);
    cudaMemsetAsync(arrivals, 0, sizeof(uint32_t) * n, stream);
    if (n > 1) {
        k_karras<<<blocks_for(n - 1), kThreads, 0, stream>>>(codes, n, left, right, parent);
    }
    k_refit<<<blocks_for(n), kThreads, 0, stream>>>(points, faces, order, n, left, right, parent,
                                                    arrivals, boxes);
    if (n > 1) k_pack_nodes<<<blocks_for(n - 1), kThreads, 0, stream>>>(left, right, boxes, n, nodes);
    k_pack_leaves<<<blocks_for(n), kThreads, 0, stream>>>(points, faces, order, n, leaves);
    if (out) {
        cudaMemcpyAsync(out->codes, codes, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(out->order, order, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, stream);
        if (n > 1) {
            cudaMemcpyAsync(out->left, left, sizeof(int32_t) * (n - 1), cudaMemcpyDeviceToHost, stream);
            cudaMemcpyAsync(out->right, right, sizeof(int32_t) * (n - 1), cudaMemcpyDeviceToHost, stream);
        }
        cudaMemcpyAsync(out->bounds, bounds, sizeof(float) * 6, cudaMemcpyDeviceToHost, stream);
    }
    return n > 1 ? 0u : (kLeafBit | 0u);
}

// ---------------------------------------------------------------------------
// Target ingestion: normalisation and vertex normals on the device
// ---------------------------------------------------------------------------
//
// The target arrives in the caller's units.  Its points are moved into the
// normalised frame in place, (p - center) * scale per coordinate with the two
// roundings of the host's normalisation (mesh.cpp:183-187), and its
// area-weighted vertex normals (mesh.cpp:71-88) are summed per vertex over
// its faces in ascending face order, as the host's face loop adds them, then
// normalised -- so both are bit-identical to the host's.  A vertex's faces
// come from a stable sort of the (vertex, face) corner pairs by vertex.

namespace {

__global__ void k_normalize(double* __restrict__ p, long count, double cx, double cy, double cz,
                            double scale) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int k = (int)(i % 3);
    const double c = k == 0 ? cx : (k == 1 ? cy : cz);
    p[i] = __dmul_rn(__dsub_rn(p[i], c), scale);
}

__global__ void k_corner_keys(const int32_t* __restrict__ faces, long corners, uint32_t* __restrict__ keys,
                              uint32_t* __restrict__ values) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= corners) return;
    keys[i] = (uint32_t)faces[i];
    values[i] = (uint32_t)(i / 3);
}

__device__ inline long lower_bound_key(const uint32_t* __restrict__ keys, long n, uint32_t x) {
    long lo = 0, hi = n;
    while (lo < hi) {
        const long mid = (lo + hi) >> 1;
        if (keys[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void k_target_normals(const double* __restrict__ p, int n, const int32_t* __restrict__ faces,
                                 const uint32_t* __restrict__ keys, const uint32_t* __restrict__ face_of,
                                 long corners, double* __restrict__ normals) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const long j0 = lower_bound_key(keys, corners, (uint32_t)v);
    const long j1 = lower_bound_key(keys, corners, (uint32_t)v + 1u);
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (long j = j0; j < j1; ++j) {
        const int32_t* f = faces + (long)face_of[j] * 3;
        const double* a = p + (long)f[0] * 3;
        const double* b = p + (long)f[1] * 3;
        const double* c = p + (long)f[2] * 3;
        const double e10 = __dsub_rn(b[0], a[0]), e11 = __dsub_rn(b[1], a[1]), e12 = __dsub_rn(b[2], a[2]);
        const double e20 = __dsub_rn(c[0], a[0]), e21 = __dsub_rn(c[1], a[1]), e22 = __dsub_rn(c[2], a[2]);
        t0 = __dadd_rn(t0, __dsub_rn(__dmul_rn(e11, e22), __dmul_rn(e12, e21)));
        t1 = __dadd_rn(t1, __dsub_rn(__dmul_rn(e12, e20), __dmul_rn(e10, e22)));
        t2 = __dadd_rn(t2, __dsub_rn(__dmul_rn(e10, e21), __dmul_rn(e11, e20)));
    }
    const double length =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(t0, t0), __dmul_rn(t1, t1)), __dmul_rn(t2, t2)));
    double* out = normals + (long)v * 3;
    if (length > 0.0) {
        out[0] = __ddiv_rn(t0, length);
        out[1] = __ddiv_rn(t1, length);
        out[2] = __ddiv_rn(t2, length);
    } else {
        out[0] = out[1] = out[2] = 0.0;
    }
}

// Radix passes that cover vertex indices below n, rounded up to an even
// count so that the sorted arrays end in the first buffer.
int corner_sort_passes(int n) {
    int bits = 1;
    while (bits < 32 && (1u << bits) < (uint32_t)n) ++bits;
    const int passes = (bits + kRadixBits - 1) / kRadixBits;
    return passes + (passes & 1);
}

}  // namespace

size_t ingest_scratch_bytes(int n, int F) {
    const size_t corners = (size_t)F * 3;
    const size_t tiles = (corners + kSortTile - 1) / kSortTile;
    const size_t pieces[] = {sizeof(uint32_t) * corners, sizeof(uint32_t) * corners,
                             sizeof(uint32_t) * corners, sizeof(uint32_t) * corners,
                             sizeof(uint32_t) * kRadix * (tiles + 1)};
    size_t total = 0;
    for (size_t bytes : pieces) total += (bytes + 255) & ~size_t(255);
    (void)n;
    return total + 256;
}

int ingest_launches(int n, int F) { return 2 + 3 * corner_sort_passes(n) + (F > 0 ? 1 : 0); }

void ingest_target(double* points, int n, const int32_t* faces, int F, const double center[3], double scale,
                   double* normals, void* scratch, cudaStream_t stream) {
    k_normalize<<<blocks_for((long)n * 3), kThreads, 0, stream>>>(points, (long)n * 3, center[0], center[1],
                                                                  center[2], scale);
    const long corners = (long)F * 3;
    char* base = static_cast<char*>(scratch);
    auto carve = [&base](size_t bytes) {
        char* q = base;
        base += (bytes + 255) & ~size_t(255);
        return q;
    };
    uint32_t* keys[2] = {reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * corners)),
                         reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * corners))};
    uint32_t* values[2] = {reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * corners)),
                           reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * corners))};
    const int tiles = (int)((corners + kSortTile - 1) / kSortTile);
    uint32_t* counts = reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * kRadix * (tiles + 1)));
    if (F > 0) {
        k_corner_keys<<<blocks_for(corners), kThreads, 0, stream>>>(faces, corners, keys[0], values[0]);
        int cur = 0;
        const int passes = corner_sort_passes(n);
        for (int pass = 0; pass < passes; ++pass) {
            const int shift = pass * kRadixBits;
            k_radix_histogram<<<tiles, kThreads, 0, stream>>>(keys[cur], (int)corners, shift, counts, tiles);
            k_radix_scan<<<1, 1024, 0, stream>>>(counts, kRadix * tiles);
            k_radix_scatter<<<tiles, kThreads, 0, stream>>>(keys[cur], values[cur], (int)corners, shift,
                                                            counts, tiles, keys[1 - cur], values[1 - cur]);
            cur = 1 - cur;
        }
    }
    k_target_normals<<<blocks_for(n), kThreads, 0, stream>>>(points, n, faces, keys[0], values[0], corners,
                                                             normals);
}

// ---------------------------------------------------------------------------
// Closest-point query
// ---------------------------------------------------------------------------

__device__ inline float box_distance(F3 p, float lx, float ly, float lz, float hx, float hy,
                                     float hz) {
    const float dx = fmaxf(fmaxf(lx - p.x, p.x - hx), 0.0f);
    const float dy = fmaxf(fmaxf(ly - p.y, p.y - hy), 0.0f);
    const float dz = fmaxf(fmaxf(lz - p.z, p.z - hz), 0.0f);
    return dx * dx + dy * dy + dz * dz;
}

// FP64 closest point with barycentrics, the reference routine's exact steps
// (closest_point.cpp:24-121), with every product and sum rounded on its own so
// the result matches the host build bit for bit.
__device__ inline double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double da(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ inline D3 vsub(D3 a, D3 b) { return {ds(a.x, b.x), ds(a.y, b.y), ds(a.z, b.z)}; }
__device__ inline D3 vadd(D3 a, D3 b) { return {da(a.x, b.x), da(a.y, b.y), da(a.z, b.z)}; }
__device__ inline D3 vmul(D3 a, double s) { return {dm(a.x, s), dm(a.y, s), dm(a.z, s)}; }
__device__ inline double vdot(D3 a, D3 b) { return da(da(dm(a.x, b.x), dm(a.y, b.y)), dm(a.z, b.z)); }

__device__ D3 closest_point_fp64(D3 p, D3 a, D3 b, D3 c, double* bary) {
    const D3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    const double d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { bary[0] = 1; bary[1] = 0; bary[2] = 0; return a; }
    const D3 bp = vsub(p, b);
    const double d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { bary[0] = 0; bary[1] = 1; bary[2] = 0; return b; }
    const double vc = ds(dm(d1, d4), dm(d3, d2));
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double den = ds(d1, d3);
        const double v = den != 0.0 ? __ddiv_rn(d1, den) : 0.0;
        bary[0] = ds(1.0, v); bary[1] = v; bary[2] = 0.0;
        return vadd(a, vmul(ab, v));
    }
    const D3 cp = vsub(p, c);
    const double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { bary[0] = 0; bary[1] = 0; bary[2] = 1; return c; }
    const double vb = ds(dm(d5, d2), dm(d1, d6));
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double den = ds(d2, d6);
        const double w = den != 0.0 ? __ddiv_rn(d2, den) : 0.0;
        bary[0] = ds(1.0, w); bary[1] = 0.0; bary[2] = w;
        return vadd(a, vmul(ac, w));
    }
    const double va = ds(dm(d3, d6), dm(d5, d4));
    if (va <= 0.0 && ds(d4, d3) >= 0.0 && ds(d5, d6) >= 0.0) {
        const double den = da(ds(d4, d3), ds(d5, d6));
        const double w = den != 0.0 ? __ddiv_rn(ds(d4, d3), den) : 0.0;
        bary[0] = 0.0; bary[1] = ds(1.0, w); bary[2] = w;
        return vadd(b, vmul(vsub(c, b), w));
    }
    const double den = da(da(va, vb), vc);
    if (fabs(den) < 1e-300) { bary[0] = 1; bary[1] = 0; bary[2] = 0; return a; }
    const double v = __ddiv_rn(vb, den), w = __ddiv_rn(vc, den);
    bary[0] = ds(ds(1.0, v), w); bary[1] = v; bary[2] = w;
    return vadd(vadd(a, vmul(ab, v)), vmul(ac, w));
}

__device__ inline D3 vnormalized(D3 a) {
    const double length = __dsqrt_rn(vdot(a, a));
    if (!(length > 0.0)) return {0.0, 0.0, 0.0};
    return {__ddiv_rn(a.x, length), __ddiv_rn(a.y, length), __ddiv_rn(a.z, length)};
}

// Robust weight, src/energy/robust.cpp:30-58.
__device__ inline double robust_weight(int kernel, double squared, double threshold) {
    if (squared < 0.0) squared = 0.0;
    if (kernel == 1) {
        if (threshold <= 0.0) return 1.0;
        if (squared <= threshold * threshold) return 1.0;
        return threshold / sqrt(squared);
    }
    if (kernel == 2) {
        if (threshold <= 0.0) return 1.0;
        const double ratio = squared / (threshold * threshold);
        const double den = 1.0 + ratio;
        return 1.0 / (den * den);
    }
    return 1.0;
}

// FP64 squared distance from q to triangle `tri` of the target.
__device__ inline double triangle_distance_fp64(const WrapDev& w, D3 q, int tri) {
    const int32_t* f = w.tgt_faces + (long)tri * 3;
    double bary[3];
    const D3 c = closest_point_fp64(q, load_d3(w.tgt_points, f[0]), load_d3(w.tgt_points, f[1]),
                                    load_d3(w.tgt_points, f[2]), bary);
    const D3 d = vsub(c, q);
    return vdot(d, d);
}

// FP64 squared distance from q to the triangle of leaf `leaf` (its corners
// are stored in FP64), and the triangle's index.
__device__ inline double leaf_distance(const WrapDev& w, int leaf, D3 q, int* tri) {
    const double2* l = reinterpret_cast<const double2*>(w.bvh_leaves) + (long)leaf * (kLeafFloat4s);
    const double2 l0 = __ldg(l), l1 = __ldg(l + 1), l2 = __ldg(l + 2), l3 = __ldg(l + 3),
                  l4 = __ldg(l + 4);
    *tri = (int)__double_as_longlong(l4.y);
    double bary[3];
    const D3 c = closest_point_fp64(q, {l0.x, l0.y, l1.x}, {l1.y, l2.x, l2.y}, {l3.x, l3.y, l4.x}, bary);
    const D3 d = vsub(c, q);
    return vdot(d, d);
}

// Nearest target triangle for `q`: the FP64 brute-force answer (smallest
// FP64 distance from the reference's closest-point routine, exact ties to the
// lowest triangle index), found by walking the hierarchy.  Boxes are pruned
// in FP32, which is well conditioned (a box distance is a clamp and three
// squares), with `w.rank_window` of slack, far above the rounding of the FP32
// boxes and query; every triangle reached is measured in FP64 -- an FP32
// closest-point routine can misplace its point on thin sliver triangles by
// far more than any fixed window.  `seed` is a triangle whose distance bounds
// the search from the start.  Returns the winner, or -1; `steps_taken` (if
// given) receives the nodes and leaves visited.
__device__ int nearest_triangle(const WrapDev& w, F3 q, D3 q64, int seed, int* overflow,
                                long* steps_taken = nullptr) {
    const double slack = (double)w.rank_window;
    double best = 1e300;     // FP64 squared distance of the best triangle so far
    float bound = 3.4e38f;   // FP32 pruning radius^2: (sqrt(best) + slack)^2, rounded up
    int best_tri = -1;
    auto consider = [&](int tri, double d) {
        if (d < best || (d == best && tri < best_tri)) {
            best = d;
            best_tri = tri;
            const double r = sqrt(best) + slack;
            bound = __double2float_ru(r * r);
        }
    };
    if (seed >= 0 && seed < w.F) consider(seed, triangle_distance_fp64(w, q64, seed));
    uint32_t stack[kStackDepth];
    float stack_d[kStackDepth];
    int sp = 0;
    uint32_t node = (uint32_t)w.bvh_root;
    // A tree visits each node at most once; the cap only guards against a
    // corrupt hierarchy, which it reports instead of looping.
    const long step_limit = 4L * (long)w.F + 1024;
    long steps = 0;
    while (true) {
        if (++steps > step_limit) {
            *overflow = 1;
            break;
        }
        if (node & kLeafBit) {
            int tri;
            const double d = leaf_distance(w, (int)(node & ~kLeafBit), q64, &tri);
            if (tri != seed) consider(tri, d);
        } else {
            const float4* nd = w.bvh_nodes + (long)node * 4;
            const float4 n0 = __ldg(nd), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3);
            const float dl = box_distance(q, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y);
            const float dr = box_distance(q, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w);
            const uint32_t cl = __float_as_uint(n3.x), cr = __float_as_uint(n3.y);
            const bool hl = dl < bound, hr = dr < bound;
            if (hl && hr) {
                const bool left_first = dl <= dr;
                if (sp < kStackDepth) {
                    stack[sp] = left_first ? cr : cl;
                    stack_d[sp] = left_first ? dr : dl;
                    ++sp;
                } else {
                    *overflow = 1;
                }
                node = left_first ? cl : cr;
                continue;
            }
            if (hl) { node = cl; continue; }
            if (hr) { node = cr; continue; }
        }
        // pop the next subtree that can still hold something closer
        bool found = false;
        while (sp > 0) {
            --sp;
            if (stack_d[sp] < bound) { node = stack[sp]; found = true; break; }
        }
        if (!found) break;
    }
    if (steps_taken) *steps_taken = steps;
    return best_tri;
}

// Walks longer than this many steps put their vertex on the wrap's list for
// its next query, where a warp walks it (a vertex over a hole in the target,
// or above the fan of slivers at a lat-long pole, stays far from the nearest
// triangles and walks hundreds to thousands of steps query after query).
constexpr long kLongWalk = 256;
// A warp's stack: 32 entries for each of 32 levels of pending subtrees.
constexpr int kWarpStack = 1024;

// The nearest triangle for `q` found by the 32 lanes of a warp together: the
// same pruning and the same winner rule as `nearest_triangle`, so the same
// answer, with up to 32 pending subtrees taken from the stack at a time, so
// that a walk of thousands of steps takes tens to a hundred dependent rounds.
// `nodes` / `dists` are the warp's stack.  Should the stack not hold a
// round's children, the rest of the walk is left to one lane
// (`*unfinished`), seeded with the winner so far, which is returned.  Every
// lane returns the same triangle; `*work` is the entries taken.
__device__ int nearest_triangle_warp(const WrapDev& w, F3 q, D3 q64, int seed, uint32_t* nodes,
                                     float* dists, int* overflow, bool* unfinished, long* work) {
    const int lane = threadIdx.x & 31;
    const double slack = (double)w.rank_window;
    double best = 1e300;
    int best_tri = -1;
    float bound = 3.4e38f;
    if (seed >= 0 && seed < w.F) {
        best = triangle_distance_fp64(w, q64, seed);
        best_tri = seed;
        const double r = sqrt(best) + slack;
        bound = __double2float_ru(r * r);
    }
    if (lane == 0) {
        nodes[0] = (uint32_t)w.bvh_root;
        dists[0] = 0.0f;
    }
    int sp = 1;  // warp-uniform
    const long round_limit = 4L * (long)w.F + 1024;
    long rounds = 0, taken = 0;
    *unfinished = false;
    __syncwarp();
    while (sp > 0) {
        if (++rounds > round_limit) {  // a corrupt hierarchy: report, do not loop
            *overflow = 1;
            break;
        }
        const int take = sp < 32 ? sp : 32;
        sp -= take;
        taken += take;
        uint32_t node = 0;
        bool live = false;
        if (lane < take) {
            node = nodes[sp + lane];
            live = dists[sp + lane] < bound;
        }
        __syncwarp();
        // leaves: FP64 distance, then the warp's winner under the exact rule
        double d = 1e300;
        int tri = 0x7fffffff;
        if (live && (node & kLeafBit)) {
            int t;
            const double x = leaf_distance(w, (int)(node & ~kLeafBit), q64, &t);
            if (t != seed) {
                d = x;
                tri = t;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double od = __shfl_xor_sync(0xffffffffu, d, o);
            const int ot = __shfl_xor_sync(0xffffffffu, tri, o);
            if (od < d || (od == d && ot < tri)) {
                d = od;
                tri = ot;
            }
        }
        if (d < best || (d == best && tri < best_tri)) {
            best = d;
            best_tri = tri;
            const double r = sqrt(best) + slack;
            bound = __double2float_ru(r * r);
        }
        // internal nodes: the children that can still hold something closer,
        // the nearer one pushed last (taken first)
        uint32_t push[2] = {0, 0};
        float push_d[2] = {0.0f, 0.0f};
        int pushes = 0;
        if (live && !(node & kLeafBit)) {
            const float4* nd = w.bvh_nodes + (long)node * 4;
            const float4 n0 = __ldg(nd), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3);
            const float dl = box_distance(q, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y);
            const float dr = box_distance(q, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w);
            const uint32_t cl = __float_as_uint(n3.x), cr = __float_as_uint(n3.y);
            const bool hl = dl < bound, hr = dr < bound;
            const bool left_first = dl <= dr;
            if (hl && hr) {
                push[0] = left_first ? cr : cl;
                push_d[0] = left_first ? dr : dl;
                push[1] = left_first ? cl : cr;
                push_d[1] = left_first ? dl : dr;
                pushes = 2;
            } else if (hl || hr) {
                push[0] = hl ? cl : cr;
                push_d[0] = hl ? dl : dr;
                pushes = 1;
            }
        }
        int at = pushes;  // inclusive prefix over the lanes, then exclusive
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, at, o);
            if (lane >= o) at += y;
        }
        const int total = __shfl_sync(0xffffffffu, at, 31);
        at -= pushes;
        if (sp + total > kWarpStack) {  // the rest by one lane, from the winner so far
            *unfinished = true;
            break;
        }
        for (int k = 0; k < pushes; ++k) {
            nodes[sp + at + k] = push[k];
            dists[sp + at + k] = push_d[k];
        }
        sp += total;
        __syncwarp();
    }
    *work = taken;
    return best_tri;
}

__device__ inline bool queries(int phase) {
    return phase == kPhaseTransfer || phase == kPhaseRefresh || phase == kPhaseFinal;
}

// The correspondence of template vertex v to triangle `tri` (-1: none), with
// the filters in the order the reference applies them
// (correspondence.cpp:35-80) and the reweighting of route_a.cpp:19-38.
__device__ void store_correspondence(const WrapDev& w, int level, int v, int tri) {
    uint8_t code = 0;
    D3 point = {0, 0, 0}, normal = {0, 0, 0};
    double distance = 0.0, robust = 1.0;
    if (tri >= 0) {
        const D3 q = load_d3(w.deformed, v);
        const int32_t* f = w.tgt_faces + (long)tri * 3;
        double bary[3];
        point = closest_point_fp64(q, load_d3(w.tgt_points, f[0]), load_d3(w.tgt_points, f[1]),
                                   load_d3(w.tgt_points, f[2]), bary);
        const D3 d = vsub(point, q);
        distance = __dsqrt_rn(vdot(d, d));
        const D3 n0 = load_d3(w.tgt_normals, f[0]), n1 = load_d3(w.tgt_normals, f[1]),
                 n2 = load_d3(w.tgt_normals, f[2]);
        normal = vnormalized(vadd(vadd(vmul(n0, bary[0]), vmul(n1, bary[1])), vmul(n2, bary[2])));
        if (distance > w.distance_threshold) {
            code = 1;
        } else if (vdot(load_d3(w.qnormals, v), normal) < w.min_normal_cosine) {
            code = 2;
        } else if (distance > 0.0) {
            const D3 offset = vsub(q, point);
            const double slope = __ddiv_rn(fabs(vdot(normal, offset)), distance);
            if (slope < w.min_slope) code = 3;
        }
        if (code == 0) {
            const D3 o = vsub(q, point);
            const double squared = vdot(o, o);
            const double threshold = w.robust_threshold[level];
            robust = threshold > 0.0 ? robust_weight(w.robust_kernel[level], squared, threshold) : 1.0;
        }
    } else {
        code = 1;
    }
    store_d3(w.corr_point, v, point);
    store_d3(w.corr_normal, v, normal);
    w.corr_distance[v] = distance;
    w.corr_triangle[v] = tri;
    w.corr_code[v] = code;
    w.robust[v] = robust;
}

// A masked vertex keeps its previous triangle and takes no correspondence.
__device__ inline void store_masked(const WrapDev& w, int v) {
    store_d3(w.corr_point, v, {0, 0, 0});
    store_d3(w.corr_normal, v, {0, 0, 0});
    w.corr_distance[v] = 0.0;
    w.corr_code[v] = 4;
    w.robust[v] = 1.0;
}

// The correspondence of template vertex v, found by one thread.
__device__ void query_vertex(const WrapDev& w, int level, int v) {
    if (w.mask && !w.mask[v]) {
        store_masked(w, v);
        return;
    }
    const float4 q32 = w.deformed32[v];
    int overflow = 0;
    const int tri = nearest_triangle(w, {q32.x, q32.y, q32.z}, load_d3(w.deformed, v), w.corr_triangle[v],
                                     &overflow);
    if (overflow) atomicOr(&w.control->error, 1);
    store_correspondence(w, level, v, tri);
}

// Thread per vertex, block row per wrap.
__global__ void k_query(const WrapDev* __restrict__ wraps) {
    const WrapDev& w = wraps[blockIdx.y];
    const WrapControl c = *w.control;
    if (!queries(c.tick_phase)) return;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= w.V) return;
    query_vertex(w, c.level, v);
}

// Puts vertex v on the wrap's list of long walks for its next query (list
// 1 - long_cur), unless the list is full.
__device__ inline void list_long_walk(const WrapDev& w, int next, int v) {
    const int at = atomicAdd(w.long_count + next, 1);
    if (at < kLongCap) {
        w.long_list[next * kLongCap + at] = v;
        w.long_flag[(long)next * w.V + v] = 1;
    }
}

// The same work as queues over a grid that fits on the device at once.
// First, the vertices whose walk was long at the wrap's previous query (its
// list), a warp each.  Then every other vertex of every querying wrap, in
// wrap then vertex order, handed out 32 at a time to whichever warp is free
// (a walk's length varies a lot from vertex to vertex, so fixed blocks would
// hold an SM until their slowest warp ends).  A launch lasts as long as its
// longest walks: the warps take those at its start, in tens of dependent
// rounds, beside the threads' walks instead of after them.  A walk longer
// than kLongWalk steps lists its vertex for the wrap's next query.
// counter[0]: the vertices' queue head; counter[1]: the long walks'; both
// start at 0.
__global__ void __launch_bounds__(128) k_query_queue(const WrapDev* __restrict__ wraps, int wrap_count,
                                                    int* __restrict__ counter) {
    extern __shared__ float4 query_shared[];  // 4 warps' stacks, then 2 x (wrap_count + 1) ints
    uint32_t* stack_nodes = reinterpret_cast<uint32_t*>(query_shared);
    float* stack_dists = reinterpret_cast<float*>(stack_nodes + 4 * kWarpStack);
    int* first = reinterpret_cast<int*>(stack_dists + 4 * kWarpStack);  // each wrap's first vertex item
    int* first_long = first + wrap_count + 1;                             // and first long-walk item
    for (int i = threadIdx.x; i < wrap_count; i += blockDim.x) {
        const WrapDev& w = wraps[i];
        const bool on = queries(w.control->tick_phase);
        first[i + 1] = on ? w.V : 0;
        first_long[i + 1] = on ? min(w.long_count[w.control->long_cur], kLongCap) : 0;
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scans by warp 0, 32 wraps at a time
        const int lane = threadIdx.x;
        for (int k = 0; k < 2; ++k) {
            int* f = k == 0 ? first : first_long;
            int carry = 0;
            for (int base = 0; base < wrap_count; base += 32) {
                int x = base + lane < wrap_count ? f[base + lane + 1] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                if (base + lane < wrap_count) f[base + lane + 1] = carry + x;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
            if (lane == 0) f[0] = 0;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    auto wrap_of = [&](const int* f, int item) {  // the last wrap whose first item is <= item
        int lo = 0, hi = wrap_count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (f[mid] <= item) lo = mid; else hi = mid - 1;
        }
        return lo;
    };
    // ---- the listed long walks, a warp each ----
    {
        const int total = first_long[wrap_count];
        uint32_t* nodes = stack_nodes + (threadIdx.x >> 5) * kWarpStack;
        float* dists = stack_dists + (threadIdx.x >> 5) * kWarpStack;
        while (true) {
            int item = 0;
            if (lane == 0) item = atomicAdd(counter + 1, 1);
            item = __shfl_sync(0xffffffffu, item, 0);
            if (item >= total) break;
            const int wi = wrap_of(first_long, item);
            const WrapDev& w = wraps[wi];
            const int cur = w.control->long_cur;
            const int v = w.long_list[cur * kLongCap + item - first_long[wi]];
            const float4 q32 = w.deformed32[v];
            const F3 q = {q32.x, q32.y, q32.z};
            const D3 q64 = load_d3(w.deformed, v);
            int overflow = 0;
            bool unfinished = false;
            long work = 0;
            int tri = nearest_triangle_warp(w, q, q64, w.corr_triangle[v], nodes, dists, &overflow,
                                            &unfinished, &work);
            if (lane == 0) {
                if (unfinished) tri = nearest_triangle(w, q, q64, tri, &overflow);
                if (overflow) atomicOr(&w.control->error, 1);
                store_correspondence(w, w.control->level, v, tri);
                if (unfinished || work > kLongWalk) list_long_walk(w, 1 - cur, v);
            }
            __syncwarp();
        }
    }
    // ---- every other vertex, a thread each ----
    const int total = first[wrap_count];
    while (true) {
        int base = 0;
        if (lane == 0) base = atomicAdd(counter, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const int item = base + lane;
        if (item >= total) continue;
        const int wi = wrap_of(first, item);
        const WrapDev& w = wraps[wi];
        const int v = item - first[wi];
        if (w.mask && !w.mask[v]) {
            store_masked(w, v);
            continue;
        }
        const int cur = w.control->long_cur;
        if (w.long_flag[(long)cur * w.V + v]) continue;  // a warp's walk, above
        const float4 q32 = w.deformed32[v];
        int overflow = 0;
        long steps = 0;
        const int tri = nearest_triangle(w, {q32.x, q32.y, q32.z}, load_d3(w.deformed, v),
                                         w.corr_triangle[v], &overflow, &steps);
        if (overflow) atomicOr(&w.control->error, 1);
        store_correspondence(w, w.control->level, v, tri);
        if (steps > kLongWalk) list_long_walk(w, 1 - cur, v);
    }
}

// Stand-alone query over a prepared hierarchy (parity tests and the
// `closest_points` entry point): FP32 ranking, FP64 winner.
__global__ void k_closest_points(const WrapDev* __restrict__ wraps, const double* __restrict__ queries,
                                 int count, double* __restrict__ out_points,
                                 double* __restrict__ out_normals, double* __restrict__ out_distances,
                                 int32_t* __restrict__ out_triangles, int* __restrict__ overflow_flag) {
    const WrapDev& w = wraps[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const D3 q = load_d3(queries, i);
    int overflow = 0;
    const int tri = nearest_triangle(w, {__double2float_rn(q.x), __double2float_rn(q.y),
                                         __double2float_rn(q.z)}, q, -1, &overflow);
    if (overflow) atomicOr(overflow_flag, 1);
    D3 point = {0, 0, 0}, normal = {0, 0, 0};
    double distance = 0.0;
    if (tri >= 0) {
        const int32_t* f = w.tgt_faces + (long)tri * 3;
        double bary[3];
        point = closest_point_fp64(q, load_d3(w.tgt_points, f[0]), load_d3(w.tgt_points, f[1]),
                                   load_d3(w.tgt_points, f[2]), bary);
        const D3 d = vsub(point, q);
        distance = __dsqrt_rn(vdot(d, d));
        normal = vnormalized(vadd(vadd(vmul(load_d3(w.tgt_normals, f[0]), bary[0]),
                                       vmul(load_d3(w.tgt_normals, f[1]), bary[1])),
                                  vmul(load_d3(w.tgt_normals, f[2]), bary[2])));
    }
    store_d3(out_points, i, point);
    store_d3(out_normals, i, normal);
    out_distances[i] = distance;
    out_triangles[i] = tri;
}

void launch_query(const WrapDev* wraps, int wrap_count, int max_vertices, cudaStream_t stream, int* counter) {
    if (!counter) {
        dim3 grid(blocks_for(max_vertices, 128), wrap_count);
        k_query<<<grid, 128, 0, stream>>>(wraps);
        return;
    }
    // the warps' stacks, then two scans over the wraps (1024 at most)
    constexpr size_t kStackBytes = (sizeof(uint32_t) + sizeof(float)) * kWarpStack * 4;
    static const int resident = [] {  // blocks of the queue that fit on the device at once
        int device = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_query_queue, 128,
                                                      kStackBytes + 2 * sizeof(int) * 1025);
        const int blocks = sms * (per_sm > 0 ? per_sm : 1);
        return blocks > 0 ? blocks : 1;
    }();
    cudaMemsetAsync(counter, 0, 2 * sizeof(int), stream);
    k_query_queue<<<resident, 128, kStackBytes + 2 * sizeof(int) * (wrap_count + 1), stream>>>(
        wraps, wrap_count, counter);
}

void launch_closest_points(const WrapDev* wrap, const double* queries, int count,
                           double* points, double* normals, double* distances, int32_t* triangles,
                           int* overflow, cudaStream_t stream) {
    k_closest_points<<<blocks_for(count, 128), 128, 0, stream>>>(
        wrap, queries, count, points, normals, distances, triangles, overflow);
}

}  // namespace nricp_b200

namespace nricp_b200 {

namespace {

// Out-of-range face indices would make the centroid pass read outside the
// caller's vertex buffer; this pass only records that they exist.
__global__ void k_check_faces(const int32_t* __restrict__ faces, int count, int vertex_count,
                              int* __restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count * 3) return;
    const int v = faces[i];
    if (v < 0 || v >= vertex_count) atomicOr(flag, 1);
}

}  // namespace

void check(cudaError_t status, const char* what);  // throws CudaError (session.cu)

size_t lbvh_export_scratch_bytes(int n) {
    const size_t tiles = (size_t)((n + kSortTile - 1) / kSortTile);
    const size_t pieces[] = {
        sizeof(float) * 3 * (size_t)n,            // centroids
        sizeof(float) * 6 * 1024,                 // bound partials
        sizeof(uint32_t) * (size_t)n,             // second key buffer
        sizeof(uint32_t) * (size_t)n,             // second value buffer
        sizeof(uint32_t) * kRadix * (tiles + 1),  // digit counts
        sizeof(int32_t) * 2 * (size_t)n,          // parent links (written by the split pass)
        256,                                      // validation flag
    };
    size_t total = 0;
    for (size_t bytes : pieces) total += (bytes + 255) & ~size_t(255);
    return total;
}

// The canonical arrays of the hierarchy (sorted codes, permutation, Karras
// children, centroid bounds) straight into caller-owned device buffers, with
// every intermediate in `scratch`.  The sort ping-pongs between the caller's
// code/permutation buffers and a scratch pair; with an even number of passes
// the result lands in the caller's.  Returns false when a face index is out of
// range (nothing past the check reads the vertices then).
bool lbvh_export_to_device(const double* points, int vertex_count, const int32_t* faces, int n,
                           void* scratch, uint32_t* codes, uint32_t* order, int32_t* left,
                           int32_t* right, float* bounds, cudaStream_t stream) {
    char* base = static_cast<char*>(scratch);
    auto carve = [&base](size_t bytes) {
        char* p = base;
        base += (bytes + 255) & ~size_t(255);
        return p;
    };
    float* centroids = reinterpret_cast<float*>(carve(sizeof(float) * 3 * n));
    float* bound_partial = reinterpret_cast<float*>(carve(sizeof(float) * 6 * 1024));
    uint32_t* keys[2] = {codes, reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n))};
    uint32_t* values[2] = {order, reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * n))};
    const int tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* counts = reinterpret_cast<uint32_t*>(carve(sizeof(uint32_t) * kRadix * (tiles + 1)));
    int32_t* parent = reinterpret_cast<int32_t*>(carve(sizeof(int32_t) * 2 * n));
    int* flag = reinterpret_cast<int*>(carve(256));

    // the array keeps the previous call's contents: clear what starts at zero
    check(cudaMemsetAsync(flag, 0, sizeof(int), stream), "hierarchy export: clearing the flag");
    k_check_faces<<<blocks_for((long)n * 3), kThreads, 0, stream>>>(faces, n, vertex_count, flag);
    check(cudaGetLastError(), "hierarchy export: face check");
    int host_flag = 0;
    check(cudaMemcpyAsync(&host_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, stream),
          "hierarchy export: reading the flag");
    // the caller's stream is synchronised here, on every call
    check(cudaStreamSynchronize(stream), "hierarchy export: face check");
    if (host_flag) return false;

    k_centroids<<<blocks_for(n), kThreads, 0, stream>>>(points, faces, n, centroids);
    const int bound_blocks = blocks_for(n) < 1024 ? blocks_for(n) : 1024;
    k_bounds_partial<<<bound_blocks, kThreads, 0, stream>>>(centroids, n, bound_partial);
    k_bounds_final<<<1, 32, 0, stream>>>(bound_partial, bound_blocks, bounds);
    k_morton<<<blocks_for(n), kThreads, 0, stream>>>(centroids, n, bounds, keys[0], values[0]);
    int cur = 0;
    for (int shift = 0; shift < 32; shift += kRadixBits) {
        k_radix_histogram<<<tiles, kThreads, 0, stream>>>(keys[cur], n, shift, counts, tiles);
        k_radix_scan<<<1, 1024, 0, stream>>>(counts, kRadix * tiles);
        k_radix_scatter<<<tiles, kThreads, 0, stream>>>(keys[cur], values[cur], n, shift, counts,
                                                        tiles, keys[1 - cur], values[1 - cur]);
        cur = 1 - cur;
    }
    // eight passes: the sorted arrays are back in the caller's buffers
    check(cudaMemsetAsync(parent, 0xff, sizeof(int32_t) * 2 * n, stream),
          "hierarchy export: clearing the parent links");
    if (n > 1) k_karras<<<blocks_for(n - 1), kThreads, 0, stream>>>(keys[cur], n, left, right, parent);
    return true;
}

}  // namespace nricp_b200
