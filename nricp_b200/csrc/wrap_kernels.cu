// The per-tick kernels of the device schedule.
//
// One tick advances every wrap of a batch by one unit of the schedule the
// reference's session runs (src/cuda/session.cu:404-576) -- a correspondence
// refresh, or one damped solve attempt with its candidate system -- and every
// kernel below serves all wraps at once: blockIdx.y is the wrap, and a wrap
// whose phase does not need a kernel leaves it immediately.  The decision
// kernel at the end of the tick is the only writer of the schedule's scalars,
// so the host never sits in the loop: it replays the tick (a CUDA graph) and
// polls one pinned flag.
//
// Reductions are fixed-order (per-block partials, then a fixed tree), so a
// wrap's result does not depend on which other wraps share its batch.
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

#include <cooperative_groups.h>

namespace nricp_b200 {

namespace cg = cooperative_groups;

namespace {

constexpr int kVertexThreads = 256;
constexpr int kNodeThreads = 256;   // 8 warps = 8 nodes per block
constexpr int kEdgeThreads = 128;
constexpr int kPcgThreads = 512;
constexpr int kStatsThreads = 512;

// Which branch of a tick handles a wrap: part 0 every wrap (one chain), 1 the
// wraps that started the tick in a solve, 2 the others.  The phase at the
// tick's start decides, so a wrap that one branch's decision moves on is not
// picked up by the other branch in the same tick.
__device__ inline bool in_part(const WrapControl& c, int part) {
    return part == 0 || (part == 1) == (c.tick_phase == kPhaseSolve);
}
__device__ inline int blocks_of_dev(long n, int threads) { return (int)((n + threads - 1) / threads); }

// Most wraps of a batch are smaller than the largest, and in any tick only
// some of them have work for a given kernel; a grid sized for the largest wrap
// times the wraps launches mostly blocks that return at once.  Instead a
// kernel's work is a list of virtual blocks -- block x of wrap y, exactly the
// blocks the full grid would run to some effect -- which a grid that fits on
// the device walks in order.  Each virtual block does the same work, with
// the same reductions and the same partial slots, as that block of the full
// grid, so results do not change.  need(w) gives the virtual blocks of wrap w
// (0: none this tick); body(wrap index, x) runs one.  The launch gives
// (wrap_count + 1) ints of dynamic shared memory.  kShared: the body uses
// shared memory, so the block meets at a barrier between virtual blocks;
// bodies without it let each warp go on to the next virtual block at once.
template <bool kShared, typename Need, typename Body>
__device__ __forceinline__ void over_virtual_blocks(const WrapDev* __restrict__ wraps, int wrap_count, Need need,
                                                    Body body) {
    extern __shared__ int first[];  // each wrap's first virtual block
    for (int i = threadIdx.x; i < wrap_count; i += blockDim.x) first[i + 1] = need(wraps[i]);
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scan by warp 0, 32 wraps at a time
        const int lane = threadIdx.x;
        int carry = 0;
        for (int base = 0; base < wrap_count; base += 32) {
            int x = base + lane < wrap_count ? first[base + lane + 1] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (base + lane < wrap_count) first[base + lane + 1] = carry + x;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) first[0] = 0;
    }
    __syncthreads();
    const int total = first[wrap_count];
    for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
        int lo = 0, hi = wrap_count - 1;  // the last wrap whose first block is <= vb
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (first[mid] <= vb) lo = mid; else hi = mid - 1;
        }
        body(lo, vb - first[lo]);
        if (kShared) __syncthreads();  // shared memory of one virtual block before the next
    }
}

__device__ inline bool refresh_like(int phase) {
    return phase == kPhaseTransfer || phase == kPhaseRefresh || phase == kPhaseFinal;
}
// Which state buffer the kernels of this tick evaluate: the candidate for a
// solve attempt, the freshly transferred state at a level start, else the
// accepted one.
__device__ inline int eval_buffer(const WrapControl& c) {
    return (c.phase == kPhaseSolve || c.phase == kPhaseTransfer) ? 1 - c.state : c.state;
}
__device__ inline bool has_candidate(const WrapControl& c) {
    return c.phase != kPhaseSolve || c.pcg_ok;
}
// Whether this tick evaluates the energy (everything but the final query).
__device__ inline bool computes_energy(const WrapControl& c) {
    return (c.phase == kPhaseTransfer || c.phase == kPhaseRefresh || c.phase == kPhaseSolve) &&
           has_candidate(c);
}
// Whether this tick assembles a system.  Route C's translation-only matrix
// does not depend on the state, so it is assembled once per refresh.
__device__ inline bool assembles(const WrapControl& c) {
    if (c.phase == kPhaseTransfer || c.phase == kPhaseRefresh) return true;
    return c.phase == kPhaseSolve && c.route == 0 && c.pcg_ok;
}

// ---- FP64 with every operation rounded on its own (host-identical) --------
__device__ inline double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double da(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ inline D3 rsub(D3 a, D3 b) { return {ds(a.x, b.x), ds(a.y, b.y), ds(a.z, b.z)}; }
__device__ inline D3 radd(D3 a, D3 b) { return {da(a.x, b.x), da(a.y, b.y), da(a.z, b.z)}; }
__device__ inline D3 rmul(D3 a, double s) { return {dm(a.x, s), dm(a.y, s), dm(a.z, s)}; }
__device__ inline double rdot(D3 a, D3 b) { return da(da(dm(a.x, b.x), dm(a.y, b.y)), dm(a.z, b.z)); }
__device__ inline D3 rcross(D3 a, D3 b) {
    return {ds(dm(a.y, b.z), dm(a.z, b.y)), ds(dm(a.z, b.x), dm(a.x, b.z)),
            ds(dm(a.x, b.y), dm(a.y, b.x))};
}
__device__ inline D3 rmat(const double* m, D3 v) {
    return {da(da(dm(m[0], v.x), dm(m[1], v.y)), dm(m[2], v.z)),
            da(da(dm(m[3], v.x), dm(m[4], v.y)), dm(m[5], v.z)),
            da(da(dm(m[6], v.x), dm(m[7], v.y)), dm(m[8], v.z))};
}

// ---- rotations (src/core/rotation.h, quaternion.h), FP64 -------------------
__device__ inline void mat_mul(const double* a, const double* b, double* out) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double sum = 0.0;
            for (int k = 0; k < 3; ++k) sum = da(sum, dm(a[r * 3 + k], b[k * 3 + c]));
            out[r * 3 + c] = sum;
        }
}
__device__ inline void skew(D3 w, double* m) {
    m[0] = 0.0; m[1] = -w.z; m[2] = w.y; m[3] = w.z; m[4] = 0.0; m[5] = -w.x;
    m[6] = -w.y; m[7] = w.x; m[8] = 0.0;
}
__device__ inline void exp_so3(D3 w, double* out) {  // rotation.h:29-47
    const double t2 = rdot(w, w);
    double h[9], h2[9];
    skew(w, h);
    mat_mul(h, h, h2);
    for (int i = 0; i < 9; ++i) out[i] = (i % 4 == 0) ? 1.0 : 0.0;
    if (t2 < 1e-24) {
        for (int i = 0; i < 9; ++i) out[i] = da(out[i], da(h[i], dm(0.5, h2[i])));
        return;
    }
    const double t = sqrt(t2);
    const double a = sin(t) / t;
    const double b = (1.0 - cos(t)) / t2;
    for (int i = 0; i < 9; ++i) out[i] = da(out[i], da(dm(a, h[i]), dm(b, h2[i])));
}
struct Quat { double w, x, y, z; };
__device__ inline Quat quat_from_matrix(const double* m) {  // quaternion.h:49-76
    const double trace = m[0] + m[4] + m[8];
    if (trace > 0.0) {
        const double s = sqrt(trace + 1.0) * 2.0;
        return {0.25 * s, (m[7] - m[5]) / s, (m[2] - m[6]) / s, (m[3] - m[1]) / s};
    }
    if (m[0] > m[4] && m[0] > m[8]) {
        const double s = sqrt(1.0 + m[0] - m[4] - m[8]) * 2.0;
        return {(m[7] - m[5]) / s, 0.25 * s, (m[1] + m[3]) / s, (m[2] + m[6]) / s};
    }
    if (m[4] > m[8]) {
        const double s = sqrt(1.0 + m[4] - m[0] - m[8]) * 2.0;
        return {(m[2] - m[6]) / s, (m[1] + m[3]) / s, 0.25 * s, (m[5] + m[7]) / s};
    }
    const double s = sqrt(1.0 + m[8] - m[0] - m[4]) * 2.0;
    return {(m[3] - m[1]) / s, (m[2] + m[6]) / s, (m[5] + m[7]) / s, 0.25 * s};
}
__device__ inline void matrix_from_quat(Quat q, double* m) {  // quaternion.h:78-94
    m[0] = 1.0 - 2.0 * (q.y * q.y + q.z * q.z);
    m[1] = 2.0 * (q.x * q.y - q.z * q.w);
    m[2] = 2.0 * (q.x * q.z + q.y * q.w);
    m[3] = 2.0 * (q.x * q.y + q.z * q.w);
    m[4] = 1.0 - 2.0 * (q.x * q.x + q.z * q.z);
    m[5] = 2.0 * (q.y * q.z - q.x * q.w);
    m[6] = 2.0 * (q.x * q.z - q.y * q.w);
    m[7] = 2.0 * (q.y * q.z + q.x * q.w);
    m[8] = 1.0 - 2.0 * (q.x * q.x + q.y * q.y);
}
__device__ inline D3 log_so3(const double* m) {  // rotation.h:51-63
    Quat q = quat_from_matrix(m);
    double len = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    if (len > 0.0) { q.w /= len; q.x /= len; q.y /= len; q.z /= len; }
    else { q = {1.0, 0.0, 0.0, 0.0}; }
    if (q.w < 0.0) { q.w = -q.w; q.x = -q.x; q.y = -q.y; q.z = -q.z; }
    const double l = sqrt(q.x * q.x + q.y * q.y + q.z * q.z);
    if (l < 1e-12) return {0.0, 0.0, 0.0};
    const double angle = 2.0 * atan2(l, q.w);
    return {q.x * (angle / l), q.y * (angle / l), q.z * (angle / l)};
}
__device__ inline void left_jacobian_inverse(D3 w, double* out) {  // rotation.h:71-105
    const double t2 = dot(w, w);
    double h[9], h2[9];
    skew(w, h);
    mat_mul(h, h, h2);
    if (t2 < 1e-12) {
        for (int i = 0; i < 9; ++i)
            out[i] = ((i % 4 == 0) ? 1.0 : 0.0) - 0.5 * h[i] + (1.0 / 12.0) * h2[i];
        return;
    }
    const double t = sqrt(t2);
    if (t > 3.14159265358979323846 - 1e-6) {
        for (int i = 0; i < 9; ++i) out[i] = ((i % 4 == 0) ? 1.0 : 0.0) - 0.5 * h[i];
        return;
    }
    const double second = 1.0 / t2 - (1.0 + cos(t)) / (2.0 * t * sin(t));
    for (int i = 0; i < 9; ++i) out[i] = ((i % 4 == 0) ? 1.0 : 0.0) - 0.5 * h[i] + second * h2[i];
}

// ---- reductions ------------------------------------------------------------
template <typename T>
__device__ inline T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Warp sums of N values at once, by recursive halving: at lane distance
// o = 16, 8, .., 1 each lane keeps half of its values (the upper half when
// its lane bit o is set) and adds its partner's copy of that half.  Each
// total is formed by the same additions as `warp_sum` of that value (x + y
// and y + x round alike), so the bits are the same, with ~N shuffles instead
// of 5N.  Afterwards this lane holds the totals of values
// [first, first + count) in v[0 .. count).
template <int N, int O = 16>
__device__ __forceinline__ void warp_sum_halving(float* v, int lane, int& first, int& count) {
    if constexpr (O >= 1) {
        constexpr int H = (N + 1) / 2;
        const bool upper = (lane & O) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const float lo = v[i];
            const float hi = i + H < N ? v[i + H] : 0.0f;
            v[i] = (upper ? hi : lo) + __shfl_xor_sync(0xffffffffu, upper ? lo : hi, O);
        }
        if (upper) {
            first += H;
            count = count > H ? count - H : 0;
        } else {
            count = count < H ? count : H;
        }
        warp_sum_halving<H, O / 2>(v, lane, first, count);
    }
}
// Block sum in a fixed order; every thread returns the total.
template <int kThreadsT>
__device__ inline double block_sum(double v, double* scratch) {
    v = warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double x = lane < kThreadsT / 32 ? scratch[lane] : 0.0;
        x = warp_sum(x);
        if (lane == 0) scratch[32] = x;
    }
    __syncthreads();
    return scratch[32];
}

// ---- symmetric 6x6 accumulation in the upper triangle ----------------------
// d[k] for (r, c), r <= c, row-major over the upper triangle.
__device__ inline int tri_index(int r, int c) { return r * 6 - r * (r - 1) / 2 + (c - r); }

// D += coef * [ |a|^2 I - a a^T, [a]x ; [a]x^T, I ]  (sum over the three rows
// of an offset residual whose node-local offset is `a`)
__device__ inline void add_offset_block(float* d, F3 a, float coef) {
    const float aa = dot(a, a);
    const float av[3] = {a.x, a.y, a.z};
    for (int r = 0; r < 3; ++r)
        for (int c = r; c < 3; ++c) d[tri_index(r, c)] += coef * ((r == c ? aa : 0.0f) - av[r] * av[c]);
    // [a]x = [[0,-az,ay],[az,0,-ax],[-ay,ax,0]] in rows 0-2, columns 3-5
    d[tri_index(0, 4)] += -coef * a.z; d[tri_index(0, 5)] += coef * a.y;
    d[tri_index(1, 3)] += coef * a.z;  d[tri_index(1, 5)] += -coef * a.x;
    d[tri_index(2, 3)] += -coef * a.y; d[tri_index(2, 4)] += coef * a.x;
    d[tri_index(3, 3)] += coef; d[tri_index(4, 4)] += coef; d[tri_index(5, 5)] += coef;
}
// D += coef * u u^T for a 6-vector u
__device__ inline void add_rank_one(float* d, const float* u, float coef) {
    for (int r = 0; r < 6; ++r)
        for (int c = r; c < 6; ++c) d[tri_index(r, c)] += coef * u[r] * u[c];
}

}  // namespace

// ---------------------------------------------------------------------------
// statistics (deform_ops.cu:135-182 / correspondence.cpp:82-94)
// ---------------------------------------------------------------------------
// The statistics pass at a tick's start (final_mode 0) also takes the tick's
// phase snapshot.
__global__ void k_stats(const WrapDev* __restrict__ wraps, int final_mode) {
    const WrapDev& w = wraps[blockIdx.y * gridDim.x + blockIdx.x];
    const WrapControl c = *w.control;
    if (!final_mode && threadIdx.x == 0) w.control->tick_phase = c.phase;
    CorrStats* target = nullptr;
    int level = -1;
    if (final_mode) {
        if (c.tick_phase != kPhaseFinal || c.phase != kPhaseFinal) return;
        target = w.final_stats;
    } else {
        if (c.stats_pending == 0) return;
        level = c.stats_pending - 1;
        target = w.level_stats + level;
    }
    __shared__ double scratch[33];
    __shared__ int hist[256];
    __shared__ unsigned long long prefix_s;
    __shared__ int rank_s;
    int counts[5] = {0, 0, 0, 0, 0};
    double sum = 0.0, maximum = 0.0;
    for (int v = threadIdx.x; v < w.V; v += blockDim.x) {
        const int code = w.corr_code[v];
        if (code >= 0 && code < 5) counts[code]++;
        if (code == 0) {
            const double d = w.corr_distance[v];
            sum += d;
            maximum = fmax(maximum, d);
        }
    }
    int totals[5];
    for (int k = 0; k < 5; ++k) totals[k] = (int)block_sum<kStatsThreads>((double)counts[k], scratch);
    const double total_sum = block_sum<kStatsThreads>(sum, scratch);
    // max via the same fixed tree on negated values is not needed: max is exact
    double m = maximum;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = 0.0;
        for (int i = 0; i < kStatsThreads / 32; ++i) mm = fmax(mm, scratch[i]);
        scratch[32] = mm;
    }
    __syncthreads();
    const double total_max = scratch[32];
    const int accepted = totals[0];
    // p95 = the floor(0.95 (n - 1))-th smallest accepted distance, found by a
    // radix select over the IEEE bits (non-negative doubles order like their
    // bit patterns).
    double p95 = 0.0;
    if (accepted > 0) {
        double pi = 0.95 * (double)(accepted - 1);
        if (pi > (double)(accepted - 1)) pi = (double)(accepted - 1);
        if (threadIdx.x == 0) { prefix_s = 0ull; rank_s = (int)pi; }
        __syncthreads();
        unsigned long long mask = 0ull;
        for (int shift = 56; shift >= 0; shift -= 8) {
            for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
            __syncthreads();
            const unsigned long long prefix = prefix_s;
            for (int v = threadIdx.x; v < w.V; v += blockDim.x) {
                if (w.corr_code[v] != 0) continue;
                const unsigned long long bits = (unsigned long long)__double_as_longlong(w.corr_distance[v]);
                if ((bits & mask) != prefix) continue;
                atomicAdd(&hist[(bits >> shift) & 255ull], 1);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int rank = rank_s;
                int digit = 0;
                for (; digit < 256; ++digit) {
                    if (rank < hist[digit]) break;
                    rank -= hist[digit];
                }
                if (digit > 255) digit = 255;
                rank_s = rank;
                prefix_s = prefix | ((unsigned long long)digit << shift);
            }
            mask |= 255ull << shift;
            __syncthreads();
        }
        p95 = __longlong_as_double((long long)prefix_s);
    }
    if (threadIdx.x == 0) {
        CorrStats s;
        s.total = totals[0] + totals[1] + totals[2] + totals[3] + totals[4];
        s.accepted = accepted;
        s.rejected_distance = totals[1];
        s.rejected_normal = totals[2];
        s.rejected_slope = totals[3];
        s.rejected_masked = totals[4];
        s.mean = accepted > 0 ? total_sum / accepted : 0.0;
        s.p95 = p95;
        s.max = accepted > 0 ? total_max : 0.0;
        *target = s;
        if (!final_mode) {
            w.records[level].correspondence_mean = s.mean;
            w.control->last_corr_mean = s.mean;
            w.control->stats_pending = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// node prologue: level warm start (deformation.cpp:141-203) and FP32 copies
// ---------------------------------------------------------------------------
__device__ __forceinline__ void k_prologue_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (!refresh_like(c.phase)) return;
    const LevelDev& L = w.levels[c.level];
    const int n = bx * blockDim.x + threadIdx.x;
    if (n >= L.node_count) return;
    double R[9];
    if (c.phase == kPhaseTransfer) {
        const LevelDev& from = w.levels[c.level - 1];
        const double* src_rot = w.rot[c.state];
        const double* src_trans = w.trans[c.state];
        const int count = L.transfer_counts[n];
        const int* nodes = L.transfer_nodes + n * 4;
        const double* weights = L.transfer_weights + n * 4;
        D3 t = {0.0, 0.0, 0.0};
        if (count > 0) {
            int heaviest = nodes[0];
            double hw = weights[0];
            for (int s = 1; s < count; ++s)
                if (weights[s] > hw) { hw = weights[s]; heaviest = nodes[s]; }
            const Quat ref = quat_from_matrix(src_rot + heaviest * 9);
            Quat b = {0.0, 0.0, 0.0, 0.0};
            D3 position = {0.0, 0.0, 0.0};
            const D3 g = load_d3(L.rest, n);
            for (int s = 0; s < count; ++s) {
                const int src = nodes[s];
                const double wt = weights[s];
                Quat q = quat_from_matrix(src_rot + src * 9);
                if (q.w * ref.w + q.x * ref.x + q.y * ref.y + q.z * ref.z < 0.0) {
                    q.w = -q.w; q.x = -q.x; q.y = -q.y; q.z = -q.z;
                }
                b.w += q.w * wt; b.x += q.x * wt; b.y += q.y * wt; b.z += q.z * wt;
                const D3 gs = load_d3(from.rest, src);
                const D3 applied = radd(radd(rmat(src_rot + src * 9, rsub(g, gs)), gs),
                                        load_d3(src_trans, src));
                position = radd(position, rmul(applied, wt));
            }
            const double len = sqrt(b.w * b.w + b.x * b.x + b.y * b.y + b.z * b.z);
            if (len > 1e-8) {
                const Quat nb = {b.w / len, b.x / len, b.y / len, b.z / len};
                matrix_from_quat(nb, R);
            } else {
                matrix_from_quat(ref, R);
            }
            t = rsub(position, g);
        } else {
            for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
        }
        double* dst = w.rot[1 - c.state] + n * 9;
        for (int i = 0; i < 9; ++i) dst[i] = R[i];
        store_d3(w.trans[1 - c.state], n, t);
    } else {
        const double* src = w.rot[c.state] + n * 9;
        for (int i = 0; i < 9; ++i) R[i] = src[i];
    }
    for (int i = 0; i < 9; ++i) w.rot32[n * 9 + i] = (float)R[i];
}

__global__ void k_prologue(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? (refresh_like(c.phase) ? blocks_of_dev(w.levels[c.level].node_count, 128) : 0) : 0;
        },
        [&](int wi, int bx) { k_prologue_body(wraps[wi], part, bx); });
}

// ---------------------------------------------------------------------------
// route C: Horn's closed-form rotation (local_global.cu:188-302), FP64
// ---------------------------------------------------------------------------
__device__ inline void horn_rotation(const double* S, double* R) {
    const double sxx = S[0], sxy = S[1], sxz = S[2], syx = S[3], syy = S[4], syz = S[5];
    const double szx = S[6], szy = S[7], szz = S[8];
    double a[4][4];
    a[0][0] = sxx + syy + szz; a[0][1] = syz - szy; a[0][2] = szx - sxz; a[0][3] = sxy - syx;
    a[1][1] = sxx - syy - szz; a[1][2] = sxy + syx; a[1][3] = szx + sxz;
    a[2][2] = -sxx + syy - szz; a[2][3] = syz + szy;
    a[3][3] = -sxx - syy + szz;
    for (int r = 1; r < 4; ++r)
        for (int c = 0; c < r; ++c) a[r][c] = a[c][r];
    double v[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) v[r][c] = r == c ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int r = 0; r < 4; ++r) {
            diag += a[r][r] * a[r][r];
            for (int c = r + 1; c < 4; ++c) off += a[r][c] * a[r][c];
        }
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < 3; ++p)
            for (int q = p + 1; q < 4; ++q) {
                if (a[p][q] == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double sign = theta >= 0.0 ? 1.0 : -1.0;
                const double t = sign / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0);
                const double sn = t * cs;
                for (int k = 0; k < 4; ++k) {
                    const double f = a[k][p], s2 = a[k][q];
                    a[k][p] = cs * f - sn * s2; a[k][q] = sn * f + cs * s2;
                }
                for (int k = 0; k < 4; ++k) {
                    const double f = a[p][k], s2 = a[q][k];
                    a[p][k] = cs * f - sn * s2; a[q][k] = sn * f + cs * s2;
                }
                for (int k = 0; k < 4; ++k) {
                    const double f = v[k][p], s2 = v[k][q];
                    v[k][p] = cs * f - sn * s2; v[k][q] = sn * f + cs * s2;
                }
            }
    }
    int best = 0;
    for (int i = 1; i < 4; ++i)
        if (a[i][i] > a[best][best]) best = i;
    const double qw = v[0][best], qx = v[1][best], qy = v[2][best], qz = v[3][best];
    const double len = sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
    if (!(len > 0.0)) {
        for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    const double w_ = qw / len, x = qx / len, y = qy / len, z = qz / len;
    R[0] = w_ * w_ + x * x - y * y - z * z; R[1] = 2.0 * (x * y - w_ * z); R[2] = 2.0 * (x * z + w_ * y);
    R[3] = 2.0 * (x * y + w_ * z); R[4] = w_ * w_ - x * x + y * y - z * z; R[5] = 2.0 * (y * z - w_ * x);
    R[6] = 2.0 * (x * z - w_ * y); R[7] = 2.0 * (y * z + w_ * x); R[8] = w_ * w_ - x * x - y * y + z * z;
}

constexpr double kRotationRelaxation = 0.2;  // local_global.cu:18

// The weighted rigid fit of point pairs (fit_rigid, deformation.cpp:86-139):
// weights clamped at zero, weighted centroids, the covariance
// sum w (p - cp)(q - cq)^T, the proper rotation that best maps the sources
// onto the targets, and t = cq - R cp.  The reference takes the rotation
// from an SVD with the reflection corrected; Horn's quaternion (the top
// eigenvector of the 4x4 matrix built from the covariance, Jacobi in FP64)
// is the same rotation.  One block, FP64 sums in a fixed order.
constexpr int kRigidThreads = 1024;
__global__ void __launch_bounds__(kRigidThreads) k_fit_rigid(const double* __restrict__ src,
                                                            const double* __restrict__ dst,
                                                            const double* __restrict__ weights, int n,
                                                            double* __restrict__ out) {
    __shared__ double scratch[33];
    double sums[7] = {0, 0, 0, 0, 0, 0, 0};  // w, w p, w q
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double w = fmax(0.0, weights[i]);
        sums[0] += w;
        for (int k = 0; k < 3; ++k) {
            sums[1 + k] += src[i * 3 + k] * w;
            sums[4 + k] += dst[i * 3 + k] * w;
        }
    }
    for (int k = 0; k < 7; ++k) sums[k] = block_sum<kRigidThreads>(sums[k], scratch);
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (!(sums[0] > 0.0)) {
        if (threadIdx.x == 0)
            for (int k = 0; k < 12; ++k) out[k] = k < 9 ? R[k] : 0.0;
        return;
    }
    const double cp[3] = {sums[1] / sums[0], sums[2] / sums[0], sums[3] / sums[0]};
    const double cq[3] = {sums[4] / sums[0], sums[5] / sums[0], sums[6] / sums[0]};
    double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double w = fmax(0.0, weights[i]);
        if (w == 0.0) continue;
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) S[r * 3 + q] += w * (src[i * 3 + r] - cp[r]) * (dst[i * 3 + q] - cq[q]);
    }
    for (int k = 0; k < 9; ++k) S[k] = block_sum<kRigidThreads>(S[k], scratch);
    if (threadIdx.x == 0) {
        horn_rotation(S, R);
        for (int k = 0; k < 9; ++k) out[k] = R[k];
        for (int r = 0; r < 3; ++r) out[9 + r] = cq[r] - (R[r * 3] * cp[0] + R[r * 3 + 1] * cp[1] + R[r * 3 + 2] * cp[2]);
    }
}

// Warp per node: the correlation of the influences that mention the node
// (bound vertices' data and landmark rows, edges it is the first endpoint of),
// Horn's rotation, and the under-relaxed update into the candidate buffer.
__device__ __forceinline__ void k_c_fit_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (c.phase != kPhaseSolve || c.route != 1) return;
    const LevelDev& L = w.levels[c.level];
    const int node = (bx * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (node >= L.node_count) return;
    const double* wt = w.weights[c.level];
    const double data_weight = wt[0] + wt[1];  // local_global.cu:546
    const double* T = w.trans[c.state];
    const D3 g = load_d3(L.rest, node);
    const D3 tn = load_d3(T, node);
    double S[9];
    for (int i = 0; i < 9; ++i) S[i] = 0.0;
    for (int i = L.gather_begin[node] + lane; i < L.gather_begin[node + 1]; i += 32) {
        const int entry = L.gather_entry[i];
        const int v = entry / kMaxSlots;
        const double own = L.bind_weights[entry];
        const D3 src = load_d3(w.tpl, v) - g;
        if (w.corr_code[v] == 0) {
            const D3 dst = load_d3(w.corr_point, v) - g - tn;
            const double s = data_weight * w.robust[v] * own;
            const double xs[3] = {src.x, src.y, src.z}, ys[3] = {dst.x, dst.y, dst.z};
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) S[r * 3 + q] += s * xs[r] * ys[q];
        }
        if (wt[4] > 0.0 && w.lm_flag[v]) {
            const D3 dst = load_d3(w.lm_target, v) - g - tn;
            const double s = wt[4] * own;
            const double xs[3] = {src.x, src.y, src.z}, ys[3] = {dst.x, dst.y, dst.z};
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) S[r * 3 + q] += s * xs[r] * ys[q];
        }
    }
    for (int i = L.node_edge_begin[node] + lane; i < L.node_edge_begin[node + 1]; i += 32) {
        const int e = L.node_edge_list[i];
        const int a = L.edges[e * 2], b = L.edges[e * 2 + 1];
        if (a != node) continue;
        const D3 gb = load_d3(L.rest, b);
        const D3 src = gb - g;
        const D3 dst = gb + load_d3(T, b) - g - tn;
        const double xs[3] = {src.x, src.y, src.z}, ys[3] = {dst.x, dst.y, dst.z};
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) S[r * 3 + q] += wt[2] * xs[r] * ys[q];
    }
    for (int i = 0; i < 9; ++i) S[i] = warp_sum(S[i]);
    if (lane == 0) {
        double fit[9], cur[9], curT[9], rel[9], step[9], out[9];
        horn_rotation(S, fit);
        for (int i = 0; i < 9; ++i) cur[i] = w.rot[c.state][node * 9 + i];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) curT[r * 3 + q] = cur[q * 3 + r];
        mat_mul(fit, curT, rel);
        const D3 omega = log_so3(rel);
        exp_so3(omega * kRotationRelaxation, step);
        mat_mul(step, cur, out);
        for (int i = 0; i < 9; ++i) w.rot[1 - c.state][node * 9 + i] = out[i];
        store_d3(w.trans[1 - c.state], node, tn);
    }
}

__global__ void k_c_fit(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? ((c.phase == kPhaseSolve && c.route == 1) ? blocks_of_dev(w.levels[c.level].node_count * 32, kNodeThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_c_fit_body(wraps[wi], part, bx); });
}

// Warp per node: the translation-only right-hand side with the fitted
// rotations (local_global.cu:317-438); the rotation half is exactly zero.
__device__ __forceinline__ void k_c_rhs_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (c.phase != kPhaseSolve || c.route != 1) return;
    const LevelDev& L = w.levels[c.level];
    const int node = (bx * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (node >= L.node_count) return;
    const double* wt = w.weights[c.level];
    const double* Rc = w.rot[1 - c.state];
    const double* Tc = w.trans[1 - c.state];
    double local[3] = {0.0, 0.0, 0.0};
    for (int i = L.gather_begin[node] + lane; i < L.gather_begin[node + 1]; i += 32) {
        const int entry = L.gather_entry[i];
        const int v = entry / kMaxSlots;
        const double own = L.bind_weights[entry];
        const D3 p = load_d3(w.tpl, v);
        D3 deformed = {0.0, 0.0, 0.0};
        const int count = L.bind_counts[v];
        for (int s = 0; s < count; ++s) {
            const int j = L.bind_nodes[v * kMaxSlots + s];
            const double ws = L.bind_weights[v * kMaxSlots + s];
            const D3 gj = load_d3(L.rest, j);
            deformed = deformed + (mul3(Rc + j * 9, p - gj) + gj + load_d3(Tc, j)) * ws;
        }
        if (w.corr_code[v] == 0) {
            const D3 off = deformed - load_d3(w.corr_point, v);
            const double u = w.robust[v];
            if (wt[0] > 0.0) {
                const double s = wt[0] * u * own;
                local[0] -= s * off.x; local[1] -= s * off.y; local[2] -= s * off.z;
            }
            if (wt[1] > 0.0) {
                const D3 n = load_d3(w.corr_normal, v);
                const double s = wt[1] * u * own * dot(n, off);
                local[0] -= s * n.x; local[1] -= s * n.y; local[2] -= s * n.z;
            }
        }
        if (wt[4] > 0.0 && w.lm_flag[v]) {
            const D3 o = deformed - load_d3(w.lm_target, v);
            const double s = wt[4] * own;
            local[0] -= s * o.x; local[1] -= s * o.y; local[2] -= s * o.z;
        }
    }
    for (int i = L.node_edge_begin[node] + lane; i < L.node_edge_begin[node + 1]; i += 32) {
        const int e = L.node_edge_list[i];
        const int a = L.edges[e * 2], b = L.edges[e * 2 + 1];
        const D3 ga = load_d3(L.rest, a), gb = load_d3(L.rest, b);
        const D3 diff = mul3(Rc + a * 9, gb - ga) + ga + load_d3(Tc, a) - gb - load_d3(Tc, b);
        const double sign = a == node ? 1.0 : -1.0;
        local[0] -= sign * wt[2] * diff.x;
        local[1] -= sign * wt[2] * diff.y;
        local[2] -= sign * wt[2] * diff.z;
    }
    for (int i = 0; i < 3; ++i) local[i] = warp_sum(local[i]);
    if (lane == 0) {
        const D3 t = load_d3(Tc, node);
        float* r = w.rhs[c.system] + node * 6;
        r[0] = r[1] = r[2] = 0.0f;
        r[3] = (float)(local[0] - wt[3] * t.x);
        r[4] = (float)(local[1] - wt[3] * t.y);
        r[5] = (float)(local[2] - wt[3] * t.z);
    }
}

__global__ void k_c_rhs(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? ((c.phase == kPhaseSolve && c.route == 1) ? blocks_of_dev(w.levels[c.level].node_count * 32, kNodeThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_c_rhs_body(wraps[wi], part, bx); });
}

// ---------------------------------------------------------------------------
// the damped solve: block-Jacobi PCG in one CTA per wrap (pcg_solver.cu:15-241)
// FP32 blocks and matvec, FP64 solution / residual / dots.
// ---------------------------------------------------------------------------
__device__ inline bool cholesky6(float* a) {
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c <= r; ++c) {
            float sum = a[r * 6 + c];
            for (int k = 0; k < c; ++k) sum -= a[r * 6 + k] * a[c * 6 + k];
            if (r == c) {
                if (!(sum > 0.0f)) return false;
                a[r * 6 + c] = sqrtf(sum);
            } else {
                a[r * 6 + c] = sum / a[c * 6 + c];
            }
        }
    return true;
}
__device__ inline void solve6(const float* l, const double* rhs, double* x) {
    float y[6];
    for (int r = 0; r < 6; ++r) {
        float s = (float)rhs[r];
        for (int k = 0; k < r; ++k) s -= l[r * 6 + k] * y[k];
        y[r] = s / l[r * 6 + r];
    }
    float z[6];
    for (int r = 5; r >= 0; --r) {
        float s = y[r];
        for (int k = r + 1; k < 6; ++k) s -= l[k * 6 + r] * z[k];
        z[r] = s / l[r * 6 + r];
    }
    for (int r = 0; r < 6; ++r) x[r] = z[r];
}

// ---- the solve's partition and shared-memory layout ------------------------
//
// Rows are grouped into segments of kSegNodes nodes (24 rows: one pass of a
// warp; 4-node segments balance the warps better than 8-node ones, 0.90 s
// against 0.93 s per 64-wrap batch, and 16-node ones are slower).  A segment is
// the unit of ownership and of reduction: one warp forms the segment's FP64
// partial dot products in a fixed lane order, and the cluster sums the
// segments' partials in a fixed order.  A CTA owns a contiguous run of
// segments, so the cluster size only decides which CTA computes which
// segment, never the order of any sum: a wrap's solve is bit-identical for
// every cluster size, and with it alone and in any batch.
constexpr int kSegNodes = 4;

// The solve's reductions -- the dot products, the residual norm, the Krylov
// scalars and the x and r vectors -- are FP64.  A build with
// NRICP_FP32_REDUCTIONS defined rounds every one of those operations to FP32
// instead (each FP64 result of a sum or product of FP32 values rounded to
// FP32 is the correctly rounded FP32 result): a variant for measuring what
// the FP64 reductions buy, never the shipped library.
#ifdef NRICP_FP32_REDUCTIONS
__device__ __forceinline__ double rnd(double x) { return (double)__double2float_rn(x); }
#else
__device__ __forceinline__ double rnd(double x) { return x; }
#endif
__device__ __forceinline__ double warp_sum_rnd(double v) {
    for (int o = 16; o > 0; o >>= 1) v = rnd(v + __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
constexpr int kPcgWarps = kPcgThreads / 32;
constexpr int kPcgOwnFloats = 78;  // per owned node: X, R (2 x 6 FP64) + Minv 36 + P, S, W 18
constexpr int kPcgMaxSmemBytes = 225 * 1024;

__host__ __device__ inline int pcg_segments(int nodes) { return (nodes + kSegNodes - 1) / kSegNodes; }
// FP64 slots for the segments' three partials, padded to 16 bytes
__host__ __device__ inline int pcg_slot_doubles(int nodes) { return (3 * pcg_segments(nodes) + 1) & ~1; }

// Owned-node capacity of one CTA when `ranks` CTAs share the solve.
__host__ __device__ inline int pcg_owned_capacity(int nodes, int ranks) {
    return (pcg_segments(nodes) + ranks - 1) / ranks * kSegNodes;
}

// Placement for one wrap within a shared-memory budget: the segment slots
// always, then the all-node direction copy U if it fits (the matvec reads it
// ~10 times per row), then the owned rows' arrays if they fit.  Whatever does
// not fit lives in the wrap's global scratch; the arithmetic is the same.
struct PcgPlacement {
    bool u_shared, own_shared;
    int floats;  // shared floats this wrap uses
};
__host__ __device__ inline PcgPlacement pcg_place(int nodes, int ranks, int budget_floats) {
    PcgPlacement p;
    int used = pcg_slot_doubles(nodes) * 2;  // 3 FP64 partials per segment
    const int u = (nodes * 6 + 3) & ~3;
    const int own = pcg_owned_capacity(nodes, ranks) * kPcgOwnFloats;
    p.u_shared = used + u <= budget_floats;
    if (p.u_shared) used += u;
    p.own_shared = used + own <= budget_floats;
    if (p.own_shared) used += own;
    p.floats = used;
    return p;
}

// Inverse of a 6x6 SPD block from its Cholesky factor L (lower): L^-T L^-1.
__device__ inline void cholesky_inverse6(const float* l, float* inv) {
    float li[36];
    for (int i = 0; i < 36; ++i) li[i] = 0.0f;
    for (int c = 0; c < 6; ++c) {
        li[c * 6 + c] = 1.0f / l[c * 6 + c];
        for (int r = c + 1; r < 6; ++r) {
            float s = 0.0f;
            for (int k = c; k < r; ++k) s -= l[r * 6 + k] * li[k * 6 + c];
            li[r * 6 + c] = s / l[r * 6 + r];
        }
    }
    for (int r = 0; r < 6; ++r)
        for (int q = 0; q < 6; ++q) {
            float s = 0.0f;
            for (int k = r > q ? r : q; k < 6; ++k) s += li[k * 6 + r] * li[k * 6 + q];
            inv[r * 6 + q] = s;
        }
}

__device__ inline float dot6(const float* a, const float* b) {
    const float2* a2 = reinterpret_cast<const float2*>(a);
    const float2* b2 = reinterpret_cast<const float2*>(b);
    const float2 a0 = a2[0], a1 = a2[1], a3 = a2[2];
    const float2 b0 = b2[0], b1 = b2[1], b3 = b2[2];
    float y = a0.x * b0.x;
    y += a0.y * b0.y;
    y += a1.x * b1.x;
    y += a1.y * b1.y;
    y += a3.x * b3.x;
    y += a3.y * b3.y;
    return y;
}

// The damped solve (pcg_solver.cu:15-241): (A + lambda diag-scale) x = b,
// x0 = 0, block-Jacobi preconditioner from the Cholesky factor of each damped
// 6x6 diagonal block (with the reference's jitter retry), stop at
// |r| / |b| <= tolerance or after the iteration cap.  One thread-block
// cluster per wrap (blockIdx.y), any cluster size.
//
// The recurrence is the single-reduction form of preconditioned CG
// (Chronopoulos & Gear, 1989): with u = M^-1 r and w = A u, the three inner
// products (r,u), (w,u), (r,r) of an iteration are formed together, so an
// iteration needs one exchange of partial sums and one exchange of u:
//
//   gamma = (r,u), delta = (w,u); beta = gamma / gamma_prev;
//   alpha = gamma / (delta - beta gamma / alpha_prev)   (beta = 0 first);
//   p = u + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s.
//
// FP32 blocks, matvec, p, s, u and w; FP64 x, r, the inner products and the
// scalars.  Each CTA writes its slice of u once into its own shared copy and
// then copies the slice, 16 bytes at a time, into every other CTA's copy
// through distributed shared memory, so the matvec reads u locally and its
// only L2 traffic is the blocks (stored in row order).  Two hardware cluster
// barriers per iteration; nothing spins.
__global__ void __launch_bounds__(kPcgThreads) k_pcg(const WrapDev* __restrict__ wraps,
                                                     const int* __restrict__ index,
                                                     int budget_floats) {
    cg::cluster_group cluster = cg::this_cluster();
    const int slot = index ? index[blockIdx.y] : (int)blockIdx.y;
    if (slot < 0) return;  // an empty entry of a class launch; uniform across the cluster
    const WrapDev& w = wraps[slot];
    const WrapControl c = *w.control;
    if (c.tick_phase != kPhaseSolve || c.phase != kPhaseSolve) return;  // uniform across the cluster
    const LevelDev& L = w.levels[c.level];
    const int N = L.node_count;
    const int rank = (int)cluster.block_rank();
    const int ranks = (int)cluster.num_blocks();
    const int segs = pcg_segments(N);
    const int cap = pcg_owned_capacity(N, ranks);
    const int seg_per = cap / kSegNodes;
    const int s0 = min(segs, rank * seg_per);
    const int s1 = min(segs, s0 + seg_per);
    const int n0 = s0 * kSegNodes;
    const int n1 = min(N, s1 * kSegNodes);
    const int own = n1 > n0 ? n1 - n0 : 0;
    const int rows = own * 6;
    const PcgPlacement place = pcg_place(N, ranks, budget_floats);

    extern __shared__ float4 dynamic_shared[];
    double* slots = reinterpret_cast<double*>(dynamic_shared);  // 3 per segment, every CTA
    float* cursor = reinterpret_cast<float*>(slots + pcg_slot_doubles(N));
    float* U;
    if (place.u_shared) {
        U = cursor;
        cursor += (N * 6 + 3) & ~3;
    } else {
        U = w.pcg_u;
    }
    double *X, *R;
    float *Minv, *P, *S, *Wv;
    if (place.own_shared) {
        X = reinterpret_cast<double*>(cursor);
        R = X + cap * 6;
        Minv = reinterpret_cast<float*>(R + cap * 6);
        P = Minv + cap * 36;
        S = P + cap * 6;
        Wv = S + cap * 6;
    } else {
        X = w.pcg_x + n0 * 6;
        R = w.pcg_r + n0 * 6;
        Minv = w.factor + n0 * 36;
        P = w.pcg_p + n0 * 6;
        S = w.pcg_s + n0 * 6;
        Wv = w.pcg_ap + n0 * 6;
    }
    const float* __restrict__ D = w.diag[c.system];
    const float* __restrict__ B = w.offdiag[c.system];
    const float* __restrict__ b = w.rhs[c.system];
    const int* __restrict__ row_begin = L.row_begin;
    const int2* __restrict__ entries = reinterpret_cast<const int2*>(L.row_entry);
    const float damping = (float)c.damping;
    const bool scaled = w.diagonal_damping != 0;
    const int max_iterations = w.pcg_max_iterations;
    const double tolerance = w.pcg_tolerance;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ double red[3][kPcgWarps];
    __shared__ double tot[3];

    // ---- damped diagonal blocks and their inverses (route A's damped():
    //      scale = max(D_rr, 1e-12)); Cholesky with the reference's jitter ----
    for (int m = threadIdx.x; m < own; m += blockDim.x) {
        const int n = n0 + m;
        float blk[36];
        for (int i = 0; i < 36; ++i) blk[i] = D[n * 36 + i];
        for (int r = 0; r < 6; ++r) blk[r * 7] += damping * (scaled ? fmaxf(blk[r * 7], 1e-12f) : 1.0f);
        float jitter = 0.0f;
        bool ok = false;
        for (int attempt = 0; attempt < 8 && !ok; ++attempt) {
            float cand[36];
            for (int i = 0; i < 36; ++i) cand[i] = blk[i];
            for (int r = 0; r < 6; ++r) cand[r * 7] += jitter;
            if (cholesky6(cand)) {
                cholesky_inverse6(cand, Minv + m * 36);
                ok = true;
            }
            jitter = jitter == 0.0f ? 1e-6f : jitter * 10.0f;
        }
        if (!ok)
            for (int i = 0; i < 36; ++i) Minv[m * 36 + i] = (i % 7 == 0) ? 1.0f : 0.0f;
    }
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        X[i] = 0.0;
        R[i] = (double)b[n0 * 6 + i];
        P[i] = 0.0f;
        S[i] = 0.0f;
    }
    __syncthreads();

    // u = M^-1 r for the owned rows into this CTA's copy, then the slice into
    // every other CTA's copy (16-byte stores; the slice starts on a segment,
    // so at a multiple of 96 bytes)
    auto precondition_and_share = [&]() {
        for (int i = threadIdx.x; i < rows; i += blockDim.x) {
            const int m = i / 6, r = i - m * 6;
            const float* mi = Minv + m * 36 + r * 6;
            float z = 0.0f;
            for (int q = 0; q < 6; ++q) z += mi[q] * (float)R[m * 6 + q];
            U[n0 * 6 + i] = z;
        }
        if (place.u_shared && ranks > 1) {
            __syncthreads();
            const float4* src = reinterpret_cast<const float4*>(U + n0 * 6);
            const int vec = rows / 4;  // rows = 6 * own, own a multiple of 4 except at the end
            for (int q = 1; q < ranks; ++q) {
                const int dst_rank = (rank + q) % ranks;
                float4* dst = reinterpret_cast<float4*>(cluster.map_shared_rank(U, dst_rank) + n0 * 6);
                for (int k = threadIdx.x; k < vec; k += blockDim.x) dst[k] = src[k];
                float* dst_tail = cluster.map_shared_rank(U, dst_rank) + n0 * 6;
                for (int k = vec * 4 + threadIdx.x; k < rows; k += blockDim.x) dst_tail[k] = U[n0 * 6 + k];
            }
        }
        if (!place.u_shared) __threadfence();  // the global copy: visible device-wide first
    };
    precondition_and_share();
    cluster.sync();

    double gamma_prev = 0.0, alpha_prev = 0.0, bnorm = 0.0, residual = 0.0;
    int iterations = 0;
    bool converged = false;
    for (int it = 0;; ++it) {
        // ---- w = A u for the owned rows; per-segment partials of (r,u), (w,u), (r,r) ----
        for (int sl = warp; sl < s1 - s0; sl += kPcgWarps) {
            const int seg = s0 + sl;
            const int sn0 = seg * kSegNodes;
            const int seg_rows = (min(N, sn0 + kSegNodes) - sn0) * 6;
            double g = 0.0, d = 0.0, rr = 0.0;
            for (int k = lane; k < seg_rows; k += 32) {
                const int n = sn0 + k / 6, r = k % 6;
                const int i = (sn0 - n0) * 6 + k;
                const float* drow = D + n * 36 + r * 6;
                const float* un = U + n * 6;
                const float dd = drow[r] + damping * (scaled ? fmaxf(drow[r], 1e-12f) : 1.0f);
                float y = 0.0f;
                for (int q = 0; q < 6; ++q) y += (q == r ? dd : drow[q]) * un[q];
                const int e1 = row_begin[n + 1];
                int e = row_begin[n];
                for (; e + 4 <= e1; e += 4) {
                    int nb[4];
                    for (int u = 0; u < 4; ++u) nb[u] = entries[e + u].y;
                    float part[4];
                    for (int u = 0; u < 4; ++u) part[u] = dot6(B + (long)(e + u) * 36 + r * 6, U + nb[u] * 6);
                    for (int u = 0; u < 4; ++u) y += part[u];
                }
                for (; e < e1; ++e) y += dot6(B + (long)e * 36 + r * 6, U + entries[e].y * 6);
                Wv[i] = y;
                const double ui = (double)un[r];
                const double ri = R[i];
                g = rnd(g + rnd(ri * ui));
                d = rnd(d + rnd((double)y * ui));
                rr = rnd(rr + rnd(ri * ri));
            }
            g = warp_sum_rnd(g);
            d = warp_sum_rnd(d);
            rr = warp_sum_rnd(rr);
            if (lane < ranks) {  // lane q stores the partials in CTA q's slots
                double* dst = cluster.map_shared_rank(slots, lane) + 3 * seg;
                dst[0] = g;
                dst[1] = d;
                dst[2] = rr;
            }
        }
        cluster.sync();
        // ---- totals over every segment, in one fixed order in every CTA ----
        {
            double g = 0.0, d = 0.0, rr = 0.0;
            for (int sg = threadIdx.x; sg < segs; sg += blockDim.x) {
                g = rnd(g + slots[3 * sg]);
                d = rnd(d + slots[3 * sg + 1]);
                rr = rnd(rr + slots[3 * sg + 2]);
            }
            g = warp_sum_rnd(g);
            d = warp_sum_rnd(d);
            rr = warp_sum_rnd(rr);
            if (lane == 0) { red[0][warp] = g; red[1][warp] = d; red[2][warp] = rr; }
            __syncthreads();
            if (warp == 0) {
                for (int k = 0; k < 3; ++k) {
                    double v = lane < kPcgWarps ? red[k][lane] : 0.0;
                    v = warp_sum_rnd(v);
                    if (lane == 0) tot[k] = v;
                }
            }
            __syncthreads();
        }
        const double gamma = tot[0], delta = tot[1], rr_total = tot[2];
        if (it == 0) {
            bnorm = rnd(sqrt(rr_total));
            if (!(bnorm > 0.0)) { converged = true; residual = 0.0; break; }
        }
        residual = rnd(rnd(sqrt(rr_total)) / bnorm);
        if (residual <= tolerance) { converged = true; break; }
        if (it >= max_iterations) break;
        const double beta = it == 0 ? 0.0 : rnd(gamma / gamma_prev);
        const double denominator = it == 0 ? delta : rnd(delta - rnd(rnd(beta * gamma) / alpha_prev));
        if (!(fabs(denominator) > 1e-300)) break;
        const double alpha = rnd(gamma / denominator);
        gamma_prev = gamma;
        alpha_prev = alpha;
        // ---- p, s, x, r for the owned rows; then u = M^-1 r, shared ----
        for (int i = threadIdx.x; i < rows; i += blockDim.x) {
            const float pn = (float)((double)U[n0 * 6 + i] + rnd(beta * (double)P[i]));
            const float sn = (float)((double)Wv[i] + rnd(beta * (double)S[i]));
            P[i] = pn;
            S[i] = sn;
            X[i] = rnd(X[i] + rnd(alpha * (double)pn));
            R[i] = rnd(R[i] - rnd(alpha * (double)sn));
        }
        __syncthreads();
        precondition_and_share();
        cluster.sync();
        iterations = it + 1;
    }
    if (rank == 0 && threadIdx.x == 0) {
        w.control->pcg_ok = converged ? 1 : 0;
        w.control->pcg_iterations = iterations;
        w.control->pcg_residual = residual;
    }
    if (converged) {
        // candidate = retract(accepted, delta): R <- exp([w]) R, t <- t + u
        // (deformation.cpp:19-32).  Route C's rotation half is zero and its
        // rotations were already fitted into the candidate buffer.
        for (int m = threadIdx.x; m < own; m += blockDim.x) {
            const int n = n0 + m;
            const double* x = X + m * 6;
            const D3 tcur = load_d3(w.trans[c.state], n);
            store_d3(w.trans[1 - c.state], n, {tcur.x + x[3], tcur.y + x[4], tcur.z + x[5]});
            double out[9];
            if (c.route == 0) {
                double e[9];
                exp_so3({x[0], x[1], x[2]}, e);
                mat_mul(e, w.rot[c.state] + n * 9, out);
                for (int i = 0; i < 9; ++i) w.rot[1 - c.state][n * 9 + i] = out[i];
            } else {
                for (int i = 0; i < 9; ++i) out[i] = w.rot[1 - c.state][n * 9 + i];
            }
            for (int i = 0; i < 9; ++i) w.rot32[n * 9 + i] = (float)out[i];
            for (int k = 0; k < 6; ++k) w.delta[n * 6 + k] = x[k];
        }
    }
    // no CTA may exit while another can still write into its shared memory
    cluster.sync();
}

// ---------------------------------------------------------------------------
// deformation evaluation (deformation.cpp:55-68) and the deformed template's
// vertex normals (mesh.cpp:71-88)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void k_evaluate_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (c.phase == kPhaseDone || !has_candidate(c)) return;
    const int v = bx * blockDim.x + threadIdx.x;
    if (v >= w.V) return;
    const LevelDev& L = w.levels[c.level];
    const int buf = eval_buffer(c);
    const double* R = w.rot[buf];
    const double* T = w.trans[buf];
    const D3 p = load_d3(w.tpl, v);
    D3 sum = {0.0, 0.0, 0.0};
    const int count = L.bind_counts[v];
    for (int s = 0; s < count; ++s) {
        const int j = L.bind_nodes[v * kMaxSlots + s];
        const double wt = L.bind_weights[v * kMaxSlots + s];
        const D3 g = load_d3(L.rest, j);
        const D3 applied = radd(radd(rmat(R + j * 9, rsub(p, g)), g), load_d3(T, j));
        sum = radd(sum, rmul(applied, wt));
    }
    if (count == 0) sum = p;
    store_d3(w.deformed, v, sum);
    w.deformed32[v] = make_float4((float)sum.x, (float)sum.y, (float)sum.z, 0.0f);
}

__global__ void k_evaluate(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? ((c.phase != kPhaseDone && has_candidate(c)) ? blocks_of_dev(w.V, kVertexThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_evaluate_body(wraps[wi], part, bx); });
}

__device__ __forceinline__ void k_normals_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (!refresh_like(c.phase)) return;
    const int v = bx * blockDim.x + threadIdx.x;
    if (v >= w.V) return;
    D3 n = {0.0, 0.0, 0.0};
    for (int i = w.vf_begin[v]; i < w.vf_begin[v + 1]; ++i) {
        const int32_t* f = w.tpl_faces + (long)w.vf_faces[i] * 3;
        const D3 a = load_d3(w.deformed, f[0]);
        const D3 b = load_d3(w.deformed, f[1]);
        const D3 cc = load_d3(w.deformed, f[2]);
        n = radd(n, rcross(rsub(b, a), rsub(cc, a)));
    }
    const double len = __dsqrt_rn(rdot(n, n));
    if (len > 0.0) n = {__ddiv_rn(n.x, len), __ddiv_rn(n.y, len), __ddiv_rn(n.z, len)};
    else n = {0.0, 0.0, 0.0};
    store_d3(w.qnormals, v, n);
}

__global__ void k_normals(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? (refresh_like(c.phase) ? blocks_of_dev(w.V, kVertexThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_normals_body(wraps[wi], part, bx); });
}

// ---------------------------------------------------------------------------
// per-vertex residuals, the data and landmark energies (FP64), and the FP32
// residual records the assembly reads (fused_assembly.cpp:185-216, 262-280)
// ---------------------------------------------------------------------------
// The node-local offset R (p_v - g_node) of vertex v bound to `node`, FP32.
__device__ inline F3 node_offset32(const WrapDev& w, const LevelDev& L, int node, int v) {
    const D3 p = load_d3(w.tpl, v) - load_d3(L.rest, node);
    return mul3f(w.rot32 + node * 9, {(float)p.x, (float)p.y, (float)p.z});
}

__device__ __forceinline__ void k_residual_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (!computes_energy(c)) return;
    if ((long)bx * blockDim.x >= w.V) return;
    const int v = bx * blockDim.x + threadIdx.x;
    const double* wt = w.weights[c.level];
    const LevelDev& L = w.levels[c.level];
    double e_p2p = 0.0, e_plane = 0.0, e_lm = 0.0;
    if (v < w.V) {
        float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0, r2 = r0;
        const bool bound = L.bind_counts[v] > 0;
        const D3 q = load_d3(w.deformed, v);
        if (bound && w.corr_code[v] == 0) {
            const D3 y = load_d3(w.corr_point, v);
            const D3 o = rsub(q, y);
            const double u = fmax(0.0, w.robust[v]);
            const D3 n = load_d3(w.corr_normal, v);
            if (wt[0] > 0.0) {
                const double s = sqrt(wt[0] * u);
                const D3 so = rmul(o, s);
                e_p2p = da(da(dm(so.x, so.x), dm(so.y, so.y)), dm(so.z, so.z));
                r0 = make_float4((float)o.x, (float)o.y, (float)o.z, (float)(wt[0] * u));
            } else {
                r0 = make_float4((float)o.x, (float)o.y, (float)o.z, 0.0f);
            }
            if (wt[1] > 0.0) {
                const double s = sqrt(wt[1] * u);
                const double value = dm(s, rdot(n, o));
                e_plane = dm(value, value);
                r1 = make_float4((float)n.x, (float)n.y, (float)n.z, (float)(wt[1] * u));
            }
        }
        if (bound && wt[4] > 0.0 && w.lm_flag[v]) {
            const D3 o = rsub(q, load_d3(w.lm_target, v));
            const double s = sqrt(wt[4]);
            const D3 so = rmul(o, s);
            e_lm = da(da(dm(so.x, so.x), dm(so.y, so.y)), dm(so.z, so.z));
            r2 = make_float4((float)o.x, (float)o.y, (float)o.z, (float)wt[4]);
        }
        w.residual32[v] = r0;
        w.resid_aux32[v] = r1;
        w.lm_resid32[v] = r2;
        // each binding's offset, once for the node and pair assembly that follow
        if (bound && assembles(c))
            for (int k = 0; k < L.bind_counts[v]; ++k) {
                const int node = L.bind_nodes[v * kMaxSlots + k];
                if (node < 0) continue;
                const F3 a = node_offset32(w, L, node, v);
                w.offsets32[v * kMaxSlots + k] = make_float4(a.x, a.y, a.z, 0.0f);
            }
    }
    __shared__ double scratch[33];
    const double s0 = block_sum<kVertexThreads>(e_p2p, scratch);
    const double s1 = block_sum<kVertexThreads>(e_plane, scratch);
    const double s4 = block_sum<kVertexThreads>(e_lm, scratch);
    if (threadIdx.x == 0) {
        double* p = w.partials + (long)bx * kPartialStride;
        p[0] = s0; p[1] = s1; p[2] = s4;
    }
}

__global__ void __launch_bounds__(kVertexThreads) k_residual(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<true>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? (computes_energy(c) ? blocks_of_dev(w.V, kVertexThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_residual_body(wraps[wi], part, bx); });
}

// ---------------------------------------------------------------------------
// Gauss-Newton blocks: warp per node for the diagonal block and the
// right-hand side (data, landmark, incident smoothness edges, anchor), thread
// per node pair for the cross blocks of shared vertices, thread per edge for
// the smoothness blocks.  Closed forms of sum_rows J^T J for an offset
// residual replace the reference's row-by-row outer products.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void k_node_assemble_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (!computes_energy(c)) return;
    const bool build = assembles(c);
    const LevelDev& L = w.levels[c.level];
    if ((long)bx * (kNodeThreads / 32) >= L.node_count) return;
    const int node = (bx * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const double* wt = w.weights[c.level];
    const int buf = eval_buffer(c);
    const int next = 1 - c.system;
    float d[21], g[6];
    for (int i = 0; i < 21; ++i) d[i] = 0.0f;
    for (int i = 0; i < 6; ++i) g[i] = 0.0f;
    double e_anchor = 0.0;
    if (node < L.node_count) {
        if (build) {
            for (int i = L.gather_begin[node] + lane; i < L.gather_begin[node + 1]; i += 32) {
                const int entry = L.gather_entry[i];
                const int v = entry / kMaxSlots;
                const float wgt = (float)L.bind_weights[entry];
                const float4 a4 = w.offsets32[entry];
                const F3 a = {a4.x, a4.y, a4.z};
                const float4 r0 = w.residual32[v];
                const float4 r1 = w.resid_aux32[v];
                const float4 r2 = w.lm_resid32[v];
                if (r0.w > 0.0f) {  // point to point
                    const F3 o = {r0.x, r0.y, r0.z};
                    add_offset_block(d, a, r0.w * wgt * wgt);
                    const F3 ao = cross(a, o);
                    const float s = r0.w * wgt;
                    g[0] -= s * ao.x; g[1] -= s * ao.y; g[2] -= s * ao.z;
                    g[3] -= s * o.x; g[4] -= s * o.y; g[5] -= s * o.z;
                }
                if (r1.w > 0.0f) {  // point to plane
                    const F3 n = {r1.x, r1.y, r1.z};
                    const F3 an = cross(a, n);
                    const float u[6] = {an.x, an.y, an.z, n.x, n.y, n.z};
                    add_rank_one(d, u, r1.w * wgt * wgt);
                    const float pv = dot(n, F3{r0.x, r0.y, r0.z});
                    const float s = r1.w * wgt * pv;
                    for (int k = 0; k < 6; ++k) g[k] -= s * u[k];
                }
                if (r2.w > 0.0f) {  // landmark
                    const F3 o = {r2.x, r2.y, r2.z};
                    add_offset_block(d, a, r2.w * wgt * wgt);
                    const F3 ao = cross(a, o);
                    const float s = r2.w * wgt;
                    g[0] -= s * ao.x; g[1] -= s * ao.y; g[2] -= s * ao.z;
                    g[3] -= s * o.x; g[4] -= s * o.y; g[5] -= s * o.z;
                }
            }
            if (wt[2] > 0.0) {
                const float ws = (float)wt[2];
                const double* R = w.rot[buf];
                const double* T = w.trans[buf];
                for (int i = L.node_edge_begin[node] + lane; i < L.node_edge_begin[node + 1]; i += 32) {
                    const int e = L.node_edge_list[i];
                    const int a = L.edges[e * 2], b = L.edges[e * 2 + 1];
                    const D3 ga = load_d3(L.rest, a), gb = load_d3(L.rest, b);
                    const D3 gd = gb - ga;
                    const D3 diff = radd(radd(rmat(R + a * 9, gd), ga), load_d3(T, a)) -
                                    (gb + load_d3(T, b));
                    const F3 dv = {(float)diff.x, (float)diff.y, (float)diff.z};
                    if (a == node) {
                        const F3 cv = mul3f(w.rot32 + a * 9, {(float)gd.x, (float)gd.y, (float)gd.z});
                        add_offset_block(d, cv, ws);
                        const F3 cd = cross(cv, dv);
                        g[0] -= ws * cd.x; g[1] -= ws * cd.y; g[2] -= ws * cd.z;
                        g[3] -= ws * dv.x; g[4] -= ws * dv.y; g[5] -= ws * dv.z;
                    } else {
                        d[tri_index(3, 3)] += ws; d[tri_index(4, 4)] += ws; d[tri_index(5, 5)] += ws;
                        g[3] += ws * dv.x; g[4] += ws * dv.y; g[5] += ws * dv.z;
                    }
                }
            }
        }
        if (lane == 0 && wt[3] > 0.0) {  // anchor (energy.cpp:239-271)
            const double* R = w.rot[buf] + node * 9;
            const D3 om = log_so3(R);
            const D3 t = load_d3(w.trans[buf], node);
            const double sc = sqrt(wt[3]);
            const double vals[6] = {sc * om.x, sc * om.y, sc * om.z, sc * t.x, sc * t.y, sc * t.z};
            for (int k = 0; k < 6; ++k) e_anchor += vals[k] * vals[k];
            if (build) {
                double J[9];
                left_jacobian_inverse(om, J);
                for (int r = 0; r < 3; ++r)
                    for (int q = r; q < 3; ++q) {
                        double s = 0.0;
                        for (int k = 0; k < 3; ++k) s += J[k * 3 + r] * J[k * 3 + q];
                        d[tri_index(r, q)] += (float)(wt[3] * s);
                    }
                for (int r = 0; r < 3; ++r) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += J[k * 3 + r] * (k == 0 ? om.x : k == 1 ? om.y : om.z);
                    g[r] -= (float)(wt[3] * s);
                }
                d[tri_index(3, 3)] += (float)wt[3]; d[tri_index(4, 4)] += (float)wt[3];
                d[tri_index(5, 5)] += (float)wt[3];
                g[3] -= (float)(wt[3] * t.x); g[4] -= (float)(wt[3] * t.y); g[5] -= (float)(wt[3] * t.z);
            }
        }
        if (build) {
            // the 21 upper-triangle sums and the 6 of the rhs, spread over the
            // lanes; each lane stores what it holds
            float v[27];
            for (int i = 0; i < 21; ++i) v[i] = d[i];
            for (int i = 0; i < 6; ++i) v[21 + i] = g[i];
            int first = 0, count = 27;
            warp_sum_halving<27>(v, lane, first, count);
            if (count > 0) {
                float* D = w.diag[next] + node * 36;
                float* G = w.rhs[next] + node * 6;
                const bool restricted = c.route == 1;
                const int j = first;
                if (j < 21) {
                    int r = 0;
                    while (tri_index(r + 1, r + 1) <= j) ++r;  // row of upper-triangle entry j
                    const int q = j - tri_index(r, r) + r;
                    float value = v[0];
                    if (restricted && (r < 3 || q < 3)) value = (r == q) ? 1.0f : 0.0f;
                    D[r * 6 + q] = value;
                    D[q * 6 + r] = value;
                } else {
                    const int k = j - 21;
                    G[k] = (restricted && k < 3) ? 0.0f : v[0];
                }
            }
        }
    }
    // the node's anchor energy; the decision kernel sums them as a block sum
    // over this block's warps would (no block barrier here)
    if (lane == 0 && node < L.node_count) w.node_partials[node] = e_anchor;
}

__global__ void __launch_bounds__(kNodeThreads, 3) k_node_assemble(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? (computes_energy(c) ? blocks_of_dev(w.levels[c.level].node_count * 32, kNodeThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_node_assemble_body(wraps[wi], part, bx); });
}

// Writes block k of the system twice, in row-entry order: B where the row
// list of node a references it, B^T where node b's does.
__device__ inline void store_block_pair(float* out, const LevelDev& L, int k, const float* blk) {
    float* A = out + (long)L.offdiag_slots[k * 2] * 36;
    float* T = out + (long)L.offdiag_slots[k * 2 + 1] * 36;
    for (int r = 0; r < 6; ++r)
        for (int q = 0; q < 6; ++q) {
            A[r * 6 + q] = blk[r * 6 + q];
            T[q * 6 + r] = blk[r * 6 + q];
        }
}

// Adds block k into the system, both ways (the smoothness edge of a node pair
// whose shared-vertex block is already there).
__device__ inline void add_block_pair(float* out, const LevelDev& L, int k, const float* blk) {
    float* A = out + (long)L.offdiag_slots[k * 2] * 36;
    float* T = out + (long)L.offdiag_slots[k * 2 + 1] * 36;
    for (int r = 0; r < 6; ++r)
        for (int q = 0; q < 6; ++q) {
            A[r * 6 + q] += blk[r * 6 + q];
            T[q * 6 + r] += blk[r * 6 + q];
        }
}

// Warp per node pair: lanes stride over the vertices the two nodes share,
// each lane keeps a 6x6 block in registers, one butterfly reduction.
__device__ __forceinline__ void k_pair_assemble_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (!assembles(c)) return;
    const LevelDev& L = w.levels[c.level];
    const int p = (bx * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= L.pair_count) return;
    float blk[36];
    for (int i = 0; i < 36; ++i) blk[i] = 0.0f;
    for (int i = L.pair_begin[p] + lane; i < L.pair_begin[p + 1]; i += 32) {
        const int code = L.pair_entry[i];
        const int v = code >> 6, sa = (code >> 3) & 7, sb = code & 7;
        const float wa = (float)L.bind_weights[v * kMaxSlots + sa];
        const float wb = (float)L.bind_weights[v * kMaxSlots + sb];
        const float4 a4 = w.offsets32[v * kMaxSlots + sa], b4 = w.offsets32[v * kMaxSlots + sb];
        const F3 aa = {a4.x, a4.y, a4.z};
        const F3 ab = {b4.x, b4.y, b4.z};
        const float4 r0 = w.residual32[v], r1 = w.resid_aux32[v], r2 = w.lm_resid32[v];
        const float coef = (r0.w + r2.w) * wa * wb;  // p2p and landmark share the form
        if (coef > 0.0f) {
            // [ (aa.ab) I - ab aa^T, [aa]x ; [ab]x^T, I ]
            const float dp = dot(aa, ab);
            const float av[3] = {aa.x, aa.y, aa.z}, bv[3] = {ab.x, ab.y, ab.z};
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q)
                    blk[r * 6 + q] += coef * ((r == q ? dp : 0.0f) - bv[r] * av[q]);
            blk[0 * 6 + 4] += -coef * aa.z; blk[0 * 6 + 5] += coef * aa.y;
            blk[1 * 6 + 3] += coef * aa.z;  blk[1 * 6 + 5] += -coef * aa.x;
            blk[2 * 6 + 3] += -coef * aa.y; blk[2 * 6 + 4] += coef * aa.x;
            // [ab]x^T = -[ab]x in rows 3-5, columns 0-2
            blk[3 * 6 + 1] += coef * ab.z;  blk[3 * 6 + 2] += -coef * ab.y;
            blk[4 * 6 + 0] += -coef * ab.z; blk[4 * 6 + 2] += coef * ab.x;
            blk[5 * 6 + 0] += coef * ab.y;  blk[5 * 6 + 1] += -coef * ab.x;
            blk[3 * 6 + 3] += coef; blk[4 * 6 + 4] += coef; blk[5 * 6 + 5] += coef;
        }
        if (r1.w > 0.0f) {
            const F3 n = {r1.x, r1.y, r1.z};
            const F3 ca = cross(aa, n), cb = cross(ab, n);
            const float ua[6] = {ca.x, ca.y, ca.z, n.x, n.y, n.z};
            const float ub[6] = {cb.x, cb.y, cb.z, n.x, n.y, n.z};
            const float s = r1.w * wa * wb;
            for (int r = 0; r < 6; ++r)
                for (int q = 0; q < 6; ++q) blk[r * 6 + q] += s * ua[r] * ub[q];
        }
    }
    // the 36 sums spread over the lanes (two each at most); each lane stores
    // what it holds, both ways
    int first = 0, count = 36;
    warp_sum_halving<36>(blk, lane, first, count);
    float* A = w.offdiag[1 - c.system] + (long)L.offdiag_slots[p * 2] * 36;
    float* T = w.offdiag[1 - c.system] + (long)L.offdiag_slots[p * 2 + 1] * 36;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        if (i >= count) break;
        const int j = first + i, r = j / 6, q = j - r * 6;
        const float value = (c.route == 1 && (r < 3 || q < 3)) ? 0.0f : blk[i];
        A[r * 6 + q] = value;
        T[q * 6 + r] = value;
    }
}

__global__ void __launch_bounds__(kNodeThreads, 3) k_pair_assemble(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? (assembles(c) ? blocks_of_dev(w.levels[c.level].pair_count * 32, kNodeThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_pair_assemble_body(wraps[wi], part, bx); });
}

__device__ __forceinline__ void k_edge_assemble_body(const WrapDev& w, int part, int bx) {
    const WrapControl c = *w.control;
    if (!in_part(c, part)) return;
    if (!computes_energy(c)) return;
    const LevelDev& L = w.levels[c.level];
    if ((long)bx * blockDim.x >= L.edge_count) return;
    const int e = bx * blockDim.x + threadIdx.x;
    const double* wt = w.weights[c.level];
    const int buf = eval_buffer(c);
    double energy = 0.0;
    if (e < L.edge_count) {
        const int a = L.edges[e * 2], b = L.edges[e * 2 + 1];
        const D3 ga = load_d3(L.rest, a), gb = load_d3(L.rest, b);
        const D3 gd = rsub(gb, ga);
        const double* R = w.rot[buf];
        const double* T = w.trans[buf];
        if (wt[2] > 0.0) {
            const double sc = sqrt(wt[2]);
            const D3 field_a = radd(radd(rmat(R + a * 9, gd), ga), load_d3(T, a));
            const D3 field_b = radd(gb, load_d3(T, b));
            const D3 diff = rmul(rsub(field_a, field_b), sc);
            energy = da(da(dm(diff.x, diff.x), dm(diff.y, diff.y)), dm(diff.z, diff.z));
        }
        if (assembles(c)) {
            float blk[36];
            for (int i = 0; i < 36; ++i) blk[i] = 0.0f;
            if (wt[2] > 0.0) {
                const float ws = (float)wt[2];
                const F3 cv = mul3f(w.rot32 + a * 9, {(float)gd.x, (float)gd.y, (float)gd.z});
                // ws * [[0, -[c]x], [0, -I]]
                if (c.route == 0) {
                    blk[0 * 6 + 4] = ws * cv.z;  blk[0 * 6 + 5] = -ws * cv.y;
                    blk[1 * 6 + 3] = -ws * cv.z; blk[1 * 6 + 5] = ws * cv.x;
                    blk[2 * 6 + 3] = ws * cv.y;  blk[2 * 6 + 4] = -ws * cv.x;
                }
                blk[3 * 6 + 3] = -ws; blk[4 * 6 + 4] = -ws; blk[5 * 6 + 5] = -ws;
            }
            // into the pair's block when the pair shares a vertex (the pair
            // assembly, launched before on the same stream, wrote it this tick)
            const int k = L.edge_block[e];
            if (k < L.pair_count) {
                add_block_pair(w.offdiag[1 - c.system], L, k, blk);
            } else {
                store_block_pair(w.offdiag[1 - c.system], L, k, blk);
            }
        }
    }
    // the edge's smoothness energy; the decision kernel sums them as a block
    // sum over this block would (no block barrier here)
    if (e < L.edge_count) w.edge_partials[e] = energy;
}

__global__ void __launch_bounds__(kEdgeThreads) k_edge_assemble(const WrapDev* __restrict__ wraps, int wrap_count, int part) {
    over_virtual_blocks<false>(
        wraps, wrap_count,
        [&](const WrapDev& w) {
            const WrapControl c = *w.control;
            return in_part(c, part) ? (computes_energy(c) ? blocks_of_dev(w.levels[c.level].edge_count, kEdgeThreads) : 0) : 0;
        },
        [&](int wi, int bx) { k_edge_assemble_body(wraps[wi], part, bx); });
}

// ---------------------------------------------------------------------------
// the decision: the schedule of route_a.cpp:99-190 / session.cu:404-576,
// taken on the device from FP64 energies
// ---------------------------------------------------------------------------
__device__ inline double relative_change(double before, double after) {  // route_shared.h:24-26
    return (before - after) / fmax(fabs(before), 1e-12);
}

__global__ void k_decide(const WrapDev* __restrict__ wraps, int part) {
    const WrapDev& w = wraps[blockIdx.x];
    WrapControl* ctl = w.control;
    if (part != 0 && (part == 1) != (ctl->tick_phase == kPhaseSolve)) return;
    const int phase = ctl->phase;
    if (phase == kPhaseDone) return;
    __shared__ double scratch[33];
    __shared__ double parts_s[kEnergyKinds];
    const WrapControl c0 = *ctl;
    if (computes_energy(c0)) {
        const LevelDev& L = w.levels[c0.level];
        const int vb = (w.V + kVertexThreads - 1) / kVertexThreads;
        const int eb = (L.edge_count + kEdgeThreads - 1) / kEdgeThreads;
        const int nb = (L.node_count + kNodeThreads / 32 - 1) / (kNodeThreads / 32);
        double s0 = 0, s1 = 0, s4 = 0, s2 = 0, s3 = 0;
        for (int i = threadIdx.x; i < vb; i += blockDim.x) {
            s0 += w.partials[(long)i * kPartialStride];
            s1 += w.partials[(long)i * kPartialStride + 1];
            s4 += w.partials[(long)i * kPartialStride + 2];
        }
        for (int i = threadIdx.x; i < eb; i += blockDim.x) {
            // edge block i's smoothness energy, summed in the order of a block
            // sum over its 128 threads: a butterfly within each warp (lane l
            // holds edge 128i + 32j + l, zero past the last edge), then the
            // four warps' sums, ((w0 + w2) + (w1 + w3)); the zeros the other
            // lanes add change nothing (energies are non-negative)
            static_assert(kEdgeThreads == 4 * 32, "four warps per edge block");
            double warp_total[4];
            for (int j = 0; j < 4; ++j) {
                double x[32];
                for (int l = 0; l < 32; ++l) {
                    const int e = i * kEdgeThreads + j * 32 + l;
                    x[l] = e < L.edge_count ? w.edge_partials[e] : 0.0;
                }
                for (int o = 16; o > 0; o >>= 1)
                    for (int l = 0; l < o; ++l) x[l] = x[l] + x[l + o];
                warp_total[j] = x[0];
            }
            s2 += (warp_total[0] + warp_total[2]) + (warp_total[1] + warp_total[3]);
        }
        for (int i = threadIdx.x; i < nb; i += blockDim.x) {
            // node block i's anchor energy, summed in the order of a block sum
            // over its 8 warps (lane 0 of warp j holds node 8i + j; the other
            // lanes add zeros, which change nothing)
            static_assert(kNodeThreads == 8 * 32, "eight nodes per node block");
            double v[8];
            for (int j = 0; j < 8; ++j) {
                const int n = i * 8 + j;
                v[j] = n < L.node_count ? w.node_partials[n] : 0.0;
            }
            s3 += ((v[0] + v[4]) + (v[2] + v[6])) + ((v[1] + v[5]) + (v[3] + v[7]));
        }
        const double t0 = block_sum<256>(s0, scratch);
        const double t1 = block_sum<256>(s1, scratch);
        const double t2 = block_sum<256>(s2, scratch);
        const double t3 = block_sum<256>(s3, scratch);
        const double t4 = block_sum<256>(s4, scratch);
        if (threadIdx.x == 0) {
            parts_s[0] = t0; parts_s[1] = t1; parts_s[2] = t2; parts_s[3] = t3; parts_s[4] = t4;
        }
        __syncthreads();
    }
    // the long walks this tick's query took from its list are done: clear
    // their flags and empty the list, which the next query but one fills
    const bool queried = c0.tick_phase == kPhaseTransfer || c0.tick_phase == kPhaseRefresh ||
                         c0.tick_phase == kPhaseFinal;
    if (queried) {
        const int cur = c0.long_cur;
        const int taken = min(w.long_count[cur], kLongCap);
        for (int i = threadIdx.x; i < taken; i += blockDim.x)
            w.long_flag[(long)cur * w.V + w.long_list[cur * kLongCap + i]] = 0;
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    WrapControl c = c0;
    c.steps += 1;
    if (queried) {
        w.long_count[c.long_cur] = 0;
        c.long_cur ^= 1;
    }
    const double total = parts_s[0] + parts_s[1] + parts_s[2] + parts_s[3] + parts_s[4];
    LevelRecord& rec = w.records[c.level];
    if (c.phase == kPhaseSolve) {
        rec.solves += 1;
        rec.pcg_iterations += c.pcg_iterations;
    }
    if (refresh_like(c.phase)) rec.queries += 1;
    if (assembles(c)) rec.assemblies += 1;
    bool close_outer = false;
    if (c.phase == kPhaseTransfer || c.phase == kPhaseRefresh) {
        if (c.phase == kPhaseTransfer) c.state = 1 - c.state;
        c.system = 1 - c.system;
        c.energy = total;
        for (int k = 0; k < kEnergyKinds; ++k) c.energy_parts[k] = parts_s[k];
        if (c.outer == 0) rec.energy_start = total;
        c.phase = kPhaseSolve;
        c.inner = 0;
        c.attempt = 0;
    } else if (c.phase == kPhaseSolve) {
        bool end_inner = false;
        if (!c.pcg_ok) {
            c.damping *= w.damping_increase;
            c.attempt += 1;
            end_inner = c.attempt >= w.max_attempts;
        } else {
            c.candidate_energy = total;
            for (int k = 0; k < kEnergyKinds; ++k) c.candidate_parts[k] = parts_s[k];
            if (total < c.energy) {
                c.state = 1 - c.state;
                if (c.route == 0) c.system = 1 - c.system;
                c.damping = fmax(c.damping * w.damping_decrease, 1e-12);
                c.inner += 1;
                rec.inner_iterations += 1;
                const double improvement = relative_change(c.energy, total);
                c.energy = total;
                for (int k = 0; k < kEnergyKinds; ++k) c.energy_parts[k] = parts_s[k];
                c.attempt = 0;
                end_inner = improvement <= w.inner_tol[c.level] || c.inner >= w.max_inner[c.level];
            } else {
                c.damping *= w.damping_increase;
                c.attempt += 1;
                end_inner = c.attempt >= w.max_attempts;
            }
        }
        close_outer = end_inner;
    } else if (c.phase == kPhaseFinal) {
        c.phase = kPhaseDone;
    }
    if (close_outer) {  // route_a.cpp:171-181
        rec.energy_end = c.energy;
        rec.outer_iterations += 1;
        bool converged = false;
        if (c.outer > 0 && relative_change(c.previous_level_energy, c.energy) <= w.outer_tol[c.level]) {
            converged = true;
            rec.converged = 1;
        } else {
            c.previous_level_energy = c.energy;
        }
        c.outer += 1;
        if (converged || c.outer >= w.max_outer[c.level]) {
            c.stats_pending = c.level + 1;
            if (c.level + 1 < c.level_count) {
                c.level += 1;
                c.phase = kPhaseTransfer;
                c.damping = w.initial_damping;
                c.outer = 0;
                c.previous_level_energy = 0.0;
                LevelRecord& next = w.records[c.level];
                next.level = c.level;
                next.nodes = w.levels[c.level].node_count;
            } else {
                c.phase = kPhaseFinal;
            }
        } else {
            c.phase = kPhaseRefresh;
        }
        c.inner = 0;
        c.attempt = 0;
    }
    *ctl = c;
}

// ---------------------------------------------------------------------------
// host launch of one tick
// ---------------------------------------------------------------------------
// Grids of the virtual-block kernels: as many blocks as fit on the device
// at once (occupancy of each kernel at its block size, times the SMs).
struct VirtualGrids {
    int prologue, c_fit, c_rhs, evaluate, normals, residual, node, pair, edge;
};
const VirtualGrids& virtual_grids() {
    static const VirtualGrids grids = [] {
        int device = 0, sms = 148;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        auto fit = [sms](auto kernel, int threads) {
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, sizeof(int) * 1025);
            return sms * (per_sm > 0 ? per_sm : 1);
        };
        VirtualGrids g;
        g.prologue = fit(k_prologue, 128);
        g.c_fit = fit(k_c_fit, kNodeThreads);
        g.c_rhs = fit(k_c_rhs, kNodeThreads);
        g.evaluate = fit(k_evaluate, kVertexThreads);
        g.normals = fit(k_normals, kVertexThreads);
        g.residual = fit(k_residual, kVertexThreads);
        g.node = fit(k_node_assemble, kNodeThreads);
        g.pair = fit(k_pair_assemble, kNodeThreads);
        g.edge = fit(k_edge_assemble, kEdgeThreads);
        return g;
    }();
    return grids;
}

void launch_tick(const WrapDev* wraps, const TickShape& s, cudaStream_t stream,
                 KernelTimers* timers) {
    const int W = s.wraps;
    const VirtualGrids& grids = virtual_grids();
    const size_t virtual_smem = sizeof(int) * (W + 1);
    const bool timed = timers && timers->active;
    // statistics of a finished level, and every wrap's phase at the tick's start
    k_stats<<<dim3(1, W), kStatsThreads, 0, stream>>>(wraps, 0);
    // A wrap that starts the tick in a solve runs the solve chain (Horn fit,
    // PCG, candidate evaluation, energy and system, decision); any other runs
    // the refresh chain (warm start, evaluation, normals, closest points,
    // energy and system, decision).  The chains touch different wraps, so
    // with a side stream they run as two parallel branches of the tick.  A
    // timed tick runs them one after the other, so that each kernel group's
    // time is its own.
    const bool split = s.side_stream != nullptr && !timed;
    const int solve_part = split ? 1 : 0, refresh_part = split ? 2 : 0;
    cudaStream_t refresh = split ? s.side_stream : stream;
    auto assemble_and_decide = [&](int part, cudaStream_t on) {
        if (timed) cudaEventRecord(timers->assemble_begin, on);
        k_residual<<<grids.residual, kVertexThreads, virtual_smem, on>>>(wraps, W, part);
        k_node_assemble<<<grids.node, kNodeThreads, virtual_smem, on>>>(wraps, W, part);
        if (s.max_pairs > 0) k_pair_assemble<<<grids.pair, kNodeThreads, virtual_smem, on>>>(wraps, W, part);
        k_edge_assemble<<<grids.edge, kEdgeThreads, virtual_smem, on>>>(wraps, W, part);
        if (timed) cudaEventRecord(timers->assemble_end, on);
        k_decide<<<W, 256, 0, on>>>(wraps, part);
    };
    if (split) {
        cudaEventRecord(s.side_fork, stream);
        cudaStreamWaitEvent(refresh, s.side_fork, 0);
    }

    // ---- the solve chain ----
    if (s.route_c) {
        k_c_fit<<<grids.c_fit, kNodeThreads, virtual_smem, stream>>>(wraps, W, solve_part);
        k_c_rhs<<<grids.c_rhs, kNodeThreads, virtual_smem, stream>>>(wraps, W, solve_part);
    }
    if (timed) cudaEventRecord(timers->pcg_begin, stream);
    auto launch_pcg = [&](int cluster, int count, int shared, const int* index, cudaStream_t on) {
        cudaLaunchConfig_t config = {};
        config.gridDim = dim3(cluster, count);
        config.blockDim = dim3(kPcgThreads);
        config.dynamicSmemBytes = shared;
        config.stream = on;
        cudaLaunchAttribute attribute[1];
        attribute[0].id = cudaLaunchAttributeClusterDimension;
        attribute[0].val.clusterDim.x = cluster;
        attribute[0].val.clusterDim.y = 1;
        attribute[0].val.clusterDim.z = 1;
        config.attrs = attribute;
        config.numAttrs = 1;
        cudaLaunchKernelEx(&config, k_pcg, wraps, index, (int)(shared / sizeof(float)));
    };
    if (s.pcg_groups <= 0) {
        launch_pcg(s.pcg_cluster, W, s.pcg_shared_bytes, nullptr, stream);
    } else {
        // fork: every class launch after everything before it on `stream`
        cudaEventRecord(s.pcg_fork, stream);
        for (int g = 1; g < s.pcg_groups; ++g) {
            cudaStreamWaitEvent(s.pcg_streams[g], s.pcg_fork, 0);
            launch_pcg(s.pcg_group_cluster[g], s.pcg_group_count[g], s.pcg_group_shared[g],
                       s.pcg_group_index[g], s.pcg_streams[g]);
            cudaEventRecord(s.pcg_join[g], s.pcg_streams[g]);
        }
        launch_pcg(s.pcg_group_cluster[0], s.pcg_group_count[0], s.pcg_group_shared[0],
                   s.pcg_group_index[0], stream);
        for (int g = 1; g < s.pcg_groups; ++g) cudaStreamWaitEvent(stream, s.pcg_join[g], 0);
    }
    if (timed) cudaEventRecord(timers->pcg_end, stream);
    if (split) {
        k_evaluate<<<grids.evaluate, kVertexThreads, virtual_smem, stream>>>(wraps, W, solve_part);
        assemble_and_decide(solve_part, stream);
    }

    // ---- the refresh chain ----
    k_prologue<<<grids.prologue, 128, virtual_smem, refresh>>>(wraps, W, refresh_part);
    k_evaluate<<<grids.evaluate, kVertexThreads, virtual_smem, refresh>>>(wraps, W, refresh_part);
    k_normals<<<grids.normals, kVertexThreads, virtual_smem, refresh>>>(wraps, W, refresh_part);
    if (timed) cudaEventRecord(timers->query_begin, refresh);
    launch_query(wraps, W, s.max_vertices, refresh, s.query_counter);
    if (timed) cudaEventRecord(timers->query_end, refresh);
    k_stats<<<dim3(1, W), kStatsThreads, 0, refresh>>>(wraps, 1);
    assemble_and_decide(refresh_part, refresh);
    if (split) {
        cudaEventRecord(s.side_join, refresh);
        cudaStreamWaitEvent(stream, s.side_join, 0);
    }
}

int tick_kernel_launches(const TickShape& s, bool timed) {
    // an untimed tick with a side stream assembles and decides in each branch
    const int per_chain = (s.max_pairs > 0 ? 5 : 4) + 1;  // residual, node, pair, edge, decide; evaluate
    return (s.max_pairs > 0 ? 14 : 13) - (s.route_c ? 0 : 2) + (s.pcg_groups > 0 ? s.pcg_groups : 1) +
           (s.side_stream && !timed ? per_chain : 0);
}

// Cluster size of the solve for one wrap of `nodes` nodes on its own: a
// power of two with about 128 nodes (32 segments, two per warp) per CTA, at
// most 16 CTAs (the non-portable maximum, enabled here).
int pcg_latency_cluster(int nodes) {
    int ranks = 1;
    while (ranks < 16 && ranks * 128 < nodes) ranks *= 2;
    return ranks;
}

void pcg_enable() {
    static const bool enabled = [] {  // once per process, thread-safe
        cudaFuncSetAttribute(k_pcg, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, kPcgMaxSmemBytes);
        return true;
    }();
    (void)enabled;
}

// Default cluster size for a batch: one wrap takes its latency cluster; many
// wraps share the SMs, so the cluster shrinks until one CTA per SM holds the
// whole batch (the result does not depend on the choice).
int pcg_cluster_size(int max_nodes, int wraps, int sm_count) {
    pcg_enable();
    int ranks = pcg_latency_cluster(max_nodes);
    while (ranks > 1 && (long)ranks * wraps > sm_count) ranks /= 2;
    return ranks;
}

// Dynamic shared memory of the solve launch: what the largest wrap would use
// at this cluster size, at most the per-CTA maximum.
int pcg_shared_bytes(const int* max_nodes, int wraps, int cluster) {
    int floats = 0;
    for (int i = 0; i < wraps; ++i)
        floats = max(floats, pcg_place(max_nodes[i], cluster, 1 << 30).floats);
    return min(floats * (int)sizeof(float), kPcgMaxSmemBytes);
}

int pcg_max_nodes() { return 32768; }

void launch_fit_rigid(const double* src, const double* dst, const double* weights, int n, double* out,
                      cudaStream_t stream) {
    k_fit_rigid<<<1, kRigidThreads, 0, stream>>>(src, dst, weights, n, out);
}

}  // namespace nricp_b200
