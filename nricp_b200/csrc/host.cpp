// Host-side preparation of a wrap.  See host.hpp.
//
// Compiled with -ffp-contract=off so that every FP64 expression rounds the way
// the reference's host code does: the template graph (seeds, bindings, edges)
// then comes out bit-identical to src/core/graph.cpp's.
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <iomanip>
#include <limits>
#include <memory>
#include <numeric>
#include <sstream>
#include <unordered_set>
#include <utility>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace nricp_b200 {

namespace {

inline double sqdist(const double* a, const double* b) {  // sampling.cpp:17-19
    const double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return x * x + y * y + z * z;
}

void keep_nearest(double* sq, int* idx, int& held, int capacity, double value, int entry) {
    // sampling.cpp:23-42
    if (held == capacity) {
        const bool beats = value < sq[capacity - 1] ||
                           (value == sq[capacity - 1] && entry < idx[capacity - 1]);
        if (!beats) return;
    }
    int at = held < capacity ? held++ : capacity - 1;
    while (at > 0 && (sq[at - 1] > value || (sq[at - 1] == value && idx[at - 1] > entry))) {
        sq[at] = sq[at - 1];
        idx[at] = idx[at - 1];
        --at;
    }
    sq[at] = value;
    idx[at] = entry;
}

// A uniform grid over a point set for exact nearest-point searches.  The
// searches below keep the k smallest (key, index) pairs under a strict total
// order, so their result does not depend on the order candidates arrive in:
// offering every point that could enter the k smallest gives exactly what a
// scan of all points gives.  A search visits cells in shells of growing
// Chebyshev radius around the query's cell and stops once every cell not yet
// visited lies farther than its k-th key.  That bound takes a margin of a
// millionth of a cell and a relative 1e-12 on squares, far above the few
// ulps by which a rounded distance can fall below the exact one.
class PointGrid {
public:
    PointGrid(const double* pts, int n) {
        double hi[3];
        for (int a = 0; a < 3; ++a) lo_[a] = hi[a] = n > 0 ? pts[a] : 0.0;
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a) {
                lo_[a] = std::min(lo_[a], pts[i * 3 + a]);
                hi[a] = std::max(hi[a], pts[i * 3 + a]);
            }
        double widest = 0.0;
        for (int a = 0; a < 3; ++a) widest = std::max(widest, hi[a] - lo_[a]);
        // cells of about one point each for a solid cloud: a few per occupied
        // cell for points on a surface; flat extents count as a thousandth
        double volume = 1.0;
        for (int a = 0; a < 3; ++a) volume *= std::max(hi[a] - lo_[a], widest * 1e-3);
        h_ = widest > 0.0 ? std::cbrt(volume / std::max(1, n)) : 1.0;
        long cells = 1;
        for (;;) {
            cells = 1;
            for (int a = 0; a < 3; ++a) {
                dim_[a] = static_cast<int>(std::floor((hi[a] - lo_[a]) / h_)) + 1;
                cells *= dim_[a];
            }
            if (cells <= 8L * n + 64) break;
            h_ *= 1.25;
        }
        begin_.assign(cells + 1, 0);
        std::vector<int32_t> cell_of(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) {
            long c = 0;
            for (int a = 2; a >= 0; --a)
                c = c * dim_[a] + std::clamp(coord(pts[i * 3 + a], a), 0, dim_[a] - 1);
            cell_of[i] = static_cast<int32_t>(c);
            begin_[c + 1]++;
        }
        for (long c = 0; c < cells; ++c) begin_[c + 1] += begin_[c];
        items_.resize(static_cast<size_t>(n));
        std::vector<int32_t> cursor(begin_.begin(), begin_.end() - 1);
        for (int i = 0; i < n; ++i) items_[cursor[cell_of[i]]++] = i;
    }

    // Calls offer(point index) for every point of the cells in shell after
    // shell around p, until done(gap) -- gap a lower bound on the distance
    // from p to any point not yet offered -- returns true, or every cell has
    // been offered.
    template <class Offer, class Done>
    void search(const double* p, Offer&& offer, Done&& done) const {
        const bool walked = search_cells(
            p, [&](long cell) { for (int32_t k = begin_[cell]; k < begin_[cell + 1]; ++k) offer(items_[k]); },
            done);
        if (!walked)  // every point, in index order: a scan's own order
            for (int32_t i = 0; i < static_cast<int32_t>(items_.size()); ++i) offer(i);
    }

    // The same walk, a cell at a time.  Returns false, having visited
    // nothing, for a query beyond twice the grid's extent or not finite.
    template <class Visit, class Done>
    bool search_cells(const double* p, Visit&& visit_cell, Done&& done) const {
        int c[3];
        for (int a = 0; a < 3; ++a) c[a] = coord(p[a], a);
        // shells nearer than the grid hold nothing
        int first = 0, widest = 1;
        for (int a = 0; a < 3; ++a) {
            first = std::max({first, -c[a], c[a] - (dim_[a] - 1)});
            widest = std::max(widest, dim_[a]);
        }
        if (first > 2 * widest || !std::isfinite(p[0] + p[1] + p[2])) return false;
        for (int r = first;; ++r) {
            const int x0 = std::max(c[0] - r, 0), x1 = std::min(c[0] + r, dim_[0] - 1);
            const int y0 = std::max(c[1] - r, 0), y1 = std::min(c[1] + r, dim_[1] - 1);
            const int z0 = std::max(c[2] - r, 0), z1 = std::min(c[2] + r, dim_[2] - 1);
            auto visit = [&](int x, int y, int z) {
                const long cell = (static_cast<long>(z) * dim_[1] + y) * dim_[0] + x;
                if (begin_[cell] < begin_[cell + 1]) visit_cell(cell);
            };
            for (int z = z0; z <= z1; ++z)
                for (int y = y0; y <= y1; ++y) {
                    if (z == c[2] - r || z == c[2] + r || y == c[1] - r || y == c[1] + r) {
                        for (int x = x0; x <= x1; ++x) visit(x, y, z);  // a face row: all of it
                    } else {                                            // else its two ends
                        if (c[0] - r >= 0 && c[0] - r < dim_[0]) visit(c[0] - r, y, z);
                        if (r > 0 && c[0] + r >= 0 && c[0] + r < dim_[0]) visit(c[0] + r, y, z);
                    }
                }
            bool covered = true;
            double gap = std::numeric_limits<double>::infinity();
            for (int a = 0; a < 3; ++a) {
                covered = covered && c[a] - r <= 0 && c[a] + r >= dim_[a] - 1;
                if (c[a] - r > 0) gap = std::min(gap, p[a] - (lo_[a] + (c[a] - r) * h_));
                if (c[a] + r < dim_[a] - 1) gap = std::min(gap, lo_[a] + (c[a] + r + 1) * h_ - p[a]);
            }
            if (covered) return true;
            if (done(std::max(0.0, gap - h_ * 1e-6))) return true;
        }
    }

    long cells() const { return static_cast<long>(begin_.size()) - 1; }
    int32_t begin(long cell) const { return begin_[cell]; }
    int32_t end(long cell) const { return begin_[cell + 1]; }
    int32_t item(int32_t k) const { return items_[k]; }  // in ascending index within a cell

private:
    int coord(double x, int a) const {
        const double t = std::floor((x - lo_[a]) / h_);
        return t == t ? static_cast<int>(std::clamp(t, -1e9, 1e9)) : 1000000000;  // NaN: far away
    }

    double lo_[3], h_;
    int dim_[3];
    std::vector<int32_t> begin_, items_;
};

// Below this many (query, point) pairs a plain scan is as fast.
constexpr long kGridPairs = 1L << 20;

// The grid holds finite points only: with a NaN among them the keys are no
// longer totally ordered and only the scan's own order gives its result.
bool all_finite(const std::vector<double>& v) {
    for (double x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

}  // namespace

void validate_mesh(const double* p, int n, const int32_t* f, int m, const char* what) {
    std::vector<std::string> problems;  // mesh.cpp:90-116
    if (n <= 0) problems.push_back("mesh has no vertices");
    if (m <= 0) problems.push_back("mesh has no faces; closest-point queries need a surface");
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(p[i * 3]) || !std::isfinite(p[i * 3 + 1]) || !std::isfinite(p[i * 3 + 2]))
            problems.push_back("vertex " + std::to_string(i) + " is not finite");
    for (int i = 0; i < m; ++i)
        for (int k = 0; k < 3; ++k) {
            const int index = f[i * 3 + k];
            if (index < 0 || index >= n)
                problems.push_back("face " + std::to_string(i) + " corner " + std::to_string(k) +
                                   " index " + std::to_string(index) + " is out of range");
        }
    if (problems.empty()) return;
    std::string message = std::string("invalid ") + what + " mesh: ";
    for (size_t i = 0; i < problems.size(); ++i) message += (i ? "; " : "") + problems[i];
    throw InvalidArgument(message);
}

void validate_settings(const NricpSolveDesc& d) {
    validate_mesh(d.template_points, d.template_vertex_count, d.template_faces,
                  d.template_face_count, "template");
    validate_mesh(d.target_points, d.target_vertex_count, d.target_faces, d.target_face_count,
                  "target");
    const int k = d.max_nodes_per_vertex > 0 ? d.max_nodes_per_vertex : 4;
    if (k > NRICP_MAX_SLOTS)
        throw InvalidArgument("max_nodes_per_vertex is " + std::to_string(k) + "; at most " +
                              std::to_string(NRICP_MAX_SLOTS) + " nodes can bind a vertex");
    if (d.graph_levels > 16)
        throw InvalidArgument("graph_levels is " + std::to_string(d.graph_levels) +
                              "; at most 16 levels are supported");
    if (d.route != NRICP_ROUTE_B && d.route != NRICP_ROUTE_C)
        throw InvalidArgument("the device session runs 'route_b' or 'route_c'");
    if (d.mask) {  // constraints.cpp:34-58
        int active = 0;
        for (int i = 0; i < d.template_vertex_count; ++i) active += d.mask[i] ? 1 : 0;
        if (active == 0)
            throw InvalidArgument(
                "invalid mask: mask excludes every vertex; the fit would be unconstrained");
    }
    if (d.landmark_count > 0) {  // constraints.cpp:8-32
        std::vector<std::string> problems;
        std::unordered_set<int> seen;
        for (int i = 0; i < d.landmark_count; ++i) {
            const int v = d.landmark_indices[i];
            if (v < 0 || v >= d.template_vertex_count) {
                problems.push_back("landmark " + std::to_string(i) + " points at template vertex " +
                                   std::to_string(v) + " but the template has " +
                                   std::to_string(d.template_vertex_count) + " vertices");
                continue;
            }
            const double* t = d.landmark_targets + i * 3;
            if (!std::isfinite(t[0]) || !std::isfinite(t[1]) || !std::isfinite(t[2]))
                problems.push_back("landmark " + std::to_string(i) + " has a non-finite target");
            if (!seen.insert(v).second)
                problems.push_back("landmark " + std::to_string(i) + " marks template vertex " +
                                   std::to_string(v) + " twice");
        }
        if (!problems.empty()) {
            std::string message = "invalid landmarks: ";
            for (size_t i = 0; i < problems.size(); ++i) message += (i ? "; " : "") + problems[i];
            throw InvalidArgument(message);
        }
    }
}

void compute_normalization(const double* p, int n, double center[3], double* scale) {
    // mesh.cpp:47-64, 174-181
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (n > 0)
        for (int k = 0; k < 3; ++k) lo[k] = hi[k] = p[k];
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], p[i * 3 + k]);
            hi[k] = std::max(hi[k], p[i * 3 + k]);
        }
    for (int k = 0; k < 3; ++k) center[k] = (lo[k] + hi[k]) * 0.5;
    const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    const double diagonal = std::sqrt(dx * dx + dy * dy + dz * dz);
    *scale = diagonal > 0.0 ? 1.0 / diagonal : 1.0;
}

void normalized_into(const double* p, int n, const double center[3], double scale, double* out) {
    for (int i = 0; i < n; ++i)  // mesh.cpp:183-187
        for (int k = 0; k < 3; ++k) out[i * 3 + k] = (p[i * 3 + k] - center[k]) * scale;
}

std::vector<double> normalized(const double* p, int n, const double center[3], double scale) {
    std::vector<double> out(static_cast<size_t>(n) * 3);
    normalized_into(p, n, center, scale, out.data());
    return out;
}

void vertex_normals_into(const double* p, int n, const int32_t* f, int m, double* out) {
    std::fill(out, out + static_cast<size_t>(n) * 3, 0.0);  // mesh.cpp:71-88
    for (int i = 0; i < m; ++i) {
        const double* a = &p[f[i * 3] * 3];
        const double* b = &p[f[i * 3 + 1] * 3];
        const double* c = &p[f[i * 3 + 2] * 3];
        const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        const double w[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                             e1[0] * e2[1] - e1[1] * e2[0]};
        for (int k = 0; k < 3; ++k) {
            double* t = &out[f[i * 3 + k] * 3];
            t[0] = t[0] + w[0];
            t[1] = t[1] + w[1];
            t[2] = t[2] + w[2];
        }
    }
    for (int i = 0; i < n; ++i) {
        double* v = &out[i * 3];
        const double length = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (length > 0.0) {
            v[0] = v[0] / length; v[1] = v[1] / length; v[2] = v[2] / length;
        } else {
            v[0] = v[1] = v[2] = 0.0;
        }
    }
}

std::vector<double> vertex_normals(const std::vector<double>& p, const int32_t* f, int m) {
    std::vector<double> out(p.size());
    vertex_normals_into(p.data(), static_cast<int>(p.size() / 3), f, m, out.data());
    return out;
}

// sampling.cpp:47-88.  Ties go to the lowest index; a parallel sweep keeps
// that rule by combining per-thread maxima in thread order.
namespace {

// The rest of the greedy sampling below, given the first seed, every point's
// squared distance to it and the first point farthest from it.  A new seed s
// can only lower the distances of points closer to it than the current
// maximum M, so each step walks the grid's cells until the gap exceeds sqrt(M)
// and updates those alone.  Every non-empty cell keeps its largest distance
// and the first point holding it, and a tournament over the cells -- larger
// distance first, then smaller index -- names the next seed: the same first
// maximum the scan over all points finds.
std::vector<int> seeds_through_grid(const std::vector<double>& pts, int count, std::vector<int> seeds,
                                    std::vector<double> nearest) {
    const int n = static_cast<int>(pts.size() / 3);
    const PointGrid grid(pts.data(), n);
    std::vector<int32_t> slot(grid.cells(), -1);
    std::vector<long> cell_of_slot;
    for (long c = 0; c < grid.cells(); ++c)
        if (grid.begin(c) < grid.end(c)) {
            slot[c] = static_cast<int32_t>(cell_of_slot.size());
            cell_of_slot.push_back(c);
        }
    int leaves = 1;
    while (leaves < static_cast<int>(cell_of_slot.size())) leaves *= 2;
    std::vector<double> value(2 * leaves, -2.0);   // below any distance
    std::vector<int> index(2 * leaves, n);
    auto wins = [&](int a, int b) {
        return value[a] > value[b] || (value[a] == value[b] && index[a] < index[b]);
    };
    auto settle = [&](long cell) {  // the cell's first maximum, then up the tree
        int at = leaves + slot[cell];
        double bs = -1.0;
        int bi = n;
        for (int32_t k = grid.begin(cell); k < grid.end(cell); ++k) {
            const int i = grid.item(k);
            if (nearest[i] > bs) { bs = nearest[i]; bi = i; }
        }
        value[at] = bs;
        index[at] = bi;
        for (at /= 2; at >= 1; at /= 2) {
            const int w = wins(2 * at, 2 * at + 1) ? 2 * at : 2 * at + 1;
            value[at] = value[w];
            index[at] = index[w];
        }
    };
    for (long c : cell_of_slot) settle(c);
    while (static_cast<int>(seeds.size()) < count) {
        const int s = index[1];
        const double reach = value[1];  // no distance is larger
        seeds.push_back(s);
        const double* chosen = &pts[s * 3];
        grid.search_cells(  // a point of the grid itself: always walked
            chosen,
            [&](long cell) {
                bool lowered = false;
                for (int32_t k = grid.begin(cell); k < grid.end(cell); ++k) {
                    const int i = grid.item(k);
                    const double d = sqdist(&pts[i * 3], chosen);
                    if (d < nearest[i]) { nearest[i] = d; lowered = true; }
                }
                if (lowered) settle(cell);
            },
            [&](double gap) { return gap * gap * (1.0 - 1e-12) >= reach; });
    }
    return seeds;
}

}  // namespace

std::vector<int> farthest_point_seeds(const std::vector<double>& pts, int count, int first) {
    const int n = static_cast<int>(pts.size() / 3);
    std::vector<int> seeds;
    if (n <= 0 || count <= 0) return seeds;
    count = std::min(count, n);
    first = std::clamp(first, 0, n - 1);
    std::vector<double> nearest(static_cast<size_t>(n));
    seeds.reserve(count);
    seeds.push_back(first);
    const double* chosen = &pts[first * 3];
    int best = first;
    double best_sq = -1.0;
    for (int i = 0; i < n; ++i) {
        nearest[i] = sqdist(&pts[i * 3], chosen);
        if (nearest[i] > best_sq) { best_sq = nearest[i]; best = i; }
    }
    // The points are split into `chunks` fixed ranges; each range keeps its
    // first maximum and the ranges are merged in order, so the seeds are the
    // sequential scan's (first maximum) for any number of chunks or threads.
    // The ranges are strided over whatever team runs the region: inside an
    // enclosing parallel region (a batch preparing wraps side by side) that
    // team is a single thread.
    if (static_cast<long>(n) * count > kGridPairs && n > 1024 && count > 16 && all_finite(pts))
        return seeds_through_grid(pts, count, std::move(seeds), std::move(nearest));
#ifdef _OPENMP
    const int chunks = n >= 20000 ? std::min(omp_get_max_threads(), 16) : 1;
#else
    const int chunks = 1;
#endif
    std::vector<double> t_best(chunks);
    std::vector<int> t_idx(chunks);
    while (static_cast<int>(seeds.size()) < count) {
        seeds.push_back(best);
        chosen = &pts[best * 3];
#pragma omp parallel num_threads(chunks)
        {
#ifdef _OPENMP
            const int first_chunk = omp_get_thread_num(), team = omp_get_num_threads();
#else
            const int first_chunk = 0, team = 1;
#endif
            for (int t = first_chunk; t < chunks; t += team) {
                const int begin = static_cast<int>((long)n * t / chunks);
                const int end = static_cast<int>((long)n * (t + 1) / chunks);
                double bs = -1.0;
                int bi = begin;
                for (int i = begin; i < end; ++i) {
                    const double d = sqdist(&pts[i * 3], chosen);
                    nearest[i] = nearest[i] < d ? nearest[i] : d;
                    if (nearest[i] > bs) { bs = nearest[i]; bi = i; }
                }
                t_best[t] = bs;
                t_idx[t] = bi;
            }
        }
        best_sq = -1.0;
        for (int t = 0; t < chunks; ++t)
            if (t_best[t] > best_sq) { best_sq = t_best[t]; best = t_idx[t]; }
    }
    return seeds;
}

std::vector<Binding> bind_vertices(const std::vector<double>& vertices,
                                   const std::vector<double>& nodes, int max_nodes, int slot_cap) {
    const int vc = static_cast<int>(vertices.size() / 3);  // sampling.cpp:90-143
    const int nc = static_cast<int>(nodes.size() / 3);
    std::vector<Binding> out(static_cast<size_t>(vc));
    for (Binding& b : out) {
        for (int s = 0; s < NRICP_MAX_SLOTS; ++s) { b.nodes[s] = -1; b.weights[s] = 0.0; }
        b.count = 0;
    }
    if (nc <= 0) return out;
    const int support = std::max(1, std::min({max_nodes, nc, slot_cap}));
    // the same k nearest by (squared distance, index) as a scan of all nodes
    std::unique_ptr<PointGrid> grid;
    if (static_cast<long>(vc) * nc > kGridPairs && nc > 64 && all_finite(nodes))
        grid = std::make_unique<PointGrid>(nodes.data(), nc);
#pragma omp parallel for schedule(static) if (static_cast<long>(vc) * nc > 2000000)
    for (int v = 0; v < vc; ++v) {
        double best_sq[NRICP_MAX_SLOTS] = {};
        int best_idx[NRICP_MAX_SLOTS] = {};
        int held = 0;  // reaches support: a search ends with every node offered, or its k nearest held
        const double* p = &vertices[v * 3];
        if (grid) {
            grid->search(
                p, [&](int n) { keep_nearest(best_sq, best_idx, held, support, sqdist(p, &nodes[n * 3]), n); },
                [&](double gap) { return held == support && best_sq[support - 1] < gap * gap * (1.0 - 1e-12); });
        } else {
            for (int n = 0; n < nc; ++n) keep_nearest(best_sq, best_idx, held, support, sqdist(p, &nodes[n * 3]), n);
        }
        Binding b;
        for (int s = 0; s < NRICP_MAX_SLOTS; ++s) { b.nodes[s] = -1; b.weights[s] = 0.0; }
        b.count = support;
        const double dmax = std::sqrt(best_sq[support - 1]);
        double total = 0.0;
        for (int s = 0; s < support; ++s) {
            const double distance = std::sqrt(best_sq[s]);
            const double ratio = dmax > 0.0 ? distance / dmax : 0.0;
            const double falloff = 1.0 - ratio;
            b.nodes[s] = best_idx[s];
            b.weights[s] = falloff * falloff;
            total += b.weights[s];
        }
        for (int s = 0; s < support; ++s)
            b.weights[s] = total > 0.0 ? b.weights[s] / total : 1.0 / static_cast<double>(support);
        out[v] = b;
    }
    return out;
}

std::vector<int32_t> node_edges(const std::vector<double>& nodes, int neighbours) {
    const int n = static_cast<int>(nodes.size() / 3);  // graph.cpp:11-39
    if (n <= 1 || neighbours <= 0) return {};
    const int taken = std::min(neighbours, n - 1);
    std::vector<std::pair<int, int>> pairs(static_cast<size_t>(n) * taken);
    // the k nearest by (distance, index), as the reference's partial sort
    // over all other nodes orders them; through a grid when n is large
    std::unique_ptr<PointGrid> grid;
    if (static_cast<long>(n) * n > kGridPairs && n > 64 && all_finite(nodes))
        grid = std::make_unique<PointGrid>(nodes.data(), n);
#pragma omp parallel for schedule(static) if (n > 512)
    for (int i = 0; i < n; ++i) {
        auto distance = [&](int o) {
            const double x = nodes[i * 3] - nodes[o * 3], y = nodes[i * 3 + 1] - nodes[o * 3 + 1],
                         z = nodes[i * 3 + 2] - nodes[o * 3 + 2];
            return std::sqrt(x * x + y * y + z * z);
        };
        std::vector<int> best_o(taken);
        if (grid) {  // finite nodes: (distance, index) is a strict total order
            std::vector<double> best_d(taken);
            int held = 0;
            grid->search(
                &nodes[i * 3],
                [&](int o) {
                    if (o != i) keep_nearest(best_d.data(), best_o.data(), held, taken, distance(o), o);
                },
                [&](double gap) { return held == taken && best_d[taken - 1] < gap * (1.0 - 1e-12); });
        } else {      // the reference's partial sort over every other node
            std::vector<std::pair<double, int>> d;
            d.reserve(n - 1);
            for (int o = 0; o < n; ++o)
                if (o != i) d.push_back({distance(o), o});
            std::partial_sort(d.begin(), d.begin() + taken, d.end());
            for (int k = 0; k < taken; ++k) best_o[k] = d[k].second;
        }
        for (int k = 0; k < taken; ++k) {
            const int o = best_o[k];
            pairs[static_cast<size_t>(i) * taken + k] = {std::min(i, o), std::max(i, o)};
        }
    }
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    std::vector<int32_t> out;
    out.reserve(pairs.size() * 2);
    for (auto& p : pairs) { out.push_back(p.first); out.push_back(p.second); }
    return out;
}

int level_node_count(int level, int nodes_initial, int growth, int vertex_count) {
    const double g = std::pow(static_cast<double>(std::max(1, growth)), static_cast<double>(level));
    const int requested = std::max(1, static_cast<int>(std::lround(nodes_initial * g)));
    return std::min(requested, vertex_count);  // graph.cpp:52-57
}

TemplateGraph build_template_graph(const double* points, int count, int levels, int nodes_initial,
                                   int growth, int max_nodes, int edge_neighbours) {
    TemplateGraph graph;  // graph.cpp:41-76
    compute_normalization(points, count, graph.center, &graph.scale);
    const std::vector<double> norm = normalized(points, count, graph.center, graph.scale);
    const int level_count = std::max(1, levels);
    // The greedy sampling does not depend on how many seeds it is asked for,
    // so every level's seeds are a prefix of the largest level's.
    int most = 0;
    for (int l = 0; l < level_count; ++l)
        most = std::max(most, level_node_count(l, nodes_initial, growth, count));
    const std::vector<int> seeds = farthest_point_seeds(norm, most, 0);
    for (int l = 0; l < level_count; ++l) {
        GraphLevel level;
        const int n = std::min<int>(level_node_count(l, nodes_initial, growth, count),
                                    static_cast<int>(seeds.size()));
        level.template_index.assign(seeds.begin(), seeds.begin() + n);
        level.rest.resize(static_cast<size_t>(n) * 3);
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) level.rest[i * 3 + k] = norm[seeds[i] * 3 + k];
        level.bindings = bind_vertices(norm, level.rest, max_nodes, NRICP_MAX_SLOTS);
        level.edges = node_edges(level.rest, edge_neighbours);
        graph.levels.push_back(std::move(level));
    }
    return graph;
}

LevelLayout build_layout(const TemplateGraph& graph, int level, int V) {
    const GraphLevel& g = graph.levels[level];
    LevelLayout L;
    const int N = g.node_count();
    L.node_count = N;
    L.rest = g.rest;
    L.bind_nodes.assign(static_cast<size_t>(V) * NRICP_MAX_SLOTS, -1);
    L.bind_weights.assign(static_cast<size_t>(V) * NRICP_MAX_SLOTS, 0.0);
    L.bind_counts.assign(V, 0);
    // usable_binding (fused_assembly.cpp:85-98): only slots that contribute
    for (int v = 0; v < V; ++v) {
        const Binding& b = g.bindings[v];
        int c = 0;
        for (int s = 0; s < b.count; ++s) {
            if (b.nodes[s] < 0 || b.nodes[s] >= N || b.weights[s] == 0.0) continue;
            L.bind_nodes[v * NRICP_MAX_SLOTS + c] = b.nodes[s];
            L.bind_weights[v * NRICP_MAX_SLOTS + c] = b.weights[s];
            ++c;
        }
        L.bind_counts[v] = c;
    }
    // node -> (vertex, slot)
    std::vector<int32_t> count(N + 1, 0);
    for (int v = 0; v < V; ++v)
        for (int s = 0; s < L.bind_counts[v]; ++s) count[L.bind_nodes[v * NRICP_MAX_SLOTS + s] + 1]++;
    L.gather_begin.assign(N + 1, 0);
    for (int n = 0; n < N; ++n) L.gather_begin[n + 1] = L.gather_begin[n] + count[n + 1];
    L.gather_entry.assign(L.gather_begin[N], 0);
    {
        std::vector<int32_t> cursor(L.gather_begin.begin(), L.gather_begin.end() - 1);
        for (int v = 0; v < V; ++v)
            for (int s = 0; s < L.bind_counts[v]; ++s) {
                const int n = L.bind_nodes[v * NRICP_MAX_SLOTS + s];
                L.gather_entry[cursor[n]++] = v * NRICP_MAX_SLOTS + s;
            }
    }
    // smoothness edges and node -> edge lists
    L.edges = g.edges;
    L.edge_count = static_cast<int>(g.edges.size() / 2);
    L.node_edge_begin.assign(N + 1, 0);
    for (int e = 0; e < L.edge_count; ++e) {
        L.node_edge_begin[L.edges[e * 2] + 1]++;
        L.node_edge_begin[L.edges[e * 2 + 1] + 1]++;
    }
    for (int n = 0; n < N; ++n) L.node_edge_begin[n + 1] += L.node_edge_begin[n];
    L.node_edge_list.assign(L.node_edge_begin[N], 0);
    {
        std::vector<int32_t> cursor(L.node_edge_begin.begin(), L.node_edge_begin.end() - 1);
        for (int e = 0; e < L.edge_count; ++e) {
            L.node_edge_list[cursor[L.edges[e * 2]]++] = e;
            L.node_edge_list[cursor[L.edges[e * 2 + 1]]++] = e;
        }
    }
    // node pairs sharing a vertex (the interactions_ map of
    // fused_assembly.cpp:68-79), grouped by (a, b) with a < b, and within a
    // group in the order the vertices' slot pairs (x < y) come.  The entry
    // code is v * 64 + (slot of a) * 8 + (slot of b).  Node a's entries come
    // from its gather list (vertex order); where a holds one slot of a vertex,
    // the slot pairs' order is the other slot's order.
    {
        size_t most = 0;
        for (int v = 0; v < V; ++v) most += static_cast<size_t>(L.bind_counts[v]) * (L.bind_counts[v] - 1) / 2;
        L.pair_entry.reserve(most);
        struct Tail { int32_t b, code; };
        struct Keyed { int key; Tail tail; };
        std::vector<Tail> run;               // node a's entries, in order
        std::vector<Keyed> several;
        std::vector<int32_t> at(N, 0);       // per b: entries, then the next place
        std::vector<int32_t> group_b;
        for (int a = 0; a < N; ++a) {
            const int32_t begin = L.gather_begin[a], end = L.gather_begin[a + 1];
            // a vertex adds at most its slot count: a bound for the run
            if (run.size() < static_cast<size_t>(end - begin) * NRICP_MAX_SLOTS)
                run.resize(static_cast<size_t>(end - begin) * NRICP_MAX_SLOTS);
            size_t n = 0;
            for (int32_t i = begin; i < end;) {
                const int v = L.gather_entry[i] / NRICP_MAX_SLOTS;
                int32_t j = i + 1;
                while (j < end && L.gather_entry[j] / NRICP_MAX_SLOTS == v) ++j;
                const int32_t* nodes = &L.bind_nodes[static_cast<size_t>(v) * NRICP_MAX_SLOTS];
                const int c = L.bind_counts[v];
                if (j == i + 1) {
                    // every slot written, the partners above a kept (no branch
                    // on the comparison: it goes either way at random)
                    const int sa = L.gather_entry[i] % NRICP_MAX_SLOTS;
                    for (int so = 0; so < c; ++so) {
                        run[n] = {nodes[so], v * 64 + sa * 8 + so};
                        n += nodes[so] > a;
                    }
                } else {  // a in several slots of v: order by the slot pair itself
                    several.clear();
                    for (int32_t k = i; k < j; ++k) {
                        const int sa = L.gather_entry[k] % NRICP_MAX_SLOTS;
                        for (int so = 0; so < c; ++so)
                            if (nodes[so] > a)
                                several.push_back({std::min(sa, so) * 8 + std::max(sa, so),
                                                   {nodes[so], v * 64 + sa * 8 + so}});
                    }
                    std::sort(several.begin(), several.end(),
                              [](const Keyed& x, const Keyed& y) { return x.key < y.key; });
                    for (const Keyed& e : several) run[n++] = e.tail;
                }
                i = j;
            }
            // stable grouping of the run by b, groups in ascending b
            group_b.clear();
            for (size_t k = 0; k < n; ++k)
                if (at[run[k].b]++ == 0) group_b.push_back(run[k].b);
            std::sort(group_b.begin(), group_b.end());
            int32_t place = static_cast<int32_t>(L.pair_entry.size());
            for (int32_t b : group_b) {
                L.pair_begin.push_back(place);
                L.pair_nodes.push_back(a);
                L.pair_nodes.push_back(b);
                const int32_t count = at[b];
                at[b] = place;
                place += count;
            }
            L.pair_entry.resize(place);
            for (size_t k = 0; k < n; ++k) L.pair_entry[at[run[k].b]++] = run[k].code;
            for (int32_t b : group_b) at[b] = 0;
        }
        L.pair_count = static_cast<int>(L.pair_nodes.size() / 2);
        L.pair_begin.push_back(static_cast<int32_t>(L.pair_entry.size()));
    }
    // off-diagonal blocks: one per node pair that shares a vertex (in pair
    // order), then one per smoothness edge whose pair shares none (in edge
    // order).  An edge whose pair shares a vertex adds into that pair's block,
    // so each node pair the system couples has exactly one block.
    L.offdiag_nodes = L.pair_nodes;
    L.edge_block.assign(L.edge_count, 0);
    for (int e = 0; e < L.edge_count; ++e) {
        const int a = L.edges[e * 2], b = L.edges[e * 2 + 1];
        int lo = 0, hi = L.pair_count;  // pairs are sorted by (a, b)
        while (lo < hi) {
            const int mid = (lo + hi) / 2;
            const int pa = L.pair_nodes[mid * 2], pb = L.pair_nodes[mid * 2 + 1];
            if (pa < a || (pa == a && pb < b)) lo = mid + 1; else hi = mid;
        }
        if (lo < L.pair_count && L.pair_nodes[lo * 2] == a && L.pair_nodes[lo * 2 + 1] == b) {
            L.edge_block[e] = lo;
        } else {
            L.edge_block[e] = static_cast<int32_t>(L.offdiag_nodes.size() / 2);
            L.offdiag_nodes.push_back(a);
            L.offdiag_nodes.push_back(b);
        }
    }
    const int B = static_cast<int>(L.offdiag_nodes.size() / 2);
    L.row_begin.assign(N + 1, 0);
    for (int k = 0; k < B; ++k) {
        L.row_begin[L.offdiag_nodes[k * 2] + 1]++;
        L.row_begin[L.offdiag_nodes[k * 2 + 1] + 1]++;
    }
    for (int n = 0; n < N; ++n) L.row_begin[n + 1] += L.row_begin[n];
    // entry pairs: (block * 2 + side, the other node of the block)
    L.row_entry.assign(static_cast<size_t>(L.row_begin[N]) * 2, 0);
    L.offdiag_slots.assign(static_cast<size_t>(B) * 2, 0);
    {
        std::vector<int32_t> cursor(L.row_begin.begin(), L.row_begin.end() - 1);
        for (int k = 0; k < B; ++k) {
            const int a = L.offdiag_nodes[k * 2], b = L.offdiag_nodes[k * 2 + 1];
            const int ia = cursor[a]++, ib = cursor[b]++;
            L.row_entry[ia * 2] = k * 2;
            L.row_entry[ia * 2 + 1] = b;
            L.row_entry[ib * 2] = k * 2 + 1;
            L.row_entry[ib * 2 + 1] = a;
            L.offdiag_slots[k * 2] = ia;       // block k, as seen from a: B
            L.offdiag_slots[k * 2 + 1] = ib;   // and from b: B^T
        }
    }
    // warm start from the previous level (deformation.cpp:141-160): the new
    // nodes bound to the old ones with the reference's four slots
    L.transfer_nodes.assign(static_cast<size_t>(N) * 4, 0);
    L.transfer_weights.assign(static_cast<size_t>(N) * 4, 0.0);
    L.transfer_counts.assign(N, 0);
    if (level > 0) {
        const GraphLevel& from = graph.levels[level - 1];
        const std::vector<Binding> tb = bind_vertices(g.rest, from.rest, 4, 4);
        for (int n = 0; n < N; ++n) {
            L.transfer_counts[n] = tb[n].count;
            for (int s = 0; s < 4; ++s) {
                L.transfer_nodes[n * 4 + s] = tb[n].nodes[s] < 0 ? 0 : tb[n].nodes[s];
                L.transfer_weights[n * 4 + s] = tb[n].weights[s];
            }
        }
    }
    return L;
}

void vertex_faces(const int32_t* faces, int m, int V, std::vector<int32_t>& begin,
                  std::vector<int32_t>& list) {
    begin.assign(V + 1, 0);
    for (int f = 0; f < m; ++f)
        for (int k = 0; k < 3; ++k) begin[faces[f * 3 + k] + 1]++;
    for (int v = 0; v < V; ++v) begin[v + 1] += begin[v];
    list.assign(begin[V], 0);
    std::vector<int32_t> cursor(begin.begin(), begin.end() - 1);
    for (int f = 0; f < m; ++f)
        for (int k = 0; k < 3; ++k) list[cursor[faces[f * 3 + k]]++] = f;
}

namespace {
std::string number(double value) {  // report.cpp:36-43
    if (!std::isfinite(value)) return "null";
    std::ostringstream out;
    out << std::setprecision(17) << value;
    return out.str();
}
}  // namespace

std::string report_json(const char* route, const char* precision, const double e[5],
                        const StatsView& c, const std::vector<LevelView>& levels,
                        const NricpSolveDesc& desc, double units, double setup_seconds,
                        double solve_seconds) {
    std::ostringstream out;  // report.cpp:46-105
    out << std::setprecision(17);
    out << "{\n";
    out << "  \"version\": \"0.1.0\",\n";
    out << "  \"route\": \"" << route << "\",\n";
    out << "  \"precision\": \"" << precision << "\",\n";
    out << "  \"setup_seconds\": " << number(setup_seconds) << ",\n";
    out << "  \"solve_seconds\": " << number(solve_seconds) << ",\n";
    out << "  \"energy\": {\n";
    out << "    \"point_to_point\": " << number(e[0]) << ",\n";
    out << "    \"point_to_plane\": " << number(e[1]) << ",\n";
    out << "    \"smoothness\": " << number(e[2]) << ",\n";
    out << "    \"anchor\": " << number(e[3]) << ",\n";
    out << "    \"landmark\": " << number(e[4]) << ",\n";
    out << "    \"total\": " << number(e[0] + e[1] + e[2] + e[3] + e[4]) << "\n";
    out << "  },\n";
    out << "  \"correspondence\": {\n";
    out << "    \"total\": " << c.total << ",\n";
    out << "    \"accepted\": " << c.accepted << ",\n";
    out << "    \"rejected_distance\": " << c.rejected_distance << ",\n";
    out << "    \"rejected_normal\": " << c.rejected_normal << ",\n";
    out << "    \"rejected_slope\": " << c.rejected_slope << ",\n";
    out << "    \"rejected_masked\": " << c.rejected_masked << ",\n";
    out << "    \"distance_mean\": " << number(c.mean) << ",\n";
    out << "    \"distance_p95\": " << number(c.p95) << ",\n";
    out << "    \"distance_max\": " << number(c.max) << "\n";
    out << "  },\n";
    out << "  \"levels\": [";
    for (size_t i = 0; i < levels.size(); ++i) {
        const LevelView& l = levels[i];
        out << (i == 0 ? "\n" : ",\n");
        out << "    {\"level\": " << l.level << ", \"nodes\": " << l.nodes
            << ", \"outer_iterations\": " << l.outer_iterations
            << ", \"inner_iterations\": " << l.inner_iterations
            << ", \"energy_start\": " << number(l.energy_start)
            << ", \"energy_end\": " << number(l.energy_end)
            << ", \"correspondence_mean\": " << number(l.correspondence_mean)
            << ", \"converged\": " << (l.converged ? "true" : "false") << "}";
    }
    out << (levels.empty() ? "],\n" : "\n  ],\n");
    out << "  \"settings\": {";
    bool first = true;
    const char* keys[6] = {"point_to_point", "point_to_plane", "smoothness", "anchor",
                           "landmark", "robust_threshold"};
    for (size_t l = 0; l < levels.size(); ++l) {
        NricpLevelSettings s;
        nricp_default_level(&s);
        if (desc.level_setting_count > 0)
            s = desc.levels[std::min<int>(static_cast<int>(l), desc.level_setting_count - 1)];
        const double robust = s.robust_threshold > 0.0 ? s.robust_threshold * units : s.robust_threshold;
        const double values[6] = {s.point_to_point, s.point_to_plane, s.smoothness, s.anchor,
                                  s.landmark, robust};
        for (int k = 0; k < 6; ++k) {
            out << (first ? "\n" : ",\n");
            first = false;
            out << "    \"level" << l << "_" << keys[k] << "\": " << number(values[k]);
        }
    }
    out << (first ? "}\n" : "\n  }\n");
    out << "}\n";
    return out.str();
}

}  // namespace nricp_b200
