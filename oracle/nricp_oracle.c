/*
 * CPU oracle for the nricp wrapping path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's FP64 route A and of the FP64 form of
 * its device route C, used as the checker for the CUDA path.  It is never
 * linked into, loaded by, or called from the product.  Function comments cite
 * the reference file:line each one restates; operation order follows the
 * reference so that double-precision results agree bit for bit where the
 * reference's own arithmetic is deterministic.
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared (see oracle/build.py).
 */
#include "nricp_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "block_cholesky.h"

#define KMAX NRICP_MAX_SLOTS
#define REF_KMAX 4 /* VertexBinding::kMaxNodes, src/core/sampling.h:17 */

static __thread char g_error[512];

static int fail(int code, const char* format, ...) {
    va_list args;
    va_start(args, format);
    vsnprintf(g_error, sizeof g_error, format, args);
    va_end(args);
    return code;
}

const char* oracle_last_error(void) { return g_error; }

/* ------------------------------------------------------------------------ */
/* Small vector algebra: src/core/vec3.h, mat3.h, rotation.h, quaternion.h    */
/* ------------------------------------------------------------------------ */

typedef struct { double x, y, z; } V3;
typedef struct { double m[9]; } M3;
typedef struct { double w, x, y, z; } Q4;

static V3 v3(double x, double y, double z) { V3 r = {x, y, z}; return r; }
static V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 scale(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 divide(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
static double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static double sqnorm(V3 a) { return dot(a, a); }
static double norm3(V3 a) { return sqrt(dot(a, a)); }
static V3 normalized(V3 a) { /* vec3.h:84-87 */
    const double length = norm3(a);
    return length > 0.0 ? divide(a, length) : v3(0, 0, 0);
}
static V3 load3(const double* p, size_t i) { return v3(p[i * 3], p[i * 3 + 1], p[i * 3 + 2]); }
static void store3(double* p, size_t i, V3 v) { p[i * 3] = v.x; p[i * 3 + 1] = v.y; p[i * 3 + 2] = v.z; }

static M3 identity3(void) { M3 r = {{1, 0, 0, 0, 1, 0, 0, 0, 1}}; return r; }
static V3 mulv(const M3* a, V3 v) { /* mat3.h:16-22 */
    return v3(a->m[0] * v.x + a->m[1] * v.y + a->m[2] * v.z,
              a->m[3] * v.x + a->m[4] * v.y + a->m[5] * v.z,
              a->m[6] * v.x + a->m[7] * v.y + a->m[8] * v.z);
}
static M3 mulm(const M3* a, const M3* b) { /* mat3.h:24-36 */
    M3 out;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double sum = 0.0;
            for (int k = 0; k < 3; ++k) sum += a->m[r * 3 + k] * b->m[k * 3 + c];
            out.m[r * 3 + c] = sum;
        }
    return out;
}
static M3 transposed(const M3* a) {
    M3 out;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) out.m[r * 3 + c] = a->m[c * 3 + r];
    return out;
}
static M3 skew(V3 w) { /* rotation.h:13-25 */
    M3 m = {{0.0, -w.z, w.y, w.z, 0.0, -w.x, -w.y, w.x, 0.0}};
    return m;
}
static M3 exp_so3(V3 omega) { /* rotation.h:29-47 */
    const double theta_squared = dot(omega, omega);
    const M3 hat = skew(omega);
    const M3 hat2 = mulm(&hat, &hat);
    M3 result = identity3();
    if (theta_squared < 1e-24) {
        for (int i = 0; i < 9; ++i) result.m[i] += hat.m[i] + 0.5 * hat2.m[i];
        return result;
    }
    const double theta = sqrt(theta_squared);
    const double a = sin(theta) / theta;
    const double b = (1.0 - cos(theta)) / theta_squared;
    for (int i = 0; i < 9; ++i) result.m[i] += a * hat.m[i] + b * hat2.m[i];
    return result;
}
static double qdot(Q4 a, Q4 b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }
static Q4 qscale(Q4 a, double s) { Q4 r = {a.w * s, a.x * s, a.y * s, a.z * s}; return r; }
static Q4 qnormalized(Q4 q) { /* quaternion.h:40-46 */
    const double length = sqrt(qdot(q, q));
    if (length <= 0.0) { Q4 r = {1, 0, 0, 0}; return r; }
    Q4 r = {q.w / length, q.x / length, q.y / length, q.z / length};
    return r;
}
static Q4 quaternion_from_matrix(const M3* m) { /* quaternion.h:49-76 */
    const double trace = m->m[0] + m->m[4] + m->m[8];
    Q4 q;
    if (trace > 0.0) {
        const double s = sqrt(trace + 1.0) * 2.0;
        q.w = 0.25 * s; q.x = (m->m[7] - m->m[5]) / s;
        q.y = (m->m[2] - m->m[6]) / s; q.z = (m->m[3] - m->m[1]) / s;
        return q;
    }
    if (m->m[0] > m->m[4] && m->m[0] > m->m[8]) {
        const double s = sqrt(1.0 + m->m[0] - m->m[4] - m->m[8]) * 2.0;
        q.w = (m->m[7] - m->m[5]) / s; q.x = 0.25 * s;
        q.y = (m->m[1] + m->m[3]) / s; q.z = (m->m[2] + m->m[6]) / s;
        return q;
    }
    if (m->m[4] > m->m[8]) {
        const double s = sqrt(1.0 + m->m[4] - m->m[0] - m->m[8]) * 2.0;
        q.w = (m->m[2] - m->m[6]) / s; q.x = (m->m[1] + m->m[3]) / s;
        q.y = 0.25 * s; q.z = (m->m[5] + m->m[7]) / s;
        return q;
    }
    const double s = sqrt(1.0 + m->m[8] - m->m[0] - m->m[4]) * 2.0;
    q.w = (m->m[3] - m->m[1]) / s; q.x = (m->m[2] + m->m[6]) / s;
    q.y = (m->m[5] + m->m[7]) / s; q.z = 0.25 * s;
    return q;
}
static M3 matrix_from_quaternion(Q4 q) { /* quaternion.h:78-94 */
    const double w = q.w, x = q.x, y = q.y, z = q.z;
    M3 m;
    m.m[0] = 1.0 - 2.0 * (y * y + z * z);
    m.m[1] = 2.0 * (x * y - z * w);
    m.m[2] = 2.0 * (x * z + y * w);
    m.m[3] = 2.0 * (x * y + z * w);
    m.m[4] = 1.0 - 2.0 * (x * x + z * z);
    m.m[5] = 2.0 * (y * z - x * w);
    m.m[6] = 2.0 * (x * z - y * w);
    m.m[7] = 2.0 * (y * z + x * w);
    m.m[8] = 1.0 - 2.0 * (x * x + y * y);
    return m;
}
static V3 log_so3(const M3* rotation) { /* rotation.h:51-63 */
    Q4 q = qnormalized(quaternion_from_matrix(rotation));
    if (q.w < 0.0) q = qscale(q, -1.0);
    const V3 vector = v3(q.x, q.y, q.z);
    const double length = norm3(vector);
    if (length < 1e-12) return v3(0, 0, 0);
    const double angle = 2.0 * atan2(length, q.w);
    return scale(vector, angle / length);
}
static M3 left_jacobian_inverse(V3 omega) { /* rotation.h:71-105 */
    const double theta_squared = dot(omega, omega);
    const M3 hat = skew(omega);
    const M3 hat2 = mulm(&hat, &hat);
    M3 result;
    if (theta_squared < 1e-12) {
        for (int i = 0; i < 9; ++i)
            result.m[i] = 1.0 * (i % 4 == 0 ? 1.0 : 0.0) + -0.5 * hat.m[i] +
                          (1.0 / 12.0) * hat2.m[i];
        return result;
    }
    const double theta = sqrt(theta_squared);
    if (theta > 3.14159265358979323846 - 1e-6) {
        for (int i = 0; i < 9; ++i) result.m[i] = (i % 4 == 0 ? 1.0 : 0.0) - 0.5 * hat.m[i];
        return result;
    }
    const double second =
        1.0 / theta_squared - (1.0 + cos(theta)) / (2.0 * theta * sin(theta));
    for (int i = 0; i < 9; ++i)
        result.m[i] = (i % 4 == 0 ? 1.0 : 0.0) - 0.5 * hat.m[i] + second * hat2.m[i];
    return result;
}

/* ------------------------------------------------------------------------ */
/* Mesh: src/core/mesh.cpp                                                   */
/* ------------------------------------------------------------------------ */

static void bounds_of(const double* p, int n, V3* lo, V3* hi) { /* mesh.cpp:47-64 */
    *lo = v3(0, 0, 0); *hi = v3(0, 0, 0);
    if (n <= 0) return;
    *lo = load3(p, 0); *hi = *lo;
    for (int i = 0; i < n; ++i) {
        const V3 v = load3(p, (size_t)i);
        lo->x = fmin(lo->x, v.x); lo->y = fmin(lo->y, v.y); lo->z = fmin(lo->z, v.z);
        hi->x = fmax(hi->x, v.x); hi->y = fmax(hi->y, v.y); hi->z = fmax(hi->z, v.z);
    }
}

void oracle_normalization(const double* points, int count, double center[3], double* s) {
    /* mesh.cpp:174-181 */
    V3 lo, hi;
    bounds_of(points, count, &lo, &hi);
    const V3 c = scale(add(lo, hi), 0.5);
    center[0] = c.x; center[1] = c.y; center[2] = c.z;
    const double diagonal = norm3(sub(hi, lo));
    *s = diagonal > 0.0 ? 1.0 / diagonal : 1.0;
}

static void apply_normalization(double* p, int n, const double center[3], double s) {
    const V3 c = v3(center[0], center[1], center[2]); /* mesh.cpp:183-187 */
    for (int i = 0; i < n; ++i) store3(p, (size_t)i, scale(sub(load3(p, (size_t)i), c), s));
}

void oracle_vertex_normals(const double* points, int point_count, const int32_t* faces,
                           int face_count, double* out) { /* mesh.cpp:71-88 */
    memset(out, 0, sizeof(double) * 3 * (size_t)point_count);
    for (int f = 0; f < face_count; ++f) {
        const V3 a = load3(points, (size_t)faces[f * 3]);
        const V3 b = load3(points, (size_t)faces[f * 3 + 1]);
        const V3 c = load3(points, (size_t)faces[f * 3 + 2]);
        const V3 w = cross(sub(b, a), sub(c, a));
        for (int k = 0; k < 3; ++k) {
            const size_t v = (size_t)faces[f * 3 + k];
            store3(out, v, add(load3(out, v), w));
        }
    }
    for (int i = 0; i < point_count; ++i) store3(out, (size_t)i, normalized(load3(out, (size_t)i)));
}

static int validate_mesh(const double* p, int n, const int32_t* f, int m, const char* what) {
    /* mesh.cpp:90-116 */
    if (n <= 0) return fail(NRICP_ERR_INVALID, "invalid %s mesh: mesh has no vertices", what);
    if (m <= 0)
        return fail(NRICP_ERR_INVALID,
                    "invalid %s mesh: mesh has no faces; closest-point queries need a surface", what);
    for (int i = 0; i < n; ++i)
        if (!isfinite(p[i * 3]) || !isfinite(p[i * 3 + 1]) || !isfinite(p[i * 3 + 2]))
            return fail(NRICP_ERR_INVALID, "invalid %s mesh: vertex %d is not finite", what, i);
    for (int i = 0; i < m; ++i)
        for (int k = 0; k < 3; ++k)
            if (f[i * 3 + k] < 0 || f[i * 3 + k] >= n)
                return fail(NRICP_ERR_INVALID,
                            "invalid %s mesh: face %d corner %d index %d is out of range", what,
                            i, k, f[i * 3 + k]);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Sampling and graph: src/core/sampling.cpp, src/core/graph.cpp             */
/* ------------------------------------------------------------------------ */

static double sqdist(V3 a, V3 b) { return sqnorm(sub(a, b)); } /* sampling.cpp:17-19 */

int oracle_farthest_point_seeds(const double* points, int count, int seeds, int first,
                                int32_t* out) { /* sampling.cpp:47-88 */
    if (count <= 0 || seeds <= 0) return 0;
    if (seeds > count) seeds = count;
    if (first < 0) first = 0;
    if (first > count - 1) first = count - 1;
    double* nearest = (double*)malloc(sizeof(double) * (size_t)count);
    int held = 0;
    out[held++] = first;
    int best = first;
    double best_squared = -1.0;
    const V3 f = load3(points, (size_t)first);
    for (int i = 0; i < count; ++i) {
        nearest[i] = sqdist(load3(points, (size_t)i), f);
        if (nearest[i] > best_squared) { best_squared = nearest[i]; best = i; }
    }
    while (held < seeds) {
        out[held++] = best;
        const V3 chosen = load3(points, (size_t)best);
        best_squared = -1.0;
        for (int i = 0; i < count; ++i) {
            const double d = sqdist(load3(points, (size_t)i), chosen);
            nearest[i] = nearest[i] < d ? nearest[i] : d; /* std::min */
            if (nearest[i] > best_squared) { best_squared = nearest[i]; best = i; }
        }
    }
    free(nearest);
    return held;
}

static void keep_nearest(double* sq, int* idx, int* held, int capacity, double value,
                         int entry) { /* sampling.cpp:23-42 */
    if (*held == capacity) {
        const int beats = value < sq[capacity - 1] ||
                          (value == sq[capacity - 1] && entry < idx[capacity - 1]);
        if (!beats) return;
    }
    int at = *held < capacity ? (*held)++ : capacity - 1;
    while (at > 0 && (sq[at - 1] > value || (sq[at - 1] == value && idx[at - 1] > entry))) {
        sq[at] = sq[at - 1];
        idx[at] = idx[at - 1];
        --at;
    }
    sq[at] = value;
    idx[at] = entry;
}

typedef struct {
    int nodes[KMAX];
    double weights[KMAX];
    int count;
} Binding;

static void bind_vertices(const double* vertices, int vertex_count, const double* nodes,
                          int node_count, int max_nodes, int slot_cap,
                          Binding* out) { /* sampling.cpp:90-143 */
    for (int v = 0; v < vertex_count; ++v) {
        for (int s = 0; s < KMAX; ++s) { out[v].nodes[s] = -1; out[v].weights[s] = 0.0; }
        out[v].count = 0;
    }
    if (node_count <= 0) return;
    int support = max_nodes < node_count ? max_nodes : node_count;
    if (support > slot_cap) support = slot_cap;
    if (support < 1) support = 1;
    double best_sq[KMAX];
    int best_idx[KMAX];
    for (int v = 0; v < vertex_count; ++v) {
        const V3 p = load3(vertices, (size_t)v);
        int held = 0;
        for (int n = 0; n < node_count; ++n)
            keep_nearest(best_sq, best_idx, &held, support, sqdist(p, load3(nodes, (size_t)n)), n);
        Binding b;
        for (int s = 0; s < KMAX; ++s) { b.nodes[s] = -1; b.weights[s] = 0.0; }
        b.count = support;
        const double dmax = sqrt(best_sq[support - 1]);
        double total = 0.0;
        for (int s = 0; s < support; ++s) {
            const double distance = sqrt(best_sq[s]);
            const double ratio = dmax > 0.0 ? distance / dmax : 0.0;
            const double falloff = 1.0 - ratio;
            b.nodes[s] = best_idx[s];
            b.weights[s] = falloff * falloff;
            total += b.weights[s];
        }
        for (int s = 0; s < support; ++s)
            b.weights[s] = total > 0.0 ? b.weights[s] / total : 1.0 / (double)support;
        out[v] = b;
    }
}

void oracle_bind_vertices(const double* vertices, int vertex_count, const double* nodes,
                          int node_count, int max_nodes, int32_t* out_nodes,
                          double* out_weights, int32_t* out_counts) {
    Binding* b = (Binding*)malloc(sizeof(Binding) * (size_t)(vertex_count > 0 ? vertex_count : 1));
    bind_vertices(vertices, vertex_count, nodes, node_count, max_nodes, KMAX, b);
    for (int v = 0; v < vertex_count; ++v) {
        for (int s = 0; s < KMAX; ++s) {
            out_nodes[v * KMAX + s] = b[v].nodes[s];
            out_weights[v * KMAX + s] = b[v].weights[s];
        }
        out_counts[v] = b[v].count;
    }
    free(b);
}

typedef struct { double d; int i; } DistIndex;
static int cmp_dist_index(const void* a, const void* b) {
    const DistIndex* x = (const DistIndex*)a;
    const DistIndex* y = (const DistIndex*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->i > y->i) - (x->i < y->i);
}
static int cmp_pair(const void* a, const void* b) {
    const int32_t* x = (const int32_t*)a;
    const int32_t* y = (const int32_t*)b;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    return (x[1] > y[1]) - (x[1] < y[1]);
}

int oracle_node_edges(const double* nodes, int node_count, int neighbours, int32_t* out,
                      int capacity) { /* graph.cpp:11-39 */
    if (node_count <= 1 || neighbours <= 0) return 0;
    const int taken = neighbours < node_count - 1 ? neighbours : node_count - 1;
    int32_t* pairs = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)node_count * (size_t)taken);
    DistIndex* d = (DistIndex*)malloc(sizeof(DistIndex) * (size_t)node_count);
    int count = 0;
    for (int n = 0; n < node_count; ++n) {
        int m = 0;
        for (int o = 0; o < node_count; ++o) {
            if (o == n) continue;
            d[m].d = norm3(sub(load3(nodes, (size_t)n), load3(nodes, (size_t)o)));
            d[m].i = o;
            ++m;
        }
        qsort(d, (size_t)m, sizeof(DistIndex), cmp_dist_index);
        for (int i = 0; i < taken; ++i) {
            const int o = d[i].i;
            pairs[count * 2] = n < o ? n : o;
            pairs[count * 2 + 1] = n < o ? o : n;
            ++count;
        }
    }
    qsort(pairs, (size_t)count, sizeof(int32_t) * 2, cmp_pair);
    int unique = 0;
    for (int i = 0; i < count; ++i) {
        if (unique > 0 && pairs[i * 2] == out[(unique - 1) * 2] &&
            pairs[i * 2 + 1] == out[(unique - 1) * 2 + 1])
            continue;
        if (unique >= capacity) { unique = -1; break; }
        out[unique * 2] = pairs[i * 2];
        out[unique * 2 + 1] = pairs[i * 2 + 1];
        ++unique;
    }
    free(pairs);
    free(d);
    return unique;
}

typedef struct {
    int node_count;
    double* rest;      /* node_count * 3 */
    int* tpl_index;
    Binding* bindings; /* vertex_count */
    int32_t* edges;    /* edge_count * 2 */
    int edge_count;
} Level;

typedef struct {
    double center[3];
    double scale;
    int level_count;
    Level* levels;
} Graph;

static int level_node_count(int level, int nodes_initial, int growth, int vertex_count) {
    /* graph.cpp:52-57 */
    const double g = pow((double)(growth > 1 ? growth : 1), (double)level);
    long requested = lround((double)nodes_initial * g);
    if (requested < 1) requested = 1;
    return requested < vertex_count ? (int)requested : vertex_count;
}

int oracle_plan(const NricpSolveDesc* desc, int32_t* level_nodes, int capacity) {
    const int levels = desc->graph_levels > 1 ? desc->graph_levels : 1;
    for (int l = 0; l < levels && l < capacity; ++l)
        level_nodes[l] = level_node_count(l, desc->nodes_initial, desc->growth,
                                          desc->template_vertex_count);
    return levels;
}

static void free_graph(Graph* g) {
    for (int l = 0; l < g->level_count; ++l) {
        free(g->levels[l].rest); free(g->levels[l].tpl_index);
        free(g->levels[l].bindings); free(g->levels[l].edges);
    }
    free(g->levels);
    memset(g, 0, sizeof *g);
}

static void build_graph(const double* normalized, int vertex_count, int levels,
                        int nodes_initial, int growth, int k, int edge_k,
                        Graph* g) { /* graph.cpp:41-76 */
    g->level_count = levels > 1 ? levels : 1;
    g->levels = (Level*)calloc((size_t)g->level_count, sizeof(Level));
    for (int l = 0; l < g->level_count; ++l) {
        Level* L = &g->levels[l];
        const int count = level_node_count(l, nodes_initial, growth, vertex_count);
        L->tpl_index = (int*)malloc(sizeof(int) * (size_t)count);
        int32_t* seeds = (int32_t*)malloc(sizeof(int32_t) * (size_t)count);
        L->node_count = oracle_farthest_point_seeds(normalized, vertex_count, count, 0, seeds);
        L->rest = (double*)malloc(sizeof(double) * 3 * (size_t)L->node_count);
        for (int n = 0; n < L->node_count; ++n) {
            L->tpl_index[n] = seeds[n];
            store3(L->rest, (size_t)n, load3(normalized, (size_t)seeds[n]));
        }
        free(seeds);
        L->bindings = (Binding*)malloc(sizeof(Binding) * (size_t)vertex_count);
        bind_vertices(normalized, vertex_count, L->rest, L->node_count, k, KMAX, L->bindings);
        const int cap = L->node_count * (edge_k > 0 ? edge_k : 1) + 1;
        L->edges = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)cap);
        L->edge_count = oracle_node_edges(L->rest, L->node_count, edge_k, L->edges, cap);
    }
}

/* ------------------------------------------------------------------------ */
/* Deformation: src/core/deformation.cpp                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    int node_count;
    const double* rest; /* borrowed */
    M3* rotation;
    V3* translation;
} Deformation;

static void deformation_init(Deformation* d, int n, const double* rest) {
    d->node_count = n;
    d->rest = rest;
    d->rotation = (M3*)malloc(sizeof(M3) * (size_t)(n > 0 ? n : 1));
    d->translation = (V3*)malloc(sizeof(V3) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) { d->rotation[i] = identity3(); d->translation[i] = v3(0, 0, 0); }
}
static void deformation_free(Deformation* d) { free(d->rotation); free(d->translation); }
static void deformation_copy(Deformation* dst, const Deformation* src) {
    dst->node_count = src->node_count;
    dst->rest = src->rest;
    memcpy(dst->rotation, src->rotation, sizeof(M3) * (size_t)src->node_count);
    memcpy(dst->translation, src->translation, sizeof(V3) * (size_t)src->node_count);
}
static V3 apply_node(const Deformation* d, int node, V3 p) { /* deformation.h:37-41 */
    const V3 rest = load3(d->rest, (size_t)node);
    return add(add(mulv(&d->rotation[node], sub(p, rest)), rest), d->translation[node]);
}
static void retract(Deformation* d, const double* delta) { /* deformation.cpp:19-32 */
    for (int n = 0; n < d->node_count; ++n) {
        const double* v = delta + (size_t)n * 6;
        const M3 e = exp_so3(v3(v[0], v[1], v[2]));
        d->rotation[n] = mulm(&e, &d->rotation[n]);
        d->translation[n] = add(d->translation[n], v3(v[3], v[4], v[5]));
    }
}
static V3 evaluate_point(V3 p, const Binding* b, const Deformation* d) { /* deformation.cpp:55-68 */
    V3 result = v3(0, 0, 0);
    for (int s = 0; s < b->count; ++s) {
        const int node = b->nodes[s];
        if (node < 0 || node >= d->node_count) continue;
        result = add(result, scale(apply_node(d, node, p), b->weights[s]));
    }
    return result;
}
static void evaluate_all(const double* pts, int n, const Binding* b, const Deformation* d,
                         double* out) {
    for (int i = 0; i < n; ++i) store3(out, (size_t)i, evaluate_point(load3(pts, (size_t)i), &b[i], d));
}

static void transfer_level(const Level* from, const Deformation* fd, const Level* to,
                           Deformation* out) { /* deformation.cpp:141-203 */
    deformation_init(out, to->node_count, to->rest);
    if (from->node_count <= 0 || to->node_count <= 0) return;
    Binding* sb = (Binding*)malloc(sizeof(Binding) * (size_t)to->node_count);
    bind_vertices(to->rest, to->node_count, from->rest, from->node_count, REF_KMAX, REF_KMAX, sb);
    for (int n = 0; n < to->node_count; ++n) {
        const Binding* b = &sb[n];
        if (b->count <= 0) continue;
        int heaviest = b->nodes[0];
        double heaviest_weight = b->weights[0];
        for (int s = 1; s < b->count; ++s)
            if (b->weights[s] > heaviest_weight) { heaviest_weight = b->weights[s]; heaviest = b->nodes[s]; }
        const Q4 reference = quaternion_from_matrix(&fd->rotation[heaviest]);
        Q4 blended = {0.0, 0.0, 0.0, 0.0};
        V3 position = v3(0, 0, 0);
        const V3 g = load3(to->rest, (size_t)n);
        for (int s = 0; s < b->count; ++s) {
            const int source = b->nodes[s];
            const double w = b->weights[s];
            Q4 r = quaternion_from_matrix(&fd->rotation[source]);
            if (qdot(r, reference) < 0.0) r = qscale(r, -1.0);
            const Q4 rw = qscale(r, w);
            blended.w += rw.w; blended.x += rw.x; blended.y += rw.y; blended.z += rw.z;
            position = add(position, scale(apply_node(fd, source, g), w));
        }
        const double length = sqrt(qdot(blended, blended));
        out->rotation[n] = length > 1e-8 ? matrix_from_quaternion(qnormalized(blended))
                                         : matrix_from_quaternion(reference);
        out->translation[n] = sub(position, g);
    }
    free(sb);
}

/* ------------------------------------------------------------------------ */
/* Closest points: src/geometry/closest_point.cpp                            */
/* ------------------------------------------------------------------------ */

static V3 closest_on_triangle(V3 p, V3 a, V3 b, V3 c, double* bary) { /* closest_point.cpp:24-121 */
    const V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { bary[0] = 1; bary[1] = 0; bary[2] = 0; return a; }
    const V3 bp = sub(p, b);
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { bary[0] = 0; bary[1] = 1; bary[2] = 0; return b; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double den = d1 - d3;
        const double v = den != 0.0 ? d1 / den : 0.0;
        bary[0] = 1.0 - v; bary[1] = v; bary[2] = 0.0;
        return add(a, scale(ab, v));
    }
    const V3 cp = sub(p, c);
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { bary[0] = 0; bary[1] = 0; bary[2] = 1; return c; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double den = d2 - d6;
        const double w = den != 0.0 ? d2 / den : 0.0;
        bary[0] = 1.0 - w; bary[1] = 0.0; bary[2] = w;
        return add(a, scale(ac, w));
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double den = (d4 - d3) + (d5 - d6);
        const double w = den != 0.0 ? (d4 - d3) / den : 0.0;
        bary[0] = 0.0; bary[1] = 1.0 - w; bary[2] = w;
        return add(b, scale(sub(c, b), w));
    }
    const double den = va + vb + vc;
    if (fabs(den) < 1e-300) { bary[0] = 1; bary[1] = 0; bary[2] = 0; return a; }
    const double v = vb / den, w = vc / den;
    bary[0] = 1.0 - v - w; bary[1] = v; bary[2] = w;
    return add(add(a, scale(ab, v)), scale(ac, w));
}

typedef struct { V3 lo, hi; int left, right, begin, count; } BNode;
typedef struct {
    const double* points; const int32_t* faces; int face_count;
    double* vnormals; V3 *ca, *cb, *cc, *centroid;
    int* order; BNode* nodes; int node_count; int root;
} Target;

static double sq_to_box(V3 p, V3 lo, V3 hi) { /* closest_point.cpp:13-20 */
    const V3 c = v3(fmin(fmax(p.x, lo.x), hi.x), fmin(fmax(p.y, lo.y), hi.y),
                    fmin(fmax(p.z, lo.z), hi.z));
    return sqnorm(sub(p, c));
}

static int g_axis;
static const V3* g_centroids;
static double coordinate_of(int t) {
    const V3 c = g_centroids[t];
    return g_axis == 0 ? c.x : (g_axis == 1 ? c.y : c.z);
}
static int cmp_by_axis(const void* a, const void* b) {
    const int x = *(const int*)a, y = *(const int*)b;
    const double cx = coordinate_of(x), cy = coordinate_of(y);
    if (cx < cy) return -1;
    if (cx > cy) return 1;
    return (x > y) - (x < y);
}

static int target_build(Target* t, int begin, int end) { /* closest_point.cpp:161-225 */
    BNode node;
    node.lo = t->ca[t->order[begin]]; node.hi = node.lo;
    for (int i = begin; i < end; ++i) {
        const int tri = t->order[i];
        const V3 cs[3] = {t->ca[tri], t->cb[tri], t->cc[tri]};
        for (int k = 0; k < 3; ++k) {
            node.lo.x = fmin(node.lo.x, cs[k].x); node.lo.y = fmin(node.lo.y, cs[k].y);
            node.lo.z = fmin(node.lo.z, cs[k].z); node.hi.x = fmax(node.hi.x, cs[k].x);
            node.hi.y = fmax(node.hi.y, cs[k].y); node.hi.z = fmax(node.hi.z, cs[k].z);
        }
    }
    node.left = node.right = -1; node.begin = 0; node.count = 0;
    const int index = t->node_count++;
    t->nodes[index] = node;
    const int count = end - begin;
    if (count <= 8) {
        t->nodes[index].begin = begin;
        t->nodes[index].count = count;
        return index;
    }
    V3 cmin = t->centroid[t->order[begin]], cmax = cmin;
    for (int i = begin; i < end; ++i) {
        const V3 c = t->centroid[t->order[i]];
        cmin.x = fmin(cmin.x, c.x); cmin.y = fmin(cmin.y, c.y); cmin.z = fmin(cmin.z, c.z);
        cmax.x = fmax(cmax.x, c.x); cmax.y = fmax(cmax.y, c.y); cmax.z = fmax(cmax.z, c.z);
    }
    const V3 e = sub(cmax, cmin);
    int axis = 0;
    if (e.y > e.x && e.y >= e.z) axis = 1;
    else if (e.z > e.x && e.z > e.y) axis = 2;
    /* nth_element under a strict total order: the two halves are unique sets;
     * a full sort gives the same halves. */
    g_axis = axis;
    g_centroids = t->centroid;
    qsort(t->order + begin, (size_t)count, sizeof(int), cmp_by_axis);
    const int middle = begin + count / 2;
    const int left = target_build(t, begin, middle);
    const int right = target_build(t, middle, end);
    t->nodes[index].left = left;
    t->nodes[index].right = right;
    return index;
}

static void target_init(Target* t, const double* points, int point_count,
                        const int32_t* faces, int face_count) { /* closest_point.cpp:123-159 */
    memset(t, 0, sizeof *t);
    t->points = points; t->faces = faces; t->face_count = face_count;
    t->vnormals = (double*)calloc((size_t)point_count * 3 + 3, sizeof(double));
    t->ca = (V3*)malloc(sizeof(V3) * (size_t)face_count);
    t->cb = (V3*)malloc(sizeof(V3) * (size_t)face_count);
    t->cc = (V3*)malloc(sizeof(V3) * (size_t)face_count);
    t->centroid = (V3*)malloc(sizeof(V3) * (size_t)face_count);
    t->order = (int*)malloc(sizeof(int) * (size_t)face_count);
    for (int f = 0; f < face_count; ++f) {
        const V3 a = load3(points, (size_t)faces[f * 3]);
        const V3 b = load3(points, (size_t)faces[f * 3 + 1]);
        const V3 c = load3(points, (size_t)faces[f * 3 + 2]);
        t->ca[f] = a; t->cb[f] = b; t->cc[f] = c;
        t->centroid[f] = divide(add(add(a, b), c), 3.0);
        t->order[f] = f;
        const V3 w = cross(sub(b, a), sub(c, a));
        for (int k = 0; k < 3; ++k) {
            const size_t v = (size_t)faces[f * 3 + k];
            store3(t->vnormals, v, add(load3(t->vnormals, v), w));
        }
    }
    for (int i = 0; i < point_count; ++i)
        store3(t->vnormals, (size_t)i, normalized(load3(t->vnormals, (size_t)i)));
    t->nodes = (BNode*)malloc(sizeof(BNode) * (size_t)(2 * face_count + 1));
    t->root = face_count > 0 ? target_build(t, 0, face_count) : -1;
}

static void target_free(Target* t) {
    free(t->vnormals); free(t->ca); free(t->cb); free(t->cc); free(t->centroid);
    free(t->order); free(t->nodes);
}

typedef struct { V3 point, normal; double distance; int triangle; } Closest;

static void consider(const Target* t, int tri, V3 p, double* best_sq, Closest* best) {
    double bary[3] = {1.0, 0.0, 0.0};
    const V3 c = closest_on_triangle(p, t->ca[tri], t->cb[tri], t->cc[tri], bary);
    const double d = sqnorm(sub(c, p));
    if (d < *best_sq) {
        *best_sq = d;
        best->point = c;
        best->distance = sqrt(d);
        best->triangle = tri;
        const int32_t* f = t->faces + tri * 3;
        best->normal = normalized(add(add(scale(load3(t->vnormals, (size_t)f[0]), bary[0]),
                                          scale(load3(t->vnormals, (size_t)f[1]), bary[1])),
                                      scale(load3(t->vnormals, (size_t)f[2]), bary[2])));
    }
}

static void query_node(const Target* t, int ni, V3 p, double* best_sq, Closest* best) {
    /* closest_point.cpp:227-262 */
    const BNode* node = &t->nodes[ni];
    if (sq_to_box(p, node->lo, node->hi) > *best_sq) return;
    if (node->left < 0) {
        for (int i = node->begin; i < node->begin + node->count; ++i)
            consider(t, t->order[i], p, best_sq, best);
        return;
    }
    const double ld = sq_to_box(p, t->nodes[node->left].lo, t->nodes[node->left].hi);
    const double rd = sq_to_box(p, t->nodes[node->right].lo, t->nodes[node->right].hi);
    const int first = ld <= rd ? node->left : node->right;
    const int second = first == node->left ? node->right : node->left;
    query_node(t, first, p, best_sq, best);
    query_node(t, second, p, best_sq, best);
}

static Closest target_query(const Target* t, V3 p, int brute) {
    Closest best;
    best.point = v3(0, 0, 0); best.normal = v3(0, 0, 0); best.distance = 0.0; best.triangle = -1;
    double best_sq = INFINITY;
    if (t->root < 0) return best;
    if (brute) {
        for (int tri = 0; tri < t->face_count; ++tri) consider(t, tri, p, &best_sq, &best);
    } else {
        query_node(t, t->root, p, &best_sq, &best);
    }
    return best;
}

void oracle_closest_points(const double* points, int point_count, const int32_t* faces,
                           int face_count, const double* queries, int query_count, int brute,
                           double* out_points, double* out_normals, double* out_distances,
                           int32_t* out_triangles) {
    Target t;
    target_init(&t, points, point_count, faces, face_count);
    for (int q = 0; q < query_count; ++q) {
        const Closest c = target_query(&t, load3(queries, (size_t)q), brute);
        store3(out_points, (size_t)q, c.point);
        store3(out_normals, (size_t)q, c.normal);
        out_distances[q] = c.distance;
        out_triangles[q] = c.triangle;
    }
    target_free(&t);
}

/* ------------------------------------------------------------------------ */
/* Correspondences and robust weights: src/solver/correspondence.cpp,        */
/* src/energy/robust.cpp, src/solver/route_a.cpp:19-38                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    int total, accepted, rejected_distance, rejected_normal, rejected_slope, rejected_masked;
    double mean, p95, max;
} Counts;

typedef struct {
    double* point;  /* V*3 */
    double* normal; /* V*3 */
    double* robust; /* V   */
    unsigned char* accepted;
} CorrSet;

static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

static double robust_weight(int kernel, double squared, double threshold) { /* robust.cpp:30-58 */
    if (squared < 0.0) squared = 0.0;
    if (kernel == NRICP_ROBUST_HUBER) {
        if (threshold <= 0.0) return 1.0;
        const double t2 = threshold * threshold;
        if (squared <= t2) return 1.0;
        return threshold / sqrt(squared);
    }
    if (kernel == NRICP_ROBUST_GEMAN_MCCLURE) {
        if (threshold <= 0.0) return 1.0;
        const double ratio = squared / (threshold * threshold);
        const double den = 1.0 + ratio;
        return 1.0 / (den * den);
    }
    return 1.0;
}

/* find_correspondences (correspondence.cpp:18-96) followed by
 * build_correspondences (route_a.cpp:19-38). */
static Counts correspond(const Target* t, const double* deformed, const double* qnormals,
                         int n, const NricpSolveDesc* desc, double distance_threshold,
                         int kernel, double robust_threshold, CorrSet* out) {
    Counts c;
    memset(&c, 0, sizeof c);
    double* accepted_d = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    int na = 0;
    for (int i = 0; i < n; ++i) {
        out->accepted[i] = 0;
        out->robust[i] = 1.0;
        store3(out->point, (size_t)i, v3(0, 0, 0));
        store3(out->normal, (size_t)i, v3(0, 0, 0));
        if (desc->mask && !desc->mask[i]) {
            c.rejected_masked++;
            c.total++;
            continue;
        }
        const V3 q = load3(deformed, (size_t)i);
        const Closest cl = target_query(t, q, 0);
        int rejection = 0;
        if (cl.distance > distance_threshold) {
            rejection = 1;
        } else if (dot(load3(qnormals, (size_t)i), cl.normal) < desc->min_normal_cosine) {
            rejection = 2;
        } else if (cl.distance > 0.0) {
            const V3 offset = sub(q, cl.point);
            const double slope = fabs(dot(cl.normal, offset)) / cl.distance;
            if (slope < desc->min_slope) rejection = 3;
        }
        c.total++;
        if (rejection == 0) {
            c.accepted++;
            accepted_d[na++] = cl.distance;
            out->accepted[i] = 1;
            store3(out->point, (size_t)i, cl.point);
            store3(out->normal, (size_t)i, cl.normal);
            const double sq = sqnorm(sub(q, cl.point));
            out->robust[i] = robust_threshold > 0.0 ? robust_weight(kernel, sq, robust_threshold) : 1.0;
        } else if (rejection == 1) c.rejected_distance++;
        else if (rejection == 2) c.rejected_normal++;
        else c.rejected_slope++;
    }
    if (na > 0) {
        qsort(accepted_d, (size_t)na, sizeof(double), cmp_double);
        double sum = 0.0;
        for (int i = 0; i < na; ++i) sum += accepted_d[i];
        c.mean = sum / na;
        double pi = 0.95 * (double)(na - 1);
        if (pi > (double)(na - 1)) pi = (double)(na - 1);
        c.p95 = accepted_d[(size_t)pi];
        c.max = accepted_d[na - 1];
    }
    free(accepted_d);
    return c;
}

/* ------------------------------------------------------------------------ */
/* Fused assembly: src/solver/fused_assembly.cpp                             */
/* ------------------------------------------------------------------------ */

typedef struct {
    int node_count;
    double* diag; /* N*36 */
    double* rhs;  /* N*6 */
    int off_count;
    int32_t* off_a; int32_t* off_b; /* sorted unique keys */
    double* off; /* off_count*36 */
    double energies[5];
    int with_jacobians;
} System;

typedef struct {
    const double* points; int vertex_count;
    const Binding* bindings;
    const Deformation* d;
    const double* node_positions;
    const CorrSet* corr;
    const int32_t* edges; int edge_count;
    const int32_t* lm_idx; const double* lm_tgt; int lm_count;
    const unsigned char* mask;
    double w[5];
} Inputs;

static int find_key(const System* s, int a, int b) {
    int lo = 0, hi = s->off_count;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (s->off_a[mid] < a || (s->off_a[mid] == a && s->off_b[mid] < b)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static void add_row(System* s, int kind, const int* nodes, double jac[][6], int slots,
                    double value) { /* fused_assembly.cpp:26-66 */
    s->energies[kind] += value * value;
    if (!s->with_jacobians) return;
    for (int slot = 0; slot < slots; ++slot) {
        const int node = nodes[slot];
        if (node < 0 || node >= s->node_count) continue;
        double* D = s->diag + (size_t)node * 36;
        for (int r = 0; r < 6; ++r) {
            for (int c = 0; c < 6; ++c) D[r * 6 + c] += jac[slot][r] * jac[slot][c];
            s->rhs[(size_t)node * 6 + r] -= jac[slot][r] * value;
        }
        for (int other = slot + 1; other < slots; ++other) {
            const int on = nodes[other];
            if (on < 0 || on >= s->node_count) continue;
            const int ka = node < on ? node : on, kb = node < on ? on : node;
            const int k = find_key(s, ka, kb);
            double* B = s->off + (size_t)k * 36;
            for (int r = 0; r < 6; ++r)
                for (int c = 0; c < 6; ++c)
                    B[r * 6 + c] += node < on ? jac[slot][r] * jac[other][c]
                                              : jac[other][r] * jac[slot][c];
        }
    }
}

static Binding usable_binding(const Binding* b, int node_count) { /* fused_assembly.cpp:85-98 */
    Binding c;
    for (int s = 0; s < KMAX; ++s) { c.nodes[s] = -1; c.weights[s] = 0.0; }
    c.count = 0;
    for (int s = 0; s < b->count; ++s) {
        const int node = b->nodes[s];
        if (node < 0 || node >= node_count || b->weights[s] == 0.0) continue;
        c.nodes[c.count] = node;
        c.weights[c.count] = b->weights[s];
        c.count++;
    }
    return c;
}

static void fill_linear_row(V3 lambda, V3 rotated, double weight, double row[6]) {
    /* fused_assembly.cpp:106-116 */
    const V3 rp = cross(lambda, rotated);
    row[0] = -weight * rp.x; row[1] = -weight * rp.y; row[2] = -weight * rp.z;
    row[3] = weight * lambda.x; row[4] = weight * lambda.y; row[5] = weight * lambda.z;
}

static V3 node_offset(const Deformation* d, int node, V3 p) { /* fused_assembly.cpp:100-104 */
    return mulv(&d->rotation[node], sub(p, load3(d->rest, (size_t)node)));
}

static const V3 AXES[3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};

static void offset_rows(System* s, int kind, const Binding* b, const Deformation* d, V3 rest,
                        V3 deformed, V3 target, double sc) { /* fused_assembly.cpp:118-143 */
    const V3 offset = scale(sub(deformed, target), sc);
    for (int row = 0; row < 3; ++row) {
        double jac[KMAX][6];
        memset(jac, 0, sizeof jac);
        for (int slot = 0; slot < b->count; ++slot)
            fill_linear_row(AXES[row], node_offset(d, b->nodes[slot], rest),
                            sc * b->weights[slot], jac[slot]);
        const double value = row == 0 ? offset.x : row == 1 ? offset.y : offset.z;
        add_row(s, kind, b->nodes, jac, b->count, value);
    }
}

/* Enumerates the off-diagonal keys the pass below will touch (the keys of
 * std::map interactions_ in fused_assembly.cpp:68-79). */
static void collect_keys(const Inputs* in, System* s) {
    const int N = in->d->node_count;
    int cap = 64, count = 0;
    int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)cap);
#define PUSH_KEY(p, q)                                                          \
    do {                                                                        \
        if (count == cap) {                                                     \
            cap *= 2;                                                           \
            keys = (int32_t*)realloc(keys, sizeof(int32_t) * 2 * (size_t)cap);  \
        }                                                                       \
        keys[count * 2] = (p) < (q) ? (p) : (q);                                \
        keys[count * 2 + 1] = (p) < (q) ? (q) : (p);                            \
        ++count;                                                                \
    } while (0)
    const int data = in->w[0] > 0.0 || in->w[1] > 0.0;
    for (int v = 0; v < in->vertex_count && data; ++v) {
        if (!in->corr->accepted[v] || (in->mask && !in->mask[v])) continue;
        const Binding b = usable_binding(&in->bindings[v], N);
        for (int x = 0; x < b.count; ++x)
            for (int y = x + 1; y < b.count; ++y)
                if (b.nodes[x] != b.nodes[y]) PUSH_KEY(b.nodes[x], b.nodes[y]);
    }
    if (in->w[2] > 0.0)
        for (int e = 0; e < in->edge_count; ++e) {
            const int a = in->edges[e * 2], b = in->edges[e * 2 + 1];
            if (a < 0 || b < 0 || a >= N || b >= N || a == b) continue;
            PUSH_KEY(a, b);
        }
    if (in->w[4] > 0.0)
        for (int l = 0; l < in->lm_count; ++l) {
            const int v = in->lm_idx[l];
            if (v < 0 || v >= in->vertex_count) continue;
            const Binding b = usable_binding(&in->bindings[v], N);
            for (int x = 0; x < b.count; ++x)
                for (int y = x + 1; y < b.count; ++y)
                    if (b.nodes[x] != b.nodes[y]) PUSH_KEY(b.nodes[x], b.nodes[y]);
        }
#undef PUSH_KEY
    qsort(keys, (size_t)count, sizeof(int32_t) * 2, cmp_pair);
    int unique = 0;
    for (int i = 0; i < count; ++i) {
        if (unique > 0 && keys[i * 2] == keys[(unique - 1) * 2] &&
            keys[i * 2 + 1] == keys[(unique - 1) * 2 + 1])
            continue;
        keys[unique * 2] = keys[i * 2];
        keys[unique * 2 + 1] = keys[i * 2 + 1];
        ++unique;
    }
    s->off_count = unique;
    s->off_a = (int32_t*)malloc(sizeof(int32_t) * (size_t)(unique + 1));
    s->off_b = (int32_t*)malloc(sizeof(int32_t) * (size_t)(unique + 1));
    s->off = (double*)calloc((size_t)(unique + 1) * 36, sizeof(double));
    for (int i = 0; i < unique; ++i) { s->off_a[i] = keys[i * 2]; s->off_b[i] = keys[i * 2 + 1]; }
    free(keys);
}

static void system_free(System* s) {
    free(s->diag); free(s->rhs); free(s->off_a); free(s->off_b); free(s->off);
    memset(s, 0, sizeof *s);
}

static void run_fused(const Inputs* in, int with_jacobians, System* s) { /* fused_assembly.cpp:159-291 */
    const int N = in->d->node_count;
    memset(s, 0, sizeof *s);
    s->node_count = N;
    s->with_jacobians = with_jacobians;
    s->diag = (double*)calloc((size_t)(N > 0 ? N : 1) * 36, sizeof(double));
    s->rhs = (double*)calloc((size_t)(N > 0 ? N : 1) * 6, sizeof(double));
    if (with_jacobians) collect_keys(in, s);
    const Deformation* d = in->d;
    for (int v = 0; v < in->vertex_count; ++v) {
        if (!in->corr->accepted[v] || (in->mask && !in->mask[v])) continue;
        const Binding b = usable_binding(&in->bindings[v], N);
        if (b.count <= 0) continue;
        const V3 rest = load3(in->points, (size_t)v);
        const V3 deformed = evaluate_point(rest, &b, d);
        const double robust = fmax(0.0, in->corr->robust[v]);
        const V3 cp = load3(in->corr->point, (size_t)v);
        if (in->w[0] > 0.0)
            offset_rows(s, 0, &b, d, rest, deformed, cp, sqrt(in->w[0] * robust));
        if (in->w[1] > 0.0) {
            const double sc = sqrt(in->w[1] * robust);
            const V3 nrm = load3(in->corr->normal, (size_t)v);
            double jac[KMAX][6];
            memset(jac, 0, sizeof jac);
            for (int slot = 0; slot < b.count; ++slot)
                fill_linear_row(nrm, node_offset(d, b.nodes[slot], rest), sc * b.weights[slot],
                                jac[slot]);
            add_row(s, 1, b.nodes, jac, b.count, sc * dot(nrm, sub(deformed, cp)));
        }
    }
    if (in->w[2] > 0.0) {
        const double sc = sqrt(in->w[2]);
        for (int e = 0; e < in->edge_count; ++e) {
            const int a = in->edges[e * 2], b = in->edges[e * 2 + 1];
            if (a < 0 || b < 0 || a >= N || b >= N) continue;
            const V3 na = load3(in->node_positions, (size_t)a);
            const V3 nb = load3(in->node_positions, (size_t)b);
            const V3 diff = scale(sub(apply_node(d, a, nb), apply_node(d, b, nb)), sc);
            const V3 rotated = mulv(&d->rotation[a], sub(nb, na));
            const int nodes[2] = {a, b};
            for (int row = 0; row < 3; ++row) {
                double jac[KMAX][6];
                memset(jac, 0, sizeof jac);
                fill_linear_row(AXES[row], rotated, sc, jac[0]);
                jac[1][row + 3] = -sc;
                const double value = row == 0 ? diff.x : row == 1 ? diff.y : diff.z;
                add_row(s, 2, nodes, jac, 2, value);
            }
        }
    }
    if (in->w[3] > 0.0) {
        const double sc = sqrt(in->w[3]);
        for (int n = 0; n < N; ++n) {
            const V3 omega = log_so3(&d->rotation[n]);
            const M3 rj = left_jacobian_inverse(omega);
            const V3 t = d->translation[n];
            const int nodes[1] = {n};
            for (int row = 0; row < 6; ++row) {
                double jac[KMAX][6];
                memset(jac, 0, sizeof jac);
                if (row < 3) {
                    for (int c = 0; c < 3; ++c) jac[0][c] = sc * rj.m[row * 3 + c];
                } else {
                    jac[0][row] = sc;
                }
                const double value = sc * (row == 0   ? omega.x
                                           : row == 1 ? omega.y
                                           : row == 2 ? omega.z
                                           : row == 3 ? t.x
                                           : row == 4 ? t.y
                                                      : t.z);
                add_row(s, 3, nodes, jac, 1, value);
            }
        }
    }
    if (in->w[4] > 0.0) {
        const double sc = sqrt(in->w[4]);
        for (int l = 0; l < in->lm_count; ++l) {
            const int v = in->lm_idx[l];
            if (v < 0 || v >= in->vertex_count) continue;
            const Binding b = usable_binding(&in->bindings[v], N);
            if (b.count <= 0) continue;
            const V3 rest = load3(in->points, (size_t)v);
            const V3 deformed = evaluate_point(rest, &b, d);
            offset_rows(s, 4, &b, d, rest, deformed, load3(in->lm_tgt, (size_t)l), sc);
        }
    }
}

static double total_energy(const double e[5]) {
    return e[0] + e[1] + e[2] + e[3] + e[4];
}

/* Energies the way block_energies sums them (energy.cpp:124-311 +
 * 313-348): per block first, then into the kind. */
static void block_energies(const Inputs* in, double e[5]) {
    memset(e, 0, sizeof(double) * 5);
    const int N = in->d->node_count;
    const Deformation* d = in->d;
    for (int v = 0; v < in->vertex_count; ++v) {
        if (!in->corr->accepted[v] || (in->mask && !in->mask[v])) continue;
        const Binding b = usable_binding(&in->bindings[v], N);
        if (b.count <= 0) continue;
        const V3 rest = load3(in->points, (size_t)v);
        const V3 deformed = evaluate_point(rest, &b, d);
        const double robust = fmax(0.0, in->corr->robust[v]);
        const V3 cp = load3(in->corr->point, (size_t)v);
        if (in->w[0] > 0.0) {
            const V3 o = scale(sub(deformed, cp), sqrt(in->w[0] * robust));
            e[0] += (0.0 + o.x * o.x + o.y * o.y) + o.z * o.z;
        }
        if (in->w[1] > 0.0) {
            const double val = sqrt(in->w[1] * robust) * dot(load3(in->corr->normal, (size_t)v),
                                                             sub(deformed, cp));
            e[1] += 0.0 + val * val;
        }
    }
    if (in->w[2] > 0.0) {
        const double sc = sqrt(in->w[2]);
        for (int e2 = 0; e2 < in->edge_count; ++e2) {
            const int a = in->edges[e2 * 2], b = in->edges[e2 * 2 + 1];
            if (a < 0 || b < 0 || a >= N || b >= N) continue;
            const V3 nb = load3(in->node_positions, (size_t)b);
            const V3 diff = scale(sub(apply_node(d, a, nb), apply_node(d, b, nb)), sc);
            e[2] += (0.0 + diff.x * diff.x + diff.y * diff.y) + diff.z * diff.z;
        }
    }
    if (in->w[3] > 0.0) {
        const double sc = sqrt(in->w[3]);
        for (int n = 0; n < N; ++n) {
            const V3 om = log_so3(&d->rotation[n]);
            const V3 t = d->translation[n];
            const double vals[6] = {sc * om.x, sc * om.y, sc * om.z, sc * t.x, sc * t.y, sc * t.z};
            double s = 0.0;
            for (int r = 0; r < 6; ++r) s += vals[r] * vals[r];
            e[3] += s;
        }
    }
    if (in->w[4] > 0.0) {
        const double sc = sqrt(in->w[4]);
        for (int l = 0; l < in->lm_count; ++l) {
            const int v = in->lm_idx[l];
            if (v < 0 || v >= in->vertex_count) continue;
            const Binding b = usable_binding(&in->bindings[v], N);
            if (b.count <= 0) continue;
            const V3 rest = load3(in->points, (size_t)v);
            const V3 o = scale(sub(evaluate_point(rest, &b, d), load3(in->lm_tgt, (size_t)l)), sc);
            e[4] += (0.0 + o.x * o.x + o.y * o.y) + o.z * o.z;
        }
    }
}

/* damped(): normal_equations.cpp:81-96 */
static void damp(System* s, double lambda, int diagonal_scaling) {
    if (lambda <= 0.0) return;
    for (int n = 0; n < s->node_count; ++n) {
        double* D = s->diag + (size_t)n * 36;
        for (int r = 0; r < 6; ++r) {
            const double sc = diagonal_scaling ? fmax(D[r * 6 + r], 1e-12) : 1.0;
            D[r * 6 + r] += lambda * sc;
        }
    }
}

static int solve_damped(const System* s, double lambda, int diagonal_scaling, double* delta) {
    double* D = (double*)malloc(sizeof(double) * 36 * (size_t)(s->node_count > 0 ? s->node_count : 1));
    memcpy(D, s->diag, sizeof(double) * 36 * (size_t)s->node_count);
    System tmp = *s;
    tmp.diag = D;
    damp(&tmp, lambda, diagonal_scaling);
    const int ok = block_cholesky_solve(s->node_count, D, s->off_count, s->off_a, s->off_b,
                                        s->off, s->rhs, delta);
    free(D);
    return ok;
}

int oracle_solve_direct(int node_count, const double* diagonal, int off_count,
                        const int32_t* off_a, const int32_t* off_b, const double* off_blocks,
                        const double* rhs, double damping, int diagonal_scaling, double* delta) {
    System s;
    memset(&s, 0, sizeof s);
    s.node_count = node_count;
    s.diag = (double*)diagonal;
    s.rhs = (double*)rhs;
    s.off_count = off_count;
    s.off_a = (int32_t*)off_a;
    s.off_b = (int32_t*)off_b;
    s.off = (double*)off_blocks;
    return solve_damped(&s, damping, diagonal_scaling, delta);
}

/* The statistics step of find_correspondences (correspondence.cpp:59-94):
 * tally each outcome; sort the accepted distances ascending, sum them in that
 * order for the mean, take element floor(min(n - 1, 0.95 (n - 1))) as the
 * 95th percentile and the last as the maximum. */
void oracle_summarize(int count, const uint8_t* codes, const double* distances,
                      int32_t counts[6], double stats[3]) {
    for (int k = 0; k < 6; ++k) counts[k] = 0;
    stats[0] = stats[1] = stats[2] = 0.0;
    double* accepted = (double*)malloc(sizeof(double) * (size_t)(count > 0 ? count : 1));
    int na = 0;
    for (int i = 0; i < count; ++i) {
        const int code = codes[i];
        if (code > 4) continue;
        counts[0]++;
        counts[code == 0 ? 1 : code + 1]++;
        if (code == 0) accepted[na++] = distances[i];
    }
    if (na > 0) {
        qsort(accepted, (size_t)na, sizeof(double), cmp_double);
        double sum = 0.0;
        for (int i = 0; i < na; ++i) sum += accepted[i];
        stats[0] = sum / na;
        double pi = 0.95 * (double)(na - 1);
        if (pi > (double)(na - 1)) pi = (double)(na - 1);
        stats[1] = accepted[(size_t)pi];
        stats[2] = accepted[na - 1];
    }
    free(accepted);
}

/* ------------------------------------------------------------------------ */
/* Route C (device global/local), FP64: src/cuda/local_global.cu             */
/* ------------------------------------------------------------------------ */

#define ROTATION_RELAXATION 0.2 /* local_global.cu:18 */

/* Largest eigenvector of Horn's 4x4 by cyclic Jacobi (local_global.cu:53-129),
 * iterated until the off-diagonal mass vanishes. */
static Q4 horn_quaternion(const double* S) {
    const double sxx = S[0], sxy = S[1], sxz = S[2];
    const double syx = S[3], syy = S[4], syz = S[5];
    const double szx = S[6], szy = S[7], szz = S[8];
    double a[4][4];
    a[0][0] = sxx + syy + szz; a[0][1] = syz - szy; a[0][2] = szx - sxz; a[0][3] = sxy - syx;
    a[1][1] = sxx - syy - szz; a[1][2] = sxy + syx; a[1][3] = szx + sxz;
    a[2][2] = -sxx + syy - szz; a[2][3] = syz + szy;
    a[3][3] = -sxx - syy + szz;
    for (int r = 1; r < 4; ++r)
        for (int c = 0; c < r; ++c) a[r][c] = a[c][r];
    double vec[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) vec[r][c] = r == c ? 1.0 : 0.0;
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
                    const double f = vec[k][p], s2 = vec[k][q];
                    vec[k][p] = cs * f - sn * s2; vec[k][q] = sn * f + cs * s2;
                }
            }
    }
    int best = 0;
    for (int i = 1; i < 4; ++i)
        if (a[i][i] > a[best][best]) best = i;
    Q4 q = {vec[0][best], vec[1][best], vec[2][best], vec[3][best]};
    return q;
}

static M3 rotation_from_quaternion(Q4 q) { /* local_global.cu:134-157 */
    const double length = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    if (!(length > 0.0)) return identity3();
    const double w = q.w / length, x = q.x / length, y = q.y / length, z = q.z / length;
    M3 r;
    r.m[0] = w * w + x * x - y * y - z * z; r.m[1] = 2.0 * (x * y - w * z);
    r.m[2] = 2.0 * (x * z + w * y); r.m[3] = 2.0 * (x * y + w * z);
    r.m[4] = w * w - x * x + y * y - z * z; r.m[5] = 2.0 * (y * z - w * x);
    r.m[6] = 2.0 * (x * z - w * y); r.m[7] = 2.0 * (y * z + w * x);
    r.m[8] = w * w - x * x - y * y + z * z;
    return r;
}

void oracle_horn_rotation(const double correlation[9], double rotation[9]) {
    const M3 r = rotation_from_quaternion(horn_quaternion(correlation));
    memcpy(rotation, r.m, sizeof r.m);
}

static void accumulate_correlation(double* S, double w, V3 x, V3 y) {
    const double xs[3] = {x.x, x.y, x.z}, ys[3] = {y.x, y.y, y.z};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) S[r * 3 + c] += w * xs[r] * ys[c];
}

/* fit_rotations_kernel, local_global.cu:188-302. */
static void fit_rotations(const Inputs* in, const double* lm_flag, const double* lm_target,
                          Deformation* d) {
    const int N = d->node_count;
    const double point_weight = in->w[0] + in->w[1]; /* local_global.cu:546 */
    M3* fitted = (M3*)malloc(sizeof(M3) * (size_t)N);
    double* S = (double*)calloc((size_t)N * 9, sizeof(double));
    for (int v = 0; v < in->vertex_count; ++v) {
        const Binding* b = &in->bindings[v];
        const V3 p = load3(in->points, (size_t)v);
        for (int s = 0; s < b->count; ++s) {
            const int node = b->nodes[s];
            if (node < 0 || node >= N || b->weights[s] == 0.0) continue;
            const V3 g = load3(d->rest, (size_t)node);
            const V3 t = d->translation[node];
            const double own = b->weights[s];
            const V3 source = sub(p, g);
            if (in->corr->accepted[v] && (!in->mask || in->mask[v]))
                accumulate_correlation(S + (size_t)node * 9,
                                       point_weight * in->corr->robust[v] * own, source,
                                       sub(sub(load3(in->corr->point, (size_t)v), g), t));
            if (in->w[4] > 0.0 && lm_flag[v] != 0.0)
                accumulate_correlation(S + (size_t)node * 9, in->w[4] * own, source,
                                       sub(sub(load3(lm_target, (size_t)v), g), t));
        }
    }
    for (int e = 0; e < in->edge_count; ++e) {
        const int a = in->edges[e * 2], b = in->edges[e * 2 + 1];
        const V3 ga = load3(d->rest, (size_t)a), gb = load3(d->rest, (size_t)b);
        accumulate_correlation(S + (size_t)a * 9, in->w[2], sub(gb, ga),
                               sub(sub(add(gb, d->translation[b]), ga), d->translation[a]));
    }
    for (int n = 0; n < N; ++n) {
        fitted[n] = rotation_from_quaternion(horn_quaternion(S + (size_t)n * 9));
        const M3 rt = transposed(&d->rotation[n]);
        const M3 rel = mulm(&fitted[n], &rt);
        const V3 omega = log_so3(&rel);
        const M3 step = exp_so3(scale(omega, ROTATION_RELAXATION));
        d->rotation[n] = mulm(&step, &d->rotation[n]);
    }
    free(S);
    free(fitted);
}

/* translation_rhs_kernel, local_global.cu:317-438. */
static void translation_rhs(const Inputs* in, const double* lm_flag, const double* lm_target,
                            const Deformation* d, double* rhs) {
    const int N = d->node_count;
    memset(rhs, 0, sizeof(double) * 6 * (size_t)N);
    for (int v = 0; v < in->vertex_count; ++v) {
        const Binding* b = &in->bindings[v];
        const V3 p = load3(in->points, (size_t)v);
        V3 deformed = v3(0, 0, 0);
        for (int s = 0; s < b->count; ++s) {
            const int o = b->nodes[s];
            if (o < 0 || b->weights[s] == 0.0) continue;
            deformed = add(deformed, scale(apply_node(d, o, p), b->weights[s]));
        }
        for (int s = 0; s < b->count; ++s) {
            const int node = b->nodes[s];
            if (node < 0 || b->weights[s] == 0.0) continue;
            const double own = b->weights[s];
            double* r = rhs + (size_t)node * 6 + 3;
            if (in->corr->accepted[v] && (!in->mask || in->mask[v])) {
                const V3 off = sub(deformed, load3(in->corr->point, (size_t)v));
                const double robust = in->corr->robust[v];
                if (in->w[0] > 0.0) {
                    const double sc = in->w[0] * robust * own;
                    r[0] -= sc * off.x; r[1] -= sc * off.y; r[2] -= sc * off.z;
                }
                if (in->w[1] > 0.0) {
                    const V3 nrm = load3(in->corr->normal, (size_t)v);
                    const double sc = in->w[1] * robust * own * dot(nrm, off);
                    r[0] -= sc * nrm.x; r[1] -= sc * nrm.y; r[2] -= sc * nrm.z;
                }
            }
            if (in->w[4] > 0.0 && lm_flag[v] != 0.0) {
                const V3 tm = sub(deformed, load3(lm_target, (size_t)v));
                const double sc = in->w[4] * own;
                r[0] -= sc * tm.x; r[1] -= sc * tm.y; r[2] -= sc * tm.z;
            }
        }
    }
    for (int e = 0; e < in->edge_count; ++e) {
        const int a = in->edges[e * 2], b = in->edges[e * 2 + 1];
        const V3 ga = load3(d->rest, (size_t)a), gb = load3(d->rest, (size_t)b);
        const V3 diff = sub(sub(add(add(mulv(&d->rotation[a], sub(gb, ga)), ga), d->translation[a]), gb),
                            d->translation[b]);
        double* ra = rhs + (size_t)a * 6 + 3;
        double* rb = rhs + (size_t)b * 6 + 3;
        ra[0] -= in->w[2] * diff.x; ra[1] -= in->w[2] * diff.y; ra[2] -= in->w[2] * diff.z;
        rb[0] += in->w[2] * diff.x; rb[1] += in->w[2] * diff.y; rb[2] += in->w[2] * diff.z;
    }
    for (int n = 0; n < N; ++n) {
        double* r = rhs + (size_t)n * 6 + 3;
        r[0] -= in->w[3] * d->translation[n].x;
        r[1] -= in->w[3] * d->translation[n].y;
        r[2] -= in->w[3] * d->translation[n].z;
    }
}

/* restrict_diagonal_kernel / restrict_offdiagonal_kernel, local_global.cu:453-507. */
static void restrict_to_translations(System* s) {
    for (int n = 0; n < s->node_count; ++n) {
        double* D = s->diag + (size_t)n * 36;
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
                if (r < 3 && c < 3) D[r * 6 + c] = r == c ? 1.0 : 0.0;
                else if (r < 3 || c < 3) D[r * 6 + c] = 0.0;
            }
    }
    for (int k = 0; k < s->off_count; ++k) {
        double* B = s->off + (size_t)k * 36;
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c)
                if (r < 3 || c < 3) B[r * 6 + c] = 0.0;
    }
}

/* ------------------------------------------------------------------------ */
/* Report JSON: src/core/report.cpp:46-105                                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    int level, nodes, outer_iterations, inner_iterations, converged;
    double energy_start, energy_end, correspondence_mean;
} LevelView;

typedef struct { char* data; size_t size, cap; } Text;
static void text_append(Text* t, const char* format, ...) {
    char buffer[512];
    va_list args;
    va_start(args, format);
    const int n = vsnprintf(buffer, sizeof buffer, format, args);
    va_end(args);
    if (t->size + (size_t)n + 1 > t->cap) {
        t->cap = (t->size + (size_t)n + 1) * 2;
        t->data = (char*)realloc(t->data, t->cap);
    }
    memcpy(t->data + t->size, buffer, (size_t)n + 1);
    t->size += (size_t)n;
}
static void text_number(Text* t, double value) {
    if (!isfinite(value)) text_append(t, "null");
    else text_append(t, "%.17g", value);
}

static void write_report(Text* t, const char* route, const double energy[5], const Counts* c,
                         const LevelView* views, int view_count, const NricpSolveDesc* desc,
                         double units) {
    text_append(t, "{\n  \"version\": \"0.1.0\",\n  \"route\": \"%s\",\n", route);
    text_append(t, "  \"precision\": \"double\",\n  \"setup_seconds\": 0,\n  \"solve_seconds\": 0,\n");
    text_append(t, "  \"energy\": {\n");
    const char* names[5] = {"point_to_point", "point_to_plane", "smoothness", "anchor", "landmark"};
    for (int i = 0; i < 5; ++i) {
        text_append(t, "    \"%s\": ", names[i]);
        text_number(t, energy[i]);
        text_append(t, ",\n");
    }
    text_append(t, "    \"total\": ");
    text_number(t, total_energy(energy));
    text_append(t, "\n  },\n  \"correspondence\": {\n");
    text_append(t, "    \"total\": %d,\n    \"accepted\": %d,\n    \"rejected_distance\": %d,\n",
                c->total, c->accepted, c->rejected_distance);
    text_append(t, "    \"rejected_normal\": %d,\n    \"rejected_slope\": %d,\n    \"rejected_masked\": %d,\n",
                c->rejected_normal, c->rejected_slope, c->rejected_masked);
    text_append(t, "    \"distance_mean\": ");
    text_number(t, c->mean);
    text_append(t, ",\n    \"distance_p95\": ");
    text_number(t, c->p95);
    text_append(t, ",\n    \"distance_max\": ");
    text_number(t, c->max);
    text_append(t, "\n  },\n  \"levels\": [");
    for (int i = 0; i < view_count; ++i) {
        const LevelView* v = &views[i];
        text_append(t, i == 0 ? "\n" : ",\n");
        text_append(t, "    {\"level\": %d, \"nodes\": %d, \"outer_iterations\": %d, \"inner_iterations\": %d, \"energy_start\": ",
                    v->level, v->nodes, v->outer_iterations, v->inner_iterations);
        text_number(t, v->energy_start);
        text_append(t, ", \"energy_end\": ");
        text_number(t, v->energy_end);
        text_append(t, ", \"correspondence_mean\": ");
        text_number(t, v->correspondence_mean);
        text_append(t, ", \"converged\": %s}", v->converged ? "true" : "false");
    }
    text_append(t, view_count == 0 ? "],\n" : "\n  ],\n");
    text_append(t, "  \"settings\": {");
    const char* keys[6] = {"point_to_point", "point_to_plane", "smoothness", "anchor", "landmark",
                           "robust_threshold"};
    int first = 1;
    for (int l = 0; l < view_count; ++l) {
        const int idx = l < desc->level_setting_count ? l : desc->level_setting_count - 1;
        const NricpLevelSettings* s = &desc->levels[idx];
        const double robust = s->robust_threshold > 0.0 ? s->robust_threshold * units : s->robust_threshold;
        const double vals[6] = {s->point_to_point, s->point_to_plane, s->smoothness, s->anchor,
                                s->landmark, robust};
        for (int k = 0; k < 6; ++k) {
            text_append(t, first ? "\n" : ",\n");
            first = 0;
            text_append(t, "    \"level%d_%s\": ", l, keys[k]);
            text_number(t, vals[k]);
        }
    }
    text_append(t, first ? "}\n" : "\n  }\n");
    text_append(t, "}\n");
}

/* ------------------------------------------------------------------------ */
/* The whole wrap: prepare_solve (bindings.cpp:584-672) + solve_route_a      */
/* (route_a.cpp:67-209) or the device schedule of route C (session.cu)       */
/* ------------------------------------------------------------------------ */

static const NricpLevelSettings* level_for(const NricpSolveDesc* d, int level) {
    if (d->level_setting_count <= 0) return NULL;
    return &d->levels[level < d->level_setting_count ? level : d->level_setting_count - 1];
}

static double relative_change(double before, double after) { /* route_shared.h:24-26 */
    return (before - after) / fmax(fabs(before), 1e-12);
}

int oracle_solve(const NricpSolveDesc* desc, int route, NricpResult* out) {
    int status;
    g_error[0] = 0;
    if ((status = validate_mesh(desc->template_points, desc->template_vertex_count,
                                desc->template_faces, desc->template_face_count, "template")))
        return status;
    if ((status = validate_mesh(desc->target_points, desc->target_vertex_count,
                                desc->target_faces, desc->target_face_count, "target")))
        return status;
    const int V = desc->template_vertex_count;
    const int k = desc->max_nodes_per_vertex > 0 ? desc->max_nodes_per_vertex : REF_KMAX;
    const int edge_k = desc->edge_neighbours > 0 ? desc->edge_neighbours : 4;
    if (k > KMAX) return fail(NRICP_ERR_INVALID, "max_nodes_per_vertex %d exceeds %d", k, KMAX);
    if (desc->level_setting_count <= 0)
        return fail(NRICP_ERR_INVALID, "level_settings must hold at least one level");
    if (desc->mask) {
        int active = 0;
        for (int i = 0; i < V; ++i) active += desc->mask[i] ? 1 : 0;
        if (active == 0)
            return fail(NRICP_ERR_INVALID,
                        "invalid mask: mask excludes every vertex; the fit would be unconstrained");
    }

    /* normalisation and graph (bindings.cpp:605-625) */
    double center[3], units;
    oracle_normalization(desc->template_points, V, center, &units);
    double* tpl = (double*)malloc(sizeof(double) * 3 * (size_t)V);
    memcpy(tpl, desc->template_points, sizeof(double) * 3 * (size_t)V);
    apply_normalization(tpl, V, center, units);
    double* tgt = (double*)malloc(sizeof(double) * 3 * (size_t)desc->target_vertex_count);
    memcpy(tgt, desc->target_points, sizeof(double) * 3 * (size_t)desc->target_vertex_count);
    apply_normalization(tgt, desc->target_vertex_count, center, units);
    Graph graph;
    build_graph(tpl, V, desc->graph_levels, desc->nodes_initial, desc->growth, k, edge_k, &graph);

    /* landmarks in the normalised frame (bindings.cpp:649-669) */
    const int L = desc->landmark_count;
    double* lm_tgt = (double*)malloc(sizeof(double) * 3 * (size_t)(L > 0 ? L : 1));
    int32_t* lm_idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(L > 0 ? L : 1));
    double* lm_flag = (double*)calloc((size_t)V, sizeof(double));
    double* lm_vtarget = (double*)calloc((size_t)V * 3, sizeof(double));
    for (int l = 0; l < L; ++l) {
        lm_idx[l] = desc->landmark_indices[l];
        const V3 t = scale(sub(load3(desc->landmark_targets, (size_t)l), v3(center[0], center[1], center[2])), units);
        store3(lm_tgt, (size_t)l, t);
        if (lm_idx[l] < 0 || lm_idx[l] >= V) {
            status = fail(NRICP_ERR_INVALID,
                          "invalid landmarks: landmark %d points at template vertex %d but the template has %d vertices",
                          l, lm_idx[l], V);
            goto cleanup_early;
        }
        if (lm_flag[lm_idx[l]] != 0.0) {
            status = fail(NRICP_ERR_INVALID, "invalid landmarks: landmark %d marks template vertex %d twice",
                          l, lm_idx[l]);
            goto cleanup_early;
        }
        lm_flag[lm_idx[l]] = 1.0;
        store3(lm_vtarget, (size_t)lm_idx[l], t);
    }

    {
        Target target;
        target_init(&target, tgt, desc->target_vertex_count, desc->target_faces, desc->target_face_count);
        const double distance_threshold = desc->distance_threshold * units;

        CorrSet corr;
        corr.point = (double*)calloc((size_t)V * 3, sizeof(double));
        corr.normal = (double*)calloc((size_t)V * 3, sizeof(double));
        corr.robust = (double*)calloc((size_t)V, sizeof(double));
        corr.accepted = (unsigned char*)calloc((size_t)V, 1);
        double* deformed = (double*)malloc(sizeof(double) * 3 * (size_t)V);
        double* qnormals = (double*)malloc(sizeof(double) * 3 * (size_t)V);
        LevelView* views = (LevelView*)calloc((size_t)graph.level_count, sizeof(LevelView));

        Deformation d;
        deformation_init(&d, graph.levels[0].node_count, graph.levels[0].rest);
        const int attempts_limit = desc->max_damping_attempts > 1 ? desc->max_damping_attempts : 1;
        const NricpLevelSettings* last_settings = NULL;
        Inputs in;
        memset(&in, 0, sizeof in);
        in.points = tpl; in.vertex_count = V; in.corr = &corr;
        in.lm_idx = lm_idx; in.lm_tgt = lm_tgt; in.lm_count = L; in.mask = desc->mask;

        for (int li = 0; li < graph.level_count; ++li) {
            const Level* level = &graph.levels[li];
            if (li > 0) {
                Deformation next;
                transfer_level(&graph.levels[li - 1], &d, level, &next);
                deformation_free(&d);
                d = next;
            }
            const NricpLevelSettings* ls = level_for(desc, li);
            last_settings = ls;
            const double robust_threshold = ls->robust_threshold > 0.0 ? ls->robust_threshold * units
                                                                       : ls->robust_threshold;
            in.bindings = level->bindings; in.d = &d; in.node_positions = level->rest;
            in.edges = level->edges; in.edge_count = level->edge_count;
            in.w[0] = ls->point_to_point; in.w[1] = ls->point_to_plane; in.w[2] = ls->smoothness;
            in.w[3] = ls->anchor; in.w[4] = ls->landmark;
            LevelView* view = &views[li];
            view->level = li; view->nodes = level->node_count;
            double damping = desc->initial_damping;
            double previous = 0.0;
            const int outer_limit = ls->max_outer_iterations > 1 ? ls->max_outer_iterations : 1;
            const int inner_limit = ls->max_inner_iterations > 1 ? ls->max_inner_iterations : 1;
            Counts counts;
            memset(&counts, 0, sizeof counts);
            const int N = level->node_count;
            double* delta = (double*)malloc(sizeof(double) * 6 * (size_t)N);
            Deformation candidate, saved;
            deformation_init(&candidate, N, level->rest);
            deformation_init(&saved, N, level->rest);

            for (int outer = 0; outer < outer_limit; ++outer) {
                evaluate_all(tpl, V, level->bindings, &d, deformed);
                oracle_vertex_normals(deformed, V, desc->template_faces, desc->template_face_count, qnormals);
                counts = correspond(&target, deformed, qnormals, V, desc, distance_threshold,
                                    ls->robust_kernel, robust_threshold, &corr);
                System sys;
                double current_energy;
                if (route == ORACLE_ROUTE_A) {
                    run_fused(&in, 0, &sys);
                    current_energy = total_energy(sys.energies);
                    system_free(&sys);
                } else {
                    run_fused(&in, 1, &sys); /* translation matrix, once per update */
                    restrict_to_translations(&sys);
                    current_energy = total_energy(sys.energies);
                }
                if (outer == 0) view->energy_start = current_energy;

                for (int inner = 0; inner < inner_limit; ++inner) {
                    if (route == ORACLE_ROUTE_A) {
                        run_fused(&in, 1, &sys); /* assemble_and_energy */
                        current_energy = total_energy(sys.energies);
                    }
                    int accepted = 0;
                    double candidate_energy = current_energy;
                    for (int attempt = 0; attempt < attempts_limit; ++attempt) {
                        if (route == ORACLE_ROUTE_A) {
                            if (!solve_damped(&sys, damping, desc->diagonal_damping, delta)) {
                                damping *= desc->damping_increase;
                                continue;
                            }
                            deformation_copy(&candidate, &d);
                            retract(&candidate, delta);
                        } else {
                            deformation_copy(&saved, &d);
                            deformation_copy(&candidate, &d);
                            in.d = &candidate;
                            fit_rotations(&in, lm_flag, lm_vtarget, &candidate);
                            translation_rhs(&in, lm_flag, lm_vtarget, &candidate, sys.rhs);
                            if (!solve_damped(&sys, damping, desc->diagonal_damping, delta)) {
                                in.d = &d;
                                damping *= desc->damping_increase;
                                continue;
                            }
                            retract(&candidate, delta);
                        }
                        in.d = &candidate;
                        System e;
                        run_fused(&in, 0, &e);
                        candidate_energy = total_energy(e.energies);
                        system_free(&e);
                        in.d = &d;
                        if (candidate_energy < current_energy) { accepted = 1; break; }
                        damping *= desc->damping_increase;
                    }
                    if (route == ORACLE_ROUTE_A) system_free(&sys);
                    if (!accepted) break;
                    deformation_copy(&d, &candidate);
                    damping = fmax(damping * desc->damping_decrease, 1e-12);
                    view->inner_iterations += 1;
                    const double improvement = relative_change(current_energy, candidate_energy);
                    current_energy = candidate_energy;
                    if (improvement <= ls->inner_tolerance) break;
                }
                if (route == ORACLE_ROUTE_C) system_free(&sys);
                System e;
                run_fused(&in, 0, &e);
                const double level_energy = total_energy(e.energies);
                system_free(&e);
                view->energy_end = level_energy;
                view->correspondence_mean = counts.mean;
                view->outer_iterations += 1;
                if (outer > 0 && relative_change(previous, level_energy) <= ls->outer_tolerance) {
                    view->converged = 1;
                    break;
                }
                previous = level_energy;
            }
            deformation_free(&candidate);
            deformation_free(&saved);
            free(delta);
        }

        /* results (route_a.cpp:192-207, bindings.cpp:674-710) */
        const Level* finest = &graph.levels[graph.level_count - 1];
        evaluate_all(tpl, V, finest->bindings, &d, deformed);
        for (int i = 0; i < V; ++i) {
            const V3 p = add(divide(load3(deformed, (size_t)i), units), v3(center[0], center[1], center[2]));
            if (out->vertices) store3(out->vertices, (size_t)i, p);
        }
        for (int n = 0; n < finest->node_count; ++n) {
            if (out->rotations) memcpy(out->rotations + (size_t)n * 9, d.rotation[n].m, sizeof(double) * 9);
            if (out->translations) store3(out->translations, (size_t)n, d.translation[n]);
            if (out->node_positions) store3(out->node_positions, (size_t)n, load3(finest->rest, (size_t)n));
        }
        if (out->level_nodes)
            for (int l = 0; l < graph.level_count; ++l) out->level_nodes[l] = graph.levels[l].node_count;

        /* fill_final_statistics (route_a.cpp:40-63) + block energies (route_a.cpp:200-206) */
        double energies[5];
        block_energies(&in, energies);
        oracle_vertex_normals(deformed, V, desc->template_faces, desc->template_face_count, qnormals);
        CorrSet final_corr;
        final_corr.point = (double*)calloc((size_t)V * 3, sizeof(double));
        final_corr.normal = (double*)calloc((size_t)V * 3, sizeof(double));
        final_corr.robust = (double*)calloc((size_t)V, sizeof(double));
        final_corr.accepted = (unsigned char*)calloc((size_t)V, 1);
        const Counts fc = correspond(&target, deformed, qnormals, V, desc, distance_threshold,
                                     last_settings->robust_kernel, 0.0, &final_corr);
        Text text = {0};
        write_report(&text, route == ORACLE_ROUTE_A ? "route_a" : "route_c", energies, &fc, views,
                     graph.level_count, desc, units);
        out->report_length = text.size;
        if (out->report_json && out->report_capacity > 0) {
            const size_t n = text.size < out->report_capacity - 1 ? text.size : out->report_capacity - 1;
            memcpy(out->report_json, text.data, n);
            out->report_json[n] = 0;
        }
        free(text.data);
        free(final_corr.point); free(final_corr.normal); free(final_corr.robust); free(final_corr.accepted);
        deformation_free(&d);
        free(views); free(deformed); free(qnormals);
        free(corr.point); free(corr.normal); free(corr.robust); free(corr.accepted);
        target_free(&target);
        status = 0;
    }
cleanup_early:
    free_graph(&graph);
    free(lm_tgt); free(lm_idx); free(lm_flag); free(lm_vtarget);
    free(tpl); free(tgt);
    return status;
}

/* ------------------------------------------------------------------------ */
/* Debug entry: the fused system at a given state                             */
/* ------------------------------------------------------------------------ */

int oracle_fused_system(const OracleSystemInputs* in, double* diagonal, double* rhs,
                        int32_t* off_a, int32_t* off_b, double* off_blocks, int capacity,
                        int* off_count, double energies[5]) {
    Binding* b = (Binding*)malloc(sizeof(Binding) * (size_t)(in->vertex_count > 0 ? in->vertex_count : 1));
    for (int v = 0; v < in->vertex_count; ++v) {
        for (int s = 0; s < KMAX; ++s) {
            b[v].nodes[s] = in->binding_nodes[v * KMAX + s];
            b[v].weights[s] = in->binding_weights[v * KMAX + s];
        }
        b[v].count = in->binding_counts[v];
    }
    Deformation d;
    deformation_init(&d, in->node_count, in->node_positions);
    for (int n = 0; n < in->node_count; ++n) {
        memcpy(d.rotation[n].m, in->rotations + (size_t)n * 9, sizeof(double) * 9);
        d.translation[n] = load3(in->translations, (size_t)n);
    }
    CorrSet corr;
    corr.point = (double*)in->corr_points;
    corr.normal = (double*)in->corr_normals;
    corr.robust = (double*)in->corr_robust;
    corr.accepted = (unsigned char*)in->corr_accepted;
    Inputs x;
    memset(&x, 0, sizeof x);
    x.points = in->template_points; x.vertex_count = in->vertex_count; x.bindings = b; x.d = &d;
    x.node_positions = in->node_positions; x.corr = &corr; x.edges = in->edges;
    x.edge_count = in->edge_count; x.lm_idx = in->landmark_indices; x.lm_tgt = in->landmark_targets;
    x.lm_count = in->landmark_count; x.mask = in->mask;
    memcpy(x.w, in->weights, sizeof x.w);
    System s;
    run_fused(&x, 1, &s);
    memcpy(diagonal, s.diag, sizeof(double) * 36 * (size_t)in->node_count);
    memcpy(rhs, s.rhs, sizeof(double) * 6 * (size_t)in->node_count);
    memcpy(energies, s.energies, sizeof(double) * 5);
    *off_count = s.off_count;
    const int status = s.off_count <= capacity ? 0 : NRICP_ERR_CAPACITY;
    if (!status) {
        memcpy(off_a, s.off_a, sizeof(int32_t) * (size_t)s.off_count);
        memcpy(off_b, s.off_b, sizeof(int32_t) * (size_t)s.off_count);
        memcpy(off_blocks, s.off, sizeof(double) * 36 * (size_t)s.off_count);
    }
    system_free(&s);
    deformation_free(&d);
    free(b);
    return status;
}

/* ------------------------------------------------------------------------ */
/* FP32 LBVH build: src/cuda/lbvh.cu:33-352                                  */
/* ------------------------------------------------------------------------ */

static uint32_t expand_bits(uint32_t v) { /* lbvh.cu:132-139 */
    v &= 0x000003ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

static int clz32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }

static int lcp(const uint32_t* codes, int n, int i, int j) { /* lbvh.cu:177-188 */
    if (j < 0 || j >= n) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + clz32((uint32_t)(i ^ j));
    return clz32(a ^ b);
}

typedef struct { uint32_t code; uint32_t index; } CodeIndex;
static int cmp_code(const void* a, const void* b) {
    const CodeIndex* x = (const CodeIndex*)a;
    const CodeIndex* y = (const CodeIndex*)b;
    if (x->code != y->code) return x->code < y->code ? -1 : 1;
    return (x->index > y->index) - (x->index < y->index);
}

void oracle_lbvh_build(const float* points, int point_count, const int32_t* faces,
                       int face_count, uint32_t* out_codes, uint32_t* out_order,
                       int32_t* out_left, int32_t* out_right, float out_bounds[6]) {
    (void)point_count;
    const int n = face_count;
    float* centroid = (float*)malloc(sizeof(float) * 3 * (size_t)n);
    for (int t = 0; t < n; ++t) { /* lbvh.cu:33-49 */
        const float* a = points + (size_t)faces[t * 3] * 3;
        const float* b = points + (size_t)faces[t * 3 + 1] * 3;
        const float* c = points + (size_t)faces[t * 3 + 2] * 3;
        for (int k = 0; k < 3; ++k) {
            volatile float s = a[k] + b[k];
            s = s + c[k];
            centroid[t * 3 + k] = s / 3.0f;
        }
    }
    float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int t = 0; t < n; ++t) /* lbvh.cu:89-127 */
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], centroid[t * 3 + k]);
            hi[k] = fmaxf(hi[k], centroid[t * 3 + k]);
        }
    for (int k = 0; k < 3; ++k) { out_bounds[k] = lo[k]; out_bounds[3 + k] = hi[k]; }
    CodeIndex* ci = (CodeIndex*)malloc(sizeof(CodeIndex) * (size_t)n);
    float sc[3];
    for (int k = 0; k < 3; ++k) {
        const float extent = hi[k] - lo[k];
        sc[k] = extent > 1e-10f ? 1023.0f / extent : 0.0f;
    }
    for (int t = 0; t < n; ++t) { /* lbvh.cu:146-168 */
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) {
            volatile float off = centroid[t * 3 + k] - lo[k];
            const float scaled = off * sc[k];
            q[k] = (uint32_t)fminf(1023.0f, fmaxf(0.0f, scaled));
        }
        ci[t].code = (expand_bits(q[2]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[0]);
        ci[t].index = (uint32_t)t;
    }
    qsort(ci, (size_t)n, sizeof(CodeIndex), cmp_code); /* stable by (code, index) */
    for (int t = 0; t < n; ++t) { out_codes[t] = ci[t].code; out_order[t] = ci[t].index; }
    for (int i = 0; i + 1 < n; ++i) { /* lbvh.cu:190-245 */
        const int pp = lcp(out_codes, n, i, i - 1);
        const int pn = lcp(out_codes, n, i, i + 1);
        const int dir = pn > pp ? 1 : -1;
        const int pmin = pp < pn ? pp : pn;
        int span = 2;
        while (lcp(out_codes, n, i, i + span * dir) > pmin) span *= 2;
        int last = 0;
        for (int step = span / 2; step >= 1; step /= 2)
            if (lcp(out_codes, n, i, i + (last + step) * dir) > pmin) last += step;
        const int j = i + last * dir;
        const int rl = i < j ? i : j, rr = i < j ? j : i;
        const int np = lcp(out_codes, n, rl, rr);
        int offset = 0, step = rr - rl;
        do {
            step = (step + 1) / 2;
            if (lcp(out_codes, n, rl, rl + offset + step) > np) offset += step;
        } while (step > 1);
        const int split = rl + offset;
        out_left[i] = rl == split ? rl : n + split;
        out_right[i] = split + 1 == rr ? rr : n + split + 1;
    }
    free(ci);
    free(centroid);
}
