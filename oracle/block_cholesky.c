/*
 * Block-sparse Cholesky -- TEST INFRASTRUCTURE ONLY.  See block_cholesky.h.
 *
 * Stands in for Eigen's SimplicialLDLT (reference src/solver/direct_solve.cpp:
 * 42-55): same job (exact solve of the damped symmetric system), restated as
 * minimum-degree ordering + right-looking 6x6-block Cholesky.
 */
#include "block_cholesky.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int* items;
    int size;
    int capacity;
} IntSet; /* sorted, unique */

static void set_insert(IntSet* set, int value) {
    int lo = 0, hi = set->size;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (set->items[mid] < value) lo = mid + 1; else hi = mid;
    }
    if (lo < set->size && set->items[lo] == value) return;
    if (set->size == set->capacity) {
        set->capacity = set->capacity ? set->capacity * 2 : 8;
        set->items = (int*)realloc(set->items, sizeof(int) * (size_t)set->capacity);
    }
    memmove(set->items + lo + 1, set->items + lo, sizeof(int) * (size_t)(set->size - lo));
    set->items[lo] = value;
    set->size += 1;
}

static void set_erase(IntSet* set, int value) {
    int lo = 0, hi = set->size;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (set->items[mid] < value) lo = mid + 1; else hi = mid;
    }
    if (lo < set->size && set->items[lo] == value) {
        memmove(set->items + lo, set->items + lo + 1,
                sizeof(int) * (size_t)(set->size - lo - 1));
        set->size -= 1;
    }
}

static int set_find(const IntSet* set, int value) {
    int lo = 0, hi = set->size;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (set->items[mid] < value) lo = mid + 1; else hi = mid;
    }
    return (lo < set->size && set->items[lo] == value) ? lo : -1;
}

/* 6x6 helpers, row-major. */
static int chol6(double* a) { /* in place, lower triangle; 0 when not PD */
    for (int r = 0; r < 6; ++r) {
        for (int c = 0; c <= r; ++c) {
            double sum = a[r * 6 + c];
            for (int k = 0; k < c; ++k) sum -= a[r * 6 + k] * a[c * 6 + k];
            if (r == c) {
                if (!(sum > 0.0)) return 0;
                a[r * 6 + c] = sqrt(sum);
            } else {
                a[r * 6 + c] = sum / a[c * 6 + c];
            }
        }
        for (int c = r + 1; c < 6; ++c) a[r * 6 + c] = 0.0;
    }
    return 1;
}

/* X := X * L^-T (L lower, 6x6), i.e. solve X L^T = B row by row. */
static void right_solve_lt(double* x, const double* l) {
    for (int r = 0; r < 6; ++r) {
        double* row = x + r * 6;
        for (int c = 0; c < 6; ++c) {
            double sum = row[c];
            for (int k = 0; k < c; ++k) sum -= row[k] * l[c * 6 + k];
            row[c] = sum / l[c * 6 + c];
        }
    }
}

/* C -= A * B^T */
static void sub_abt(double* c, const double* a, const double* b) {
    for (int r = 0; r < 6; ++r)
        for (int s = 0; s < 6; ++s) {
            double sum = 0.0;
            for (int k = 0; k < 6; ++k) sum += a[r * 6 + k] * b[s * 6 + k];
            c[r * 6 + s] -= sum;
        }
}

int block_cholesky_solve(int n, const double* diagonal, int count,
                         const int32_t* a, const int32_t* b,
                         const double* blocks, const double* rhs, double* x) {
    if (n <= 0) return 0;
    /* ---- minimum-degree ordering on the explicit elimination graph ---- */
    IntSet* graph = (IntSet*)calloc((size_t)n, sizeof(IntSet));
    for (int i = 0; i < count; ++i) {
        if (a[i] == b[i] || a[i] < 0 || b[i] < 0 || a[i] >= n || b[i] >= n) continue;
        set_insert(&graph[a[i]], b[i]);
        set_insert(&graph[b[i]], a[i]);
    }
    int* order = (int*)malloc(sizeof(int) * (size_t)n);
    int* position = (int*)malloc(sizeof(int) * (size_t)n);
    IntSet* pattern = (IntSet*)calloc((size_t)n, sizeof(IntSet));
    char* done = (char*)calloc((size_t)n, 1);
    for (int step = 0; step < n; ++step) {
        int best = -1;
        for (int v = 0; v < n; ++v) {
            if (done[v]) continue;
            if (best < 0 || graph[v].size < graph[best].size) best = v;
        }
        order[step] = best;
        position[best] = step;
        done[best] = 1;
        /* the column pattern of `best` is its current neighbour set */
        pattern[best] = graph[best];
        graph[best].items = NULL;
        graph[best].size = graph[best].capacity = 0;
        const IntSet* neighbours = &pattern[best];
        for (int i = 0; i < neighbours->size; ++i) {
            const int u = neighbours->items[i];
            set_erase(&graph[u], best);
            for (int j = 0; j < neighbours->size; ++j) {
                const int w = neighbours->items[j];
                if (w != u) set_insert(&graph[u], w);
            }
        }
    }
    free(done);
    for (int v = 0; v < n; ++v) free(graph[v].items);
    free(graph);

    /* ---- working storage: column v holds A(u, v) for u in pattern(v) ---- */
    double** column = (double**)malloc(sizeof(double*) * (size_t)n);
    double* pivot = (double*)malloc(sizeof(double) * 36 * (size_t)n);
    memcpy(pivot, diagonal, sizeof(double) * 36 * (size_t)n);
    for (int v = 0; v < n; ++v)
        column[v] = (double*)calloc((size_t)(pattern[v].size > 0 ? pattern[v].size : 1) * 36,
                                    sizeof(double));
    for (int i = 0; i < count; ++i) {
        const int p = a[i], q = b[i];
        if (p == q || p < 0 || q < 0 || p >= n || q >= n) continue;
        const double* block = blocks + (size_t)i * 36; /* A(p, q) */
        if (position[p] < position[q]) {
            /* stored in column p as A(q, p) = block^T */
            const int slot = set_find(&pattern[p], q);
            double* target = column[p] + (size_t)slot * 36;
            for (int r = 0; r < 6; ++r)
                for (int c = 0; c < 6; ++c) target[r * 6 + c] += block[c * 6 + r];
        } else {
            const int slot = set_find(&pattern[q], p);
            double* target = column[q] + (size_t)slot * 36;
            for (int r = 0; r < 36; ++r) target[r] += block[r];
        }
    }

    /* ---- right-looking factorisation in elimination order ---- */
    int ok = 1;
    for (int step = 0; step < n && ok; ++step) {
        const int v = order[step];
        double* lvv = pivot + (size_t)v * 36;
        if (!chol6(lvv)) { ok = 0; break; }
        const IntSet* pv = &pattern[v];
        for (int i = 0; i < pv->size; ++i) right_solve_lt(column[v] + (size_t)i * 36, lvv);
        for (int i = 0; i < pv->size; ++i) {
            const int u = pv->items[i];
            const double* luv = column[v] + (size_t)i * 36;
            for (int j = 0; j < pv->size; ++j) {
                const int w = pv->items[j];
                if (position[w] < position[u]) continue;
                const double* lwv = column[v] + (size_t)j * 36;
                if (w == u) {
                    sub_abt(pivot + (size_t)u * 36, luv, luv);
                } else {
                    const int slot = set_find(&pattern[u], w); /* A(w, u) */
                    sub_abt(column[u] + (size_t)slot * 36, lwv, luv);
                }
            }
        }
    }

    if (ok) {
        double* y = x;
        memcpy(y, rhs, sizeof(double) * 6 * (size_t)n);
        for (int step = 0; step < n; ++step) { /* L y = b */
            const int v = order[step];
            const double* l = pivot + (size_t)v * 36;
            double* yv = y + (size_t)v * 6;
            for (int r = 0; r < 6; ++r) {
                double sum = yv[r];
                for (int k = 0; k < r; ++k) sum -= l[r * 6 + k] * yv[k];
                yv[r] = sum / l[r * 6 + r];
            }
            const IntSet* pv = &pattern[v];
            for (int i = 0; i < pv->size; ++i) {
                const double* luv = column[v] + (size_t)i * 36;
                double* yu = y + (size_t)pv->items[i] * 6;
                for (int r = 0; r < 6; ++r) {
                    double sum = 0.0;
                    for (int k = 0; k < 6; ++k) sum += luv[r * 6 + k] * yv[k];
                    yu[r] -= sum;
                }
            }
        }
        for (int step = n - 1; step >= 0; --step) { /* L^T x = y */
            const int v = order[step];
            const double* l = pivot + (size_t)v * 36;
            double* xv = x + (size_t)v * 6;
            const IntSet* pv = &pattern[v];
            for (int i = 0; i < pv->size; ++i) {
                const double* luv = column[v] + (size_t)i * 36;
                const double* xu = x + (size_t)pv->items[i] * 6;
                for (int c = 0; c < 6; ++c) {
                    double sum = 0.0;
                    for (int r = 0; r < 6; ++r) sum += luv[r * 6 + c] * xu[r];
                    xv[c] -= sum;
                }
            }
            for (int r = 5; r >= 0; --r) {
                double sum = xv[r];
                for (int k = r + 1; k < 6; ++k) sum -= l[k * 6 + r] * xv[k];
                xv[r] = sum / l[r * 6 + r];
            }
        }
        for (int i = 0; i < 6 * n; ++i)
            if (!isfinite(x[i])) { ok = 0; break; }
    }

    for (int v = 0; v < n; ++v) { free(column[v]); free(pattern[v].items); }
    free(column); free(pattern); free(pivot); free(order); free(position);
    return ok;
}
