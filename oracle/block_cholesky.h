/*
 * Block-sparse Cholesky for the 6x6-block reduced systems -- TEST
 * INFRASTRUCTURE ONLY (the oracle's linear solve).
 *
 * The reference's route A solves with Eigen 3.4.0 SimplicialLDLT
 * (src/solver/direct_solve.cpp:42-55).  Eigen is a git submodule that is not
 * vendored with the reference, so this is a restatement of the published
 * algorithm -- a sparse symmetric factorisation with a fill-reducing ordering --
 * at 6x6-block granularity: minimum-degree ordering of the node graph, a
 * right-looking block Cholesky, then two triangular solves.  The reference's
 * results at this boundary are pinned only against a dense numpy solve
 * (tests/test_normal_equations.py:107-135), not against Eigen's bits.
 */
#ifndef NRICP_BLOCK_CHOLESKY_H
#define NRICP_BLOCK_CHOLESKY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Solves A x = rhs.  A is symmetric with `diagonal[n*36]` row-major 6x6
 * blocks and `count` off-diagonal blocks A(a[i], b[i]) (row-major, rows of
 * a[i]); A(b, a) is the transpose.  Returns 1 on success, 0 when a pivot
 * block is not positive definite (the caller then damps harder). */
int block_cholesky_solve(int n, const double* diagonal, int count,
                         const int32_t* a, const int32_t* b,
                         const double* blocks, const double* rhs, double* x);

#ifdef __cplusplus
}
#endif

#endif
