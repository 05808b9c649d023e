// Replacement for the reference's src/solver/direct_solve.cpp -- TEST
// INFRASTRUCTURE ONLY.  Same signature (src/solver/direct_solve.h:18), same
// job: an exact solve of the damped block-sparse system.  The reference does
// it with Eigen 3.4.0 SimplicialLDLT, which is not vendored with it; this calls
// the oracle's block Cholesky (oracle/block_cholesky.c) instead.
#include <cmath>
#include <cstdint>
#include <vector>

#include "solver/direct_solve.h"

extern "C" {
#include "block_cholesky.h"
}

namespace nricp {

DirectSolveResult solve_direct(const NormalEquations& system) {
    DirectSolveResult result;
    const int n = system.node_count;
    if (n <= 0) {
        return result;
    }
    std::vector<double> diagonal(static_cast<std::size_t>(n) * 36);
    for (int node = 0; node < n; ++node) {
        for (int i = 0; i < 36; ++i) {
            diagonal[static_cast<std::size_t>(node) * 36 + i] =
                system.diagonal[static_cast<std::size_t>(node)].m[i];
        }
    }
    const std::size_t count = system.off_diagonal.size();
    std::vector<int32_t> a(count), b(count);
    std::vector<double> blocks(count * 36);
    for (std::size_t i = 0; i < count; ++i) {
        a[i] = system.off_diagonal[i].a;
        b[i] = system.off_diagonal[i].b;
        for (int k = 0; k < 36; ++k) {
            blocks[i * 36 + k] = system.off_diagonal[i].value.m[k];
        }
    }
    result.delta.assign(static_cast<std::size_t>(n) * 6, 0.0);
    result.ok = block_cholesky_solve(n, diagonal.data(), static_cast<int>(count), a.data(),
                                     b.data(), blocks.data(), system.rhs.data(),
                                     result.delta.data()) != 0;
    if (!result.ok) {
        result.delta.clear();
    }
    return result;
}

}  // namespace nricp
