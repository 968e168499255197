// Smoothed-aggregation algebraic multigrid hierarchy (host, FP64) for the
// symmetric M-matrix of the relaxation's inner solve.
//
// A multigrid V-cycle used as the preconditioner of the inner conjugate
// gradients removes the smooth far field of a removal's correction, which a
// pointwise (Jacobi) preconditioner leaves to many iterations.  The
// construction is Vanek, Mandel and Brezina's (Computing 56, 1996): strength
// of connection |a_ij| >= theta sqrt(a_ii a_jj), greedy aggregation,
// piecewise-constant tentative prolongator smoothed by one damped Jacobi
// step on the filtered matrix, Galerkin coarse operators R A P with R = P^T
// whose weakest entries are lumped into the diagonal, down to a coarsest
// level solved with a dense inverse.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tg_host {

struct AmgCsr {
    int rows = 0, cols = 0;
    std::vector<int32_t> ptr, col;
    std::vector<double> val;
};

struct AmgLevel {
    AmgCsr A;   // the level's operator (level 0: the fine matrix it was built from)
    AmgCsr P;   // rows x next level's rows
    AmgCsr R;   // P^T
};

struct AmgHierarchy {
    std::vector<AmgLevel> levels;   // the last level has no P / R
    std::vector<double> coarse_inv; // dense inverse of the last level's operator, row-major
};

struct AmgOptions {
    double theta = 0.08;       // strength threshold on the finest level
    double theta_coarse = 0.0; // and on the coarser ones, whose Galerkin rows spread over more entries
    double omega = 0.8;        // prolongator smoothing weight, 4/3 over rho(D_F^-1 A_F) for rho ~ 1.7
    // coarse-operator entries |a_ij| < coarse_drop sqrt(a_ii a_jj) are dropped
    // and lumped into a_ii: on the 3.2M-row system of the 7.3M-cell tip 0.01
    // halves level 1's entries per row (50 -> 24) and lowers the CG
    // iterations to 1e-8 from 21 to 16
    double coarse_drop = 0.01;
    int max_coarse = 1000;     // rows at which coarsening stops
    int max_levels = 12;
    int threads = 0;           // 0: hardware concurrency
};

// Builds the hierarchy of the n x n matrix A (full CSR with its diagonal;
// rows without off-diagonal entries are left out of the coarse levels),
// taking A over as the finest level's operator.  Returns an empty string or
// the error.
std::string amg_build(AmgCsr&& A, const AmgOptions& opt, AmgHierarchy* out);

// Test hook: while on, one worker thread of every threaded pass of the build
// throws std::bad_alloc (an allocation failure inside a worker), which the
// build must turn into an error on the calling thread.
void amg_inject_worker_failure(bool on);

}  // namespace tg_host
