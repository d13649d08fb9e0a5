// Smoothed-aggregation set-up on the device (internal): host graph helpers
// (sa_graph.cpp) and the device set-up driver (sa_setup.cu).
#pragma once
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace exfem {

// rows of sorted int32 column lists (CSR pattern without values)
struct Rows {
  std::vector<int64_t> ptr;  // (nrows + 1)
  std::vector<int32_t> idx;
  int64_t nrows() const { return ptr.empty() ? 0 : (int64_t)ptr.size() - 1; }
};

// node adjacency of a mesh: row n lists, ascending, every node that shares an
// element with n (n itself included)
int host_node_adjacency(int64_t nn, int64_t ne, int nnode, const int32_t* conn, Rows& out);
// the entries q of pattern `pat` whose flag[q] is set, row by row in their order:
// S holds their columns, keep their positions in pat (rows filtered on threads)
void host_filter_pattern(const Rows& pat, const uint8_t* flag, Rows& S, std::vector<int64_t>& keep);
// six rigid-body modes of nodes X (nn, 3) centred at their mean: (3 nn, 6) row-major
void host_rigid_body_modes(int64_t nn, const double* X, std::vector<double>& B);
// tentative prolongator of an aggregation: per aggregate, modified Gram-Schmidt of
// the near-null-space rows (K columns) of its DOFs (bs per node, in increasing DOF
// order); columns whose norm drops below drop x their original norm are zeroed.
// Q (nb*bs, K): the orthonormal rows of each DOF (zero for unaggregated nodes);
// Bc (nagg*K, K): the coarse near-null space (the R factors).
void host_fit_candidates(int64_t nb, int bs, int K, const int32_t* agg, int64_t nagg, const double* B,
                         std::vector<double>& Q, std::vector<double>& Bc, double drop = 1e-10);
// prolongator pattern: row n lists the aggregates of n and of its strength-graph
// neighbours (unaggregated nodes left out)
void host_p_pattern(const Rows& S, const int32_t* agg, int64_t nagg, Rows& P);
// row i of out = union over j in outer(i) of inner(j), ascending (columns < ncols)
void host_union_pattern(const Rows& outer, const Rows& inner, int64_t ncols, Rows& out);
// transpose of a pattern with ncols columns: row g lists the rows n that hold g
// (ascending), and slot[k] the position of g inside row n's list
void host_transpose_pattern(const Rows& P, int64_t ncols, Rows& PT, std::vector<int32_t>& slot);
// inverse of the coarsest matrix (n x n, row-major, symmetrised in place) through
// a regularised Cholesky factor L: Ainv = L^-T L^-1
int host_coarse_inverse(int64_t n, std::vector<double>& A, std::vector<double>& Ainv);

// device set-up of a smoothed-aggregation hierarchy for a block's current
// element matrices (sa_setup.cu)
int amg_setup_block(exfem_amg_s* h, exfem_block_s* b, const double* Ke, int max_coarse, int keep_level0,
                    cudaStream_t s);
int amg_setup_blocks(exfem_amg_s* h, const std::vector<exfem_block_s*>& blks, const std::vector<const double*>& Kes,
                     int max_coarse, int keep_level0, cudaStream_t s);

}  // namespace exfem
