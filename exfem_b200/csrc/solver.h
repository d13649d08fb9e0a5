// AMG hierarchy and solver handle layouts (internal).
#pragma once
#include <algorithm>
#include <memory>
#include <vector>

#include "internal.h"

namespace exfem {

// a level matrix kept in block-sparse form (R x C dense blocks, row-major) by the
// device set-up: the V-cycle applies it with one index per block instead of one
// per entry (the scalar CSR copy stays for exports and replicated unions)
struct Bsr {
  int R = 0, C = 0;
  int64_t nb = 0, nnzb = 0;  // block rows, stored blocks
  DevBuf<int64_t> ptr;
  DevBuf<int32_t> idx;
  DevBuf<double> v64;
  DevBuf<float> v32;
  bool on() const { return nnzb > 0; }
};

struct AmgLevel {
  enum { WB = 0, WX = 1, WR = 2, WD = 3, WD2 = 4, WTMP = 5, NW = 6 };
  int64_t n = 0, nc = 0;
  double rho = 1.0;
  int64_t op_nnz = 0;     // nonzeros of the level operator when it is not stored (device set-up)
  Csr64 A, P, R;
  Bsr bA, bP, bR;         // the same matrices in block form (device set-up only)
  DevBuf<double> dinv64;
  DevBuf<float> dinv32;
  DevBuf<double> coef64;  // optional per-row Chebyshev coefficients (5 per row)
  DevBuf<float> coef32;
  DevBuf<double> w64[NW];
  DevBuf<float> w32[NW];
};

// a block's element matrices assembled into one CSR matrix (EXFEM_OP_CSR_F64):
// 3x3 node blocks on the node-adjacency pattern (built once, so the device
// pointers a captured graph holds stay valid), expanded to scalar CSR
struct BlockCsr {
  bool ready = false;
  int64_t nnzb = 0;
  DevBuf<int64_t> bptr;
  DevBuf<int32_t> bidx;
  DevBuf<double> bval;
  Csr64 A;
};
int block_csr_assemble(exfem_block_s* b, const double* Ke, BlockCsr& c, cudaStream_t s);
// the same for several blocks over one node set, summed block after block in
// gather-plan order (the prescribed DOFs of the first block)
int blocks_csr_assemble(const std::vector<exfem_block_s*>& blks, const std::vector<const double*>& Kes, BlockCsr& c,
                        cudaStream_t s);
int amg_setup_blocks(exfem_amg_s* h, const std::vector<exfem_block_s*>& blks, const std::vector<const double*>& Kes,
                     int max_coarse, int keep_level0, cudaStream_t s);
int csr_apply(const Csr64& A, const double* x, double* y, const int* skip, cudaStream_t s);

// level-0 operator override: y = A0(x) and its inverse diagonal
template <class T>
struct Level0Op {
  int (*apply)(void* ctx, const T* x, T* y, const int* skip, cudaStream_t s) = nullptr;
  void* ctx = nullptr;
  const T* dinv = nullptr;
};

template <class T>
int amg_vcycle(exfem_amg_s* h, const T* b, T* x, const Level0Op<T>* op0, const int* skip, cudaStream_t s);
int amg_prepare(exfem_amg_s* h, int dtype);
int amg_set_level_rows(exfem_amg_s* h, size_t l, const double* rho_rows);
int amg_replicate(exfem_amg_s* h, int nmesh, const int64_t* level_offsets, int ninst, const int32_t* inst_mesh);
int amg_add_level(exfem_amg_s* h, int64_t n, int64_t nc, const int64_t* Ap, const int32_t* Ai, const double* Av,
                  const int64_t* Pp, const int32_t* Pi, const double* Pv, const int64_t* Rp, const int32_t* Ri,
                  const double* Rv, const double* dinv, double rho);

// device scalars of one PCG run (FP64 step scalars and dot products)
struct PcgScal {
  double rz, pAp, rr, bb, tol2, alpha, beta, spare;
  int k, maxiter, done, pad;
};

// device scalars of the Newton increment run as one graph
struct NewtonScal {
  double rtol, fn_t, qref, rt, ft, ut_n, ratio, dut, alpha, rls, n2, nrm_r, nrm_f, nrm_u, nrm_du, nrm_t;
  int it, max_iter, done, converged, failed, corrections, line_search, ls_count, ls_done, loops;
  int lin_its, lin_nup;  // FP32 iterations and replacements of the last linear solve
  double hist[64];
};

// device scalars of the reliable-update mixed solve run as one graph
struct MixedScal {
  double tol, delta, bn, rn, rn_prev, sc, inv_sc, nrm2;
  float pscale;
  int maxiter, max_updates, its, nup, restart, done, loops;
};

}  // namespace exfem

struct exfem_amg_s {
  int degree = 2;
  std::vector<std::unique_ptr<exfem::AmgLevel>> levels;
  int64_t nc = 0;
  int64_t coarse_nnz = 0;  // nonzeros of the coarsest operator (device set-up)
  exfem::DevBuf<double> Ainv;
  exfem::DevBuf<int64_t> crow_s, crow_m, crow_a;  // block-diagonal coarse solve: per-row block start, size, offset
  bool replicated = false;                          // levels address shared blocks through row maps
  exfem::DevBuf<double> cb64, cx64;
  exfem::DevBuf<float> cb32, cx32;
};

struct exfem_solver_s {
  exfem_block_s* blk = nullptr;
  // further element blocks over the same nodes (a model of several blocks,
  // gfem/model.py:466-486): the operator is the sum of every block's product, the
  // prescribed DOFs (identity rows of opA) those of the first block
  std::vector<exfem_block_s*> more;
  std::vector<const double*> more_Ke;
  exfem::DevBuf<double> mb64;  // product of one further block
  exfem::DevBuf<float> mb32;
  bool csr_dirty = false;      // EXFEM_OP_CSR_F64: element matrices changed since the last assembly
  exfem_amg_s* amg = nullptr;
  int op = EXFEM_OP_MF_F32, pc = EXFEM_PC_AMG;
  const double* Ke = nullptr;
  exfem::BlockCsr csr;  // EXFEM_OP_CSR_F64: the assembled operator
  int64_t n = 0;
  // workspace
  exfem::DevBuf<double> x64, r64, z64, p64, Ap64, b64, t64, dinv64, diag64;
  exfem::DevBuf<float> x32, r32, z32, p32, Ap32, b32, t32, dinv32;
  exfem::DevBuf<double> partial, dscr;
  exfem::DevBuf<unsigned> counter;
  exfem::DevBuf<exfem::PcgScal> scal;
  exfem::PcgScal* h_scal = nullptr;  // pinned
  exfem::DevBuf<double> cx64, cr64, cd64;  // EXFEM_PC_CHEBY work vectors
  exfem::DevBuf<float> cx32, cr32, cd32;
  double cheb_lmax = 0.0;                  // EXFEM_PC_CHEBY spectral bound of D^-1 A
  double g_lmax[2] = {0.0, 0.0};           // the bound each captured graph was recorded with
  bool diag_ready = false;
  int mixed_mode = 1;  // exfem_solver_mixed: 1 = reliable updates, 0 = restarted refinement (the reference's)
  double mixed_delta = 0.1;  // reliable updates: replace the residual after this reduction
  uint64_t diag_tan_gen = 0, diag_bc_gen = 0, graph_bc_gen = 0;
  // CUDA graphs of the PCG iterations, one per precision: with device_loop a
  // graph whose conditional while node repeats one iteration until the device
  // scalars say done (no host round trips between iterations), else a graph of
  // `chunk` iterations launched from the host until done
  int use_graph = 1, chunk = 8, device_loop = 1;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool gloop[2] = {false, false};
  uint64_t graph_gen = 0;  // counts (re)builds of the PCG graphs
  // the reliable-update mixed solve as one graph (built with device_loop)
  cudaGraphExec_t gmixed = nullptr;
  uint64_t gmixed_gen = 0;
  exfem::DevBuf<exfem::MixedScal> mx_scal;
  exfem::DevBuf<double> mx_b, mx_x;
  // the Newton increment as one graph (exfem_newton_increment)
  cudaGraphExec_t gnewton = nullptr;
  uint64_t gnewton_gen = 0;
  exfem::DevBuf<exfem::NewtonScal> nw_scal;
  exfem::DevBuf<double> nw_u, nw_ut, nw_du, nw_r, nw_f, nw_t, nw_fext, nw_start, nw_s_old, nw_s_new, nw_s_trial;
  std::vector<const double*> g_Ke[2];
  ~exfem_solver_s();
};
