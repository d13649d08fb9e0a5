/*
 * exfem_b200 — C ABI of the B200 structural hot path (element force / tangent
 * kernels, element-by-element matvecs, smoothed-aggregation V-cycle, PCG and
 * mixed-precision refinement) behind the interfaces of EXFEM's ``gfem`` 0.3.0.
 *
 * Conventions (all entry points):
 *   - plain C types only; no exceptions cross the boundary;
 *   - every call returns an int status: EXFEM_OK (0), EXFEM_NOT_CONVERGED (1,
 *     results still written), or a negative error; exfem_last_error() gives a
 *     message for the calling host thread;
 *   - device pointers passed in are borrowed for the duration of the call and
 *     owned by the caller; host pointers are read before the call returns;
 *   - "stream" is a cudaStream_t passed as void*; NULL means the legacy default
 *     stream; work is stream ordered and calls return without a device sync
 *     unless they must read a device scalar (solvers, which say so);
 *   - handles (block, amg, solver) own their device memory and are not thread
 *     safe: one host thread per handle;
 *   - DOF numbering is node-interleaved, dof = 3*node + component, as in the
 *     reference (gfem/model.py:157-158).
 */
#ifndef EXFEM_B200_H
#define EXFEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  EXFEM_OK = 0,
  EXFEM_NOT_CONVERGED = 1,
  EXFEM_ERR_ARG = -1,
  EXFEM_ERR_CUDA = -2,
  EXFEM_ERR_OOM = -3,
  EXFEM_ERR_TIMEOUT = -4,
  EXFEM_ERR_NONFINITE = -5,
  EXFEM_ERR_UNSUPPORTED = -6
};

/* element types: gfem/elements.py:124-125 (HEX8, fbar=True -> B-bar for small
 * strain) and gfem/elements.py:177-179 (TET10); ELEMENTS map 194-197 */
enum { EXFEM_C3D8 = 0, EXFEM_C3D10 = 1 };
/* materials: gfem/materials.py:56-68 LinearElastic, 228-302 J2Plasticity */
enum { EXFEM_LINEAR_ELASTIC = 0, EXFEM_J2 = 1 };
/* arithmetic types of buffers passed as void* */
enum { EXFEM_F64 = 0, EXFEM_F32 = 1, EXFEM_BF16 = 2 };
/* assembly of element vectors into nodal vectors */
enum { EXFEM_ASSEMBLE_GATHER = 0, EXFEM_ASSEMBLE_COLOUR = 1 };
/* linear-operator kinds of a solver */
enum { EXFEM_OP_EBE_F64 = 0, EXFEM_OP_MF_F64 = 1, EXFEM_OP_MF_F32 = 2, EXFEM_OP_CSR_F64 = 3 };
/* preconditioners of a solver; EXFEM_PC_CHEBY is the set-up-free Chebyshev-Jacobi
 * polynomial of gfem/solvers.py:289-306 (degree 6 in D^-1 A over [lmax/30, lmax],
 * lmax from 25 power iterations x 1.1, gfem/solvers.py:328-342) */
enum { EXFEM_PC_NONE = 0, EXFEM_PC_JACOBI = 1, EXFEM_PC_AMG = 2, EXFEM_PC_CHEBY = 3 };

#define EXFEM_MAX_TABLE 32

/* Material parameters.  Mirrors the constructor arguments of
 * gfem/materials.py:56-68 (LinearElastic(E, nu)) and 236-256
 * (J2Plasticity(E, nu, table, Hk)).  For J2, (sy_tab, ep_tab) is the hardening
 * table *after* the reference's extension (one-row tables become perfect
 * plasticity, and a last point at eps_p = 1e6 continues the final slope). */
typedef struct {
  int kind;
  double E, nu;
  double Hk;
  int ntab;
  double sy_tab[EXFEM_MAX_TABLE];
  double ep_tab[EXFEM_MAX_TABLE];
} exfem_material;

typedef struct exfem_block_s* exfem_block;
typedef struct exfem_amg_s* exfem_amg;
typedef struct exfem_solver_s* exfem_solver;
typedef struct exfem_batch_s* exfem_batch;
typedef struct exfem_queue_s* exfem_queue;

/* ------------------------------------------------------------ library */
int exfem_version(void);
const char* exfem_last_error(void);

/* ------------------------------------------------------------ blocks
 * One element block = one element type + one material over a node set
 * (gfem/model.py:21-26 Block.__init__, :362-365 Model.add_block).  Creation
 * uploads coordinates and connectivity, builds the atomic-free gather plan
 * (gfem/model.py:241-261, bit-identical), a greedy element colouring, and the
 * per-element geometry streams of the matrix-free operator. */
int exfem_block_create(int etype, const exfem_material* mat, int64_t nn, const double* X_host,
                       int64_t ne, const int32_t* conn_host, exfem_block* out);
int exfem_block_destroy(exfem_block b);
/* the block's kernels wait on asynchronous copies and tensor-core operations with
 * bounded waits; one that gives up sets a device flag instead of hanging.  Returns
 * EXFEM_ERR_TIMEOUT (and clears the flag) if that happened since the last check,
 * EXFEM_OK otherwise; the solver calls check it themselves.  No counterpart in the
 * reference. */
int exfem_block_status(exfem_block b, void* stream);
/* failure detection self-test: a kernel waits, with a limit of `polls` polls, on a
 * barrier nothing arrives on; returns EXFEM_ERR_TIMEOUT when the wait gave up and the
 * kernel returned (the expected result; the context stays usable). */
int exfem_selftest_bounded_wait(int polls, void* stream);
/* sizes: ne, nn, nnode, ngp, nstate, gather-plan width vmax, colour count,
 * affine (1 if every C3D10 has straight edges), device bytes held */
int exfem_block_query(exfem_block b, int64_t* ne, int64_t* nn, int* nnode, int* ngp, int* nstate,
                      int* vmax, int* ncolour, int* affine, int64_t* device_bytes);
/* index maps, copied to host: gather plan (nn, vmax) int32 with sentinel ne*nnode
 * (gfem/model.py:241-261); element colours (ne,) */
int exfem_block_gather_plan(exfem_block b, int32_t* plan_host);
int exfem_block_colours(exfem_block b, int32_t* colour_host);
/* element-tile maps of the matrix-free operator.  The block's elements are put
 * in a tile order (grouped by mesh component, in the order of each component's
 * first element, then along a Morton curve of the corner-coordinate sums, ties by
 * element index); a tile is `tile` consecutive positions of that order, and slot
 * s = a*tile + p is local node a of the element at tile position p.  tile_info:
 * tile count, total length of the node lists and the longest list; tile_maps,
 * copied to host: ptr (ntile+1), the sorted distinct nodes of every tile (the
 * order of its shared-memory records), for each listed node the end of its run of slots
 * (uint16), and per tile the slots grouped by node in node order, increasing
 * within a node (ntile, nnode*tile, zero padded); tile_order: the tile size and
 * the order (ne,) as position -> element.  No counterpart in the reference. */
int exfem_block_tile_info(exfem_block b, int64_t* ntile, int64_t* nlist, int* maxu);
int exfem_block_tile_maps(exfem_block b, int32_t* ptr_host, int32_t* nodes_host, uint16_t* nend_host,
                          uint16_t* perm_host);
int exfem_block_tile_order(exfem_block b, int* tile, int32_t* order_host);
/* connectivity of every tile position (ne, nnode) in the local numbering the
 * tiles use: linear-elastic C3D10 blocks renumber face-sharing pairs (see
 * exfem_host_tile_pairs), other blocks keep each element's own numbering. */
int exfem_block_tile_conn(exfem_block b, int32_t* conn_tile_host);
/* elements per matrix-free tile (128 or 256) for blocks of element type etype
 * created after the call, process-wide; chosen by the autotuner
 * (exfem_b200.tuning).  No counterpart in the reference. */
int exfem_set_tile(int etype, int tile);
int exfem_get_tile(int etype, int* tile);
/* per-element stiffness scale (gfem/model.py:449-463, fields["scale"]); NULL = 1 */
int exfem_block_set_scale(exfem_block b, const double* scale_host);
/* per-element Lame parameters (ne each) of a linear-elastic block, used by every
 * element kernel (forces, stresses, Ke, the matrix-free operator and its
 * diagonal) in place of the material's; lets one block hold many
 * independent instances with different E and nu.  NULL, NULL = the material's.
 * No counterpart in the reference (one material per block, gfem/model.py:21-26). */
int exfem_block_set_lame(exfem_block b, const double* lam_host, const double* mu_host);
/* prescribed-DOF mask (ndof bytes, 1 = fixed): operators apply the reference's
 * opA, y = free*K(free*v) + fixed*v (gfem/solvers.py:257-267); NULL = all free */
int exfem_block_set_fixed(exfem_block b, const uint8_t* fixed_host);

/* ------------------------------------------------------------ element kernels (FP64)
 * Internal force f(u) with new Gauss-point states (gfem/model.py:466-477
 * Model.internal_force over Block.force 70-81).  u, f: (ndof); state_old,
 * state_new: (ne, ngp, nstate) or NULL for the linear-elastic material;
 * fe: optional (ne, nnode, 3) element forces.  assembly = EXFEM_ASSEMBLE_GATHER
 * reduces through the gather plan (reference order), EXFEM_ASSEMBLE_COLOUR by
 * a colour-by-colour scatter; both are deterministic.  Also refreshes the
 * block's per-Gauss-point consistent-tangent data at (u, state_old). */
int exfem_internal_force(exfem_block b, const double* u, const double* state_old,
                         double* state_new, double* fe, double* f, int assembly, void* stream);
/* Element tangents Ke (ne, 3*nnode, 3*nnode) row-major in dtype F64/F32/BF16
 * (gfem/model.py:83-111 Block.stiff, 479-483 Model.element_stiffness). */
int exfem_element_stiffness(exfem_block b, const double* u, const double* state_old, int dtype,
                            void* Ke, void* stream);
/* Refresh only the per-Gauss-point tangent data of the matrix-free operator at
 * (u, state_old) — what ``jax.jvp`` re-derives on every product in
 * gfem/model.py:488-490 (Model.tangent_jvp). */
int exfem_tangent_update(exfem_block b, const double* u, const double* state_old, void* stream);
/* Matrix-free tangent product with the block's current tangent data, dtype F64
 * or F32: y = opA(v) when apply_bc != 0 (gfem/solvers.py:257-267), else the bare
 * y = K(u) v of Model.tangent_jvp (gfem/model.py:488-490), which it replaces. */
int exfem_tangent_matvec(exfem_block b, int dtype, const void* v, void* y, int apply_bc, void* stream);
/* Diagonal of the matrix-free tangent (FP64, ndof); fixed DOFs get 1. */
int exfem_tangent_diagonal(exfem_block b, double* diag, void* stream);
/* Stored-tangent EbE product with Ke (ne, nd, nd) FP64 and reference-order
 * gather assembly: y = opA(v) when apply_bc != 0 (gfem/model.py:264-267
 * gather_matvec within opA, gfem/solvers.py:257-267), else y = K v
 * (gfem/model.py:162-166 ops_matvec). */
int exfem_ebe_matvec(exfem_block b, const double* Ke, const double* v, double* y, int apply_bc, void* stream);
/* stored-Ke product for nrhs (1, 2, 3, 4, 8 or 16) right-hand sides at once on the tensor cores:
 * Ke (ne, nd, nd) BF16 as written by exfem_element_stiffness with EXFEM_BF16, V and
 * Y (ndof, nrhs) FP32 with the right-hand sides fastest; V is rounded to BF16 and
 * the products accumulate in FP32 (tcgen05.mma).  apply_bc as exfem_ebe_matvec.
 * The multi-load-case form of gfem/model.py:264-267 (gfem/optimize.py:116-143
 * vmaps the single product over load cases). */
int exfem_ebe_matvec_bf16_multi(exfem_block b, const void* Ke_bf16, int nrhs, const float* V, float* Y,
                                int apply_bc, void* stream);
/* Stored-Ke product for nrhs (1..16) right-hand sides at once on the CUDA cores:
 * Ke (ne, nd, nd) in ke_dtype (EXFEM_BF16, EXFEM_F32 or EXFEM_F64, as written by
 * exfem_element_stiffness), V and Y (ndof, nrhs) with the right-hand sides fastest,
 * FP32 for BF16 / FP32 Ke (FP32 accumulation) and FP64 for FP64 Ke.  One read of Ke
 * serves every right-hand side; element rows are summed per node through the
 * gather plan in the reference's order.  apply_bc as exfem_ebe_matvec.  The
 * multi-load-case form of gfem/model.py:264-267 (gfem/optimize.py:116-143 vmaps the
 * single product over load cases). */
int exfem_ebe_matvec_multi(exfem_block b, const void* Ke, int ke_dtype, int nrhs, const void* V, void* Y,
                           int apply_bc, void* stream);
/* Jacobi PCG over nrhs (1, 2, 3, 4, 8 or 16) load cases at once with the stored FP64
 * element matrices Ke and the block's prescribed DOFs (gfem/optimize.py:116-143:
 * linalg.pcg, gfem/linalg.py:21-47, vmapped over the cases, with A(v) = free K
 * (free v) + (1 - free) v and the inverse assembled diagonal, 1 on prescribed
 * rows): B, X (ndof, nrhs) FP64 with the cases fastest; B should be zero on
 * prescribed DOFs (the reference passes free * f).  One product per iteration for
 * all cases; each case keeps its own scalars and stops on its own test (r.r <=
 * tol^2 max(b.b, 1e-300) or k >= maxiter); iters and relres (nrhs) per case.  The
 * loop runs on the device (one graph launch).  EXFEM_NOT_CONVERGED if a case
 * stopped on maxiter.  Synchronises the stream. */
int exfem_multi_pcg(exfem_block b, const double* Ke, int nrhs, const double* B, double* X, double tol, int maxiter,
                    int* iters, double* relres, void* stream);
/* Diagonal of stored Ke (gfem/model.py:169-173 ops_diagonal), FP64 (ndof). */
int exfem_ebe_diagonal(exfem_block b, const double* Ke, double* diag, void* stream);
/* Initial-stress (geometric) stiffness of every element under its constant
 * Cauchy stress S (ne, 3, 3) FP64 (gfem/model.py:113-117 geo_stiff, 541-553
 * geometric_ops, with the stresses of Model.stresses): Kg (ne, 3 nnode, 3 nnode)
 * FP64 row-major, K[3a+i, 3b+j] = delta_ij sum_g vol_g dN_a/dX . S . dN_b/dX. */
int exfem_geometric_stiffness(exfem_block b, const double* S, double* Kg, void* stream);
/* Volume-averaged Cauchy stress (ne, 3, 3), von Mises (ne) and PEEQ (ne)
 * (gfem/model.py:530-539 Model.stresses over Block.cauchy 129-137). */
int exfem_stresses(exfem_block b, const double* u, const double* state, double* S,
                   double* mises, double* peeq, void* stream);

/* ------------------------------------------------------------ AMG hierarchy
 * Device copy of a smoothed-aggregation hierarchy set up on the host
 * (gfem/linalg.py:103-136 AMG.__init__/params).  Levels are added fine to
 * coarse as CSR (int64 indptr, int32 indices, FP64 data): level matrix A
 * (n x n), prolongator P (n x nc), restriction R = P^T (nc x n), Jacobi
 * inverse diagonal dinv (n) and the Chebyshev bound rho.  The coarsest matrix is
 * given densely; its regularised Cholesky factor's inverse is formed on the
 * host (gfem/linalg.py:126-133). */
int exfem_amg_create(exfem_amg* out);
int exfem_amg_destroy(exfem_amg h);
int exfem_amg_add_level(exfem_amg h, int64_t n, int64_t nc,
                        const int64_t* A_ptr, const int32_t* A_idx, const double* A_val,
                        const int64_t* P_ptr, const int32_t* P_idx, const double* P_val,
                        const int64_t* R_ptr, const int32_t* R_idx, const double* R_val,
                        const double* dinv, double rho);
int exfem_amg_set_coarse(exfem_amg h, int64_t nc, const double* Ainv_dense);
/* Smoothed-aggregation hierarchy set up on the device from a block's element
 * matrices Ke (ne, 3 nnode, 3 nnode) FP64 (device pointer) and its prescribed
 * DOFs (exfem_set_fixed): the set-up of AMG.__init__ (gfem/linalg.py:103-136,
 * pyamg.smoothed_aggregation_solver with rigid-body modes, theta = 0 strength,
 * standard aggregation, Jacobi-smoothed prolongator omega = 4/3 with absolute
 * row-sum weighting, Galerkin R A P, max_coarse rows, <= 10 levels, 15-step
 * power-iteration rho x 1.1, regularised Cholesky of the coarsest matrix) with
 * the assembly and every matrix product on the GPU and only graph work on the
 * host.  h must be empty (exfem_amg_create).  The mesh level stores no matrix
 * unless keep_level0 is set; it is then smoothed with the block's matrix-free
 * product (solvers, exfem_amg_vcycle with level0).  Synchronises the stream. */
int exfem_amg_setup_block(exfem_amg h, exfem_block b, const double* Ke, int max_coarse, int keep_level0,
                          void* stream);
/* The same set-up for a model of several blocks over one node set (a list of
 * element blocks, gfem/model.py:466-486, assembled into one matrix as
 * gfem/model.py:176-192 does from the stiffness ops of all blocks): blocks[i] with
 * its element matrices Kes[i]; A_0 sums the blocks in order through each block's
 * gather plan; the prescribed DOFs are those of blocks[0]. */
int exfem_amg_setup_blocks(exfem_amg h, int nblk, const exfem_block* blocks, const double* const* Kes,
                           int max_coarse, int keep_level0, void* stream);
/* level count (coarsest included) and, for the first cap levels, rows and
 * operator nonzeros (AMG.info, gfem/linalg.py:135, 148-154). */
int exfem_amg_info(exfem_amg h, int cap, int* nlevels, int64_t* rows, int64_t* nnz);
/* copy one level of a (not replicated) hierarchy to the host: what 0 = A, 1 = P,
 * 2 = R (scalar CSR: rows, cols, nnz; ptr (rows+1), idx, val when not NULL; a level
 * without a stored matrix reports nnz 0), 3 = the inverse diagonal (rows values in
 * val); rho (may be NULL) receives the level's spectral bound.  The coarsest
 * level's dense inverse: exfem_amg_export_coarse (Ainv nc*nc, may be NULL).  Used to
 * merge hierarchies set up on the device into a batched union. */
int exfem_amg_export_level(exfem_amg h, int level, int what, int64_t* rows, int64_t* cols, int64_t* nnz,
                           int64_t* ptr, int32_t* idx, double* val, double* rho);
int exfem_amg_export_coarse(exfem_amg h, int64_t* nc, double* Ainv);
/* Union of independent hierarchies (batched solves, no counterpart in the
 * reference): per-row spectral bounds of level `level` (n doubles; each row
 * smoothed with its own instance's Chebyshev coefficients, degree 2; a bound of 0
 * marks a pass-through row with smoothing switched off, used where an instance
 * has fewer levels than the union and identity levels relay it), and a
 * block-diagonal coarsest solve: nblk blocks at row offsets (nblk+1, int64) whose
 * inverses are concatenated row-major in Ainv_blocks. */
int exfem_amg_set_level_rows(exfem_amg h, int level, const double* rho_rows);
int exfem_amg_set_coarse_blocks(exfem_amg h, int64_t nblk, const int64_t* offsets, const double* Ainv_blocks);
/* Replicate a block-diagonal hierarchy of nblk independent blocks into ninst
 * instances, instance i a copy of block inst_block[i], laid out one after the
 * other at every level (batched solves of several right-hand sides per mesh; no
 * counterpart in the reference).  level_offsets holds (levels + 1) rows of
 * nblk + 1 row offsets of the blocks, the last row for the coarsest level.  The
 * stored matrices are shared by the copies; call after every level and the
 * coarse solve are set, once. */
int exfem_amg_replicate(exfem_amg h, int nblk, const int64_t* level_offsets, int ninst, const int32_t* inst_block);
/* One V-cycle z = M(r) (gfem/linalg.py:156-195, Chebyshev degree 2 over
 * [rho/30, rho]) in dtype F64 or F32; the coarse solve is FP64 in both.  When
 * level0 is a block, level 0 is smoothed with that block's matrix-free tangent
 * and the given inverse diagonal dinv0 (same dtype) instead of the stored level
 * matrix (gfem/solvers.py:311-314). */
int exfem_amg_vcycle(exfem_amg h, int dtype, const void* r, void* z, exfem_block level0,
                     const void* dinv0, void* stream);
/* Allocation-free V-cycle (no counterpart in the reference).  Same result and
 * arguments as exfem_amg_vcycle, for callers that must not allocate device
 * memory during a call: code recording a CUDA graph by stream capture, where
 * cudaMalloc is not permitted, and hosts whose device memory belongs to another
 * allocator.  exfem_amg_vcycle allocates its per-level work vectors on first use;
 * this variant takes them from one static device array of
 * EXFEM_VCYCLE_NOALLOC_BYTES that every GPU loading the library holds until exit,
 * and calls no cudaMalloc, cudaFree or allocating routine.  A hierarchy whose
 * work vectors (6 per level and 2 coarse, each rounded up to 256 bytes) exceed
 * the array is rejected with EXFEM_ERR_ARG, and so, before any launch, is a
 * level without a stored matrix that no level-0 block smooths (the device set-up
 * without keep_level0).  A call outside a stream capture looks up the array's
 * device address (cudaGetSymbolAddress) on the current device; a call inside a
 * capture uses the address of the last call on that device outside one, so the
 * first call on a device should come before any stream capture.  All calls
 * share the array: calls that overlap on the GPU race, so the caller must
 * serialise them. */
#define EXFEM_VCYCLE_NOALLOC_BYTES (8u << 20)
int exfem_amg_vcycle_noalloc(exfem_amg h, int dtype, const void* r, void* z, exfem_block level0,
                             const void* dinv0, void* stream);

/* ------------------------------------------------------------ solvers
 * A solver binds an operator (EXFEM_OP_*) of a block, a preconditioner
 * (EXFEM_PC_*; an AMG handle for EXFEM_PC_AMG) and device workspace.
 * EXFEM_OP_EBE_F64 needs exfem_solver_set_ke before solving.  EXFEM_OP_CSR_F64 (the
 * reference's operator="csr", gfem/model.py:195-238, gfem/solvers.py:406-412): the
 * element matrices passed to exfem_solver_set_ke are assembled on the device into
 * one FP64 CSR matrix (node-adjacency pattern, built once; prescribed DOFs as
 * identity rows and columns), and the solver multiplies by it. */
int exfem_solver_create(exfem_block b, int op_kind, int pc_kind, exfem_amg amg, exfem_solver* out);
int exfem_solver_destroy(exfem_solver s);
int exfem_solver_set_ke(exfem_solver s, const double* Ke);
/* A model of several element blocks (gfem/model.py:466-486: the reference's
 * operators loop over the blocks and its gather plan covers all of them,
 * gfem/model.py:241-261): add_block adds a further block over the solver block's
 * node set; every operator of the solver (products, diagonal, the FP64 residual
 * of the mixed solves, the level-0 smoothing) is then the sum over the blocks, with
 * the prescribed DOFs of the first block (give every block the same mask).
 * set_ke_block sets the stored element matrices of block i (0 = the solver's own
 * block, as exfem_solver_set_ke); EXFEM_OP_CSR_F64 assembles all blocks into one
 * matrix at the next solve. */
int exfem_solver_add_block(exfem_solver s, exfem_block b);
int exfem_solver_set_ke_block(exfem_solver s, int block, const double* Ke);
/* Refresh the Jacobi / level-0 inverse diagonal from the current operator
 * (gfem/solvers.py:312-313 dinv0). Called automatically by the first solve. */
int exfem_solver_refresh_diagonal(exfem_solver s, void* stream);
/* EXFEM_PC_CHEBY: the spectral bound in use (refreshed with the diagonal, i.e. when
 * the operator's tangent or prescribed DOFs change; 0 before the first solve). */
int exfem_solver_cheby_bound(exfem_solver s, double* lmax);
/* Use CUDA graphs for the PCG iteration loop (default on) and the number of
 * iterations captured per graph launch (host-driven loop only). */
int exfem_solver_set_graph(exfem_solver s, int enable, int chunk);
/* With graphs on: 1 (default) runs the whole PCG loop inside one graph launch, a
 * conditional while node repeating one captured iteration until the device-side
 * stopping test (r.r <= tol^2 b.b or k >= maxiter) ends it, so no host round trip
 * falls between iterations; 0 launches graphs of `chunk` iterations from the host
 * and reads the stopping test after each. */
int exfem_solver_set_loop(exfem_solver s, int device_loop);
/* PCG in the operator's precision with FP64 scalars and dot products
 * (gfem/linalg.py:21-47): x0 = 0, stop when r.r <= tol^2 b.b or k >= maxiter.
 * b, x: FP64 device (ndof).  Synchronises the stream to read the iteration count.
 * Returns EXFEM_NOT_CONVERGED when relres > 1e-3 or is not finite (the
 * reference's warning condition, gfem/solvers.py:472-473). */
int exfem_solver_pcg(exfem_solver s, const double* b, double* x, double tol, int maxiter,
                     int* iters, double* relres, void* stream);
/* FP32 matrix-free PCG with FP32 V-cycle inside FP64 iterative refinement with an
 * FP64 matrix-free residual, until ||b - A x|| <= tol ||b|| (gfem/solvers.py:344-384
 * _LinearSystem._mixed); how the FP32 work is organised: exfem_solver_set_mixed_mode. */
int exfem_solver_mixed(exfem_solver s, const double* b, double* x, double tol, double inner_tol,
                       int max_pass, int maxiter, int* iters, int* passes, double* relres,
                       void* stream);
/* How exfem_solver_mixed runs its FP32 work.  Mode 1 (default): one FP32 PCG
 * recursion whose residual is replaced by the FP64 residual b - A x whenever it
 * has dropped by delta (default 0.1) since the last replacement, the search direction kept
 * (reliable updates, Sleijpen & van der Vorst 1996); inner_tol is not used, `passes`
 * returns the number of replacements (at most 100 x max_pass).  Mode 0: the
 * reference's restarted refinement (gfem/solvers.py:344-384): each pass a new FP32
 * PCG to inner_tol on the scaled FP64 residual (passes after the first stop at 4x
 * the first pass's iterations). */
int exfem_solver_set_mixed_mode(exfem_solver s, int mode, double delta);
/* One increment of the static Newton procedure (gfem/solvers.py:607-683:
 * StaticSolver._predictor and _newton with the reference's convergence test and
 * 4-step backtracking line search) as one graph launch: the residual norms, the
 * convergence test, the step lengths and every linear solve (the reliable-update
 * mixed solve, FP32 matrix-free with the AMG V-cycle inside FP64 replacements, to
 * cg_tol) run on the device; the host reads the result once.  For a solver with
 * EXFEM_OP_MF_F32, EXFEM_PC_AMG, reliable updates, graphs and the device loop on, of
 * one block or several (exfem_solver_add_block: forces, tangents and products are
 * summed over the blocks in order); the blocks' prescribed DOFs are the step's.  u:
 * converged displacements of the previous increment (the predictor's start),
 * states_old: per block its J2 states (ne, ngp, nstate; the entry of an elastic block
 * is ignored and may be NULL, as may the whole array for a model without J2 blocks),
 * fext: the external force at the end of the increment, start: u with the prescribed
 * values of the increment's end on the prescribed DOFs; qref: the running force
 * scale (in and out).  Out: u_out and states_out (per block, like states_old) at the
 * last residual evaluation, corrections (Newton corrections when
 * converged, max_iter otherwise), converged (0 when the increment failed: not
 * converged in max_iter <= 64 iterations or a non-finite residual), ratios (the
 * residual ratio of every iteration, max_iter values at most), lin_stats (2: FP32
 * iterations and FP64 replacements of the increment's last linear solve; may be
 * NULL). */
int exfem_newton_increment(exfem_solver s, const double* u, const double* const* states_old, const double* fext,
                           const double* start, double rtol, int max_iter, int line_search, double cg_tol,
                           int cg_maxiter, double* qref, double* u_out, double* const* states_out, int* corrections,
                           int* converged, double* ratios, int* lin_stats, void* stream);

/* ------------------------------------------------------------ batched solves
 * Many independent linear-elastic systems in one set of launches (no counterpart
 * in the reference, which solves one Model at a time; nearest is the vmapped
 * multi-RHS PCG of gfem/optimize.py:116-143).  `blk` is the union of the
 * instances' meshes (per-element Lame parameters, prescribed-DOF mask), `amg` the
 * block-diagonal union of their hierarchies (exfem_amg_set_level_rows,
 * exfem_amg_set_coarse_blocks), dof_offsets (ninst+1) the instances' contiguous
 * DOF ranges.  The solve runs FP32 matrix-free AMG-PCG per instance inside FP64
 * iterative refinement with per-instance scaling, scalars and stopping rule
 * ||b_i - A x_i|| <= tol ||b_i||; iters (ninst) and relres (ninst) are per
 * instance.  Synchronises the stream. */
int exfem_batch_create(exfem_block blk, exfem_amg amg, int ninst, const int64_t* dof_offsets, exfem_batch* out);
int exfem_batch_destroy(exfem_batch b);
int exfem_batch_solve(exfem_batch b, const double* rhs, double* x, double tol, double inner_tol, int max_pass,
                      int maxiter, int* iters, int* passes, double* relres, void* stream);

/* ------------------------------------------------------------ request queue
 * Linear solves queued against resident solver handles, for hosts that are not
 * Python (the served stream behind the C ABI; no counterpart in the reference,
 * which solves one model per StaticSolver.solve call, gfem/solvers.py:481-605).
 * exfem_queue_create starts `workers` host threads on the current device, each
 * with its own CUDA stream.  exfem_queue_submit copies a right-hand side (the
 * solver's ndof FP64 values, host memory) and returns a request id; a worker
 * takes the oldest pending request whose solver is idle (one request per solver
 * handle at a time; requests of different handles run concurrently) and runs
 * exfem_solver_mixed with it to `tol` (the handle must be EXFEM_OP_MF_F32 with its
 * preconditioner set; the handle must not be used elsewhere while the queue holds
 * requests for it).  poll reports the state (EXFEM_REQ_*), iterations and relative
 * residual; wait blocks up to timeout_s seconds; result copies a finished request's
 * solution to x_host and forgets the request (returns the solve's status, or the
 * error of a failed or withdrawn one); cancel withdraws a request that has not
 * started (*withdrawn = 1) and leaves running or finished ones alone
 * (*withdrawn = 0).  destroy withdraws what is pending and waits for the running. */
enum { EXFEM_REQ_PENDING = 0, EXFEM_REQ_RUNNING = 1, EXFEM_REQ_DONE = 2, EXFEM_REQ_FAILED = 3,
       EXFEM_REQ_CANCELLED = 4 };
int exfem_queue_create(int workers, exfem_queue* out);
int exfem_queue_destroy(exfem_queue q);
int exfem_queue_submit(exfem_queue q, exfem_solver s, const double* rhs_host, double tol, int64_t* id);
int exfem_queue_poll(exfem_queue q, int64_t id, int* state, int* iters, double* relres);
int exfem_queue_wait(exfem_queue q, int64_t id, double timeout_s, int* state);
int exfem_queue_result(exfem_queue q, int64_t id, double* x_host, int* iters, int* passes, double* relres);
int exfem_queue_cancel(exfem_queue q, int64_t id, int* withdrawn);

/* ------------------------------------------------------------ host index builders
 * Host-side, no device work.  Gather plan of one connectivity exactly as
 * gfem/model.py:241-261 (plan must hold nn*vmax entries; call with plan = NULL to
 * get vmax; the plan of several blocks is that of their connectivities
 * concatenated as one flat list: ne = 1, nnode = the total slot count); greedy
 * colouring; standard aggregation of a symmetric strength graph (CSR pattern)
 * for the smoothed-aggregation set-up. */
int exfem_host_gather_plan(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int32_t* plan,
                           int* vmax);
int exfem_host_colouring(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int32_t* colour,
                         int* ncolour);
int exfem_host_standard_aggregation(int64_t n, const int64_t* ptr, const int32_t* idx,
                                    int32_t* agg, int64_t* nagg);
/* Host graph steps of the device smoothed-aggregation set-up (exfem_amg_setup_block),
 * exported for checking (no counterpart in the reference; pyamg does these steps
 * inside smoothed_aggregation_solver, gfem/linalg.py:113-116):
 * node adjacency of a mesh (row n: every node sharing an element with n, itself
 * included, ascending) — call with idx NULL for ptr (nn+1) and *nnz, then with idx;
 * tentative prolongator of an aggregation (per aggregate, modified Gram-Schmidt of
 * the K near-null-space columns B (nb*bs, K) over its DOFs in increasing order,
 * columns below 1e-10 of their norm dropped): Q (nb*bs, K) orthonormal rows of each
 * DOF, Bc (nagg*K, K) the coarse near-null space;
 * coarsest inverse: A (n, n) symmetrised, 1e-13 max|A| added to the diagonal,
 * Cholesky, Ainv = L^-T L^-1 (gfem/linalg.py:122-133). */
int exfem_host_node_adjacency(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int64_t* nnz, int64_t* ptr,
                              int32_t* idx);
int exfem_host_fit_candidates(int64_t nb, int bs, int K, const int32_t* agg, int64_t nagg, const double* B,
                              double* Q, double* Bc);
int exfem_host_coarse_inverse(int64_t n, const double* A, double* Ainv);
/* Strength filter of the device set-up (theta = 0: the blocks of a level matrix that
 * are not all zero), exported for checking: the entries q of the pattern (nrows,
 * ptr, idx) with flag[q] set, row by row in their order.  *nnz = their count;
 * ptr_out (nrows + 1), idx_out (their columns) and keep_out (their positions in
 * idx) are written when idx_out is not NULL.  No counterpart in the reference
 * (pyamg's classical strength with theta = 0 inside smoothed_aggregation_solver,
 * gfem/linalg.py:113-116). */
int exfem_host_filter_pattern(int64_t nrows, const int64_t* ptr, const int32_t* idx, const uint8_t* flag,
                              int64_t* nnz, int64_t* ptr_out, int32_t* idx_out, int64_t* keep_out);
/* tile order of the matrix-free operator (see exfem_block_tile_order) for a mesh
 * of ne elements with nnode nodes each, the first ncorner of them corners:
 * order (ne,) position -> element.  No counterpart in the reference. */
int exfem_host_tile_order(int64_t nn, int64_t ne, int nnode, int ncorner, const double* X,
                          const int32_t* conn, int32_t* order);
/* face pairs of a C3D10 tile order (linear-elastic blocks): order (ne,) in/out,
 * conn_tile (ne, 10) out.  Elements sharing a face are put at positions 2j, 2j+1
 * with the face's corners (p, q, r) at local 0, 1, 2 of the first and 1, 0, 2 of
 * the second (both positively oriented), so the product loads and adds their six
 * shared nodes once.  No counterpart in the reference. */
int exfem_host_tile_pairs(int64_t ne, const int32_t* conn, int32_t* order, int32_t* conn_tile);
/* tile maps of the matrix-free product (see exfem_block_tile_maps) for a
 * connectivity already in tile order: per tile its sorted distinct nodes, nend
 * and perm.  Call with ptr = NULL for ntile and nlist (the total list length),
 * then with ptr (ntile+1), nodes (nlist), nend (nlist) and perm
 * (ntile * nnode * tile).  No counterpart in the reference. */
int exfem_host_tile_maps(int64_t nn, int64_t ne, int nnode, const int32_t* conn, int tile, int64_t* ntile,
                         int64_t* nlist, int32_t* ptr, int32_t* nodes, uint16_t* nend, uint16_t* perm);
/* boundary faces: keys (nface, 4) int64, each face's corner nodes sorted
 * ascending (triangles padded in front with -1); once[f] = 1 when no other face
 * has the same key, else 0.  The face matching of gfem/surfaces.py:182-221
 * (skin), by hashing the keys. */
int exfem_host_face_once(int64_t nface, const int64_t* keys, uint8_t* once);

#ifdef __cplusplus
}
#endif
#endif /* EXFEM_B200_H */
