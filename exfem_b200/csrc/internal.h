// Internal handle layouts and cross-file launchers of the exfem_b200 library.
#pragma once
#include <cuda_bf16.h>

#include <memory>
#include <vector>

#include "common.cuh"
#include "element_math.cuh"

struct exfem_block_s {
  int device = 0;
  int etype = 0, nnode = 0, ngp = 0, nstate = 1, nd = 0;
  int64_t ne = 0, nn = 0;
  exfem::MatDev mat{};
  exfem_material mat_in{};
  // mesh
  exfem::DevBuf<double> X;            // (nn, 3)
  exfem::DevBuf<int32_t> conn;        // (ne, nnode)
  exfem::DevBuf<double> scale;        // (ne), empty = 1
  exfem::DevBuf<double> lam_e, mu_e;  // (ne) per-element Lame parameters, empty = material's
  // index maps
  int vmax = 0;
  exfem::DevBuf<int32_t> plan;        // (nn, vmax), sentinel ne*nnode
  std::vector<int32_t> plan_host;
  int ncolour = 0;
  std::vector<int64_t> colour_ptr;    // (ncolour+1) into colour_elems
  exfem::DevBuf<int32_t> colour_elems;
  std::vector<int32_t> colour_host;
  // boundary conditions
  exfem::DevBuf<uint8_t> fixed;       // (ndof) 1 = prescribed; empty = all free
  exfem::DevBuf<uint8_t> node_fixed;  // (nn) bit c set = dof c prescribed
  // matrix-free operator data: tiles of `tile` consecutive positions of the tile
  // order (elements by mesh component, then along a Morton curve), each with the
  // sorted list of distinct nodes it touches and per-slot local indices
  int affine = 1;
  int tile = 128;                     // elements per tile (128 or 256)
  int64_t ntile = 0;
  int maxu = 0;                       // largest distinct-node count of a tile
  std::vector<int32_t> order_host;    // (ne) tile position -> element
  exfem::DevBuf<int32_t> tpos;        // (ne) element -> tile position
  exfem::DevBuf<int32_t> order_dev;   // (ne) tile position -> element
  exfem::DevBuf<int32_t> conn_tile;   // (ne, nnode) connectivity per position, in the tiles' local numbering
  exfem::DevBuf<int32_t> tile_ptr;    // (ntile+1)
  exfem::DevBuf<int32_t> tile_nodes;  // concatenated sorted node lists
  exfem::DevBuf<int32_t> tile_nodes_bc;  // same, node | fixed-DOF bits << 29
  std::vector<int32_t> tile_nodes_host;
  exfem::DevBuf<uint16_t> lidx;       // tile-major (ntile, nnode*tile): list position of each slot's node
  exfem::DevBuf<uint16_t> tile_nend;  // per listed node: end of its slot run in tile_perm
  exfem::DevBuf<uint16_t> tile_perm;  // tile-major (ntile, nnode*tile) slots grouped by node
  exfem::DevBuf<int32_t> tile_dest;   // per tile-list entry: 0x80000000|node (only tile of the node) or its partials position
  exfem::DevBuf<int32_t> tile_dest_bc;  // same, fixed-DOF bits of directly written nodes at bits 28-30
  std::vector<int32_t> tile_dest_host;
  int64_t nmulti = 0;                 // nodes not listed by exactly one tile
  exfem::DevBuf<int32_t> multi_nodes; // (nmulti) those nodes, ascending
  exfem::DevBuf<int32_t> multi_nodes_bc;  // same, fixed-DOF bits at 28-30
  std::vector<int32_t> multi_nodes_host;
  exfem::DevBuf<int32_t> multi_ptr;   // (nmulti+1) their runs of partials
  exfem::DevBuf<double> partial;      // per-entry tile sums, (x, y, z, 0) per entry (FP64 or FP32 view)
  exfem::DevBuf<int> dev_err;         // set by bounded waits that give up
  int geo_stride = 0;                 // per-element geometry entries (without the Lame pair when uniform)
  exfem::DevBuf<double> geo64;        // tile-major (ntile, geo_stride, tile)
  exfem::DevBuf<float> geo32;
  int plastic_tangent = 0;            // 1 once tangent data differs from elastic
  exfem::DevBuf<double> tan64;        // tile-major (ntile, ngp*8, tile)
  exfem::DevBuf<float> tan32;
  // generations: tangent data and boundary-condition buffers (solvers compare)
  uint64_t tan_gen = 0, bc_gen = 0;
  // scratch
  exfem::DevBuf<double> ys;           // (ne*nnode*3) element vectors for gather assembly
  exfem::DevBuf<double> mp_work;      // multi-case Jacobi PCG: inverse diagonal, R, P, Q, partial sums, scalars
  exfem::DevBuf<double> ys_m64;       // (ne*nnode*3*nrhs) element rows of the FP64 multi-right-hand-side product
  exfem::DevBuf<float> ys_tc;         // (ne*nnode*3*nrhs) element rows of the tensor-core stored-Ke product
  int64_t ndof() const { return 3 * nn; }
};

namespace exfem {

struct Csr64 {  // device CSR, FP64 values and an FP32 copy
  int64_t n = 0, ncols = 0, nnz = 0;
  DevBuf<int64_t> ptr;
  DevBuf<int32_t> idx;
  DevBuf<double> v64;
  DevBuf<float> v32;
  // replicated blocks (optional): row r reads stored row rmap[r] and shifts its
  // column indices by cshift[r], so copies of a block share one set of entries
  DevBuf<int64_t> rmap, cshift;
};

// element kernels (element_ops.cu)
int launch_force(exfem_block_s* b, int mode, const double* u, const double* st_old, double* st_new,
                 double* fe, double* S, double* mises, double* peeq, cudaStream_t s);
int launch_gather_assemble(exfem_block_s* b, const double* ys, double* f, const double* v_opa,
                           const int* skip, cudaStream_t s);
int build_geometry(exfem_block_s* b);
int launch_stiffness(exfem_block_s* b, const double* u, const double* st_old, int dtype, void* Ke,
                     double* ediag, cudaStream_t s, const double* tan_in = nullptr);
int launch_colour_assemble(exfem_block_s* b, const double* fe, double* f, cudaStream_t s);
int launch_ebe_matvec(exfem_block_s* b, const double* Ke, const double* v, double* y,
                      const int* skip, cudaStream_t s, bool bc = true);
int launch_ebe_diagonal(exfem_block_s* b, const double* Ke, double* diag, cudaStream_t s);
int launch_geo_stiffness(exfem_block_s* b, const double* S, double* Kg, cudaStream_t s);
// matrix-free operator (matfree.cu)
template <class T>
int launch_mf_matvec(exfem_block_s* b, const T* v, T* y, const int* skip, cudaStream_t s, bool bc = true);
int launch_mf_diagonal(exfem_block_s* b, double* diag, cudaStream_t s);
// bounded device waits: read and clear a block's wait-failure flag (capi.cu); a
// kernel whose only wait can never complete (matfree.cu)
int block_wait_status(exfem_block_s* b, cudaStream_t s);
int launch_wait_selftest(int polls, int* err, cudaStream_t s);
// stored-Ke product for several right-hand sides on the tensor cores (ebe_tc.cu)
int launch_ebe_matvec_tc(exfem_block_s* b, const __nv_bfloat16* Ke, int nrhs, const float* V, float* Y,
                         cudaStream_t s, bool bc);
// multi-right-hand-side stored-Ke product on the CUDA cores (ebe_multi.cu); Ke in
// EXFEM_BF16 / EXFEM_F32 (V, Y FP32) or EXFEM_F64 (V, Y FP64)
int launch_ebe_matvec_multi(exfem_block_s* b, const void* Ke, int ke_dtype, int nrhs, const void* V, void* Y,
                            bool bc, cudaStream_t s);
// multi-case Jacobi PCG with stored FP64 Ke (ebe_multi.cu): B, X (ndof, nrhs) FP64
int multi_pcg(exfem_block_s* b, const double* Ke, int nrhs, const double* B, double* X, double tol, int maxiter,
              int* iters, double* relres, cudaStream_t s);
template <class VT>
int launch_gather_multi(exfem_block_s* b, const VT* ys, const VT* V, VT* Y, int nrhs, bool bc, cudaStream_t s);

// reductions and vector kernels (krylov.cu)
enum ModeForce { FORCE_FULL = 0, FORCE_TANGENT = 1, FORCE_STRESS = 2 };

}  // namespace exfem
