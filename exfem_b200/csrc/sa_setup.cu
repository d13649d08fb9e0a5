// Smoothed-aggregation hierarchy set up on the device for a block's element
// matrices (no counterpart in the reference, which sets up on the host through
// pyamg.smoothed_aggregation_solver, gfem/linalg.py:103-136, with the
// parameters restated here: rigid-body near-null space, theta = 0 symmetric
// strength, standard aggregation, one Jacobi smoothing step of the tentative
// prolongator with omega = 4/3 and the local (absolute row sum) weighting,
// Galerkin coarse operators R A P with R = P^T, max_coarse rows, at most 10
// levels).  The host does the graph work (sa_graph.cpp); every product with
// matrix values runs here, block-sparse with bs x bs node blocks (3 on the
// mesh level, 6 = the number of near-null-space vectors below it):
//
//   A_0   = sum_e K_e, assembled node row by node row through the gather plan,
//           prescribed DOFs replaced by identity rows/columns (bc_matrix,
//           gfem/linalg.py:213-217)
//   P     = T - omega D^-1 (A T),  D = absolute row sums of A
//   A P   then  A_c = P^T (A P)    (one warp per node / coarse node, fixed order)
//
// Every sum runs in a fixed order in one thread, so the hierarchy is bit-wise
// reproducible.  The levels are handed to the V-cycle as scalar CSR (FP64 + an
// FP32 copy); the mesh level keeps no stored matrix unless asked to (the
// solvers smooth it with the matrix-free product).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "sa.h"
#include "solver.h"

namespace exfem {

int host_standard_aggregation(int64_t n, const int64_t* ptr, const int32_t* idx, int32_t* agg, int64_t& nagg);

namespace {

__device__ __forceinline__ int find_sorted(const int32_t* a, int n, int32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int64_t warp_id() { return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int64_t warp_count() { return ((int64_t)gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ int64_t thread_id() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t thread_count() { return (int64_t)gridDim.x * blockDim.x; }

// A_0 node row n (3x3 blocks on the node adjacency row) = sum over the elements
// of the gather plan row n (increasing slot order) of their Ke blocks; a lane
// owns one (neighbour, entry) pair of an element at a time, and the warp
// synchronises between elements, so every entry is summed in plan order.  With
// `accumulate` the rows are added to (the next block of a model of several blocks,
// whose slots follow the previous blocks' in the model's plan) instead of set.
__global__ void sa_assemble0_kernel(int64_t nn, int nnode, int vmax, const int32_t* __restrict__ plan,
                                    int32_t sentinel, const int32_t* __restrict__ conn,
                                    const double* __restrict__ Ke, const uint8_t* __restrict__ nfix,
                                    const int64_t* __restrict__ aptr, const int32_t* __restrict__ aidx,
                                    double* __restrict__ A, int accumulate) {
  const int lane = threadIdx.x & 31;
  const int nd = 3 * nnode;
  for (int64_t n = warp_id(); n < nn; n += warp_count()) {
    const int64_t r0 = aptr[n];
    const int len = (int)(aptr[n + 1] - r0);
    const int32_t* row = aidx + r0;
    double* Ar = A + r0 * 9;
    if (!accumulate)
      for (int k = lane; k < len * 9; k += 32) Ar[k] = 0.0;
    __syncwarp();
    const uint32_t fn = nfix ? nfix[n] : 0u;
    for (int v = 0; v < vmax; ++v) {
      const int32_t slot = plan[n * vmax + v];
      if (slot == sentinel) break;
      const int64_t e = slot / nnode;
      const int a = slot - (int)e * nnode;
      const double* Kr = Ke + e * (int64_t)nd * nd + (int64_t)(3 * a) * nd;
      for (int k = lane; k < nnode * 9; k += 32) {
        const int bb = k / 9, ij = k - 9 * bb, i = ij / 3, j = ij - 3 * i;
        const int32_t m = conn[e * nnode + bb];
        const uint32_t fm = nfix ? nfix[m] : 0u;
        if (((fn >> i) & 1u) || ((fm >> j) & 1u)) continue;
        const int p = find_sorted(row, len, m);
        Ar[p * 9 + ij] += Kr[i * nd + 3 * bb + j];
      }
      __syncwarp();
    }
    if (lane < 3 && ((fn >> lane) & 1u)) {
      const int p = find_sorted(row, len, (int32_t)n);
      Ar[p * 9 + lane * 4] = 1.0;
    }
    __syncwarp();
  }
}

// per scalar row: diagonal entry and absolute row sum
__global__ void sa_rowinfo_kernel(int64_t nb, int bs, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                  const double* __restrict__ A, double* __restrict__ diag, double* __restrict__ dabs) {
  for (int64_t t = thread_id(); t < nb * bs; t += thread_count()) {
    const int64_t n = t / bs;
    const int r = (int)(t - n * bs);
    double s = 0.0, d = 0.0;
    for (int64_t q = ptr[n]; q < ptr[n + 1]; ++q) {
      const double* blk = A + q * bs * bs + r * bs;
      for (int c = 0; c < bs; ++c) s += fabs(blk[c]);
      if (idx[q] == n) d = blk[r];
    }
    diag[t] = d;
    dabs[t] = s;
  }
}

// nonzero flag per block, and the number of all-zero blocks
__global__ void sa_nzflag_kernel(int64_t nblk, int bb, const double* __restrict__ A, uint8_t* __restrict__ f,
                                 unsigned long long* __restrict__ nzero) {
  unsigned long long z = 0;
  for (int64_t q = thread_id(); q < nblk; q += thread_count()) {
    uint8_t nz = 0;
    for (int k = 0; k < bb; ++k) nz |= (A[q * bb + k] != 0.0);
    f[q] = nz;
    z += !nz;
  }
  if (z) atomicAdd(nzero, z);
}

__global__ void sa_gather_blocks_kernel(int64_t nkeep, int bb, const int64_t* __restrict__ keep,
                                        const double* __restrict__ Ain, double* __restrict__ Aout) {
  for (int64_t t = thread_id(); t < nkeep * bb; t += thread_count()) {
    const int64_t q = t / bb;
    Aout[t] = Ain[keep[q] * bb + (t - q * bb)];
  }
}

__global__ void sa_dinv_kernel(int64_t n, const double* __restrict__ diag, double* __restrict__ d64,
                               float* __restrict__ d32) {
  for (int64_t i = thread_id(); i < n; i += thread_count()) {
    const double d = diag[i];
    const double v = fabs(d) > 0.0 ? 1.0 / d : 0.0;
    d64[i] = v;
    d32[i] = (float)v;
  }
}

// P = T - omega D^-1 (A T): node row n holds one BS x K block per aggregate of its
// pattern; lane e owns entry e of each block, A T summed over the strength
// neighbours in increasing order
template <int BS, int K>
__global__ void sa_smooth_p_kernel(int64_t nb, const int64_t* __restrict__ sptr, const int32_t* __restrict__ sidx,
                                   const double* __restrict__ A, const int32_t* __restrict__ agg,
                                   const double* __restrict__ Q, const double* __restrict__ dabs, double omega,
                                   const int64_t* __restrict__ pptr, const int32_t* __restrict__ pidx,
                                   double* __restrict__ P) {
  constexpr int E = BS * K;
  const int lane = threadIdx.x & 31;
  for (int64_t n = warp_id(); n < nb; n += warp_count()) {
    const int64_t p0 = pptr[n];
    const int plen = (int)(pptr[n + 1] - p0);
    double* Pr = P + p0 * E;
    for (int k = lane; k < plen * E; k += 32) Pr[k] = 0.0;
    __syncwarp();
    for (int64_t q = sptr[n]; q < sptr[n + 1]; ++q) {
      const int32_t m = sidx[q];
      const int32_t g = agg[m];
      if (g < 0) continue;
      const int s = find_sorted(pidx + p0, plen, g);
      const double* Am = A + q * BS * BS;
      const double* Qm = Q + (int64_t)m * E;
      for (int e = lane; e < E; e += 32) {
        const int r = e / K, k = e - r * K;
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < BS; ++j) acc += Am[r * BS + j] * Qm[j * K + k];
        Pr[s * E + e] += acc;
      }
    }
    const int32_t gn = agg[n];
    const int sn = gn >= 0 ? find_sorted(pidx + p0, plen, gn) : -1;
    for (int s = 0; s < plen; ++s)
      for (int e = lane; e < E; e += 32) {
        const int r = e / K;
        const double d = dabs[n * BS + r];
        const double di = d != 0.0 ? 1.0 / d : 0.0;
        const double t = s == sn ? Q[n * E + e] : 0.0;
        Pr[s * E + e] = t - omega * (di * Pr[s * E + e]);
      }
    __syncwarp();
  }
}

// A P: node row n holds one BS x K block per aggregate of its pattern (the union
// of its neighbours' P patterns)
template <int BS, int K>
__global__ void sa_ap_kernel(int64_t nb, const int64_t* __restrict__ sptr, const int32_t* __restrict__ sidx,
                             const double* __restrict__ A, const int64_t* __restrict__ pptr,
                             const int32_t* __restrict__ pidx, const double* __restrict__ P,
                             const int64_t* __restrict__ qptr, const int32_t* __restrict__ qidx,
                             double* __restrict__ AP) {
  constexpr int E = BS * K;
  const int lane = threadIdx.x & 31;
  for (int64_t n = warp_id(); n < nb; n += warp_count()) {
    const int64_t q0 = qptr[n];
    const int qlen = (int)(qptr[n + 1] - q0);
    double* R = AP + q0 * E;
    for (int k = lane; k < qlen * E; k += 32) R[k] = 0.0;
    __syncwarp();
    for (int64_t q = sptr[n]; q < sptr[n + 1]; ++q) {
      const int32_t m = sidx[q];
      const double* Am = A + q * BS * BS;
      for (int64_t t = pptr[m]; t < pptr[m + 1]; ++t) {
        const int pos = find_sorted(qidx + q0, qlen, pidx[t]);
        const double* Pm = P + t * E;
        for (int e = lane; e < E; e += 32) {
          const int r = e / K, k = e - r * K;
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < BS; ++j) acc += Am[r * BS + j] * Pm[j * K + k];
          R[pos * E + e] += acc;
        }
      }
    }
    __syncwarp();
  }
}

// A_c = P^T (A P): coarse node row g sums, over the fine nodes n whose P row
// holds g (increasing n), P[n, g]^T AP[n, h] into its K x K block of h
template <int BS, int K>
__global__ void sa_rap_kernel(int64_t nagg, const int64_t* __restrict__ tptr, const int32_t* __restrict__ tidx,
                              const int32_t* __restrict__ tslot, const int64_t* __restrict__ pptr,
                              const double* __restrict__ P, const int64_t* __restrict__ qptr,
                              const int32_t* __restrict__ qidx, const double* __restrict__ AP,
                              const int64_t* __restrict__ cptr, const int32_t* __restrict__ cidx,
                              double* __restrict__ Ac) {
  constexpr int E = BS * K, EC = K * K;
  const int lane = threadIdx.x & 31;
  for (int64_t g = warp_id(); g < nagg; g += warp_count()) {
    const int64_t c0 = cptr[g];
    const int clen = (int)(cptr[g + 1] - c0);
    double* C = Ac + c0 * EC;
    for (int k = lane; k < clen * EC; k += 32) C[k] = 0.0;
    __syncwarp();
    for (int64_t u = tptr[g]; u < tptr[g + 1]; ++u) {
      const int32_t n = tidx[u];
      const double* Pn = P + (pptr[n] + tslot[u]) * E;
      for (int64_t t = qptr[n]; t < qptr[n + 1]; ++t) {
        const int pos = find_sorted(cidx + c0, clen, qidx[t]);
        const double* Qn = AP + t * E;
        for (int e = lane; e < EC; e += 32) {
          const int k = e / K, l = e - k * K;
          double acc = 0.0;
#pragma unroll
          for (int r = 0; r < BS; ++r) acc += Pn[r * K + k] * Qn[r * K + l];
          C[pos * EC + e] += acc;
        }
      }
    }
    __syncwarp();
  }
}

// block rows (R x C blocks) -> scalar CSR rows, columns ascending
__global__ void sa_expand_kernel(int64_t nbr, int R, int C, const int64_t* __restrict__ bptr,
                                 const int32_t* __restrict__ bidx, const double* __restrict__ blk,
                                 int64_t* __restrict__ ptr, int32_t* __restrict__ idx, double* __restrict__ v64,
                                 float* __restrict__ v32) {
  for (int64_t t = thread_id(); t < nbr * R; t += thread_count()) {
    const int64_t n = t / R;
    const int r = (int)(t - n * R);
    const int64_t q0 = bptr[n], len = bptr[n + 1] - q0;
    int64_t o = q0 * R * C + r * len * C;
    ptr[t] = o;
    if (t == nbr * R - 1) ptr[nbr * R] = bptr[nbr] * R * C;
    for (int64_t q = 0; q < len; ++q)
      for (int c = 0; c < C; ++c, ++o) {
        const double v = blk[(q0 + q) * R * C + r * C + c];
        idx[o] = bidx[q0 + q] * C + c;
        v64[o] = v;
        v32[o] = (float)v;
      }
  }
}

// R = P^T as scalar CSR: row g*K + k lists, for the fine nodes n holding g
// (increasing), the BS DOFs of n with P[n, g][r][k]
// FP32 copy of FP64 values
__global__ void sa_to_f32_kernel(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// blocks of R = P^T in block form: block q of aggregate row a (fine node tidx[q])
// is the transpose of P's block at position tslot[q] of that node's row
// (BS x K -> K x BS), FP64 and FP32
__global__ void sa_transpose_blocks_kernel(int64_t nq, int BS, int K, const int32_t* __restrict__ tidx,
                                           const int32_t* __restrict__ tslot, const int64_t* __restrict__ pptr,
                                           const double* __restrict__ P, double* __restrict__ r64,
                                           float* __restrict__ r32) {
  const int E = BS * K;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nq * E; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / E;
    const int e = (int)(t - q * E), i = e / BS, j = e - i * BS;   // entry (i, j) of the K x BS block
    const int64_t blk = pptr[tidx[q]] + tslot[q];
    const double v = P[blk * E + j * K + i];
    r64[t] = v;
    r32[t] = (float)v;
  }
}

__global__ void sa_expand_rt_kernel(int64_t nagg, int BS, int K, const int64_t* __restrict__ tptr,
                                    const int32_t* __restrict__ tidx, const int32_t* __restrict__ tslot,
                                    const int64_t* __restrict__ pptr, const double* __restrict__ P,
                                    int64_t* __restrict__ ptr, int32_t* __restrict__ idx, double* __restrict__ v64,
                                    float* __restrict__ v32) {
  for (int64_t t = thread_id(); t < nagg * K; t += thread_count()) {
    const int64_t g = t / K;
    const int k = (int)(t - g * K);
    const int64_t u0 = tptr[g], len = tptr[g + 1] - u0;
    int64_t o = u0 * BS * K + k * len * BS;
    ptr[t] = o;
    if (t == nagg * K - 1) ptr[nagg * K] = tptr[nagg] * BS * K;
    for (int64_t u = 0; u < len; ++u) {
      const int32_t n = tidx[u0 + u];
      const double* b = P + (pptr[n] + tslot[u0 + u]) * BS * K;
      for (int r = 0; r < BS; ++r, ++o) {
        const double v = b[r * K + k];
        idx[o] = n * BS + r;
        v64[o] = v;
        v32[o] = (float)v;
      }
    }
  }
}

// y = D^-1 A x on block rows
__global__ void sa_dinv_spmv_kernel(int64_t nb, int bs, const int64_t* __restrict__ ptr,
                                    const int32_t* __restrict__ idx, const double* __restrict__ A,
                                    const double* __restrict__ dinv, const double* __restrict__ x,
                                    double* __restrict__ y) {
  for (int64_t t = thread_id(); t < nb * bs; t += thread_count()) {
    const int64_t n = t / bs;
    const int r = (int)(t - n * bs);
    double s = 0.0;
    for (int64_t q = ptr[n]; q < ptr[n + 1]; ++q) {
      const double* blk = A + q * bs * bs + r * bs;
      const double* xm = x + (int64_t)idx[q] * bs;
      for (int c = 0; c < bs; ++c) s += blk[c] * xm[c];
    }
    y[t] = dinv[t] * s;
  }
}

constexpr int NPART = 512;

// per-block partial sums of squares (fixed grid, fixed order)
__global__ void sa_sumsq_kernel(int64_t n, const double* __restrict__ x, double* __restrict__ part) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)NPART * 256) s += x[i] * x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void sa_scale_kernel(int64_t n, double a, const double* __restrict__ y, double* __restrict__ x) {
  for (int64_t i = thread_id(); i < n; i += thread_count()) x[i] = a * y[i];
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// seeded standard normal start vector (splitmix64 counters, Box-Muller)
__global__ void sa_randn_kernel(int64_t n, uint64_t seed, double* __restrict__ x) {
  for (int64_t i = thread_id(); i < n; i += thread_count()) {
    const uint64_t h1 = splitmix64(seed ^ (2 * (uint64_t)i)), h2 = splitmix64(seed ^ (2 * (uint64_t)i + 1));
    const double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53, u2 = (double)(h2 >> 11) * 0x1.0p-53;
    x[i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

}  // namespace
namespace {

template <class T>
int up(DevBuf<T>& d, const std::vector<T>& h) {
  return d.upload(h.empty() ? nullptr : h.data(), h.size());
}

template <class T>
int down(std::vector<T>& h, const T* d, size_t n, cudaStream_t s) {
  h.resize(n);
  if (n) {
    EX_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    EX_CUDA(cudaStreamSynchronize(s));
  }
  return EXFEM_OK;
}

// phase timing of the set-up, printed to stderr when EXFEM_SETUP_TIMING is set
struct PhaseClock {
  bool on = std::getenv("EXFEM_SETUP_TIMING") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(const char* what, cudaStream_t s, int level) {
    if (!on) return;
    cudaStreamSynchronize(s);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[sa setup] level %d %-22s %8.1f ms\n", level, what,
                 std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

unsigned sa_grid(int64_t work, int block) { return grid_for((size_t)std::max<int64_t>(work, 1), block, 148u * 32u); }

// block-sparse operator of one level while it is being coarsened
struct BlockOp {
  int bs = 3;
  int64_t nb = 0;
  Rows pat;
  DevBuf<int64_t> ptr;
  DevBuf<int32_t> idx;
  DevBuf<double> val;
  int set_pattern(Rows&& r) {
    pat = std::move(r);
    int st;
    if ((st = up(ptr, pat.ptr))) return st;
    return up(idx, pat.idx);
  }
};

// 1.1 x the largest eigenvalue of D^-1 A estimated by 15 power iterations from a
// seeded normal vector (the reference's estimate, gfem/linalg.py:138-146)
int power_rho(const BlockOp& A, const double* dinv, cudaStream_t s, double& rho) {
  const int64_t n = A.nb * A.bs;
  DevBuf<double> x, y, part;
  int st;
  if ((st = x.alloc(n)) || (st = y.alloc(n)) || (st = part.alloc(NPART))) return st;
  sa_randn_kernel<<<sa_grid(n, 256), 256, 0, s>>>(n, 0x5eed5eedull, x.p);
  EX_LAUNCH_CHECK();
  std::vector<double> hp;
  auto norm = [&](const double* v, double& out) -> int {
    sa_sumsq_kernel<<<NPART, 256, 0, s>>>(n, v, part.p);
    EX_LAUNCH_CHECK();
    int q;
    if ((q = down(hp, part.p, NPART, s))) return q;
    double t = 0.0;
    for (double v2 : hp) t += v2;
    out = std::sqrt(t);
    return EXFEM_OK;
  };
  double lam = 1.0, nx = 0.0, ny = 0.0;
  if ((st = norm(x.p, nx))) return st;
  for (int it = 0; it < 15; ++it) {
    sa_dinv_spmv_kernel<<<sa_grid(n, 256), 256, 0, s>>>(A.nb, A.bs, A.ptr.p, A.idx.p, A.val.p, dinv, x.p, y.p);
    EX_LAUNCH_CHECK();
    if ((st = norm(y.p, ny))) return st;
    lam = ny / std::max(nx, 1e-300);
    sa_scale_kernel<<<sa_grid(n, 256), 256, 0, s>>>(n, 1.0 / std::max(ny, 1e-300), y.p, x.p);
    EX_LAUNCH_CHECK();
    nx = ny / std::max(ny, 1e-300);
  }
  EX_CUDA(cudaStreamSynchronize(s));  // x and y are freed on return
  rho = 1.1 * lam;
  return EXFEM_OK;
}

int expand_blocks(Csr64& M, int64_t nbr, int R, int C, int64_t ncols, const DevBuf<int64_t>& bptr,
                  const DevBuf<int32_t>& bidx, const double* blk, int64_t nblk, cudaStream_t s) {
  M.n = nbr * R;
  M.ncols = ncols;
  M.nnz = nblk * R * C;
  int st;
  if ((st = M.ptr.alloc(M.n + 1)) || (st = M.idx.alloc(M.nnz)) || (st = M.v64.alloc(M.nnz)) ||
      (st = M.v32.alloc(M.nnz)))
    return st;
  if (M.n == 0) {
    EX_CUDA(cudaMemsetAsync(M.ptr.p, 0, sizeof(int64_t), s));
    return EXFEM_OK;
  }
  sa_expand_kernel<<<sa_grid(M.n, 256), 256, 0, s>>>(nbr, R, C, bptr.p, bidx.p, blk, M.ptr.p, M.idx.p, M.v64.p,
                                                       M.v32.p);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template <int BS>
int coarsen(const BlockOp& A, const DevBuf<int32_t>& dagg, const DevBuf<double>& dQ, const DevBuf<double>& dabs,
            int64_t nagg, const Rows& Pp, const Rows& APp, const Rows& PT, const std::vector<int32_t>& slot,
            BlockOp& Ac, AmgLevel& L, cudaStream_t s) {
  constexpr int K = 6, E = BS * K;
  DevBuf<int64_t> pptr, qptr, tptr;
  DevBuf<int32_t> pidx, qidx, tidx, tslot;
  DevBuf<double> P, AP;
  int st;
  if ((st = up(pptr, Pp.ptr)) || (st = up(pidx, Pp.idx)) || (st = up(qptr, APp.ptr)) || (st = up(qidx, APp.idx)) ||
      (st = up(tptr, PT.ptr)) || (st = up(tidx, PT.idx)) || (st = up(tslot, slot)))
    return st;
  if ((st = P.alloc(std::max<size_t>(Pp.idx.size() * E, 1))) || (st = AP.alloc(std::max<size_t>(APp.idx.size() * E, 1))) ||
      (st = Ac.val.alloc(std::max<size_t>(Ac.pat.idx.size() * K * K, 1))))
    return st;
  const unsigned wg = sa_grid(A.nb * 32, 256);
  sa_smooth_p_kernel<BS, K><<<wg, 256, 0, s>>>(A.nb, A.ptr.p, A.idx.p, A.val.p, dagg.p, dQ.p, dabs.p, 4.0 / 3.0,
                                               pptr.p, pidx.p, P.p);
  EX_LAUNCH_CHECK();
  sa_ap_kernel<BS, K><<<wg, 256, 0, s>>>(A.nb, A.ptr.p, A.idx.p, A.val.p, pptr.p, pidx.p, P.p, qptr.p, qidx.p, AP.p);
  EX_LAUNCH_CHECK();
  sa_rap_kernel<BS, K><<<sa_grid(nagg * 32, 256), 256, 0, s>>>(nagg, tptr.p, tidx.p, tslot.p, pptr.p, P.p, qptr.p,
                                                                 qidx.p, AP.p, Ac.ptr.p, Ac.idx.p, Ac.val.p);
  EX_LAUNCH_CHECK();
  // P and R = P^T as scalar CSR for the V-cycle
  if ((st = expand_blocks(L.P, A.nb, BS, K, nagg * K, pptr, pidx, P.p, (int64_t)Pp.idx.size(), s))) return st;
  Csr64& R = L.R;
  R.n = nagg * K;
  R.ncols = A.nb * BS;
  R.nnz = (int64_t)Pp.idx.size() * E;
  if ((st = R.ptr.alloc(R.n + 1)) || (st = R.idx.alloc(R.nnz)) || (st = R.v64.alloc(R.nnz)) ||
      (st = R.v32.alloc(R.nnz)))
    return st;
  if (R.n) {
    sa_expand_rt_kernel<<<sa_grid(R.n, 256), 256, 0, s>>>(nagg, BS, K, tptr.p, tidx.p, tslot.p, pptr.p, P.p, R.ptr.p,
                                                           R.idx.p, R.v64.p, R.v32.p);
    EX_LAUNCH_CHECK();
  }
  // the same P and R in block form for the V-cycle (one index per block)
  {
    const int64_t nq = (int64_t)Pp.idx.size();
    Bsr& bp = L.bP;
    bp.R = BS, bp.C = K, bp.nb = A.nb, bp.nnzb = nq;
    if ((st = bp.v32.alloc(std::max<int64_t>(nq * E, 1))) || (st = L.bR.v64.alloc(std::max<int64_t>(nq * E, 1))) ||
        (st = L.bR.v32.alloc(std::max<int64_t>(nq * E, 1))))
      return st;
    if (nq) {
      sa_to_f32_kernel<<<sa_grid(nq * E, 256), 256, 0, s>>>(nq * E, P.p, bp.v32.p);
      EX_LAUNCH_CHECK();
      sa_transpose_blocks_kernel<<<sa_grid(nq * E, 256), 256, 0, s>>>(nq, BS, K, tidx.p, tslot.p, pptr.p, P.p,
                                                                        L.bR.v64.p, L.bR.v32.p);
      EX_LAUNCH_CHECK();
    }
    Bsr& br = L.bR;
    br.R = K, br.C = BS, br.nb = nagg, br.nnzb = nq;
    EX_CUDA(cudaStreamSynchronize(s));
    bp.ptr = std::move(pptr);
    bp.idx = std::move(pidx);
    bp.v64 = std::move(P);
    br.ptr = std::move(tptr);
    br.idx = std::move(tidx);
  }
  EX_CUDA(cudaStreamSynchronize(s));  // the temporaries are freed on return
  return EXFEM_OK;
}

}  // namespace

// node adjacency of several blocks over one node set: each element's node list
// padded to the widest element with its own first node (repeats are ignored)
static int blocks_adjacency(const std::vector<exfem_block_s*>& blks, cudaStream_t s, Rows& adj) {
  const int64_t nn = blks[0]->nn;
  int wmax = 0;
  int64_t ne = 0;
  for (auto* b : blks) {
    EX_ARG(b->nn == nn, "blocks of one operator must share their node set (%lld vs %lld nodes)",
           (long long)b->nn, (long long)nn);
    wmax = std::max(wmax, b->nnode);
    ne += b->ne;
  }
  std::vector<int32_t> conn((size_t)ne * wmax), cb;
  int64_t e0 = 0;
  int st;
  for (auto* b : blks) {
    if ((st = down(cb, b->conn.p, (size_t)b->ne * b->nnode, s))) return st;
    for (int64_t e = 0; e < b->ne; ++e)
      for (int a = 0; a < wmax; ++a)
        conn[(size_t)(e0 + e) * wmax + a] = cb[(size_t)e * b->nnode + (a < b->nnode ? a : 0)];
    e0 += b->ne;
  }
  return host_node_adjacency(nn, ne, wmax, conn.data(), adj);
}

static void assemble_blocks(const std::vector<exfem_block_s*>& blks, const std::vector<const double*>& Kes,
                            int64_t nn, const int64_t* aptr, const int32_t* aidx, double* A, cudaStream_t s) {
  const uint8_t* nfix = blks[0]->node_fixed.n ? blks[0]->node_fixed.p : nullptr;
  for (size_t i = 0; i < blks.size(); ++i) {
    exfem_block_s* b = blks[i];
    sa_assemble0_kernel<<<sa_grid(nn * 32, 256), 256, 0, s>>>(nn, b->nnode, b->vmax, b->plan.p,
                                                               (int32_t)(b->ne * b->nnode), b->conn.p, Kes[i], nfix,
                                                               aptr, aidx, A, i > 0 ? 1 : 0);
  }
}

int blocks_csr_assemble(const std::vector<exfem_block_s*>& blks, const std::vector<const double*>& Kes, BlockCsr& c,
                        cudaStream_t s) {
  EX_ARG(!blks.empty() && blks.size() == Kes.size(), "need one element-matrix array per block");
  for (size_t i = 0; i < blks.size(); ++i) EX_ARG(Kes[i] || blks[i]->ne == 0, "element matrices are NULL");
  const int64_t nn = blks[0]->nn, n = 3 * nn;
  int st;
  if (!c.ready) {
    Rows adj;
    if ((st = blocks_adjacency(blks, s, adj))) return st;
    c.nnzb = (int64_t)adj.idx.size();
    if ((st = up(c.bptr, adj.ptr)) || (st = up(c.bidx, adj.idx)) ||
        (st = c.bval.alloc(std::max<int64_t>(c.nnzb * 9, 1))))
      return st;
    c.A.n = c.A.ncols = n;
    c.A.nnz = c.nnzb * 9;
    if ((st = c.A.ptr.alloc(n + 1)) || (st = c.A.idx.alloc(std::max<int64_t>(c.A.nnz, 1))) ||
        (st = c.A.v64.alloc(std::max<int64_t>(c.A.nnz, 1))) || (st = c.A.v32.alloc(std::max<int64_t>(c.A.nnz, 1))))
      return st;
    c.ready = true;
  }
  if (nn == 0) return EXFEM_OK;
  assemble_blocks(blks, Kes, nn, c.bptr.p, c.bidx.p, c.bval.p, s);
  EX_LAUNCH_CHECK();
  sa_expand_kernel<<<sa_grid(n, 256), 256, 0, s>>>(nn, 3, 3, c.bptr.p, c.bidx.p, c.bval.p, c.A.ptr.p, c.A.idx.p,
                                                     c.A.v64.p, c.A.v32.p);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

int block_csr_assemble(exfem_block_s* b, const double* Ke, BlockCsr& c, cudaStream_t s) {
  EX_ARG(Ke || b->ne == 0, "element matrices are NULL");
  const int64_t nn = b->nn, n = 3 * nn;
  int st;
  if (!c.ready) {
    std::vector<int32_t> conn;
    if ((st = down(conn, b->conn.p, (size_t)b->ne * b->nnode, s))) return st;
    Rows adj;
    if ((st = host_node_adjacency(nn, b->ne, b->nnode, conn.data(), adj))) return st;
    c.nnzb = (int64_t)adj.idx.size();
    if ((st = up(c.bptr, adj.ptr)) || (st = up(c.bidx, adj.idx)) ||
        (st = c.bval.alloc(std::max<int64_t>(c.nnzb * 9, 1))))
      return st;
    c.A.n = c.A.ncols = n;
    c.A.nnz = c.nnzb * 9;
    if ((st = c.A.ptr.alloc(n + 1)) || (st = c.A.idx.alloc(std::max<int64_t>(c.A.nnz, 1))) ||
        (st = c.A.v64.alloc(std::max<int64_t>(c.A.nnz, 1))) || (st = c.A.v32.alloc(std::max<int64_t>(c.A.nnz, 1))))
      return st;
    c.ready = true;
  }
  if (nn == 0) return EXFEM_OK;
  sa_assemble0_kernel<<<sa_grid(nn * 32, 256), 256, 0, s>>>(
      nn, b->nnode, b->vmax, b->plan.p, (int32_t)(b->ne * b->nnode), b->conn.p, Ke,
      b->node_fixed.n ? b->node_fixed.p : nullptr, c.bptr.p, c.bidx.p, c.bval.p, 0);
  EX_LAUNCH_CHECK();
  sa_expand_kernel<<<sa_grid(n, 256), 256, 0, s>>>(nn, 3, 3, c.bptr.p, c.bidx.p, c.bval.p, c.A.ptr.p, c.A.idx.p,
                                                     c.A.v64.p, c.A.v32.p);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

int amg_setup_block(exfem_amg_s* h, exfem_block_s* b, const double* Ke, int max_coarse, int keep_level0,
                    cudaStream_t s) {
  return amg_setup_blocks(h, std::vector<exfem_block_s*>{b}, std::vector<const double*>{Ke}, max_coarse,
                          keep_level0, s);
}

int amg_setup_blocks(exfem_amg_s* h, const std::vector<exfem_block_s*>& blks, const std::vector<const double*>& Kes,
                     int max_coarse, int keep_level0, cudaStream_t s) {
  EX_ARG(h->levels.empty() && h->nc == 0, "AMG handle already holds a hierarchy");
  EX_ARG(!blks.empty() && blks.size() == Kes.size(), "need one element-matrix array per block");
  int64_t ne = 0;
  for (size_t i = 0; i < blks.size(); ++i) {
    EX_ARG(blks[i]->ne == 0 || Kes[i], "block %zu needs its element matrices", i);
    ne += blks[i]->ne;
  }
  EX_ARG(ne > 0, "the blocks need elements");
  EX_ARG(max_coarse >= 6, "max_coarse must be at least 6");
  exfem_block_s* b = blks[0];
  std::vector<double> X;
  int st;
  PhaseClock clk;
  if ((st = down(X, b->X.p, (size_t)b->nn * 3, s))) return st;
  // level 0: node adjacency pattern, A_0 assembled from the element matrices
  BlockOp A;
  A.bs = 3;
  A.nb = b->nn;
  {
    Rows adj;
    if (blks.size() == 1) {
      std::vector<int32_t> conn;
      if ((st = down(conn, b->conn.p, (size_t)b->ne * b->nnode, s))) return st;
      if ((st = host_node_adjacency(b->nn, b->ne, b->nnode, conn.data(), adj))) return st;
    } else if ((st = blocks_adjacency(blks, s, adj))) {
      return st;
    }
    clk.mark("node adjacency (host)", s, 0);
    if ((st = A.set_pattern(std::move(adj)))) return st;
  }
  if ((st = A.val.alloc(std::max<size_t>(A.pat.idx.size() * 9, 1)))) return st;
  assemble_blocks(blks, Kes, A.nb, A.ptr.p, A.idx.p, A.val.p, s);
  EX_LAUNCH_CHECK();
  clk.mark("assembly", s, 0);
  std::vector<double> B;
  host_rigid_body_modes(b->nn, X.data(), B);
  std::vector<double>().swap(X);
  constexpr int K = 6;
  const int max_levels = 10;
  while (A.nb * A.bs > max_coarse && (int)h->levels.size() < max_levels - 1) {
    const int bs = A.bs;
    const int64_t n = A.nb * bs, nblk = (int64_t)A.pat.idx.size();
    DevBuf<double> diag, dabs;
    DevBuf<uint8_t> flag;
    DevBuf<unsigned long long> nzero;
    if ((st = diag.alloc(n)) || (st = dabs.alloc(n)) || (st = flag.alloc(std::max<int64_t>(nblk, 1))) ||
        (st = nzero.alloc(1)))
      return st;
    EX_CUDA(cudaMemsetAsync(nzero.p, 0, sizeof(unsigned long long), s));
    sa_rowinfo_kernel<<<sa_grid(n, 256), 256, 0, s>>>(A.nb, bs, A.ptr.p, A.idx.p, A.val.p, diag.p, dabs.p);
    EX_LAUNCH_CHECK();
    sa_nzflag_kernel<<<sa_grid(nblk, 256), 256, 0, s>>>(nblk, bs * bs, A.val.p, flag.p, nzero.p);
    EX_LAUNCH_CHECK();
    std::vector<unsigned long long> hz;
    if ((st = down(hz, nzero.p, 1, s))) return st;
    // strength graph (theta = 0): the nonzero blocks; A keeps only those (the
    // pattern as it is when no block is all zero)
    if (hz[0] > 0) {
      std::vector<uint8_t> f;
      if ((st = down(f, flag.p, (size_t)nblk, s))) return st;
      Rows S;
      std::vector<int64_t> keep;
      host_filter_pattern(A.pat, f.data(), S, keep);
      if ((int64_t)keep.size() < nblk) {
        DevBuf<int64_t> dkeep;
        DevBuf<double> v;
        if ((st = up(dkeep, keep)) || (st = v.alloc(std::max<size_t>(keep.size() * bs * bs, 1)))) return st;
        const int64_t nk = (int64_t)keep.size();
        sa_gather_blocks_kernel<<<sa_grid(nk * bs * bs, 256), 256, 0, s>>>(nk, bs * bs, dkeep.p, A.val.p, v.p);
        EX_LAUNCH_CHECK();
        EX_CUDA(cudaStreamSynchronize(s));
        A.val = std::move(v);
        if ((st = A.set_pattern(std::move(S)))) return st;
      }
    }
    const int lev = (int)h->levels.size();
    clk.mark("strength graph", s, lev);
    std::vector<int32_t> agg(A.nb);
    int64_t nagg = 0;
    if ((st = host_standard_aggregation(A.nb, A.pat.ptr.data(), A.pat.idx.data(), agg.data(), nagg))) return st;
    if (nagg == 0) break;
    std::vector<double> Q, Bc;
    clk.mark("aggregation (host)", s, lev);
    host_fit_candidates(A.nb, bs, K, agg.data(), nagg, B.data(), Q, Bc);
    clk.mark("tentative P (host)", s, lev);
    Rows Pp, APp, PT, Acp;
    std::vector<int32_t> slot;
    host_p_pattern(A.pat, agg.data(), nagg, Pp);
    host_union_pattern(A.pat, Pp, nagg, APp);
    host_transpose_pattern(Pp, nagg, PT, slot);
    host_union_pattern(PT, APp, nagg, Acp);
    clk.mark("patterns (host)", s, lev);
    auto L = std::make_unique<AmgLevel>();
    L->n = n;
    L->nc = nagg * K;
    L->op_nnz = (int64_t)A.pat.idx.size() * bs * bs;
    BlockOp Ac;
    Ac.bs = K;
    Ac.nb = nagg;
    if ((st = Ac.set_pattern(std::move(Acp)))) return st;
    DevBuf<int32_t> dagg;
    DevBuf<double> dQ;
    if ((st = up(dagg, agg)) || (st = up(dQ, Q))) return st;
    st = bs == 3 ? coarsen<3>(A, dagg, dQ, dabs, nagg, Pp, APp, PT, slot, Ac, *L, s)
                 : coarsen<6>(A, dagg, dQ, dabs, nagg, Pp, APp, PT, slot, Ac, *L, s);
    if (st) return st;
    clk.mark("P, AP, RAP, P/R CSR", s, lev);
    // smoother data of this level: inverse diagonal, spectral bound, stored matrix
    if ((st = L->dinv64.alloc(n)) || (st = L->dinv32.alloc(n))) return st;
    sa_dinv_kernel<<<sa_grid(n, 256), 256, 0, s>>>(n, diag.p, L->dinv64.p, L->dinv32.p);
    EX_LAUNCH_CHECK();
    if ((st = power_rho(A, L->dinv64.p, s, L->rho))) return st;
    clk.mark("spectral bound", s, lev);
    if (!h->levels.empty() || keep_level0) {
      if ((st = expand_blocks(L->A, A.nb, bs, bs, n, A.ptr, A.idx, A.val.p, (int64_t)A.pat.idx.size(), s))) return st;
      // and in block form (A is replaced by the coarse operator below, so its
      // device arrays move into the level)
      Bsr& ba = L->bA;
      ba.R = ba.C = bs;
      ba.nb = A.nb;
      ba.nnzb = (int64_t)A.pat.idx.size();
      if ((st = ba.v32.alloc(std::max<int64_t>(ba.nnzb * bs * bs, 1)))) return st;
      if (ba.nnzb) {
        sa_to_f32_kernel<<<sa_grid(ba.nnzb * bs * bs, 256), 256, 0, s>>>(ba.nnzb * bs * bs, A.val.p, ba.v32.p);
        EX_LAUNCH_CHECK();
      }
      EX_CUDA(cudaStreamSynchronize(s));
      ba.ptr = std::move(A.ptr);
      ba.idx = std::move(A.idx);
      ba.v64 = std::move(A.val);
    } else {
      L->A.n = n;
      L->A.ncols = n;
      L->A.nnz = 0;
    }
    EX_CUDA(cudaStreamSynchronize(s));
    h->levels.push_back(std::move(L));
    const bool stop = nagg * K >= n;  // no reduction: the next operator is the coarsest
    A = std::move(Ac);
    B = std::move(Bc);
    if (stop) break;
  }
  // coarsest level: dense inverse through a regularised Cholesky factor
  const int64_t nc = A.nb * A.bs;
  EX_ARG(nc <= 5000, "coarsest level of %lld rows is too large for a dense solve", (long long)nc);
  std::vector<double> v;
  if ((st = down(v, A.val.p, A.pat.idx.size() * A.bs * A.bs, s))) return st;
  std::vector<double> D((size_t)nc * nc, 0.0), Ainv;
  for (int64_t r = 0; r < A.nb; ++r)
    for (int64_t q = A.pat.ptr[r]; q < A.pat.ptr[r + 1]; ++q)
      for (int i = 0; i < A.bs; ++i)
        for (int j = 0; j < A.bs; ++j)
          D[(r * A.bs + i) * nc + (int64_t)A.pat.idx[q] * A.bs + j] = v[(q * A.bs + i) * A.bs + j];
  if ((st = host_coarse_inverse(nc, D, Ainv))) return st;
  clk.mark("coarsest inverse", s, (int)h->levels.size());
  if ((st = h->Ainv.upload(Ainv.data(), Ainv.size()))) return st;
  h->nc = nc;
  h->coarse_nnz = nc * nc;
  return EXFEM_OK;
}

}  // namespace exfem
