// Device V-cycle of a smoothed-aggregation hierarchy (gfem/linalg.py:156-195).
//
// Per level: Chebyshev smoothing of D^-1 A over [rho/30, rho] with degree 2
// (3 operator products per call, the first one on a zero guess is skipped since
// A*0 = 0), residual, restriction R = P^T, recursion, prolongation, and
// post-smoothing.  The coarsest level is solved in FP64 with the inverse of the
// regularised dense Cholesky factor formed on the host (two triangular solves in
// the reference, gfem/linalg.py:179-181; the product is the same up to rounding).
//
// CSR products run with a group of 4-32 lanes per row (chosen from the mean row
// length) and a fixed shuffle tree, so results are deterministic.  The Chebyshev
// step is fused into the row loop: x += d, r -= dinv*(A d), d' = a d + b r.
// Level 0 can instead be smoothed with the current matrix-free tangent
// (gfem/solvers.py:311-314), in which case the products go through the
// element kernel and the vector updates through small elementwise kernels.
#include <array>
#include <mutex>

#include "internal.h"
#include "solver.h"

namespace exfem {

// SP_CHEBLAST: the last Chebyshev step of a smoothing, which also adds the new
// direction to x (x = (x + d) + d2) and stores neither r nor d2; SP_SETDIFF (block
// products): y = M (b - x), the restriction of a residual whose product A x is in x.
enum SpmvMode { SP_SET = 0, SP_ADD = 1, SP_RES = 2, SP_RESINIT = 3, SP_CHEB = 4, SP_CHEBLAST = 5, SP_SETDIFF = 6 };

template <class T, int LANES, int MODE>
__global__ void __launch_bounds__(256)
spmv_kernel(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
            const T* __restrict__ val, const T* __restrict__ x, T* __restrict__ y,
            const T* __restrict__ b, const T* __restrict__ dinv, T* __restrict__ d2,
            T* __restrict__ xo, T c1, T c2, const T* __restrict__ rc1, const T* __restrict__ rc2,
            const int64_t* __restrict__ rmap, const int64_t* __restrict__ cshift, const int* __restrict__ skip) {
  static_assert(MODE <= SP_CHEB, "the scalar product has the first five modes only");
  if (skip && *skip) return;
  constexpr int GPW = 32 / LANES;  // row groups per warp
  const int lane = threadIdx.x & (LANES - 1);
  const int grp = (threadIdx.x & 31) / LANES;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp * GPW; base < n; base += nwarps * GPW) {
    const int64_t row = base + grp;
    T s = T(0);
    if (row < n) {
      const int64_t sr = rmap ? rmap[row] : row;
      const int64_t cs = rmap ? cshift[row] : 0;
      const int64_t k1 = ptr[sr + 1];
      for (int64_t k = ptr[sr] + lane; k < k1; k += LANES) s += val[k] * x[idx[k] + cs];
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LANES);
    if (row < n && lane == 0) {
      if (MODE == SP_SET) {
        y[row] = s;
      } else if (MODE == SP_ADD) {
        y[row] += s;
      } else if (MODE == SP_RES) {
        y[row] = b[row] - s;
      } else if (MODE == SP_RESINIT) {
        const T r = dinv[row] * (b[row] - s);
        y[row] = r;
        d2[row] = r * (rc1 ? rc1[5 * row] : c1);
      } else {  // SP_CHEB: x is the direction d
        const T d = x[row];
        xo[row] += d;
        const T r = y[row] - dinv[row] * s;
        y[row] = r;
        d2[row] = (rc1 ? rc1[5 * row] : c1) * d + (rc2 ? rc2[5 * row] : c2) * r;
      }
    }
  }
}

template <class T, int MODE>
static int spmv_lanes(const Csr64& A, const T* val, const T* x, T* y, const T* b, const T* dinv, T* d2,
                      T* xo, T c1, T c2, const int* skip, cudaStream_t s, const T* rc1 = nullptr,
                      const T* rc2 = nullptr) {
  if (A.n == 0) return EXFEM_OK;
  const int64_t nsrc = A.ptr.n ? (int64_t)A.ptr.n - 1 : A.n;  // stored rows (fewer when blocks are replicated)
  const double avg = nsrc ? (double)A.nnz / (double)nsrc : 0.0;
  const int threads = 256;
  // one group of L lanes per row: 32 / L rows per warp
#define EXF_SP(L) spmv_kernel<T, L, MODE><<<grid_for((size_t)((A.n + 32 / L - 1) / (32 / L)) * 32, threads, 148u * 24u), threads, 0, s>>>(A.n, A.ptr.p, A.idx.p, val, x, y, b, dinv, d2, xo, c1, c2, rc1, rc2, A.rmap.p, A.cshift.p, skip)
  if (avg <= 8) EXF_SP(4);
  else if (avg <= 24) EXF_SP(8);
  else if (avg <= 64) EXF_SP(16);
  else EXF_SP(32);
#undef EXF_SP
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

// N values of T from p into registers with the widest loads that p's alignment A
// (bytes, a multiple of 4) allows: 16-byte, 8-byte or single loads.
template <class T, int N, int A>
__device__ __forceinline__ void load_regs(const T* __restrict__ p, T (&o)[N]) {
  constexpr int BYTES = N * (int)sizeof(T);
  if constexpr (A % 16 == 0 && BYTES % 16 == 0) {
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(p) + i);
      memcpy(reinterpret_cast<char*>(o) + 16 * i, &v, 16);
    }
  } else if constexpr (A % 8 == 0 && BYTES % 8 == 0) {
#pragma unroll
    for (int i = 0; i < BYTES / 8; ++i) {
      const float2 v = __ldg(reinterpret_cast<const float2*>(p) + i);
      memcpy(reinterpret_cast<char*>(o) + 8 * i, &v, 8);
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = __ldg(p + i);
  }
}

// alignment in bytes of element k * n of a 256-byte aligned array of T
template <class T, int N>
constexpr int stride_align() {
  return (N * (int)sizeof(T)) % 16 == 0 ? 16 : (N * (int)sizeof(T)) % 8 == 0 ? 8 : 4;
}

// Block-sparse product with the same fused modes as spmv_kernel: L lanes per block
// row stride over its blocks (consecutive blocks are contiguous in memory, so a
// group's loads coalesce), each lane keeps the R row sums of its blocks, and the
// group reduces them in a fixed order; lane 0 finishes the R rows.
template <class T, int R, int C, int L, int MODE>
__global__ void __launch_bounds__(256)
bsr_kernel(int64_t nb, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val,
           const T* __restrict__ x, T* __restrict__ y, const T* __restrict__ b, const T* __restrict__ dinv,
           T* __restrict__ d2, T* __restrict__ xo, T c1, T c2, const int* __restrict__ skip) {
  if (skip && *skip) return;
  constexpr int GPW = 32 / L;
  const int lane = threadIdx.x & (L - 1);
  const int grp = (threadIdx.x & 31) / L;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp * GPW; base < nb; base += nwarps * GPW) {
    const int64_t br = base + grp;
    T acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = T(0);
    if (br < nb) {
      const int64_t k1 = ptr[br + 1];
      for (int64_t k = ptr[br] + lane; k < k1; k += L) {
        T v[R * C], xv[C];
        load_regs<T, R * C, stride_align<T, R * C>()>(val + k * (R * C), v);
        load_regs<T, C, stride_align<T, C>()>(x + (int64_t)idx[k] * C, xv);
        if constexpr (MODE == SP_SETDIFF) {
          T bv[C];
          load_regs<T, C, stride_align<T, C>()>(b + (int64_t)idx[k] * C, bv);
#pragma unroll
          for (int j = 0; j < C; ++j) xv[j] = bv[j] - xv[j];
        }
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
          for (int j = 0; j < C; ++j) acc[i] += v[i * C + j] * xv[j];
      }
    }
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int o = L / 2; o > 0; o >>= 1) acc[i] += __shfl_down_sync(0xffffffffu, acc[i], o, L);
    if (br < nb && lane == 0) {
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int64_t row = br * R + i;
        const T sv = acc[i];
        if (MODE == SP_SET) {
          y[row] = sv;
        } else if (MODE == SP_ADD) {
          y[row] += sv;
        } else if (MODE == SP_RES) {
          y[row] = b[row] - sv;
        } else if (MODE == SP_RESINIT) {
          const T r = dinv[row] * (b[row] - sv);
          y[row] = r;
          d2[row] = r * c1;
        } else if (MODE == SP_CHEB) {  // x is the direction d
          const T d = x[row];
          xo[row] += d;
          const T r = y[row] - dinv[row] * sv;
          y[row] = r;
          d2[row] = c1 * d + c2 * r;
        } else if (MODE == SP_CHEBLAST) {
          const T d = x[row];
          const T r = y[row] - dinv[row] * sv;
          const T dn = c1 * d + c2 * r;
          xo[row] = (xo[row] + d) + dn;
        } else {  // SP_SETDIFF
          y[row] = sv;
        }
      }
    }
  }
}

template <class T, int R, int C, int MODE>
static int bsr_launch(const Bsr& M, const T* val, const T* x, T* y, const T* b, const T* dinv, T* d2, T* xo, T c1,
                       T c2, const int* skip, cudaStream_t s) {
  // the vector loads of the kernel assume the alignment of a 256-byte aligned array
  if ((uintptr_t)x % stride_align<T, C>() || (uintptr_t)val % stride_align<T, R * C>() ||
      (MODE == SP_SETDIFF && (uintptr_t)b % stride_align<T, C>())) {
    set_error("block-sparse product: misaligned operand (x %p, blocks %p)", (const void*)x, (const void*)val);
    return EXFEM_ERR_ARG;
  }
  const double avg = M.nb ? (double)M.nnzb / (double)M.nb : 0.0;
  const int threads = 256;
  // one group of L lanes per block row: 32 / L block rows per warp
#define EXF_BSR(L) bsr_kernel<T, R, C, L, MODE><<<grid_for((size_t)((M.nb + 32 / L - 1) / (32 / L)) * 32, threads, 148u * 24u), threads, 0, s>>>(M.nb, M.ptr.p, M.idx.p, val, x, y, b, dinv, d2, xo, c1, c2, skip)
  if (avg <= 2) EXF_BSR(1);
  else if (avg <= 6) EXF_BSR(4);
  else if (avg <= 16) EXF_BSR(8);
  else if (avg <= 40) EXF_BSR(16);
  else EXF_BSR(32);
#undef EXF_BSR
  return EXFEM_OK;
}

template <class T, int MODE>
static int bsr_apply(const Bsr& M, const T* x, T* y, const T* b, const T* dinv, T* d2, T* xo, T c1, T c2,
                     const int* skip, cudaStream_t s) {
  const T* val;
  if constexpr (sizeof(T) == 8) val = M.v64.p;
  else val = M.v32.p;
  int st;
  if (M.R == 3 && M.C == 6) st = bsr_launch<T, 3, 6, MODE>(M, val, x, y, b, dinv, d2, xo, c1, c2, skip, s);
  else if (M.R == 6 && M.C == 3) st = bsr_launch<T, 6, 3, MODE>(M, val, x, y, b, dinv, d2, xo, c1, c2, skip, s);
  else if (M.R == 6 && M.C == 6) st = bsr_launch<T, 6, 6, MODE>(M, val, x, y, b, dinv, d2, xo, c1, c2, skip, s);
  else if (M.R == 3 && M.C == 3) st = bsr_launch<T, 3, 3, MODE>(M, val, x, y, b, dinv, d2, xo, c1, c2, skip, s);
  else {
    set_error("no block-sparse product for %d x %d blocks", M.R, M.C);
    return EXFEM_ERR_UNSUPPORTED;
  }
  if (st) return st;
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template <class T>
static const T* csr_vals(const Csr64& A);
template <> const double* csr_vals<double>(const Csr64& A) { return A.v64.p; }
template <> const float* csr_vals<float>(const Csr64& A) { return A.v32.p; }

// ---------------------------------------------------------------- elementwise kernels
template <class T>
__global__ void cheb_init0_kernel(int64_t n, const T* __restrict__ b, const T* __restrict__ dinv,
                                  T* __restrict__ x, T* __restrict__ r, T* __restrict__ d, T ith,
                                  const int* __restrict__ skip, const T* __restrict__ rith = nullptr) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = dinv[i] * b[i];
    x[i] = T(0);
    r[i] = ri;
    d[i] = ri * (rith ? rith[5 * i] : ith);
  }
}

template <class T>
__global__ void cheb_update_kernel(int64_t n, T* __restrict__ x, const T* __restrict__ d, T* __restrict__ r,
                                   const T* __restrict__ Ad, const T* __restrict__ dinv, T* __restrict__ d2,
                                   T c1, T c2, const int* __restrict__ skip, const T* __restrict__ rc1 = nullptr,
                                   const T* __restrict__ rc2 = nullptr, int last = 0) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T di = d[i];
    const T ri = r[i] - dinv[i] * Ad[i];
    const T dn = (rc1 ? rc1[5 * i] : c1) * di + (rc2 ? rc2[5 * i] : c2) * ri;
    if (last) {  // the smoothing's last step: x = (x + d) + d2, r and d2 not kept
      x[i] = (x[i] + di) + dn;
    } else {
      x[i] += di;
      r[i] = ri;
      d2[i] = dn;
    }
  }
}

template <class T>
__global__ void resinit_kernel(int64_t n, const T* __restrict__ b, const T* __restrict__ Ax,
                               const T* __restrict__ dinv, T* __restrict__ r, T* __restrict__ d, T ith,
                               const int* __restrict__ skip, const T* __restrict__ rith = nullptr) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = dinv[i] * (b[i] - Ax[i]);
    r[i] = ri;
    d[i] = ri * (rith ? rith[5 * i] : ith);
  }
}

template <class T>
__global__ void sub_kernel(int64_t n, const T* __restrict__ b, T* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = b[i] - y[i];
}

template <class T>
__global__ void add_kernel(int64_t n, const T* __restrict__ d, T* __restrict__ x, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += d[i];
}

// x = Ainv * b, FP64 arithmetic, one warp per row
template <class T>
__global__ void coarse_kernel(int64_t nc, const double* __restrict__ Ainv, const T* __restrict__ b,
                              T* __restrict__ x, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= nc) return;
  double s = 0.0;
  for (int64_t j = lane; j < nc; j += 32) s += Ainv[row * nc + j] * (double)b[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[row] = (T)s;
}

// block-diagonal coarse solve: row r lies in block [s, s+m) whose inverse starts at a
template <class T>
__global__ void coarse_blocks_kernel(int64_t nc, const double* __restrict__ Ainv, const int64_t* __restrict__ rs,
                                     const int64_t* __restrict__ rm, const int64_t* __restrict__ ra,
                                     const T* __restrict__ b, T* __restrict__ x, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= nc) return;
  const int64_t s0 = rs[row], m = rm[row], a = ra[row] + (row - s0) * m;
  double s = 0.0;
  for (int64_t j = lane; j < m; j += 32) s += Ainv[a + j] * (double)b[s0 + j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[row] = (T)s;
}

// ---------------------------------------------------------------- V-cycle driver
template <class T>
static T* lvbuf(AmgLevel& L, int k);
template <> double* lvbuf<double>(AmgLevel& L, int k) { return L.w64[k].p; }
template <> float* lvbuf<float>(AmgLevel& L, int k) { return L.w32[k].p; }
template <class T>
static const T* lvcoef(AmgLevel& L);
template <> const double* lvcoef<double>(AmgLevel& L) { return L.coef64.p; }
template <> const float* lvcoef<float>(AmgLevel& L) { return L.coef32.p; }
template <class T>
static const T* lvdinv(AmgLevel& L);
template <> const double* lvdinv<double>(AmgLevel& L) { return L.dinv64.p; }
template <> const float* lvdinv<float>(AmgLevel& L) { return L.dinv32.p; }

int amg_prepare(exfem_amg_s* h, int dtype) {
  int st;
  for (auto& Lp : h->levels) {
    AmgLevel& L = *Lp;
    const int64_t nb = std::max<int64_t>(L.n, 1);
    for (int k = 0; k < AmgLevel::NW; ++k) {
      if (dtype == EXFEM_F64 && L.w64[k].n < (size_t)nb && (st = L.w64[k].alloc(nb))) return st;
      if (dtype == EXFEM_F32 && L.w32[k].n < (size_t)nb && (st = L.w32[k].alloc(nb))) return st;
    }
  }
  const int64_t nb = std::max<int64_t>(h->nc, 1);
  if (dtype == EXFEM_F64) {
    if (h->cb64.n < (size_t)nb && (st = h->cb64.alloc(nb))) return st;
    if (h->cx64.n < (size_t)nb && (st = h->cx64.alloc(nb))) return st;
  } else {
    if (h->cb32.n < (size_t)nb && (st = h->cb32.alloc(nb))) return st;
    if (h->cx32.n < (size_t)nb && (st = h->cx32.alloc(nb))) return st;
  }
  return EXFEM_OK;
}

template <class T>
static int coarse_solve(exfem_amg_s* h, const T* b, T* x, const int* skip, cudaStream_t s) {
  if (h->nc == 0) return EXFEM_OK;
  const int threads = 128;
  if (h->crow_s.p) {
    coarse_blocks_kernel<T><<<(unsigned)((h->nc * 32 + threads - 1) / threads), threads, 0, s>>>(
        h->nc, h->Ainv.p, h->crow_s.p, h->crow_m.p, h->crow_a.p, b, x, skip);
    EX_LAUNCH_CHECK();
    return EXFEM_OK;
  }
  coarse_kernel<T><<<(unsigned)((h->nc * 32 + threads - 1) / threads), threads, 0, s>>>(h->nc, h->Ainv.p, b, x, skip);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template <class T>
static int vcycle_level(exfem_amg_s* h, size_t l, const T* b, T* x, const Level0Op<T>* op0,
                        const int* skip, cudaStream_t s) {
  if (l == h->levels.size()) return coarse_solve<T>(h, b, x, skip, s);
  AmgLevel& L = *h->levels[l];
  const bool mf = (l == 0 && op0 && op0->apply);
  if (!mf && L.A.nnz == 0) {
    set_error("AMG level %zu holds no stored matrix: smooth it with a level-0 block", l);
    return EXFEM_ERR_ARG;
  }
  const T* dinv = (l == 0 && op0 && op0->dinv) ? op0->dinv : lvdinv<T>(L);
  const T* rc = lvcoef<T>(L);  // per-row Chebyshev coefficients (union of independent hierarchies)
  // block-sparse forms where the device set-up kept them (never with per-row
  // coefficients or replicated levels, whose scalar rows are remapped)
  const bool blocks_ok = !rc && !h->replicated;
  const bool useA = blocks_ok && L.bA.on();
  const bool useT = blocks_ok && L.bP.on() && L.bR.on();
  const int64_t n = L.n;
  T* r = lvbuf<T>(L, AmgLevel::WR);
  T* d = lvbuf<T>(L, AmgLevel::WD);
  T* d2 = lvbuf<T>(L, AmgLevel::WD2);
  T* t = lvbuf<T>(L, AmgLevel::WTMP);
  const double lmax = L.rho, lmin = L.rho / 30.0;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  double ca[8], cb[8];
  {
    double rh = 1.0 / sigma;
    for (int j = 0; j < h->degree; ++j) {
      const double rn = 1.0 / (2.0 * sigma - rh);
      ca[j] = rn * rh;
      cb[j] = 2.0 * rn / delta;
      rh = rn;
    }
  }
  const T ith = (T)(1.0 / theta);
  const unsigned eg = grid_for(n, 256);
  const T* vals = csr_vals<T>(L.A);
  int st;
  // the last step of the matrix-free and block-sparse smoothings adds the final
  // direction itself (x = (x + d) + d2); the scalar-CSR smoothing adds it after
  auto smooth_steps = [&]() -> int {
    const bool fused_last = mf || useA;
    for (int j = 0; j < h->degree; ++j) {
      const bool last = fused_last && j == h->degree - 1;
      if (mf) {
        if ((st = op0->apply(op0->ctx, d, t, skip, s))) return st;
        cheb_update_kernel<T><<<eg, 256, 0, s>>>(n, x, d, r, t, dinv, d2, (T)ca[j], (T)cb[j], skip,
                                                 rc ? rc + 2 * j : nullptr, rc ? rc + 2 * j + 1 : nullptr,
                                                 last ? 1 : 0);
        EX_LAUNCH_CHECK();
      } else {
        if (useA) {
          if (last) {
            if ((st = bsr_apply<T, SP_CHEBLAST>(L.bA, d, r, nullptr, dinv, d2, x, (T)ca[j], (T)cb[j], skip, s)))
              return st;
          } else if ((st = bsr_apply<T, SP_CHEB>(L.bA, d, r, nullptr, dinv, d2, x, (T)ca[j], (T)cb[j], skip, s))) {
            return st;
          }
        } else if ((st = spmv_lanes<T, SP_CHEB>(L.A, vals, d, r, nullptr, dinv, d2, x, (T)ca[j], (T)cb[j], skip, s,
                                                rc ? rc + 2 * j : nullptr, rc ? rc + 2 * j + 1 : nullptr))) {
          return st;
        }
      }
      std::swap(d, d2);
    }
    if (!(fused_last && h->degree > 0)) {
      add_kernel<T><<<eg, 256, 0, s>>>(n, d, x, skip);
      EX_LAUNCH_CHECK();
    }
    return EXFEM_OK;
  };
  // pre-smoothing from x = 0
  cheb_init0_kernel<T><<<eg, 256, 0, s>>>(n, b, dinv, x, r, d, ith, skip, rc ? rc + 4 : nullptr);
  EX_LAUNCH_CHECK();
  if ((st = smooth_steps())) return st;
  // residual and restriction
  if (mf) {
    if ((st = op0->apply(op0->ctx, x, t, skip, s))) return st;
    if (!useT) {  // the block-sparse restriction below forms b - t itself
      sub_kernel<T><<<eg, 256, 0, s>>>(n, b, t, skip);
      EX_LAUNCH_CHECK();
    }
  } else {
    if (useA) {
      if ((st = bsr_apply<T, SP_RES>(L.bA, x, t, b, nullptr, nullptr, nullptr, T(0), T(0), skip, s))) return st;
    } else if ((st = spmv_lanes<T, SP_RES>(L.A, vals, x, t, b, nullptr, nullptr, nullptr, T(0), T(0), skip, s))) {
      return st;
    }
  }
  T* bc;
  T* xc;
  if (l + 1 < h->levels.size()) {
    AmgLevel& C = *h->levels[l + 1];
    bc = lvbuf<T>(C, AmgLevel::WB);
    xc = lvbuf<T>(C, AmgLevel::WX);
  } else {
    if constexpr (sizeof(T) == 8) { bc = (T*)h->cb64.p; xc = (T*)h->cx64.p; }
    else { bc = (T*)h->cb32.p; xc = (T*)h->cx32.p; }
  }
  if (useT) {
    if (mf) {
      if ((st = bsr_apply<T, SP_SETDIFF>(L.bR, t, bc, b, nullptr, nullptr, nullptr, T(0), T(0), skip, s))) return st;
    } else if ((st = bsr_apply<T, SP_SET>(L.bR, t, bc, nullptr, nullptr, nullptr, nullptr, T(0), T(0), skip, s))) {
      return st;
    }
  } else if ((st = spmv_lanes<T, SP_SET>(L.R, csr_vals<T>(L.R), t, bc, nullptr, nullptr, nullptr, nullptr, T(0), T(0),
                                         skip, s))) {
    return st;
  }
  if ((st = vcycle_level<T>(h, l + 1, bc, xc, nullptr, skip, s))) return st;
  if (useT) {
    if ((st = bsr_apply<T, SP_ADD>(L.bP, xc, x, nullptr, nullptr, nullptr, nullptr, T(0), T(0), skip, s))) return st;
  } else if ((st = spmv_lanes<T, SP_ADD>(L.P, csr_vals<T>(L.P), xc, x, nullptr, nullptr, nullptr, nullptr, T(0), T(0),
                                         skip, s))) {
    return st;
  }
  // post-smoothing from the corrected x
  if (mf) {
    if ((st = op0->apply(op0->ctx, x, t, skip, s))) return st;
    resinit_kernel<T><<<eg, 256, 0, s>>>(n, b, t, dinv, r, d, ith, skip, rc ? rc + 4 : nullptr);
    EX_LAUNCH_CHECK();
  } else {
    if (useA) {
      if ((st = bsr_apply<T, SP_RESINIT>(L.bA, x, r, b, dinv, d, nullptr, ith, T(0), skip, s))) return st;
    } else if ((st = spmv_lanes<T, SP_RESINIT>(L.A, vals, x, r, b, dinv, d, nullptr, ith, T(0), skip, s,
                                               rc ? rc + 4 : nullptr))) {
      return st;
    }
  }
  return smooth_steps();
}

template <class T>
int amg_vcycle(exfem_amg_s* h, const T* b, T* x, const Level0Op<T>* op0, const int* skip, cudaStream_t s) {
  if (h->levels.empty()) {
    if (h->nc == 0) { set_error("empty AMG hierarchy"); return EXFEM_ERR_ARG; }
    return coarse_solve<T>(h, b, x, skip, s);
  }
  int st;
  if ((st = amg_prepare(h, sizeof(T) == 8 ? EXFEM_F64 : EXFEM_F32))) return st;
  return vcycle_level<T>(h, 0, b, x, op0, skip, s);
}

template int amg_vcycle<double>(exfem_amg_s*, const double*, double*, const Level0Op<double>*, const int*, cudaStream_t);
template int amg_vcycle<float>(exfem_amg_s*, const float*, float*, const Level0Op<float>*, const int*, cudaStream_t);

// y = A x with a stored FP64 CSR matrix (the assembled-operator solvers)
int csr_apply(const Csr64& A, const double* x, double* y, const int* skip, cudaStream_t s) {
  return spmv_lanes<double, SP_SET>(A, A.v64.p, x, y, nullptr, nullptr, nullptr, nullptr, 0.0, 0.0, skip, s);
}

// ---------------------------------------------------------------- upload
static int upload_csr(Csr64& M, int64_t n, int64_t ncols, const int64_t* ptr, const int32_t* idx, const double* val) {
  M.n = n;
  M.ncols = ncols;
  M.nnz = ptr[n];
  int st;
  if ((st = M.ptr.upload(ptr, n + 1))) return st;
  if ((st = M.idx.upload(idx, M.nnz))) return st;
  if ((st = M.v64.upload(val, M.nnz))) return st;
  std::vector<float> v32(val, val + M.nnz);
  for (int64_t k = 0; k < M.nnz; ++k) v32[k] = (float)val[k];
  return M.v32.upload(v32.data(), M.nnz);
}

// per-row Chebyshev coefficients (degree 2) from per-row spectral bounds (0 marks a
// pass-through row whose smoother is switched off): for each
// row [ca0, cb0, ca1, cb1, 1/theta] of the reference's recurrence (linalg.py:161-175)
int amg_set_level_rows(exfem_amg_s* h, size_t l, const double* rho_rows) {
  EX_ARG(l < h->levels.size(), "level %zu out of range", l);
  EX_ARG(h->degree == 2, "per-row Chebyshev coefficients cover degree 2");
  AmgLevel& L = *h->levels[l];
  std::vector<double> c((size_t)L.n * 5);
  std::vector<float> c32((size_t)L.n * 5);
  for (int64_t i = 0; i < L.n; ++i) {
    const double rho = rho_rows[i];
    EX_ARG(rho >= 0 && std::isfinite(rho), "invalid spectral bound %g at row %lld", rho, (long long)i);
    if (rho == 0.0) {  // pass-through row: no smoothing, the level only relays to the next
      for (int k = 0; k < 5; ++k) c[5 * i + k] = 0.0;
      continue;
    }
    const double lmax = rho, lmin = rho / 30.0;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
    double rh = 1.0 / sigma;
    for (int j = 0; j < 2; ++j) {
      const double rn = 1.0 / (2.0 * sigma - rh);
      c[5 * i + 2 * j] = rn * rh;
      c[5 * i + 2 * j + 1] = 2.0 * rn / delta;
      rh = rn;
    }
    c[5 * i + 4] = 1.0 / theta;
  }
  for (size_t k = 0; k < c.size(); ++k) c32[k] = (float)c[k];
  int st;
  if ((st = L.coef64.upload(c.data(), c.size()))) return st;
  return L.coef32.upload(c32.data(), c32.size());
}

int amg_add_level(exfem_amg_s* h, int64_t n, int64_t nc, const int64_t* Ap, const int32_t* Ai, const double* Av,
                  const int64_t* Pp, const int32_t* Pi, const double* Pv, const int64_t* Rp, const int32_t* Ri,
                  const double* Rv, const double* dinv, double rho) {
  auto L = std::make_unique<AmgLevel>();
  L->n = n;
  L->nc = nc;
  L->rho = rho;
  int st;
  if ((st = upload_csr(L->A, n, n, Ap, Ai, Av))) return st;
  if ((st = upload_csr(L->P, n, nc, Pp, Pi, Pv))) return st;
  if ((st = upload_csr(L->R, nc, n, Rp, Ri, Rv))) return st;
  if ((st = L->dinv64.upload(dinv, n))) return st;
  std::vector<float> d32(dinv, dinv + n);
  if ((st = L->dinv32.upload(d32.data(), n))) return st;
  h->levels.push_back(std::move(L));
  return EXFEM_OK;
}

// Replicate a hierarchy of nmesh independent blocks into ninst copies (instance i
// copies block inst_mesh[i]).  Matrices keep one stored copy per block; the copies
// address it through per-row maps.  Vectors (inverse diagonals, per-row Chebyshev
// coefficients) and the block-diagonal coarse solve are expanded.
template <class T>
static int download(std::vector<T>& h, const DevBuf<T>& d) {
  h.resize(d.n);
  if (d.n) EX_CUDA(cudaMemcpy(h.data(), d.p, d.bytes(), cudaMemcpyDeviceToHost));
  return EXFEM_OK;
}

template <class T>
static int expand_rows(DevBuf<T>& d, const std::vector<int64_t>& rmap, int per_row) {
  if (!d.p) return EXFEM_OK;
  std::vector<T> h, out(rmap.size() * per_row);
  int st;
  if ((st = download(h, d))) return st;
  for (size_t r = 0; r < rmap.size(); ++r)
    for (int k = 0; k < per_row; ++k) out[r * per_row + k] = h[(size_t)rmap[r] * per_row + k];
  return d.upload(out.data(), out.size());
}

int amg_replicate(exfem_amg_s* h, int nmesh, const int64_t* level_offsets, int ninst, const int32_t* inst_mesh) {
  const size_t nl = h->levels.size();
  const int64_t* off = level_offsets;  // (nl + 1) rows of nmesh + 1 offsets
  EX_ARG(h->nc > 0, "set the coarse solve before replicating");
  for (size_t l = 0; l <= nl; ++l) {
    const int64_t* o = off + l * (nmesh + 1);
    const int64_t want = l < nl ? h->levels[l]->n : h->nc;
    EX_ARG(o[0] == 0 && o[nmesh] == want, "level %zu offsets do not cover its %lld rows", l, (long long)want);
    for (int m = 0; m < nmesh; ++m) EX_ARG(o[m + 1] > o[m], "block %d is empty at level %zu", m, l);
  }
  for (int i = 0; i < ninst; ++i) EX_ARG(inst_mesh[i] >= 0 && inst_mesh[i] < nmesh, "instance %d: bad block", i);
  if (h->crow_s.p) {  // an existing block-diagonal coarse solve must use the same blocks
    std::vector<int64_t> rs;
    int st;
    if ((st = download(rs, h->crow_s))) return st;
    const int64_t* o = off + nl * (nmesh + 1);
    for (int m = 0; m < nmesh; ++m)
      EX_ARG(rs[o[m]] == o[m] && rs[o[m + 1] - 1] == o[m], "coarse blocks differ from the level offsets");
  } else {
    EX_ARG(nmesh == 1, "a dense coarse solve replicates a single block only");
  }
  // per level: stored row of each union row and the instance of each union row
  std::vector<std::vector<int64_t>> rmap(nl + 1), shift(nl + 1), ishift(nl + 1);
  for (size_t l = 0; l <= nl; ++l) {
    const int64_t* o = off + l * (nmesh + 1);
    int64_t u = 0;
    ishift[l].resize(ninst);
    for (int i = 0; i < ninst; ++i) {
      const int m = inst_mesh[i];
      ishift[l][i] = u - o[m];
      for (int64_t k = o[m]; k < o[m + 1]; ++k, ++u) {
        rmap[l].push_back(k);
        shift[l].push_back(u - k);  // constant over the instance's rows
      }
    }
  }
  auto inst_of_rows = [&](size_t l) {  // instance index per union row
    std::vector<int> w;
    w.reserve(rmap[l].size());
    const int64_t* o = off + l * (nmesh + 1);
    for (int i = 0; i < ninst; ++i)
      for (int64_t k = o[inst_mesh[i]]; k < o[inst_mesh[i] + 1]; ++k) w.push_back(i);
    return w;
  };
  int st;
  for (size_t l = 0; l < nl; ++l) {
    AmgLevel& L = *h->levels[l];
    const std::vector<int> wi = inst_of_rows(l), wc = inst_of_rows(l + 1);
    std::vector<int64_t> cs_p(wi.size()), cs_r(wc.size());
    for (size_t r = 0; r < wi.size(); ++r) cs_p[r] = ishift[l + 1][wi[r]];
    for (size_t r = 0; r < wc.size(); ++r) cs_r[r] = ishift[l][wc[r]];
    const int64_t n = (int64_t)rmap[l].size(), nc = (int64_t)rmap[l + 1].size();
    if ((st = L.A.rmap.upload(rmap[l].data(), n)) || (st = L.A.cshift.upload(shift[l].data(), n))) return st;
    if ((st = L.P.rmap.upload(rmap[l].data(), n)) || (st = L.P.cshift.upload(cs_p.data(), n))) return st;
    if ((st = L.R.rmap.upload(rmap[l + 1].data(), nc)) || (st = L.R.cshift.upload(cs_r.data(), nc))) return st;
    if ((st = expand_rows(L.dinv64, rmap[l], 1)) || (st = expand_rows(L.dinv32, rmap[l], 1))) return st;
    if ((st = expand_rows(L.coef64, rmap[l], 5)) || (st = expand_rows(L.coef32, rmap[l], 5))) return st;
    L.n = L.A.n = L.A.ncols = L.P.n = L.R.ncols = n;
    L.nc = L.P.ncols = L.R.n = nc;
  }
  // block-diagonal coarse solve over the instances
  const std::vector<int64_t>& rc = rmap[nl];
  const int64_t nu = (int64_t)rc.size();
  std::vector<int64_t> s0(nu), sm(nu), sa(nu), us(nu), um(nu), ua(nu);
  if (h->crow_s.p) {
    if ((st = download(s0, h->crow_s)) || (st = download(sm, h->crow_m)) || (st = download(sa, h->crow_a))) return st;
  } else {
    s0.assign(h->nc, 0);
    sm.assign(h->nc, h->nc);
    sa.assign(h->nc, 0);
  }
  for (int64_t r = 0; r < nu; ++r) {
    const int64_t k = rc[r];
    us[r] = s0[k] + shift[nl][r];
    um[r] = sm[k];
    ua[r] = sa[k];
  }
  if ((st = h->crow_s.upload(us.data(), nu)) || (st = h->crow_m.upload(um.data(), nu)) ||
      (st = h->crow_a.upload(ua.data(), nu)))
    return st;
  h->nc = nu;
  h->replicated = true;
  return EXFEM_OK;
}

}  // namespace exfem

// ================================================================= allocation-free V-cycle
// exfem_amg_vcycle_noalloc: the same V-cycle as exfem_amg_vcycle, for callers
// that must not allocate device memory during the call — code recording a CUDA
// graph by stream capture (cudaMalloc is not permitted while a capture is open)
// and hosts whose device memory is owned by another allocator.  The per-level
// work vectors (6 per level plus 2 coarse vectors) are carved from one
// file-scope device array of EXFEM_VCYCLE_NOALLOC_BYTES (8 MiB), which every GPU
// that loads the library holds until the process exits.  Hierarchies whose work
// vectors do not fit are rejected with EXFEM_ERR_ARG.  All calls share the
// array: calls whose work overlaps on the GPU (other streams, other host
// threads) race with each other and must be serialised by the caller.  Nothing
// in the array needs to start at zero: each call writes every work entry before
// reading it, so contents left by the previous call are never read.
namespace exfem {

static __device__ __align__(256) unsigned char g_vcycle_scratch[EXFEM_VCYCLE_NOALLOC_BYTES];

// device address of the scratch array, with the device current (the host-side
// name of the array is not a device address).  Outside a stream capture the
// address is looked up on every call, so a context that was destroyed and made
// again (cudaDeviceReset) gets its new address; inside a capture the address
// remembered from the last call on that device outside a capture is used, because
// the look-up may load the module, which a capture does not permit.
static std::mutex g_scratch_mu;
static void* g_scratch_dev[64] = {nullptr};

static int vcycle_scratch_address(cudaStream_t s, void** out) {
  int dev = 0;
  EX_CUDA(cudaGetDevice(&dev));
  EX_ARG(dev >= 0 && dev < 64, "device ordinal %d out of range", dev);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  EX_CUDA(cudaStreamIsCapturing(s, &cap));
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    EX_CUDA(cudaGetSymbolAddress(&p, g_vcycle_scratch));
    g_scratch_dev[dev] = p;
  }
  EX_ARG(g_scratch_dev[dev] != nullptr,
         "allocation-free V-cycle: first call on device %d is inside a stream capture; call it once before capturing",
         dev);
  *out = g_scratch_dev[dev];
  return EXFEM_OK;
}

template <class T>
struct NoallocWork {
  std::vector<std::array<T*, AmgLevel::NW>> lv;
  T* cb = nullptr;
  T* cx = nullptr;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

template <class T>
static int noalloc_carve(exfem_amg_s* h, unsigned char* base, NoallocWork<T>& w) {
  size_t off = 0;
  w.lv.resize(h->levels.size());
  for (size_t l = 0; l < h->levels.size(); ++l)
    for (int k = 0; k < AmgLevel::NW; ++k) {
      w.lv[l][k] = reinterpret_cast<T*>(base + off);
      off += align256(sizeof(T) * (size_t)std::max<int64_t>(h->levels[l]->n, 1));
    }
  w.cb = reinterpret_cast<T*>(base + off);
  off += align256(sizeof(T) * (size_t)std::max<int64_t>(h->nc, 1));
  w.cx = reinterpret_cast<T*>(base + off);
  off += align256(sizeof(T) * (size_t)std::max<int64_t>(h->nc, 1));
  if (off > (size_t)EXFEM_VCYCLE_NOALLOC_BYTES) {
    set_error("allocation-free V-cycle: the hierarchy needs %zu bytes of work vectors, the static scratch holds %zu",
              off, (size_t)EXFEM_VCYCLE_NOALLOC_BYTES);
    return EXFEM_ERR_ARG;
  }
  return EXFEM_OK;
}

template <class T>
static int vcycle_level_noalloc(exfem_amg_s* h, size_t l, const T* b, T* x, const Level0Op<T>* op0,
                                NoallocWork<T>& w, cudaStream_t s) {
  if (l == h->levels.size()) return coarse_solve<T>(h, b, x, nullptr, s);
  AmgLevel& L = *h->levels[l];
  const bool mf = (l == 0 && op0 && op0->apply);
  if (!mf && L.A.nnz == 0) {
    set_error("AMG level %zu holds no stored matrix: smooth it with a level-0 block", l);
    return EXFEM_ERR_ARG;
  }
  const T* dinv = (l == 0 && op0 && op0->dinv) ? op0->dinv : lvdinv<T>(L);
  const T* rc = lvcoef<T>(L);  // per-row Chebyshev coefficients (union of independent hierarchies)
  const int64_t n = L.n;
  T* r = w.lv[l][AmgLevel::WR];
  T* d = w.lv[l][AmgLevel::WD];
  T* d2 = w.lv[l][AmgLevel::WD2];
  T* t = w.lv[l][AmgLevel::WTMP];
  const double lmax = L.rho, lmin = L.rho / 30.0;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  double ca[8], cb[8];
  {
    double rh = 1.0 / sigma;
    for (int j = 0; j < h->degree; ++j) {
      const double rn = 1.0 / (2.0 * sigma - rh);
      ca[j] = rn * rh;
      cb[j] = 2.0 * rn / delta;
      rh = rn;
    }
  }
  const T ith = (T)(1.0 / theta);
  const unsigned eg = grid_for(n, 256);
  const T* vals = csr_vals<T>(L.A);
  int st;
  auto smooth_steps = [&]() -> int {
    for (int j = 0; j < h->degree; ++j) {
      if (mf) {
        if ((st = op0->apply(op0->ctx, d, t, nullptr, s))) return st;
        cheb_update_kernel<T><<<eg, 256, 0, s>>>(n, x, d, r, t, dinv, d2, (T)ca[j], (T)cb[j], nullptr,
                                                 rc ? rc + 2 * j : nullptr, rc ? rc + 2 * j + 1 : nullptr);
        EX_LAUNCH_CHECK();
      } else {
        if ((st = spmv_lanes<T, SP_CHEB>(L.A, vals, d, r, nullptr, dinv, d2, x, (T)ca[j], (T)cb[j], nullptr, s,
                                         rc ? rc + 2 * j : nullptr, rc ? rc + 2 * j + 1 : nullptr)))
          return st;
      }
      std::swap(d, d2);
    }
    add_kernel<T><<<eg, 256, 0, s>>>(n, d, x, nullptr);
    EX_LAUNCH_CHECK();
    return EXFEM_OK;
  };
  cheb_init0_kernel<T><<<eg, 256, 0, s>>>(n, b, dinv, x, r, d, ith, nullptr, rc ? rc + 4 : nullptr);
  EX_LAUNCH_CHECK();
  if ((st = smooth_steps())) return st;
  if (mf) {
    if ((st = op0->apply(op0->ctx, x, t, nullptr, s))) return st;
    sub_kernel<T><<<eg, 256, 0, s>>>(n, b, t, nullptr);
    EX_LAUNCH_CHECK();
  } else {
    if ((st = spmv_lanes<T, SP_RES>(L.A, vals, x, t, b, nullptr, nullptr, nullptr, T(0), T(0), nullptr, s))) return st;
  }
  T* bc = (l + 1 < h->levels.size()) ? w.lv[l + 1][AmgLevel::WB] : w.cb;
  T* xc = (l + 1 < h->levels.size()) ? w.lv[l + 1][AmgLevel::WX] : w.cx;
  if ((st = spmv_lanes<T, SP_SET>(L.R, csr_vals<T>(L.R), t, bc, nullptr, nullptr, nullptr, nullptr, T(0), T(0), nullptr, s)))
    return st;
  if ((st = vcycle_level_noalloc<T>(h, l + 1, bc, xc, nullptr, w, s))) return st;
  if ((st = spmv_lanes<T, SP_ADD>(L.P, csr_vals<T>(L.P), xc, x, nullptr, nullptr, nullptr, nullptr, T(0), T(0), nullptr, s)))
    return st;
  if (mf) {
    if ((st = op0->apply(op0->ctx, x, t, nullptr, s))) return st;
    resinit_kernel<T><<<eg, 256, 0, s>>>(n, b, t, dinv, r, d, ith, nullptr, rc ? rc + 4 : nullptr);
    EX_LAUNCH_CHECK();
  } else {
    if ((st = spmv_lanes<T, SP_RESINIT>(L.A, vals, x, r, b, dinv, d, nullptr, ith, T(0), nullptr, s,
                                        rc ? rc + 4 : nullptr)))
      return st;
  }
  return smooth_steps();
}

template <class T>
static int mf_apply_noalloc(void* ctx, const T* x, T* y, const int* skip, cudaStream_t s) {
  return launch_mf_matvec<T>((exfem_block_s*)ctx, x, y, skip, s);
}

template <class T>
static int vcycle_noalloc(exfem_amg_s* h, const T* r, T* z, exfem_block_s* level0, const T* dinv0, cudaStream_t s) {
  EX_ARG(!h->levels.empty() || h->nc > 0, "empty AMG hierarchy");
  // every level smoothed with a stored matrix must hold one; checked before any
  // launch (a hierarchy set up without its mesh-level matrix needs a level-0 block)
  for (size_t l = 0; l < h->levels.size(); ++l)
    if (!(l == 0 && level0) && h->levels[l]->A.nnz == 0) {
      set_error("AMG level %zu holds no stored matrix: smooth it with a level-0 block", l);
      return EXFEM_ERR_ARG;
    }
  void* base = nullptr;
  int st;
  if ((st = vcycle_scratch_address(s, &base))) return st;
  NoallocWork<T> w;
  if ((st = noalloc_carve<T>(h, static_cast<unsigned char*>(base), w))) return st;
  if (h->levels.empty()) return coarse_solve<T>(h, r, z, nullptr, s);
  Level0Op<T> op;
  if (level0) {
    op.apply = &mf_apply_noalloc<T>;
    op.ctx = level0;
    op.dinv = dinv0;
  }
  return vcycle_level_noalloc<T>(h, 0, r, z, level0 ? &op : nullptr, w, s);
}

}  // namespace exfem

extern "C" int exfem_amg_vcycle_noalloc(exfem_amg h, int dtype, const void* r, void* z, exfem_block level0,
                                        const void* dinv0, void* stream) {
  using namespace exfem;
  EX_ARG(h && r && z, "NULL argument");
  EX_ARG(!level0 || dinv0, "a level-0 block needs dinv0");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == EXFEM_F64)
    return vcycle_noalloc<double>(h, (const double*)r, (double*)z, level0, (const double*)dinv0, s);
  if (dtype == EXFEM_F32)
    return vcycle_noalloc<float>(h, (const float*)r, (float*)z, level0, (const float*)dinv0, s);
  set_error("V-cycle supports F64 and F32, got %d", dtype);
  return EXFEM_ERR_ARG;
}
