// PCG and mixed-precision iterative refinement on the device.
//
// PCG follows gfem/linalg.py:21-47 exactly: x0 = 0, r = b, z = M(r), p = z,
// loop while r.r > tol^2 max(b.b, 1e-300) and k < maxiter: Ap = A p,
// alpha = rz / p.Ap, x += alpha p, r -= alpha Ap, rr = r.r, z = M(r),
// beta = r.z / rz, p = z + beta p.  All dot products accumulate in FP64 with a
// fixed two-level reduction order (deterministic), and all step scalars live in
// device memory as FP64, so the host never sits in the loop: iterations are
// issued in chunks (captured once as a CUDA graph), every kernel first reads the
// device "done" flag, and the host reads the flag once per chunk.
//
// Mixed refinement follows gfem/solvers.py:344-384 (_LinearSystem._mixed): an
// FP32 inner PCG on the normalised residual, the correction accumulated in FP64,
// and the FP64 residual b - A x recomputed with the FP64 operator each pass.
#include <algorithm>
#include <cmath>
#include <vector>

#include "solver.h"

namespace exfem {

constexpr int RT = 256;          // reduction block size
constexpr int RED_MAX_BLOCKS = 592;   // 4 CTAs of 256 per SM

enum Fin { FIN_BB = 0, FIN_RZ0, FIN_RR0, FIN_ALPHA, FIN_RR, FIN_BETA, FIN_STORE };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void fin_apply(int F, double s, PcgScal* sc, double* out) {
  switch (F) {
    case FIN_BB:
      sc->bb = s;
      sc->tol2 = sc->spare * fmax(s, 1e-300);
      break;
    case FIN_RZ0: sc->rz = s; break;
    case FIN_RR0:
      sc->rr = s;
      sc->done = !(s > sc->tol2 && sc->k < sc->maxiter);
      break;
    case FIN_ALPHA:
      sc->pAp = s;
      sc->alpha = sc->rz / s;
      break;
    case FIN_RR: sc->rr = s; break;
    case FIN_BETA:
      sc->beta = s / sc->rz;
      sc->rz = s;
      sc->k += 1;
      sc->done = !(sc->rr > sc->tol2 && sc->k < sc->maxiter);
      break;
    default: *out = s;
  }
}

// block partial sums + last-block final sum in index order
__device__ __forceinline__ void block_finish(double v, double* partial, unsigned* counter, int F,
                                             PcgScal* sc, double* out) {
  __shared__ double sw[RT / 32];
  __shared__ int last;
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < RT / 32; ++w) t += sw[w];
    partial[blockIdx.x] = t;
    __threadfence();
    const unsigned tk = atomicAdd(counter, 1u);
    last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    double t = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += 32) t += ((volatile double*)partial)[i];
    t = warp_sum(t);
    if (threadIdx.x == 0) {
      fin_apply(F, t, sc, out);
      *counter = 0u;
    }
  }
}

template <class T>
__global__ void __launch_bounds__(RT)
dot_kernel(int64_t n, const T* __restrict__ a, const T* __restrict__ b, double* partial, unsigned* counter,
           PcgScal* sc, double* out, int F, int check_done) {
  if (check_done && sc->done) return;
  // four independent strided loads in flight per thread, four accumulators summed
  // in a fixed order at the end (deterministic for a given grid)
  const int64_t S = (int64_t)gridDim.x * RT;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int64_t i = blockIdx.x * (int64_t)RT + threadIdx.x;
  for (; i + 3 * S < n; i += 4 * S) {
    const T x0 = a[i], x1 = a[i + S], x2 = a[i + 2 * S], x3 = a[i + 3 * S];
    const T y0 = b[i], y1 = b[i + S], y2 = b[i + 2 * S], y3 = b[i + 3 * S];
    a0 += (double)x0 * (double)y0;
    a1 += (double)x1 * (double)y1;
    a2 += (double)x2 * (double)y2;
    a3 += (double)x3 * (double)y3;
  }
  for (; i < n; i += S) a0 += (double)a[i] * (double)b[i];
  block_finish((a0 + a1) + (a2 + a3), partial, counter, F, sc, out);
}

template <class T>
__global__ void __launch_bounds__(RT)
update_xr_kernel(int64_t n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                 const T* __restrict__ Ap, double* partial, unsigned* counter, PcgScal* sc) {
  if (sc->done) return;
  const T alpha = (T)sc->alpha;
  const int64_t S = (int64_t)gridDim.x * RT;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int64_t i = blockIdx.x * (int64_t)RT + threadIdx.x;
  for (; i + 3 * S < n; i += 4 * S) {
    T xv[4], pv[4], rv[4], av[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      xv[u] = x[i + u * S];
      pv[u] = p[i + u * S];
      rv[u] = r[i + u * S];
      av[u] = Ap[i + u * S];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x[i + u * S] = xv[u] + alpha * pv[u];
      const T ri = rv[u] - alpha * av[u];
      r[i + u * S] = ri;
      acc[u] += (double)ri * (double)ri;
    }
  }
  for (; i < n; i += S) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
  }
  block_finish((acc[0] + acc[1]) + (acc[2] + acc[3]), partial, counter, FIN_RR, sc, nullptr);
}

template <class T>
__global__ void update_p_kernel(int64_t n, T* __restrict__ p, const T* __restrict__ z, const PcgScal* sc) {
  if (sc->done) return;
  const T beta = (T)sc->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

template <class TS, class TD>
__global__ void convert_kernel(int64_t n, const TS* __restrict__ s, TD* __restrict__ d, double scale,
                               const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (TD)((double)s[i] * scale);
}

template <class T>
__global__ void mask_kernel(int64_t n, const uint8_t* __restrict__ fixed, const T* __restrict__ v,
                            T* __restrict__ out, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = fixed[i] ? T(0) : v[i];
}

template <class T>
__global__ void pc_out_kernel(int64_t n, const uint8_t* __restrict__ fixed, const T* __restrict__ r,
                              T* __restrict__ z, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (fixed[i]) z[i] = r[i];
}

template <class T>
__global__ void jacobi_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r, T* __restrict__ z,
                              const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = dinv[i] * r[i];
}

// y += t on the free DOFs (the product of a further block, whose prescribed rows
// hold the identity the first block's product already wrote)
template <class T>
__global__ void add_free_kernel(int64_t n, const uint8_t* __restrict__ fixed, const T* __restrict__ t,
                                T* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!(fixed && fixed[i])) y[i] += t[i];
}

// Chebyshev-Jacobi polynomial preconditioner z = M(r) (the reference's "cheby",
// gfem/solvers.py:289-306): res = D^-1 r, d = res / theta, x = 0; six times
// x += d, res -= D^-1 A d, d = c_a d + c_b res; z = x + d
template <class T>
__global__ void cheb_pc_init_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r,
                                    T* __restrict__ x, T* __restrict__ res, T* __restrict__ d, T ith,
                                    const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T q = dinv[i] * r[i];
    res[i] = q;
    d[i] = q * ith;
    x[i] = T(0);
  }
}

template <class T>
__global__ void cheb_pc_step_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ Ad,
                                    T* __restrict__ x, T* __restrict__ res, T* __restrict__ d, T ca, T cb,
                                    const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T di = d[i];
    x[i] += di;
    const T q = res[i] - dinv[i] * Ad[i];
    res[i] = q;
    d[i] = ca * di + cb * q;
  }
}

template <class T>
__global__ void cheb_pc_out_kernel(int64_t n, const T* __restrict__ x, const T* __restrict__ d, T* __restrict__ z,
                                   const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = x[i] + d[i];
}

// power-iteration start vector of the Chebyshev bound (gfem/solvers.py:333):
// v_i = sin(0.37 i + 0.1) free_i + 1e-3
__global__ void cheb_start_kernel(int64_t n, const uint8_t* __restrict__ fixed, double* __restrict__ v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = ((fixed && fixed[i]) ? 0.0 : sin(0.37 * (double)i + 0.1)) + 1e-3;
}

// w = D^-1 y, or v = w / |w| (scale given)
__global__ void cheb_scale_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                  double* __restrict__ out, double sc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (b ? a[i] * b[i] : a[i]) * sc;
}

__global__ void dinv_kernel(int64_t n, const double* __restrict__ d, const uint8_t* __restrict__ fixed,
                            double* __restrict__ d64, float* __restrict__ d32) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool fx = fixed && fixed[i];
    const double v = fx ? 1.0 : (fabs(d[i]) > 0.0 ? 1.0 / d[i] : 1.0);
    d64[i] = v;
    d32[i] = (float)v;
  }
}

__global__ void axpy_f32_kernel(int64_t n, double* __restrict__ x, const float* __restrict__ d, double sc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += (double)d[i] * sc;
}

__global__ void sub64_kernel(int64_t n, const double* __restrict__ b, const double* __restrict__ t,
                             double* __restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - t[i];
}

__global__ void init_scal_kernel(PcgScal* sc, double tol, int maxiter) {
  sc->rz = sc->pAp = sc->rr = sc->bb = sc->alpha = sc->beta = 0.0;
  sc->spare = tol * tol;
  sc->tol2 = 0.0;
  sc->k = 0;
  sc->maxiter = maxiter;
  sc->done = 0;
}

// start of a new segment of a PCG recursion that keeps its search direction:
// stopping tolerance and iteration budget (the other scalars carry over)
__global__ void segment_scal_kernel(PcgScal* sc, double tol, int maxiter) {
  sc->spare = tol * tol;
  sc->k = 0;
  sc->maxiter = maxiter;
  sc->done = 0;
}

// Condition of the device-side iteration loop (the conditional while node of the
// PCG graph): run the body again while the recursion is not done.  `pad` counts the
// passes of this launch; maxiter + 2 passes end the loop even if the done flag were
// never set, so the loop always terminates.
__global__ void loop_cond_kernel(cudaGraphConditionalHandle h, PcgScal* sc, int head) {
  if (head) sc->pad = 0;
  else sc->pad += 1;
  const bool more = !sc->done && sc->k < sc->maxiter && (long long)sc->pad <= (long long)sc->maxiter + 1;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void scale_f32_kernel(int64_t n, float* __restrict__ v, float a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] *= a;
}

// ---------------------------------------------------------------- helpers
static unsigned red_grid(int64_t n) {
  int64_t g = (n + RT * 4 - 1) / (RT * 4);
  if (g < 1) g = 1;
  if (g > RED_MAX_BLOCKS) g = RED_MAX_BLOCKS;
  return (unsigned)g;
}

template <class T>
static int dot(exfem_solver_s* S, const T* a, const T* b, int F, double* out, int check_done, cudaStream_t st) {
  dot_kernel<T><<<red_grid(S->n), RT, 0, st>>>(S->n, a, b, S->partial.p, S->counter.p, S->scal.p, out, F, check_done);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

static double* ws64(exfem_solver_s* S, int k) {
  DevBuf<double>* v[] = {&S->x64, &S->r64, &S->z64, &S->p64, &S->Ap64, &S->b64, &S->t64};
  return v[k]->p;
}
static float* ws32(exfem_solver_s* S, int k) {
  DevBuf<float>* v[] = {&S->x32, &S->r32, &S->z32, &S->p32, &S->Ap32, &S->b32, &S->t32};
  return v[k]->p;
}
enum { WX = 0, WR, WZ, WP, WAP, WB, WT };
template <class T> static T* ws(exfem_solver_s* S, int k);
template <> double* ws<double>(exfem_solver_s* S, int k) { return ws64(S, k); }
template <> float* ws<float>(exfem_solver_s* S, int k) { return ws32(S, k); }
template <class T> static const T* sdinv(exfem_solver_s* S);
template <> const double* sdinv<double>(exfem_solver_s* S) { return S->dinv64.p; }
template <> const float* sdinv<float>(exfem_solver_s* S) { return S->dinv32.p; }

template <class T> static T* more_buf(exfem_solver_s* S);
template <> double* more_buf<double>(exfem_solver_s* S) { return S->mb64.p; }
template <> float* more_buf<float>(exfem_solver_s* S) { return S->mb32.p; }

// generations of the tangent data / prescribed-DOF buffers over all blocks
static uint64_t tan_gen_all(const exfem_solver_s* S) {
  uint64_t g = S->blk->tan_gen;
  for (auto* b : S->more) g += b->tan_gen;
  return g;
}
static uint64_t bc_gen_all(const exfem_solver_s* S) {
  uint64_t g = S->blk->bc_gen;
  for (auto* b : S->more) g += b->bc_gen;
  return g;
}

// matrix-free product of every block: y = opA_0(v) + sum over the further blocks of
// free * K_b(free * v)
template <class T>
static int mf_apply_all(exfem_solver_s* S, const T* v, T* y, const int* skip, cudaStream_t st) {
  int s;
  if ((s = launch_mf_matvec<T>(S->blk, v, y, skip, st))) return s;
  for (auto* b : S->more) {
    T* t = more_buf<T>(S);
    if ((s = launch_mf_matvec<T>(b, v, t, skip, st))) return s;
    add_free_kernel<T><<<grid_for(S->n, 256), 256, 0, st>>>(S->n, S->blk->fixed.p, t, y, skip);
    EX_LAUNCH_CHECK();
  }
  return EXFEM_OK;
}

template <class T>
static int op_apply(exfem_solver_s* S, const T* v, T* y, const int* skip, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    if (S->op == EXFEM_OP_EBE_F64) {
      if (!S->Ke) { set_error("solver: stored-Ke operator without Ke (call exfem_solver_set_ke)"); return EXFEM_ERR_ARG; }
      int s;
      if ((s = launch_ebe_matvec(S->blk, S->Ke, v, y, skip, st))) return s;
      for (size_t i = 0; i < S->more.size(); ++i) {
        if (!S->more_Ke[i]) {
          set_error("solver: stored-Ke operator without Ke of block %zu (call exfem_solver_set_ke_block)", i + 1);
          return EXFEM_ERR_ARG;
        }
        if ((s = launch_ebe_matvec(S->more[i], S->more_Ke[i], v, S->mb64.p, skip, st))) return s;
        add_free_kernel<double><<<grid_for(S->n, 256), 256, 0, st>>>(S->n, S->blk->fixed.p, S->mb64.p, y, skip);
        EX_LAUNCH_CHECK();
      }
      return EXFEM_OK;
    }
    if (S->op == EXFEM_OP_CSR_F64) {
      if (!S->csr.ready) { set_error("solver: CSR operator not assembled (call exfem_solver_set_ke)"); return EXFEM_ERR_ARG; }
      return csr_apply(S->csr.A, v, y, skip, st);
    }
  }
  return mf_apply_all<T>(S, v, y, skip, st);
}

template <class T>
static int op0_apply(void* ctx, const T* x, T* y, const int* skip, cudaStream_t st) {
  return op_apply<T>((exfem_solver_s*)ctx, x, y, skip, st);
}

template <class T>
static int pc_apply(exfem_solver_s* S, const T* r, T* z, const int* skip, cudaStream_t st) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  if (S->pc == EXFEM_PC_NONE) {
    EX_CUDA(cudaMemcpyAsync(z, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
    return EXFEM_OK;
  }
  if (S->pc == EXFEM_PC_JACOBI) {
    jacobi_kernel<T><<<eg, 256, 0, st>>>(n, sdinv<T>(S), r, z, skip);
    EX_LAUNCH_CHECK();
    return EXFEM_OK;
  }
  if (S->pc == EXFEM_PC_CHEBY) {
    T *x, *res, *d;
    if constexpr (sizeof(T) == 8) {
      x = S->cx64.p, res = S->cr64.p, d = S->cd64.p;
    } else {
      x = S->cx32.p, res = S->cr32.p, d = S->cd32.p;
    }
    T* Ad = z;  // z is free until the final sum: it holds A d meanwhile
    const double hi = S->cheb_lmax, lo = hi / 30.0;
    const double th = 0.5 * (hi + lo), de = 0.5 * (hi - lo), sg = th / de;
    double rh = 1.0 / sg;
    cheb_pc_init_kernel<T><<<eg, 256, 0, st>>>(n, sdinv<T>(S), r, x, res, d, (T)(1.0 / th), skip);
    EX_LAUNCH_CHECK();
    int s;
    for (int j = 0; j < 6; ++j) {
      if ((s = op_apply<T>(S, d, Ad, skip, st))) return s;
      const double rn = 1.0 / (2.0 * sg - rh);
      cheb_pc_step_kernel<T><<<eg, 256, 0, st>>>(n, sdinv<T>(S), Ad, x, res, d, (T)(rn * rh), (T)(2.0 * rn / de),
                                                 skip);
      EX_LAUNCH_CHECK();
      rh = rn;
    }
    cheb_pc_out_kernel<T><<<eg, 256, 0, st>>>(n, x, d, z, skip);
    EX_LAUNCH_CHECK();
    return EXFEM_OK;
  }
  const uint8_t* fixed = S->blk->fixed.p;
  const T* rin = r;
  if (fixed) {
    T* t = ws<T>(S, WT);
    mask_kernel<T><<<eg, 256, 0, st>>>(n, fixed, r, t, skip);
    EX_LAUNCH_CHECK();
    rin = t;
  }
  Level0Op<T> op0;
  op0.apply = &op0_apply<T>;
  op0.ctx = S;
  op0.dinv = sdinv<T>(S);
  int s;
  if ((s = amg_vcycle<T>(S->amg, rin, z, &op0, skip, st))) return s;
  if (fixed) {
    pc_out_kernel<T><<<eg, 256, 0, st>>>(n, fixed, r, z, skip);
    EX_LAUNCH_CHECK();
  }
  return EXFEM_OK;
}

template <class T>
static int pcg_iteration(exfem_solver_s* S, cudaStream_t st) {
  const int* skip = &S->scal.p->done;
  T *x = ws<T>(S, WX), *r = ws<T>(S, WR), *z = ws<T>(S, WZ), *p = ws<T>(S, WP), *Ap = ws<T>(S, WAP);
  int s;
  if ((s = op_apply<T>(S, p, Ap, skip, st))) return s;
  if ((s = dot<T>(S, p, Ap, FIN_ALPHA, nullptr, 1, st))) return s;
  update_xr_kernel<T><<<red_grid(S->n), RT, 0, st>>>(S->n, x, r, p, Ap, S->partial.p, S->counter.p, S->scal.p);
  EX_LAUNCH_CHECK();
  if ((s = pc_apply<T>(S, r, z, skip, st))) return s;
  if ((s = dot<T>(S, r, z, FIN_BETA, nullptr, 1, st))) return s;
  update_p_kernel<T><<<grid_for(S->n, 256), 256, 0, st>>>(S->n, p, z, S->scal.p);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

static int norm64(exfem_solver_s* S, const double* v, double* out, cudaStream_t st);

// Spectral bound of D^-1 A for the Chebyshev-Jacobi preconditioner: 25 power
// iterations from the reference's start vector, times 1.1 (gfem/solvers.py:328-342),
// with the solver's FP64 operator when it has one (the FP32 one otherwise)
static int cheby_bound(exfem_solver_s* S, cudaStream_t st) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  double* v = S->cx64.p;
  double* w = S->cr64.p;
  int s;
  cheb_start_kernel<<<eg, 256, 0, st>>>(n, S->blk->fixed.p, v);
  EX_LAUNCH_CHECK();
  double vn, wn, lam = 1.0;
  if ((s = norm64(S, v, &vn, st))) return s;
  for (int it = 0; it < 25; ++it) {
    if (S->op == EXFEM_OP_MF_F32) {
      convert_kernel<double, float><<<eg, 256, 0, st>>>(n, v, S->cx32.p, 1.0, nullptr);
      EX_LAUNCH_CHECK();
      if ((s = op_apply<float>(S, S->cx32.p, S->cr32.p, nullptr, st))) return s;
      convert_kernel<float, double><<<eg, 256, 0, st>>>(n, S->cr32.p, w, 1.0, nullptr);
      EX_LAUNCH_CHECK();
    } else if ((s = op_apply<double>(S, v, w, nullptr, st))) {
      return s;
    }
    cheb_scale_kernel<<<eg, 256, 0, st>>>(n, w, S->dinv64.p, w, 1.0);
    EX_LAUNCH_CHECK();
    if ((s = norm64(S, w, &wn, st))) return s;
    lam = wn / vn;
    if (!(wn > 0.0) || !std::isfinite(wn)) break;
    cheb_scale_kernel<<<eg, 256, 0, st>>>(n, w, nullptr, v, 1.0 / wn);
    EX_LAUNCH_CHECK();
    vn = 1.0;
  }
  EX_ARG(std::isfinite(lam) && lam > 0.0, "Chebyshev bound: power iteration gave %g", lam);
  S->cheb_lmax = 1.1 * lam;
  return EXFEM_OK;
}

int solver_refresh_diagonal(exfem_solver_s* S, cudaStream_t st) {
  int s;
  const bool stored = S->op == EXFEM_OP_EBE_F64 || S->op == EXFEM_OP_CSR_F64;
  for (size_t i = 0; i <= S->more.size(); ++i) {
    exfem_block_s* b = i ? S->more[i - 1] : S->blk;
    const double* Ke = i ? S->more_Ke[i - 1] : S->Ke;
    double* d = i ? S->mb64.p : S->diag64.p;
    if (stored && !Ke) { set_error("solver: stored-Ke operator without Ke of block %zu", i); return EXFEM_ERR_ARG; }
    if ((s = stored ? launch_ebe_diagonal(b, Ke, d, st) : launch_mf_diagonal(b, d, st))) return s;
    if (i) {
      add_free_kernel<double><<<grid_for(S->n, 256), 256, 0, st>>>(S->n, S->blk->fixed.p, S->mb64.p, S->diag64.p,
                                                                   nullptr);
      EX_LAUNCH_CHECK();
    }
  }
  dinv_kernel<<<grid_for(S->n, 256), 256, 0, st>>>(S->n, S->diag64.p, S->blk->fixed.p, S->dinv64.p, S->dinv32.p);
  EX_LAUNCH_CHECK();
  if (S->pc == EXFEM_PC_CHEBY && (s = cheby_bound(S, st))) return s;
  S->diag_ready = true;
  S->diag_tan_gen = tan_gen_all(S);
  S->diag_bc_gen = bc_gen_all(S);
  return EXFEM_OK;
}

// Graph of the whole PCG loop: a head kernel sets the loop condition from the
// device scalars, then a conditional while node runs one captured iteration plus
// the condition kernel until the recursion is done (or maxiter + 2 passes)
template <class T>
static int loop_graph(exfem_solver_s* S, cudaStream_t st, cudaGraph_t* out) {
  cudaGraph_t g = nullptr;
  EX_CUDA(cudaGraphCreate(&g, 0));
  auto fail = [&](cudaError_t e, const char* what) {
    cudaGraphDestroy(g);
    set_error("PCG loop graph: %s: %s", what, cudaGetErrorString(e));
    return EXFEM_ERR_CUDA;
  };
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
  if (e != cudaSuccess) return fail(e, "condition handle");
  PcgScal* sc = S->scal.p;
  int head = 1;
  void* args[] = {&h, &sc, &head};
  cudaKernelNodeParams kp = {};
  kp.func = (void*)loop_cond_kernel;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = args;
  cudaGraphNode_t n_head, n_loop;
  if ((e = cudaGraphAddKernelNode(&n_head, g, nullptr, 0, &kp)) != cudaSuccess) return fail(e, "head node");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if ((e = cudaGraphAddNode(&n_loop, g, &n_head, 1, &cp)) != cudaSuccess) return fail(e, "while node");
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return fail(e, "capture of the loop body");
  int cs = pcg_iteration<T>(S, st);
  if (!cs) {
    loop_cond_kernel<<<1, 1, 0, st>>>(h, sc, 0);
    if (cudaGetLastError() != cudaSuccess) cs = EXFEM_ERR_CUDA;
  }
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(st, &captured);
  if (cs) {
    cudaGraphDestroy(g);
    return cs;
  }
  if (e != cudaSuccess) return fail(e, "end of the body capture");
  *out = g;
  return EXFEM_OK;
}

// hierarchy work vectors, inverse diagonal of the current operator, and (graphs
// on) the captured PCG iterations in precision T
template <class T>
static int pcg_prepare(exfem_solver_s* S, cudaStream_t st) {
  const int gi = sizeof(T) == 8 ? 0 : 1;
  int s;
  if (S->pc == EXFEM_PC_AMG && !S->amg) { set_error("solver: AMG preconditioner without hierarchy"); return EXFEM_ERR_ARG; }
  if (S->pc == EXFEM_PC_AMG && (s = amg_prepare(S->amg, sizeof(T) == 8 ? EXFEM_F64 : EXFEM_F32))) return s;
  if (S->op == EXFEM_OP_CSR_F64 && S->csr_dirty) {  // element matrices changed: assemble them again
    std::vector<exfem_block_s*> blks{S->blk};
    std::vector<const double*> kes{S->Ke};
    blks.insert(blks.end(), S->more.begin(), S->more.end());
    kes.insert(kes.end(), S->more_Ke.begin(), S->more_Ke.end());
    for (size_t i = 0; i < kes.size(); ++i)
      if (!kes[i]) { set_error("solver: CSR operator without Ke of block %zu", i); return EXFEM_ERR_ARG; }
    if ((s = blocks_csr_assemble(blks, kes, S->csr, st))) return s;
    S->csr_dirty = false;
  }
  const bool stale = !S->diag_ready || S->diag_tan_gen != tan_gen_all(S) || S->diag_bc_gen != bc_gen_all(S);
  if (stale && S->pc != EXFEM_PC_NONE && (s = solver_refresh_diagonal(S, st))) return s;
  const int chunk = S->chunk > 0 ? S->chunk : 8;
  if (S->use_graph) {
    std::vector<const double*> keptr;  // the element matrices a captured stored-Ke graph reads
    if (S->op == EXFEM_OP_EBE_F64) {
      keptr.push_back(S->Ke);
      keptr.insert(keptr.end(), S->more_Ke.begin(), S->more_Ke.end());
    }
    if (S->graph_bc_gen != bc_gen_all(S)) {
      for (auto& ge : S->gexec)
        if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
      S->graph_bc_gen = bc_gen_all(S);
    }
    if (S->gexec[gi] && (S->g_Ke[gi] != keptr || S->g_lmax[gi] != S->cheb_lmax)) {
      cudaGraphExecDestroy(S->gexec[gi]);
      S->gexec[gi] = nullptr;
    }
    if (!S->gexec[gi]) {
      CaptureScope cap;
      cudaGraph_t g = nullptr;
      if (S->device_loop) {
        if ((s = loop_graph<T>(S, st, &g))) return s;
      } else {
        EX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int cs = EXFEM_OK;
        for (int i = 0; i < chunk && !cs; ++i) cs = pcg_iteration<T>(S, st);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (cs) { if (ce == cudaSuccess) cudaGraphDestroy(g); return cs; }
        EX_CUDA(ce);
      }
      cudaError_t ce = cudaGraphInstantiate(&S->gexec[gi], g, 0);
      cudaGraphDestroy(g);
      EX_CUDA(ce);
      S->gloop[gi] = S->device_loop != 0;
      ++S->graph_gen;
      S->g_Ke[gi] = keptr;
      S->g_lmax[gi] = S->cheb_lmax;
    }
  }
  return EXFEM_OK;
}

// chunks of PCG iterations until the device "done" flag is set (at most maxiter
// iterations); the scalars are left in S->h_scal
template <class T>
static int pcg_chunks(exfem_solver_s* S, int maxiter, cudaStream_t st) {
  const int gi = sizeof(T) == 8 ? 0 : 1;
  const int chunk = S->chunk > 0 ? S->chunk : 8;
  int s;
  if (S->use_graph && S->gexec[gi] && S->gloop[gi]) {  // one launch runs the loop to the end
    EX_CUDA(cudaGraphLaunch(S->gexec[gi], st));
    EX_CUDA(cudaMemcpyAsync(S->h_scal, S->scal.p, sizeof(PcgScal), cudaMemcpyDeviceToHost, st));
    EX_CUDA(cudaStreamSynchronize(st));
    return EXFEM_OK;
  }
  const int max_chunks = maxiter / chunk + 2;
  for (int c = 0; c < max_chunks; ++c) {
    EX_CUDA(cudaMemcpyAsync(S->h_scal, S->scal.p, sizeof(PcgScal), cudaMemcpyDeviceToHost, st));
    EX_CUDA(cudaStreamSynchronize(st));
    if (S->h_scal->done) break;
    if (S->use_graph) {
      EX_CUDA(cudaGraphLaunch(S->gexec[gi], st));
    } else {
      for (int i = 0; i < chunk; ++i)
        if ((s = pcg_iteration<T>(S, st))) return s;
    }
  }
  EX_CUDA(cudaMemcpyAsync(S->h_scal, S->scal.p, sizeof(PcgScal), cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaStreamSynchronize(st));
  return EXFEM_OK;
}

// PCG on workspace vectors b (WB) -> x (WX) in precision T
template <class T>
static int pcg_run(exfem_solver_s* S, double tol, int maxiter, int* iters, double* relres, cudaStream_t st) {
  const int64_t n = S->n;
  int s;
  if ((s = pcg_prepare<T>(S, st))) return s;
  T *x = ws<T>(S, WX), *r = ws<T>(S, WR), *z = ws<T>(S, WZ), *p = ws<T>(S, WP), *b = ws<T>(S, WB);
  init_scal_kernel<<<1, 1, 0, st>>>(S->scal.p, tol, maxiter);
  EX_LAUNCH_CHECK();
  EX_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, st));
  EX_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
  if ((s = dot<T>(S, b, b, FIN_BB, nullptr, 0, st))) return s;
  if ((s = pc_apply<T>(S, r, z, nullptr, st))) return s;
  EX_CUDA(cudaMemcpyAsync(p, z, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
  if ((s = dot<T>(S, r, z, FIN_RZ0, nullptr, 0, st))) return s;
  if ((s = dot<T>(S, r, r, FIN_RR0, nullptr, 0, st))) return s;
  if ((s = pcg_chunks<T>(S, maxiter, st))) return s;
  const PcgScal& h = *S->h_scal;
  if (iters) *iters = h.k;
  const double rel = sqrt(h.rr / fmax(h.bb, 1e-300));
  if (relres) *relres = rel;
  return (std::isfinite(rel) && rel <= 1e-3) ? EXFEM_OK : EXFEM_NOT_CONVERGED;
}

int solver_pcg(exfem_solver_s* S, const double* b, double* x, double tol, int maxiter, int* iters,
               double* relres, cudaStream_t st) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  int s;
  if (S->op == EXFEM_OP_MF_F32) {
    convert_kernel<double, float><<<eg, 256, 0, st>>>(n, b, S->b32.p, 1.0, nullptr);
    EX_LAUNCH_CHECK();
    s = pcg_run<float>(S, tol, maxiter, iters, relres, st);
    if (s < 0) return s;
    convert_kernel<float, double><<<eg, 256, 0, st>>>(n, S->x32.p, x, 1.0, nullptr);
    EX_LAUNCH_CHECK();
    return s;
  }
  EX_CUDA(cudaMemcpyAsync(S->b64.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  s = pcg_run<double>(S, tol, maxiter, iters, relres, st);
  if (s < 0) return s;
  EX_CUDA(cudaMemcpyAsync(x, S->x64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  return s;
}

static int norm64(exfem_solver_s* S, const double* v, double* out, cudaStream_t st) {
  int s;
  if ((s = dot<double>(S, v, v, FIN_STORE, S->dscr.p, 0, st))) return s;
  double h;
  EX_CUDA(cudaMemcpyAsync(&h, S->dscr.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaStreamSynchronize(st));
  *out = sqrt(h);
  return EXFEM_OK;
}

int solver_mixed(exfem_solver_s* S, const double* b, double* x, double tol, double inner_tol, int max_pass,
                 int maxiter, int* iters, int* passes, double* relres, cudaStream_t st) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  if (S->op == EXFEM_OP_EBE_F64 || S->op == EXFEM_OP_CSR_F64) {
    set_error("mixed refinement needs a matrix-free operator (EXFEM_OP_MF_F32)");
    return EXFEM_ERR_ARG;
  }
  // r64 holds the FP64 residual, x the FP64 solution; t64 is scratch for A64(x)
  int s;
  EX_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
  EX_CUDA(cudaMemcpyAsync(S->r64.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  double bn;
  if ((s = norm64(S, b, &bn, st))) return s;
  if (bn == 0.0) bn = 1.0;
  int its = 0, p = 0;
  double rn = bn;
  // Passes after the first stop at 4x the first pass's iteration count: a pass can
  // only lower the FP64 residual by the FP32 operator's attainable accuracy (about
  // 1e-3 relative on a 12.5M-DOF C3D10 cube), and the recursion of a later pass,
  // whose right-hand side is the rounding-level residual of the previous one, can
  // stall above inner_tol there (the reference runs it to cg_maxiter).
  int cap = maxiter;
  const double itol = inner_tol;
  for (p = 0; p < max_pass; ++p) {
    double sc;
    if ((s = norm64(S, S->r64.p, &sc, st))) return s;
    if (sc == 0.0) sc = 1.0;
    convert_kernel<double, float><<<eg, 256, 0, st>>>(n, S->r64.p, S->b32.p, 1.0 / sc, nullptr);
    EX_LAUNCH_CHECK();
    int k = 0;
    double rr;
    s = pcg_run<float>(S, itol, cap, &k, &rr, st);
    if (s < 0) return s;
    its += k;
    axpy_f32_kernel<<<eg, 256, 0, st>>>(n, x, S->x32.p, sc);
    EX_LAUNCH_CHECK();
    if ((s = mf_apply_all<double>(S, x, S->Ap64.p, nullptr, st))) return s;
    sub64_kernel<<<eg, 256, 0, st>>>(n, b, S->Ap64.p, S->r64.p);
    EX_LAUNCH_CHECK();
    if ((s = norm64(S, S->r64.p, &rn, st))) return s;
    if (!std::isfinite(rn)) break;
    if (rn <= tol * bn) { ++p; break; }
    if (p == 0) cap = std::min(maxiter, std::max(4 * k, 32));
  }
  if (iters) *iters = its;
  if (passes) *passes = p;
  if (relres) *relres = rn / bn;
  return (std::isfinite(rn) && rn <= tol * bn) ? EXFEM_OK : EXFEM_NOT_CONVERGED;
}

// Mixed precision with reliable updates (Sleijpen & van der Vorst, "Reliable
// updated residuals in hybrid Bi-CG methods", Computing 56, 1996; used for
// mixed-precision CG by Clark, Babich, Barros, Brower & Rebbi, Comput. Phys.
// Commun. 181, 2010): one FP32 PCG recursion (FP32 matrix-free product and V-cycle,
// FP64 scalars) whose residual is replaced by the FP64 residual b - A64 x every
// time the recursion has lowered it by `delta` since the last replacement; x is
// accumulated in FP64 at each replacement.  Unlike restarted refinement the search
// direction is kept across replacements (rescaled to the new residual's units), so
// the FP32 iterations stay close to the FP64 PCG count instead of rebuilding the
// Krylov space in every pass.  A replacement that does not halve the FP64 residual
// restarts the recursion from the preconditioned residual.  Stops when
// ||b - A64 x|| <= tol ||b||.  `updates` receives the number of replacements.
int solver_mixed_ru(exfem_solver_s* S, const double* b, double* x, double tol, double delta, int max_updates,
                    int maxiter, int* iters, int* updates, double* relres, cudaStream_t st) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  if (S->op == EXFEM_OP_EBE_F64 || S->op == EXFEM_OP_CSR_F64) {
    set_error("mixed refinement needs a matrix-free operator (EXFEM_OP_MF_F32)");
    return EXFEM_ERR_ARG;
  }
  int s;
  if ((s = pcg_prepare<float>(S, st))) return s;
  float *x32 = S->x32.p, *r32 = S->r32.p, *z32 = S->z32.p, *p32 = S->p32.p;
  EX_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
  EX_CUDA(cudaMemcpyAsync(S->r64.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  double bn;
  if ((s = norm64(S, b, &bn, st))) return s;
  int its = 0, nup = 0;
  double rn = bn;
  if (bn == 0.0) {
    if (iters) *iters = 0;
    if (updates) *updates = 0;
    if (relres) *relres = 0.0;
    return EXFEM_OK;
  }
  double sc = bn, rn_prev = bn;
  bool restart = true;
  init_scal_kernel<<<1, 1, 0, st>>>(S->scal.p, 1.0, maxiter);
  EX_LAUNCH_CHECK();
  for (;;) {
    // (re)start a segment from the FP64 residual r64, in units of sc
    convert_kernel<double, float><<<eg, 256, 0, st>>>(n, S->r64.p, r32, 1.0 / sc, nullptr);
    EX_LAUNCH_CHECK();
    EX_CUDA(cudaMemsetAsync(x32, 0, sizeof(float) * n, st));
    const double seg_tol = std::max(delta, tol * bn / rn);
    segment_scal_kernel<<<1, 1, 0, st>>>(S->scal.p, seg_tol, std::max(maxiter - its, 0));
    EX_LAUNCH_CHECK();
    if ((s = dot<float>(S, r32, r32, FIN_BB, nullptr, 0, st))) return s;
    if ((s = pc_apply<float>(S, r32, z32, nullptr, st))) return s;
    if (restart) {
      EX_CUDA(cudaMemcpyAsync(p32, z32, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    } else {
      // the iteration that ended the last segment skipped its direction update
      // (p = z + beta p, beta of that iteration): do it with the replaced residual
      update_p_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(n, p32, z32, S->scal.p);
      EX_LAUNCH_CHECK();
    }
    if ((s = dot<float>(S, r32, z32, FIN_RZ0, nullptr, 0, st))) return s;
    if ((s = dot<float>(S, r32, r32, FIN_RR0, nullptr, 0, st))) return s;
    if ((s = pcg_chunks<float>(S, std::max(maxiter - its, 0), st))) return s;
    its += S->h_scal->k;
    // replacement: x += sc x32, r64 = b - A64 x
    axpy_f32_kernel<<<eg, 256, 0, st>>>(n, x, x32, sc);
    EX_LAUNCH_CHECK();
    if ((s = mf_apply_all<double>(S, x, S->Ap64.p, nullptr, st))) return s;
    sub64_kernel<<<eg, 256, 0, st>>>(n, b, S->Ap64.p, S->r64.p);
    EX_LAUNCH_CHECK();
    if ((s = norm64(S, S->r64.p, &rn, st))) return s;
    ++nup;
    if (!std::isfinite(rn) || rn <= tol * bn || its >= maxiter || nup >= max_updates) break;
    // keep the search direction in the new residual's units; restart when the
    // replacement did not halve the FP64 residual (the recursion has stalled)
    restart = !(rn <= 0.5 * rn_prev);
    if (!restart) {
      scale_f32_kernel<<<eg, 256, 0, st>>>(n, p32, (float)(sc / rn));
      EX_LAUNCH_CHECK();
    }
    rn_prev = rn;
    sc = rn;
  }
  if (iters) *iters = its;
  if (updates) *updates = nup;
  if (relres) *relres = rn / bn;
  return (std::isfinite(rn) && rn <= tol * bn) ? EXFEM_OK : EXFEM_NOT_CONVERGED;
}

// ---------------------------------------------------------------- reliable updates as one graph
//
// The same recursion as solver_mixed_ru with every decision taken on the device:
// the replacement segments are a conditional while node whose body holds the
// segment start (scaled FP32 residual, fresh or rescaled direction), the PCG loop
// (a nested conditional while node over one captured iteration), the FP64
// replacement x += sc x32, r64 = b - A64 x, and the test for the next segment.  The
// scalars (||b||, ||r||, the scale, the restart flag, iteration and replacement
// counts) live in a MixedScal in device memory; every formula is the host path's, in
// the same order and precision, so both give the same iterates.  One graph per
// solver handle, built on first use and rebuilt with the PCG graph (prescribed DOFs,
// element matrices, Chebyshev bound); b and x pass through the handle's own vectors
// so that the graph's addresses stay fixed.

__global__ void mx_params_kernel(MixedScal* ms, double tol, double delta, int maxiter, int max_updates) {
  ms->tol = tol;
  ms->delta = delta;
  ms->maxiter = maxiter;
  ms->max_updates = max_updates;
}

// after ||b||^2 landed in nrm2: the recursion's starting scalars
__global__ void mx_start_kernel(MixedScal* ms) {
  const double bn = sqrt(ms->nrm2);
  ms->bn = bn;
  ms->rn = bn;
  ms->rn_prev = bn;
  ms->sc = bn;
  ms->restart = 1;
  ms->its = 0;
  ms->nup = 0;
  ms->done = bn == 0.0;
}

// segment start: 1/sc for the scaled residual, the segment's tolerance and budget
// (segment_scal_kernel's fields)
__global__ void mx_seg_begin_kernel(MixedScal* ms, PcgScal* sc) {
  ms->inv_sc = 1.0 / ms->sc;
  const double seg_tol = fmax(ms->delta, ms->tol * ms->bn / ms->rn);
  sc->spare = seg_tol * seg_tol;
  sc->k = 0;
  sc->maxiter = max(ms->maxiter - ms->its, 0);
  sc->done = 0;
}

__global__ void mx_scale_down_kernel(int64_t n, const double* __restrict__ r64, float* __restrict__ r32,
                                     const MixedScal* ms) {
  const double s = ms->inv_sc;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r32[i] = (float)((double)r64[i] * s);
}

// direction of the new segment: the preconditioned residual after a restart, else
// the skipped update of the last iteration, p = z + beta p
__global__ void mx_dir_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ z, const PcgScal* sc,
                              const MixedScal* ms) {
  const bool fresh = ms->restart != 0;
  const float beta = (float)sc->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = fresh ? z[i] : z[i] + beta * p[i];
}

__global__ void mx_count_kernel(MixedScal* ms, const PcgScal* sc) { ms->its += sc->k; }

__global__ void mx_axpy_kernel(int64_t n, double* __restrict__ x, const float* __restrict__ d, const MixedScal* ms) {
  const double sc = ms->sc;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += (double)d[i] * sc;
}

// after ||r64||^2 landed in nrm2: stop, or prepare the next segment (restart when the
// replacement did not halve the residual, else rescale the kept direction)
__global__ void mx_seg_end_kernel(MixedScal* ms) {
  const double rn = sqrt(ms->nrm2);
  ms->rn = rn;
  ms->nup += 1;
  ms->done = !isfinite(rn) || rn <= ms->tol * ms->bn || ms->its >= ms->maxiter || ms->nup >= ms->max_updates;
  if (!ms->done) {
    ms->restart = !(rn <= 0.5 * ms->rn_prev);
    ms->pscale = ms->restart ? 1.0f : (float)(ms->sc / rn);
    ms->rn_prev = rn;
    ms->sc = rn;
  }
}

__global__ void mx_rescale_kernel(int64_t n, float* __restrict__ p, const MixedScal* ms) {
  if (ms->done || ms->restart) return;
  const float a = ms->pscale;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] *= a;
}

// segment loop condition: another segment while not done, at most max_updates + 1
__global__ void mx_cond_kernel(cudaGraphConditionalHandle h, MixedScal* ms, int head) {
  if (head) ms->loops = 0;
  else ms->loops += 1;
  const bool more = !ms->done && (long long)ms->loops <= (long long)ms->max_updates;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

// nodes of g that no edge leaves
static int graph_leaves(cudaGraph_t g, std::vector<cudaGraphNode_t>& out) {
  size_t nn = 0, ne = 0;
  EX_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) EX_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
  EX_CUDA(cudaGraphGetEdges(g, nullptr, nullptr, &ne));
  std::vector<cudaGraphNode_t> from(ne), to(ne);
  if (ne) EX_CUDA(cudaGraphGetEdges(g, from.data(), to.data(), &ne));
  out.clear();
  for (auto nd : nodes)
    if (std::find(from.begin(), from.end(), nd) == from.end()) out.push_back(nd);
  return EXFEM_OK;
}

// capture the work of f on stream st into g after the nodes deps
template <class F>
static int capture_into(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, cudaStream_t st, F f) {
  cudaError_t e = cudaStreamBeginCaptureToGraph(st, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                                cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    set_error("graph capture could not start: %s", cudaGetErrorString(e));
    return EXFEM_ERR_CUDA;
  }
  int cs = f();
  if (!cs && cudaGetLastError() != cudaSuccess) cs = EXFEM_ERR_CUDA;
  cudaGraph_t out = nullptr;
  e = cudaStreamEndCapture(st, &out);
  if (cs) return cs;
  if (e != cudaSuccess) {
    set_error("graph capture failed: %s", cudaGetErrorString(e));
    return EXFEM_ERR_CUDA;
  }
  return EXFEM_OK;
}

// the nodes of one reliable-update solve of mx_b into mx_x, appended to g after its
// current leaves (g may be the body of an enclosing conditional node)
static int mixed_nodes(exfem_solver_s* S, cudaStream_t st, cudaGraph_t g) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  MixedScal* ms = S->mx_scal.p;
  PcgScal* sc = S->scal.p;
  float *x32 = S->x32.p, *r32 = S->r32.p, *z32 = S->z32.p, *p32 = S->p32.p;
  const double* b = S->mx_b.p;
  double* x = S->mx_x.p;
  auto fail = [&](int s) { return s; };
  int s;
  cudaGraphConditionalHandle hs, hp;
  cudaGraph_t seg, body;
  cudaGraphNode_t n_seg, n_pcg;
  std::vector<cudaGraphNode_t> leaves;
  if ((s = graph_leaves(g, leaves))) return s;
  // head: x = 0, r64 = b, ||b||, start scalars, the PCG scalars' reset
  s = capture_into(g, leaves, st, [&]() -> int {
    EX_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    EX_CUDA(cudaMemcpyAsync(S->r64.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    int q;
    if ((q = dot<double>(S, b, b, FIN_STORE, &ms->nrm2, 0, st))) return q;
    mx_start_kernel<<<1, 1, 0, st>>>(ms);
    init_scal_kernel<<<1, 1, 0, st>>>(sc, 1.0, 0);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  // the segment loop
  if ((s = graph_leaves(g, leaves))) return fail(s);
  {
    cudaError_t e = cudaGraphConditionalHandleCreate(&hs, g, 0, 0);
    if (e != cudaSuccess) return fail((set_error("condition handle: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
  }
  s = capture_into(g, leaves, st, [&]() -> int {
    mx_cond_kernel<<<1, 1, 0, st>>>(hs, ms, 1);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  {
    std::vector<cudaGraphNode_t> deps;
    if ((s = graph_leaves(g, deps))) return fail(s);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hs;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(&n_seg, g, deps.data(), deps.size(), &cp);
    if (e != cudaSuccess) return fail((set_error("while node: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
    seg = cp.conditional.phGraph_out[0];
  }
  // segment start
  s = capture_into(seg, {}, st, [&]() -> int {
    mx_seg_begin_kernel<<<1, 1, 0, st>>>(ms, sc);
    mx_scale_down_kernel<<<eg, 256, 0, st>>>(n, S->r64.p, r32, ms);
    EX_CUDA(cudaMemsetAsync(x32, 0, sizeof(float) * n, st));
    int q;
    if ((q = dot<float>(S, r32, r32, FIN_BB, nullptr, 0, st))) return q;
    if ((q = pc_apply<float>(S, r32, z32, nullptr, st))) return q;
    mx_dir_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, p32, z32, sc, ms);
    if ((q = dot<float>(S, r32, z32, FIN_RZ0, nullptr, 0, st))) return q;
    if ((q = dot<float>(S, r32, r32, FIN_RR0, nullptr, 0, st))) return q;
    return EXFEM_OK;
  });
  if (s) return fail(s);
  // the PCG loop of the segment
  if ((s = graph_leaves(seg, leaves))) return fail(s);
  {
    cudaError_t e = cudaGraphConditionalHandleCreate(&hp, seg, 0, 0);
    if (e != cudaSuccess) return fail((set_error("condition handle: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
  }
  s = capture_into(seg, leaves, st, [&]() -> int {
    loop_cond_kernel<<<1, 1, 0, st>>>(hp, sc, 1);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  {
    std::vector<cudaGraphNode_t> deps;
    if ((s = graph_leaves(seg, deps))) return fail(s);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hp;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(&n_pcg, seg, deps.data(), deps.size(), &cp);
    if (e != cudaSuccess) return fail((set_error("while node: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
    body = cp.conditional.phGraph_out[0];
  }
  s = capture_into(body, {}, st, [&]() -> int {
    int q;
    if ((q = pcg_iteration<float>(S, st))) return q;
    loop_cond_kernel<<<1, 1, 0, st>>>(hp, sc, 0);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  // segment end: replacement, FP64 residual, test, rescale, loop condition
  s = capture_into(seg, {n_pcg}, st, [&]() -> int {
    mx_count_kernel<<<1, 1, 0, st>>>(ms, sc);
    mx_axpy_kernel<<<eg, 256, 0, st>>>(n, x, x32, ms);
    int q;
    if ((q = mf_apply_all<double>(S, x, S->Ap64.p, nullptr, st))) return q;
    sub64_kernel<<<eg, 256, 0, st>>>(n, b, S->Ap64.p, S->r64.p);
    if ((q = dot<double>(S, S->r64.p, S->r64.p, FIN_STORE, &ms->nrm2, 0, st))) return q;
    mx_seg_end_kernel<<<1, 1, 0, st>>>(ms);
    mx_rescale_kernel<<<eg, 256, 0, st>>>(n, p32, ms);
    mx_cond_kernel<<<1, 1, 0, st>>>(hs, ms, 0);
    return EXFEM_OK;
  });
  return s;
}

static int mixed_graph_build(exfem_solver_s* S, cudaStream_t st, cudaGraph_t* out) {
  cudaGraph_t g = nullptr;
  EX_CUDA(cudaGraphCreate(&g, 0));
  int s = mixed_nodes(S, st, g);
  if (s) {
    cudaGraphDestroy(g);
    return s;
  }
  *out = g;
  return EXFEM_OK;
}

int solver_mixed_graph(exfem_solver_s* S, const double* b, double* x, double tol, double delta, int max_updates,
                       int maxiter, int* iters, int* updates, double* relres, cudaStream_t st) {
  const int64_t n = S->n;
  if (S->op == EXFEM_OP_EBE_F64 || S->op == EXFEM_OP_CSR_F64) {
    set_error("mixed refinement needs a matrix-free operator (EXFEM_OP_MF_F32)");
    return EXFEM_ERR_ARG;
  }
  int s;
  if ((s = pcg_prepare<float>(S, st))) return s;
  if (!S->mx_b.p && ((s = S->mx_b.alloc(std::max<int64_t>(n, 1))) || (s = S->mx_x.alloc(std::max<int64_t>(n, 1))) ||
                     (s = S->mx_scal.alloc(1))))
    return s;
  // the PCG graph's validity covers this one (same captured iteration)
  if (S->gmixed && S->gmixed_gen != S->graph_gen) {
    cudaGraphExecDestroy(S->gmixed);
    S->gmixed = nullptr;
  }
  if (!S->gmixed) {
    CaptureScope cap;
    cudaGraph_t g = nullptr;
    if ((s = mixed_graph_build(S, st, &g))) return s;
    cudaError_t e = cudaGraphInstantiate(&S->gmixed, g, 0);
    cudaGraphDestroy(g);
    EX_CUDA(e);
    S->gmixed_gen = S->graph_gen;
  }
  EX_CUDA(cudaMemcpyAsync(S->mx_b.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  mx_params_kernel<<<1, 1, 0, st>>>(S->mx_scal.p, tol, delta, maxiter, max_updates);
  EX_LAUNCH_CHECK();
  EX_CUDA(cudaGraphLaunch(S->gmixed, st));
  EX_CUDA(cudaMemcpyAsync(x, S->mx_x.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  MixedScal h;
  EX_CUDA(cudaMemcpyAsync(&h, S->mx_scal.p, sizeof(MixedScal), cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaStreamSynchronize(st));
  if (h.bn == 0.0) {
    if (iters) *iters = 0;
    if (updates) *updates = 0;
    if (relres) *relres = 0.0;
    return EXFEM_OK;
  }
  if (iters) *iters = h.its;
  if (updates) *updates = h.nup;
  if (relres) *relres = h.rn / h.bn;
  return (std::isfinite(h.rn) && h.rn <= tol * h.bn) ? EXFEM_OK : EXFEM_NOT_CONVERGED;
}

// ---------------------------------------------------------------- Newton increment as one graph
//
// One increment of StaticSolver (gfem/solvers.py:607-683: the tangent predictor,
// then Newton corrections with the reference's convergence test and its 4-step
// backtracking line search) for a single-block model with the matrix-free tangent
// and the reliable-update mixed solve, as one graph launch: every norm, test and
// step length is computed on the device, the Newton loop and the line search are
// conditional while nodes, each correction's linear solve sits under a conditional
// if node (skipped once the increment has converged) and is the graph form of the
// mixed solve (mixed_nodes).  Elementwise updates use unfused multiply and add, as
// the host driver's array arithmetic does; norms are fixed-order device sums.

__global__ void nw_init_kernel(NewtonScal* ns, double rtol, int max_iter, int line_search, double qref) {
  ns->rtol = rtol;
  ns->max_iter = max_iter;
  ns->line_search = line_search;
  ns->qref = qref;
  ns->it = 0;
  ns->done = 0;
  ns->converged = 0;
  ns->failed = 0;
  ns->corrections = max_iter;
  ns->dut = 0.0;
  ns->loops = 0;
}

// d = a - b
__global__ void nw_sub_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                              double* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = __dsub_rn(a[i], b[i]);
}

// r = free * (f [+ k] - fext); with neg also rhs = -r
__global__ void nw_residual_kernel(int64_t n, const uint8_t* __restrict__ fixed, const double* __restrict__ f,
                                   const double* __restrict__ k, const double* __restrict__ fext, double* __restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = k ? __dadd_rn(f[i], k[i]) : f[i];
    const double fr = (fixed && fixed[i]) ? 0.0 : 1.0;
    r[i] = __dmul_rn(fr, __dsub_rn(a, fext[i]));
  }
}

__global__ void nw_neg_kernel(int64_t n, const double* __restrict__ r, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = -r[i];
}

// predictor: qref = max(qref, ||r||)
__global__ void nw_pred_kernel(NewtonScal* ns) { ns->qref = fmax(ns->qref, sqrt(ns->nrm_r)); }

// u = ut + free * du
__global__ void nw_pred_step_kernel(int64_t n, const uint8_t* __restrict__ fixed, const double* __restrict__ ut,
                                    const double* __restrict__ du, double* __restrict__ u) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double fr = (fixed && fixed[i]) ? 0.0 : 1.0;
    u[i] = __dadd_rn(ut[i], __dmul_rn(fr, du[i]));
  }
}

__global__ void nw_fn_kernel(NewtonScal* ns) { ns->fn_t = sqrt(ns->nrm_t); }

__global__ void nw_lin_kernel(NewtonScal* ns, const MixedScal* ms) {
  ns->lin_its = ms->its;
  ns->lin_nup = ms->nup;
}

// the convergence test of one Newton iteration (gfem/solvers.py:640-660); sets the
// condition of the correction that follows
__global__ void nw_test_kernel(NewtonScal* ns, cudaGraphConditionalHandle h_solve) {
  ns->it += 1;
  const double rt = sqrt(ns->nrm_r), ft = sqrt(ns->nrm_f), utn = sqrt(ns->nrm_u);
  ns->rt = rt;
  ns->ft = ft;
  const double ref = fmax(fmax(ns->fn_t, ft), fmax(1e-3 * ns->qref, 1e-30));
  ns->qref = fmax(ns->qref, fmax(ns->fn_t, ft));
  const double ratio = rt / ref;
  ns->ratio = ratio;
  if (ns->it <= 64) ns->hist[ns->it - 1] = ratio;
  if (!isfinite(rt)) {
    ns->failed = 1;
    ns->done = 1;
  } else {
    const bool small_du = ns->dut <= 1e-2 * fmax(utn, 1e-30);
    if (ratio <= ns->rtol * 1e-2 || (ns->it > 1 && ratio <= ns->rtol && small_du)) {
      ns->converged = 1;
      ns->done = 1;
      ns->corrections = ns->it - 1;
    }
  }
  ns->alpha = 1.0;
  ns->rls = rt;
  ns->ls_count = 0;
  ns->ls_done = !ns->line_search;
  cudaGraphSetConditional(h_solve, ns->done ? 0u : 1u);
}

// trial point of the line search: ut = u + alpha du
__global__ void nw_trial_kernel(int64_t n, const double* __restrict__ u, const double* __restrict__ du,
                                double* __restrict__ ut, const NewtonScal* ns) {
  const double a = ns->alpha;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    ut[i] = __dadd_rn(u[i], __dmul_rn(a, du[i]));
}

// accept the step when the trial residual fell below the current one or alpha < 0.2
__global__ void nw_ls_test_kernel(NewtonScal* ns, cudaGraphConditionalHandle h) {
  ns->ls_count += 1;
  const double n2 = sqrt(ns->nrm_r);
  ns->n2 = n2;
  if (n2 < ns->rls || ns->alpha < 0.2) ns->ls_done = 1;
  else ns->alpha *= 0.5;
  cudaGraphSetConditional(h, (!ns->ls_done && ns->ls_count < 4) ? 1u : 0u);
}

__global__ void nw_ls_head_kernel(NewtonScal* ns, cudaGraphConditionalHandle h) {
  cudaGraphSetConditional(h, ns->ls_done ? 0u : 1u);
}

// u = u + alpha du; dut = |alpha| ||du|| (alpha is a power of two: the same as ||alpha du||)
__global__ void nw_step_kernel(int64_t n, double* __restrict__ u, const double* __restrict__ du,
                               const NewtonScal* ns) {
  const double a = ns->alpha;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    u[i] = __dadd_rn(u[i], __dmul_rn(a, du[i]));
}

__global__ void nw_dut_kernel(NewtonScal* ns) { ns->dut = fabs(ns->alpha) * sqrt(ns->nrm_du); }

// Newton loop condition: another iteration while not done, at most max_iter
__global__ void nw_cond_kernel(cudaGraphConditionalHandle h, NewtonScal* ns, int head) {
  if (head) ns->loops = 0;
  else ns->loops += 1;
  cudaGraphSetConditional(h, (!ns->done && ns->it < ns->max_iter && ns->loops <= ns->max_iter) ? 1u : 0u);
}

// a += b
__global__ void nw_add_kernel(int64_t n, double* __restrict__ a, const double* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = __dadd_rn(a[i], b[i]);
}

// the model's blocks in order (the solver's first block, then the further ones)
static exfem_block_s* nw_block(const exfem_solver_s* S, size_t i) { return i ? S->more[i - 1] : S->blk; }
static size_t nw_nblock(const exfem_solver_s* S) { return 1 + S->more.size(); }
static bool nw_j2(const exfem_block_s* b) { return b->mat.kind == EXFEM_J2; }
// offset of block i's J2 states in the concatenated state buffers (0 entries for an
// elastic block)
static int64_t nw_state_off(const exfem_solver_s* S, size_t i) {
  int64_t o = 0;
  for (size_t k = 0; k < i; ++k) {
    const exfem_block_s* b = nw_block(S, k);
    if (nw_j2(b)) o += b->ne * b->ngp * b->nstate;
  }
  return o;
}

// internal force f = sum over the blocks, in block order (and, for J2 blocks, the
// new states and the consistent tangent data) at u
static int nw_fint(exfem_solver_s* S, const double* u, double* s_new, double* f, cudaStream_t st) {
  int s;
  for (size_t i = 0; i < nw_nblock(S); ++i) {
    exfem_block_s* b = nw_block(S, i);
    const bool j2 = nw_j2(b);
    const int64_t o = nw_state_off(S, i);
    double* fb = i ? S->mb64.p : f;
    if ((s = launch_force(b, FORCE_FULL, u, j2 ? S->nw_s_old.p + o : nullptr, j2 ? s_new + o : nullptr, b->ys.p,
                          nullptr, nullptr, nullptr, st)))
      return s;
    if ((s = launch_gather_assemble(b, b->ys.p, fb, nullptr, nullptr, st))) return s;
    if (i) {
      nw_add_kernel<<<grid_for(S->n, 256), 256, 0, st>>>(S->n, f, fb);
      EX_LAUNCH_CHECK();
    }
  }
  return EXFEM_OK;
}

// consistent tangent data of every J2 block at (u, states of the last converged increment)
static int nw_tangent(exfem_solver_s* S, const double* u, cudaStream_t st) {
  int s;
  for (size_t i = 0; i < nw_nblock(S); ++i) {
    exfem_block_s* b = nw_block(S, i);
    if (nw_j2(b) && (s = launch_force(b, FORCE_TANGENT, u, S->nw_s_old.p + nw_state_off(S, i), nullptr, nullptr,
                                      nullptr, nullptr, nullptr, st)))
      return s;
  }
  return EXFEM_OK;
}

// y = sum over the blocks of their FP64 matrix-free tangent products of v (no
// prescribed rows), in block order
static int nw_jvp(exfem_solver_s* S, const double* v, double* y, cudaStream_t st) {
  int s;
  for (size_t i = 0; i < nw_nblock(S); ++i) {
    double* yb = i ? S->mb64.p : y;
    if ((s = launch_mf_matvec<double>(nw_block(S, i), v, yb, nullptr, st, false))) return s;
    if (i) {
      nw_add_kernel<<<grid_for(S->n, 256), 256, 0, st>>>(S->n, y, yb);
      EX_LAUNCH_CHECK();
    }
  }
  return EXFEM_OK;
}

static bool nw_any_j2(const exfem_solver_s* S) {
  for (size_t i = 0; i < nw_nblock(S); ++i)
    if (nw_j2(nw_block(S, i))) return true;
  return false;
}

static int newton_graph_build(exfem_solver_s* S, cudaStream_t st, cudaGraph_t* out) {
  const int64_t n = S->n;
  const unsigned eg = grid_for(n, 256);
  exfem_block_s* b = S->blk;
  const bool j2 = nw_any_j2(S);
  const uint8_t* fx = b->fixed.p;
  NewtonScal* ns = S->nw_scal.p;
  double *U = S->nw_u.p, *UT = S->nw_ut.p, *DU = S->nw_du.p, *R = S->nw_r.p, *F = S->nw_f.p, *T = S->nw_t.p;
  const double *FEXT = S->nw_fext.p, *START = S->nw_start.p;
  cudaGraph_t g = nullptr;
  EX_CUDA(cudaGraphCreate(&g, 0));
  auto fail = [&](int s) {
    cudaGraphDestroy(g);
    return s;
  };
  int s;
  std::vector<cudaGraphNode_t> leaves;
  // predictor (gfem/solvers.py:607-624): r = free (fint(uc) + K(uc)(ut - uc) - fext),
  // du from the mixed solve of -r (a zero r solves to zero), u = ut + free du
  s = capture_into(g, {}, st, [&]() -> int {
    int q;
    EX_CUDA(cudaMemcpyAsync(UT, START, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    nw_sub_kernel<<<eg, 256, 0, st>>>(n, UT, U, DU);
    if ((q = nw_fint(S, U, S->nw_s_trial.p, F, st))) return q;
    if ((q = nw_tangent(S, U, st))) return q;
    if ((q = nw_jvp(S, DU, T, st))) return q;
    nw_residual_kernel<<<eg, 256, 0, st>>>(n, fx, F, T, FEXT, R);
    if ((q = dot<double>(S, R, R, FIN_STORE, &ns->nrm_r, 0, st))) return q;
    nw_pred_kernel<<<1, 1, 0, st>>>(ns);
    // the tangent of a J2 block changes with u and the states: its diagonal with it
    // (an elastic block's diagonal is refreshed before the launch when stale)
    if (j2 && (q = solver_refresh_diagonal(S, st))) return q;
    nw_neg_kernel<<<eg, 256, 0, st>>>(n, R, S->mx_b.p);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  if ((s = mixed_nodes(S, st, g))) return fail(s);
  if ((s = graph_leaves(g, leaves))) return fail(s);
  s = capture_into(g, leaves, st, [&]() -> int {
    nw_lin_kernel<<<1, 1, 0, st>>>(ns, S->mx_scal.p);
    nw_pred_step_kernel<<<eg, 256, 0, st>>>(n, fx, UT, S->mx_x.p, U);
    int q;
    if ((q = dot<double>(S, FEXT, FEXT, FIN_STORE, &ns->nrm_t, 0, st))) return q;
    nw_fn_kernel<<<1, 1, 0, st>>>(ns);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  // Newton loop
  cudaGraphConditionalHandle h_loop, h_solve, h_ls;
  cudaGraph_t loop, solve, ls;
  cudaGraphNode_t n_loop, n_solve, n_ls;
  if ((s = graph_leaves(g, leaves))) return fail(s);
  {
    cudaError_t e = cudaGraphConditionalHandleCreate(&h_loop, g, 0, 0);
    if (e != cudaSuccess) return fail((set_error("condition handle: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
  }
  s = capture_into(g, leaves, st, [&]() -> int {
    nw_cond_kernel<<<1, 1, 0, st>>>(h_loop, ns, 1);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  {
    std::vector<cudaGraphNode_t> deps;
    if ((s = graph_leaves(g, deps))) return fail(s);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h_loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(&n_loop, g, deps.data(), deps.size(), &cp);
    if (e != cudaSuccess) return fail((set_error("while node: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
    loop = cp.conditional.phGraph_out[0];
  }
  // residual and convergence test; the if node's handle belongs to the loop body
  {
    cudaError_t e = cudaGraphConditionalHandleCreate(&h_solve, loop, 0, 0);
    if (e != cudaSuccess) return fail((set_error("condition handle: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
  }
  s = capture_into(loop, {}, st, [&]() -> int {
    int q;
    if ((q = nw_fint(S, U, S->nw_s_new.p, F, st))) return q;
    nw_residual_kernel<<<eg, 256, 0, st>>>(n, fx, F, nullptr, FEXT, R);
    if ((q = dot<double>(S, R, R, FIN_STORE, &ns->nrm_r, 0, st))) return q;
    if ((q = dot<double>(S, F, F, FIN_STORE, &ns->nrm_f, 0, st))) return q;
    if ((q = dot<double>(S, U, U, FIN_STORE, &ns->nrm_u, 0, st))) return q;
    nw_test_kernel<<<1, 1, 0, st>>>(ns, h_solve);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  {
    std::vector<cudaGraphNode_t> deps;
    if ((s = graph_leaves(loop, deps))) return fail(s);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h_solve;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(&n_solve, loop, deps.data(), deps.size(), &cp);
    if (e != cudaSuccess) return fail((set_error("if node: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
    solve = cp.conditional.phGraph_out[0];
  }
  // the correction: tangent and diagonal at (u, states of the last converged
  // increment), du from the mixed solve of -r
  s = capture_into(solve, {}, st, [&]() -> int {
    int q;
    if ((q = nw_tangent(S, U, st))) return q;
    if (j2 && (q = solver_refresh_diagonal(S, st))) return q;
    nw_neg_kernel<<<eg, 256, 0, st>>>(n, R, S->mx_b.p);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  if ((s = mixed_nodes(S, st, solve))) return fail(s);
  // line search (gfem/solvers.py:670-677): up to four trial points
  if ((s = graph_leaves(solve, leaves))) return fail(s);
  {
    cudaError_t e = cudaGraphConditionalHandleCreate(&h_ls, solve, 0, 0);
    if (e != cudaSuccess) return fail((set_error("condition handle: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
  }
  s = capture_into(solve, leaves, st, [&]() -> int {
    nw_lin_kernel<<<1, 1, 0, st>>>(ns, S->mx_scal.p);
    nw_ls_head_kernel<<<1, 1, 0, st>>>(ns, h_ls);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  {
    std::vector<cudaGraphNode_t> deps;
    if ((s = graph_leaves(solve, deps))) return fail(s);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h_ls;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(&n_ls, solve, deps.data(), deps.size(), &cp);
    if (e != cudaSuccess) return fail((set_error("while node: %s", cudaGetErrorString(e)), EXFEM_ERR_CUDA));
    ls = cp.conditional.phGraph_out[0];
  }
  s = capture_into(ls, {}, st, [&]() -> int {
    int q;
    nw_trial_kernel<<<eg, 256, 0, st>>>(n, U, S->mx_x.p, UT, ns);
    if ((q = nw_fint(S, UT, S->nw_s_trial.p, T, st))) return q;
    nw_residual_kernel<<<eg, 256, 0, st>>>(n, fx, T, nullptr, FEXT, DU);
    if ((q = dot<double>(S, DU, DU, FIN_STORE, &ns->nrm_r, 0, st))) return q;
    nw_ls_test_kernel<<<1, 1, 0, st>>>(ns, h_ls);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  s = capture_into(solve, {n_ls}, st, [&]() -> int {
    nw_step_kernel<<<eg, 256, 0, st>>>(n, U, S->mx_x.p, ns);
    int q;
    if ((q = dot<double>(S, S->mx_x.p, S->mx_x.p, FIN_STORE, &ns->nrm_du, 0, st))) return q;
    nw_dut_kernel<<<1, 1, 0, st>>>(ns);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  // loop condition after the (possibly skipped) correction
  s = capture_into(loop, {n_solve}, st, [&]() -> int {
    nw_cond_kernel<<<1, 1, 0, st>>>(h_loop, ns, 0);
    return EXFEM_OK;
  });
  if (s) return fail(s);
  *out = g;
  return EXFEM_OK;
}

int newton_increment(exfem_solver_s* S, const double* u, const double* const* s_old, const double* fext,
                     const double* start, double rtol, int max_iter, int line_search, double cg_tol, int cg_maxiter,
                     double* qref, double* u_out, double* const* s_out, int* corrections, int* converged,
                     double* hist, int* lin_stats, cudaStream_t st) {
  const int64_t n = S->n;
  const size_t nb = nw_nblock(S);
  const bool j2 = nw_any_j2(S);
  if (S->op != EXFEM_OP_MF_F32 || S->pc != EXFEM_PC_AMG || !S->amg) {
    set_error("the device Newton increment needs a solver with the FP32 matrix-free operator and an AMG hierarchy");
    return EXFEM_ERR_ARG;
  }
  if (max_iter < 1 || max_iter > 64) {
    set_error("max_iter must lie in 1..64, got %d", max_iter);
    return EXFEM_ERR_ARG;
  }
  for (size_t i = 0; i < nb; ++i)
    if (nw_j2(nw_block(S, i)) && (!s_old || !s_out || !s_old[i] || !s_out[i])) {
      set_error("block %zu is J2: its state_old and state_out are needed", i);
      return EXFEM_ERR_ARG;
    }
  const int64_t nst = nw_state_off(S, nb);
  int s;
  // everything the captured work touches exists before the capture
  if ((s = pcg_prepare<float>(S, st))) return s;
  if (!S->mx_b.p && ((s = S->mx_b.alloc(std::max<int64_t>(n, 1))) || (s = S->mx_x.alloc(std::max<int64_t>(n, 1))) ||
                     (s = S->mx_scal.alloc(1))))
    return s;
  if (!S->nw_scal.p) {
    DevBuf<double>* v[] = {&S->nw_u, &S->nw_ut, &S->nw_du, &S->nw_r, &S->nw_f, &S->nw_t, &S->nw_fext, &S->nw_start};
    for (auto* p : v)
      if ((s = p->alloc(std::max<int64_t>(n, 1)))) return s;
    if ((s = S->nw_scal.alloc(1))) return s;
  }
  if (nb > 1 && S->mb64.n < (size_t)n && (s = S->mb64.alloc(std::max<int64_t>(n, 1)))) return s;
  if (j2 && S->nw_s_old.n < (size_t)nst) {
    DevBuf<double>* v[] = {&S->nw_s_old, &S->nw_s_new, &S->nw_s_trial};
    for (auto* p : v)
      if ((s = p->alloc(nst))) return s;
  }
  for (size_t i = 0; i < nb; ++i) {
    exfem_block_s* b = nw_block(S, i);
    if (b->ys.n < (size_t)(b->ne * b->nnode * 3) && (s = b->ys.alloc(b->ne * b->nnode * 3))) return s;
  }
  if (S->gnewton && S->gnewton_gen != S->graph_gen) {
    cudaGraphExecDestroy(S->gnewton);
    S->gnewton = nullptr;
  }
  if (!S->gnewton) {
    // one eager FP64 product per block sets up the matrix-free operators' maps before the capture
    for (size_t i = 0; i < nb; ++i)
      if ((s = launch_mf_matvec<double>(nw_block(S, i), S->nw_u.p, S->nw_t.p, nullptr, st, false))) return s;
    CaptureScope cap;
    cudaGraph_t g = nullptr;
    if ((s = newton_graph_build(S, st, &g))) return s;
    cudaError_t e = cudaGraphInstantiate(&S->gnewton, g, 0);
    cudaGraphDestroy(g);
    EX_CUDA(e);
    S->gnewton_gen = S->graph_gen;
  }
  EX_CUDA(cudaMemcpyAsync(S->nw_u.p, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  EX_CUDA(cudaMemcpyAsync(S->nw_fext.p, fext, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  EX_CUDA(cudaMemcpyAsync(S->nw_start.p, start, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  for (size_t i = 0; i < nb; ++i) {
    const exfem_block_s* b = nw_block(S, i);
    if (nw_j2(b))
      EX_CUDA(cudaMemcpyAsync(S->nw_s_old.p + nw_state_off(S, i), s_old[i],
                              sizeof(double) * b->ne * b->ngp * b->nstate, cudaMemcpyDeviceToDevice, st));
  }
  nw_init_kernel<<<1, 1, 0, st>>>(S->nw_scal.p, rtol, max_iter, line_search, *qref);
  EX_CUDA(cudaMemsetAsync(&S->nw_scal.p->lin_its, 0, 2 * sizeof(int), st));
  mx_params_kernel<<<1, 1, 0, st>>>(S->mx_scal.p, cg_tol, S->mixed_delta, cg_maxiter, 1200);
  EX_LAUNCH_CHECK();
  EX_CUDA(cudaGraphLaunch(S->gnewton, st));
  EX_CUDA(cudaMemcpyAsync(u_out, S->nw_u.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  for (size_t i = 0; i < nb; ++i) {
    const exfem_block_s* b = nw_block(S, i);
    if (nw_j2(b))
      EX_CUDA(cudaMemcpyAsync(s_out[i], S->nw_s_new.p + nw_state_off(S, i),
                              sizeof(double) * b->ne * b->ngp * b->nstate, cudaMemcpyDeviceToDevice, st));
  }
  NewtonScal h;
  EX_CUDA(cudaMemcpyAsync(&h, S->nw_scal.p, sizeof(NewtonScal), cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaStreamSynchronize(st));
  // the graph changed the J2 blocks' tangent data: the next host solve refreshes its diagonal
  for (size_t i = 0; i < nb; ++i)
    if (nw_j2(nw_block(S, i))) ++nw_block(S, i)->tan_gen;
  *qref = h.qref;
  if (corrections) *corrections = h.corrections;
  if (converged) *converged = h.converged && !h.failed;
  if (hist)
    for (int k = 0; k < std::min(h.it, 64); ++k) hist[k] = h.hist[k];
  if (lin_stats) {
    lin_stats[0] = h.lin_its;
    lin_stats[1] = h.lin_nup;
  }
  return EXFEM_OK;
}

int solver_alloc(exfem_solver_s* S) {
  const int64_t n = S->n;
  int s;
  DevBuf<double>* v64[] = {&S->x64, &S->r64, &S->z64, &S->p64, &S->Ap64, &S->b64, &S->t64, &S->dinv64, &S->diag64};
  for (auto* v : v64)
    if ((s = v->alloc(std::max<int64_t>(n, 1)))) return s;
  DevBuf<float>* v32[] = {&S->x32, &S->r32, &S->z32, &S->p32, &S->Ap32, &S->b32, &S->t32, &S->dinv32};
  for (auto* v : v32)
    if ((s = v->alloc(std::max<int64_t>(n, 1)))) return s;
  if ((s = S->mb64.alloc(std::max<int64_t>(n, 1))) || (s = S->mb32.alloc(std::max<int64_t>(n, 1)))) return s;
  if (S->pc == EXFEM_PC_CHEBY) {
    DevBuf<double>* c64[] = {&S->cx64, &S->cr64, &S->cd64};
    DevBuf<float>* c32[] = {&S->cx32, &S->cr32, &S->cd32};
    for (auto* v : c64)
      if ((s = v->alloc(std::max<int64_t>(n, 1)))) return s;
    for (auto* v : c32)
      if ((s = v->alloc(std::max<int64_t>(n, 1)))) return s;
  }
  if ((s = S->partial.alloc(RED_MAX_BLOCKS))) return s;
  if ((s = S->dscr.alloc(4))) return s;
  if ((s = S->counter.alloc(1))) return s;
  EX_CUDA(cudaMemset(S->counter.p, 0, sizeof(unsigned)));
  if ((s = S->scal.alloc(1))) return s;
  EX_CUDA(outside_captures([&] { return cudaMallocHost(&S->h_scal, sizeof(PcgScal)); }));
  return EXFEM_OK;
}

}  // namespace exfem

exfem_solver_s::~exfem_solver_s() {
  for (auto& g : gexec)
    if (g) cudaGraphExecDestroy(g);
  if (gmixed) cudaGraphExecDestroy(gmixed);
  if (h_scal) exfem::outside_captures([&] { return cudaFreeHost(h_scal); });
}
