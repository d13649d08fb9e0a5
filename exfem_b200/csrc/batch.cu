// Batched solves: many independent linear-elastic systems of uneven sizes in one
// set of launches (no counterpart in the reference, which solves one Model at a
// time; its closest relative is the vmapped multi-RHS Jacobi-PCG of
// gfem/optimize.py:116-143).
//
// The instances are concatenated into one "union" block (node and element
// offsets per instance, per-element Lame parameters), so one tile-queue launch of
// the matrix-free product serves all of them, and their smoothed-aggregation
// hierarchies are merged level by level into one block-diagonal union hierarchy
// (per-row Chebyshev coefficients, block-diagonal FP64 coarse solve).  The
// instances' DOFs are contiguous ranges [off[i], off[i+1]) of the union vectors.
// This file adds what must stay per instance: PCG step scalars, dot products and
// convergence flags (one CTA per instance for every segmented reduction, so the
// order is fixed and results do not depend on the other instances), and the FP64
// iterative refinement with per-instance scaling and stopping.  Converged
// instances are frozen: their updates are skipped while the others continue.
#include "solver.h"

namespace exfem {

constexpr int BT = 256;

struct BatchScal {  // device arrays, one entry per instance
  double *rz, *pAp, *rr, *bb, *tol2, *alpha, *beta, *sc, *bn, *rn, *tmp;
  int *k, *done, *odone, *iters;
  double* itol;  // inner tolerance of the current pass
  int* cap;      // inner iteration limit of the current pass
};

enum BFin { BF_BB = 0, BF_RZ0, BF_RR0, BF_ALPHA, BF_BETA, BF_STORE };

__device__ __forceinline__ double bwarp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sw[BT / 32];
  __shared__ double tot;
  v = bwarp_sum(v);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < BT / 32; ++w) t += sw[w];
    tot = t;
  }
  __syncthreads();
  return tot;
}

// per-instance dot product a.b over the instance's range, then the step update
template <class T>
__global__ void __launch_bounds__(BT)
bdot_kernel(const int64_t* __restrict__ off, const T* __restrict__ a, const T* __restrict__ b, BatchScal S,
            int F, double tol, int maxiter, int check_done) {
  const int i = blockIdx.x;
  if (check_done && S.done[i]) return;
  double acc = 0.0;
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) acc += (double)a[j] * (double)b[j];
  const double s = block_sum(acc);
  if (threadIdx.x) return;
  switch (F) {
    case BF_BB:
      S.bb[i] = s;
      S.tol2[i] = S.itol[i] * S.itol[i] * fmax(s, 1e-300);
      break;
    case BF_RZ0: S.rz[i] = s; break;
    case BF_RR0:
      S.rr[i] = s;
      S.k[i] = 0;
      S.done[i] = S.odone[i] || !(s > S.tol2[i] && 0 < S.cap[i]);
      break;
    case BF_ALPHA:
      S.pAp[i] = s;
      S.alpha[i] = S.rz[i] / s;
      break;
    case BF_BETA:
      S.beta[i] = s / S.rz[i];
      S.rz[i] = s;
      S.k[i] += 1;
      S.done[i] = !(S.rr[i] > S.tol2[i] && S.k[i] < S.cap[i]);
      break;
    default: S.tmp[i] = s;
  }
}

template <class T>
__global__ void __launch_bounds__(BT)
bupdate_xr_kernel(const int64_t* __restrict__ off, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                  const T* __restrict__ Ap, BatchScal S) {
  const int i = blockIdx.x;
  if (S.done[i]) return;
  const T alpha = (T)S.alpha[i];
  double acc = 0.0;
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) {
    x[j] += alpha * p[j];
    const T rj = r[j] - alpha * Ap[j];
    r[j] = rj;
    acc += (double)rj * (double)rj;
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) S.rr[i] = s;
}

template <class T>
__global__ void bupdate_p_kernel(const int64_t* __restrict__ off, T* __restrict__ p, const T* __restrict__ z,
                                 BatchScal S) {
  const int i = blockIdx.x;
  if (S.done[i]) return;
  const T beta = (T)S.beta[i];
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) p[j] = z[j] + beta * p[j];
}

__global__ void count_kernel(int n, const int* __restrict__ flags, int* __restrict__ out) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) c += flags[i] ? 1 : 0;
  atomicAdd(&cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = cnt;
}

// r32 = r64 / sc_i (instances already converged get zeros), sc_i = ||r64_i|| or 1
__global__ void bscale_kernel(const int64_t* __restrict__ off, const double* __restrict__ r64, float* __restrict__ r32,
                              BatchScal S) {
  const int i = blockIdx.x;
  const double n = sqrt(S.tmp[i]);
  const double sc = n > 0.0 ? n : 1.0, isc = 1.0 / sc;
  if (threadIdx.x == 0) S.sc[i] = sc;
  const bool od = S.odone[i];
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) r32[j] = od ? 0.0f : (float)(r64[j] * isc);
}

__global__ void baccum_kernel(const int64_t* __restrict__ off, double* __restrict__ x, const float* __restrict__ d,
                              BatchScal S) {
  const int i = blockIdx.x;
  if (S.odone[i]) return;
  const double sc = S.sc[i];
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) x[j] += (double)d[j] * sc;
  if (threadIdx.x == 0) S.iters[i] += S.k[i];
}

// r = b - t; per-instance residual norm and outer convergence test
__global__ void bresidual_kernel(const int64_t* __restrict__ off, const double* __restrict__ b,
                                 const double* __restrict__ t, double* __restrict__ r, BatchScal S, double tol) {
  const int i = blockIdx.x;
  double acc = 0.0;
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) {
    const double rj = b[j] - t[j];
    r[j] = rj;
    acc += rj * rj;
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) {
    const double rn = sqrt(s);
    S.rn[i] = rn;
    if (!S.odone[i] && rn <= tol * S.bn[i]) S.odone[i] = 1;
  }
}

__global__ void bnorm_init_kernel(const int64_t* __restrict__ off, const double* __restrict__ b, BatchScal S,
                                  double inner_tol, int maxiter) {
  const int i = blockIdx.x;
  double acc = 0.0;
  for (int64_t j = off[i] + threadIdx.x; j < off[i + 1]; j += BT) acc += b[j] * b[j];
  const double s = block_sum(acc);
  if (threadIdx.x == 0) {
    const double n = sqrt(s);
    S.bn[i] = n > 0.0 ? n : 1.0;
    S.rn[i] = n;
    S.tmp[i] = s;
    S.odone[i] = 0;
    S.iters[i] = 0;
    S.itol[i] = inner_tol;
    S.cap[i] = maxiter;
  }
}

// after the first pass, per instance (the rule of the single-solve restarted
// refinement): later passes stop at 4x the first pass's iterations
__global__ void badapt_kernel(int m, BatchScal S, double inner_tol, int maxiter) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  S.cap[i] = min(maxiter, max(4 * S.k[i], 32));
}

}  // namespace exfem

struct exfem_batch_s {
  exfem_block_s* blk = nullptr;
  exfem_amg_s* amg = nullptr;
  int ninst = 0;
  int64_t n = 0;
  exfem::DevBuf<int64_t> off;
  exfem::DevBuf<double> sd;  // scalars: 11 double arrays
  exfem::DevBuf<int> si;     // 4 int arrays + counter
  exfem::DevBuf<double> x64, r64, t64, diag64, dinv64;
  exfem::DevBuf<float> x32, r32, z32, p32, Ap32, t32, dinv32;
  int* h_cnt = nullptr;
  cudaGraphExec_t gexec = nullptr;
  uint64_t graph_bc_gen = ~0ull;
  int chunk = 8;
  exfem::BatchScal S{};
  ~exfem_batch_s() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (h_cnt) exfem::outside_captures([&] { return cudaFreeHost(h_cnt); });
  }
};

namespace exfem {

int launch_mf_diagonal(exfem_block_s* b, double* diag, cudaStream_t s);

template <class T>
static int batch_op(void* ctx, const T* x, T* y, const int* skip, cudaStream_t s) {
  return launch_mf_matvec<T>((exfem_block_s*)ctx, x, y, skip, s);
}

__global__ void bdinv_kernel(int64_t n, const double* __restrict__ d, const uint8_t* __restrict__ fixed,
                             double* __restrict__ d64, float* __restrict__ d32) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool fx = fixed && fixed[i];
    const double v = fx ? 1.0 : (fabs(d[i]) > 0.0 ? 1.0 / d[i] : 1.0);
    d64[i] = v;
    d32[i] = (float)v;
  }
}

__global__ void bmask_kernel(int64_t n, const uint8_t* __restrict__ fixed, const float* __restrict__ v,
                             float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = fixed[i] ? 0.0f : v[i];
}

__global__ void bpcout_kernel(int64_t n, const uint8_t* __restrict__ fixed, const float* __restrict__ r,
                              float* __restrict__ z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (fixed[i]) z[i] = r[i];
}

static int batch_precond(exfem_batch_s* B, const float* r, float* z, cudaStream_t st) {
  const uint8_t* fixed = B->blk->fixed.p;
  const float* rin = r;
  const unsigned eg = grid_for(B->n, 256);
  if (fixed) {
    bmask_kernel<<<eg, 256, 0, st>>>(B->n, fixed, r, B->t32.p);
    EX_LAUNCH_CHECK();
    rin = B->t32.p;
  }
  Level0Op<float> op0;
  op0.apply = &batch_op<float>;
  op0.ctx = B->blk;
  op0.dinv = B->dinv32.p;
  int s;
  if ((s = amg_vcycle<float>(B->amg, rin, z, &op0, nullptr, st))) return s;
  if (fixed) {
    bpcout_kernel<<<eg, 256, 0, st>>>(B->n, fixed, r, z);
    EX_LAUNCH_CHECK();
  }
  return EXFEM_OK;
}

static int batch_iteration(exfem_batch_s* B, int maxiter, cudaStream_t st) {
  const unsigned g = (unsigned)B->ninst;
  int s;
  if ((s = launch_mf_matvec<float>(B->blk, B->p32.p, B->Ap32.p, nullptr, st))) return s;
  bdot_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->p32.p, B->Ap32.p, B->S, BF_ALPHA, 0.0, maxiter, 1);
  bupdate_xr_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->x32.p, B->r32.p, B->p32.p, B->Ap32.p, B->S);
  if ((s = batch_precond(B, B->r32.p, B->z32.p, st))) return s;
  bdot_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->r32.p, B->z32.p, B->S, BF_BETA, 0.0, maxiter, 1);
  bupdate_p_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->p32.p, B->z32.p, B->S);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

static int batch_count(exfem_batch_s* B, const int* flags, int* out, cudaStream_t st) {
  count_kernel<<<1, 256, 0, st>>>(B->ninst, flags, B->si.p + 5 * B->ninst);
  EX_LAUNCH_CHECK();
  EX_CUDA(cudaMemcpyAsync(B->h_cnt, B->si.p + 5 * B->ninst, sizeof(int), cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaStreamSynchronize(st));
  *out = *B->h_cnt;
  return EXFEM_OK;
}

// inner FP32 PCG on r32 (already scaled) for all instances not yet converged
static int batch_pcg32(exfem_batch_s* B, double tol, int maxiter, cudaStream_t st) {
  const unsigned g = (unsigned)B->ninst;
  const int64_t n = B->n;
  int s;
  EX_CUDA(cudaMemsetAsync(B->x32.p, 0, sizeof(float) * n, st));
  bdot_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->r32.p, B->r32.p, B->S, BF_BB, tol, maxiter, 0);
  if ((s = batch_precond(B, B->r32.p, B->z32.p, st))) return s;
  EX_CUDA(cudaMemcpyAsync(B->p32.p, B->z32.p, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
  bdot_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->r32.p, B->z32.p, B->S, BF_RZ0, tol, maxiter, 0);
  bdot_kernel<float><<<g, BT, 0, st>>>(B->off.p, B->r32.p, B->r32.p, B->S, BF_RR0, tol, maxiter, 0);
  EX_LAUNCH_CHECK();
  if (B->graph_bc_gen != B->blk->bc_gen && B->gexec) {
    cudaGraphExecDestroy(B->gexec);
    B->gexec = nullptr;
  }
  if (!B->gexec) {
    CaptureScope cap;
    cudaGraph_t gr;
    EX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int cs = EXFEM_OK;
    for (int i = 0; i < B->chunk && !cs; ++i) cs = batch_iteration(B, maxiter, st);
    cudaError_t ce = cudaStreamEndCapture(st, &gr);
    if (cs) { if (ce == cudaSuccess) cudaGraphDestroy(gr); return cs; }
    EX_CUDA(ce);
    ce = cudaGraphInstantiate(&B->gexec, gr, 0);
    cudaGraphDestroy(gr);
    EX_CUDA(ce);
    B->graph_bc_gen = B->blk->bc_gen;
  }
  const int max_chunks = maxiter / B->chunk + 2;
  for (int c = 0; c < max_chunks; ++c) {
    int ndone;
    if ((s = batch_count(B, B->S.done, &ndone, st))) return s;
    if (ndone == B->ninst) break;
    EX_CUDA(cudaGraphLaunch(B->gexec, st));
  }
  return EXFEM_OK;
}

int batch_solve(exfem_batch_s* B, const double* b, double* x, double tol, double inner_tol, int max_pass, int maxiter,
                int* iters, int* passes, double* relres, cudaStream_t st) {
  const unsigned g = (unsigned)B->ninst;
  const int64_t n = B->n;
  int s;
  // inverse diagonal of the current operator for the level-0 smoother
  if ((s = launch_mf_diagonal(B->blk, B->diag64.p, st))) return s;
  bdinv_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, B->diag64.p, B->blk->fixed.p, B->dinv64.p, B->dinv32.p);
  EX_LAUNCH_CHECK();
  if ((s = amg_prepare(B->amg, EXFEM_F32))) return s;
  EX_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
  EX_CUDA(cudaMemcpyAsync(B->r64.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  bnorm_init_kernel<<<g, BT, 0, st>>>(B->off.p, b, B->S, inner_tol, maxiter);
  EX_LAUNCH_CHECK();
  int p = 0;
  for (p = 0; p < max_pass; ++p) {
    bscale_kernel<<<g, BT, 0, st>>>(B->off.p, B->r64.p, B->r32.p, B->S);
    EX_LAUNCH_CHECK();
    if ((s = batch_pcg32(B, inner_tol, maxiter, st))) return s;
    baccum_kernel<<<g, BT, 0, st>>>(B->off.p, x, B->x32.p, B->S);
    EX_LAUNCH_CHECK();
    if ((s = launch_mf_matvec<double>(B->blk, x, B->t64.p, nullptr, st))) return s;
    bresidual_kernel<<<g, BT, 0, st>>>(B->off.p, b, B->t64.p, B->r64.p, B->S, tol);
    EX_LAUNCH_CHECK();
    if (p == 0) {
      badapt_kernel<<<(B->ninst + 255) / 256, 256, 0, st>>>(B->ninst, B->S, inner_tol, maxiter);
      EX_LAUNCH_CHECK();
    }
    // next pass scales by the new residual norms
    bdot_kernel<double><<<g, BT, 0, st>>>(B->off.p, B->r64.p, B->r64.p, B->S, BF_STORE, 0.0, 0, 0);
    EX_LAUNCH_CHECK();
    int nod;
    if ((s = batch_count(B, B->S.odone, &nod, st))) return s;
    if (nod == B->ninst) { ++p; break; }
  }
  std::vector<double> rn(B->ninst), bn(B->ninst);
  std::vector<int> it(B->ninst), od(B->ninst);
  EX_CUDA(cudaMemcpyAsync(rn.data(), B->S.rn, sizeof(double) * B->ninst, cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaMemcpyAsync(bn.data(), B->S.bn, sizeof(double) * B->ninst, cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaMemcpyAsync(it.data(), B->S.iters, sizeof(int) * B->ninst, cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaMemcpyAsync(od.data(), B->S.odone, sizeof(int) * B->ninst, cudaMemcpyDeviceToHost, st));
  EX_CUDA(cudaStreamSynchronize(st));
  bool all = true;
  for (int i = 0; i < B->ninst; ++i) {
    if (iters) iters[i] = it[i];
    if (relres) relres[i] = rn[i] / bn[i];
    all = all && od[i];
  }
  if (passes) *passes = p;
  return all ? EXFEM_OK : EXFEM_NOT_CONVERGED;
}

int batch_alloc(exfem_batch_s* B, const int64_t* off_host) {
  int s;
  const int m = B->ninst;
  if ((s = B->off.upload(off_host, m + 1))) return s;
  if ((s = B->sd.alloc((size_t)12 * m))) return s;
  if ((s = B->si.alloc((size_t)5 * m + 1))) return s;
  EX_CUDA(cudaMemset(B->sd.p, 0, B->sd.bytes()));
  EX_CUDA(cudaMemset(B->si.p, 0, B->si.bytes()));
  double* d = B->sd.p;
  B->S = BatchScal{d, d + m, d + 2 * m, d + 3 * m, d + 4 * m, d + 5 * m, d + 6 * m, d + 7 * m, d + 8 * m, d + 9 * m,
                   d + 10 * m, B->si.p, B->si.p + m, B->si.p + 2 * m, B->si.p + 3 * m, d + 11 * m,
                   B->si.p + 4 * m};
  DevBuf<double>* v64[] = {&B->x64, &B->r64, &B->t64, &B->diag64, &B->dinv64};
  for (auto* v : v64)
    if ((s = v->alloc(std::max<int64_t>(B->n, 1)))) return s;
  DevBuf<float>* v32[] = {&B->x32, &B->r32, &B->z32, &B->p32, &B->Ap32, &B->t32, &B->dinv32};
  for (auto* v : v32)
    if ((s = v->alloc(std::max<int64_t>(B->n, 1)))) return s;
  EX_CUDA(outside_captures([&] { return cudaMallocHost(&B->h_cnt, sizeof(int)); }));
  return EXFEM_OK;
}

}  // namespace exfem

using namespace exfem;

extern "C" {

int exfem_batch_create(exfem_block blk, exfem_amg amg, int ninst, const int64_t* dof_offsets, exfem_batch* out) try {
  EX_ARG(blk && amg && dof_offsets && out, "NULL argument");
  *out = nullptr;
  EX_ARG(ninst >= 1, "need at least one instance");
  EX_ARG(blk->mat.kind == EXFEM_LINEAR_ELASTIC, "batched solves cover linear-elastic blocks");
  EX_ARG(dof_offsets[0] == 0 && dof_offsets[ninst] == blk->ndof(), "DOF offsets must cover the union block");
  for (int i = 0; i < ninst; ++i) EX_ARG(dof_offsets[i + 1] > dof_offsets[i], "empty instance %d", i);
  EX_ARG(amg->levels.empty() || amg->levels[0]->n == blk->ndof(), "hierarchy does not match the union block");
  auto B = std::make_unique<exfem_batch_s>();
  B->blk = blk;
  B->amg = amg;
  B->ninst = ninst;
  B->n = blk->ndof();
  int s;
  if ((s = batch_alloc(B.get(), dof_offsets))) return s;
  *out = B.release();
  return EXFEM_OK;
} catch (...) {
  return host_exception();
}

int exfem_batch_destroy(exfem_batch b) {
  delete b;
  return EXFEM_OK;
}

int exfem_batch_solve(exfem_batch b, const double* rhs, double* x, double tol, double inner_tol, int max_pass,
                      int maxiter, int* iters, int* passes, double* relres, void* stream) try {
  EX_ARG(b && rhs && x, "NULL argument");
  EX_ARG(tol >= 0 && inner_tol > 0 && max_pass >= 1 && maxiter >= 1, "invalid refinement parameters");
  cudaStream_t user = (cudaStream_t)stream, work = user;
  cudaEvent_t ev = nullptr;
  const bool own = (user == nullptr || user == cudaStreamLegacy);
  if (own) {  // graphs cannot be captured on the legacy default stream
    EX_CUDA(cudaStreamCreateWithFlags(&work, cudaStreamNonBlocking));
    EX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    EX_CUDA(cudaEventRecord(ev, user));
    EX_CUDA(cudaStreamWaitEvent(work, ev, 0));
  }
  const int s = batch_solve(b, rhs, x, tol, inner_tol, max_pass, maxiter, iters, passes, relres, work);
  if (own) {
    cudaEventRecord(ev, work);
    cudaStreamWaitEvent(user, ev, 0);
    cudaEventDestroy(ev);
    cudaStreamDestroy(work);
  }
  return s;
} catch (...) {
  return host_exception();
}

}  // extern "C"
