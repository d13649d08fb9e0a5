// Stored-Ke product for several right-hand sides on the CUDA cores, and the
// multi-load-case Jacobi PCG built on it.
//
// Y = opA(V) for nrhs = 1..16 right-hand sides at once, with the element matrices
// Ke (ne, nd, nd) stored in BF16, FP32 or FP64 (the output of
// exfem_element_stiffness) and V, Y (ndof, nrhs) with the right-hand sides fastest:
// FP32 for BF16 / FP32 Ke, FP64 for FP64 Ke.  This is the multi-load-case form of
// the reference's stored-Ke product (gfem/model.py:264-267 gather_matvec inside
// opA; gfem/optimize.py:116-143 vmaps it, with Jacobi PCG, over the load cases):
// one read of Ke serves every right-hand side.
//
// Per element the work is Ke (nd x nd) times U_e (nd x nrhs): 2 FMA per byte of
// BF16 Ke at four right-hand sides, far below what the tensor cores need to be the
// bound, so the contraction runs on the CUDA cores and the kernel is bound by
// streaming Ke.  Each warp takes elements in turn (grid-stride, two per pass for BF16
// and FP32 Ke): it gathers their nodal values (prescribed DOFs zeroed) into its
// shared-memory slice, lane i < nd multiplies row i of Ke — read with the widest
// aligned loads — by them (broadcast reads) and stores the nrhs results of its row;
// the element rows are then summed per node through the gather plan in the
// reference's order (gfem/model.py:241-267) and opA's prescribed rows applied
// (gather_multi_kernel).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "internal.h"
#include "solver.h"

namespace exfem {

namespace {

template <class KT>
__device__ __forceinline__ float to_acc(KT v, float) { return (float)v; }
template <>
__device__ __forceinline__ float to_acc<__nv_bfloat16>(__nv_bfloat16 v, float) { return __bfloat162float(v); }
__device__ __forceinline__ double to_acc(double v, double) { return v; }

// N values of T at p into registers with the widest loads the alignment A allows
template <class T, int N, int A>
__device__ __forceinline__ void ld_row(const T* __restrict__ p, T (&o)[N]) {
  constexpr int BYTES = N * (int)sizeof(T);
  if constexpr (A % 16 == 0 && BYTES % 16 == 0) {
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(p) + i);
      memcpy(reinterpret_cast<char*>(o) + 16 * i, &v, 16);
    }
  } else if constexpr (A % 8 == 0 && BYTES % 8 == 0) {
#pragma unroll
    for (int i = 0; i < BYTES / 8; ++i) {
      const uint2 v = __ldg(reinterpret_cast<const uint2*>(p) + i);
      memcpy(reinterpret_cast<char*>(o) + 8 * i, &v, 8);
    }
  } else if constexpr (A % 4 == 0 && BYTES % 4 == 0) {
#pragma unroll
    for (int i = 0; i < BYTES / 4; ++i) {
      const unsigned v = __ldg(reinterpret_cast<const unsigned*>(p) + i);
      memcpy(reinterpret_cast<char*>(o) + 4 * i, &v, 4);
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = p[i];
  }
}

// byte alignment of row i of a 256-byte aligned array of rows of N values of T
template <class T, int N>
constexpr int row_align() {
  return (N * (int)sizeof(T)) % 16 == 0 ? 16
         : (N * (int)sizeof(T)) % 8 == 0 ? 8
         : (N * (int)sizeof(T)) % 4 == 0 ? 4
                                         : 2;
}

constexpr int MW = 8;  // warps per CTA

}  // namespace

// ys[(e*nd + i)*NR + r] = sum_j Ke[e, i, j] * (free * V)[dof(e, j), r]
//
// Each warp takes EP elements per pass (EP = 2 for BF16 / FP32 Ke, 1 for FP64): the
// Ke rows of all of them are requested first, then their nodal values are gathered
// together (16-byte vectors of right-hand sides where nrhs allows), so that every
// lane has EP rows and EP gathers in flight at once.  FP32 products of an even
// number of right-hand sides issue packed FFMA2 (two right-hand sides per
// instruction, each rounded as its own FMA).
template <int ET, int NR, class KT, class VT>
__global__ void __launch_bounds__(32 * MW)
ebe_multi_kernel(int64_t ne, const int32_t* __restrict__ conn, const KT* __restrict__ Ke,
                 const VT* __restrict__ V, const uint8_t* __restrict__ fixed, VT* __restrict__ ys, int vecv) {
  constexpr int NN = ElemTraits<ET>::nnode, ND = 3 * NN;
  constexpr int EP = sizeof(KT) <= 4 ? 2 : 1;
  constexpr int W = (NR * sizeof(VT)) % 16 == 0 ? 16 / (int)sizeof(VT) : 1;  // values per gathered vector
  constexpr int NV = ND * NR / W;
  constexpr bool PAIRED = sizeof(VT) == 4 && NR % 2 == 0;
  __shared__ __align__(16) VT us[MW][EP][ND * NR];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * MW;
  for (int64_t e0 = (int64_t)blockIdx.x * MW + warp; e0 < ne; e0 += EP * stride) {
    KT row[EP][ND];
#pragma unroll
    for (int p = 0; p < EP; ++p) {
      const int64_t e = e0 + p * stride;
      if (e < ne && lane < ND) ld_row<KT, ND, row_align<KT, ND>()>(Ke + (e * ND + lane) * ND, row[p]);
    }
#pragma unroll
    for (int p = 0; p < EP; ++p) {
      const int64_t e = e0 + p * stride;
      if (e < ne) {
        for (int q = lane; q < NV; q += 32) {
          const int i = (q * W) / NR, r = (q * W) % NR;
          const int64_t d = 3 * (int64_t)__ldg(conn + e * NN + i / 3) + i % 3;
          const bool off = fixed && __ldg(fixed + d);
          if constexpr (W > 1) {
            uint4 v;
            if (vecv) {  // V 16-byte aligned (checked on the host)
              v = __ldg(reinterpret_cast<const uint4*>(V + d * NR + r));
            } else {
              VT t[W];
#pragma unroll
              for (int k = 0; k < W; ++k) t[k] = __ldg(V + d * NR + r + k);
              memcpy(&v, t, 16);
            }
            if (off) v = make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4*>(&us[warp][p][q * W]) = v;
          } else {
            const VT v = __ldg(V + d * NR + r);
            us[warp][p][q] = off ? VT(0) : v;
          }
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int p = 0; p < EP; ++p) {
      const int64_t e = e0 + p * stride;
      if (e < ne && lane < ND) {
        const VT* u = us[warp][p];
        VT y[NR];
        if constexpr (PAIRED) {
          float2 y2[NR / 2];
#pragma unroll
          for (int j = 0; j < NR / 2; ++j) y2[j] = make_float2(0.f, 0.f);
#pragma unroll
          for (int c = 0; c < ND; ++c) {
            const float k = to_acc(row[p][c], 0.f);
            const float2 k2 = make_float2(k, k);
            const float2* u2 = reinterpret_cast<const float2*>(u + c * NR);
#pragma unroll
            for (int j = 0; j < NR / 2; ++j) y2[j] = __ffma2_rn(k2, u2[j], y2[j]);
          }
#pragma unroll
          for (int j = 0; j < NR / 2; ++j) {
            y[2 * j] = y2[j].x;
            y[2 * j + 1] = y2[j].y;
          }
        } else {
#pragma unroll
          for (int r = 0; r < NR; ++r) y[r] = VT(0);
#pragma unroll
          for (int c = 0; c < ND; ++c) {
            const VT k = to_acc(row[p][c], VT(0));
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] += k * u[c * NR + r];
          }
        }
        VT* out = ys + (e * ND + lane) * NR;
        if constexpr ((NR * sizeof(VT)) % 16 == 0) {
#pragma unroll
          for (int r = 0; r < NR; r += 16 / (int)sizeof(VT)) {
            uint4 w;
            memcpy(&w, y + r, 16);
            *reinterpret_cast<uint4*>(out + r) = w;
          }
        } else {
#pragma unroll
          for (int r = 0; r < NR; ++r) out[r] = y[r];
        }
      }
    }
    __syncwarp();
  }
}

// Y[3n+c, r] = fixed ? V : sum over node n's gather-plan slots of the element rows,
// the slots in the plan's order; one thread per node and group of four right-hand
// sides (16-byte loads and stores) for FP32 with nrhs a multiple of 4 and aligned
// V, Y (vec4), else per node and right-hand side.  The plan entries are read four
// at a time and the rows of all four slots requested before any is added.
template <class VT>
__global__ void __launch_bounds__(256) gather_multi_kernel(int64_t nn, int vmax, int nnode, const int32_t* __restrict__ plan,
                                    int64_t sentinel, const VT* __restrict__ ys, const uint8_t* __restrict__ fixed,
                                    const VT* __restrict__ V, int nrhs, VT* __restrict__ Y, int vec4) {
  constexpr int K = 4;
  const int nd = 3 * nnode;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if constexpr (sizeof(VT) == 4) {
    if (vec4) {
      const int nq = nrhs >> 2;
      if (t >= nn * nq) return;
      const int64_t n = t / nq;
      const int r4 = (int)(t - n * nq) * 4;
      float4 s[3] = {make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0)};
      bool more = true;
      for (int k0 = 0; k0 < vmax && more; k0 += K) {
        int64_t sl[K];
#pragma unroll
        for (int u = 0; u < K; ++u) sl[u] = k0 + u < vmax ? (int64_t)plan[n * vmax + k0 + u] : sentinel;
        float4 w[K][3];
#pragma unroll
        for (int u = 0; u < K; ++u) {
          if (sl[u] != sentinel) {
            const int64_t e = sl[u] / nnode;
            const int a = (int)(sl[u] - e * nnode);
#pragma unroll
            for (int c = 0; c < 3; ++c)
              w[u][c] = *reinterpret_cast<const float4*>(ys + (e * nd + 3 * a + c) * nrhs + r4);
          }
        }
#pragma unroll
        for (int u = 0; u < K; ++u) {
          if (sl[u] == sentinel) {
            more = false;
            break;
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            s[c].x += w[u][c].x;
            s[c].y += w[u][c].y;
            s[c].z += w[u][c].z;
            s[c].w += w[u][c].w;
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t d = 3 * n + c;
        float4* out = reinterpret_cast<float4*>(Y + d * nrhs + r4);
        *out = (fixed && fixed[d]) ? *reinterpret_cast<const float4*>(V + d * nrhs + r4) : s[c];
      }
      return;
    }
  }
  if (t >= nn * nrhs) return;
  const int64_t n = t / nrhs;
  const int r = (int)(t - n * nrhs);
  VT s[3] = {VT(0), VT(0), VT(0)};
  bool more = true;
  for (int k0 = 0; k0 < vmax && more; k0 += K) {
    int64_t sl[K];
#pragma unroll
    for (int u = 0; u < K; ++u) sl[u] = k0 + u < vmax ? (int64_t)plan[n * vmax + k0 + u] : sentinel;
    VT w[K][3];
#pragma unroll
    for (int u = 0; u < K; ++u) {
      if (sl[u] != sentinel) {
        const int64_t e = sl[u] / nnode;
        const int a = (int)(sl[u] - e * nnode);
#pragma unroll
        for (int c = 0; c < 3; ++c) w[u][c] = ys[(e * nd + 3 * a + c) * nrhs + r];
      }
    }
#pragma unroll
    for (int u = 0; u < K; ++u) {
      if (sl[u] == sentinel) {
        more = false;
        break;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) s[c] += w[u][c];
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t d = 3 * n + c;
    Y[d * nrhs + r] = (fixed && fixed[d]) ? V[d * nrhs + r] : s[c];
  }
}

template <class VT>
int launch_gather_multi(exfem_block_s* b, const VT* ys, const VT* V, VT* Y, int nrhs, bool bc, cudaStream_t s) {
  // 16-byte accesses need nrhs a multiple of 4 and 16-byte aligned V and Y
  const int vec4 = sizeof(VT) == 4 && (nrhs & 3) == 0 && ((uintptr_t)V | (uintptr_t)Y) % 16 == 0;
  const int64_t work = vec4 ? b->nn * (nrhs / 4) : b->nn * nrhs;
  if (!work) return EXFEM_OK;
  gather_multi_kernel<VT><<<(unsigned)((work + 255) / 256), 256, 0, s>>>(
      b->nn, b->vmax, b->nnode, b->plan.p, b->ne * b->nnode, ys, bc ? b->fixed.p : nullptr, V, nrhs, Y, vec4);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template int launch_gather_multi<float>(exfem_block_s*, const float*, const float*, float*, int, bool, cudaStream_t);
template int launch_gather_multi<double>(exfem_block_s*, const double*, const double*, double*, int, bool,
                                         cudaStream_t);

namespace {

template <int ET, class KT, class VT>
int multi_launch(exfem_block_s* b, const KT* Ke, int nrhs, const VT* V, VT* ys, const uint8_t* fx, cudaStream_t s) {
  int dev, nsm;
  EX_CUDA(cudaGetDevice(&dev));
  EX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((b->ne + MW - 1) / MW, (int64_t)nsm * 8));
  const int vecv = (uintptr_t)V % 16 == 0;  // 16-byte gathers of V need it aligned
#define EXF_MULTI(NR)                                                                                   \
  case NR:                                                                                              \
    ebe_multi_kernel<ET, NR, KT, VT><<<grid, 32 * MW, 0, s>>>(b->ne, b->conn.p, Ke, V, fx, ys, vecv); \
    break;
  switch (nrhs) {
    EXF_MULTI(1) EXF_MULTI(2) EXF_MULTI(3) EXF_MULTI(4) EXF_MULTI(5) EXF_MULTI(6) EXF_MULTI(7) EXF_MULTI(8)
    EXF_MULTI(9) EXF_MULTI(10) EXF_MULTI(11) EXF_MULTI(12) EXF_MULTI(13) EXF_MULTI(14) EXF_MULTI(15)
    EXF_MULTI(16)
    default:
      set_error("the multi-right-hand-side stored-Ke product takes 1..16 right-hand sides, got %d", nrhs);
      return EXFEM_ERR_ARG;
  }
#undef EXF_MULTI
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template <class KT, class VT>
int multi_dispatch(exfem_block_s* b, const KT* Ke, int nrhs, const VT* V, VT* Y, bool bc, DevBuf<VT>& rows,
                   cudaStream_t s) {
  if (nrhs < 1 || nrhs > 16) {
    set_error("the multi-right-hand-side stored-Ke product takes 1..16 right-hand sides, got %d", nrhs);
    return EXFEM_ERR_ARG;
  }
  int st;
  const size_t need = (size_t)b->ne * b->nd * nrhs;
  if (rows.n < need && (st = rows.alloc(need))) return st;
  if (b->ne) {
    const uint8_t* fx = bc ? b->fixed.p : nullptr;
    st = b->etype == EXFEM_C3D8 ? multi_launch<EXFEM_C3D8>(b, Ke, nrhs, V, rows.p, fx, s)
                                : multi_launch<EXFEM_C3D10>(b, Ke, nrhs, V, rows.p, fx, s);
    if (st) return st;
  }
  return launch_gather_multi<VT>(b, rows.p, V, Y, nrhs, bc, s);
}

}  // namespace

int launch_ebe_matvec_multi(exfem_block_s* b, const void* Ke, int ke_dtype, int nrhs, const void* V, void* Y,
                            bool bc, cudaStream_t s) {
  switch (ke_dtype) {
    case EXFEM_BF16:
      return multi_dispatch<__nv_bfloat16, float>(b, (const __nv_bfloat16*)Ke, nrhs, (const float*)V, (float*)Y, bc,
                                                  b->ys_tc, s);
    case EXFEM_F32:
      return multi_dispatch<float, float>(b, (const float*)Ke, nrhs, (const float*)V, (float*)Y, bc, b->ys_tc, s);
    case EXFEM_F64:
      return multi_dispatch<double, double>(b, (const double*)Ke, nrhs, (const double*)V, (double*)Y, bc, b->ys_m64,
                                            s);
    default:
      set_error("unknown element-matrix type %d", ke_dtype);
      return EXFEM_ERR_ARG;
  }
}

// ---------------------------------------------------------------- multi-case Jacobi PCG
//
// gfem/optimize.py:116-143: linalg.pcg (gfem/linalg.py:21-47) vmapped over the load
// cases, with A(v) = free K (free v) + (1 - free) v, the right-hand sides free * f
// and the preconditioner inv = free ? 1 / (d != 0 ? d : 1) : 1 from the assembled
// diagonal d.  Here every case is a column of (ndof, NR) arrays and each iteration
// issues one stored-Ke product for all of them; every case keeps its own scalars and
// stops on its own test (r.r <= tol^2 max(b.b, 1e-300) or k >= maxiter), after
// which its column is left as it is — the iterates of a vmapped while loop, whose
// finished lanes stop changing.  Reductions: per-block partial sums of each column
// in a fixed order, then the last block sums the partials in block order
// (deterministic for a given grid).

namespace {

constexpr int MP_T = 256;           // threads per reduction block
constexpr int MP_MAX_BLOCKS = 592;  // 4 per SM

struct MultiScal {
  double rz[16], rr[16], bb[16], tol2[16], alpha[16], beta[16];
  int k[16], done[16], act[16];
  int maxiter, loops;
};

enum MpOp { MP_INIT = 0, MP_ALPHA, MP_XR, MP_RZ };

// per-column block sums of `acc`, then the final sums (in block order) handed to fin
template <int NR, class Fin>
__device__ __forceinline__ void mp_finish(double (&acc)[NR], double* partial, unsigned* counter, Fin fin) {
  __shared__ double sw[MP_T / 32][NR];
  __shared__ int last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sw[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < NR) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < MP_T / 32; ++w) t += sw[w][threadIdx.x];
    partial[(int64_t)blockIdx.x * NR + threadIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last) {
    __threadfence();
    if (threadIdx.x < NR) {
      double t = 0.0;
      for (unsigned b = 0; b < gridDim.x; ++b) t += ((volatile double*)partial)[(int64_t)b * NR + threadIdx.x];
      fin(threadIdx.x, t);
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
  }
}

// MP_INIT:  what 0: sums B.B; 1: R = B, P = dinv R, sums R.P; 2: sums R.R (and the
//           first stopping test)
// MP_ALPHA: sums P.Q -> alpha, act = !done
// MP_XR:    X += alpha P, R -= alpha Q (active columns); sums R.R
// MP_RZ:    sums R.(dinv R) -> beta, rz, k, done
template <int NR, int OP>
__global__ void __launch_bounds__(MP_T)
mp_reduce_kernel(int64_t n, const double* __restrict__ B, const double* __restrict__ dinv, double* __restrict__ X,
                 double* __restrict__ R, double* __restrict__ P, const double* __restrict__ Q, MultiScal* sc,
                 double* partial, unsigned* counter, int what) {
  double acc[NR];
  double al[NR];
  bool on[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    acc[j] = 0.0;
    al[j] = OP == MP_XR ? sc->alpha[j] : 0.0;
    on[j] = OP == MP_XR ? sc->act[j] != 0 : true;
  }
  for (int64_t i = blockIdx.x * (int64_t)MP_T + threadIdx.x; i < n; i += (int64_t)gridDim.x * MP_T) {
    const double di = dinv[i];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      const int64_t q = i * NR + j;
      if constexpr (OP == MP_INIT) {
        const double b = B[q];
        if (what == 1) {
          R[q] = b;
          P[q] = di * b;
          acc[j] += b * (di * b);
        } else {
          acc[j] += b * b;
        }
      } else if constexpr (OP == MP_ALPHA) {
        acc[j] += P[q] * Q[q];
      } else if constexpr (OP == MP_XR) {
        double r = R[q];
        if (on[j]) {
          X[q] += al[j] * P[q];
          r -= al[j] * Q[q];
          R[q] = r;
        }
        acc[j] += r * r;
      } else {
        const double r = R[q];
        acc[j] += r * (di * r);
      }
    }
  }
  mp_finish<NR>(acc, partial, counter, [&](int j, double t) {
    if constexpr (OP == MP_INIT) {
      if (what == 0) {
        sc->bb[j] = fmax(t, 1e-300);
      } else if (what == 1) {
        sc->rz[j] = t;
      } else {
        sc->rr[j] = t;
        sc->k[j] = 0;
        sc->done[j] = !(t > sc->tol2[j] && 0 < sc->maxiter);
      }
    } else if constexpr (OP == MP_ALPHA) {
      sc->act[j] = !sc->done[j];
      sc->alpha[j] = sc->act[j] ? sc->rz[j] / t : 0.0;
    } else if constexpr (OP == MP_XR) {
      if (sc->act[j]) sc->rr[j] = t;
    } else {
      if (sc->act[j]) {
        sc->beta[j] = t / sc->rz[j];
        sc->rz[j] = t;
        sc->k[j] += 1;
        sc->done[j] = !(sc->rr[j] > sc->tol2[j] && sc->k[j] < sc->maxiter);
      }
    }
  });
}

// P = dinv R + beta P on the columns active in this iteration
template <int NR>
__global__ void mp_update_p_kernel(int64_t n, const double* __restrict__ dinv, const double* __restrict__ R,
                                   double* __restrict__ P, const MultiScal* sc) {
  double be[NR];
  bool on[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    be[j] = sc->beta[j];
    on[j] = sc->act[j] != 0;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double di = dinv[i];
#pragma unroll
    for (int j = 0; j < NR; ++j)
      if (on[j]) P[i * NR + j] = di * R[i * NR + j] + be[j] * P[i * NR + j];
  }
}

__global__ void mp_scal_init_kernel(MultiScal* sc, int maxiter) {
  for (int j = 0; j < 16; ++j) {
    sc->rz[j] = sc->rr[j] = sc->bb[j] = sc->tol2[j] = sc->alpha[j] = sc->beta[j] = 0.0;
    sc->k[j] = 0;
    sc->done[j] = 1;
    sc->act[j] = 0;
  }
  sc->maxiter = maxiter;
  sc->loops = 0;
}

__global__ void mp_tol_kernel(MultiScal* sc, int nr, double tol) {
  for (int j = 0; j < nr; ++j) sc->tol2[j] = tol * tol * sc->bb[j];
}

// inverse diagonal of the reference's preconditioner: free ? 1 / (d != 0 ? d : 1) : 1
__global__ void mp_dinv_kernel(int64_t n, const double* __restrict__ d, const uint8_t* __restrict__ fixed,
                               double* __restrict__ dinv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool fr = !(fixed && fixed[i]);
    dinv[i] = fr ? 1.0 / (fabs(d[i]) > 0.0 ? d[i] : 1.0) : 1.0;
  }
}

// loop condition: another pass while some column is active, at most maxiter + 2 passes
__global__ void mp_cond_kernel(cudaGraphConditionalHandle h, MultiScal* sc, int nr, int head) {
  if (head) sc->loops = 0;
  else sc->loops += 1;
  bool any = false;
  for (int j = 0; j < nr; ++j) any = any || !sc->done[j];
  cudaGraphSetConditional(h, (any && (long long)sc->loops <= (long long)sc->maxiter + 1) ? 1u : 0u);
}

template <int NR>
int mp_iteration(exfem_block_s* b, const double* Ke, const double* dinv, double* X, double* R, double* P, double* Q,
                 MultiScal* sc, double* partial, unsigned* counter, unsigned grid, cudaStream_t s) {
  const int64_t n = b->ndof();
  int st;
  if ((st = launch_ebe_matvec_multi(b, Ke, EXFEM_F64, NR, P, Q, true, s))) return st;
  mp_reduce_kernel<NR, MP_ALPHA><<<grid, MP_T, 0, s>>>(n, nullptr, dinv, X, R, P, Q, sc, partial, counter, 0);
  mp_reduce_kernel<NR, MP_XR><<<grid, MP_T, 0, s>>>(n, nullptr, dinv, X, R, P, Q, sc, partial, counter, 0);
  mp_reduce_kernel<NR, MP_RZ><<<grid, MP_T, 0, s>>>(n, nullptr, dinv, X, R, P, Q, sc, partial, counter, 0);
  mp_update_p_kernel<NR><<<grid_for(n, 256), 256, 0, s>>>(n, dinv, R, P, sc);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template <int NR>
int mp_solve(exfem_block_s* b, const double* Ke, const double* Bm, double* X, double tol, int maxiter, int* iters,
             double* relres, cudaStream_t s) {
  const int64_t n = b->ndof();
  int st;
  // workspace: dinv (n), R, P, Q (n NR each), partial sums, scalars, counter
  // (every array starts on 256 bytes: the product reads P with 16-byte loads)
  DevBuf<double>& w = b->mp_work;
  const int64_t np = (n + 31) / 32 * 32;
  const size_t need = (size_t)np * (1 + 3 * NR) + (size_t)MP_MAX_BLOCKS * 16 + sizeof(MultiScal) / 8 + 64;
  if (w.n < need && (st = w.alloc(need))) return st;
  double* dinv = w.p;
  double* R = dinv + np;
  double* P = R + np * NR;
  double* Q = P + np * NR;
  double* partial = Q + np * NR;
  MultiScal* sc = reinterpret_cast<MultiScal*>(partial + MP_MAX_BLOCKS * 16);
  unsigned* counter = reinterpret_cast<unsigned*>(sc + 1);
  const unsigned grid =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + MP_T * 4 - 1) / (MP_T * 4), MP_MAX_BLOCKS));
  // element rows of the product, allocated before the capture below
  const size_t nrows = (size_t)b->ne * b->nd * NR;
  if (b->ys_m64.n < nrows && (st = b->ys_m64.alloc(nrows))) return st;
  EX_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
  if ((st = launch_ebe_diagonal(b, Ke, Q, s))) return st;
  mp_dinv_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, Q, b->fixed.p, dinv);
  mp_scal_init_kernel<<<1, 1, 0, s>>>(sc, maxiter);
  EX_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * n * NR, s));
  for (int what = 0; what < 3; ++what) {
    mp_reduce_kernel<NR, MP_INIT><<<grid, MP_T, 0, s>>>(n, Bm, dinv, X, R, P, nullptr, sc, partial, counter, what);
    if (what == 0) mp_tol_kernel<<<1, 1, 0, s>>>(sc, NR, tol);
  }
  EX_LAUNCH_CHECK();
  // the iteration loop as one graph: a conditional while node repeats one captured
  // iteration while some column is active
  cudaGraph_t g = nullptr;
  EX_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphExec_t ge = nullptr;
  auto fail = [&](cudaError_t e, const char* what) {
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    set_error("multi-case PCG graph: %s: %s", what, cudaGetErrorString(e));
    return EXFEM_ERR_CUDA;
  };
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
  if (e != cudaSuccess) return fail(e, "condition handle");
  int nr = NR, head = 1;
  void* args[] = {&h, &sc, &nr, &head};
  cudaKernelNodeParams kp = {};
  kp.func = (void*)mp_cond_kernel;
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
  {
    CaptureScope cap;
    if ((e = cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return fail(e, "capture of the loop body");
    int cs = mp_iteration<NR>(b, Ke, dinv, X, R, P, Q, sc, partial, counter, grid, s);
    if (!cs) {
      mp_cond_kernel<<<1, 1, 0, s>>>(h, sc, NR, 0);
      if (cudaGetLastError() != cudaSuccess) cs = EXFEM_ERR_CUDA;
    }
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s, &captured);
    if (cs) {
      cudaGraphDestroy(g);
      return cs;
    }
    if (e != cudaSuccess) return fail(e, "end of the body capture");
  }
  if ((e = cudaGraphInstantiate(&ge, g, 0)) != cudaSuccess) return fail(e, "instantiation");
  if ((e = cudaGraphLaunch(ge, s)) != cudaSuccess) return fail(e, "launch");
  MultiScal hs;
  e = cudaMemcpyAsync(&hs, sc, sizeof(MultiScal), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  EX_CUDA(e);
  bool all = true;
  for (int j = 0; j < NR; ++j) {
    const double rel = std::sqrt(hs.rr[j] / hs.bb[j]);
    if (iters) iters[j] = hs.k[j];
    if (relres) relres[j] = rel;
    all = all && std::isfinite(rel) && hs.rr[j] <= hs.tol2[j];
  }
  return all ? EXFEM_OK : EXFEM_NOT_CONVERGED;
}

}  // namespace

int multi_pcg(exfem_block_s* b, const double* Ke, int nrhs, const double* B, double* X, double tol, int maxiter,
              int* iters, double* relres, cudaStream_t s) {
  switch (nrhs) {
    case 1: return mp_solve<1>(b, Ke, B, X, tol, maxiter, iters, relres, s);
    case 2: return mp_solve<2>(b, Ke, B, X, tol, maxiter, iters, relres, s);
    case 3: return mp_solve<3>(b, Ke, B, X, tol, maxiter, iters, relres, s);
    case 4: return mp_solve<4>(b, Ke, B, X, tol, maxiter, iters, relres, s);
    case 8: return mp_solve<8>(b, Ke, B, X, tol, maxiter, iters, relres, s);
    case 16: return mp_solve<16>(b, Ke, B, X, tol, maxiter, iters, relres, s);
    default:
      set_error("the multi-case PCG takes 1, 2, 3, 4, 8 or 16 load cases per call, got %d", nrhs);
      return EXFEM_ERR_ARG;
  }
}

}  // namespace exfem
