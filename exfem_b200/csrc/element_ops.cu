// FP64 element kernels: internal force with the J2 return map (and the
// per-Gauss-point consistent-tangent data it produces), element tangents Ke,
// element-averaged stresses, deterministic assembly (gather plan or colour
// scatter), and the stored-Ke element-by-element product.
//
// Reference: gfem/model.py:35-111 (geom, B-bar defgrad, force, stiff),
// 129-137 (cauchy), 162-173 (ops_matvec / ops_diagonal), 241-267 (gather plan
// assembly), 466-486 (Model.internal_force / element_stiffness).
#include <cuda_bf16.h>

#include "internal.h"

namespace exfem {

// dN_b / dxi_i of the trilinear hexahedron at corner-ordered Gauss point g
__device__ __forceinline__ double hex_dN(int g, int b, int i) {
  const double p0 = HEX_GQ * hex_sign(g, 0), p1 = HEX_GQ * hex_sign(g, 1), p2 = HEX_GQ * hex_sign(g, 2);
  const double s0 = hex_sign(b, 0), s1 = hex_sign(b, 1), s2 = hex_sign(b, 2);
  const double f0 = 1.0 + s0 * p0, f1 = 1.0 + s1 * p1, f2 = 1.0 + s2 * p2;
  return i == 0 ? 0.125 * s0 * f1 * f2 : (i == 1 ? 0.125 * f0 * s1 * f2 : 0.125 * f0 * f1 * s2);
}

template <class T>
__device__ __forceinline__ void matmul3(const T (&A)[9], const T (&B)[9], T (&C)[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// Q = C * iJ^T for symmetric C given as 6 components, scaled by w
template <class T>
__device__ __forceinline__ void cotangent(const T (&c)[6], T w, const T (&iJ)[9], T (&Q)[9]) {
  const T r[3][3] = {{c[0], c[3], c[5]}, {c[3], c[1], c[4]}, {c[5], c[4], c[2]}};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      Q[3 * i + k] = w * (r[i][0] * iJ[3 * k] + r[i][1] * iJ[3 * k + 1] + r[i][2] * iJ[3 * k + 2]);
}

// ---------------------------------------------------------------- force / tangent / stress
template <int ET, int MODE>
__global__ void __launch_bounds__(128)
force_kernel(int64_t ne, const double* __restrict__ X, const int32_t* __restrict__ conn,
             const double* __restrict__ u, const double* __restrict__ scale,
             const double* __restrict__ st_old, double* __restrict__ st_new, double* __restrict__ fe,
             double* __restrict__ tan64, float* __restrict__ tan32, double* __restrict__ S,
             double* __restrict__ mises, double* __restrict__ peeq, const MatDev mat,
             const double* __restrict__ lam_e, const double* __restrict__ mu_e,
             const int32_t* __restrict__ tpos, int tile) {
  using Tr = ElemTraits<ET>;
  constexpr int NN = Tr::nnode, NG = Tr::ngp;
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  // per-element Lame parameters (linear elasticity) override the material's
  const double lam_k = lam_e ? lam_e[e] : mat.lam, mu_k = lam_e ? mu_e[e] : mat.mu;
  const int ns = mat.kind == EXFEM_J2 ? 19 : 1;
  const double sc = (MODE != FORCE_STRESS && scale) ? scale[e] : 1.0;
  int nod[NN];
#pragma unroll
  for (int a = 0; a < NN; ++a) nod[a] = conn[e * NN + a];
  double Sacc[6] = {0, 0, 0, 0, 0, 0}, vsum = 0.0, pacc = 0.0;
  const double* st_e = st_old ? st_old + e * (int64_t)NG * ns : nullptr;
  double* sn_e = (MODE == FORCE_FULL && st_new) ? st_new + e * (int64_t)NG * ns : nullptr;
  double zero_state[19];
#pragma unroll
  for (int k = 0; k < 19; ++k) zero_state[k] = 0.0;

  if constexpr (ET == EXFEM_C3D8) {
    double xa[8][3], ua[8][3], cm[7][3], um[7][3];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xa[a][c] = X[3 * (int64_t)nod[a] + c];
        ua[a][c] = u[3 * (int64_t)nod[a] + c];
      }
    hex_to_modal(xa, cm);
    hex_to_modal(ua, um);
    double J0[9], iJ0[9], G0[9], H0[9];
#pragma unroll
    for (int n = 0; n < 3; ++n)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        J0[3 * n + i] = cm[i][n];
        G0[3 * n + i] = um[i][n];
      }
    inv3(J0, iJ0);
    matmul3(G0, iJ0, H0);
    const double tr0 = H0[0] + H0[4] + H0[8];
    double Fm[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k) Fm[k][0] = Fm[k][1] = Fm[k][2] = 0.0;
    double tacc = 0.0;
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
      const double x = HEX_GQ * hex_sign(g, 0), y = HEX_GQ * hex_sign(g, 1), z = HEX_GQ * hex_sign(g, 2);
      double J[9], iJ[9], G[9], H[9];
      hex_modal_grad(cm, x, y, z, J);
      const double detJ = inv3(J, iJ);
      hex_modal_grad(um, x, y, z, G);
      matmul3(G, iJ, H);
      const double bb = (tr0 - (H[0] + H[4] + H[8])) / 3.0;
      H[0] += bb;
      H[4] += bb;
      H[8] += bb;
      double sig[6], tn[8];
      const double* st = st_e ? st_e + g * ns : zero_state;
      material_stress(mat, lam_k, mu_k, H, st, sn_e ? sn_e + g * ns : nullptr, sig, tn);
      if (MODE != FORCE_STRESS) {
        if (tan64)
#pragma unroll
          for (int k = 0; k < 8; ++k) tan64[tile_index(tpos[e], g * 8 + k, NG * 8, tile)] = tn[k];
        if (tan32)
#pragma unroll
          for (int k = 0; k < 8; ++k) tan32[tile_index(tpos[e], g * 8 + k, NG * 8, tile)] = (float)tn[k];
      }
      if (MODE == FORCE_FULL) {
        const double vol = detJ * sc;
        const double t = vol * (sig[0] + sig[1] + sig[2]) / 3.0;
        tacc += t;
        double cdev[6] = {vol * sig[0] - t, vol * sig[1] - t, vol * sig[2] - t,
                          vol * sig[3], vol * sig[4], vol * sig[5]};
        double Q[9];
        cotangent(cdev, 1.0, iJ, Q);
        hex_modal_grad_adj(Q, x, y, z, Fm);
      } else if (MODE == FORCE_STRESS) {
        double snew[19];
        material_stress(mat, lam_k, mu_k, H, st, snew, sig, tn);
#pragma unroll
        for (int k = 0; k < 6; ++k) Sacc[k] += detJ * sig[k];
        vsum += detJ;
        if (mat.kind == EXFEM_J2) pacc += detJ * snew[9];
      }
    }
    if (MODE == FORCE_FULL && fe) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) Fm[i][c] += tacc * iJ0[3 * i + c];
      double f[8][3];
      hex_from_modal(Fm, f);
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) fe[(e * 8 + a) * 3 + c] = f[a][c];
    }
  } else {
    double f[10][3];
#pragma unroll
    for (int a = 0; a < 10; ++a) f[a][0] = f[a][1] = f[a][2] = 0.0;
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
      double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, iJ[9], H[9];
#pragma unroll
      for (int a = 0; a < 10; ++a) {
        const int64_t n3 = 3 * (int64_t)nod[a];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          double dn = 0.0;
          // compile-time table lookup (g is a runtime loop index)
          switch (g) {
            case 0: dn = tet10_dN(0, a, i); break;
            case 1: dn = tet10_dN(1, a, i); break;
            case 2: dn = tet10_dN(2, a, i); break;
            default: dn = tet10_dN(3, a, i); break;
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            J[3 * c + i] += X[n3 + c] * dn;
            G[3 * c + i] += u[n3 + c] * dn;
          }
        }
      }
      const double detJ = inv3(J, iJ);
      matmul3(G, iJ, H);
      double sig[6], tn[8];
      const double* st = st_e ? st_e + g * ns : zero_state;
      material_stress(mat, lam_k, mu_k, H, st, sn_e ? sn_e + g * ns : nullptr, sig, tn);
      if (MODE != FORCE_STRESS) {
        if (tan64)
#pragma unroll
          for (int k = 0; k < 8; ++k) tan64[tile_index(tpos[e], g * 8 + k, NG * 8, tile)] = tn[k];
        if (tan32)
#pragma unroll
          for (int k = 0; k < 8; ++k) tan32[tile_index(tpos[e], g * 8 + k, NG * 8, tile)] = (float)tn[k];
      }
      if (MODE == FORCE_FULL) {
        const double vol = detJ / 24.0 * sc;
        double Q[9];
        cotangent(sig, vol, iJ, Q);
#pragma unroll
        for (int a = 0; a < 10; ++a)
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            double dn = 0.0;
            switch (g) {
              case 0: dn = tet10_dN(0, a, i); break;
              case 1: dn = tet10_dN(1, a, i); break;
              case 2: dn = tet10_dN(2, a, i); break;
              default: dn = tet10_dN(3, a, i); break;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) f[a][c] += Q[3 * c + i] * dn;
          }
      } else if (MODE == FORCE_STRESS) {
        double snew[19];
        material_stress(mat, lam_k, mu_k, H, st, snew, sig, tn);
        const double w = detJ / 24.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) Sacc[k] += w * sig[k];
        vsum += w;
        if (mat.kind == EXFEM_J2) pacc += w * snew[9];
      }
    }
    if (MODE == FORCE_FULL && fe) {
#pragma unroll
      for (int a = 0; a < 10; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) fe[(e * 10 + a) * 3 + c] = f[a][c];
    }
  }
  if (MODE == FORCE_STRESS) {
    double s[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = Sacc[k] / vsum;
    if (S) {
      double* o = S + e * 9;
      o[0] = s[0]; o[1] = s[3]; o[2] = s[5];
      o[3] = s[3]; o[4] = s[1]; o[5] = s[4];
      o[6] = s[5]; o[7] = s[4]; o[8] = s[2];
    }
    const double m3 = (s[0] + s[1] + s[2]) / 3.0;
    const double d0 = s[0] - m3, d1 = s[1] - m3, d2 = s[2] - m3;
    if (mises)
      mises[e] = sqrt(1.5 * (d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5])));
    if (peeq) peeq[e] = pacc / vsum;
  }
}

template <int ET, int MODE>
static int force_dispatch(exfem_block_s* b, const double* u, const double* st_old, double* st_new,
                          double* fe, double* S, double* mises, double* peeq, cudaStream_t s) {
  const int threads = 128;
  const unsigned grid = (unsigned)((b->ne + threads - 1) / threads);
  const bool j2 = b->mat.kind == EXFEM_J2;
  double* t64 = (MODE != FORCE_STRESS && j2) ? b->tan64.p : nullptr;
  float* t32 = (MODE != FORCE_STRESS && j2) ? b->tan32.p : nullptr;
  force_kernel<ET, MODE><<<grid, threads, 0, s>>>(b->ne, b->X.p, b->conn.p, u, b->scale.p, st_old,
                                                  st_new, fe, t64, t32, S, mises, peeq, b->mat, b->lam_e.p,
                                                  b->mu_e.p, b->tpos.p, b->tile);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

int launch_force(exfem_block_s* b, int mode, const double* u, const double* st_old, double* st_new,
                 double* fe, double* S, double* mises, double* peeq, cudaStream_t s) {
  if (b->ne == 0) return EXFEM_OK;
#define EXF_CASE(ET)                                                                           \
  if (b->etype == ET) {                                                                        \
    if (mode == FORCE_FULL) return force_dispatch<ET, FORCE_FULL>(b, u, st_old, st_new, fe, S, mises, peeq, s); \
    if (mode == FORCE_TANGENT) return force_dispatch<ET, FORCE_TANGENT>(b, u, st_old, st_new, fe, S, mises, peeq, s); \
    return force_dispatch<ET, FORCE_STRESS>(b, u, st_old, st_new, fe, S, mises, peeq, s);      \
  }
  EXF_CASE(EXFEM_C3D8)
  EXF_CASE(EXFEM_C3D10)
#undef EXF_CASE
  set_error("unknown element type %d", b->etype);
  return EXFEM_ERR_ARG;
}

// ---------------------------------------------------------------- assembly
// f[3n+c] = sum over the gather plan of node n (reference order); optional opA
// finalisation y = fixed ? v : sum.
__global__ void gather_assemble_kernel(int64_t nn, int vmax, const int32_t* __restrict__ plan,
                                       int64_t sentinel, const double* __restrict__ ys,
                                       double* __restrict__ f, const uint8_t* __restrict__ fixed,
                                       const double* __restrict__ v, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  const int32_t* row = plan + n * vmax;
  for (int k = 0; k < vmax; ++k) {
    const int64_t slot = row[k];
    if (slot == sentinel) break;
    s0 += ys[3 * slot];
    s1 += ys[3 * slot + 1];
    s2 += ys[3 * slot + 2];
  }
  const double s[3] = {s0, s1, s2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t d = 3 * n + c;
    f[d] = (v && fixed && fixed[d]) ? v[d] : s[c];
  }
}

int launch_gather_assemble(exfem_block_s* b, const double* ys, double* f, const double* v_opa,
                           const int* skip, cudaStream_t s) {
  if (b->nn == 0) return EXFEM_OK;
  const int threads = 256;
  gather_assemble_kernel<<<(unsigned)((b->nn + threads - 1) / threads), threads, 0, s>>>(
      b->nn, b->vmax, b->plan.p, b->ne * b->nnode, ys, f, v_opa ? b->fixed.p : nullptr, v_opa, skip);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

// one colour: elements of the colour share no node, so plain read-modify-write is exact
__global__ void colour_scatter_kernel(int64_t cnt, const int32_t* __restrict__ elems,
                                      const int32_t* __restrict__ conn, int nnode,
                                      const double* __restrict__ fe, double* __restrict__ f) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const int64_t e = elems[i];
  for (int a = 0; a < nnode; ++a) {
    const int64_t n = conn[e * nnode + a];
    for (int c = 0; c < 3; ++c) f[3 * n + c] += fe[(e * nnode + a) * 3 + c];
  }
}

int launch_colour_assemble(exfem_block_s* b, const double* fe, double* f, cudaStream_t s) {
  EX_CUDA(cudaMemsetAsync(f, 0, sizeof(double) * b->ndof(), s));
  for (int c = 0; c < b->ncolour; ++c) {
    const int64_t a0 = b->colour_ptr[c], cnt = b->colour_ptr[c + 1] - a0;
    if (!cnt) continue;
    colour_scatter_kernel<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(cnt, b->colour_elems.p + a0,
                                                                        b->conn.p, b->nnode, fe, f);
    EX_LAUNCH_CHECK();
  }
  return EXFEM_OK;
}

// ---------------------------------------------------------------- geometry streams
// Per element: C3D8 the 7 modal coordinate vectors (21) and the stiffness scale;
// C3D10 the inverse Jacobian (9) and vol * scale; then, only for blocks with
// per-element Lame parameters, lambda and mu (the matrix-free kernels otherwise
// take the material's from their arguments).
template <int ET>
__global__ void geometry_kernel(int64_t ne, const double* __restrict__ X, const int32_t* __restrict__ conn_tile,
                                const int32_t* __restrict__ order, const double* __restrict__ scale,
                                const double* __restrict__ lam_e, const double* __restrict__ mu_e, int GS,
                                double* __restrict__ g64, float* __restrict__ g32, int tile) {
  using Tr = ElemTraits<ET>;
  constexpr int NN = Tr::nnode, GF = Tr::geo_stride;
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;   // tile position
  if (p >= ne) return;
  const int64_t e = order[p];
  const int32_t* cn = conn_tile + p * NN;                              // this position's nodes
  const double sc = scale ? scale[e] : 1.0;
  double out[GF];
#pragma unroll
  for (int k = 0; k < GF; ++k) out[k] = 0.0;
  if constexpr (ET == EXFEM_C3D8) {
    double xa[8][3], cm[7][3];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) xa[a][c] = X[3 * (int64_t)cn[a] + c];
    hex_to_modal(xa, cm);
#pragma unroll
    for (int k = 0; k < 7; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) out[3 * k + c] = cm[k][c];
    out[21] = sc;
  } else {
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, iJ[9];
#pragma unroll
    for (int a = 0; a < 10; ++a) {
      const int64_t n3 = 3 * (int64_t)cn[a];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) J[3 * c + i] += X[n3 + c] * tet10_dN(0, a, i);
    }
    const double det = inv3(J, iJ);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k] = iJ[k];
    out[9] = det / 24.0 * sc;
  }
  if (lam_e) {
    out[GF - 2] = lam_e[e];
    out[GF - 1] = mu_e[e];
  }
  for (int k = 0; k < GS; ++k) {
    g64[tile_index(p, k, GS, tile)] = out[k];
    g32[tile_index(p, k, GS, tile)] = (float)out[k];
  }
}

int build_geometry(exfem_block_s* b) {
  const int GF = b->etype == EXFEM_C3D8 ? ElemTraits<EXFEM_C3D8>::geo_stride : ElemTraits<EXFEM_C3D10>::geo_stride;
  const int GS = b->lam_e.p ? GF : GF - 2;
  int st;
  const int64_t padded = b->ntile * b->tile * GS;
  if (b->geo64.n != (size_t)padded || b->geo_stride != GS) {
    if ((st = b->geo64.alloc(padded))) return st;
    if ((st = b->geo32.alloc(padded))) return st;
    EX_CUDA(cudaMemset(b->geo64.p, 0, b->geo64.bytes()));
    EX_CUDA(cudaMemset(b->geo32.p, 0, b->geo32.bytes()));
  }
  b->geo_stride = GS;
  if (b->ne == 0) return EXFEM_OK;
  const int threads = 128;
  const unsigned grid = (unsigned)((b->ne + threads - 1) / threads);
  if (b->etype == EXFEM_C3D8)
    geometry_kernel<EXFEM_C3D8><<<grid, threads>>>(b->ne, b->X.p, b->conn_tile.p, b->order_dev.p, b->scale.p,
                                                   b->lam_e.p, b->mu_e.p, GS, b->geo64.p, b->geo32.p, b->tile);
  else
    geometry_kernel<EXFEM_C3D10><<<grid, threads>>>(b->ne, b->X.p, b->conn_tile.p, b->order_dev.p, b->scale.p,
                                                    b->lam_e.p, b->mu_e.p, GS, b->geo64.p, b->geo32.p, b->tile);
  EX_LAUNCH_CHECK();
  // the legacy stream only: a device-wide synchronisation would invalidate a graph
  // capture in progress on another host thread
  EX_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  return EXFEM_OK;
}

// ---------------------------------------------------------------- element tangents
__device__ __forceinline__ double elem_dN(int et, int g, int a, int i) {
  if (et == EXFEM_C3D8) return hex_dN(g, a, i);
  switch (g) {
    case 0: return tet10_dN(0, a, i);
    case 1: return tet10_dN(1, a, i);
    case 2: return tet10_dN(2, a, i);
    default: return tet10_dN(3, a, i);
  }
}

template <class OutT>
__device__ __forceinline__ void store_out(OutT* p, double v);
template <> __device__ __forceinline__ void store_out<double>(double* p, double v) { *p = v; }
template <> __device__ __forceinline__ void store_out<float>(float* p, double v) { *p = (float)v; }
template <> __device__ __forceinline__ void store_out<__nv_bfloat16>(__nv_bfloat16* p, double v) {
  *p = __float2bfloat16((float)v);
}

// One block = EPB elements x NN threads.  Phase 1: one thread per Gauss point
// computes the inverse Jacobian, weighted volume and material tangent data into
// shared memory.  Phase 2: one thread per element node a computes the three rows
// 3a..3a+2 of Ke = sum_g w_g dF_a : C_g : dF_b (the reference's G^T A G).
template <int ET, int MODE, class OutT>
__global__ void __launch_bounds__(64)
stiffness_kernel(int64_t ne, const double* __restrict__ X, const int32_t* __restrict__ conn,
                 const double* __restrict__ u, const double* __restrict__ scale,
                 const double* __restrict__ st_old, const double* __restrict__ tan_in,
                 const MatDev mat, const double* __restrict__ lam_e, const double* __restrict__ mu_e,
                 OutT* __restrict__ Ke, double* __restrict__ ediag, const int32_t* __restrict__ tpos, int tile) {
  using Tr = ElemTraits<ET>;
  constexpr int NN = Tr::nnode, NG = Tr::ngp, ND = 3 * NN, EPB = 64 / NN;
  constexpr bool BBAR = ET == EXFEM_C3D8;
  __shared__ double s_iJ[EPB][NG][9];
  __shared__ double s_vol[EPB][NG];
  __shared__ double s_tn[EPB][NG][8];
  __shared__ double s_iJ0[EPB][9];
  const int le = threadIdx.x / NN, a = threadIdx.x % NN;
  const int64_t e = (int64_t)blockIdx.x * EPB + le;
  const bool valid = le < EPB && e < ne;
  const bool own = valid && lam_e;  // per-element Lame parameters override the material's
  const double lam_k = own ? lam_e[e] : mat.lam, mu_k = own ? mu_e[e] : mat.mu;
  const int ns = mat.kind == EXFEM_J2 ? 19 : 1;
  if (valid && a < NG) {
    const int g = a;
    const double sc = scale ? scale[e] : 1.0;
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double J0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, G0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < NN; ++b) {
      const int64_t n3 = 3 * (int64_t)conn[e * NN + b];
      for (int i = 0; i < 3; ++i) {
        const double dn = elem_dN(ET, g, b, i);
        const double dn0 = BBAR ? 0.125 * hex_sign(b, i) : 0.0;
        for (int c = 0; c < 3; ++c) {
          const double xv = X[n3 + c], uv = u ? u[n3 + c] : 0.0;
          J[3 * c + i] += xv * dn;
          G[3 * c + i] += uv * dn;
          if (BBAR) {
            J0[3 * c + i] += xv * dn0;
            G0[3 * c + i] += uv * dn0;
          }
        }
      }
    }
    double iJ[9], H[9];
    const double detJ = inv3(J, iJ);
    matmul3(G, iJ, H);
    if (BBAR) {
      double iJ0[9], H0[9];
      inv3(J0, iJ0);
      matmul3(G0, iJ0, H0);
      const double bb = ((H0[0] + H0[4] + H0[8]) - (H[0] + H[4] + H[8])) / 3.0;
      H[0] += bb;
      H[4] += bb;
      H[8] += bb;
      if (g == 0)
        for (int k = 0; k < 9; ++k) s_iJ0[le][k] = iJ0[k];
    }
    double zero_state[19];
    for (int k = 0; k < 19; ++k) zero_state[k] = 0.0;
    const double* st = st_old ? st_old + (e * NG + g) * ns : zero_state;
    double sig[6], tn[8];
    if (tan_in) {
      for (int k = 0; k < 8; ++k) tn[k] = tan_in[tile_index(tpos[e], g * 8 + k, NG * 8, tile)];
    } else {
      material_stress(mat, lam_k, mu_k, H, st, nullptr, sig, tn);
    }
    for (int k = 0; k < 9; ++k) s_iJ[le][g][k] = iJ[k];
    s_vol[le][g] = (ET == EXFEM_C3D8 ? 1.0 : 1.0 / 24.0) * detJ * sc;
    for (int k = 0; k < 8; ++k) s_tn[le][g][k] = tn[k];
  }
  __syncthreads();
  if (!valid) return;
  double dNa[NG][3], dN0a[3] = {0, 0, 0};
#pragma unroll
  for (int g = 0; g < NG; ++g)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i) s += elem_dN(ET, g, a, i) * s_iJ[le][g][3 * i + j];
      dNa[g][j] = s;
    }
  if (BBAR)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i) s += 0.125 * hex_sign(a, i) * s_iJ0[le][3 * i + j];
      dN0a[j] = s;
    }
  const double Kb = own ? lam_k + 2.0 * mu_k / 3.0 : mat.K, mu = mu_k;
  for (int b = (MODE == 1 ? a : 0); b < (MODE == 1 ? a + 1 : NN); ++b) {
    double dNb[NG][3], dN0b[3] = {0, 0, 0};
#pragma unroll
    for (int g = 0; g < NG; ++g)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) s += elem_dN(ET, g, b, i) * s_iJ[le][g][3 * i + j];
        dNb[g][j] = s;
      }
    if (BBAR)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) s += 0.125 * hex_sign(b, i) * s_iJ0[le][3 * i + j];
        dN0b[j] = s;
      }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double acc[3] = {0, 0, 0};
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        H[3 * k + 0] = dNb[g][0];
        H[3 * k + 1] = dNb[g][1];
        H[3 * k + 2] = dNb[g][2];
        if (BBAR) {
          const double bb = (dN0b[k] - dNb[g][k]) / 3.0;
          H[0] += bb;
          H[4] += bb;
          H[8] += bb;
        }
        double de[6], ds[6];
        sym_from_grad(H, de);
        tangent_stress(Kb, mu, s_tn[le][g], de, ds);
        const double trs = ds[0] + ds[1] + ds[2];
        const double rows[3][3] = {{ds[0], ds[3], ds[5]}, {ds[3], ds[1], ds[4]}, {ds[5], ds[4], ds[2]}};
        const double w = s_vol[le][g];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          double v = rows[i][0] * dNa[g][0] + rows[i][1] * dNa[g][1] + rows[i][2] * dNa[g][2];
          if (BBAR) v += (dN0a[i] - dNa[g][i]) / 3.0 * trs;
          acc[i] += w * v;
        }
      }
      if (MODE == 0) {
#pragma unroll
        for (int i = 0; i < 3; ++i) store_out(Ke + e * ND * ND + (3 * a + i) * ND + 3 * b + k, acc[i]);
      } else {
        ediag[(e * NN + a) * 3 + k] = acc[k];
      }
    }
  }
}

template <int ET, class OutT>
static void stiffness_go(exfem_block_s* b, const double* u, const double* st_old, const double* tan_in,
                         OutT* Ke, double* ediag, cudaStream_t s) {
  constexpr int EPB = 64 / ElemTraits<ET>::nnode;
  const unsigned grid = (unsigned)((b->ne + EPB - 1) / EPB);
  if (ediag)
    stiffness_kernel<ET, 1, OutT><<<grid, 64, 0, s>>>(b->ne, b->X.p, b->conn.p, u, b->scale.p, st_old,
                                                      tan_in, b->mat, b->lam_e.p, b->mu_e.p, Ke, ediag,
                                                      b->tpos.p, b->tile);
  else
    stiffness_kernel<ET, 0, OutT><<<grid, 64, 0, s>>>(b->ne, b->X.p, b->conn.p, u, b->scale.p, st_old,
                                                      tan_in, b->mat, b->lam_e.p, b->mu_e.p, Ke, ediag,
                                                      b->tpos.p, b->tile);
}

int launch_stiffness(exfem_block_s* b, const double* u, const double* st_old, int dtype, void* Ke,
                     double* ediag, cudaStream_t s, const double* tan_in) {
  if (b->ne == 0) return EXFEM_OK;
  if (dtype == EXFEM_F64) {
    if (b->etype == EXFEM_C3D8) stiffness_go<EXFEM_C3D8>(b, u, st_old, tan_in, (double*)Ke, ediag, s);
    else stiffness_go<EXFEM_C3D10>(b, u, st_old, tan_in, (double*)Ke, ediag, s);
  } else if (dtype == EXFEM_F32) {
    if (b->etype == EXFEM_C3D8) stiffness_go<EXFEM_C3D8>(b, u, st_old, tan_in, (float*)Ke, ediag, s);
    else stiffness_go<EXFEM_C3D10>(b, u, st_old, tan_in, (float*)Ke, ediag, s);
  } else if (dtype == EXFEM_BF16) {
    if (b->etype == EXFEM_C3D8) stiffness_go<EXFEM_C3D8>(b, u, st_old, tan_in, (__nv_bfloat16*)Ke, ediag, s);
    else stiffness_go<EXFEM_C3D10>(b, u, st_old, tan_in, (__nv_bfloat16*)Ke, ediag, s);
  } else {
    set_error("unsupported Ke dtype %d", dtype);
    return EXFEM_ERR_ARG;
  }
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

// ---------------------------------------------------------------- initial-stress stiffness
// K_sigma of an element under a constant Cauchy stress sigma (gfem/model.py:113-117
// geo_stiff): k_ab = sum_g vol_g dN_a/dX . sigma . dN_b/dX with the plain
// (not B-bar) shape-function gradients and vol_g = w_g det J, expanded as
// K[3a+i, 3b+j] = k_ab delta_ij.  One thread per (element, node a) writes rows
// 3a .. 3a+2.
template <int ET>
__global__ void __launch_bounds__(128)
geo_stiffness_kernel(int64_t ne, const double* __restrict__ X, const int32_t* __restrict__ conn,
                     const double* __restrict__ S, double* __restrict__ Kg) {
  constexpr int NN = ElemTraits<ET>::nnode, NG = ElemTraits<ET>::ngp, ND = 3 * NN;
  const double w = ET == EXFEM_C3D8 ? 1.0 : 1.0 / 24.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ne * NN; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / NN;
    const int a = (int)(t - e * NN);
    const int32_t* ce = conn + e * NN;
    double sg[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) sg[k] = S[e * 9 + k];
    double k_ab[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) k_ab[b] = 0.0;
    for (int g = 0; g < NG; ++g) {
      double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, iJ[9];
      for (int c = 0; c < NN; ++c) {
        const double* xc = X + 3 * (int64_t)ce[c];
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
          for (int i = 0; i < 3; ++i) J[3 * n + i] += xc[n] * elem_dN(ET, g, c, i);
      }
      const double vol = w * inv3(J, iJ);
      double ga[3], sa[3];                                   // dN_a/dX and sigma . dN_a/dX
#pragma unroll
      for (int j = 0; j < 3; ++j)
        ga[j] = elem_dN(ET, g, a, 0) * iJ[j] + elem_dN(ET, g, a, 1) * iJ[3 + j] + elem_dN(ET, g, a, 2) * iJ[6 + j];
#pragma unroll
      for (int j = 0; j < 3; ++j) sa[j] = ga[0] * sg[j] + ga[1] * sg[3 + j] + ga[2] * sg[6 + j];
      for (int b = 0; b < NN; ++b) {
        double gb[3];
#pragma unroll
        for (int j = 0; j < 3; ++j)
          gb[j] = elem_dN(ET, g, b, 0) * iJ[j] + elem_dN(ET, g, b, 1) * iJ[3 + j] + elem_dN(ET, g, b, 2) * iJ[6 + j];
        k_ab[b] += vol * (sa[0] * gb[0] + sa[1] * gb[1] + sa[2] * gb[2]);
      }
    }
    double* K = Kg + e * (int64_t)ND * ND;
    for (int i = 0; i < 3; ++i)
      for (int b = 0; b < NN; ++b)
#pragma unroll
        for (int j = 0; j < 3; ++j) K[(int64_t)(3 * a + i) * ND + 3 * b + j] = i == j ? k_ab[b] : 0.0;
  }
}

int launch_geo_stiffness(exfem_block_s* b, const double* S, double* Kg, cudaStream_t s) {
  if (b->ne == 0) return EXFEM_OK;
  const int64_t work = b->ne * b->nnode;
  const unsigned grid = (unsigned)std::min<int64_t>((work + 127) / 128, 1 << 20);
  if (b->etype == EXFEM_C3D8) geo_stiffness_kernel<EXFEM_C3D8><<<grid, 128, 0, s>>>(b->ne, b->X.p, b->conn.p, S, Kg);
  else geo_stiffness_kernel<EXFEM_C3D10><<<grid, 128, 0, s>>>(b->ne, b->X.p, b->conn.p, S, Kg);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

// ---------------------------------------------------------------- stored-Ke products
// ys[e, r] = sum_j Ke[e, r, j] * (free*v)[dofs[e, j]]   (one thread per element row)
__global__ void ebe_rows_kernel(int64_t ne, int nnode, const int32_t* __restrict__ conn,
                                const double* __restrict__ Ke, const double* __restrict__ v,
                                const uint8_t* __restrict__ fixed, double* __restrict__ ys,
                                const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int nd = 3 * nnode;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ne * nd) return;
  const int64_t e = t / nd;
  const int r = (int)(t - e * nd);
  const double* K = Ke + e * nd * nd + (int64_t)r * nd;
  double s = 0.0;
  for (int a = 0; a < nnode; ++a) {
    const int64_t n3 = 3 * (int64_t)conn[e * nnode + a];
    for (int c = 0; c < 3; ++c) {
      const double vv = (fixed && fixed[n3 + c]) ? 0.0 : v[n3 + c];
      s += K[3 * a + c] * vv;
    }
  }
  ys[t] = s;
}

int launch_ebe_matvec(exfem_block_s* b, const double* Ke, const double* v, double* y,
                      const int* skip, cudaStream_t s, bool bc) {
  int st;
  if (b->ys.n < (size_t)(b->ne * b->nnode * 3) && (st = b->ys.alloc(b->ne * b->nnode * 3))) return st;
  const int64_t rows = b->ne * b->nnode * 3;
  if (rows) {
    ebe_rows_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(b->ne, b->nnode, b->conn.p, Ke, v,
                                                                   bc ? b->fixed.p : nullptr, b->ys.p, skip);
    EX_LAUNCH_CHECK();
  }
  return launch_gather_assemble(b, b->ys.p, y, bc ? v : nullptr, skip, s);
}

__global__ void ebe_diag_kernel(int64_t nn, int vmax, int nnode, const int32_t* __restrict__ plan,
                                int64_t sentinel, const double* __restrict__ Ke, const double* __restrict__ ediag,
                                double* __restrict__ diag) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const int nd = 3 * nnode;
  double s[3] = {0, 0, 0};
  for (int k = 0; k < vmax; ++k) {
    const int64_t slot = plan[n * vmax + k];
    if (slot == sentinel) break;
    const int64_t e = slot / nnode;
    const int a = (int)(slot - e * nnode);
    for (int c = 0; c < 3; ++c)
      s[c] += Ke ? Ke[e * nd * nd + (3 * a + c) * (int64_t)nd + 3 * a + c] : ediag[slot * 3 + c];
  }
  for (int c = 0; c < 3; ++c) diag[3 * n + c] = s[c];
}

int launch_ebe_diagonal(exfem_block_s* b, const double* Ke, double* diag, cudaStream_t s) {
  if (b->nn == 0) return EXFEM_OK;
  ebe_diag_kernel<<<(unsigned)((b->nn + 255) / 256), 256, 0, s>>>(b->nn, b->vmax, b->nnode, b->plan.p,
                                                                  b->ne * b->nnode, Ke, nullptr, diag);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

int launch_mf_diagonal(exfem_block_s* b, double* diag, cudaStream_t s) {
  int st;
  if (b->ys.n < (size_t)(b->ne * b->nnode * 3) && (st = b->ys.alloc(b->ne * b->nnode * 3))) return st;
  // element diagonals of the current matrix-free tangent: the stiffness kernel
  // in diagonal-only mode reading the stored per-Gauss-point tangent data (the
  // displacement enters the tangent only through that data)
  if (b->ne) {
    const double* tan_in = b->mat.kind == EXFEM_J2 ? b->tan64.p : nullptr;
    if ((st = launch_stiffness(b, nullptr, nullptr, EXFEM_F64, nullptr, b->ys.p, s, tan_in))) return st;
  }
  ebe_diag_kernel<<<(unsigned)((b->nn + 255) / 256), 256, 0, s>>>(b->nn, b->vmax, b->nnode, b->plan.p,
                                                                  b->ne * b->nnode, nullptr, b->ys.p, diag);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

}  // namespace exfem
