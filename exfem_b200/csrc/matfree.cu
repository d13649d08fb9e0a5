// Matrix-free element-by-element tangent product y = opA(v) in FP32 or FP64.
//
// This replaces the reference's forward-mode AD product K(u) v
// (gfem/model.py:488-490 Model.tangent_jvp) and its stored-Ke product
// (gfem/model.py:264-267) inside opA (gfem/solvers.py:257-267):
//     y = free * K (free * v) + fixed * v.
// Per element the kernel reads a geometry stream (C3D8: the 7 modal coordinate
// vectors, i.e. coordinates with the centroid removed, plus the stiffness scale;
// C3D10 with straight edges: the constant inverse Jacobian and scaled volume),
// gathers v at the element nodes, evaluates the B-bar (C3D8) or standard (C3D10)
// strain at every Gauss point, applies the elastic law or the stored J2
// consistent tangent, and scatters the element vector with atomic adds.
#include "internal.h"

namespace exfem {

template <class T>
__device__ __forceinline__ void mf_stress(bool j2, const T* __restrict__ tn, T lam, T mu, T Kb,
                                          const T (&e)[6], T (&s)[6]) {
  if (j2) {
    T t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = tn[k];
    tangent_stress(Kb, mu, t, e, s);
  } else {
    elastic_stress(lam, mu, e, s);
  }
}

template <class T>
__device__ __forceinline__ void matmul3t(const T (&A)[9], const T (&B)[9], T (&C)[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

template <class T, int ET, bool J2>
__global__ void __launch_bounds__(128)
mf_matvec_kernel(int64_t ne, const T* __restrict__ geo, const int32_t* __restrict__ conn,
                 const T* __restrict__ tan, const uint8_t* __restrict__ nfix, const T* __restrict__ v,
                 T* __restrict__ y, T lam, T mu, T Kb, const int* __restrict__ skip) {
  using Tr = ElemTraits<ET>;
  constexpr int NN = Tr::nnode, NG = Tr::ngp, GS = Tr::geo_stride;
  if (skip && *skip) return;
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int nod[NN];
  uint8_t fx[NN];
#pragma unroll
  for (int a = 0; a < NN; ++a) {
    nod[a] = __ldg(conn + e * NN + a);
    fx[a] = nfix ? __ldg(nfix + nod[a]) : (uint8_t)0;
  }
  T va[NN][3];
#pragma unroll
  for (int a = 0; a < NN; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) va[a][c] = ((fx[a] >> c) & 1) ? T(0) : __ldg(v + 3 * (int64_t)nod[a] + c);
  T g[GS];
#pragma unroll
  for (int k = 0; k < GS; ++k) g[k] = __ldg(geo + e * GS + k);
  T f[NN][3];
  if constexpr (ET == EXFEM_C3D8) {
    T cm[7][3], um[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) cm[k][c] = g[3 * k + c];
    const T sc = g[21];
    hex_to_modal(va, um);
    T J0[9], iJ0[9], G0[9], H0[9];
#pragma unroll
    for (int n = 0; n < 3; ++n)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        J0[3 * n + i] = cm[i][n];
        G0[3 * n + i] = um[i][n];
      }
    inv3(J0, iJ0);
    matmul3t(G0, iJ0, H0);
    const T tr0 = H0[0] + H0[4] + H0[8];
    T Fm[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k) Fm[k][0] = Fm[k][1] = Fm[k][2] = T(0);
    T tacc = T(0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const T x = T(HEX_GQ * hex_sign(q, 0)), yy = T(HEX_GQ * hex_sign(q, 1)), z = T(HEX_GQ * hex_sign(q, 2));
      T J[9], iJ[9], G[9], H[9];
      hex_modal_grad(cm, x, yy, z, J);
      const T detJ = inv3(J, iJ);
      hex_modal_grad(um, x, yy, z, G);
      matmul3t(G, iJ, H);
      const T bb = (tr0 - (H[0] + H[4] + H[8])) * T(1.0 / 3.0);
      H[0] += bb;
      H[4] += bb;
      H[8] += bb;
      T ee[6], s[6];
      sym_from_grad(H, ee);
      mf_stress<T>(J2, J2 ? tan + (e * NG + q) * 8 : nullptr, lam, mu, Kb, ee, s);
      const T vol = detJ * sc;
      const T t = vol * (s[0] + s[1] + s[2]) * T(1.0 / 3.0);
      tacc += t;
      const T r[3][3] = {{vol * s[0] - t, vol * s[3], vol * s[5]},
                         {vol * s[3], vol * s[1] - t, vol * s[4]},
                         {vol * s[5], vol * s[4], vol * s[2] - t}};
      T Q[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) Q[3 * i + k] = r[i][0] * iJ[3 * k] + r[i][1] * iJ[3 * k + 1] + r[i][2] * iJ[3 * k + 2];
      hex_modal_grad_adj(Q, x, yy, z, Fm);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int i = 0; i < 3; ++i) Fm[i][c] += tacc * iJ0[3 * i + c];
    T fo[8][3];
    hex_from_modal(Fm, fo);
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) f[a][c] = fo[a][c];
  } else {
    T iJ[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) iJ[k] = g[k];
    const T vol = g[9];
#pragma unroll
    for (int a = 0; a < NN; ++a) f[a][0] = f[a][1] = f[a][2] = T(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      T G[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) G[k] = T(0);
#pragma unroll
      for (int a = 0; a < 10; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const T dn = T(tet10_dN(q, a, i));
          if (dn != T(0))
#pragma unroll
            for (int c = 0; c < 3; ++c) G[3 * c + i] += va[a][c] * dn;
        }
      T H[9];
      matmul3t(G, iJ, H);
      T ee[6], s[6];
      sym_from_grad(H, ee);
      mf_stress<T>(J2, J2 ? tan + (e * NG + q) * 8 : nullptr, lam, mu, Kb, ee, s);
      const T r[3][3] = {{vol * s[0], vol * s[3], vol * s[5]},
                         {vol * s[3], vol * s[1], vol * s[4]},
                         {vol * s[5], vol * s[4], vol * s[2]}};
      T Q[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) Q[3 * i + k] = r[i][0] * iJ[3 * k] + r[i][1] * iJ[3 * k + 1] + r[i][2] * iJ[3 * k + 2];
#pragma unroll
      for (int a = 0; a < 10; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const T dn = T(tet10_dN(q, a, i));
          if (dn != T(0))
#pragma unroll
            for (int c = 0; c < 3; ++c) f[a][c] += Q[3 * c + i] * dn;
        }
    }
  }
#pragma unroll
  for (int a = 0; a < NN; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (!((fx[a] >> c) & 1)) atomicAdd(y + 3 * (int64_t)nod[a] + c, f[a][c]);
}

// y = fixed ? v : 0 before the scatter
template <class T>
__global__ void mf_init_kernel(int64_t ndof, const uint8_t* __restrict__ fixed, const T* __restrict__ v,
                               T* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ndof; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (fixed && fixed[i]) ? v[i] : T(0);
}

template <class T>
int launch_mf_matvec(exfem_block_s* b, const T* v, T* y, const int* skip, cudaStream_t s, bool bc) {
  const int64_t ndof = b->ndof();
  if (ndof == 0) return EXFEM_OK;
  mf_init_kernel<T><<<grid_for(ndof, 256), 256, 0, s>>>(ndof, bc ? b->fixed.p : nullptr, v, y, skip);
  EX_LAUNCH_CHECK();
  if (b->ne == 0) return EXFEM_OK;
  const T* geo;
  const T* tan;
  if constexpr (sizeof(T) == 8) {
    geo = (const T*)b->geo64.p;
    tan = (const T*)b->tan64.p;
  } else {
    geo = (const T*)b->geo32.p;
    tan = (const T*)b->tan32.p;
  }
  const bool j2 = b->mat.kind == EXFEM_J2;
  const T lam = (T)b->mat.lam, mu = (T)b->mat.mu, Kb = (T)b->mat.K;
  const int threads = 128;
  const unsigned grid = (unsigned)((b->ne + threads - 1) / threads);
  const uint8_t* nf = bc ? b->node_fixed.p : nullptr;
  if (b->etype == EXFEM_C3D8) {
    if (j2) mf_matvec_kernel<T, EXFEM_C3D8, true><<<grid, threads, 0, s>>>(b->ne, geo, b->conn.p, tan, nf, v, y, lam, mu, Kb, skip);
    else mf_matvec_kernel<T, EXFEM_C3D8, false><<<grid, threads, 0, s>>>(b->ne, geo, b->conn.p, tan, nf, v, y, lam, mu, Kb, skip);
  } else {
    if (!b->affine) {
      set_error("matrix-free C3D10 needs straight-edged elements (mid-nodes at edge midpoints)");
      return EXFEM_ERR_UNSUPPORTED;
    }
    if (j2) mf_matvec_kernel<T, EXFEM_C3D10, true><<<grid, threads, 0, s>>>(b->ne, geo, b->conn.p, tan, nf, v, y, lam, mu, Kb, skip);
    else mf_matvec_kernel<T, EXFEM_C3D10, false><<<grid, threads, 0, s>>>(b->ne, geo, b->conn.p, tan, nf, v, y, lam, mu, Kb, skip);
  }
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template int launch_mf_matvec<float>(exfem_block_s*, const float*, float*, const int*, cudaStream_t, bool);
template int launch_mf_matvec<double>(exfem_block_s*, const double*, double*, const int*, cudaStream_t, bool);

}  // namespace exfem
