// Element and material arithmetic shared by the element kernels.
//
// C3D8 (gfem/elements.py:113-125): 8-node trilinear hexahedron, 2x2x2 Gauss
// points at the corners scaled by 1/sqrt(3) (same order as the corners), unit
// weights, B-bar for small strain (gfem/model.py:42-51): the volumetric part of
// the displacement gradient at each Gauss point is replaced by its value at the
// element centre.
//
// The hexahedron is handled in a modal basis: with the corner signs s_a, any
// trilinear field is v(xi) = m0 + m1 xi + m2 eta + m3 zeta + m4 xi eta +
// m5 eta zeta + m6 xi zeta + m7 xi eta zeta with m_k = 1/8 sum_a S_k(a) v_a.
// Reference-coordinate gradients then need 3-4 terms per column instead of a
// sum over 8 nodes, and the adjoint (force) is accumulated in the same basis and
// mapped back to the nodes by one signed 8x8 transform.  Mathematically
// identical to the reference's einsum over dN (agreement to rounding).
//
// C3D10 (gfem/elements.py:166-179): quadratic tetrahedron, 4-point rule with
// barycentric a = 0.5854101966249685, b = 0.1381966011250105, weights 1/24.
//
// Materials (gfem/materials.py): LinearElastic sigma = lam tr(eps) I + 2 mu eps;
// J2Plasticity radial return with a fixed 25-iteration local Newton on dgamma
// (materials.py:270-296).  The consistent tangent the reference obtains with
// jax.jacfwd through that loop is written in closed form:
//   dsigma = K tr(de) I + 2 mu c1 dev(de) + c2 n (n : de),
//   c1 = 1 - 3 mu dg / q,  c2 = 4 mu^2 (dg / q - 1 / (3 mu + Hk + H')),
// with H' the table slope at the last local iterate (exactly what forward-mode
// AD through the final iteration yields), c1 = 1 and c2 = 0 on elastic points.
#pragma once
#include "common.cuh"

namespace exfem {

// ---------------------------------------------------------------- C3D8 tables
// corner signs of gfem/elements.py:114-115
__host__ __device__ constexpr int hex_sign(int a, int axis) {
  return axis == 0 ? ((a == 1 || a == 2 || a == 5 || a == 6) ? 1 : -1)
       : axis == 1 ? ((a == 2 || a == 3 || a == 6 || a == 7) ? 1 : -1)
                   : (a >= 4 ? 1 : -1);
}
// modal sign S_k(a), k = 1..7 : x, y, z, xy, yz, xz, xyz
__host__ __device__ constexpr int hex_mode_sign(int k, int a) {
  return k == 1 ? hex_sign(a, 0)
       : k == 2 ? hex_sign(a, 1)
       : k == 3 ? hex_sign(a, 2)
       : k == 4 ? hex_sign(a, 0) * hex_sign(a, 1)
       : k == 5 ? hex_sign(a, 1) * hex_sign(a, 2)
       : k == 6 ? hex_sign(a, 0) * hex_sign(a, 2)
                : hex_sign(a, 0) * hex_sign(a, 1) * hex_sign(a, 2);
}
constexpr double HEX_GQ = 0.57735026918962576451;  // 1/sqrt(3)

// nodal (8 x 3) -> modal m[k-1][c] for k = 1..7
template <class T>
__device__ __forceinline__ void hex_to_modal(const T (&v)[8][3], T (&m)[7][3]) {
#pragma unroll
  for (int k = 1; k <= 7; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T s = T(0);
#pragma unroll
      for (int a = 0; a < 8; ++a) s += T(hex_mode_sign(k, a)) * v[a][c];
      m[k - 1][c] = T(0.125) * s;
    }
}

// modal adjoint F[k-1][c] -> nodal f_a = 1/8 sum_k S_k(a) F_k
template <class T>
__device__ __forceinline__ void hex_from_modal(const T (&F)[7][3], T (&f)[8][3]) {
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T s = T(0);
#pragma unroll
      for (int k = 1; k <= 7; ++k) s += T(hex_mode_sign(k, a)) * F[k - 1][c];
      f[a][c] = T(0.125) * s;
    }
}

// gradient of a modal field at (x, y, z): G[c][i] = d v_c / d xi_i
template <class T>
__device__ __forceinline__ void hex_modal_grad(const T (&m)[7][3], T x, T y, T z, T (&G)[9]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    G[3 * c + 0] = m[0][c] + y * m[3][c] + z * m[5][c] + y * z * m[6][c];
    G[3 * c + 1] = m[1][c] + x * m[3][c] + z * m[4][c] + x * z * m[6][c];
    G[3 * c + 2] = m[2][c] + y * m[4][c] + x * m[5][c] + x * y * m[6][c];
  }
}

// accumulate the modal adjoint of hex_modal_grad for cotangent Q[c][i]
template <class T>
__device__ __forceinline__ void hex_modal_grad_adj(const T (&Q)[9], T x, T y, T z, T (&F)[7][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T q0 = Q[3 * c + 0], q1 = Q[3 * c + 1], q2 = Q[3 * c + 2];
    F[0][c] += q0;
    F[1][c] += q1;
    F[2][c] += q2;
    F[3][c] += y * q0 + x * q1;
    F[4][c] += z * q1 + y * q2;
    F[5][c] += z * q0 + x * q2;
    F[6][c] += y * z * q0 + x * z * q1 + x * y * q2;
  }
}

// ---------------------------------------------------------------- C3D10 tables
constexpr double TET_A = 0.5854101966249685;
constexpr double TET_B = 0.1381966011250105;
__host__ __device__ constexpr double tet_gp(int g, int i) {  // gfem/elements.py:177
  return (g == i + 1) ? TET_A : TET_B;
}
// barycentric L_c at Gauss point g, computed as the reference does from xi
__host__ __device__ constexpr double tet_L(int g, int c) {
  return c == 0 ? 1.0 - tet_gp(g, 0) - tet_gp(g, 1) - tet_gp(g, 2) : tet_gp(g, c - 1);
}
__host__ __device__ constexpr double tet_dL(int c, int i) {  // d L_c / d xi_i
  return c == 0 ? -1.0 : (c - 1 == i ? 1.0 : 0.0);
}
__host__ __device__ constexpr int tet_edge(int k, int end) {  // gfem/elements.py:167
  return end == 0 ? (k == 0 ? 0 : k == 1 ? 1 : k == 2 ? 2 : k == 3 ? 0 : k == 4 ? 1 : 2)
                  : (k == 0 ? 1 : k == 1 ? 2 : k == 2 ? 0 : 3);
}
// mid-edge node (4..9) between corners j != k (edge order of gfem/elements.py:167)
__host__ __device__ constexpr int tet_edge_node(int j, int k) {
  return (j == 0 && k == 1) || (j == 1 && k == 0)   ? 4
       : (j == 1 && k == 2) || (j == 2 && k == 1) ? 5
       : (j == 0 && k == 2) || (j == 2 && k == 0) ? 6
       : (j == 0 && k == 3) || (j == 3 && k == 0) ? 7
       : (j == 1 && k == 3) || (j == 3 && k == 1) ? 8
                                                  : 9;
}
// dN_a / d xi_i at Gauss point g (corner: L(2L-1); edge: 4 L_p L_q)
__host__ __device__ constexpr double tet10_dN(int g, int a, int i) {
  return a < 4 ? (4.0 * tet_L(g, a) - 1.0) * tet_dL(a, i)
               : 4.0 * (tet_dL(tet_edge(a - 4, 0), i) * tet_L(g, tet_edge(a - 4, 1)) +
                        tet_L(g, tet_edge(a - 4, 0)) * tet_dL(tet_edge(a - 4, 1), i));
}

// ---------------------------------------------------------------- tile-major streams
// Per-element streams of the matrix-free operator (geometry, J2 tangent data) are
// stored tile-major ("AoSoA") over the block's tile order: tiles of `tile`
// consecutive positions, and inside a tile component k of the element at
// position p at k*tile + p.  A tile's stream is one contiguous block (one bulk
// copy), and the thread that evaluates positions 2j and 2j+1 reads component k of
// both with one 8- (FP32) or 16-byte (FP64) load.
__host__ __device__ __forceinline__ int64_t tile_index(int64_t pos, int k, int width, int tile) {
  return ((pos / tile) * width + k) * tile + (pos % tile);
}

// ---------------------------------------------------------------- element traits
template <int ET> struct ElemTraits;
template <> struct ElemTraits<EXFEM_C3D8> {
  static constexpr int nnode = 8, ngp = 8, nd = 24;
  static constexpr int geo_stride = 24;  // modal c1..c7 (21), scale, lambda, mu
};
template <> struct ElemTraits<EXFEM_C3D10> {
  static constexpr int nnode = 10, ngp = 4, nd = 30;
  static constexpr int geo_stride = 12;  // inverse Jacobian (9), vol*scale, lambda, mu
};

// ---------------------------------------------------------------- materials
struct MatDev {
  int kind;
  double mu, lam, K, Hk;
  int ntab;
  double ep[EXFEM_MAX_TABLE], sy[EXFEM_MAX_TABLE];
};

// np.interp on the hardening table and its derivative (0 where clamped)
__device__ __forceinline__ void table_interp(const MatDev& m, double x, double& f, double& slope) {
  const int n = m.ntab;
  int c = 0;
  for (int j = 0; j < n; ++j) c += (m.ep[j] <= x) ? 1 : 0;
  int i = c < 1 ? 1 : (c > n - 1 ? n - 1 : c);
  const double x0 = m.ep[i - 1], x1 = m.ep[i], f0 = m.sy[i - 1], f1 = m.sy[i];
  const double dx = x1 - x0, df = f1 - f0;
  const bool dx0 = fabs(dx) <= 4.930380657631324e-32;  // spacing(eps) of float64
  f = dx0 ? f0 : f0 + ((x - x0) / dx) * df;
  slope = dx0 ? 0.0 : df / dx;
  if (x < m.ep[0]) { f = m.sy[0]; slope = 0.0; }
  if (x > m.ep[n - 1]) { f = m.sy[n - 1]; slope = 0.0; }
}

// symmetric 3x3 as 6 (xx, yy, zz, xy, yz, xz)
template <class T>
__device__ __forceinline__ void sym_from_grad(const T (&H)[9], T (&e)[6]) {
  e[0] = H[0];
  e[1] = H[4];
  e[2] = H[8];
  e[3] = T(0.5) * (H[1] + H[3]);
  e[4] = T(0.5) * (H[5] + H[7]);
  e[5] = T(0.5) * (H[2] + H[6]);
}

template <class T>
__device__ __forceinline__ void elastic_stress(T lam, T mu, const T (&e)[6], T (&s)[6]) {
  const T tr = e[0] + e[1] + e[2];
  s[0] = lam * tr + T(2) * mu * e[0];
  s[1] = lam * tr + T(2) * mu * e[1];
  s[2] = lam * tr + T(2) * mu * e[2];
  s[3] = T(2) * mu * e[3];
  s[4] = T(2) * mu * e[4];
  s[5] = T(2) * mu * e[5];
}

// linearised J2 stress with tangent data tn = (n[6], c1, c2)
template <class T>
__device__ __forceinline__ void tangent_stress(T Kb, T mu, const T* tn, const T (&e)[6], T (&s)[6]) {
  const T tr = e[0] + e[1] + e[2];
  const T m3 = tr * T(1.0 / 3.0);
  const T nde = tn[0] * e[0] + tn[1] * e[1] + tn[2] * e[2] +
                T(2) * (tn[3] * e[3] + tn[4] * e[4] + tn[5] * e[5]);
  const T a = T(2) * mu * tn[6], b = tn[7] * nde;
  s[0] = Kb * tr + a * (e[0] - m3) + b * tn[0];
  s[1] = Kb * tr + a * (e[1] - m3) + b * tn[1];
  s[2] = Kb * tr + a * (e[2] - m3) + b * tn[2];
  s[3] = a * e[3] + b * tn[3];
  s[4] = a * e[4] + b * tn[4];
  s[5] = a * e[5] + b * tn[5];
}

// J2 radial return (gfem/materials.py:270-296) at one Gauss point.
// eps: symmetric strain (6); st: state in (19) = [eps_p (3x3), alpha, beta (3x3)];
// sn: state out (may alias nothing); sig: stress (6); tn: tangent data (8).
__device__ __forceinline__ void j2_return(const MatDev& m, const double (&eps)[6], const double* st,
                                          double* sn, double (&sig)[6], double (&tn)[8]) {
  const double mu = m.mu;
  double ee[9];
  ee[0] = eps[0] - st[0]; ee[1] = eps[3] - st[1]; ee[2] = eps[5] - st[2];
  ee[3] = eps[3] - st[3]; ee[4] = eps[1] - st[4]; ee[5] = eps[4] - st[5];
  ee[6] = eps[5] - st[6]; ee[7] = eps[4] - st[7]; ee[8] = eps[2] - st[8];
  const double a0 = st[9];
  const double tr = ee[0] + ee[4] + ee[8];
  double xi[9], s_tr[9];
  double ss = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double dev = ee[k] - ((k == 0 || k == 4 || k == 8) ? tr / 3.0 : 0.0);
    s_tr[k] = 2.0 * mu * dev;
    xi[k] = s_tr[k] - st[10 + k];
    ss += xi[k] * xi[k];
  }
  const double q_tr = 1.2247448713915890491 * sqrt(ss + 1e-30);
  double sy0, tmp;
  table_interp(m, a0, sy0, tmp);
  const double f_tr = q_tr - sy0;
  const double H3 = 3.0 * mu + m.Hk;
  double dg = 0.0, hp = 0.0;
  for (int it = 0; it < 25; ++it) {
    double syv, dsy;
    table_interp(m, a0 + dg, syv, dsy);
    const double g = q_tr - H3 * dg - syv;
    const double nd = dg + g / (H3 + dsy);
    hp = dsy;
    dg = nd > 0.0 ? nd : 0.0;
  }
  const bool plastic = f_tr > 0.0;
  if (!plastic) dg = 0.0;
  const double qn = q_tr + 1e-30;
  double n[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) n[k] = 1.5 * xi[k] / qn;
  const double Kb = m.K;
  double sg[9];
#pragma unroll
  for (int k = 0; k < 9; ++k)
    sg[k] = s_tr[k] - 2.0 * mu * dg * n[k] + ((k == 0 || k == 4 || k == 8) ? Kb * tr : 0.0);
  sig[0] = sg[0]; sig[1] = sg[4]; sig[2] = sg[8];
  sig[3] = sg[1]; sig[4] = sg[5]; sig[5] = sg[2];
  if (sn) {
#pragma unroll
    for (int k = 0; k < 9; ++k) sn[k] = st[k] + dg * n[k];
    sn[9] = a0 + dg;
#pragma unroll
    for (int k = 0; k < 9; ++k) sn[10 + k] = st[10 + k] + (2.0 / 3.0) * m.Hk * dg * n[k];
  }
  if (plastic) {
    tn[0] = n[0]; tn[1] = n[4]; tn[2] = n[8]; tn[3] = n[1]; tn[4] = n[5]; tn[5] = n[2];
    tn[6] = 1.0 - 3.0 * mu * dg / q_tr;
    tn[7] = 4.0 * mu * mu * (dg / q_tr - 1.0 / (H3 + hp));
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k) tn[k] = 0.0;
    tn[6] = 1.0;
    tn[7] = 0.0;
  }
}

// stress at a Gauss point for the FP64 residual; writes the state and the tangent data.
// lam, mu: the element's Lame parameters (linear elasticity; J2 uses the material's)
__device__ __forceinline__ void material_stress(const MatDev& m, double lam, double mu, const double (&H)[9],
                                                const double* st, double* sn, double (&sig)[6],
                                                double (&tn)[8]) {
  double e[6];
  sym_from_grad(H, e);
  if (m.kind == EXFEM_J2) {
    j2_return(m, e, st, sn, sig, tn);
  } else {
    elastic_stress(lam, mu, e, sig);
    if (sn) sn[0] = st ? st[0] : 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) tn[k] = 0.0;
    tn[6] = 1.0;
    tn[7] = 0.0;
  }
}

}  // namespace exfem
