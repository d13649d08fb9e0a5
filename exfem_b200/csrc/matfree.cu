// Matrix-free element-by-element tangent product y = opA(v) in FP32 or FP64.
//
// Replaces the reference's forward-mode AD product K(u) v (gfem/model.py:488-490
// Model.tangent_jvp) and its stored-Ke product (gfem/model.py:264-267) inside
// opA (gfem/solvers.py:257-267):  y = free * K (free * v) + fixed * v.
//
// Work unit: a tile of TT consecutive positions of the block's tile order
// (elements grouped by mesh component and sorted along a Morton curve, so that a
// tile is a compact patch), one CTA of TT/2 threads per tile, persistent over
// tiles.  Per tile:
//   1. the tile's streams (geometry, slot -> node-list position, the slots
//      grouped by node and the end of each node's run) are one contiguous block
//      each; in the FP32 kernel one thread moves them into shared memory with
//      bulk TMA copies (cp.async.bulk, mbarrier completion), double buffered so
//      that the copy of the next tile overlaps the work on this one;
//   2. v is gathered once per distinct node of the tile into shared memory with
//      asynchronous cp.async copies issued one tile ahead (fixed DOFs, whose bits
//      sit above the node id in the tile list, are zero filled);
//   3. thread j evaluates the products of the elements at tile positions 2j and
//      2j+1 together, every arithmetic operation on a lane pair (in FP32 one
//      packed FFMA2/FADD2/FMUL2 instruction for both elements), and writes the 2 x
//      nnode nodal force vectors into its own slots;
//   4. each distinct node of the tile sums its slots in increasing slot order
//      (no atomics, a fixed order) and stores the sum at its precomputed position
//      in a node-major partials buffer;
// and a second, node-centric pass forms y[n] = fixed ? v : the sum of node n's
// contiguous run of tile entries, in tile order (the reference's atomic-free
// gather-plan assembly, gfem/model.py:241-267, at tile granularity).  The
// product is deterministic: every sum has a fixed order.
// Geometry: C3D8 stores the 7 modal coordinate vectors (coordinates with the
// centroid removed) and the stiffness scale; C3D10 stores the inverse Jacobian
// and scaled volume, formed in FP64 from the nodal coordinates and rounded once.
#include <limits>
#include <mutex>
#include <type_traits>

#include "internal.h"
#include "pair_math.cuh"

namespace exfem {

// ---------------------------------------------------------------- async-copy helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: gives up after `polls` polls (default ~2^24, seconds at most),
// records the failure in *err and returns false
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, int polls = 1 << 24) {
  for (int i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, 1);
  return false;
}

// Self-test of the bounded wait: nothing ever arrives on the barrier, so every
// thread's wait must give up after `polls` polls and record it; the kernel then
// returns normally and the context stays usable.
__global__ void wait_selftest_kernel(int polls, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  mbar_wait_bounded(&bar, 0, err, polls);
}

int launch_wait_selftest(int polls, int* err, cudaStream_t s) {
  wait_selftest_kernel<<<1, 32, 0, s>>>(polls, err);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

// 4- or 8-byte asynchronous global->shared copy; src_bytes = 0 writes zeros
template <int N>
__device__ __forceinline__ void cp_async(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src), "n"(N), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <class T>
__device__ __forceinline__ void matmul3t(const T (&A)[9], const T (&B)[9], T (&C)[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// stress at a Gauss point from the strain: elastic or the stored J2 tangent
// (tn points to component 0 of this element pair and point, stride S pairs)
template <class P, int S, bool J2>
__device__ __forceinline__ void mf_stress(const P* tn, P lam, P mu, P Kb, const P (&e)[6], P (&s)[6]) {
  if constexpr (J2) {
    P t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = tn[k * S];
    tangent_stress(Kb, mu, t, e, s);
  } else {
    elastic_stress(lam, mu, e, s);
  }
}

// products f = Ke v_e of an element (pair) from its streams (g, tn: component 0
// of the element (pair), stride S); P is a lane pair (F2, D2) or a scalar.  With
// ELAME the Lame parameters follow the geometry, otherwise lam and mu are the
// material's (J2 uses mu and the bulk modulus Kb).
template <class P, int ET, bool J2, bool ELAME, int S>
__device__ __forceinline__ void element_product(const P* g, const P* tn, const P (&va)[ElemTraits<ET>::nnode][3],
                                                P lam, P mu, P Kb, P (&f)[ElemTraits<ET>::nnode][3]) {
  if constexpr (ET == EXFEM_C3D8) {
    P cm[7][3], um[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) cm[k][c] = g[(3 * k + c) * S];
    const P sc = g[21 * S];
    const P le = ELAME ? g[22 * S] : lam, me = (J2 || !ELAME) ? mu : g[23 * S];
    hex_to_modal(va, um);
    P J0[9], iJ0[9], G0[9], H0[9];
#pragma unroll
    for (int n = 0; n < 3; ++n)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        J0[3 * n + i] = cm[i][n];
        G0[3 * n + i] = um[i][n];
      }
    inv3(J0, iJ0);
    matmul3t(G0, iJ0, H0);
    const P tr0 = H0[0] + H0[4] + H0[8];
    P Fm[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k) Fm[k][0] = Fm[k][1] = Fm[k][2] = P(0.0);
    P tacc = P(0.0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const P x = P(HEX_GQ * hex_sign(q, 0)), yy = P(HEX_GQ * hex_sign(q, 1)), z = P(HEX_GQ * hex_sign(q, 2));
      P J[9], iJ[9], G[9], H[9];
      hex_modal_grad(cm, x, yy, z, J);
      const P detJ = inv3(J, iJ);
      hex_modal_grad(um, x, yy, z, G);
      matmul3t(G, iJ, H);
      const P bb = P((tr0 - (H[0] + H[4] + H[8])) * P(1.0 / 3.0));
      H[0] += bb;
      H[4] += bb;
      H[8] += bb;
      P ee[6], s[6];
      sym_from_grad(H, ee);
      mf_stress<P, S, J2>(tn + q * 8 * S, le, me, Kb, ee, s);
      const P vol = P(detJ * sc);
      const P t = P(vol * (s[0] + s[1] + s[2]) * P(1.0 / 3.0));
      tacc += t;
      const P r[3][3] = {{vol * s[0] - t, P(vol * s[3]), P(vol * s[5])},
                         {P(vol * s[3]), vol * s[1] - t, P(vol * s[4])},
                         {P(vol * s[5]), P(vol * s[4]), vol * s[2] - t}};
      P Q[9];
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
    hex_from_modal(Fm, f);
  } else if constexpr (!J2) {
    // linear-elastic C3D10 with a constant Jacobian (straight edges): the
    // displacement gradient is linear in the barycentric coordinates L, so the
    // stress is too, and the 4-point rule integrates the degree-2 integrand
    // exactly.  With sigma_k the stress at corner k, g_i = grad L_i (rows of the
    // inverse Jacobian, g_0 = -(g_1 + g_2 + g_3)), V = 4 vol the element volume
    // and s_k = (V/20) sigma_k, S = sum_k s_k, the exact integrals
    //   f_i  = (4 s_i - S) g_i                     (corner i)
    //   f_ij = 4 ((S + s_j) g_i + (S + s_i) g_j)   (mid-node of edge ij)
    // equal the quadrature sums of the reference.  The corner gradients follow
    // from du/dL_i at corner k: 3 u_k for i = k, 4 u_ik - u_i otherwise.
    P iJ[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) iJ[k] = g[k * S];
    const P vol = g[9 * S];
    const P lt = P(P(0.2) * vol * (ELAME ? g[10 * S] : lam)), mt = P(P(0.2) * vol * (ELAME ? g[11 * S] : mu));
    const P m2 = P(P(2.0) * mt);
    P sv[4][6];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      P nw[3];                                          // -du/dL_0 at corner k
#pragma unroll
      for (int c = 0; c < 3; ++c) nw[c] = k == 0 ? P(P(-3.0) * va[0][c]) : P(-4.0) * va[tet_edge_node(0, k)][c] + va[0][c];
      P G[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int m = 1; m < 4; ++m)
          G[3 * c + m - 1] = m == k ? P(3.0) * va[k][c] + nw[c] : P(4.0) * va[tet_edge_node(m, k)][c] + (nw[c] - va[m][c]);
      P Hk[9];
      matmul3t(G, iJ, Hk);
      const P tr = Hk[0] + Hk[4] + Hk[8];
      const P ltr = P(lt * tr);
      sv[k][0] = m2 * Hk[0] + ltr;
      sv[k][1] = m2 * Hk[4] + ltr;
      sv[k][2] = m2 * Hk[8] + ltr;
      sv[k][3] = P(mt * (Hk[1] + Hk[3]));
      sv[k][4] = P(mt * (Hk[5] + Hk[7]));
      sv[k][5] = P(mt * (Hk[2] + Hk[6]));
    }
    P NSs[6], S4[6];                                    // -S, 4 S
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const P Ss = sv[0][j] + sv[1][j] + sv[2][j] + sv[3][j];
      NSs[j] = -Ss;
      S4[j] = P(P(4.0) * Ss);
    }
    P gr[4][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      gr[1][j] = iJ[j];
      gr[2][j] = iJ[3 + j];
      gr[3][j] = iJ[6 + j];
      gr[0][j] = -(gr[1][j] + gr[2][j] + gr[3][j]);
    }
    // symmetric (xx yy zz xy yz xz) times vector
    auto smv = [](const P (&m)[6], const P (&x)[3], P (&y)[3]) {
      y[0] = m[0] * x[0] + m[3] * x[1] + m[5] * x[2];
      y[1] = m[3] * x[0] + m[1] * x[1] + m[4] * x[2];
      y[2] = m[5] * x[0] + m[4] * x[1] + m[2] * x[2];
    };
    auto smv_acc = [](const P (&m)[6], const P (&x)[3], P (&y)[3]) {
      y[0] += m[0] * x[0] + m[3] * x[1] + m[5] * x[2];
      y[1] += m[3] * x[0] + m[1] * x[1] + m[4] * x[2];
      y[2] += m[5] * x[0] + m[4] * x[1] + m[2] * x[2];
    };
    P U[4][6];                                          // 4 (S + s_k)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      P Z[6];                                           // 4 s_k - S
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        Z[j] = P(4.0) * sv[k][j] + NSs[j];
        U[k][j] = P(4.0) * sv[k][j] + S4[j];
      }
      smv(Z, gr[k], f[k]);
    }
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      const int i = tet_edge(e, 0), j = tet_edge(e, 1);
      smv(U[j], gr[i], f[4 + e]);
      smv_acc(U[i], gr[j], f[4 + e]);
    }
  } else {
    // C3D10 with a constant Jacobian, in barycentric form: with L the
    // barycentric coordinates, w_j = du/dL_j = base_j + D * (g == j ? v_j : v_e(j,g))
    // at Gauss point g (L_g = A, others B), base_j = (4B-1) v_j + 4B sum of the
    // edge nodes at corner j, D = 4(A-B); the reference gradient is
    // G_i = w_{i+1} - w_0.  The force is the adjoint of the same steps.
    const P D = P(4.0 * (TET_A - TET_B)), C0 = P(4.0 * TET_B - 1.0), C1 = P(4.0 * TET_B);
    P iJ[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) iJ[k] = g[k * S];
    const P vol = g[9 * S];
    const P le = ELAME ? g[10 * S] : lam, me = (J2 || !ELAME) ? mu : g[11 * S];
    P base[4][3], vbar[10][3], bbar[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      base[0][c] = C0 * va[0][c] + C1 * (va[4][c] + va[6][c] + va[7][c]);
      base[1][c] = C0 * va[1][c] + C1 * (va[4][c] + va[5][c] + va[8][c]);
      base[2][c] = C0 * va[2][c] + C1 * (va[5][c] + va[6][c] + va[9][c]);
      base[3][c] = C0 * va[3][c] + C1 * (va[7][c] + va[8][c] + va[9][c]);
    }
#pragma unroll
    for (int a = 0; a < 10; ++a) vbar[a][0] = vbar[a][1] = vbar[a][2] = P(0.0);
#pragma unroll
    for (int j = 0; j < 4; ++j) bbar[j][0] = bbar[j][1] = bbar[j][2] = P(0.0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      P w[4][3];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int src = jj == q ? jj : tet_edge_node(jj, q);
#pragma unroll
        for (int c = 0; c < 3; ++c) w[jj][c] = base[jj][c] + D * va[src][c];
      }
      P G[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) G[3 * c + i] = w[i + 1][c] - w[0][c];
      P H[9];
      matmul3t(G, iJ, H);
      P ee[6], s[6];
      sym_from_grad(H, ee);
      mf_stress<P, S, J2>(tn + q * 8 * S, le, me, Kb, ee, s);
      const P r[3][3] = {{P(vol * s[0]), P(vol * s[3]), P(vol * s[5])},
                         {P(vol * s[3]), P(vol * s[1]), P(vol * s[4])},
                         {P(vol * s[5]), P(vol * s[4]), P(vol * s[2])}};
      P Q[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) Q[3 * i + k] = r[i][0] * iJ[3 * k] + r[i][1] * iJ[3 * k + 1] + r[i][2] * iJ[3 * k + 2];
      // adjoint: wbar_{i+1} = Q[:, i], wbar_0 = -sum_i Q[:, i]
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        P wb[4];
        wb[1] = Q[3 * c + 0];
        wb[2] = Q[3 * c + 1];
        wb[3] = Q[3 * c + 2];
        wb[0] = -(wb[1] + wb[2] + wb[3]);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          bbar[jj][c] += wb[jj];
          const int src = jj == q ? jj : tet_edge_node(jj, q);
          vbar[src][c] += D * wb[jj];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      vbar[0][c] += C0 * bbar[0][c];
      vbar[1][c] += C0 * bbar[1][c];
      vbar[2][c] += C0 * bbar[2][c];
      vbar[3][c] += C0 * bbar[3][c];
      const P e0 = C1 * bbar[0][c], e1 = C1 * bbar[1][c], e2 = C1 * bbar[2][c], e3 = C1 * bbar[3][c];
      vbar[4][c] += e0 + e1;   // edge (0,1)
      vbar[5][c] += e1 + e2;   // edge (1,2)
      vbar[6][c] += e0 + e2;   // edge (2,0)
      vbar[7][c] += e0 + e3;   // edge (0,3)
      vbar[8][c] += e1 + e3;   // edge (1,3)
      vbar[9][c] += e2 + e3;   // edge (2,3)
    }
#pragma unroll
    for (int a = 0; a < 10; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) f[a][c] = vbar[a][c];
  }
}

// Fixed-point accumulation of the tile's node sums: every nodal force of the
// tile is scaled by q = 2^(B - e), with 2^e > vmax * max|f| over the tile (vmax
// the largest number of element slots at one node), rounded to an integer and
// added with native shared-memory integer atomics; the sums are exact integers,
// independent of the order of the additions, and |sum| < 2^B fits the integer.
// Converted back they carry a rounding error of at most vmax / (2q) <
// 2^-B vmax^2 max|f|, below the rounding of the FP32 / FP64 sums they replace.
template <class T> struct FixedOf;
template <> struct FixedOf<float> {
  using type = int32_t;
  static constexpr int B = 30;
};
template <> struct FixedOf<double> {
  using type = unsigned long long;
  static constexpr int B = 62;
};
__device__ __forceinline__ float max_nan(float a, float b) {
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ double max_nan(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }
__device__ __forceinline__ int32_t to_fixed(float x) { return __float2int_rn(x); }
__device__ __forceinline__ unsigned long long to_fixed(double x) { return (unsigned long long)__double2ll_rn(x); }
__device__ __forceinline__ float from_fixed(int32_t i, float) { return __int2float_rn(i); }
__device__ __forceinline__ double from_fixed(unsigned long long i, double) { return __ll2double_rn((long long)i); }

// local node of the second element of a face pair that may hold the same node as
// local node a of the first (and conversely: the map is an involution), -1 if
// none.  C3D10 face pairs put the shared face's corners at (0,1,2) and (1,0,2),
// so the shared edge nodes are 4<->4 (edge 01), 5<->6 (edges 12 and 20); the
// kernel compares the two nodes before sharing anything.
template <int ET>
__host__ __device__ constexpr int pair_partner(int a) {
  if constexpr (ET == EXFEM_C3D10)
    return a == 0 ? 1 : a == 1 ? 0 : a == 2 ? 2 : a == 4 ? 4 : a == 5 ? 6 : a == 6 ? 5 : -1;
  else
    return -1;
}

template <class T, int ET, int TT, int LANES, bool ELAME>
struct TileLayout {
  using Tr = ElemTraits<ET>;
  using I = typename FixedOf<T>::type;
  static constexpr int NN = Tr::nnode, NG = Tr::ngp, NSLOT = NN * TT, NT = TT / LANES;
  static constexpr int GS = ELAME ? Tr::geo_stride : Tr::geo_stride - 2;
  static constexpr uint32_t GEO_B = GS * TT * sizeof(T);
  static constexpr uint32_t LIDX_B = NSLOT * sizeof(uint16_t);
  static constexpr uint32_t STAGE_B = GEO_B + LIDX_B;
  static_assert(GEO_B % 16 == 0 && LIDX_B % 16 == 0, "bulk copies need 16-byte multiples");
  // one shared-memory record per distinct node of the tile: v (3) and the
  // fixed-point sums (3), padded to an odd number of elements (FP32: 7 words;
  // FP64: 7 eight-byte words, which keeps every double 8-byte aligned) so that a
  // warp's scattered record accesses spread over all banks; one address serves a
  // node's loads and its atomic additions
  static constexpr int RW = sizeof(T) == 4 ? 7 : 14;                  // record size in 4-byte words
  static_assert((RW * 4) % sizeof(T) == 0 && (RW * 4) % sizeof(I) == 0, "records keep their members aligned");
  static constexpr int ROFF = 3 * sizeof(T);                          // byte offset of the sums
  // shared memory: [2 stages (TMA only): geometry | lidx] [records: mu]
  // [destinations: 2 x mu], mu = maxu rounded up to 8
  static size_t smem_bytes(bool tma, int mu) {
    return (tma ? 2 * (size_t)STAGE_B : 0) + (size_t)mu * RW * 4 + 2 * (size_t)mu * sizeof(int32_t);
  }
  // lane pairs: registers capped so that 3 CTAs of 128 (6 of 64) threads fit an SM
  static constexpr int MINB = (LANES == 2) ? 384 / NT : 1;
};

// LANES = 2: thread j evaluates the elements at tile positions 2j and 2j+1 as one
// lane pair; LANES = 1: thread j evaluates the element at position j alone, for
// element types and precisions whose pair arithmetic would not fit in registers.
template <class T, int ET, bool J2, bool ELAME, int TT, int LANES, bool TMA>
__global__ void __launch_bounds__(TT / LANES, TileLayout<T, ET, TT, LANES, ELAME>::MINB)
mf_tile_kernel(int64_t ne, int64_t ntile, const T* __restrict__ geo, const uint16_t* __restrict__ lidx,
               const T* __restrict__ tan, const int32_t* __restrict__ tptr, const int32_t* __restrict__ tpack,
               const int32_t* __restrict__ tdest, const T* __restrict__ v, T* __restrict__ y, T* __restrict__ part,
               T lam_m, T mu_m, T K_m, int mu, int vmax, const int* __restrict__ skip, int* __restrict__ err) {
  using L = TileLayout<T, ET, TT, LANES, ELAME>;
  using I = typename L::I;
  using P = std::conditional_t<LANES == 2, typename PairOf<T>::type, T>;
  constexpr int NN = L::NN, NG = L::NG, GS = L::GS, NSLOT = L::NSLOT, NT = L::NT, NW = NT / 32;
  constexpr int B = FixedOf<T>::B, GK = 8;
  if (skip && *skip) return;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ T wmax[NW];
  const int tid = threadIdx.x;
  unsigned char* base = smem + (TMA ? 2 * L::STAGE_B : 0);
  unsigned char* rec = base;                                                        // [mu] records
  int32_t* tdb = reinterpret_cast<int32_t*>(base + (size_t)mu * L::RW * 4);         // [2][mu]
  auto vval = [&](int k) { return reinterpret_cast<T*>(rec + k * (L::RW * 4)); };
  auto sums = [&](int k) { return reinterpret_cast<I*>(rec + k * (L::RW * 4) + L::ROFF); };
  auto stage = [&](int s) { return smem + s * L::STAGE_B; };
  auto issue = [&](int64_t t, int s) {
    fence_proxy_async();
    mbar_expect_tx(&bar[s], L::STAGE_B);
    bulk_g2s(stage(s), geo + t * (GS * TT), L::GEO_B, &bar[s]);
    bulk_g2s(stage(s) + L::GEO_B, lidx + t * NSLOT, L::LIDX_B, &bar[s]);
  };
  // node lists run ahead: the packed ids of tile t+2 are loaded into registers
  // while tile t is processed, and the asynchronous copies of tile t+1's node
  // values and destinations (fixed DOFs zero filled) are issued, from the ids
  // loaded one tile earlier, as soon as tile t's elements have read theirs
  struct Ids {
    int32_t u0, nu;
    uint32_t pk[GK];
  };
  // (the list bounds come from registers loaded one tile earlier, so the id loads
  // never wait on a dependent load of tptr)
  auto load_ids = [&](int32_t u0, int32_t u1, Ids& d) {
    d.u0 = u0;
    d.nu = u1 - u0;
#pragma unroll
    for (int i = 0; i < GK; ++i) {
      const int k = tid + i * NT;
      d.pk[i] = k < d.nu ? (uint32_t)tpack[d.u0 + k] : 0u;
    }
  };
  auto copies = [&](const Ids& d, int buf) {
    auto one = [&](int k, uint32_t pk) {
      const T* vp = v + 3 * (int64_t)(pk & 0x1FFFFFFFu);
      const uint32_t bits = pk >> 29;
      T* xk = vval(k);
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async<sizeof(T)>(xk + c, vp + c, ((bits >> c) & 1) ? 0 : (int)sizeof(T));
      cp_async<4>(tdb + buf * mu + k, tdest + d.u0 + k, 4);
    };
#pragma unroll
    for (int i = 0; i < GK; ++i) {
      const int k = tid + i * NT;
      if (k < d.nu) one(k, d.pk[i]);
    }
    for (int k = tid + GK * NT; k < d.nu; k += NT) one(k, (uint32_t)tpack[d.u0 + k]);
  };
  for (int k = tid; k < mu; k += NT) {
    I* a = sums(k);
    a[0] = a[1] = a[2] = I(0);
  }
  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0 && (int64_t)blockIdx.x < ntile) issue(blockIdx.x, 0);
  }
  Ids cur, nxt;
  cur.nu = nxt.nu = 0;
  if ((int64_t)blockIdx.x < ntile) {
    load_ids(tptr[blockIdx.x], tptr[blockIdx.x + 1], cur);
    copies(cur, 0);
  }
  cp_async_commit();
  if ((int64_t)blockIdx.x + gridDim.x < ntile)
    load_ids(tptr[blockIdx.x + gridDim.x], tptr[blockIdx.x + gridDim.x + 1], nxt);
  int32_t pu0 = 0, pu1 = 0;                                           // list bounds three tiles ahead
  if ((int64_t)blockIdx.x + 2 * (int64_t)gridDim.x < ntile) {
    pu0 = tptr[blockIdx.x + 2 * (int64_t)gridDim.x];
    pu1 = tptr[blockIdx.x + 2 * (int64_t)gridDim.x + 1];
  }
  int it = 0;
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x, ++it) {
    const int s = it & 1;
    const int64_t tn = t + gridDim.x;
    if constexpr (TMA) {
      if (tid == 0 && tn < ntile) issue(tn, s ^ 1);
    }
    const int nu = cur.nu;
    cp_async_wait<0>();                                                // this tile's copies have landed
    const T* g;
    const uint16_t* li;
    if constexpr (TMA) {
      const bool ok = mbar_wait_bounded(&bar[s], (uint32_t)((it >> 1) & 1), err);
      if (__syncthreads_or(!ok)) {
        // let the copies into the other stage finish (bounded) before leaving
        if (tid == 0 && tn < ntile) mbar_wait_bounded(&bar[s ^ 1], (uint32_t)(((it + 1) >> 1) & 1), nullptr);
        cp_async_wait<0>();
        return;
      }
      g = reinterpret_cast<const T*>(stage(s));
      li = reinterpret_cast<const uint16_t*>(stage(s) + L::GEO_B);
    } else {
      __syncthreads();
      g = geo + t * (GS * TT);
      li = lidx + t * NSLOT;
    }
    const int64_t rem = ne - t * TT;
    const int cnt = rem < TT ? (int)rem : TT;                         // elements in this tile
    // LANES = 2: the element pair at positions 2 tid, 2 tid + 1; LANES = 1: the
    // element at position tid (slots a*TT + position)
    uint32_t r0[NN], r1[NN];                                           // record byte offsets
    P f[NN][3];
    {
      P va[NN][3];
      if constexpr (LANES == 2) {
#pragma unroll
        for (int a = 0; a < NN; ++a) {
          const uint32_t lp = reinterpret_cast<const uint32_t*>(li + a * TT)[tid];   // both slots in one load
          r0[a] = (lp & 0xFFFFu) * (L::RW * 4);
          r1[a] = (lp >> 16) * (L::RW * 4);
        }
        T x0[NN][3];
#pragma unroll
        for (int a = 0; a < NN; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) x0[a][c] = reinterpret_cast<const T*>(rec + r0[a])[c];
#pragma unroll
        for (int b = 0; b < NN; ++b) {
          // a node the pair shares (face pairs: fixed local partner) is loaded once
          const int sb = pair_partner<ET>(b);
          const bool sh = sb >= 0 && r1[b] == r0[sb >= 0 ? sb : 0];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const T x1 = sh ? x0[sb >= 0 ? sb : 0][c] : reinterpret_cast<const T*>(rec + r1[b])[c];
            va[b][c] = P(x0[b][c], x1);
          }
        }
      } else {
#pragma unroll
        for (int a = 0; a < NN; ++a) {
          r0[a] = li[a * TT + tid] * (L::RW * 4);
          const T* x0 = reinterpret_cast<const T*>(rec + r0[a]);
#pragma unroll
          for (int c = 0; c < 3; ++c) va[a][c] = x0[c];
        }
      }
      const P* gp = reinterpret_cast<const P*>(g) + tid;
      const P* tp = J2 ? reinterpret_cast<const P*>(tan + t * (NG * 8 * TT)) + tid : nullptr;
      element_product<P, ET, J2, ELAME, NT>(gp, tp, va, P(lam_m), P(mu_m), P(K_m), f);
    }
    // positions past the end of the mesh (zero geometry, last tile only)
    // contribute nothing
    if (cnt < TT) {
      const bool ok0 = LANES * tid < cnt, ok1 = LANES * tid + 1 < cnt;
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if constexpr (LANES == 2) f[a][c] = P(ok0 ? f[a][c].lo() : T(0), ok1 ? f[a][c].hi() : T(0));
          else f[a][c] = ok0 ? f[a][c] : T(0);
        }
    }
    // tile-wide max |f| (NaN and infinity propagate)
    T m = T(0);
#pragma unroll
    for (int a = 0; a < NN; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if constexpr (LANES == 2) {
          m = max_nan(m, fabs(f[a][c].lo()));
          m = max_nan(m, fabs(f[a][c].hi()));
        } else {
          m = max_nan(m, fabs(f[a][c]));
        }
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) wmax[tid >> 5] = m;
    __syncthreads();
    T M = wmax[0];
#pragma unroll
    for (int w = 1; w < NW; ++w) M = max_nan(M, wmax[w]);
    // every element has read its node values: the next tile's may come in
    if (tn < ntile) copies(nxt, s ^ 1);
    cp_async_commit();
    cur = nxt;
    if (tn + gridDim.x < ntile) load_ids(pu0, pu1, nxt);
    if (tn + 2 * (int64_t)gridDim.x < ntile) {
      pu0 = tptr[tn + 2 * (int64_t)gridDim.x];
      pu1 = tptr[tn + 2 * (int64_t)gridDim.x + 1];
    }
    const bool bad = !(M <= std::numeric_limits<T>::max());            // NaN or infinity in the tile
    int e = 0;
    if (!bad && M > T(0)) {
      frexp(M * T(vmax), &e);                                          // vmax * M < 2^e
      e = max(e, B + std::numeric_limits<T>::min_exponent);          // keep q finite
    }
    const T q = bad ? T(1) : scalbn(T(1), B - e), iq = scalbn(T(1), e - B);
    if constexpr (LANES == 2) {
      P fq[NN][3];
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) fq[a][c] = P(f[a][c] * P(q));
      // the pair's shared nodes take one addition of both forces
#pragma unroll
      for (int a = 0; a < NN; ++a) {
        const int sa = pair_partner<ET>(a);
        const bool sh = sa >= 0 && r0[a] == r1[sa >= 0 ? sa : 0];
        I* d0 = reinterpret_cast<I*>(rec + r0[a] + L::ROFF);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T w = sh ? fq[a][c].lo() + fq[sa >= 0 ? sa : 0][c].hi() : fq[a][c].lo();
          atomicAdd(d0 + c, to_fixed(w));
        }
      }
#pragma unroll
      for (int b = 0; b < NN; ++b) {
        const int sb = pair_partner<ET>(b);
        const bool sh = sb >= 0 && r1[b] == r0[sb >= 0 ? sb : 0];
        if (!sh) {
          I* d1 = reinterpret_cast<I*>(rec + r1[b] + L::ROFF);
#pragma unroll
          for (int c = 0; c < 3; ++c) atomicAdd(d1 + c, to_fixed(fq[b][c].hi()));
        }
      }
    } else {
#pragma unroll
      for (int a = 0; a < NN; ++a) {
        I* a0 = reinterpret_cast<I*>(rec + r0[a] + L::ROFF);
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(a0 + c, to_fixed(f[a][c] * q));
      }
    }
    __syncthreads();
    // node sums back to T: a node listed by this tile only goes to y directly
    // (prescribed DOFs take v), the others' sums are stored (not added) at their
    // partials positions; the accumulators are cleared for the next tile
    const int32_t* td = tdb + s * mu;
    const T nan = std::numeric_limits<T>::quiet_NaN();
    for (int k = tid; k < nu; k += NT) {
      I* a = sums(k);
      T r[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r[c] = bad ? nan : from_fixed(a[c], T(0)) * iq;
        a[c] = I(0);
      }
      const int32_t d = td[k];
      if (d < 0) {
        const int64_t n3 = 3 * (int64_t)(d & 0x0FFFFFFF);
#pragma unroll
        for (int c = 0; c < 3; ++c) y[n3 + c] = (((uint32_t)d >> (28 + c)) & 1u) ? v[n3 + c] : r[c];
      } else {
        reinterpret_cast<Node4<T>*>(part)[d] = Node4<T>{r[0], r[1], r[2], T(0)};   // one 16-byte entry
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

// pass 2 over the nodes not listed by exactly one tile (ids with fixed-DOF bits
// at 28-30): y[3n+c] = fixed ? v : sum of node n's partials (a contiguous run of
// (x, y, z, 0) entries, tile order).  Each thread takes U nodes a grid stride apart, so that their loads are
// in flight together.
template <class T>
__global__ void mf_gather_kernel(int64_t nm, const int32_t* __restrict__ mnodes, const int32_t* __restrict__ mptr,
                                 const T* __restrict__ part, const T* __restrict__ v, T* __restrict__ y,
                                 const int* __restrict__ skip) {
  // U nodes per thread, the first R entries of each run loaded before any is added
  // (every load in flight at once); entries are still added in run order
  constexpr int U = 4, R = 2;
  if (skip && *skip) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const Node4<T>* P = reinterpret_cast<const Node4<T>*>(part);
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < nm; i0 += U * stride) {
    uint32_t id[U];
    int32_t q0[U], q1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * stride;
      id[u] = i < nm ? (uint32_t)mnodes[i] : 0u;
      q0[u] = i < nm ? mptr[i] : 0;
      q1[u] = i < nm ? mptr[i + 1] : 0;
    }
    Node4<T> w[U][R];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (q0[u] + r < q1[u]) w[u][r] = P[q0[u] + r];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (i0 + u * stride >= nm) break;
      T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (q0[u] + r < q1[u]) {
          s0 += w[u][r].x;
          s1 += w[u][r].y;
          s2 += w[u][r].z;
        }
      for (int32_t q = q0[u] + R; q < q1[u]; ++q) {
        const Node4<T> e = P[q];
        s0 += e.x;
        s1 += e.y;
        s2 += e.z;
      }
      const int64_t d = 3 * (int64_t)(id[u] & 0x0FFFFFFFu);
      const uint32_t bits = id[u] >> 28;
      y[d] = (bits & 1u) ? v[d] : s0;
      y[d + 1] = (bits & 2u) ? v[d + 1] : s1;
      y[d + 2] = (bits & 4u) ? v[d + 2] : s2;
    }
  }
}

// ---------------------------------------------------------------- launch
template <class T, int ET, bool J2, bool ELAME, int TT>
static int mf_go(exfem_block_s* b, const T* geo, const T* tan, const int32_t* tpack, const T* v, T* y, T* part,
                 const int* skip, cudaStream_t s) {
  constexpr bool TMA = sizeof(T) == 4;
  // lane pairs for the FP32 C3D10 product; one element per thread where pair
  // arithmetic would spill (C3D8's modal form, FP64)
  constexpr int LANES = (sizeof(T) == 4 && ET == EXFEM_C3D10) ? 2 : 1;
  using L = TileLayout<T, ET, TT, LANES, ELAME>;
  auto kern = mf_tile_kernel<T, ET, J2, ELAME, TT, LANES, TMA>;
  if (b->geo_stride != L::GS) {
    set_error("geometry stream stride %d does not match the kernel's %d", b->geo_stride, L::GS);
    return EXFEM_ERR_ARG;
  }
  const int mu = (b->maxu + 7) & ~7;
  const size_t smem = L::smem_bytes(TMA, mu);
  // The kernel's dynamic shared-memory limit is a process-wide attribute (per
  // device): it only ever grows, under a lock, so that a launch on one host thread
  // never finds it lowered by another thread's smaller mesh.  The persistent grid
  // is sized per (shared-memory size, device) from the occupancy query.
  static std::mutex attr_mu;
  static size_t opted_dev[64] = {0};
  static thread_local size_t q_smem = 0;
  static thread_local int per_sm = 0, nsm = 0, q_dev = -1;
  int cur;
  EX_CUDA(cudaGetDevice(&cur));
  if (cur < 0 || cur >= 64) {
    set_error("device ordinal %d out of range", cur);
    return EXFEM_ERR_UNSUPPORTED;
  }
  {
    std::lock_guard<std::mutex> lock(attr_mu);
    if (smem > opted_dev[cur]) {
      const size_t want = std::max<size_t>(smem, 48 * 1024);
      EX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want));
      opted_dev[cur] = want;
    }
  }
  if (smem != q_smem || cur != q_dev) {
    EX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cur));
    EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L::NT, smem));
    q_smem = smem;
    q_dev = cur;
  }
  if (per_sm < 1) {
    set_error("matrix-free tile kernel does not fit on an SM (%zu bytes of shared memory)", smem);
    return EXFEM_ERR_UNSUPPORTED;
  }
  const int64_t grid = std::min<int64_t>(b->ntile, (int64_t)nsm * per_sm);
  const int32_t* tdest = tpack == b->tile_nodes_bc.p ? b->tile_dest_bc.p : b->tile_dest.p;
  kern<<<(unsigned)grid, L::NT, smem, s>>>(b->ne, b->ntile, geo, b->lidx.p, tan, b->tile_ptr.p, tpack, tdest, v,
                                           y, part, (T)b->mat.lam, (T)b->mat.mu, (T)b->mat.K, mu, b->vmax, skip,
                                           b->dev_err.p);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template <class T, int ET, bool J2, bool ELAME>
static int mf_tile(exfem_block_s* b, const T* geo, const T* tan, const int32_t* tpack, const T* v, T* y, T* part,
                   const int* skip, cudaStream_t s) {
  switch (b->tile) {
    case 128: return mf_go<T, ET, J2, ELAME, 128>(b, geo, tan, tpack, v, y, part, skip, s);
    case 256: return mf_go<T, ET, J2, ELAME, 256>(b, geo, tan, tpack, v, y, part, skip, s);
    default:
      set_error("unsupported matrix-free tile size %d", b->tile);
      return EXFEM_ERR_UNSUPPORTED;
  }
}

template <class T, int ET>
static int mf_dispatch(exfem_block_s* b, const T* geo, const T* tan, const int32_t* tpack, const T* v, T* y,
                       T* part, const int* skip, cudaStream_t s) {
  if (b->mat.kind == EXFEM_J2) return mf_tile<T, ET, true, false>(b, geo, tan, tpack, v, y, part, skip, s);
  if (b->lam_e.p) return mf_tile<T, ET, false, true>(b, geo, tan, tpack, v, y, part, skip, s);
  return mf_tile<T, ET, false, false>(b, geo, tan, tpack, v, y, part, skip, s);
}

template <class T>
int launch_mf_matvec(exfem_block_s* b, const T* v, T* y, const int* skip, cudaStream_t s, bool bc) {
  const int64_t ndof = b->ndof();
  if (ndof == 0) return EXFEM_OK;
  if (b->etype == EXFEM_C3D10 && !b->affine) {
    set_error("matrix-free C3D10 needs straight-edged elements (mid-nodes at edge midpoints)");
    return EXFEM_ERR_UNSUPPORTED;
  }
  T* part = reinterpret_cast<T*>(b->partial.p);
  if (b->ne) {
    const T* geo;
    const T* tan;
    if constexpr (sizeof(T) == 8) {
      geo = (const T*)b->geo64.p;
      tan = (const T*)b->tan64.p;
    } else {
      geo = (const T*)b->geo32.p;
      tan = (const T*)b->tan32.p;
    }
    const int32_t* nf = (bc && b->fixed.p) ? b->tile_nodes_bc.p : b->tile_nodes.p;
    const int st = b->etype == EXFEM_C3D8 ? mf_dispatch<T, EXFEM_C3D8>(b, geo, tan, nf, v, y, part, skip, s)
                                          : mf_dispatch<T, EXFEM_C3D10>(b, geo, tan, nf, v, y, part, skip, s);
    if (st) return st;
  }
  if (b->nmulti) {
    const int32_t* mn = (bc && b->fixed.p) ? b->multi_nodes_bc.p : b->multi_nodes.p;
    mf_gather_kernel<T><<<grid_for((b->nmulti + 3) / 4, 256), 256, 0, s>>>(b->nmulti, mn, b->multi_ptr.p, part, v, y,
                                                                           skip);
  }
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template int launch_mf_matvec<float>(exfem_block_s*, const float*, float*, const int*, cudaStream_t, bool);
template int launch_mf_matvec<double>(exfem_block_s*, const double*, double*, const int*, cudaStream_t, bool);

}  // namespace exfem
