// Matrix-free element-by-element tangent product y = opA(v) in FP32 or FP64.
//
// Replaces the reference's forward-mode AD product K(u) v (gfem/model.py:488-490
// Model.tangent_jvp) and its stored-Ke product (gfem/model.py:264-267) inside
// opA (gfem/solvers.py:257-267):  y = free * K (free * v) + fixed * v.
//
// Work unit: a tile of MF_TILE = 128 consecutive elements, one CTA of 128 threads
// per tile, persistent over tiles.  Per tile:
//   1. element streams (geometry, tile-local node indices, J2 tangent data) are
//      one contiguous block each in the tile-major layout; in the FP32 kernel a
//      single thread moves them into shared memory with bulk TMA copies
//      (cp.async.bulk, mbarrier completion), double buffered so that the copy of
//      the next tile overlaps the work on this one;
//   2. v is gathered once per distinct node of the tile into shared memory —
//      ~3 distinct nodes per element instead of 8/10 node slots — with
//      asynchronous cp.async copies issued one tile ahead (fixed DOFs, whose bits
//      sit above the node id in the tile list, are zero filled), so the gather
//      of the next tile overlaps the arithmetic of this one;
//   3. one thread per element evaluates the element product from shared memory
//      (C3D8: modal B-bar form; C3D10: constant inverse Jacobian of the
//      straight-edged element) and accumulates it into per-node shared-memory
//      sums;
//   4. the tile's per-node sums are stored (plain stores, no atomics) at their
//      precomputed positions in a node-major partials buffer;
// and a second, node-centric pass forms y[n] = fixed ? v : the sum of node n's
// contiguous run of tile entries, in tile order (the reference's atomic-free
// gather-plan assembly, gfem/model.py:241-267, at tile granularity).  The
// product is deterministic.
// Geometry: C3D8 stores the 7 modal coordinate vectors (coordinates with the
// centroid removed) and the stiffness scale; C3D10 stores the inverse Jacobian
// and scaled volume, formed in FP64 from the nodal coordinates and rounded once.
#include "internal.h"

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
// bounded wait: gives up after ~2^24 polls, records the failure and returns false
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err) {
  for (int i = 0; i < (1 << 24); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, 1);
  return false;
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
// (tn points to component 0 of this element/point, stride MF_TILE)
template <class T, bool J2>
__device__ __forceinline__ void mf_stress(const T* tn, T lam, T mu, T Kb, const T (&e)[6], T (&s)[6]) {
  if constexpr (J2) {
    T t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = tn[k * MF_TILE];
    tangent_stress(Kb, mu, t, e, s);
  } else {
    elastic_stress(lam, mu, e, s);
  }
}

// element product f = Ke v_e from the element's streams (strided by MF_TILE)
template <class T, int ET, bool J2>
__device__ __forceinline__ void element_product(const T* g, const T* tn, const T (&va)[ElemTraits<ET>::nnode][3],
                                                T lam, T mu, T Kb, T (&f)[ElemTraits<ET>::nnode][3]) {
  if constexpr (ET == EXFEM_C3D8) {
    T cm[7][3], um[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) cm[k][c] = g[(3 * k + c) * MF_TILE];
    const T sc = g[21 * MF_TILE];
    const T le = g[22 * MF_TILE], me = J2 ? mu : g[23 * MF_TILE];
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
      mf_stress<T, J2>(tn + q * 8 * MF_TILE, le, me, Kb, ee, s);
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
    hex_from_modal(Fm, f);
  } else {
    // C3D10 with a constant Jacobian, in barycentric form: with L the
    // barycentric coordinates, w_j = du/dL_j = base_j + D * (g == j ? v_j : v_e(j,g))
    // at Gauss point g (L_g = A, others B), base_j = (4B-1) v_j + 4B sum of the
    // edge nodes at corner j, D = 4(A-B); the reference gradient is
    // G_i = w_{i+1} - w_0.  The force is the adjoint of the same steps.
    constexpr T A = T(TET_A), B = T(TET_B);
    constexpr T D = T(4.0 * (TET_A - TET_B)), C0 = T(4.0 * TET_B - 1.0), C1 = T(4.0 * TET_B);
    T iJ[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) iJ[k] = g[k * MF_TILE];
    const T vol = g[9 * MF_TILE];
    const T le = g[10 * MF_TILE], me = J2 ? mu : g[11 * MF_TILE];
    (void)A;
    (void)B;
    T base[4][3], vbar[10][3], bbar[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      base[0][c] = C0 * va[0][c] + C1 * (va[4][c] + va[6][c] + va[7][c]);
      base[1][c] = C0 * va[1][c] + C1 * (va[4][c] + va[5][c] + va[8][c]);
      base[2][c] = C0 * va[2][c] + C1 * (va[5][c] + va[6][c] + va[9][c]);
      base[3][c] = C0 * va[3][c] + C1 * (va[7][c] + va[8][c] + va[9][c]);
    }
#pragma unroll
    for (int a = 0; a < 10; ++a) vbar[a][0] = vbar[a][1] = vbar[a][2] = T(0);
#pragma unroll
    for (int j = 0; j < 4; ++j) bbar[j][0] = bbar[j][1] = bbar[j][2] = T(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      T w[4][3];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int src = jj == q ? jj : tet_edge_node(jj, q);
#pragma unroll
        for (int c = 0; c < 3; ++c) w[jj][c] = base[jj][c] + D * va[src][c];
      }
      T G[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) G[3 * c + i] = w[i + 1][c] - w[0][c];
      T H[9];
      matmul3t(G, iJ, H);
      T ee[6], s[6];
      sym_from_grad(H, ee);
      mf_stress<T, J2>(tn + q * 8 * MF_TILE, le, me, Kb, ee, s);
      const T r[3][3] = {{vol * s[0], vol * s[3], vol * s[5]},
                         {vol * s[3], vol * s[1], vol * s[4]},
                         {vol * s[5], vol * s[4], vol * s[2]}};
      T Q[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) Q[3 * i + k] = r[i][0] * iJ[3 * k] + r[i][1] * iJ[3 * k + 1] + r[i][2] * iJ[3 * k + 2];
      // adjoint: wbar_{i+1} = Q[:, i], wbar_0 = -sum_i Q[:, i]
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T wb[4];
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
      const T e0 = C1 * bbar[0][c], e1 = C1 * bbar[1][c], e2 = C1 * bbar[2][c], e3 = C1 * bbar[3][c];
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

template <class T, int ET, bool J2>
struct TileLayout {
  using Tr = ElemTraits<ET>;
  static constexpr int NN = Tr::nnode, NG = Tr::ngp, GS = Tr::geo_stride, NSLOT = NN * MF_TILE;
  static constexpr uint32_t GEO_B = GS * MF_TILE * sizeof(T);
  static constexpr uint32_t LIDX_B = NSLOT * sizeof(uint16_t);
  static constexpr uint32_t TAN_B = J2 ? NG * 8 * MF_TILE * sizeof(T) : 0;
  static constexpr uint32_t STAGE_B = GEO_B + LIDX_B + TAN_B;
  static_assert(GEO_B % 16 == 0 && LIDX_B % 16 == 0 && TAN_B % 16 == 0, "bulk copies need 16-byte multiples");
};

template <class T, int ET, bool J2, bool TMA>
__global__ void __launch_bounds__(MF_TILE)
mf_tile_kernel(int64_t ne, int64_t ntile, const T* __restrict__ geo, const uint16_t* __restrict__ lidx,
               const T* __restrict__ tan, const int32_t* __restrict__ tptr, const int32_t* __restrict__ tpack,
               const int32_t* __restrict__ tdest, const T* __restrict__ v, T* __restrict__ part, T lam, T mu,
               T Kb, int maxu, const int* __restrict__ skip, int* __restrict__ err) {
  using L = TileLayout<T, ET, J2>;
  constexpr int NN = L::NN, NG = L::NG, GS = L::GS, NSLOT = L::NSLOT;
  if (skip && *skip) return;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  const int tid = threadIdx.x;
  // element of the tile handled by this thread: lanes of a warp take every 4th
  // element, so the elements that share corner nodes (neighbours in the mesh
  // order) fall into different warps and their shared-memory additions to the
  // same node rarely collide inside one warp instruction
  const int lt = 4 * (tid & 31) + (tid >> 5);
  T* xsb[2];                                                          // gathered v, double buffered
  xsb[0] = reinterpret_cast<T*>(smem + (TMA ? 2 * L::STAGE_B : 0));
  xsb[1] = xsb[0] + 3 * maxu;
  T* ys = xsb[1] + 3 * maxu;                                          // accumulated products
  auto stage_geo = [&](int s) { return reinterpret_cast<T*>(smem + s * L::STAGE_B); };
  auto stage_lidx = [&](int s) { return reinterpret_cast<uint16_t*>(smem + s * L::STAGE_B + L::GEO_B); };
  auto stage_tan = [&](int s) { return reinterpret_cast<T*>(smem + s * L::STAGE_B + L::GEO_B + L::LIDX_B); };
  auto issue = [&](int64_t t, int s) {
    fence_proxy_async();
    mbar_expect_tx(&bar[s], L::STAGE_B);
    bulk_g2s(stage_geo(s), geo + t * (GS * MF_TILE), L::GEO_B, &bar[s]);
    bulk_g2s(stage_lidx(s), lidx + t * NSLOT, L::LIDX_B, &bar[s]);
    if constexpr (J2) bulk_g2s(stage_tan(s), tan + t * (NG * 8 * MF_TILE), L::TAN_B, &bar[s]);
  };
  // asynchronous gather of the tile's distinct nodes (fixed DOFs zero filled)
  auto gather = [&](int64_t t, T* xs) {
    const int64_t u0 = tptr[t];
    const int nu = tptr[t + 1] - (int32_t)u0;
    for (int k = tid; k < nu; k += MF_TILE) {
      const uint32_t pk = (uint32_t)tpack[u0 + k];
      const int64_t n = pk & 0x1FFFFFFFu;
      const uint32_t bits = pk >> 29;
      const T* vp = v + 3 * n;
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async<sizeof(T)>(xs + c * maxu + k, vp + c, ((bits >> c) & 1) ? 0 : (int)sizeof(T));
    }
    cp_async_commit();
  };
  for (int k = tid; k < 3 * maxu; k += MF_TILE) ys[k] = T(0);
  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0 && (int64_t)blockIdx.x < ntile) issue(blockIdx.x, 0);
  }
  if ((int64_t)blockIdx.x < ntile) gather(blockIdx.x, xsb[0]);
  __syncthreads();
  int it = 0;
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x, ++it) {
    const int s = it & 1;
    const int64_t tn = t + gridDim.x;
    if constexpr (TMA) {
      if (tid == 0 && tn < ntile) issue(tn, s ^ 1);
    }
    if (tn < ntile) gather(tn, xsb[s ^ 1]);
    else cp_async_commit();                                            // keep one group per iteration
    cp_async_wait<1>();                                                // this tile's gather has landed
    const T* g;
    const uint16_t* li;
    const T* tnp;
    if constexpr (TMA) {
      const bool ok = mbar_wait_bounded(&bar[s], (uint32_t)((it >> 1) & 1), err);
      if (__syncthreads_or(!ok)) {
        cp_async_wait<0>();
        return;
      }
      g = stage_geo(s);
      li = stage_lidx(s);
      tnp = J2 ? stage_tan(s) : nullptr;
    } else {
      __syncthreads();
      g = geo + t * (GS * MF_TILE);
      li = lidx + t * NSLOT;
      tnp = J2 ? tan + t * (NG * 8 * MF_TILE) : nullptr;
    }
    const T* xs = xsb[s];
    const int64_t e = t * MF_TILE + lt;
    if (e < ne) {
      int l[NN];
      T va[NN][3];
#pragma unroll
      for (int a = 0; a < NN; ++a) {
        l[a] = li[a * MF_TILE + lt];
#pragma unroll
        for (int c = 0; c < 3; ++c) va[a][c] = xs[c * maxu + l[a]];
      }
      T f[NN][3];
      element_product<T, ET, J2>(g + lt, J2 ? tnp + lt : nullptr, va, lam, mu, Kb, f);
#pragma unroll
      for (int a = 0; a < NN; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(&ys[c * maxu + l[a]], f[a][c]);
    }
    __syncthreads();
    // the tile's per-node sums, stored (not added) at their node-major positions
    const int64_t u0 = tptr[t];
    const int nu = tptr[t + 1] - (int32_t)u0;
    for (int k = tid; k < nu; k += MF_TILE) {
      T* p = part + 3 * (int64_t)tdest[u0 + k];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        p[c] = ys[c * maxu + k];
        ys[c * maxu + k] = T(0);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

// pass 2: y[3n+c] = fixed ? v : sum of node n's tile entries (a contiguous run
// in node-major order, tile order inside the run)
template <class T>
__global__ void mf_gather_kernel(int64_t nn, const int32_t* __restrict__ node_ptr, const T* __restrict__ part,
                                 const uint8_t* __restrict__ fixed, const T* __restrict__ v, T* __restrict__ y,
                                 const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    T s0 = T(0), s1 = T(0), s2 = T(0);
    const int32_t q1 = node_ptr[n + 1];
    for (int32_t q = node_ptr[n]; q < q1; q += 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (q + u < q1) {
          const T* p = part + 3 * (int64_t)(q + u);
          s0 += p[0];
          s1 += p[1];
          s2 += p[2];
        }
    }
    const int64_t d = 3 * n;
    if (fixed) {
      y[d] = fixed[d] ? v[d] : s0;
      y[d + 1] = fixed[d + 1] ? v[d + 1] : s1;
      y[d + 2] = fixed[d + 2] ? v[d + 2] : s2;
    } else {
      y[d] = s0;
      y[d + 1] = s1;
      y[d + 2] = s2;
    }
  }
}

// ---------------------------------------------------------------- launch
template <class T, int ET, bool J2>
static int mf_go(exfem_block_s* b, const T* geo, const T* tan, const int32_t* tpack, const T* v, T* part,
                 const int* skip, cudaStream_t s) {
  constexpr bool TMA = sizeof(T) == 4;
  using L = TileLayout<T, ET, J2>;
  auto kern = mf_tile_kernel<T, ET, J2, TMA>;
  const size_t smem = (TMA ? 2 * (size_t)L::STAGE_B : 0) + 3 * 3 * (size_t)b->maxu * sizeof(T);
  // per (kernel, shared-memory size): opt in above 48 KB and size the persistent grid
  static thread_local size_t opted = 0;
  static thread_local int per_sm = 0, nsm = 0, dev = -1;
  int cur;
  EX_CUDA(cudaGetDevice(&cur));
  if (smem > opted || cur != dev) {
    EX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
    EX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cur));
    EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MF_TILE, smem));
    opted = smem;
    dev = cur;
  }
  if (per_sm < 1) {
    set_error("matrix-free tile kernel does not fit on an SM (%zu bytes of shared memory)", smem);
    return EXFEM_ERR_UNSUPPORTED;
  }
  const int64_t grid = std::min<int64_t>(b->ntile, (int64_t)nsm * per_sm);
  kern<<<(unsigned)grid, MF_TILE, smem, s>>>(b->ne, b->ntile, geo, b->lidx.p, tan, b->tile_ptr.p, tpack,
                                             b->tile_dest.p, v, part, (T)b->mat.lam, (T)b->mat.mu, (T)b->mat.K,
                                             b->maxu, skip, b->dev_err.p);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
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
    const bool j2 = b->mat.kind == EXFEM_J2;
    const int32_t* nf = (bc && b->fixed.p) ? b->tile_nodes_bc.p : b->tile_nodes.p;
    int st;
    if (b->etype == EXFEM_C3D8)
      st = j2 ? mf_go<T, EXFEM_C3D8, true>(b, geo, tan, nf, v, part, skip, s)
              : mf_go<T, EXFEM_C3D8, false>(b, geo, tan, nf, v, part, skip, s);
    else
      st = j2 ? mf_go<T, EXFEM_C3D10, true>(b, geo, tan, nf, v, part, skip, s)
              : mf_go<T, EXFEM_C3D10, false>(b, geo, tan, nf, v, part, skip, s);
    if (st) return st;
  }
  mf_gather_kernel<T><<<grid_for(b->nn, 256), 256, 0, s>>>(b->nn, b->node_ptr.p, part, bc ? b->fixed.p : nullptr,
                                                           v, y, skip);
  EX_LAUNCH_CHECK();
  return EXFEM_OK;
}

template int launch_mf_matvec<float>(exfem_block_s*, const float*, float*, const int*, cudaStream_t, bool);
template int launch_mf_matvec<double>(exfem_block_s*, const double*, double*, const int*, cudaStream_t, bool);

}  // namespace exfem
