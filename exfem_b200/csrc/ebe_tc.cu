// Stored-Ke product for many right-hand sides on the 5th-generation tensor cores.
//
// Y = opA(V) for nrhs <= 16 right-hand sides at once, with the element matrices Ke
// stored in BF16 (the output of exfem_element_stiffness with dtype BF16) and the
// right-hand sides rounded to BF16, accumulated in FP32 in tensor memory
// (tcgen05.mma kind::f16).  This is the multi-right-hand-side variant of the
// reference's stored-Ke product (gfem/model.py:264-267 gather_matvec; the vmapped
// multi-load-case solve of gfem/optimize.py:116-143), where Ke.U is a dense
// contraction: one BF16 Ke read serves every right-hand side.
//
// Work unit: a group of G elements (C3D8: 5 x 24 rows, C3D10: 4 x 32 rows with
// 2 zero rows each) forms one M = 128 x K = 128 tile.  A (shared memory) is
// block-diagonal with the G element matrices on its diagonal, B holds the G
// elements' nodal values, K-major, N = 16 columns (right-hand sides, zero
// padded).  Eight MMAs of K = 16 issued by one thread accumulate D = A B in
// tensor memory (128 lanes x 16 FP32 columns); each warp reads its 32 lanes back
// with tcgen05.ld and writes the element product rows.  A second kernel sums the
// element rows of every node through the gather plan (gfem/model.py:241-267, the
// reference's atomic-free order) and applies opA's prescribed-DOF rows.
//
// Shared-memory operands use the no-swizzle K-major canonical layout: 8 x 16-byte
// core matrices, the 8-row groups 128 bytes apart (SBO) and the 16-byte K chunks
// of a row group 128*(rows/8) bytes apart (LBO).  Only the diagonal core matrices
// of A are rewritten per group; the zeros elsewhere are written once.
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.h"

namespace exfem {

namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: gives up after ~2^24 polls and returns false
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  for (int i = 0; i < (1 << 24); ++i)
    if (bar_try_wait(bar, parity)) return true;
  return false;
}

// shared-memory matrix descriptor, no swizzle, K-major (canonical layout above)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;                           // descriptor version of sm_100
  return d;                                         // base offset 0, layout type 0 (no swizzle)
}

constexpr int TC_M = 128, TC_K = 128, TC_N = 16;
// instruction descriptor: D F32, A and B BF16, both K-major, N = 16, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);
constexpr uint32_t A_BYTES = TC_M * TC_K * 2;       // 32 KB
constexpr uint32_t B_BYTES = TC_N * TC_K * 2;       // 4 KB
constexpr uint32_t A_LBO = (TC_M / 8) * 128, A_SBO = 128;
constexpr uint32_t B_LBO = (TC_N / 8) * 128, B_SBO = 128;

// byte offset of element (row, k) of a K-major operand with `rows` rows
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int rows) {
  return (uint32_t)(((row >> 3) + (k >> 3) * (rows >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

template <int ET>
struct TcShape {
  static constexpr int NN = ElemTraits<ET>::nnode, ND = 3 * NN;
  static constexpr int NDP = (ND + 7) & ~7;         // rows per element in the tile (multiple of 8)
  static constexpr int G = TC_M / NDP;              // elements per tile
};

}  // namespace

// ys[(e*nd + i)*nrhs + r] = sum_j Ke[e, i, j] * bf16(free * V)[dof(e, j), r]
//
// Two-stage pipeline per CTA over its groups (stage s = group parity): while the
// tensor cores run group i out of shared-memory stage s into tensor-memory columns
// 16 s .. 16 s + 15, the CTA waits for group i-1's MMAs, starts the asynchronous
// copies of group i+1's Ke into the other stage, loads group i+1's nodal values
// into registers, and reads group i-1's products out of tensor memory.
template <int ET, int NR>
__global__ void __launch_bounds__(128)
ebe_tc_kernel(int64_t ne, const int32_t* __restrict__ conn, const __nv_bfloat16* __restrict__ Ke,
              const float* __restrict__ V, const uint8_t* __restrict__ fixed, float* __restrict__ ys,
              int* __restrict__ err) {
  using S = TcShape<ET>;
  constexpr int NN = S::NN, ND = S::ND, NDP = S::NDP, G = S::G;
  constexpr int nrhs = NR;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr int VPT = (G * ND * NR + 127) / 128;      // prefetched nodal values per thread
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023);
  auto As = [&](int s) { return base + s * STAGE; };
  auto Bs = [&](int s) { return base + s * STAGE + A_BYTES; };
  __shared__ __align__(8) uint64_t mma_bar[2];
  __shared__ uint32_t tmem_base_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t ngroup = (ne + G - 1) / G;

  for (int k = tid; k < 2 * STAGE / 16; k += 128) reinterpret_cast<uint4*>(base)[k] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    bar_init(&mma_bar[0], 1);
    bar_init(&mma_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base_s)),
                 "r"(32));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  bool failed = false;                                // CTA-uniform: a bounded wait gave up

  // Ke of a group into stage s: asynchronous 16-byte copies where the element rows
  // allow (C3D8: 48-byte rows), 4-byte copies otherwise; rows past the mesh are zero
  auto fill_a = [&](int64_t grp, int s) {
    const int64_t e0 = grp * G;
    unsigned char* A = As(s);
    if constexpr ((ND * 2) % 16 == 0) {
      constexpr int CH = ND * 2 / 16;                 // 16-byte chunks per row
      for (int q = tid; q < G * ND * CH; q += 128) {
        const int g = q / (ND * CH), rem = q - g * (ND * CH), i = rem / CH, j = 8 * (rem - i * CH);
        const int64_t e = e0 + g;
        const uint32_t dst = smem_addr(A + kmajor_off(g * NDP + i, g * NDP + j, TC_M));
        const __nv_bfloat16* src = Ke + ((e < ne ? e : 0) * ND + i) * ND + j;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(e < ne ? 16 : 0)
                     : "memory");
      }
    } else {
      for (int q = tid; q < G * ND * (ND / 2); q += 128) {
        const int g = q / (ND * (ND / 2)), rem = q - g * (ND * (ND / 2)), i = rem / (ND / 2);
        const int j = 2 * (rem - i * (ND / 2));
        const int64_t e = e0 + g;
        const uint32_t dst = smem_addr(A + kmajor_off(g * NDP + i, g * NDP + j, TC_M));
        const __nv_bfloat16* src = Ke + ((e < ne ? e : 0) * ND + i) * ND + j;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(e < ne ? 4 : 0)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // nodal values of a group (prescribed DOFs zero) into registers
  float vr[VPT];
  // (all node ids first, then every value and mask load in flight together; the
  // mask is applied with a select so that no load waits for another's result)
  auto load_v = [&](int64_t grp) {
    const int64_t e0 = grp * G;
    int64_t dv[VPT];
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const int q = tid + 128 * u;
      dv[u] = -1;
      if (q < G * ND * nrhs) {
        const int g = q / (ND * nrhs), rem = q - g * (ND * nrhs), i = rem / nrhs, r = rem - i * nrhs;
        const int64_t e = e0 + g;
        if (e < ne) dv[u] = (3 * (int64_t)__ldg(conn + e * NN + i / 3) + i % 3) * nrhs + r;
      }
    }
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const int64_t k = dv[u] < 0 ? 0 : dv[u];
      const float x = __ldg(V + k);
      const bool off = dv[u] < 0 || (fixed && __ldg(fixed + k / nrhs));
      vr[u] = off ? 0.0f : x;
    }
  };
  auto store_b = [&](int s) {
    unsigned char* B = Bs(s);
#pragma unroll
    for (int u = 0; u < VPT; ++u) {
      const int q = tid + 128 * u;
      if (q < G * ND * nrhs) {
        const int g = q / (ND * nrhs), rem = q - g * (ND * nrhs), i = rem / nrhs, r = rem - i * nrhs;
        *reinterpret_cast<__nv_bfloat16*>(B + kmajor_off(r, g * NDP + i, TC_N)) = __float2bfloat16_rn(vr[u]);
      }
    }
  };
  auto epilogue = [&](int64_t grp, int s) {
    uint32_t d[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
          "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
        : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(TC_N * s)));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int row = 32 * warp + lane;
    const int g = row / NDP, i = row - g * NDP;
    const int64_t e = grp * G + g;
    if (g < G && i < ND && e < ne) {
      float* out = ys + (e * ND + i) * nrhs;
      if ((nrhs & 3) == 0) {
#pragma unroll
        for (int r = 0; r < TC_N; r += 4)
          if (r < nrhs)
            *reinterpret_cast<float4*>(out + r) = make_float4(__uint_as_float(d[r]), __uint_as_float(d[r + 1]),
                                                              __uint_as_float(d[r + 2]), __uint_as_float(d[r + 3]));
      } else {
#pragma unroll
        for (int r = 0; r < TC_N; ++r)
          if (r < nrhs) out[r] = __uint_as_float(d[r]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };

  const int64_t g0 = blockIdx.x, gs = gridDim.x;
  if (g0 < ngroup) {
    fill_a(g0, 0);
    load_v(g0);
  }
  int it = 0;
  for (int64_t grp = g0; grp < ngroup; grp += gs, ++it) {
    const int s = it & 1;
    // 1. this group's operands are in stage s
    store_b(s);
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic / async-copy stores -> tensor-core reads
    __syncthreads();
    // 2. its MMAs into tensor-memory columns 16 s ..
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_addr(As(s)), b0 = smem_addr(Bs(s));
#pragma unroll
      for (int k = 0; k < TC_K / 16; ++k) {
        const uint64_t ad = smem_desc(a0 + k * 2 * A_LBO, A_LBO, A_SBO);
        const uint64_t bd = smem_desc(b0 + k * 2 * B_LBO, B_LBO, B_SBO);
        const uint32_t acc = k > 0 ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(
                tmem + (uint32_t)(TC_N * s)),
            "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&mma_bar[s]))
                   : "memory");
    }
    // 3. the previous group's MMAs have finished: its stage and columns are free
    if (it > 0) {
      const bool ok = bar_wait(&mma_bar[s ^ 1], (uint32_t)(((it - 1) >> 1) & 1));
      if (__syncthreads_or(!ok)) {
        failed = true;
        ++it;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // 4. the next group's Ke and nodal values start coming in
    const int64_t nxt = grp + gs;
    if (nxt < ngroup) {
      fill_a(nxt, s ^ 1);
      load_v(nxt);
    }
    // 5. the previous group's products out of tensor memory
    if (it > 0) epilogue(grp - gs, s ^ 1);
  }
  // the last group
  if (it > 0 && !failed) {
    const int s = (it - 1) & 1;
    const bool ok = bar_wait(&mma_bar[s], (uint32_t)(((it - 1) >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      epilogue(g0 + (int64_t)(it - 1) * gs, s);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  if (failed && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32));
  }
}

template <int ET>
static int tc_launch(exfem_block_s* b, const __nv_bfloat16* Ke, int nrhs, const float* V, const uint8_t* fx,
                     cudaStream_t s) {
  const size_t smem = 2 * (A_BYTES + B_BYTES) + 1024;
  int dev, nsm;
  EX_CUDA(cudaGetDevice(&dev));
  EX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int64_t ng = (b->ne + TcShape<ET>::G - 1) / TcShape<ET>::G;
  const unsigned grid = (unsigned)std::min<int64_t>(ng, (int64_t)nsm * 3);
  auto go = [&](auto kern) -> int {
    EX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, 128, smem, s>>>(b->ne, b->conn.p, Ke, V, fx, b->ys_tc.p, b->dev_err.p);
    EX_LAUNCH_CHECK();
    return EXFEM_OK;
  };
  switch (nrhs) {
    case 1: return go(ebe_tc_kernel<ET, 1>);
    case 2: return go(ebe_tc_kernel<ET, 2>);
    case 3: return go(ebe_tc_kernel<ET, 3>);
    case 4: return go(ebe_tc_kernel<ET, 4>);
    case 8: return go(ebe_tc_kernel<ET, 8>);
    case 16: return go(ebe_tc_kernel<ET, 16>);
    default:
      set_error("the tensor-core stored-Ke product takes 1, 2, 3, 4, 8 or 16 right-hand sides, got %d", nrhs);
      return EXFEM_ERR_ARG;
  }
}

int launch_ebe_matvec_tc(exfem_block_s* b, const __nv_bfloat16* Ke, int nrhs, const float* V, float* Y,
                         cudaStream_t s, bool bc) {
  if (nrhs < 1 || nrhs > TC_N) {
    set_error("the tensor-core stored-Ke product takes 1..%d right-hand sides, got %d", TC_N, nrhs);
    return EXFEM_ERR_ARG;
  }
  int st;
  const size_t need = (size_t)b->ne * b->nd * nrhs;
  if (b->ys_tc.n < need && (st = b->ys_tc.alloc(need))) return st;
  if (b->ne) {
    const uint8_t* fx = bc ? b->fixed.p : nullptr;
    const int st = b->etype == EXFEM_C3D8 ? tc_launch<EXFEM_C3D8>(b, Ke, nrhs, V, fx, s)
                                          : tc_launch<EXFEM_C3D10>(b, Ke, nrhs, V, fx, s);
    if (st) return st;
  }
  return launch_gather_multi<float>(b, b->ys_tc.p, V, Y, nrhs, bc, s);
}

}  // namespace exfem
