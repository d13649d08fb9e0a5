// Shared definitions for the exfem_b200 CUDA library: status codes, error
// capture, an owning device buffer, and small 3x3 tensor helpers used by the
// element kernels.  Everything here is internal; the public C ABI lives in
// include/exfem_b200.h.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <vector>

#include "../../include/exfem_b200.h"

namespace exfem {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what, const char* file, int line);
// status of the C++ exception being handled (call inside a catch clause): a C++
// exception never crosses the C ABI; host allocations that fail become
// EXFEM_ERR_OOM, sizes no host array can hold EXFEM_ERR_ARG
int host_exception();

#define EX_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) return ::exfem::cuda_status(_e, #call, __FILE__, __LINE__); \
  } while (0)

#define EX_LAUNCH_CHECK()                                                          \
  do {                                                                             \
    cudaError_t _e = cudaGetLastError();                                           \
    if (_e != cudaSuccess) return ::exfem::cuda_status(_e, "kernel launch", __FILE__, __LINE__); \
  } while (0)

#define EX_ARG(cond, ...)                                                          \
  do {                                                                             \
    if (!(cond)) {                                                                 \
      ::exfem::set_error(__VA_ARGS__);                                             \
      return EXFEM_ERR_ARG;                                                        \
    }                                                                              \
  } while (0)

// ---------------------------------------------------------------- captures and allocations
// cudaFree and cudaFreeHost synchronise the whole device, and a device-wide
// synchronisation invalidates a CUDA-graph capture that another host thread has in
// progress.  Captures hold capture_lock() shared for their duration; allocations
// and frees take it exclusively, so they wait for the captures in flight.  A
// thread never allocates inside its own capture (the capture would fail anyway),
// so it does not take the lock there (capturing_here()).
std::shared_mutex& capture_lock();
int& capturing_here();

struct CaptureScope {
  std::shared_lock<std::shared_mutex> lk;
  CaptureScope() : lk(capture_lock()) { capturing_here() = 1; }
  ~CaptureScope() { capturing_here() = 0; }
  CaptureScope(const CaptureScope&) = delete;
  CaptureScope& operator=(const CaptureScope&) = delete;
};

// run an allocation or free outside every other thread's capture
template <class F>
auto outside_captures(F f) -> decltype(f()) {
  if (capturing_here()) return f();
  std::unique_lock<std::shared_mutex> lk(capture_lock());
  return f();
}

// ---------------------------------------------------------------- device buffer
// Owning, non-copyable device allocation.  Allocation failures are reported
// through the status of the function that asked for the buffer.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) outside_captures([&] { return cudaFree(p); });
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    release();
    if (count == 0) return EXFEM_OK;
    cudaError_t e = outside_captures([&] { return cudaMalloc(&p, count * sizeof(T)); });
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
      return EXFEM_ERR_OOM;
    }
    n = count;
    return EXFEM_OK;
  }
  int upload(const T* host, size_t count) {
    int s = alloc(count);
    if (s) return s;
    if (count && host) EX_CUDA(cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    else if (count) EX_CUDA(cudaMemset(p, 0, count * sizeof(T)));   // nothing to copy: zero filled
    return EXFEM_OK;
  }
  size_t bytes() const { return n * sizeof(T); }
};

inline unsigned grid_for(size_t n, int block, unsigned cap = 148u * 16u) {
  size_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// ---------------------------------------------------------------- 3x3 helpers
// Matrices are row-major T[9]: m[3*i + j].
template <class T>
__host__ __device__ __forceinline__ T det3(const T* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// inverse by the adjugate; returns the determinant
template <class T>
__host__ __device__ __forceinline__ T inv3(const T* m, T* r) {
  T c00 = m[4] * m[8] - m[5] * m[7];
  T c01 = m[5] * m[6] - m[3] * m[8];
  T c02 = m[3] * m[7] - m[4] * m[6];
  T d = m[0] * c00 + m[1] * c01 + m[2] * c02;
  T id = T(1) / d;
  r[0] = c00 * id;
  r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = c01 * id;
  r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = c02 * id;
  r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return d;
}

}  // namespace exfem
