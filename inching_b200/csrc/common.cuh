// Shared helpers for the inching_b200 kernels: status handling, warp utilities.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <cuda_runtime.h>

#include "../../include/inching_b200.h"

namespace inch {

// Thread-local message of the last error returned to this host thread.
void set_error(const char* fmt, ...);

#define INCH_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess) {                                                         \
      ::inch::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
      return INCH_CUDA_ERROR;                                                        \
    }                                                                                \
  } while (0)

#define INCH_LAUNCH_CHECK() INCH_CUDA(cudaGetLastError())

#define INCH_REQUIRE(cond, code, ...)                                                \
  do {                                                                               \
    if (!(cond)) {                                                                   \
      ::inch::set_error(__VA_ARGS__);                                                \
      return (code);                                                                 \
    }                                                                                \
  } while (0)

// Carve aligned sub-buffers out of a caller workspace.
struct Carver {
  char* base;
  size_t cap;
  size_t off = 0;
  bool ok = true;
  Carver(void* p, size_t n) : base(static_cast<char*>(p)), cap(n) {}
  template <class T>
  T* take(size_t count) {
    size_t a = (off + 255) & ~size_t(255);
    size_t need = a + count * sizeof(T);
    if (base == nullptr || need > cap) {
      ok = false;
      off = need;
      return nullptr;
    }
    off = need;
    return reinterpret_cast<T*>(base + a);
  }
};

// Size-only counterpart of Carver.
struct Sizer {
  size_t off = 0;
  template <class T>
  void take(size_t count) {
    off = ((off + 255) & ~size_t(255)) + count * sizeof(T);
  }
  size_t bytes() const { return off + 256; }
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

inline int grid_for(int64_t work, int per_block, int cap = 148 * 32) {
  int64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}

}  // namespace inch
