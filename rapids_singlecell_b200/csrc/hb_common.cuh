// Shared definitions for the B200 Harmony engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/harmony_b200.h"

namespace hb {

constexpr int kNumBins = 4096;      // first radix level of the block splitter select (12 key bits)
constexpr int kBinShift = 20;
constexpr int kPartTile = 2048;     // cells per tile of the stable block partition
constexpr int kMaxBlocks = 512;     // most block updates per k-means iteration
constexpr int kMaxIterChunk = 8;    // k-means iterations whose block lists are built per launch
constexpr int kMaxBuckets = 4096;   // (block, batch) buckets of the stable partition

// Shuffle key of cell i for one k-means iteration.  This is the PCG-RXS-M-XS
// 32-bit hash (M. O'Neill, "PCG: a family of simple fast space-efficient
// statistically good algorithms for random number generation", 2014) applied
// to i ^ seed; the reference orders cells by exactly this key
// (_cuda/harmony/clustering/kernels_clustering.cuh:106-117), so the constants
// are part of the algorithm's definition.  The map is a bijection on 32-bit
// words: keys of distinct cells never tie.
__host__ __device__ __forceinline__ uint32_t pcg_key(uint32_t i, uint32_t seed) {
  uint32_t st = i ^ seed;
  st = st * 747796405u + 2891336453u;
  uint32_t w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
  return (w >> 22u) ^ w;
}

template <typename T> struct num;
template <> struct num<float> {
  static __device__ __forceinline__ float exp_(float x) { return expf(x); }
  static __device__ __forceinline__ float log_(float x) { return logf(x); }
  static __device__ __forceinline__ float pow_(float a, float b) { return powf(a, b); }
  static __device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
};
template <> struct num<double> {
  static __device__ __forceinline__ double exp_(double x) { return exp(x); }
  static __device__ __forceinline__ double log_(double x) { return log(x); }
  static __device__ __forceinline__ double pow_(double a, double b) { return pow(a, b); }
  static __device__ __forceinline__ double rsqrt_(double x) { return rsqrt(x); }
};

// storage <-> compute conversions
__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ double to_f(double x) { return x; }
__device__ __forceinline__ float to_f(__half x) { return __half2float(x); }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
template <typename S> __device__ __forceinline__ S from_f(float x);
template <typename S> __device__ __forceinline__ S from_f(double x);
template <> __device__ __forceinline__ float from_f<float>(float x) { return x; }
template <> __device__ __forceinline__ double from_f<double>(double x) { return x; }
template <> __device__ __forceinline__ float from_f<float>(double x) { return (float)x; }
template <> __device__ __forceinline__ double from_f<double>(float x) { return x; }
template <> __device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }

// A launch gated on a device flag (the run has stopped): true when the kernel must return at once.
// The flag is written by an earlier launch on the same stream, so every CTA reads the same value.
__device__ __forceinline__ bool gated(const int* gate) { return gate && *(volatile const int*)gate; }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum over all threads of a (1-, 2- or 3-D) block; every thread
// receives the total.  `red` needs 32 slots; the thread count must be a
// multiple of 32.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, w = tid >> 5;
  const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T t = (tid < nw) ? red[tid] : T(0);
  if (w == 0) t = warp_sum(t);
  if (tid == 0) red[0] = t;
  __syncthreads();
  T r = red[0];
  __syncthreads();
  return r;
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Bump allocator over the caller's workspace (the library never calls cudaMalloc).
struct Carver {
  char* base;
  size_t off = 0;
  size_t cap;
  bool dry;
  Carver(void* b, size_t c) : base((char*)b), cap(c), dry(b == nullptr) {}
  template <typename T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = dry ? nullptr : (T*)(base + off);
    off += count * sizeof(T);
    return p;
  }
  bool ok() const { return dry || off <= cap; }
};

void set_error(const char* fmt, ...);

#define HB_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::hb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
      return HB_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

extern thread_local int64_t g_launches;  // kernels launched by this thread (profiling)

#define HB_LAUNCH_CHECK()                                                          \
  do {                                                                             \
    ++::hb::g_launches;                                                            \
    cudaError_t _e = cudaGetLastError();                                           \
    if (_e != cudaSuccess) {                                                       \
      ::hb::set_error("%s:%d launch failed: %s", __FILE__, __LINE__, cudaGetErrorString(_e)); \
      return HB_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

#define HB_TRY(...)             \
  do {                          \
    int _s = (__VA_ARGS__);     \
    if (_s != HB_OK) return _s; \
  } while (0)

int num_sms();
// Raises fn's dynamic shared-memory limit to the largest the device allows, once per
// (function, device).  The limit is one per-function setting shared by every thread of the
// process: plans of different shapes running at the same time must never lower it under
// each other's launches, so it is only ever set to this one value.
int allow_max_dyn_smem(const void* fn);

}  // namespace hb
