// psg_common.cuh -- shared types and helpers of the psgpu_b200 CUDA layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace psg {

template <typename T>
struct __align__(2 * sizeof(T)) cpx {
  T x, y;
};

template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
  return cpx<T>{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cpx<T> cadd(cpx<T> a, cpx<T> b) { return cpx<T>{a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> csub(cpx<T> a, cpx<T> b) { return cpx<T>{a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> cscale(cpx<T> a, T s) { return cpx<T>{a.x * s, a.y * s}; }
template <typename T>
__device__ __forceinline__ cpx<T> cconj(cpx<T> a) { return cpx<T>{a.x, -a.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> czero() { return cpx<T>{(T)0, (T)0}; }

// block-wide and warp-wide barriers as callables for LineFFT::run
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
// barrier of `count` threads (whole warps) on hardware barrier `id` (1..15;
// 0 is the one __syncthreads uses)
struct NamedSync {
  int id, count;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
  }
};

}  // namespace psg

// status codes shared with include/psgpu.h
#define PSG_OK 0
#define PSG_ERR_ARG 1
#define PSG_ERR_CUDA 2
#define PSG_ERR_UNSUPPORTED 3
#define PSG_ERR_STATE 4

#define PSG_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      psg_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
      return PSG_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

extern "C" void psg_set_error(const char* fmt, ...);
