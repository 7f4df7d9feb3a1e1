// psg_tan2d_run.cuh -- launch side of the 2D base + tangent integrator
// (psg_tan2d.cuh) for the batched UPO search: the persistent and cluster
// kernels in FP64 and FP32, their launch helpers and the per-precision
// integration resources.  The kernels are instantiated in psg_tan2d_f64.cu
// and psg_tan2d_f32.cu (one translation unit per precision, compiled in
// parallel); other files see only the explicit-instantiation declarations
// below.
#pragma once
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "psg_tan2d.cuh"
#include "psgpu_internal.h"

namespace psg {

// the integrations with CS blocks per instance (a cluster of CS), for
// batches too small to fill the device one block per instance; cluster c
// takes instances c, c + C, ... (all blocks run the same instance sequence).
// FP32 instances (the exact-tangent Krylov products in FP32) ask for two
// blocks per SM.
template <typename T, int N, int CS>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(256, (sizeof(T) == 4 ? 2 : 1))
    tan2d_cluster(const InstTan2D<T>* __restrict__ insts, int ninst,
                  const cpx<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* smem = reinterpret_cast<cpx<T>*>(smem_raw);
  unsigned rank;
  asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
  const Team t{(int)rank, CS};
  const int ncl = gridDim.x / CS;
  for (int i = blockIdx.x / CS; i < ninst; i += ncl) Tan2D<T, N>::run(insts[i], tw, smem, t);
}

template <typename T, int N>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 2 : 1))
    tan2d_persistent(const InstTan2D<T>* __restrict__ insts, int ninst, int* __restrict__ next,
                     const cpx<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* smem = reinterpret_cast<cpx<T>*>(smem_raw);
  __shared__ int s_idx;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_idx = atomicAdd(next, 1);
    __syncthreads();
    const int i = s_idx;
    if (i >= ninst) break;
    Tan2D<T, N>::run(insts[i], tw, smem);
  }
}

// precision conversion of whole state vectors (one job per blockIdx.y)
struct CvtJob {
  const void* src;
  void* dst;
};
template <typename S, typename D>
__global__ void cvt_vec(const CvtJob* __restrict__ jobs, int nkt) {
  const CvtJob J = jobs[blockIdx.y];
  const cpx<S>* a = reinterpret_cast<const cpx<S>*>(J.src);
  cpx<D>* b = reinterpret_cast<cpx<D>*>(J.dst);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nkt; i += gridDim.x * blockDim.x)
    b[i] = cpx<D>{(D)a[i].x, (D)a[i].y};
}

// njobs conversions into precision T from the other one
template <typename T>
void cvt_launch(const CvtJob* d_jobs, int njobs, int nkt, cudaStream_t st) {
  const dim3 grid((nkt + 255) / 256, (unsigned)njobs);
  if (sizeof(T) == 4) cvt_vec<double, float><<<grid, 256, 0, st>>>(d_jobs, nkt);
  else cvt_vec<float, double><<<grid, 256, 0, st>>>(d_jobs, nkt);
}

// kernel of one precision, grid size and cluster size (1: the persistent form)
template <typename T, int CS>
const void* tan2d_fn(int n) {
  if (CS == 1) {
    switch (n) {
      case 16: return (const void*)tan2d_persistent<T, 16>;
      case 32: return (const void*)tan2d_persistent<T, 32>;
      case 64: return (const void*)tan2d_persistent<T, 64>;
      case 128: return (const void*)tan2d_persistent<T, 128>;
      default: return (const void*)tan2d_persistent<T, 256>;
    }
  }
  switch (n) {
    case 16: return (const void*)tan2d_cluster<T, 16, (CS == 1 ? 2 : CS)>;
    case 32: return (const void*)tan2d_cluster<T, 32, (CS == 1 ? 2 : CS)>;
    case 64: return (const void*)tan2d_cluster<T, 64, (CS == 1 ? 2 : CS)>;
    case 128: return (const void*)tan2d_cluster<T, 128, (CS == 1 ? 2 : CS)>;
    default: return (const void*)tan2d_cluster<T, 256, (CS == 1 ? 2 : CS)>;
  }
}

template <typename T, int N>
void tan2d_launch_n(int cs, int m, int grid, size_t smem, cudaStream_t st,
                    const InstTan2D<T>* d, int* next, const cpx<T>* tw) {
  if (cs == 4) tan2d_cluster<T, N, 4><<<4 * m, 256, smem, st>>>(d, m, tw);
  else if (cs == 2) tan2d_cluster<T, N, 2><<<2 * m, 256, smem, st>>>(d, m, tw);
  else tan2d_persistent<T, N><<<grid, 256, smem, st>>>(d, m, next, tw);
}

template <typename T>
void tan2d_launch(int n, int cs, int m, int grid, size_t smem, cudaStream_t st,
                  const InstTan2D<T>* d, int* next, const cpx<T>* tw) {
  switch (n) {
    case 16: tan2d_launch_n<T, 16>(cs, m, grid, smem, st, d, next, tw); break;
    case 32: tan2d_launch_n<T, 32>(cs, m, grid, smem, st, d, next, tw); break;
    case 64: tan2d_launch_n<T, 64>(cs, m, grid, smem, st, d, next, tw); break;
    case 128: tan2d_launch_n<T, 128>(cs, m, grid, smem, st, d, next, tw); break;
    default: tan2d_launch_n<T, 256>(cs, m, grid, smem, st, d, next, tw); break;
  }
}

template <typename T>
inline size_t tan2d_smem(int n) {
  int gg = 0, sm = 0;
  switch (n) {
    case 16: gg = LineFFT<16, 1, T>::G; sm = LineFFT<16, 1, T>::SMEM; break;
    case 32: gg = LineFFT<32, 1, T>::G; sm = LineFFT<32, 1, T>::SMEM; break;
    case 64: gg = LineFFT<64, 1, T>::G; sm = LineFFT<64, 1, T>::SMEM; break;
    case 128: gg = LineFFT<128, 1, T>::G; sm = LineFFT<128, 1, T>::SMEM; break;
    default: gg = LineFFT<256, 1, T>::G; sm = LineFFT<256, 1, T>::SMEM; break;
  }
  return sizeof(cpx<T>) * (2 * n + (256 / gg) * sm);
}

template <typename T>
inline void tan2d_tables(int n, cpx<T>* h) {
  switch (n) {
    case 16: LineFFT<16, 1, T>::host_table(h); LineFFT<16, 1, T, true>::host_table(h + n); break;
    case 32: LineFFT<32, 1, T>::host_table(h); LineFFT<32, 1, T, true>::host_table(h + n); break;
    case 64: LineFFT<64, 1, T>::host_table(h); LineFFT<64, 1, T, true>::host_table(h + n); break;
    case 128: LineFFT<128, 1, T>::host_table(h); LineFFT<128, 1, T, true>::host_table(h + n); break;
    default: LineFFT<256, 1, T>::host_table(h); LineFFT<256, 1, T, true>::host_table(h + n); break;
  }
}

// the integration resources of one precision: twiddles, launch descriptors,
// dynamic shared memory and the resident-block capacity of the device
template <typename T>
struct IntPlan {
  cpx<T>* tw = nullptr;
  InstTan2D<T>* d_inst = nullptr;
  size_t smem = 0;
  int grid_cap = 148;

  int init(int n, int ng, cpx<T>* tw_dev) {
    tw = tw_dev;
    std::vector<cpx<T>> h(2 * n);
    tan2d_tables<T>(n, h.data());
    PSG_CUDA_TRY(cudaMemcpy(tw, h.data(), sizeof(cpx<T>) * 2 * n, cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMalloc(&d_inst, sizeof(InstTan2D<T>) * ng));
    smem = tan2d_smem<T>(n);
    const void* fns[3] = {tan2d_fn<T, 1>(n), tan2d_fn<T, 2>(n), tan2d_fn<T, 4>(n)};
    for (const void* f : fns)
      PSG_CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fns[0], 256, smem);
    // PSG_UPO_BLOCKS_PER_SM caps the blocks the dealing counts on per SM (the
    // FP32 integrator fits two)
    if (const char* e = getenv("PSG_UPO_BLOCKS_PER_SM")) occ = std::min(occ, std::max(1, atoi(e)));
    grid_cap = nsm * std::max(occ, 1);
    return PSG_OK;
  }
  void release() {
    if (d_inst) cudaFree(d_inst);
    d_inst = nullptr;
  }
};


// instantiated in psg_tan2d_f64.cu / psg_tan2d_f32.cu
#define PSG_TAN2D_EXTERN(T)                                                                   \
  extern template const void* tan2d_fn<T, 1>(int);                                           \
  extern template const void* tan2d_fn<T, 2>(int);                                           \
  extern template const void* tan2d_fn<T, 4>(int);                                           \
  extern template void tan2d_launch<T>(int, int, int, int, size_t, cudaStream_t,             \
                                       const InstTan2D<T>*, int*, const cpx<T>*);            \
  extern template void cvt_launch<T>(const CvtJob*, int, int, cudaStream_t);
#define PSG_TAN2D_INSTANTIATE(T)                                                              \
  template const void* tan2d_fn<T, 1>(int);                                                  \
  template const void* tan2d_fn<T, 2>(int);                                                  \
  template const void* tan2d_fn<T, 4>(int);                                                  \
  template void tan2d_launch<T>(int, int, int, int, size_t, cudaStream_t,                    \
                                const InstTan2D<T>*, int*, const cpx<T>*);                   \
  template void cvt_launch<T>(const CvtJob*, int, int, cudaStream_t);

}  // namespace psg
