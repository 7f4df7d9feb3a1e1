// psg_ns2d.cu -- 2D vorticity RK4/CN step as one persistent CTA per instance
// (kernel body in psg_ns2d.cuh).  Any number of instances of any supported
// size run in one launch: blocks take instances from a work counter, largest
// first as ordered by the host.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "psg_ns2d.cuh"
#include "psgpu_internal.h"

namespace psg {

template <typename T>
struct Twiddles2D {
  const cpx<T>* t[5];  // n = 16, 32, 64, 128, 256
  int pk = 0;          // bit q: size class q runs the packed transforms (FP32)
};

template <typename T, int NN, bool HASPK>
__device__ __forceinline__ void rhs2d_run(const Inst2D<T>& I, const cpx<T>* tw, cpx<T>* smem,
                                          bool pk) {
  if constexpr (sizeof(T) == 4 && HASPK) {
    if (pk) {
      Rhs2D<T, NN, 1>::run(I, tw, smem);
      return;
    }
  }
  Rhs2D<T, NN>::run(I, tw, smem);
}

// block sizes of the persistent kernel the autotuner chooses from
constexpr int kBlock2D[3] = {128, 256, 512};

// HASPK: the packed transform schedules are compiled in (a schedule with no
// packed size class launches the build without them, whose registers are
// those of the scalar transforms alone)
template <typename T, int NT, bool HASPK = false>
__global__ void __launch_bounds__(NT)
ns2d_persistent(const Inst2D<T>* __restrict__ insts, int ninst, int* __restrict__ next,
                Twiddles2D<T> tws) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* smem = reinterpret_cast<cpx<T>*>(smem_raw);
  __shared__ int s_idx;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_idx = atomicAdd(next, 1);
    __syncthreads();
    const int i = s_idx;
    if (i >= ninst) break;
    const Inst2D<T> I = insts[i];
    switch (I.n) {
      case 16: rhs2d_run<T, 16, HASPK>(I, tws.t[0], smem, tws.pk & 1); break;
      case 32: rhs2d_run<T, 32, HASPK>(I, tws.t[1], smem, tws.pk & 2); break;
      case 64: rhs2d_run<T, 64, HASPK>(I, tws.t[2], smem, tws.pk & 4); break;
      case 128: rhs2d_run<T, 128, HASPK>(I, tws.t[3], smem, tws.pk & 8); break;
      default: rhs2d_run<T, 256, HASPK>(I, tws.t[4], smem, tws.pk & 16); break;
    }
  }
}

// FP64 reference boxes <-> state; `low` (FP32 engine) holds the part of each
// value below the state's precision
template <typename T>
__global__ void ref_to_dev2(const double2* __restrict__ src, cpx<T>* __restrict__ dst, long n,
                            cpx<T>* __restrict__ low) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const cpx<T> v = cpx<T>{(T)src[i].x, (T)src[i].y};
    dst[i] = v;
    if (low) low[i] = cpx<T>{(T)(src[i].x - (double)v.x), (T)(src[i].y - (double)v.y)};
  }
}
template <typename T>
__global__ void dev_to_ref2(const cpx<T>* __restrict__ src, double2* __restrict__ dst, long n,
                            const cpx<T>* __restrict__ low) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 v = make_double2((double)src[i].x, (double)src[i].y);
    if (low) { v.x += (double)low[i].x; v.y += (double)low[i].y; }
    dst[i] = v;
  }
}

// ---------------------------------------------------------------------------
// batched host engine
// ---------------------------------------------------------------------------
struct Batch2DBase {
  virtual ~Batch2DBase() {}
  virtual int upload(int i, const double* Z) = 0;
  virtual int download(int i, double* Z) = 0;
  virtual int run(const double* nu, const double* dt, const int* nsteps) = 0;
  virtual int set_params(const double* nu, const double* dt, const int* nsteps) = 0;
  virtual int launch() = 0;
  virtual int autotune(int* variant, float* ms) = 0;
  virtual int tuning(int* variant, float* ms) const = 0;
  virtual int schedule(int* pk, float* ms) const = 0;
  virtual int set_schedule(const int* pk) = 0;
  virtual int sync() = 0;
  virtual long launch_count() const = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  virtual int device_state(int i, void** Z) = 0;
};

template <typename T>
struct Batch2D final : Batch2DBase {
  int ninst = 0;
  std::vector<int> sizes;
  std::vector<long> offs;     // state offset of each instance (complex words)
  std::vector<long> woffs;    // work offset
  cpx<T>* pool = nullptr;
  cpx<T>* twp = nullptr;
  Inst2D<T>* d_insts = nullptr;
  int* d_next = nullptr;
  double2* staging = nullptr;
  long staging_len = 0;
  cudaStream_t stream = 0;
  long launches = 0;
  std::vector<int> order;     // instances sorted by cost, largest first
  size_t smem_v[3] = {0, 0, 0};  // dynamic shared memory per block-size variant
  int grid_v[3] = {0, 0, 0};     // resident blocks per variant (0: does not fit)
  int grid_pk[3] = {0, 0, 0};    // the same for the build with packed schedules
  int variant = 1;               // 256 threads unless the autotuner picks another
  float tune_ms[3] = {-1.f, -1.f, -1.f};
  // transform schedule per size class (n = 16 .. 256): bit q packed f32x2
  // transforms (FP32), chosen by the autotuner; sched_ms[q][0 / 1] the timing of
  // the batch with class q scalar / packed (-1: class absent or not timed)
  int pk_mask = 0;
  float sched_ms[5][2] = {{-1.f, -1.f}, {-1.f, -1.f}, {-1.f, -1.f}, {-1.f, -1.f}, {-1.f, -1.f}};
  int gexec_pk = -1;
  long state_words = 0;          // states (+ carried errors) of all instances
  bool params_set = false;
  // the persistent launch as a CUDA graph: reset the work counter, launch
  cudaGraphExec_t gexec = nullptr;
  int gexec_variant = -1;
  cudaStream_t cap = nullptr;

  ~Batch2D() override {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (cap) cudaStreamDestroy(cap);
    if (pool) cudaFree(pool);
    if (d_insts) cudaFree(d_insts);
    if (d_next) cudaFree(d_next);
    if (staging) cudaFree(staging);
  }

  int init(int n_, const int* sizes_) {
    ninst = n_;
    sizes.assign(sizes_, sizes_ + n_);
    long total = 0, work = 0, maxk = 0;
    for (int i = 0; i < ninst; ++i) {
      const int n = sizes[i];
      if (!(n == 16 || n == 32 || n == 64 || n == 128 || n == 256)) {
        psg_set_error("2D grid size %d unsupported (powers of two 16..256)", n);
        return PSG_ERR_UNSUPPORTED;
      }
      offs.push_back(total);
      total += (std::is_same<T, float>::value ? 6L : 5L) * nkt2(n);
      maxk = std::max<long>(maxk, nkt2(n));
    }
    state_words = total;
    for (int i = 0; i < ninst; ++i) {
      woffs.push_back(total + work);
      work += 3L * sizes[i] * (sizes[i] / 3 + 1);
    }
    const long twlen = 2 * (16 + 32 + 64 + 128 + 256);
    PSG_CUDA_TRY(cudaMalloc(&pool, sizeof(cpx<T>) * (total + work + twlen)));
    PSG_CUDA_TRY(cudaMemset(pool, 0, sizeof(cpx<T>) * (total + work + twlen)));
    twp = pool + total + work;
    std::vector<cpx<T>> h(twlen);
    tables2d(h.data());
    PSG_CUDA_TRY(cudaMemcpy(twp, h.data(), sizeof(cpx<T>) * twlen, cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMalloc(&d_insts, sizeof(Inst2D<T>) * ninst));
    PSG_CUDA_TRY(cudaMalloc(&d_next, sizeof(int)));
    staging_len = maxk;
    PSG_CUDA_TRY(cudaMalloc(&staging, sizeof(double2) * staging_len));
    order.resize(ninst);
    for (int i = 0; i < ninst; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sizes[a] > sizes[b]; });
    int maxn = 16;
    for (int n : sizes) maxn = std::max(maxn, n);
    int g = 4, sm = 0;
    switch (maxn) {
      case 16: g = LineFFT<16, 1, T>::G; sm = LineFFT<16, 1, T>::SMEM; break;
      case 32: g = LineFFT<32, 1, T>::G; sm = LineFFT<32, 1, T>::SMEM; break;
      case 64: g = LineFFT<64, 1, T>::G; sm = LineFFT<64, 1, T>::SMEM; break;
      case 128: g = LineFFT<128, 1, T>::G; sm = LineFFT<128, 1, T>::SMEM; break;
      default: g = LineFFT<256, 1, T>::G; sm = LineFFT<256, 1, T>::SMEM; break;
    }
    // exchange space for the densest packing of groups over all sizes present
    size_t worst = 0;
    for (int n : sizes) {
      int gg = 4, ss = 0;
      switch (n) {
        case 16: gg = LineFFT<16, 1, T>::G; ss = LineFFT<16, 1, T>::SMEM; break;
        case 32: gg = LineFFT<32, 1, T>::G; ss = LineFFT<32, 1, T>::SMEM; break;
        case 64: gg = LineFFT<64, 1, T>::G; ss = LineFFT<64, 1, T>::SMEM; break;
        case 128: gg = LineFFT<128, 1, T>::G; ss = LineFFT<128, 1, T>::SMEM; break;
        default: gg = LineFFT<256, 1, T>::G; ss = LineFFT<256, 1, T>::SMEM; break;
      }
      for (int v = 0; v < 3; ++v)
        smem_v[v] = std::max(smem_v[v], sizeof(cpx<T>) * (size_t)(2 * n + (kBlock2D[v] / gg) * ss));
    }
    (void)g; (void)sm;
    int dev = 0, nsm = 148, big = 0;
    PSG_CUDA_TRY(cudaGetDevice(&dev));
    PSG_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    PSG_CUDA_TRY(cudaDeviceGetAttribute(&big, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    for (int v = 0; v < 3; ++v) {
      const void* k = kernel(v);
      grid_v[v] = 0;
      if (smem_v[v] + 1024 > (size_t)big) continue;
      PSG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem_v[v]));
      int per_sm = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kBlock2D[v], smem_v[v]);
      grid_v[v] = std::max(0, std::min(ninst, nsm * per_sm));
      grid_pk[v] = 0;
      if constexpr (sizeof(T) == 4) {
        const void* kp = kernel_pk(v);
        PSG_CUDA_TRY(cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_v[v]));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, kBlock2D[v], smem_v[v]);
        grid_pk[v] = std::max(0, std::min(ninst, nsm * per_sm));
      }
    }
    if (!grid_v[variant]) {
      variant = -1;
      for (int v = 0; v < 3 && variant < 0; ++v)
        if (grid_v[v]) variant = v;
      if (variant < 0) {
        psg_set_error("2D batch: no block size fits this device");
        return PSG_ERR_UNSUPPORTED;
      }
    }
    PSG_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    return PSG_OK;
  }

  static const void* kernel(int v) {
    switch (v) {
      case 0: return (const void*)ns2d_persistent<T, 128>;
      case 1: return (const void*)ns2d_persistent<T, 256>;
      default: return (const void*)ns2d_persistent<T, 512>;
    }
  }
  static const void* kernel_pk(int v) {
    switch (v) {
      case 0: return (const void*)ns2d_persistent<T, 128, true>;
      case 1: return (const void*)ns2d_persistent<T, 256, true>;
      default: return (const void*)ns2d_persistent<T, 512, true>;
    }
  }

  Twiddles2D<T> twiddles() const {
    Twiddles2D<T> tws;
    long o = 0;
    for (int q = 0, n = 16; q < 5; ++q, n *= 2) { tws.t[q] = twp + o; o += 2 * n; }
    tws.pk = pk_mask;
    return tws;
  }

  void launch_kernel(int v, cudaStream_t st) {
    const Twiddles2D<T> tws = twiddles();
    if constexpr (sizeof(T) == 4) {
      if (tws.pk) {
      switch (v) {
        case 0: ns2d_persistent<T, 128, true><<<grid_pk[0], 128, smem_v[0], st>>>(d_insts, ninst, d_next, tws); break;
        case 1: ns2d_persistent<T, 256, true><<<grid_pk[1], 256, smem_v[1], st>>>(d_insts, ninst, d_next, tws); break;
        default: ns2d_persistent<T, 512, true><<<grid_pk[2], 512, smem_v[2], st>>>(d_insts, ninst, d_next, tws); break;
      }
      return;
      }
    }
    switch (v) {
      case 0: ns2d_persistent<T, 128><<<grid_v[0], 128, smem_v[0], st>>>(d_insts, ninst, d_next, tws); break;
      case 1: ns2d_persistent<T, 256><<<grid_v[1], 256, smem_v[1], st>>>(d_insts, ninst, d_next, tws); break;
      default: ns2d_persistent<T, 512><<<grid_v[2], 512, smem_v[2], st>>>(d_insts, ninst, d_next, tws); break;
    }
  }

  // (re)build the graph of one persistent launch for the current variant
  int build_graph() {
    if (gexec && gexec_variant == variant && gexec_pk == pk_mask) return PSG_OK;
    if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
    cudaGraph_t graph = nullptr;
    PSG_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(d_next, 0, sizeof(int), cap);
    launch_kernel(variant, cap);
    cudaError_t e = cudaStreamEndCapture(cap, &graph);
    if (e != cudaSuccess) { psg_set_error("graph capture: %s", cudaGetErrorString(e)); return PSG_ERR_CUDA; }
    e = cudaGraphInstantiate(&gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { psg_set_error("graph instantiate: %s", cudaGetErrorString(e)); return PSG_ERR_CUDA; }
    gexec_variant = variant;
    gexec_pk = pk_mask;
    return PSG_OK;
  }

  // carried rounding error of instance i's state (FP32 engine), or null
  cpx<T>* comp(int i) {
    if (!std::is_same<T, float>::value) return nullptr;
    return pool + offs[i] + 5L * nkt2(sizes[i]);
  }

  int upload(int i, const double* Z) override {
    if (i < 0 || i >= ninst) { psg_set_error("instance %d out of range", i); return PSG_ERR_ARG; }
    const long nk = nkt2(sizes[i]);
    PSG_CUDA_TRY(cudaMemcpyAsync(staging, Z, sizeof(double2) * nk, cudaMemcpyHostToDevice, stream));
    ref_to_dev2<T><<<148, 256, 0, stream>>>(staging, pool + offs[i], nk, comp(i));
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  int download(int i, double* Z) override {
    if (i < 0 || i >= ninst) { psg_set_error("instance %d out of range", i); return PSG_ERR_ARG; }
    const long nk = nkt2(sizes[i]);
    dev_to_ref2<T><<<148, 256, 0, stream>>>(pool + offs[i], staging, nk, comp(i));
    ++launches;
    PSG_CUDA_TRY(cudaMemcpyAsync(Z, staging, sizeof(double2) * nk, cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }

  int run(const double* nu, const double* dt, const int* nsteps) override {
    int rc = set_params(nu, dt, nsteps);
    return rc ? rc : launch();
  }

  int launch() override {
    if (!params_set) { psg_set_error("2D batch: parameters not set"); return PSG_ERR_STATE; }
    if (int rc = build_graph()) return rc;
    PSG_CUDA_TRY(cudaGraphLaunch(gexec, stream));
    ++launches;
    return PSG_OK;
  }

  // time every block size on the current parameters (3 timed launches of a
  // 2-step copy of the run after one warm-up), restoring the states after
  // each, and keep the fastest; then, at that block size and in FP32, the
  // transform schedule of each size class present (scalar or packed f32x2
  // transforms), one class at a time, keeping the faster
  int autotune(int* v_out, float* ms) override {
    if (!params_set) { psg_set_error("2D batch: parameters not set"); return PSG_ERR_STATE; }
    std::vector<Inst2D<T>> h(hparams), shortp(hparams);
    for (auto& I : shortp) I.nsteps = std::min(I.nsteps, 2);
    cpx<T>* save = nullptr;
    PSG_CUDA_TRY(cudaMalloc(&save, sizeof(cpx<T>) * state_words));
    PSG_CUDA_TRY(cudaMemcpyAsync(save, pool, sizeof(cpx<T>) * state_words, cudaMemcpyDeviceToDevice, stream));
    PSG_CUDA_TRY(cudaMemcpyAsync(d_insts, shortp.data(), sizeof(Inst2D<T>) * ninst,
                                 cudaMemcpyHostToDevice, stream));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    // ms per launch of the short run with block-size variant v and the current schedule
    auto time_v = [&](int v, float* out) -> int {
      cudaMemsetAsync(d_next, 0, sizeof(int), stream);
      launch_kernel(v, stream);
      cudaEventRecord(a, stream);
      for (int r = 0; r < 3; ++r) {
        cudaMemsetAsync(d_next, 0, sizeof(int), stream);
        launch_kernel(v, stream);
      }
      cudaEventRecord(b, stream);
      launches += 4;
      cudaError_t e = cudaEventSynchronize(b);
      if (e != cudaSuccess) { psg_set_error("autotune: %s", cudaGetErrorString(e)); return PSG_ERR_CUDA; }
      float t = 0.f;
      cudaEventElapsedTime(&t, a, b);
      *out = t / 3.f;
      return PSG_OK;
    };
    int rc = PSG_OK;
    float best = 1e30f;
    int pick = variant;
    for (int v = 0; v < 3 && !rc; ++v) {
      tune_ms[v] = -1.f;
      if (!grid_v[v]) continue;
      rc = time_v(v, &tune_ms[v]);
      if (!rc && tune_ms[v] < best) { best = tune_ms[v]; pick = v; }
    }
    for (int q = 0; q < 5; ++q) sched_ms[q][0] = sched_ms[q][1] = -1.f;
    if (sizeof(T) == 4) {
      int present = 0;
      for (int n : sizes)
        for (int q = 0; q < 5; ++q)
          if (n == (16 << q)) present |= 1 << q;
      for (int q = 0; q < 5 && !rc && grid_pk[pick] > 0; ++q) {
        if (!(present & (1 << q))) continue;
        for (int p = 0; p < 2 && !rc; ++p) {
          pk_mask = p ? (pk_mask | (1 << q)) : (pk_mask & ~(1 << q));
          rc = time_v(pick, &sched_ms[q][p]);
        }
        if (!rc && sched_ms[q][1] >= 0.f && sched_ms[q][1] < sched_ms[q][0]) pk_mask |= 1 << q;
        else pk_mask &= ~(1 << q);
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) { cudaFree(save); return rc; }
    PSG_CUDA_TRY(cudaMemcpyAsync(pool, save, sizeof(cpx<T>) * state_words, cudaMemcpyDeviceToDevice, stream));
    PSG_CUDA_TRY(cudaMemcpyAsync(d_insts, h.data(), sizeof(Inst2D<T>) * ninst,
                                 cudaMemcpyHostToDevice, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    cudaFree(save);
    variant = pick;
    if (v_out) *v_out = variant;
    if (ms) for (int v = 0; v < 3; ++v) ms[v] = tune_ms[v];
    return PSG_OK;
  }

  int set_schedule(const int* pk) override {
    int m = 0;
    for (int q = 0; q < 5; ++q)
      if (pk[q]) m |= 1 << q;
    if (m && (sizeof(T) != 4 || !grid_pk[variant])) {
      psg_set_error("packed transforms need an FP32 batch whose packed build fits");
      return PSG_ERR_UNSUPPORTED;
    }
    pk_mask = m;
    return PSG_OK;
  }

  int schedule(int* pk, float* ms) const override {
    for (int q = 0; q < 5; ++q) {
      if (pk) pk[q] = (pk_mask >> q) & 1;
      if (ms) { ms[2 * q] = sched_ms[q][0]; ms[2 * q + 1] = sched_ms[q][1]; }
    }
    return PSG_OK;
  }

  std::vector<Inst2D<T>> hparams;

  int set_params(const double* nu, const double* dt, const int* nsteps) override {
    std::vector<Inst2D<T>> h(ninst);
    for (int j = 0; j < ninst; ++j) {
      const int i = order[j];
      const long nk = nkt2(sizes[i]);
      Inst2D<T>& I = h[j];
      I.n = sizes[i]; I.nsteps = nsteps[i]; I.nu = (T)nu[i]; I.dt = (T)dt[i];
      cpx<T>* b = pool + offs[i];
      I.Z = b; I.Z0 = b + nk; I.Z1 = b + 2 * nk; I.Z2 = b + 3 * nk; I.Z3 = b + 4 * nk;
      I.work = pool + woffs[i];
      I.ZC = comp(i);
    }
    PSG_CUDA_TRY(cudaMemcpyAsync(d_insts, h.data(), sizeof(Inst2D<T>) * ninst,
                                 cudaMemcpyHostToDevice, stream));
    // the copy reads pageable host memory: finish it before h goes away
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    hparams = h;
    params_set = true;
    return PSG_OK;
  }

  int tuning(int* v_out, float* ms) const override {
    if (v_out) *v_out = variant;
    if (ms) for (int v = 0; v < 3; ++v) ms[v] = tune_ms[v];
    return PSG_OK;
  }

  int sync() override {
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }
  long launch_count() const override { return launches; }
  void set_stream(cudaStream_t s) override { stream = s; }
  int device_state(int i, void** Z) override {
    if (i < 0 || i >= ninst) { psg_set_error("instance %d out of range", i); return PSG_ERR_ARG; }
    *Z = (void*)(pool + offs[i]);
    return PSG_OK;
  }
};

}  // namespace psg

using namespace psg;

struct psg_batch2d {
  Batch2DBase* b = nullptr;
  int ninst = 0;
};

extern "C" int psg_batch2d_create(psg_batch2d** out, int ninst, const int* sizes, int precision) {
  if (!out || ninst <= 0 || !sizes) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  *out = nullptr;
  if (precision != 32 && precision != 64) { psg_set_error("precision must be 32 or 64"); return PSG_ERR_ARG; }
  psg_batch2d* h = new psg_batch2d();
  int rc;
  if (precision == 64) { auto* b = new Batch2D<double>(); h->b = b; rc = b->init(ninst, sizes); }
  else { auto* b = new Batch2D<float>(); h->b = b; rc = b->init(ninst, sizes); }
  if (rc) { delete h->b; delete h; return rc; }
  h->ninst = ninst;
  *out = h;
  return PSG_OK;
}

extern "C" void psg_batch2d_destroy(psg_batch2d* h) {
  if (!h) return;
  delete h->b;
  delete h;
}

#define PSG_B2(h)                                                   \
  do {                                                              \
    if (!(h) || !(h)->b) { psg_set_error("null batch handle"); return PSG_ERR_ARG; } \
  } while (0)

extern "C" int psg_batch2d_upload(psg_batch2d* h, int i, const double* Z) {
  PSG_B2(h);
  return h->b->upload(i, Z);
}
extern "C" int psg_batch2d_download(psg_batch2d* h, int i, double* Z) {
  PSG_B2(h);
  return h->b->download(i, Z);
}
extern "C" int psg_batch2d_run(psg_batch2d* h, const double* nu, const double* dt, const int* nsteps) {
  PSG_B2(h);
  if (!nu || !dt || !nsteps) { psg_set_error("null parameter arrays"); return PSG_ERR_ARG; }
  return h->b->run(nu, dt, nsteps);
}
extern "C" int psg_batch2d_set_params(psg_batch2d* h, const double* nu, const double* dt,
                                      const int* nsteps) {
  PSG_B2(h);
  if (!nu || !dt || !nsteps) { psg_set_error("null parameter arrays"); return PSG_ERR_ARG; }
  return h->b->set_params(nu, dt, nsteps);
}
extern "C" int psg_batch2d_launch(psg_batch2d* h) {
  PSG_B2(h);
  return h->b->launch();
}
extern "C" int psg_batch2d_autotune(psg_batch2d* h, int* variant, float* ms) {
  PSG_B2(h);
  return h->b->autotune(variant, ms);
}
extern "C" int psg_batch2d_tuning(psg_batch2d* h, int* variant, float* ms) {
  PSG_B2(h);
  return h->b->tuning(variant, ms);
}

// the transform schedule the autotuner chose per size class
extern "C" int psg_batch2d_schedule(psg_batch2d* h, int* packed, float* ms) {
  PSG_B2(h);
  return h->b->schedule(packed, ms);
}

// pin the transform schedule per grid size (packed[5], as psg_batch2d_schedule)
extern "C" int psg_batch2d_set_schedule(psg_batch2d* h, const int* packed) {
  PSG_B2(h);
  if (!packed) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  return h->b->set_schedule(packed);
}

extern "C" int psg_batch2d_sync(psg_batch2d* h) {
  PSG_B2(h);
  return h->b->sync();
}
extern "C" int psg_batch2d_set_stream(psg_batch2d* h, void* s) {
  PSG_B2(h);
  h->b->set_stream((cudaStream_t)s);
  return PSG_OK;
}
extern "C" long psg_batch2d_launches(psg_batch2d* h) { return (h && h->b) ? h->b->launch_count() : -1; }
extern "C" int psg_batch2d_device_state(psg_batch2d* h, int i, void** Z) {
  PSG_B2(h);
  if (!Z) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->b->device_state(i, Z);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the 2D step.
//
// Some hosts cannot call cudaMalloc from the code that drives the step: a
// plugin running inside another runtime that owns all device memory, a
// callback invoked while a CUDA graph is being captured, or an embedded
// driver whose memory budget is fixed at start-up.  psg_ns2d_step_noalloc
// serves them: it runs the same per-instance kernel body as the batched engine
// (Rhs2D::run), but its stage registers, row scratch and twiddle tables live
// in the file-scope array below instead of buffers allocated at run time.  The
// caller passes only the state, in device memory it already owns.
//
// Size limit: grids up to 128 x 128 (FP32 or FP64).  The array is part of the
// library image, so every GPU that loads the library holds these 512 KiB until
// the process exits.  The FP32 step also keeps, in the array, the rounding
// error its state updates carry (as psg_batch2d_run's FP32 engine does),
// cleared at the start of every call, so a call's state is its FP32 input.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr int kNoallocMaxN = 128;
constexpr size_t kNoallocBytes = 512 * 1024;
constexpr size_t kTw64Off = 0;          // 480 complex doubles (n = 16..128, two plans each)
constexpr size_t kTw32Off = 8192;       // 480 complex floats
constexpr size_t kWorkOff = 12288;      // Z0..Z3, the carried error (FP32) and row scratch

constexpr long nkt2c(int n) { return (long)(n / 3 + 1) * (2 * (n / 3) + 1); }
// bytes of the work area at the largest grid: FP64 (4 stage registers + 3 scratch
// rows) and FP32 (the same plus the carried rounding error)
constexpr size_t kWork64 = 16 * (4 * nkt2c(kNoallocMaxN) + 3L * kNoallocMaxN * (kNoallocMaxN / 3 + 1));
constexpr size_t kWork32 = 8 * (5 * nkt2c(kNoallocMaxN) + 3L * kNoallocMaxN * (kNoallocMaxN / 3 + 1));
static_assert(kWorkOff + kWork64 <= kNoallocBytes && kWorkOff + kWork32 <= kNoallocBytes,
              "static scratch too small for the largest grid");
static_assert(kTw64Off + 480 * 16 <= kTw32Off && kTw32Off + 480 * 8 <= kWorkOff, "twiddle tables");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// device address of g_noalloc_scratch, looked up once per device
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[kMaxDevices] = {nullptr};

template <typename T>
__global__ void __launch_bounds__(256) ns2d_single(Inst2D<T> I, const cpx<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* smem = reinterpret_cast<cpx<T>*>(smem_raw);
  switch (I.n) {
    case 16: Rhs2D<T, 16>::run(I, tw, smem); break;
    case 32: Rhs2D<T, 32>::run(I, tw, smem); break;
    case 64: Rhs2D<T, 64>::run(I, tw, smem); break;
    default: Rhs2D<T, 128>::run(I, tw, smem); break;
  }
}

template <typename T>
size_t noalloc_smem() {
  // the densest exchange layout among the supported sizes
  size_t worst = 0;
  worst = std::max(worst, (size_t)(32 + (256 / LineFFT<16, 1, T>::G) * LineFFT<16, 1, T>::SMEM));
  worst = std::max(worst, (size_t)(64 + (256 / LineFFT<32, 1, T>::G) * LineFFT<32, 1, T>::SMEM));
  worst = std::max(worst, (size_t)(128 + (256 / LineFFT<64, 1, T>::G) * LineFFT<64, 1, T>::SMEM));
  worst = std::max(worst, (size_t)(256 + (256 / LineFFT<128, 1, T>::G) * LineFFT<128, 1, T>::SMEM));
  return worst * sizeof(cpx<T>);
}

// One-time set-up on the current device: find the array's device address,
// write the twiddle tables into it, raise the kernels' shared-memory limit.
// Nothing here allocates device memory.  The table copies are synchronous, so
// a first call made while `stream` is being captured is refused (the capture
// would be invalidated) with a message asking for a warm-up call.
int noalloc_setup(unsigned char** out, cudaStream_t stream) {
  int dev = 0;
  PSG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    psg_set_error("device ordinal %d beyond %d", dev, kMaxDevices);
    return PSG_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_addr[dev]) { *out = g_noalloc_addr[dev]; return PSG_OK; }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PSG_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    psg_set_error("psg_ns2d_step_noalloc: the first call on device %d sets up the static scratch "
                  "with synchronous copies and cannot run during stream capture; make one call "
                  "before capturing", dev);
    return PSG_ERR_UNSUPPORTED;
  }
  void* addr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
  if (e != cudaSuccess) {
    psg_set_error("cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
    return PSG_ERR_CUDA;
  }
  cpx<double> t64[480];
  cpx<float> t32[480];
  tables2d<double>(t64, kNoallocMaxN);
  tables2d<float>(t32, kNoallocMaxN);
  PSG_CUDA_TRY(cudaMemcpy((unsigned char*)addr + kTw64Off, t64, sizeof t64, cudaMemcpyHostToDevice));
  PSG_CUDA_TRY(cudaMemcpy((unsigned char*)addr + kTw32Off, t32, sizeof t32, cudaMemcpyHostToDevice));
  PSG_CUDA_TRY(cudaFuncSetAttribute(ns2d_single<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)noalloc_smem<double>()));
  PSG_CUDA_TRY(cudaFuncSetAttribute(ns2d_single<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)noalloc_smem<float>()));
  g_noalloc_addr[dev] = (unsigned char*)addr;
  *out = (unsigned char*)addr;
  return PSG_OK;
}

template <typename T>
int noalloc_run(unsigned char* base, int n, double nu, double dt, int nsteps, const void* z_in,
                void* z_out, cudaStream_t stream) {
  const long nk = nkt2(n);
  if (z_in != z_out)
    PSG_CUDA_TRY(cudaMemcpyAsync(z_out, z_in, sizeof(cpx<T>) * nk, cudaMemcpyDeviceToDevice, stream));
  cpx<T>* work = reinterpret_cast<cpx<T>*>(base + kWorkOff);
  Inst2D<T> I;
  I.n = n; I.nsteps = nsteps; I.nu = (T)nu; I.dt = (T)dt;
  I.Z = reinterpret_cast<cpx<T>*>(z_out);
  I.Z0 = work; I.Z1 = work + nk; I.Z2 = work + 2 * nk; I.Z3 = work + 3 * nk;
  if (sizeof(T) == 4) {
    // the carried rounding error starts at zero: the state is the caller's FP32 value
    I.ZC = work + 4 * nk;
    PSG_CUDA_TRY(cudaMemsetAsync(I.ZC, 0, sizeof(cpx<T>) * nk, stream));
    I.work = work + 5 * nk;
  } else {
    I.ZC = nullptr;
    I.work = work + 4 * nk;
  }
  const cpx<T>* tw = reinterpret_cast<const cpx<T>*>(base + (sizeof(T) == 8 ? kTw64Off : kTw32Off));
  int off = 0;
  for (int m = 16; m < n; m *= 2) off += 2 * m;
  ns2d_single<T><<<1, 256, noalloc_smem<T>(), stream>>>(I, tw + off);
  PSG_CUDA_TRY(cudaGetLastError());
  return PSG_OK;
}

}  // namespace

// No counterpart in the reference: see include/psgpu.h.
extern "C" int psg_ns2d_step_noalloc(int n, int precision, double nu, double dt, int nsteps,
                                     const void* z_in, void* z_out, void* stream) {
  if (!(n == 16 || n == 32 || n == 64 || n == 128)) {
    psg_set_error("psg_ns2d_step_noalloc: grid %d unsupported; the static scratch holds grids "
                  "of 16, 32, 64 or 128 points per direction at most", n);
    return PSG_ERR_UNSUPPORTED;
  }
  if (precision != 32 && precision != 64) {
    psg_set_error("psg_ns2d_step_noalloc: precision must be 32 or 64");
    return PSG_ERR_ARG;
  }
  if (nsteps < 0 || !z_in || !z_out) {
    psg_set_error("psg_ns2d_step_noalloc: bad arguments");
    return PSG_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* base = nullptr;
  int rc = noalloc_setup(&base, s);
  if (rc) return rc;
  return precision == 64 ? noalloc_run<double>(base, n, nu, dt, nsteps, z_in, z_out, s)
                         : noalloc_run<float>(base, n, nu, dt, nsteps, z_in, z_out, s);
}
