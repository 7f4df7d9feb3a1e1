// psg_ns2d.cu -- 2D vorticity RK4/CN step as one persistent CTA per instance.
//
// A 2D instance (N <= 256) is small enough that one thread block integrates it
// for all of its steps without leaving the kernel: every right-hand side is
// three phases separated by block barriers,
//   1. y-inverse of w, u = i ky w / k^2, v = -i kx w / k^2  (X columns each)
//   2. x rows: C2R of (w,u) and (v), products v w and u w scaled by 1/N^2,
//      R2C of the packed pair, kx <= K kept (in place in the row scratch)
//   3. y-forward of both products per column, kept ky rows, then
//      N = -i (kx F(u w) + ky F(v w)), the Kolmogorov forcing and the RK4 stage
// and the intermediate rows live in a per-instance scratch that stays in L2.
// Any number of instances of any supported size run in one launch: blocks
// take instances from a work counter (largest first, ordered by the host).
//
// The scheme restates 2D_NavierStokes/src_RK4/kernels.h:112-435 (setVelocity,
// Step1, Step2, Step) and the transforms replace conj -> setFFN -> Z2D,
// multReal, batched D2Z -> normFF1 (2D_NavierStokes/src_RK4/functions.h:33-149).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "psg_common.cuh"
#include "psg_fft.cuh"
#include "psgpu_internal.h"

namespace psg {

template <typename T>
struct Inst2D {
  int n;        // grid points per direction
  int nsteps;   // RK4 steps to take
  T nu, dt;     // viscosity, time step
  cpx<T>* Z;    // state [2K+1][K+1]
  cpx<T>* Z0;   // stage state
  cpx<T>* Z1;
  cpx<T>* Z2;
  cpx<T>* Z3;
  cpx<T>* work;  // [3][n][K+1] row scratch
};

__device__ __forceinline__ int row_to_box2(int r, int K, int n) {
  if (r <= K) return r + K;
  if (r >= n - K) return r - n + K;
  return -1;
}

// mask of 2D_NavierStokes/src_RK4/src_gmres/init.F90:30-36 (alpha = 1)
__device__ __forceinline__ bool keep2(int ikx, int ky, int K) {
  if (ikx == 0 && ky <= 0) return false;
  const int wk = ikx * ikx + ky * ky;
  return 4 * wk <= (2 * K - 1) * (2 * K - 1);   // |k| <= K - 1/2
}

template <typename T>
__device__ __forceinline__ T wkinv2(T wk) {
  return (T)1 / (wk > (T)0.001 ? wk : (T)0.001);
}

// field f (0: w, 1: u, 2: v) at box mode (ikx, iky) of the stage state, with
// the kx = 0 lower half filled by conjugates (2D_NavierStokes/src_RK4/kernels.h:82-96)
template <typename T>
__device__ __forceinline__ cpx<T> field2(const cpx<T>* __restrict__ Z0, int f, int ikx, int iky,
                                          int K, int X) {
  bool cj = false;
  if (ikx == 0 && iky < K) { iky = 2 * K - iky; cj = true; }
  const int ky = iky - K;
  if (!keep2(ikx, ky, K)) return czero<T>();
  const cpx<T> z = Z0[iky * X + ikx];
  cpx<T> r;
  if (f == 0) {
    r = z;
  } else {
    const T kx = (T)ikx, kyT = (T)ky;
    const T wki = wkinv2(kx * kx + kyT * kyT);
    // UK = i ky Z / k^2, VK = -i kx Z / k^2 (2D_NavierStokes/src_RK4/kernels.h:126-130)
    if (f == 1) r = cpx<T>{-kyT * z.y * wki, kyT * z.x * wki};
    else r = cpx<T>{kx * z.y * wki, -kx * z.x * wki};
  }
  if (cj) r.y = -r.y;
  return r;
}

template <typename T, int N>
struct Rhs2D {
  using FI = LineFFT<N, +1, T>;
  using FO = LineFFT<N, -1, T>;
  using FX = LineFFT<N, -1, T, true>;  // forward transform of phase 2: consumes FI's output
  static constexpr int G = FI::G, E = FI::E;
  static constexpr int K = N / 3, X = K + 1, Y = 2 * K + 1;

  // phase 1: y-inverse of the three fields, written to work[f][y][kx]
  static __device__ void phase1(const Inst2D<T>& I, const cpx<T>* tw, cpx<T>* ex) {
    const int gid = threadIdx.x / G, gi = threadIdx.x % G, ng = blockDim.x / G;
    for (int base = 0; base < 3 * X; base += ng) {
      const int col = base + gid;
      const bool live = col < 3 * X;
      const int f = live ? col / X : 0, ikx = live ? col % X : 0;
      cpx<T> v[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int iky = row_to_box2(FI::in_index(gi, e), K, N);
        v[e] = (live && iky >= 0) ? field2(I.Z0, f, ikx, iky, K, X) : czero<T>();
      }
      FI::run(v, gi, tw, ex, WarpSync());
      if (live) {
        cpx<T>* dst = I.work + (long)f * N * X + ikx;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[FI::out_index(gi, e) * X] = v[e];
      }
    }
  }

  // phase 2: x rows, products, back to spectral rows (fields 0: F(v w), 1: F(u w))
  static __device__ void phase2(const Inst2D<T>& I, const cpx<T>* tw, cpx<T>* ex) {
    const int gid = threadIdx.x / G, gi = threadIdx.x % G, ng = blockDim.x / G;
    const T scale = (T)1 / ((T)N * (T)N);
    for (int base = 0; base < N; base += ng) {
      const int y = base + gid;
      const bool live = y < N;
      const cpx<T>* rw = I.work + (long)(live ? y : 0) * X;
      const cpx<T>* ru = rw + (long)N * X;
      const cpx<T>* rv = rw + 2L * N * X;
      cpx<T> v[E];
      // (w, u) packed: w + i u
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int r = FI::in_index(gi, e);
        cpx<T> z = czero<T>();
        if (live) {
          if (r == 0) z = cpx<T>{rw[0].x, ru[0].x};
          else if (r <= K) { const cpx<T> a = rw[r], b = ru[r]; z = cpx<T>{a.x - b.y, a.y + b.x}; }
          else if (r >= N - K) { const cpx<T> a = rw[N - r], b = ru[N - r]; z = cpx<T>{a.x + b.y, -a.y + b.x}; }
        }
        v[e] = z;
      }
      FI::run(v, gi, tw, ex, WarpSync());
      T w[E], u[E];
#pragma unroll
      for (int e = 0; e < E; ++e) { w[e] = v[e].x; u[e] = v[e].y; }
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int r = FI::in_index(gi, e);
        cpx<T> z = czero<T>();
        if (live) {
          if (r == 0) z = cpx<T>{rv[0].x, (T)0};
          else if (r <= K) z = rv[r];
          else if (r >= N - K) { const cpx<T> a = rv[N - r]; z = cpx<T>{a.x, -a.y}; }
        }
        v[e] = z;
      }
      FI::run(v, gi, tw, ex, WarpSync());
      // products (multReal, 2D_NavierStokes/src_RK4/kernels.h:187-201): p = v w, q = u w
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cpx<T>{v[e].x * w[e] * scale, u[e] * w[e] * scale};
      FX::run(v, gi, tw + N, ex, WarpSync());
#pragma unroll
      for (int e = 0; e < E; ++e) ex[FX::out_index(gi, e)] = v[e];
      __syncwarp();
      if (live) {
        cpx<T>* P = I.work + (long)y * X;
        cpx<T>* Q = P + (long)N * X;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int k = FX::out_index(gi, e);
          if (k <= K) {
            const cpx<T> a = v[e], b = ex[(N - k) & (N - 1)];
            P[k] = cpx<T>{(T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y)};
            Q[k] = cpx<T>{(T)0.5 * (a.y + b.y), (T)(-0.5) * (a.x - b.x)};
          }
        }
      }
      __syncwarp();
    }
  }

  // phase 3: y-forward of both products, spectral finish and RK4 stage s
  static __device__ void phase3(const Inst2D<T>& I, const cpx<T>* tw, cpx<T>* ex, int s) {
    const int gid = threadIdx.x / G, gi = threadIdx.x % G, ng = blockDim.x / G;
    for (int base = 0; base < X; base += ng) {
      const int ikx = base + gid;
      const bool live = ikx < X;
      cpx<T> a[E], b[E];
      const cpx<T>* src = I.work + (live ? ikx : 0);
#pragma unroll
      for (int e = 0; e < E; ++e) a[e] = live ? src[FO::in_index(gi, e) * X] : czero<T>();
      FO::run(a, gi, tw, ex, WarpSync());
#pragma unroll
      for (int e = 0; e < E; ++e)
        b[e] = live ? src[(long)N * X + FO::in_index(gi, e) * X] : czero<T>();
      FO::run(b, gi, tw, ex, WarpSync());
      if (!live) continue;
      const T dt = I.dt;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int iky = row_to_box2(FO::out_index(gi, e), K, N);
        if (iky < 0) continue;
        const int ky = iky - K;
        const int ik = iky * X + ikx;
        if (!keep2(ikx, ky, K)) {
          // masked modes: Z = 0, Z0 untouched (kernels.h:285-295)
          I.Z[ik] = czero<T>();
          continue;
        }
        const T kx = (T)ikx, kyT = (T)ky;
        // N = -i (kx F(u w) + ky F(v w)) (kernels.h:260-261); forcing -2 at (0, +-4)
        T NX = kx * b[e].y + kyT * a[e].y;
        const T NY = -kx * b[e].x - kyT * a[e].x;
        if (ikx == 0 && (ky == 4 || ky == -4)) NX -= (T)2;
        const cpx<T> d = cpx<T>{dt * NX, dt * NY};
        const cpx<T> z = I.Z[ik];
        if (s == 0) {
          I.Z1[ik] = d;
          I.Z0[ik] = cpx<T>{z.x + (T)0.5 * d.x, z.y + (T)0.5 * d.y};
        } else if (s == 1) {
          I.Z2[ik] = d;
          I.Z0[ik] = cpx<T>{z.x + (T)0.5 * d.x, z.y + (T)0.5 * d.y};
        } else if (s == 2) {
          I.Z3[ik] = d;
          I.Z0[ik] = cpx<T>{z.x + d.x, z.y + d.y};
        } else {
          const T wk = kx * kx + kyT * kyT;
          const T damp1 = (T)1 - (T)0.5 * dt * I.nu * wk;
          const T damp2 = (T)1 / ((T)1 + (T)0.5 * dt * I.nu * wk);
          const cpx<T> z1 = I.Z1[ik], z2 = I.Z2[ik], z3 = I.Z3[ik];
          const cpx<T> zn = cpx<T>{
              damp2 * (damp1 * z.x + (z1.x + (T)2 * z2.x + (T)2 * z3.x + d.x) / (T)6),
              damp2 * (damp1 * z.y + (z1.y + (T)2 * z2.y + (T)2 * z3.y + d.y) / (T)6)};
          I.Z[ik] = zn;
          I.Z0[ik] = zn;
        }
      }
    }
  }

  // gtw: the plain plan's twiddle table followed by the swapped plan's (2N entries)
  static __device__ void run(const Inst2D<T>& I, const cpx<T>* __restrict__ gtw, cpx<T>* smem) {
    cpx<T>* tw = smem;
    cpx<T>* ex = smem + 2 * N + (threadIdx.x / G) * FI::SMEM;
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) tw[i] = gtw[i];
    // setVelocity: Z0 = Z on kept modes, 0 elsewhere (kernels.h:112-147)
    for (int ik = threadIdx.x; ik < X * Y; ik += blockDim.x) {
      const int iky = ik / X, ikx = ik % X;
      I.Z0[ik] = keep2(ikx, iky - K, K) ? I.Z[ik] : czero<T>();
    }
    __syncthreads();
    for (int step = 0; step < I.nsteps; ++step) {
      for (int s = 0; s < 4; ++s) {
        phase1(I, tw, ex);
        __syncthreads();
        phase2(I, tw, ex);
        __syncthreads();
        phase3(I, tw, ex, s);
        __syncthreads();
      }
    }
  }
};

template <typename T>
struct Twiddles2D {
  const cpx<T>* t[5];  // n = 16, 32, 64, 128, 256
};

template <typename T>
__global__ void __launch_bounds__(256)
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
      case 16: Rhs2D<T, 16>::run(I, tws.t[0], smem); break;
      case 32: Rhs2D<T, 32>::run(I, tws.t[1], smem); break;
      case 64: Rhs2D<T, 64>::run(I, tws.t[2], smem); break;
      case 128: Rhs2D<T, 128>::run(I, tws.t[3], smem); break;
      default: Rhs2D<T, 256>::run(I, tws.t[4], smem); break;
    }
  }
}

template <typename T>
__global__ void ref_to_dev2(const double2* __restrict__ src, cpx<T>* __restrict__ dst, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = cpx<T>{(T)src[i].x, (T)src[i].y};
}
template <typename T>
__global__ void dev_to_ref2(const cpx<T>* __restrict__ src, double2* __restrict__ dst, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = make_double2((double)src[i].x, (double)src[i].y);
}

inline int nkt2(int n) { const int K = n / 3; return (K + 1) * (2 * K + 1); }

// twiddle tables of every 2D size up to nmax, each as [plain plan | swapped plan]
template <typename T>
void tables2d(cpx<T>* h, int nmax = 256) {
  long o = 0;
  if (nmax >= 16) { LineFFT<16, 1, T>::host_table(h + o); LineFFT<16, 1, T, true>::host_table(h + o + 16); o += 32; }
  if (nmax >= 32) { LineFFT<32, 1, T>::host_table(h + o); LineFFT<32, 1, T, true>::host_table(h + o + 32); o += 64; }
  if (nmax >= 64) { LineFFT<64, 1, T>::host_table(h + o); LineFFT<64, 1, T, true>::host_table(h + o + 64); o += 128; }
  if (nmax >= 128) { LineFFT<128, 1, T>::host_table(h + o); LineFFT<128, 1, T, true>::host_table(h + o + 128); o += 256; }
  if (nmax >= 256) { LineFFT<256, 1, T>::host_table(h + o); LineFFT<256, 1, T, true>::host_table(h + o + 256); o += 512; }
}

// ---------------------------------------------------------------------------
// batched host engine
// ---------------------------------------------------------------------------
struct Batch2DBase {
  virtual ~Batch2DBase() {}
  virtual int upload(int i, const double* Z) = 0;
  virtual int download(int i, double* Z) = 0;
  virtual int run(const double* nu, const double* dt, const int* nsteps) = 0;
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
  size_t smem = 0;

  ~Batch2D() override {
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
      total += 5L * nkt2(n);
      maxk = std::max<long>(maxk, nkt2(n));
    }
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
      worst = std::max(worst, (size_t)(2 * n + (256 / gg) * ss));
    }
    (void)g; (void)sm;
    smem = sizeof(cpx<T>) * worst;
    PSG_CUDA_TRY(cudaFuncSetAttribute(ns2d_persistent<T>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return PSG_OK;
  }

  int upload(int i, const double* Z) override {
    if (i < 0 || i >= ninst) { psg_set_error("instance %d out of range", i); return PSG_ERR_ARG; }
    const long nk = nkt2(sizes[i]);
    PSG_CUDA_TRY(cudaMemcpyAsync(staging, Z, sizeof(double2) * nk, cudaMemcpyHostToDevice, stream));
    ref_to_dev2<T><<<148, 256, 0, stream>>>(staging, pool + offs[i], nk);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  int download(int i, double* Z) override {
    if (i < 0 || i >= ninst) { psg_set_error("instance %d out of range", i); return PSG_ERR_ARG; }
    const long nk = nkt2(sizes[i]);
    dev_to_ref2<T><<<148, 256, 0, stream>>>(pool + offs[i], staging, nk);
    ++launches;
    PSG_CUDA_TRY(cudaMemcpyAsync(Z, staging, sizeof(double2) * nk, cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }

  int run(const double* nu, const double* dt, const int* nsteps) override {
    std::vector<Inst2D<T>> h(ninst);
    for (int j = 0; j < ninst; ++j) {
      const int i = order[j];
      const long nk = nkt2(sizes[i]);
      Inst2D<T>& I = h[j];
      I.n = sizes[i]; I.nsteps = nsteps[i]; I.nu = (T)nu[i]; I.dt = (T)dt[i];
      cpx<T>* b = pool + offs[i];
      I.Z = b; I.Z0 = b + nk; I.Z1 = b + 2 * nk; I.Z2 = b + 3 * nk; I.Z3 = b + 4 * nk;
      I.work = pool + woffs[i];
    }
    PSG_CUDA_TRY(cudaMemcpyAsync(d_insts, h.data(), sizeof(Inst2D<T>) * ninst,
                                 cudaMemcpyHostToDevice, stream));
    PSG_CUDA_TRY(cudaMemsetAsync(d_next, 0, sizeof(int), stream));
    Twiddles2D<T> tws;
    long o = 0;
    for (int q = 0, n = 16; q < 5; ++q, n *= 2) { tws.t[q] = twp + o; o += 2 * n; }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ns2d_persistent<T>, 256, smem);
    const int grid = std::max(1, std::min(ninst, nsm * std::max(per_sm, 1)));
    ns2d_persistent<T><<<grid, 256, smem, stream>>>(d_insts, ninst, d_next, tws);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
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
// the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr int kNoallocMaxN = 128;
constexpr size_t kNoallocBytes = 512 * 1024;
constexpr size_t kTw64Off = 0;          // 480 complex doubles (n = 16..128, two plans each)
constexpr size_t kTw32Off = 8192;       // 480 complex floats
constexpr size_t kWorkOff = 12288;      // Z0..Z3 and row scratch

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
// Nothing here allocates device memory.
int noalloc_setup(unsigned char** out) {
  int dev = 0;
  PSG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    psg_set_error("device ordinal %d beyond %d", dev, kMaxDevices);
    return PSG_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_addr[dev]) { *out = g_noalloc_addr[dev]; return PSG_OK; }
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
  I.work = work + 4 * nk;
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
  // the largest footprint must fit the array: 4 stage registers + 3 scratch rows
  const size_t need = kWorkOff + (size_t)16 * (4 * nkt2(kNoallocMaxN) + 3L * kNoallocMaxN * (kNoallocMaxN / 3 + 1));
  static_assert(kWorkOff + 16ull * (4 * 3655 + 3 * 128 * 43) <= kNoallocBytes, "scratch too small");
  static_assert(kTw64Off + 480 * 16 <= kTw32Off && kTw32Off + 480 * 8 <= kWorkOff, "twiddle tables");
  (void)need;
  unsigned char* base = nullptr;
  int rc = noalloc_setup(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  return precision == 64 ? noalloc_run<double>(base, n, nu, dt, nsteps, z_in, z_out, s)
                         : noalloc_run<float>(base, n, nu, dt, nsteps, z_in, z_out, s);
}
