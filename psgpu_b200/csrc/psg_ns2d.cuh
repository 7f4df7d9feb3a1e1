// psg_ns2d.cuh -- device building blocks of the 2D vorticity step shared by
// the batched engine (psg_ns2d.cu) and the UPO solver (psg_newton2d.cu).
//
// A 2D instance (N <= 256) is integrated by one thread block; every right-hand
// side is three phases separated by block barriers,
//   1. y-inverse of w, u = i ky w / k^2, v = -i kx w / k^2  (K+1 columns each)
//   2. x rows: C2R of (w,u) and (v), products v w and u w scaled by 1/N^2,
//      R2C of the packed pair, kx <= K kept (in place in the row scratch)
//   3. y-forward of both products per column, kept ky rows, then
//      N = -i (kx F(u w) + ky F(v w)), the Kolmogorov forcing and the RK4 stage
// with the intermediate rows in a per-instance scratch that stays in L2.
//
// The scheme restates 2D_NavierStokes/src_RK4/kernels.h:112-435 (setVelocity,
// Step1, Step2, Step) and the transforms replace conj -> setFFN -> Z2D,
// multReal, batched D2Z -> normFF1 (2D_NavierStokes/src_RK4/functions.h:33-149).
#pragma once
#include <math.h>

#include "psg_common.cuh"
#include "psg_fft.cuh"
#include "psg_fft2.cuh"

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
  cpx<T>* ZC;    // carried rounding error of the state updates (FP32), or null
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

// PK (FP32 only): the transforms of two lines at once as packed f32x2 ones
// (psg_fft2.cuh): phase 1 two columns per lane group, phase 2 the inverse rows
// of (w + i u) and v together, phase 3 the two product columns together.  The
// batch's autotuner picks PK per grid size (Batch2D::autotune).
template <typename T, int N, int PK = 0>
struct Rhs2D {
  static_assert(PK == 0 || sizeof(T) == 4, "packed transforms are FP32");
  using FI = LineFFT<N, +1, T>;
  using FO = LineFFT<N, -1, T>;
  using FX = LineFFT<N, -1, T, true>;  // forward transform of phase 2: consumes FI's output
  static constexpr int G = FI::G, E = FI::E;
  static constexpr int K = N / 3, X = K + 1, Y = 2 * K + 1;

  // phase 1, packed: columns 2p and 2p + 1 of the 3X (three fields) together
  static __device__ void phase1_pk(const Inst2D<T>& I, const cpx<T>* tw, cpx<T>* ex) {
    const int gid = threadIdx.x / G, gi = threadIdx.x % G, ng = blockDim.x / G;
    constexpr int NP = (3 * X + 1) / 2;
    for (int base = 0; base < NP; base += ng) {
      const int p = base + gid;
      const int c0 = 2 * p, c1 = 2 * p + 1;
      const bool l0 = c0 < 3 * X, l1 = c1 < 3 * X;
      const int f0 = l0 ? c0 / X : 0, x0 = l0 ? c0 % X : 0;
      const int f1 = l1 ? c1 / X : 0, x1 = l1 ? c1 % X : 0;
      Pk v[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int iky = row_to_box2(FI::in_index(gi, e), K, N);
        const cpx<T> a = (l0 && iky >= 0) ? field2(I.Z0, f0, x0, iky, K, X) : czero<T>();
        const cpx<T> b = (l1 && iky >= 0) ? field2(I.Z0, f1, x1, iky, K, X) : czero<T>();
        v[e] = Pk{make_float2(a.x, b.x), make_float2(a.y, b.y)};
      }
      LineFFT2<N, +1>::run(v, gi, tw, reinterpret_cast<float2*>(ex), WarpSync());
      if (l0) {
        cpx<T>* dst = I.work + (long)f0 * N * X + x0;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[FI::out_index(gi, e) * X] = cpx<T>{v[e].re.x, v[e].im.x};
      }
      if (l1) {
        cpx<T>* dst = I.work + (long)f1 * N * X + x1;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[FI::out_index(gi, e) * X] = cpx<T>{v[e].re.y, v[e].im.y};
      }
    }
  }

  // phase 1: y-inverse of the three fields, written to work[f][y][kx]
  static __device__ void phase1(const Inst2D<T>& I, const cpx<T>* tw, cpx<T>* ex) {
    if constexpr (PK != 0) { phase1_pk(I, tw, ex); return; }
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
      T w[E], u[E];
      if constexpr (PK != 0) {
        // (w + i u) and v (its Hermitian line) through one packed transform
        Pk pv[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int r = FI::in_index(gi, e);
          cpx<T> za = czero<T>(), zb = czero<T>();
          if (live) {
            if (r == 0) {
              za = cpx<T>{rw[0].x, ru[0].x};
              zb = cpx<T>{rv[0].x, (T)0};
            } else if (r <= K) {
              const cpx<T> a = rw[r], b = ru[r];
              za = cpx<T>{a.x - b.y, a.y + b.x};
              zb = rv[r];
            } else if (r >= N - K) {
              const cpx<T> a = rw[N - r], b = ru[N - r], c = rv[N - r];
              za = cpx<T>{a.x + b.y, -a.y + b.x};
              zb = cpx<T>{c.x, -c.y};
            }
          }
          pv[e] = Pk{make_float2(za.x, zb.x), make_float2(za.y, zb.y)};
        }
        LineFFT2<N, +1>::run(pv, gi, tw, reinterpret_cast<float2*>(ex), WarpSync());
#pragma unroll
        for (int e = 0; e < E; ++e) {
          w[e] = pv[e].re.x; u[e] = pv[e].im.x;
          v[e] = cpx<T>{pv[e].re.y, pv[e].im.y};
        }
      } else {
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
      }
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
      if constexpr (PK != 0) {
        // both product columns through one packed transform
        Pk pv[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const cpx<T> x = live ? src[FO::in_index(gi, e) * X] : czero<T>();
          const cpx<T> y = live ? src[(long)N * X + FO::in_index(gi, e) * X] : czero<T>();
          pv[e] = Pk{make_float2(x.x, y.x), make_float2(x.y, y.y)};
        }
        LineFFT2<N, -1>::run(pv, gi, tw, reinterpret_cast<float2*>(ex), WarpSync());
#pragma unroll
        for (int e = 0; e < E; ++e) {
          a[e] = cpx<T>{pv[e].re.x, pv[e].im.x};
          b[e] = cpx<T>{pv[e].re.y, pv[e].im.y};
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) a[e] = live ? src[FO::in_index(gi, e) * X] : czero<T>();
        FO::run(a, gi, tw, ex, WarpSync());
#pragma unroll
        for (int e = 0; e < E; ++e)
          b[e] = live ? src[(long)N * X + FO::in_index(gi, e) * X] : czero<T>();
        FO::run(b, gi, tw, ex, WarpSync());
      }
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
          if (I.ZC) I.ZC[ik] = czero<T>();
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
          // ((1 - x/2) z + incr) / (1 + x/2), x = nu k^2 dt, evaluated as
          // (z - eS z) + (incr - eI incr) so that only the small eS, eI are
          // rounded (the factor repeats every step and its rounding would
          // compound over a run)
          const T wk = kx * kx + kyT * kyT;
          const T x = dt * I.nu * wk, hx = (T)0.5 * x;
          const T eS = x / ((T)1 + hx), eI = hx / ((T)1 + hx);
          const cpx<T> z1 = I.Z1[ik], z2 = I.Z2[ik], z3 = I.Z3[ik];
          const T ix = (z1.x + (T)2 * z2.x + (T)2 * z3.x + d.x) / (T)6;
          const T iy = (z1.y + (T)2 * z2.y + (T)2 * z3.y + d.y) / (T)6;
          const T yx = (ix - eI * ix) - eS * z.x, yy = (iy - eI * iy) - eS * z.y;
          cpx<T> zn;
          if (I.ZC) {  // carry the rounding error of z + y to the next step
            const cpx<T> c = I.ZC[ik];
            const T ax = yx + c.x, ay = yy + c.y;
            zn.x = z.x + ax;
            zn.y = z.y + ay;
            const T bx = zn.x - z.x, by = zn.y - z.y;
            I.ZC[ik] = cpx<T>{(z.x - (zn.x - bx)) + (ax - bx), (z.y - (zn.y - by)) + (ay - by)};
          } else {
            zn = cpx<T>{z.x + yx, z.y + yy};
          }
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


}  // namespace psg
