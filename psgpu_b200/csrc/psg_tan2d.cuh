// psg_tan2d.cuh -- tangent-linear 2D step and the 2D time derivative.
//
// The tangent of the reference's 2D RK4/CN step (2D_NavierStokes/src_RK4/
// kernels.h:247-435) is integrated together with the base trajectory: every
// stage transforms the base fields (w, u, v) and the perturbation fields
// (dw, du, dv), forms the products and their linearisation
//     d(v w) = dv w + v dw,   d(u w) = du w + u dw
// and applies the same stage coefficients to the base and the perturbation
// (the forcing is constant and drops out of the perturbation).  Integrating
// the pair over a period T gives Phi_T(z) and the exact Jacobian-vector
// product J(z) q of the discrete step, with no finite-difference error.
//
// The time derivative dz/dt = -nu k^2 z + N(z) + forcing restates the Newton
// solver's TIMEDERIV (2D_NavierStokes/src_RK4/src_gmres/timederiv.F90:2-32),
// with nu k^2 in place of the driver's 10**(log10 nu + 2 log10 |k|).
#pragma once
#include "psg_ns2d.cuh"

namespace psg {

template <typename T>
struct InstTan2D {
  int n;       // grid points per direction
  int nsteps;  // RK4 steps
  T nu, dt;
  int mode;    // 0: base + tangent steps; 1: base only; 2: time derivative of Z into D
  cpx<T>* Z;   // base state (in/out)
  cpx<T>* Z0;  // base stage state
  cpx<T>* Z1;
  cpx<T>* Z2;
  cpx<T>* Z3;
  cpx<T>* D;   // perturbation (in/out); mode 2: the derivative
  cpx<T>* D0;
  cpx<T>* D1;
  cpx<T>* D2;
  cpx<T>* D3;
  cpx<T>* work;  // [6][n][K+1]
};

// The thread blocks that integrate one instance together: one block, or the
// two blocks of a cluster, each taking every other group of lines in every
// phase (the row scratch is in global memory, so no shared memory crosses
// blocks); the phases are separated by a block or a cluster barrier.
struct Team {
  int rank, size;
};

__device__ __forceinline__ void team_sync(const Team& t) {
  if (t.size == 1) {
    __syncthreads();
  } else {
    // release this block's global writes at cluster scope, then wait for the
    // other block's (barrier.cluster with release / acquire semantics)
    asm volatile(
        "fence.acq_rel.cluster;\n\t"
        "barrier.cluster.arrive.release.aligned;\n\t"
        "barrier.cluster.wait.acquire.aligned;" ::: "memory");
  }
}

template <typename T, int N>
struct Tan2D {
  using FI = LineFFT<N, +1, T>;
  using FO = LineFFT<N, -1, T>;
  using FX = LineFFT<N, -1, T, true>;
  static constexpr int G = FI::G, E = FI::E;
  static constexpr int K = N / 3, X = K + 1, Y = 2 * K + 1;

  // phase 1: y-inverse of nf fields (0..2 base from Z0, 3..5 perturbation from D0)
  static __device__ void phase1(const InstTan2D<T>& I, const cpx<T>* tw, cpx<T>* ex, int nf,
                                const Team& t) {
    const int gid = t.rank * (blockDim.x / G) + threadIdx.x / G, gi = threadIdx.x % G;
    const int ng = t.size * (blockDim.x / G);
    for (int base = 0; base < nf * X; base += ng) {
      const int col = base + gid;
      const bool live = col < nf * X;
      const int f = live ? col / X : 0, ikx = live ? col % X : 0;
      const cpx<T>* src = (f < 3) ? I.Z0 : I.D0;
      const int ff = f % 3;
      cpx<T> v[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int iky = row_to_box2(FI::in_index(gi, e), K, N);
        v[e] = (live && iky >= 0) ? field2(src, ff, ikx, iky, K, X) : czero<T>();
      }
      FI::run(v, gi, tw, ex, WarpSync());
      if (live) {
        cpx<T>* dst = I.work + (long)f * N * X + ikx;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[FI::out_index(gi, e) * X] = v[e];
      }
    }
  }

  static __device__ __forceinline__ void load_pair(const cpx<T>* ra, const cpx<T>* rb, int gi,
                                                   bool live, cpx<T> (&v)[E]) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int r = FI::in_index(gi, e);
      cpx<T> z = czero<T>();
      if (live) {
        if (r == 0) {
          z = cpx<T>{ra[0].x, rb ? rb[0].x : (T)0};
        } else if (r <= K) {
          const cpx<T> a = ra[r], b = rb ? rb[r] : czero<T>();
          z = cpx<T>{a.x - b.y, a.y + b.x};
        } else if (r >= N - K) {
          const cpx<T> a = ra[N - r], b = rb ? rb[N - r] : czero<T>();
          z = cpx<T>{a.x + b.y, -a.y + b.x};
        }
      }
      v[e] = z;
    }
  }

  // forward transform of p + i q and split into P, Q (kx <= K)
  static __device__ __forceinline__ void store_pair(cpx<T> (&v)[E], int gi, bool live,
                                                    const cpx<T>* tw2, cpx<T>* ex, cpx<T>* P,
                                                    cpx<T>* Q) {
    FX::run(v, gi, tw2, ex, WarpSync());
#pragma unroll
    for (int e = 0; e < E; ++e) ex[FX::out_index(gi, e)] = v[e];
    __syncwarp();
    if (live) {
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

  // phase 2: rows.  Base products (v w, u w) -> work[0], work[1]; with the
  // perturbation, their linearisation -> work[2], work[3].
  static __device__ void phase2(const InstTan2D<T>& I, const cpx<T>* tw, cpx<T>* ex, bool tan,
                                const Team& t) {
    const int gid = t.rank * (blockDim.x / G) + threadIdx.x / G, gi = threadIdx.x % G;
    const int ng = t.size * (blockDim.x / G);
    const T scale = (T)1 / ((T)N * (T)N);
    const long fs = (long)N * X;
    for (int base = 0; base < N; base += ng) {
      const int y = base + gid;
      const bool live = y < N;
      const cpx<T>* r0 = I.work + (long)(live ? y : 0) * X;
      cpx<T> v[E];
      load_pair(r0, r0 + fs, gi, live, v);  // (w, u)
      FI::run(v, gi, tw, ex, WarpSync());
      T w[E], u[E];
#pragma unroll
      for (int e = 0; e < E; ++e) { w[e] = v[e].x; u[e] = v[e].y; }
      load_pair(r0 + 2 * fs, tan ? r0 + 5 * fs : nullptr, gi, live, v);  // (v, dv)
      FI::run(v, gi, tw, ex, WarpSync());
      T vv[E], dp[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        vv[e] = v[e].x;
        dp[e] = v[e].y * w[e];  // dv w
        v[e] = cpx<T>{vv[e] * w[e] * scale, u[e] * w[e] * scale};
      }
      cpx<T>* P = I.work + (long)(live ? y : 0) * X;
      store_pair(v, gi, live, tw + N, ex, P, P + fs);
      if (!tan) continue;
      load_pair(r0 + 3 * fs, r0 + 4 * fs, gi, live, v);  // (dw, du)
      FI::run(v, gi, tw, ex, WarpSync());
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const T dw = v[e].x, du = v[e].y;
        v[e] = cpx<T>{(dp[e] + vv[e] * dw) * scale, (du * w[e] + u[e] * dw) * scale};
      }
      store_pair(v, gi, live, tw + N, ex, P + 2 * fs, P + 3 * fs);
    }
  }

  // N(z) at (ikx, ky) from F(v w) = a, F(u w) = b (2D_NavierStokes/src_RK4/kernels.h:260-261)
  static __device__ __forceinline__ cpx<T> nl(cpx<T> a, cpx<T> b, int ikx, int ky) {
    const T kx = (T)ikx, kyT = (T)ky;
    return cpx<T>{kx * b.y + kyT * a.y, -kx * b.x - kyT * a.x};
  }

  // RK4 stage s applied to (Z, Z0, Z1..Z3) with increment d = dt * rhs
  static __device__ __forceinline__ void stage(cpx<T>* Zs, cpx<T>* Z0s, cpx<T>* Z1s, cpx<T>* Z2s,
                                               cpx<T>* Z3s, int ik, int s, cpx<T> d, T damp1,
                                               T damp2) {
    const cpx<T> z = Zs[ik];
    if (s == 0) {
      Z1s[ik] = d;
      Z0s[ik] = cpx<T>{z.x + (T)0.5 * d.x, z.y + (T)0.5 * d.y};
    } else if (s == 1) {
      Z2s[ik] = d;
      Z0s[ik] = cpx<T>{z.x + (T)0.5 * d.x, z.y + (T)0.5 * d.y};
    } else if (s == 2) {
      Z3s[ik] = d;
      Z0s[ik] = cpx<T>{z.x + d.x, z.y + d.y};
    } else {
      const cpx<T> z1 = Z1s[ik], z2 = Z2s[ik], z3 = Z3s[ik];
      const cpx<T> zn = cpx<T>{
          damp2 * (damp1 * z.x + (z1.x + (T)2 * z2.x + (T)2 * z3.x + d.x) / (T)6),
          damp2 * (damp1 * z.y + (z1.y + (T)2 * z2.y + (T)2 * z3.y + d.y) / (T)6)};
      Zs[ik] = zn;
      Z0s[ik] = zn;
    }
  }

  // phase 3: y-forward, spectral finish, stage update (s >= 0) or derivative (s < 0)
  static __device__ void phase3(const InstTan2D<T>& I, const cpx<T>* tw, cpx<T>* ex, int s,
                                bool tan, const Team& t) {
    const int gid = t.rank * (blockDim.x / G) + threadIdx.x / G, gi = threadIdx.x % G;
    const int ng = t.size * (blockDim.x / G);
    const long fs = (long)N * X;
    for (int base = 0; base < X; base += ng) {
      const int ikx = base + gid;
      const bool live = ikx < X;
      const cpx<T>* src = I.work + (live ? ikx : 0);
      for (int part = 0; part < (tan ? 2 : 1); ++part) {
        cpx<T> a[E], b[E];
        const cpx<T>* sp = src + 2 * part * fs;
#pragma unroll
        for (int e = 0; e < E; ++e) a[e] = live ? sp[FO::in_index(gi, e) * X] : czero<T>();
        FO::run(a, gi, tw, ex, WarpSync());
#pragma unroll
        for (int e = 0; e < E; ++e) b[e] = live ? sp[fs + FO::in_index(gi, e) * X] : czero<T>();
        FO::run(b, gi, tw, ex, WarpSync());
        if (!live) continue;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int iky = row_to_box2(FO::out_index(gi, e), K, N);
          if (iky < 0) continue;
          const int ky = iky - K;
          const int ik = iky * X + ikx;
          const bool keep = keep2(ikx, ky, K);
          if (s < 0) {  // time derivative of the base state
            cpx<T> d = czero<T>();
            if (keep) {
              cpx<T> r = nl(a[e], b[e], ikx, ky);
              if (ikx == 0 && ky == 4) r.x -= (T)2;
              const T wk = (T)(ikx * ikx + ky * ky);
              const cpx<T> z = I.Z[ik];
              d = cpx<T>{-I.nu * wk * z.x + r.x, -I.nu * wk * z.y + r.y};
            }
            I.D[ik] = d;
            continue;
          }
          cpx<T>* Zs = part ? I.D : I.Z;
          if (!keep) { Zs[ik] = czero<T>(); continue; }
          cpx<T> r = nl(a[e], b[e], ikx, ky);
          if (part == 0 && ikx == 0 && (ky == 4 || ky == -4)) r.x -= (T)2;
          const T wk = (T)(ikx * ikx + ky * ky);
          const T damp1 = (T)1 - (T)0.5 * I.dt * I.nu * wk;
          const T damp2 = (T)1 / ((T)1 + (T)0.5 * I.dt * I.nu * wk);
          const cpx<T> d = cpx<T>{I.dt * r.x, I.dt * r.y};
          if (part == 0) stage(I.Z, I.Z0, I.Z1, I.Z2, I.Z3, ik, s, d, damp1, damp2);
          else stage(I.D, I.D0, I.D1, I.D2, I.D3, ik, s, d, damp1, damp2);
        }
      }
    }
  }

  static __device__ void run(const InstTan2D<T>& I, const cpx<T>* __restrict__ gtw, cpx<T>* smem,
                             Team t = Team{0, 1}) {
    cpx<T>* tw = smem;
    cpx<T>* ex = smem + 2 * N + (threadIdx.x / G) * FI::SMEM;
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) tw[i] = gtw[i];
    const bool tan = (I.mode == 0);
    for (int ik = t.rank * blockDim.x + threadIdx.x; ik < X * Y; ik += t.size * blockDim.x) {
      const int iky = ik / X, ikx = ik % X;
      const bool keep = keep2(ikx, iky - K, K);
      I.Z0[ik] = keep ? I.Z[ik] : czero<T>();
      if (tan) I.D0[ik] = keep ? I.D[ik] : czero<T>();
    }
    team_sync(t);
    if (I.mode == 2) {
      phase1(I, tw, ex, 3, t);
      team_sync(t);
      phase2(I, tw, ex, false, t);
      team_sync(t);
      phase3(I, tw, ex, -1, false, t);
      team_sync(t);
      return;
    }
    for (int step = 0; step < I.nsteps; ++step) {
      for (int s = 0; s < 4; ++s) {
        phase1(I, tw, ex, tan ? 6 : 3, t);
        team_sync(t);
        phase2(I, tw, ex, tan, t);
        team_sync(t);
        phase3(I, tw, ex, s, tan, t);
        team_sync(t);
      }
    }
  }
};

}  // namespace psg
