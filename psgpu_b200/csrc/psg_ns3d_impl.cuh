// psg_ns3d_impl.cuh -- sm_100a kernels and host engine of the 3D pseudospectral step
// (Navier-Stokes Heun/CN, Euler Heun, Navier-Stokes RK4/CN, Boussinesq RK4/CN).
//
// See psg_ns3d.cuh for the pass structure.  Each scheme update restates the
// reference kernel cited beside it; the transforms replace the reference's
// conj -> setFFN -> cufftExecZ2D -> multReal -> cufftExecD2Z -> normFF1
// sequence (3D_NavierStokes/src/functions.h:26-108).
//
// Data layout (complex T, W = 8 kx columns per tile, XT = XP / W tiles):
//   state / registers  S[c][xt][ky][kz][W]     pass A reads, pass E writes one tile
//   B1 (A -> B)        [f][xt][z][ky][W]       pass B reads one [ky][W] tile
//   B2 (B -> C)        [f][z][y][XP]           pass C reads L whole rows
//   B3 (C -> D)        [f][xt][z][y][W]        pass D reads one [y][W] tile
//   B4 (D -> E)        [f][xt][ky][z][W]       pass E reads one [z][W] tile
// so that every pass's input tile is one contiguous chunk of HBM, moved into
// shared memory by a single TMA bulk copy (cp.async.bulk) per field; outputs
// are written as full 64-byte segments.
#pragma once
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <type_traits>
#include <vector>

#include "psg_fft2.cuh"
#include "psg_ns3d.cuh"
#include "psg_tma.cuh"
#include "psgpu_internal.h"

namespace psg {

constexpr int kTileW = 8;

// The truncated box of an N^3 grid as compile-time constants (the engine sets
// Geom3 to the same values: K = N/3, X = K+1, Y = 2K+1, XP = X rounded up to
// kTileW), so that the row <-> box index arithmetic of the passes folds.
template <int N>
struct Box {
  static constexpr int K = N / 3, X = K + 1, Y = 2 * K + 1;
  static constexpr int XP = (X + kTileW - 1) / kTileW * kTileW, XT = XP / kTileW;
};

// FFT row (0..n-1) -> box index (0..2K) or -1 when the row is truncated
__device__ __forceinline__ int row_to_box(int r, int K, int n) {
  if (r <= K) return r + K;
  if (r >= n - K) return r - n + K;
  return -1;
}

// 2/3-rule mask of the reference (3D_NavierStokes/src/init.F90:43-46) for
// integer box indices; alpha scales kx.
template <typename T>
__device__ __forceinline__ bool keep_mode(int ix, int ky, int kz, int K, T alpha) {
  if (ix == 0 && ky < 0) return false;
  if (ix == 0 && ky == 0 && kz <= 0) return false;
  const T kx = (T)ix * alpha;
  const T wk = kx * kx + (T)(ky * ky + kz * kz);
  const T lim = (T)K - (T)0.5;
  return !(wk > lim * lim);
}

template <typename T>
__device__ __forceinline__ T wkinv(T wk) {
  return (T)1 / (wk > (T)0.001 ? wk : (T)0.001);
}

// exchange stride per column of a column-pass tile: congruent to 2 mod 16
// complex words, so that the 8 columns x 4 threads of a warp fall on distinct
// banks in both exchange directions
template <int S>
struct ColStride {
  static constexpr int value = S + ((2 - (S % 16)) + 16) % 16;
};
// exchange stride per row of the row pass: groups of G lanes share a warp
template <int S, int G>
struct RowStride {
  static constexpr int off = (G >= 16) ? 0 : (G == 8 ? 8 : 4);
  static constexpr int value = S + ((off - (S % 16)) + 16) % 16;
};

// Programmatic dependent launch.  pdl_trigger: the next kernel of the stream
// may be launched once every block of this one has executed it (its blocks
// then take the SM slots this grid's last blocks free, and run their set-up).
// pdl_wait: block until the kernels this launch depends on have completed and
// their writes are visible.  Every pass calls pdl_wait before its first global
// access other than the constant twiddle table, reads and writes alike (the
// next pass writes buffers the previous one reads), and issues its tile copy
// right after it, so that the table set-up runs while the copy is in flight in
// every wave of blocks.  Both are no-ops for a launch without the
// programmatic-serialisation attribute.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Load `n` contiguous chunks into shared memory with one mbarrier; returns
// false (uniformly) if the copy did not complete within the wait bound.
__device__ __forceinline__ bool tile_load(uint64_t* bar, int* s_ok, void* const* dst,
                                          const void* const* src, const uint32_t* bytes, int n,
                                          int* status) {
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int i = 0; i < n; ++i) tot += bytes[i];
    mbar_expect_tx(bar, tot);
    for (int i = 0; i < n; ++i) bulk_g2s(dst[i], src[i], bytes[i], bar);
  }
  return true;
}

__device__ __forceinline__ bool tile_wait(uint64_t* bar, int* s_ok, int* status) {
  if (threadIdx.x == 0) *s_ok = mbar_wait_bounded(bar, 0, status) ? 1 : 0;
  __syncthreads();
  return *s_ok != 0;
}

// ---------------------------------------------------------------------------
// pass A: z-inverse of the stage state with the velocity (and density
// gradient) formed in registers; Hermitian completion of the kx = 0 plane.
// grid (XT, Y): one [kz][W] tile of each state component.
//
// MODE 1 (pair): the two 3-vectors of a bilinear product, b = in (written to
// the w slots 0-2 that pass C reads as w) and a = in2 (the u slots 3-5), each
// passed through the spectral operator of `ops` (bits 0-3 for b, 4-7 for a:
// OP_ID, OP_CURL = i k x, OP_BS = i k x / k^2) and masked to the kept modes.
// MODE 2 (scale): the fields of the Boussinesq adjoint's scalar products,
// [psi, i k rho, B w] from psi = in2.c[0] and (w, rho) = in.c[0..3].
// ---------------------------------------------------------------------------
enum SpecOp : int { OP_ID = 0, OP_CURL = 1, OP_BS = 2 };

template <typename T>
__device__ __forceinline__ cpx<T> spec_op(int op, int comp, const cpx<T>* x, T kx, T ky, T kz, T wki) {
  if (op == OP_ID) return x[comp];
  cpx<T> r;  // (i k x x)_comp
  if (comp == 0) r = cpx<T>{-(ky * x[2].y - kz * x[1].y), ky * x[2].x - kz * x[1].x};
  else if (comp == 1) r = cpx<T>{-(kz * x[0].y - kx * x[2].y), kz * x[0].x - kx * x[2].x};
  else r = cpx<T>{-(kx * x[1].y - ky * x[0].y), kx * x[1].x - ky * x[0].x};
  if (op == OP_BS) { r.x *= wki; r.y *= wki; }
  return r;
}

// pass A's staging of one (xt, ky) tile: twiddles and the signed 1/k^2 table
// (negated where the 2/3 rule drops the mode), then the NC state tiles by bulk
// copy, and the kx = 0 column of tile 0 for ky <= 0 patched with the conjugate
// of the stored mode at (-ky, -kz) (Hermitian completion).  False (uniformly)
// if the copy did not complete within the wait bound.
template <typename T, int N, int NC, typename Src>
__device__ __forceinline__ bool a_stage(const Geom3<T>& g, Src src_comp, const cpx<T>* __restrict__ tw,
                                        cpx<T>* s_in, cpx<T>* s_tw, T* s_wk, uint64_t* s_bar,
                                        int* s_ok, int* status) {
  constexpr int W = kTileW;
  constexpr int Y = Box<N>::Y, K = Box<N>::K;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int xt = blockIdx.x, iky = blockIdx.y;
  const long tile = ((long)xt * Y + iky) * Y * W;
  pdl_trigger();
  if (tid == 0) mbar_init(s_bar, 1);
  __syncthreads();
  pdl_wait();
  if (tid == 0) {
    mbar_expect_tx(s_bar, (uint32_t)(NC * Y * W * sizeof(cpx<T>)));
    for (int q = 0; q < NC; ++q)
      bulk_g2s(s_in + q * Y * W, src_comp(q) + tile, (uint32_t)(Y * W * sizeof(cpx<T>)), s_bar);
  }
  // the tables while the copy is in flight
  for (int i = tid; i < N; i += nth) s_tw[i] = tw[i];
  const bool mirror = (xt == 0) && (iky <= K);
  for (int idx = tid; idx < Y * W; idx += nth) {
    const int ikz = idx / W, cc = idx % W, ikx = xt * W + cc;
    bool ll;
    if (ikx >= Box<N>::X) ll = false;
    else if (ikx == 0 && mirror && !(iky == K && ikz > K))  // value taken from the mirror mode
      ll = (iky == K && ikz == K) ? false : keep_mode<T>(0, K - iky, K - ikz, K, g.alpha);
    else ll = keep_mode<T>(ikx, iky - K, ikz - K, K, g.alpha);
    const T kx = (T)ikx * g.alpha, ky = (T)(iky - K), kz = (T)(ikz - K);
    const T wki = wkinv(kx * kx + ky * ky + kz * kz);
    s_wk[idx] = ll ? wki : -wki;
  }
  if (!tile_wait(s_bar, s_ok, status)) return false;
  if (mirror) {
    const long mt = (long)(2 * K - iky) * Y * W;
    for (int i = tid; i < NC * Y; i += nth) {
      const int q = i / Y, ikz = i % Y;
      cpx<T>* d = s_in + q * Y * W + ikz * W;
      if (iky == K && ikz == K) *d = czero<T>();
      else if (!(iky == K && ikz > K)) *d = cconj(src_comp(q)[mt + (long)(2 * K - ikz) * W]);
    }
    __syncthreads();
  }
  return true;
}

template <typename T, int N, int NC, int NF, int MODE = 0, int NG = 2>
__global__ void __launch_bounds__(NG * kTileW * LineFFT<N, 1, T>::G,
                                  sizeof(T) > 4 ? (N >= 256 ? 1 : 2) : (NG == 2 ? 3 : 2))
pass_a(Geom3<T> g, Fields4<T> in, cpx<T>* __restrict__ out, const cpx<T>* __restrict__ tw,
       int mask_vel, int* status, Fields4<T> in2 = Fields4<T>{}, int ops = 0) {
  using F = LineFFT<N, +1, T>;
  constexpr int W = kTileW;
  constexpr int SX = ColStride<F::SMEM>::value;
  constexpr int Y = Box<N>::Y, K = Box<N>::K, XT = Box<N>::XT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_ok;
  cpx<T>* s_in = reinterpret_cast<cpx<T>*>(smem_raw);   // [NC][Y][W]
  cpx<T>* s_tw = s_in + NC * Y * W;                       // [N]
  cpx<T>* s_ex = s_tw + N;                                // [NG][W][SX]
  // 1/k^2 of every mode of the tile, negated where the 2/3 rule drops the mode
  T* s_wk = reinterpret_cast<T*>(s_ex + NG * W * SX);     // [Y][W]

  // NG groups of W x G threads transform NG output fields at a time
  const int tid = threadIdx.x;
  const int grp = tid / (W * F::G), ht = tid % (W * F::G);
  const int c = ht % W, gi = ht / W;
  const int xt = blockIdx.x, iky = blockIdx.y;
  auto src_comp = [&](int q) -> const cpx<T>* {
    if (MODE == 1 && q >= 3) return in2.c[q - 3];
    if (MODE == 2 && q == 4) return in2.c[0];
    return in.c[q];
  };
  if (!a_stage<T, N, NC>(g, src_comp, tw, s_in, s_tw, s_wk, &s_bar, &s_ok, status)) return;

  const int ikx = xt * W + c;
  const T kx = (T)ikx * g.alpha;
  const T ky = (T)(iky - K);
  const bool live_col = ikx < Box<N>::X;
#pragma unroll 1
  for (int f0 = 0; f0 < NF; f0 += NG) {
    const int f = f0 + grp;
    const bool live = live_col && f < NF;
    cpx<T> v[F::E];
#pragma unroll
    for (int e = 0; e < F::E; ++e) {
      const int ikz = row_to_box(F::in_index(gi, e), K, N);
      const int o = ikz * W + c;
      cpx<T> r = czero<T>();
      if (ikz >= 0 && live) {
        const T kz = (T)(ikz - K);
        const T tk = s_wk[o];
        if (MODE == 1) {
          if (tk > (T)0) {
            const int sl = f / 3, comp = f % 3;
            const cpx<T> x[3] = {s_in[(3 * sl) * Y * W + o], s_in[(3 * sl + 1) * Y * W + o],
                                 s_in[(3 * sl + 2) * Y * W + o]};
            r = spec_op<T>((ops >> (4 * sl)) & 15, comp, x, kx, ky, kz, tk);
          }
        } else if (MODE == 2) {
          if (tk > (T)0) {
            if (f == 0) {
              r = s_in[4 * Y * W + o];
            } else if (f <= 3) {  // i k_j rho
              const cpx<T> rho = s_in[3 * Y * W + o];
              const T kk = (f == 1) ? kx : (f == 2) ? ky : kz;
              r = cpx<T>{-kk * rho.y, kk * rho.x};
            } else {
              const cpx<T> x[3] = {s_in[o], s_in[Y * W + o], s_in[2 * Y * W + o]};
              r = spec_op<T>(OP_BS, f - 4, x, kx, ky, kz, tk);
            }
          }
        } else if (f < 3) {
          r = s_in[f * Y * W + o];
        } else if (f < 6) {
          // u = i k x w / k^2 (3D_NavierStokes/src/kernels.h:194-201)
          const T wki = (mask_vel && tk < (T)0) ? (T)0 : fabs(tk);
          const cpx<T> xi = s_in[o], et = s_in[Y * W + o], zt = s_in[2 * Y * W + o];
          if (f == 3) r = cpx<T>{-(ky * zt.y - kz * et.y) * wki, -(kz * et.x - ky * zt.x) * wki};
          else if (f == 4) r = cpx<T>{-(kz * xi.y - kx * zt.y) * wki, -(kx * zt.x - kz * xi.x) * wki};
          else r = cpx<T>{-(kx * et.y - ky * xi.y) * wki, -(ky * xi.x - kx * et.x) * wki};
        } else if (NC > 3) {
          // i k_j rho (setFFK, 3D_Boussinesq/src/kernels.h:75-93)
          const cpx<T> rho = s_in[3 * Y * W + o];
          const T kk = (f == 6) ? kx : (f == 7) ? ky : kz;
          r = cpx<T>{-kk * rho.y, kk * rho.x};
        }
      }
      v[e] = r;
    }
    // each group syncs only its own threads (barrier 1 + grp)
    F::run(v, gi, s_tw, s_ex + (grp * W + c) * SX, NamedSync{1 + grp, W * F::G});
    if (live) {
      cpx<T>* o = out + ((((long)f * XT + xt) * N) * Y + iky) * W + c;
#pragma unroll
      for (int e = 0; e < F::E; ++e) o[(long)F::out_index(gi, e) * Y * W] = v[e];
    }
  }
}

// pass A with two fields per thread on packed f32x2 arithmetic (FP32 engine,
// the step's own right-hand side, MODE 0 of pass_a): one group of W x G
// threads takes the output fields in pairs (f, f+1) through one LineFFT2
// transform, so every butterfly and twiddle instruction serves two fields.
// Staging, field values and output layout are pass_a's; the exchange holds
// the pair's values side by side (16-byte words, row stride odd mod 8 so that
// the eight columns of a quarter warp fall on distinct bank groups).
template <int N, int NC, int NF>
__global__ void __launch_bounds__(kTileW * LineFFT<N, 1, float>::G, 3)
pass_a_pk(Geom3<float> g, Fields4<float> in, cpx<float>* __restrict__ out,
          const cpx<float>* __restrict__ tw, int mask_vel, int* status) {
  using T = float;
  using F = LineFFT<N, +1, T>;
  using F2 = LineFFT2<N, +1>;
  constexpr int W = kTileW;
  constexpr int SX = F::SMEM + ((1 - F::SMEM % 8) + 8) % 8;
  constexpr int Y = Box<N>::Y, K = Box<N>::K, XT = Box<N>::XT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_ok;
  cpx<T>* s_in = reinterpret_cast<cpx<T>*>(smem_raw);  // [NC][Y][W]
  cpx<T>* s_tw = s_in + NC * Y * W;                      // [N]
  float4* s_ex = reinterpret_cast<float4*>(s_tw + N);    // [W][SX]
  T* s_wk = reinterpret_cast<T*>(s_ex + W * SX);         // [Y][W]
  const int tid = threadIdx.x, c = tid % W, gi = tid / W;
  const int xt = blockIdx.x, iky = blockIdx.y;
  auto src_comp = [&](int q) -> const cpx<T>* { return in.c[q]; };
  if (!a_stage<T, N, NC>(g, src_comp, tw, s_in, s_tw, s_wk, &s_bar, &s_ok, status)) return;
  const int ikx = xt * W + c;
  const T kx = (T)ikx * g.alpha, ky = (T)(iky - K);
  const bool live = ikx < Box<N>::X;
  // field f at staged mode o (pass_a, MODE 0)
  auto value = [&](int f, int o, T kz, T tk) -> cpx<T> {
    if (f < 3) return s_in[f * Y * W + o];
    if (f < 6) {
      const T wki = (mask_vel && tk < (T)0) ? (T)0 : fabsf(tk);
      const cpx<T> xi = s_in[o], et = s_in[Y * W + o], zt = s_in[2 * Y * W + o];
      if (f == 3) return cpx<T>{-(ky * zt.y - kz * et.y) * wki, -(kz * et.x - ky * zt.x) * wki};
      if (f == 4) return cpx<T>{-(kz * xi.y - kx * zt.y) * wki, -(kx * zt.x - kz * xi.x) * wki};
      return cpx<T>{-(kx * et.y - ky * xi.y) * wki, -(ky * xi.x - kx * et.x) * wki};
    }
    if (NC > 3 && f < 9) {
      const cpx<T> rho = s_in[3 * Y * W + o];
      const T kk = (f == 6) ? kx : (f == 7) ? ky : kz;
      return cpx<T>{-kk * rho.y, kk * rho.x};
    }
    return czero<T>();
  };
#pragma unroll 1
  for (int f0 = 0; f0 < NF; f0 += 2) {
    const bool two = f0 + 1 < NF;
    Pk v[F::E];
#pragma unroll
    for (int e = 0; e < F::E; ++e) {
      const int ikz = row_to_box(F::in_index(gi, e), K, N);
      const int o = ikz * W + c;
      cpx<T> a = czero<T>(), b = czero<T>();
      if (ikz >= 0 && live) {
        const T kz = (T)(ikz - K), tk = s_wk[o];
        a = value(f0, o, kz, tk);
        if (two) b = value(f0 + 1, o, kz, tk);
      }
      v[e] = Pk{make_float2(a.x, b.x), make_float2(a.y, b.y)};
    }
    F2::run(v, gi, s_tw, s_ex + c * SX, BlockSync());
    if (live) {
      cpx<T>* o0 = out + ((((long)f0 * XT + xt) * N) * Y + iky) * W + c;
      cpx<T>* o1 = o0 + (long)XT * N * Y * W;
#pragma unroll
      for (int e = 0; e < F::E; ++e) {
        const long off = (long)F::out_index(gi, e) * Y * W;
        o0[off] = cpx<T>{v[e].re.x, v[e].im.x};
        if (two) o1[off] = cpx<T>{v[e].re.y, v[e].im.y};
      }
    }
  }
}

// ---------------------------------------------------------------------------
// pass B: y-inverse.  grid (XT, N, NF): tile B1[f][xt][z] = [ky][W] -> B2 rows
// ---------------------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(kTileW * LineFFT<N, 1, T>::G)
pass_b(Geom3<T> g, const cpx<T>* __restrict__ in, cpx<T>* __restrict__ out,
       const cpx<T>* __restrict__ tw, int* status) {
  using F = LineFFT<N, +1, T>;
  constexpr int W = kTileW;
  constexpr int SX = ColStride<F::SMEM>::value;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_ok;
  constexpr int Y = Box<N>::Y, K = Box<N>::K, XP = Box<N>::XP, XT = Box<N>::XT;
  // the staged tile, then (every input in registers) the exchange space
  constexpr int AREA = Y * W > W * SX ? Y * W : W * SX;
  cpx<T>* s_in = reinterpret_cast<cpx<T>*>(smem_raw);  // [Y][W]
  cpx<T>* s_tw = s_in + AREA;
  const int tid = threadIdx.x, c = tid % W, gi = tid / W;
  const int xt = blockIdx.x, z = blockIdx.y, f = blockIdx.z;
  pdl_trigger();
  if (tid == 0) mbar_init(&s_bar, 1);
  __syncthreads();
  pdl_wait();
  if (tid == 0) {
    mbar_expect_tx(&s_bar, (uint32_t)(Y * W * sizeof(cpx<T>)));
    bulk_g2s(s_in, in + (((long)f * XT + xt) * N + z) * Y * W, (uint32_t)(Y * W * sizeof(cpx<T>)),
             &s_bar);
  }
  for (int i = tid; i < N; i += blockDim.x) s_tw[i] = tw[i];
  if (!tile_wait(&s_bar, &s_ok, status)) return;
  cpx<T> v[F::E];
#pragma unroll
  for (int e = 0; e < F::E; ++e) {
    const int iky = row_to_box(F::in_index(gi, e), K, N);
    v[e] = iky >= 0 ? s_in[iky * W + c] : czero<T>();
  }
  __syncthreads();
  F::run(v, gi, s_tw, s_in + c * SX, BlockSync());
  cpx<T>* dst = out + (((long)f * N + z) * N) * XP + xt * W + c;
#pragma unroll
  for (int e = 0; e < F::E; ++e) dst[(long)F::out_index(gi, e) * XP] = v[e];
}

// ---------------------------------------------------------------------------
// pass C: x rows.  C2R of the fields (two real signals per complex transform),
// the products -(u x w) (multReal, 3D_NavierStokes/src/kernels.h:281-306) and
// u.grad rho (3D_Boussinesq/src/kernels.h:298-328) in registers, scaled by
// 1/N^3 (normFF1), R2C back keeping kx <= K.  L rows per block (one row per
// group of G lanes), the block's rows of every field fetched by bulk copies.
// out: B3 [g][xt][z][y][W]
// ---------------------------------------------------------------------------
template <typename T, int N>
struct RowOps {
  using FI = LineFFT<N, +1, T>;
  using FO = LineFFT<N, -1, T, true>;  // consumes FI's output distribution
  static constexpr int G = FI::G, E = FI::E;
  static constexpr int SX = RowStride<FI::SMEM, FI::G>::value;

  // row position r of the complex line a + i b whose inverse transform gives the
  // real fields a, b (half spectra A, B in shared memory; B == nullptr: b = 0)
  static __device__ __forceinline__ cpx<T> line_in(const cpx<T>* A, const cpx<T>* B, int r, int K) {
    cpx<T> z = czero<T>();
    if (r == 0) {
      z = cpx<T>{A[0].x, B ? B[0].x : (T)0};
    } else if (r <= K) {
      const cpx<T> a = A[r], b = B ? B[r] : czero<T>();
      z = cpx<T>{a.x - b.y, a.y + b.x};  // a + i b
    } else if (r >= N - K) {
      const cpx<T> a = A[N - r], b = B ? B[N - r] : czero<T>();
      z = cpx<T>{a.x + b.y, -a.y + b.x};  // conj(a) + i conj(b)
    }
    return z;
  }

  // inverse transform of two real fields a, b given by their half spectra (smem rows)
  static __device__ __forceinline__ void c2r_pair(const cpx<T>* A, const cpx<T>* B, int K,
                                                  int gi, const cpx<T>* tw, cpx<T>* ex,
                                                  T (&ra)[E], T (&rb)[E]) {
    cpx<T> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = line_in(A, B, FI::in_index(gi, e), K);
    FI::run(v, gi, tw, ex, WarpSync());
#pragma unroll
    for (int e = 0; e < E; ++e) { ra[e] = v[e].x; rb[e] = v[e].y; }
  }

  // FP32: four real fields as two complex lines (a + i b, c + i d) through one
  // packed f32x2 transform, the instruction count of one scalar line.  PK 1:
  // the exchange crosses the scalar-sized buffer in two halves; PK 2: one
  // pass through a buffer of twice the size.
  template <int PK>
  static __device__ __forceinline__ void c2r_quad(const cpx<T>* A, const cpx<T>* B, const cpx<T>* C,
                                                  const cpx<T>* D, int K, int gi, const cpx<T>* tw,
                                                  cpx<T>* ex, T (&ra)[E], T (&rb)[E], T (&rc)[E],
                                                  T (&rd)[E]) {
    static_assert(sizeof(T) == 4 && PK >= 1 && PK <= 2, "packed transforms are FP32");
    Pk v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int r = FI::in_index(gi, e);
      const cpx<T> z1 = line_in(A, B, r, K), z2 = line_in(C, D, r, K);
      v[e] = Pk{make_float2(z1.x, z2.x), make_float2(z1.y, z2.y)};
    }
    if constexpr (PK == 2) LineFFT2<N, +1>::run(v, gi, tw, reinterpret_cast<float4*>(ex), WarpSync());
    else LineFFT2<N, +1>::run(v, gi, tw, reinterpret_cast<float2*>(ex), WarpSync());
#pragma unroll
    for (int e = 0; e < E; ++e) {
      ra[e] = v[e].re.x; rb[e] = v[e].im.x; rc[e] = v[e].re.y; rd[e] = v[e].im.y;
    }
  }

  // the split of a forward-transformed pair line Z = FFT(p + i q) into P, Q for
  // k < XP (zero beyond K); z: this lane's outputs, ex: N words of exchange
  static __device__ __forceinline__ void split_store(const cpx<T> (&z)[E], int K, int XP, int gi,
                                                     cpx<T>* ex, cpx<T>* __restrict__ P,
                                                     cpx<T>* __restrict__ Q, long tstride) {
#pragma unroll
    for (int e = 0; e < E; ++e) ex[FO::out_index(gi, e)] = z[e];
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = FO::out_index(gi, e);
      if (k < XP) {
        cpx<T> pk = czero<T>(), qk = czero<T>();
        if (k <= K) {
          const cpx<T> a = z[e], b = ex[(N - k) & (N - 1)];
          pk = cpx<T>{a.x + b.x, a.y - b.y};
          qk = cpx<T>{a.y + b.y, b.x - a.x};
        }
        const long o = (long)(k / kTileW) * tstride + (k % kTileW);
        P[o] = pk;
        Q[o] = qk;
      }
    }
    __syncwarp();
  }

  // FP32: forward transforms of (p + i q) and (r + i s) as one packed line pair;
  // p, q (and r, s with s) pre-scaled by 1/2 for the split; s == nullptr: r
  // alone, stored directly into Rr
  template <int PK>
  static __device__ __forceinline__ void r2c_quad(const T (&p)[E], const T (&q)[E], const T (&r)[E],
                                                  const T* s, int K, int XP, int gi,
                                                  const cpx<T>* tw, cpx<T>* ex,
                                                  cpx<T>* __restrict__ P, cpx<T>* __restrict__ Q,
                                                  cpx<T>* __restrict__ Rr, cpx<T>* __restrict__ S,
                                                  long tstride) {
    static_assert(sizeof(T) == 4 && PK >= 1 && PK <= 2, "packed transforms are FP32");
    Pk v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = Pk{make_float2(p[e], r[e]), make_float2(q[e], s ? s[e] : 0.f)};
    using FO2 = LineFFT2<N, -1, true>;
    if constexpr (PK == 2) FO2::run(v, gi, tw, reinterpret_cast<float4*>(ex), WarpSync());
    else FO2::run(v, gi, tw, reinterpret_cast<float2*>(ex), WarpSync());
    cpx<T> z[E];
#pragma unroll
    for (int e = 0; e < E; ++e) z[e] = cpx<T>{v[e].re.x, v[e].im.x};
    split_store(z, K, XP, gi, ex, P, Q, tstride);
#pragma unroll
    for (int e = 0; e < E; ++e) z[e] = cpx<T>{v[e].re.y, v[e].im.y};
    if (s) {
      split_store(z, K, XP, gi, ex, Rr, S, tstride);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = FO::out_index(gi, e);
        if (k < XP) Rr[(long)(k / kTileW) * tstride + (k % kTileW)] = (k <= K) ? z[e] : czero<T>();
      }
    }
  }

  // forward transform of two real signals p, q (q == nullptr: p alone); writes
  // P_k, Q_k for k < XP into the [xt][..][W] layout (zero beyond K).  With q,
  // p and q come pre-scaled by 1/2 (exact), which is the 1/2 of the split.
  static __device__ __forceinline__ void r2c_pair(const T (&p)[E], const T* q, int K, int XP,
                                                  int gi, const cpx<T>* tw, cpx<T>* ex,
                                                  cpx<T>* __restrict__ P, cpx<T>* __restrict__ Q,
                                                  long tstride) {
    cpx<T> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cpx<T>{p[e], q ? q[e] : (T)0};
    FO::run(v, gi, tw, ex, WarpSync());
    if (q) {
#pragma unroll
      for (int e = 0; e < E; ++e) ex[FO::out_index(gi, e)] = v[e];
      __syncwarp();
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = FO::out_index(gi, e);
        if (k < XP) {
          cpx<T> pk = czero<T>(), qk = czero<T>();
          if (k <= K) {
            const cpx<T> a = v[e], b = ex[(N - k) & (N - 1)];
            // P = (Z_k + conj Z_{N-k}) / 2,  Q = -i (Z_k - conj Z_{N-k}) / 2
            pk = cpx<T>{a.x + b.x, a.y - b.y};
            qk = cpx<T>{a.y + b.y, b.x - a.x};
          }
          const long o = (long)(k / kTileW) * tstride + (k % kTileW);
          P[o] = pk;
          Q[o] = qk;
        }
      }
      __syncwarp();
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = FO::out_index(gi, e);
        if (k < XP) P[(long)(k / kTileW) * tstride + (k % kTileW)] = (k <= K) ? v[e] : czero<T>();
      }
    }
  }
};

// Template knobs picked by the engine's autotuner: L rows per block (one group
// of G lanes per row, so L*G threads) and ST buffers per warp.  Every warp
// runs its own pipeline over "warp tiles" of 32/G rows (RPW): its lane 0
// fetches the tile's rows of every field by bulk copies into the warp's own
// buffer and all lanes wait on the warp's mbarrier, so no warp ever waits for
// another.  ST = 1: the next tile's copy is issued as soon as the last C2R has
// gathered its inputs, overlapping the forward transforms and stores; ST = 2:
// it is issued at the top of the iteration into the other buffer.
// The nine-field (Boussinesq) FP32 build at 128 threads asks for three blocks
// per SM, which caps it at 168 registers (it spills 8 bytes instead of holding
// 255); every other build, FP64 included (one block per SM by its shared
// memory), leaves the block count to the compiler (0).  Passes A and E in
// FP64 at 256^3 likewise ask for one block per SM: their shared memory allows
// no more, and the register cap of three would only make them spill.
// PK (FP32 only): 0 one scalar transform per complex line; 1 or 2 two lines per
// packed f32x2 transform (RowOps::c2r_quad / r2c_quad), with the exchange in
// two halves through the scalar-sized buffer (1) or in one pass through a
// buffer twice that size (2).
template <typename T, int N, int NF, int L, int ST, int PK = 0>
__global__ void __launch_bounds__(L * LineFFT<N, 1, T>::G,
                                  (sizeof(T) == 4 && NF == 9 && L * LineFFT<N, 1, T>::G <= 128) ? 3 : 0)
pass_c(Geom3<T> g, const cpx<T>* __restrict__ in, cpx<T>* __restrict__ out,
       const cpx<T>* __restrict__ tw, T scale, T* __restrict__ dump, int* status, int nwt,
       unsigned long long* __restrict__ umax, int dnf) {
  static_assert(PK == 0 || (sizeof(T) == 4 && NF != 7), "packed x-pass: FP32 forward fields");
  using R = RowOps<T, N>;
  constexpr int G = R::G, E = R::E;
  constexpr int RPW = 32 / G, WPB = L / RPW;  // rows per warp tile, warps per block
  static_assert(L % RPW == 0, "whole warps per block");
  constexpr bool BOUS = (NF == 9);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar[WPB][2];
  constexpr int K = Box<N>::K, XP = Box<N>::XP, XT = Box<N>::XT;
  constexpr int wtile_words = NF * RPW * XP;
  cpx<T>* s_buf = reinterpret_cast<cpx<T>*>(smem_raw);  // [WPB][ST][NF][RPW][XP]
  cpx<T>* s_tw = s_buf + WPB * ST * wtile_words;         // [2N]: plain | swapped plan
  cpx<T>* s_ex = s_tw + 2 * N;                           // [L][SX]
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int j = lane / G, gi = lane % G;
  cpx<T>* s_w = s_buf + warp * ST * wtile_words;  // this warp's buffers
  uint64_t* bar = s_bar[warp];
  const long plane = (long)N * N * XP;
  const uint32_t bytes = (uint32_t)(RPW * XP * sizeof(cpx<T>));
  if (lane == 0) { mbar_init(&bar[0], 1); mbar_init(&bar[1], 1); }
  for (int i = tid; i < 2 * N; i += blockDim.x) s_tw[i] = tw[i];
  __syncthreads();
  pdl_wait();
  // warp tile t = rows [t*RPW, t*RPW + RPW) of every field, one bulk copy per
  // field; the buffer's earlier contents were read by this warp's lanes before
  // the __syncwarp that precedes every call
  auto issue = [&](int t, int b) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[b], NF * bytes);
    for (int f = 0; f < NF; ++f)
      bulk_g2s(s_w + b * wtile_words + f * RPW * XP, in + f * plane + (long)t * RPW * XP, bytes,
               &bar[b]);
  };
  const int wstride = gridDim.x * WPB;
  int t = blockIdx.x * WPB + warp;
  if (lane == 0 && t < nwt) issue(t, 0);
  const long tstride = (long)N * N * kTileW;  // B3: successive xt tiles
  const long fstride = (long)XT * tstride;
  cpx<T>* ex = s_ex + (warp * RPW + j) * R::SX * (PK == 2 ? 2 : 1);
  for (int i = 0; t < nwt; ++i, t += wstride) {
    const int b = (ST == 2) ? (i & 1) : 0;
    const uint32_t parity = (ST == 2) ? ((i >> 1) & 1) : (i & 1);
    const int tn = t + wstride;
    // two buffers: buffer b^1 was released by the __syncwarp ending iteration i-1
    if (ST == 2 && lane == 0 && tn < nwt) issue(tn, b ^ 1);
    const bool ok = mbar_wait_bounded(&bar[b], parity, status);
    if (!__all_sync(0xffffffffu, ok)) {
      if (ST == 2 && lane == 0 && tn < nwt) mbar_wait_bounded(&bar[b ^ 1], ((i + 1) >> 1) & 1, nullptr);
      return;
    }
    // one buffer: free once the last C2R has gathered its rows
    auto release = [&]() {
      if (ST == 1) {
        __syncwarp();
        if (lane == 0 && tn < nwt) issue(tn, 0);
      }
    };
    const long row = (long)t * RPW + j;
    const int z = (int)(row / N), y = (int)(row % N);
    const cpx<T>* src = s_w + b * wtile_words + j * XP;
    constexpr int fs = RPW * XP;  // field stride in shared memory
    cpx<T>* dst = out + ((long)z * N + y) * kTileW;
    const cpx<T>* two = s_tw + N;  // swapped plan for the forward transforms
    const T hscale = (T)0.5 * scale;  // products of a paired forward transform
    if (NF == 7) {
      // scalar products of the Boussinesq adjoint: psi * (i k rho), psi * u
      T ps[E], ga[E], gb[E], p0[E], p1[E], p2[E];
      R::c2r_pair(src, src + fs, K, gi, s_tw, ex, ps, ga);
#pragma unroll
      for (int e = 0; e < E; ++e) p0[e] = ps[e] * ga[e] * hscale;
      R::c2r_pair(src + 2 * fs, src + 3 * fs, K, gi, s_tw, ex, ga, gb);
#pragma unroll
      for (int e = 0; e < E; ++e) { p1[e] = ps[e] * ga[e] * hscale; p2[e] = ps[e] * gb[e] * hscale; }
      R::r2c_pair(p0, p1, K, XP, gi, two, ex, dst, dst + fstride, tstride);
      R::c2r_pair(src + 4 * fs, src + 5 * fs, K, gi, s_tw, ex, ga, gb);
#pragma unroll
      for (int e = 0; e < E; ++e) { p0[e] = ps[e] * ga[e] * hscale; p1[e] = ps[e] * gb[e] * hscale; }
      R::r2c_pair(p2, p0, K, XP, gi, two, ex, dst + 2 * fstride, dst + 3 * fstride, tstride);
      R::c2r_pair(src + 6 * fs, nullptr, K, gi, s_tw, ex, ga, gb);
      release();
#pragma unroll
      for (int e = 0; e < E; ++e) p2[e] = ps[e] * ga[e] * hscale;
      R::r2c_pair(p1, p2, K, XP, gi, two, ex, dst + 4 * fstride, dst + 5 * fstride, tstride);
      __syncwarp();
      continue;
    }
    T xi[E], et[E], zt[E], u[E], v[E], w[E];
    if constexpr (PK != 0) {
      // packed: (u + i rho_x, v + i rho_y) -> (w + i rho_z, xi + i eta) -> zeta
      // alone for the Boussinesq fields (u.grad rho first, so that at most six
      // physical fields are live); (xi + i eta, zeta + i u) -> (v + i w) else
      if constexpr (BOUS) {
        T rx[E], ry[E], n4[E];
        R::template c2r_quad<PK>(src + 3 * fs, src + 6 * fs, src + 4 * fs, src + 7 * fs, K, gi,
                                 s_tw, ex, u, rx, v, ry);
#pragma unroll
        for (int e = 0; e < E; ++e) n4[e] = u[e] * rx[e] + v[e] * ry[e];
        R::template c2r_quad<PK>(src + 5 * fs, src + 8 * fs, src, src + fs, K, gi, s_tw, ex, w, rx,
                                 xi, et);
#pragma unroll
        for (int e = 0; e < E; ++e) n4[e] = (n4[e] + w[e] * rx[e]) * hscale;
        R::c2r_pair(src + 2 * fs, nullptr, K, gi, s_tw, ex, zt, ry);
        release();
        if (umax) {
          double m = 0.0;
#pragma unroll
          for (int e = 0; e < E; ++e) m = fmax(m, fabs((double)u[e]));
          for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
          if (lane == 0) atomicMax(umax, (unsigned long long)__double_as_longlong(m));
        }
        if (dump) {
          const long base = row * N;
          const long nr = (long)N * N * N;
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const int x = R::FI::out_index(gi, e);
            dump[base + x] = xi[e];
            dump[nr + base + x] = et[e];
            dump[2 * nr + base + x] = zt[e];
            if (dnf == 6) {
              dump[3 * nr + base + x] = u[e];
              dump[4 * nr + base + x] = v[e];
              dump[5 * nr + base + x] = w[e];
            }
          }
        }
        T n1[E], n2[E], n3[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          n1[e] = -(v[e] * zt[e] - w[e] * et[e]) * hscale;
          n2[e] = -(w[e] * xi[e] - u[e] * zt[e]) * hscale;
          n3[e] = -(u[e] * et[e] - v[e] * xi[e]) * hscale;
        }
        R::template r2c_quad<PK>(n1, n2, n3, n4, K, XP, gi, two, ex, dst, dst + fstride,
                                 dst + 2 * fstride, dst + 3 * fstride, tstride);
        __syncwarp();
        continue;
      }
      R::template c2r_quad<PK>(src, src + fs, src + 2 * fs, src + 3 * fs, K, gi, s_tw, ex, xi, et,
                               zt, u);
    } else {
      R::c2r_pair(src, src + fs, K, gi, s_tw, ex, xi, et);
      R::c2r_pair(src + 2 * fs, src + 3 * fs, K, gi, s_tw, ex, zt, u);
    }
    R::c2r_pair(src + 4 * fs, src + 5 * fs, K, gi, s_tw, ex, v, w);
    if (!BOUS) release();
    if (umax) {
      // max |u| of the physical x-velocity (the Boussinesq DNS's CFL input,
      // 3D_Boussinesq/src/out_low.h:14): non-negative doubles order as their bits
      double m = 0.0;
#pragma unroll
      for (int e = 0; e < E; ++e) m = fmax(m, fabs((double)u[e]));
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) atomicMax(umax, (unsigned long long)__double_as_longlong(m));
    }
    if (dump) {
      const long base = row * N;
      const long nr = (long)N * N * N;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = R::FI::out_index(gi, e);
        dump[base + x] = xi[e];
        dump[nr + base + x] = et[e];
        dump[2 * nr + base + x] = zt[e];
        if (dnf == 6) {  // the velocity too (the DNS's mean-square statistics)
          dump[3 * nr + base + x] = u[e];
          dump[4 * nr + base + x] = v[e];
          dump[5 * nr + base + x] = w[e];
        }
      }
    }
    T n1[E], n2[E], n3[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      // U,V,W <- -(u x w)  (multReal)
      n1[e] = -(v[e] * zt[e] - w[e] * et[e]) * hscale;
      n2[e] = -(w[e] * xi[e] - u[e] * zt[e]) * hscale;
      n3[e] = -(u[e] * et[e] - v[e] * xi[e]) * (BOUS ? hscale : scale);
    }
    if constexpr (PK != 0 && !BOUS) {
      R::template r2c_quad<PK>(n1, n2, n3, nullptr, K, XP, gi, two, ex, dst, dst + fstride,
                               dst + 2 * fstride, nullptr, tstride);
    } else if (!BOUS) {
      R::r2c_pair(n1, n2, K, XP, gi, two, ex, dst, dst + fstride, tstride);
      R::r2c_pair(n3, nullptr, K, XP, gi, two, ex, dst + 2 * fstride, nullptr, tstride);
    } else {
      T rx[E], ry[E], n4[E];
      R::c2r_pair(src + 6 * fs, src + 7 * fs, K, gi, s_tw, ex, rx, ry);
#pragma unroll
      for (int e = 0; e < E; ++e) n4[e] = u[e] * rx[e] + v[e] * ry[e];
      R::c2r_pair(src + 8 * fs, nullptr, K, gi, s_tw, ex, rx, ry);
      release();
#pragma unroll
      for (int e = 0; e < E; ++e) n4[e] = (n4[e] + w[e] * rx[e]) * hscale;
      R::r2c_pair(n1, n2, K, XP, gi, two, ex, dst, dst + fstride, tstride);
      R::r2c_pair(n3, n4, K, XP, gi, two, ex, dst + 2 * fstride, dst + 3 * fstride, tstride);
    }
    __syncwarp();
  }
  // The x-pass runs as one wave of resident blocks: a trigger at entry would
  // let the next pass's blocks take the room left on these SMs and wait there
  // for the whole pass.  Each block triggers when its rows are done.
  pdl_trigger();
}

// ---------------------------------------------------------------------------
// pass D: y-forward.  grid (XT, N, NO): tile B3[f][xt][z] = [y][W] -> B4
// ---------------------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(kTileW * LineFFT<N, 1, T>::G)
pass_d(Geom3<T> g, const cpx<T>* __restrict__ in, cpx<T>* __restrict__ out,
       const cpx<T>* __restrict__ tw, int* status) {
  using F = LineFFT<N, -1, T>;
  constexpr int W = kTileW;
  constexpr int SX = ColStride<F::SMEM>::value;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_ok;
  constexpr int Y = Box<N>::Y, K = Box<N>::K, XT = Box<N>::XT;
  // the staged tile, then (every input in registers) the exchange space
  constexpr int AREA = N * W > W * SX ? N * W : W * SX;
  cpx<T>* s_in = reinterpret_cast<cpx<T>*>(smem_raw);  // [N][W]
  cpx<T>* s_tw = s_in + AREA;
  const int tid = threadIdx.x, c = tid % W, gi = tid / W;
  const int xt = blockIdx.x, z = blockIdx.y, f = blockIdx.z;
  pdl_trigger();
  if (tid == 0) mbar_init(&s_bar, 1);
  __syncthreads();
  pdl_wait();
  if (tid == 0) {
    mbar_expect_tx(&s_bar, (uint32_t)(N * W * sizeof(cpx<T>)));
    bulk_g2s(s_in, in + (((long)f * XT + xt) * N + z) * N * W, (uint32_t)(N * W * sizeof(cpx<T>)),
             &s_bar);
  }
  for (int i = tid; i < N; i += blockDim.x) s_tw[i] = tw[i];
  if (!tile_wait(&s_bar, &s_ok, status)) return;
  cpx<T> v[F::E];
#pragma unroll
  for (int e = 0; e < F::E; ++e) v[e] = s_in[F::in_index(gi, e) * W + c];
  __syncthreads();
  F::run(v, gi, s_tw, s_in + c * SX, BlockSync());
  // B4[f][xt][ky][z][W]
  cpx<T>* dst = out + (((long)f * XT + xt) * Y * N + z) * W + c;
#pragma unroll
  for (int e = 0; e < F::E; ++e) {
    const int iky = row_to_box(F::out_index(gi, e), K, N);
    if (iky >= 0) dst[(long)iky * N * W] = v[e];
  }
}

// ---------------------------------------------------------------------------
// pass E: z-forward of the NO fields of one (xt, ky) tile, then the spectral
// finish and the scheme update for every mode of the tile.
// ---------------------------------------------------------------------------
template <typename T>
struct Regs {
  Fields4<T> S, X0, K1, K2, K3;
  // FP32 engine: the rounding error of every state update, carried to the
  // next one (state = S + SC), so that increments far below one ulp of the
  // state still add up over a long run; null pointers in FP64
  Fields4<T> SC;
};

// s + y as a rounded sum and its exact error (Knuth's TwoSum)
template <typename T>
__device__ __forceinline__ void two_sum(T a, T b, T& s, T& err) {
  s = a + b;
  const T bp = s - a;
  err = (a - (s - bp)) + (b - bp);
}

// state value s (+ carried error c) plus the small increment y: returns the
// new state and stores the new carried error; plain s + y without SC, and for
// a mode the update does not keep (its carried error is cleared)
template <typename T>
__device__ __forceinline__ cpx<T> comp_add(const Fields4<T>& SC, int q, long ik, cpx<T> s, cpx<T> y,
                                           bool keep = true) {
  if (!SC.c[q]) return cpx<T>{s.x + y.x, s.y + y.y};
  if (!keep) {
    SC.c[q][ik] = czero<T>();
    return cpx<T>{s.x + y.x, s.y + y.y};
  }
  const cpx<T> c = SC.c[q][ik];
  cpx<T> r, e;
  two_sum(s.x, y.x + c.x, r.x, e.x);
  two_sum(s.y, y.y + c.y, r.y, e.y);
  SC.c[q][ik] = e;
  return r;
}

// v (1 - e) evaluated as v - e v
template <typename T>
__device__ __forceinline__ cpx<T> damp(cpx<T> v, T e) {
  return cpx<T>{v.x - e * v.x, v.y - e * v.y};
}

template <typename T, int SCHEME>
__device__ __forceinline__ void scheme_point(const Geom3<T>& g, const Regs<T>& R,
                                             const StepParams<T>& p, int stage, long ik, int ikx,
                                             int iy, int iz, T xiX, T xiY, T etX, T etY, T ztX,
                                             T ztY, cpx<T> RKv) {
  const T kx = (T)ikx * g.alpha, ky = (T)iy, kz = (T)iz;
  const T wk = kx * kx + ky * ky + kz * kz;
  const T wki = wkinv(wk);
  const T LL = keep_mode<T>(ikx, iy, iz, g.K, g.alpha) ? (T)1 : (T)0;
  if (SCHEME == SCHEME_NS_HEUN || SCHEME == SCHEME_EULER_HEUN) {
    cpx<T>* S0 = R.S.c[0]; cpx<T>* S1 = R.S.c[1]; cpx<T>* S2 = R.S.c[2];
    cpx<T>* H0 = R.K1.c[0]; cpx<T>* H1 = R.K1.c[1]; cpx<T>* H2 = R.K1.c[2];
    const cpx<T> s0 = S0[ik], s1 = S1[ik], s2 = S2[ik];
    if (SCHEME == SCHEME_NS_HEUN) {
      if (p.fform == 0) {  // 3D_NavierStokes/src/kernels.h:342-343, 419-420
        if (kx == (T)0 && kz == p.kf && ky == p.kf) xiX += p.ampfor;
        if (kx == (T)0 && kz == -p.kf && ky == p.kf) xiX -= p.ampfor;
      } else if (kx == (T)0 && ky == p.kf) {  // 3D_NavierStokes/src_gmres/kernels.h:234-238, 320-324
        if (kz == p.kf) { etY += p.ampfor; ztY -= p.ampfor; }
        if (kz == -p.kf) { etY += p.ampfor; ztY += p.ampfor; }
      }
      // nuzn = (1 - nu k^2 dt/2)/dt, nu1 = dt/(1 + nu k^2 dt/2) (3D_NavierStokes/src/init.F90:194-198)
      const T NU = p.nu * wk;
      const T nuzn = LL * (((T)1 - (T)0.5 * NU * p.dt) / p.dt);
      const T nu1 = LL * (p.dt / ((T)1 + (T)0.5 * NU * p.dt));
      if (stage == STAGE_HEUN_PRED) {
        H0[ik] = cpx<T>{xiX, xiY}; H1[ik] = cpx<T>{etX, etY}; H2[ik] = cpx<T>{ztX, ztY};
        // nu1 (nuzn s + N) = (s - e s) + nu1 N with nu1 nuzn = 1 - e,
        // e = NU dt / (1 + NU dt / 2): only the small e is rounded
        (void)nuzn;
        const T x = NU * p.dt;
        const T e = x / ((T)1 + (T)0.5 * x);
        const T NU1 = LL * nu1;
        const T eL = LL * e;
        const bool kp = LL != (T)0;
        S0[ik] = comp_add(R.SC, 0, ik, cpx<T>{LL * s0.x, LL * s0.y},
                          cpx<T>{NU1 * xiX - eL * s0.x, NU1 * xiY - eL * s0.y}, kp);
        S1[ik] = comp_add(R.SC, 1, ik, cpx<T>{LL * s1.x, LL * s1.y},
                          cpx<T>{NU1 * etX - eL * s1.x, NU1 * etY - eL * s1.y}, kp);
        S2[ik] = comp_add(R.SC, 2, ik, cpx<T>{LL * s2.x, LL * s2.y},
                          cpx<T>{NU1 * ztX - eL * s2.x, NU1 * ztY - eL * s2.y}, kp);
      } else {
        const T NU2 = LL * (T)0.5 * nu1;
        const cpx<T> h0 = H0[ik], h1 = H1[ik], h2 = H2[ik];
        const bool kp = LL != (T)0;
        S0[ik] = comp_add(R.SC, 0, ik, cpx<T>{LL * s0.x, LL * s0.y},
                          cpx<T>{NU2 * (xiX - h0.x), NU2 * (xiY - h0.y)}, kp);
        S1[ik] = comp_add(R.SC, 1, ik, cpx<T>{LL * s1.x, LL * s1.y},
                          cpx<T>{NU2 * (etX - h1.x), NU2 * (etY - h1.y)}, kp);
        S2[ik] = comp_add(R.SC, 2, ik, cpx<T>{LL * s2.x, LL * s2.y},
                          cpx<T>{NU2 * (ztX - h2.x), NU2 * (ztY - h2.y)}, kp);
      }
    } else {  // Euler (3D_Euler/src/kernels.h:324-341, 396-406)
      if (stage == STAGE_HEUN_PRED) {
        H0[ik] = cpx<T>{LL * xiX, LL * xiY}; H1[ik] = cpx<T>{LL * etX, LL * etY};
        H2[ik] = cpx<T>{LL * ztX, LL * ztY};
        S0[ik] = comp_add(R.SC, 0, ik, s0, cpx<T>{p.dt * xiX, p.dt * xiY});
        S1[ik] = comp_add(R.SC, 1, ik, s1, cpx<T>{p.dt * etX, p.dt * etY});
        S2[ik] = comp_add(R.SC, 2, ik, s2, cpx<T>{p.dt * ztX, p.dt * ztY});
      } else {
        const T hd = LL * (T)0.5 * p.dt;
        const cpx<T> h0 = H0[ik], h1 = H1[ik], h2 = H2[ik];
        const bool kp = LL != (T)0;
        S0[ik] = comp_add(R.SC, 0, ik, cpx<T>{LL * s0.x, LL * s0.y},
                          cpx<T>{hd * (xiX - h0.x), hd * (xiY - h0.y)}, kp);
        S1[ik] = comp_add(R.SC, 1, ik, cpx<T>{LL * s1.x, LL * s1.y},
                          cpx<T>{hd * (etX - h1.x), hd * (etY - h1.y)}, kp);
        S2[ik] = comp_add(R.SC, 2, ik, cpx<T>{LL * s2.x, LL * s2.y},
                          cpx<T>{hd * (ztX - h2.x), hd * (ztY - h2.y)}, kp);
      }
    }
  } else {
    // RK4 with per-stage CN factors (3D_Boussinesq/src/kernels.h:331-621)
    constexpr bool BOUS = (SCHEME == SCHEME_BOUS_RK4);
    T rXR = 0, rXC = 0;  // density right-hand side
    const bool final_stage = (stage == STAGE_RK4);
    const T LC = final_stage ? (T)1 : LL;
    const cpx<T> x0 = R.X0.c[0][ik], e0 = R.X0.c[1][ik], z0 = R.X0.c[2][ik];
    if (BOUS) {
      const cpx<T> r0 = R.X0.c[3][ik];
      const cpx<T> RK = RKv;
      const T gXR = -kx * r0.y, gXC = kx * r0.x, gYR = -ky * r0.y, gYC = ky * r0.x;
      const T gZR = -kz * r0.y, gZC = kz * r0.x;
      xiX = LC * (xiX - p.ri * (gYR * p.sinth - gZR * p.costh));
      xiY = LC * (xiY - p.ri * (gYC * p.sinth - gZC * p.costh));
      etX = LC * (etX + p.ri * gXR * p.sinth);
      etY = LC * (etY + p.ri * gXC * p.sinth);
      ztX = LC * (ztX - p.ri * gXR * p.costh);
      ztY = LC * (ztY - p.ri * gXC * p.costh);
      rXR = -LC * (RK.x + (kz * x0.y - kx * z0.y) * wki * p.costh +
                   (kx * e0.y - ky * x0.y) * wki * p.sinth);
      rXC = -LC * (RK.y + (kx * z0.x - kz * x0.x) * wki * p.costh +
                   (ky * x0.x - kx * e0.x) * wki * p.sinth);
    } else {
      xiX *= LC; xiY *= LC; etX *= LC; etY *= LC; ztX *= LC; ztY *= LC;
    }
    if (kx == (T)0 && kz == (T)0 && ky == p.kf) ztX += p.ampfor;
    const T dt = p.dt;
    const T nk = dt * p.nu * wk;
    const T nks = BOUS ? nk / p.sc : (T)0;
    if (stage == STAGE_DERIV) {  // RHS kernel: dz/dt = -nu k^2 z + N
      const cpx<T> s0 = R.S.c[0][ik], s1 = R.S.c[1][ik], s2 = R.S.c[2][ik];
      const T d1 = -p.nu * wk;
      R.K1.c[0][ik] = cpx<T>{d1 * s0.x + xiX, d1 * s0.y + xiY};
      R.K1.c[1][ik] = cpx<T>{d1 * s1.x + etX, d1 * s1.y + etY};
      R.K1.c[2][ik] = cpx<T>{d1 * s2.x + ztX, d1 * s2.y + ztY};
      if (BOUS) {
        const cpx<T> s3 = R.S.c[3][ik];
        const T d2 = -p.nu * wk / p.sc;
        R.K1.c[3][ik] = cpx<T>{d2 * s3.x + rXR, d2 * s3.y + rXC};
      }
    } else if (!final_stage) {
      // X0 = d (S + fr dt N) with d = (1 - q nk)/(1 + q nk), applied as
      // v - e v, e = 2 q nk / (1 + q nk): the factor is the same every step,
      // so its rounding would compound coherently over a run; written this
      // way only e (small) is rounded
      const T q = (stage == STAGE_RK3) ? (T)0.5 : (T)0.25;
      const T fr = (stage == STAGE_RK3) ? (T)1 : (T)0.5;
      const T e1 = (T)2 * q * nk / ((T)1 + q * nk);
      const Fields4<T>& KR = (stage == STAGE_RK1) ? R.K1 : (stage == STAGE_RK2) ? R.K2 : R.K3;
      KR.c[0][ik] = cpx<T>{dt * xiX, dt * xiY};
      KR.c[1][ik] = cpx<T>{dt * etX, dt * etY};
      KR.c[2][ik] = cpx<T>{dt * ztX, dt * ztY};
      const cpx<T> s0 = R.S.c[0][ik], s1 = R.S.c[1][ik], s2 = R.S.c[2][ik];
      R.X0.c[0][ik] = damp(cpx<T>{s0.x + fr * dt * xiX, s0.y + fr * dt * xiY}, e1);
      R.X0.c[1][ik] = damp(cpx<T>{s1.x + fr * dt * etX, s1.y + fr * dt * etY}, e1);
      R.X0.c[2][ik] = damp(cpx<T>{s2.x + fr * dt * ztX, s2.y + fr * dt * ztY}, e1);
      if (BOUS) {
        const T e2 = (T)2 * q * nks / ((T)1 + q * nks);
        KR.c[3][ik] = cpx<T>{dt * rXR, dt * rXC};
        const cpx<T> s3 = R.S.c[3][ik];
        R.X0.c[3][ik] = damp(cpx<T>{s3.x + fr * dt * rXR, s3.y + fr * dt * rXC}, e2);
      }
    } else {
      // S' = ((1 - nk/2) S + incr) / (1 + nk/2) = (S - eS S) + (incr - eI incr)
      // with eS = nk / (1 + nk/2), eI = (nk/2) / (1 + nk/2)
      const T sixth = (T)(1.0 / 6.0), third = (T)(1.0 / 3.0);
      const T hn = (T)0.5 * nk;
      const T eS = nk / ((T)1 + hn), eI = hn / ((T)1 + hn);
      T o[4][2];
      const T nr[3][2] = {{xiX, xiY}, {etX, etY}, {ztX, ztY}};
      const bool kp = LL != (T)0;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const cpx<T> s = R.S.c[q][ik], a = R.K1.c[q][ik], b = R.K2.c[q][ik], cc3 = R.K3.c[q][ik];
        const T ix = sixth * (a.x + dt * nr[q][0]) + third * (b.x + cc3.x);
        const T iy = sixth * (a.y + dt * nr[q][1]) + third * (b.y + cc3.y);
        const cpx<T> r = comp_add(R.SC, q, ik, cpx<T>{LL * s.x, LL * s.y},
                                  cpx<T>{LL * ((ix - eI * ix) - eS * s.x),
                                         LL * ((iy - eI * iy) - eS * s.y)}, kp);
        o[q][0] = r.x;
        o[q][1] = r.y;
      }
      if (BOUS) {
        const T hs = (T)0.5 * nks;
        const T eS2 = nks / ((T)1 + hs), eI2 = hs / ((T)1 + hs);
        const cpx<T> s = R.S.c[3][ik], a = R.K1.c[3][ik], b = R.K2.c[3][ik], cc3 = R.K3.c[3][ik];
        const T ix = sixth * (a.x + dt * rXR) + third * (b.x + cc3.x);
        const T iy = sixth * (a.y + dt * rXC) + third * (b.y + cc3.y);
        const cpx<T> r = comp_add(R.SC, 3, ik, cpx<T>{LL * s.x, LL * s.y},
                                  cpx<T>{LL * ((ix - eI2 * ix) - eS2 * s.x),
                                         LL * ((iy - eI2 * iy) - eS2 * s.y)}, kp);
        o[3][0] = r.x;
        o[3][1] = r.y;
        R.X0.c[3][ik] = cpx<T>{o[3][0], o[3][1]};
        R.S.c[3][ik] = cpx<T>{o[3][0], o[3][1]};
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) R.X0.c[q][ik] = cpx<T>{o[q][0], o[q][1]};
      // remove the divergence of the vorticity (3D_Boussinesq/src/kernels.h:597-606)
      const T phiR = (kx * o[0][1] + ky * o[1][1] + kz * o[2][1]) * wki;
      const T phiC = -(kx * o[0][0] + ky * o[1][0] + kz * o[2][0]) * wki;
      R.S.c[0][ik] = cpx<T>{o[0][0] - (-kx * phiC), o[0][1] - kx * phiR};
      R.S.c[1][ik] = cpx<T>{o[1][0] - (-ky * phiC), o[1][1] - ky * phiR};
      R.S.c[2][ik] = cpx<T>{o[2][0] - (-kz * phiC), o[2][1] - kz * phiR};
    }
  }

}

// barrier of the first `count` threads of the block only (hardware barrier 1)
struct GroupSync {
  int count;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync 1, %0;" ::"r"(count) : "memory");
  }
};

// Pass E runs 2 W G threads: for three fields both halves transform the tile,
// for more the first half alone (named barriers of their own), then all of
// them do the update, whose state loads are what the pass waits on.
template <typename T, int N, int NO, int SCHEME>
__global__ void __launch_bounds__(2 * kTileW * LineFFT<N, 1, T>::G, sizeof(T) > 4 ? (N >= 256 ? 1 : 2) : 3)
pass_e(Geom3<T> g, const cpx<T>* __restrict__ in, const cpx<T>* __restrict__ tw, Regs<T> R,
       StepParams<T> p, int stage, int* status) {
  using F = LineFFT<N, -1, T>;
  constexpr int W = kTileW;
  constexpr int SX = ColStride<F::SMEM>::value;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_ok;
  constexpr int Y = Box<N>::Y, K = Box<N>::K, XT = Box<N>::XT;
  // Fields are transformed last to first.  Field f's kept rows go to the last
  // Y rows of its own input tile.  With ALIAS its exchange space is the start
  // of that tile (its inputs are in registers by then), running on into the
  // first rows of field f+1 (dead: already transformed, outputs further on)
  // or, for the last field, into a pad after the tiles.
  constexpr int EXW = W * SX, OVER = EXW > N * W ? EXW - N * W : 0;
  constexpr bool ALIAS = OVER <= (N - Y) * W;
  constexpr int R0 = N - Y;  // first output row
  cpx<T>* s_in = reinterpret_cast<cpx<T>*>(smem_raw);  // [NO][N][W] (+ pad)
  cpx<T>* s_tw = s_in + NO * N * W + (ALIAS ? OVER : 0);
  constexpr int TG = (NO == 3) ? 2 : 1;                // transform groups
  cpx<T>* s_ex = s_tw + N;  // without ALIAS: the first group's; then the second's
  const int tid = threadIdx.x, nth = blockDim.x, c = tid % W;
  const int xt = blockIdx.x, iky = blockIdx.y;
  pdl_trigger();
  if (tid == 0) mbar_init(&s_bar, 1);
  __syncthreads();
  const long tile = ((long)xt * Y + iky) * Y * W;
  pdl_wait();
  if (tid == 0) {
    const uint32_t bytes = (uint32_t)(N * W * sizeof(cpx<T>));
    mbar_expect_tx(&s_bar, NO * bytes);
    for (int f = 0; f < NO; ++f)
      bulk_g2s(s_in + f * N * W, in + (((long)f * XT + xt) * Y + iky) * N * W, bytes, &s_bar);
    // the state tiles the update will read: fetch them into L2 while the
    // transforms run
    const uint32_t sb = (uint32_t)(Y * W * sizeof(cpx<T>));
    const int nc = (NO > 3) ? 4 : 3;
    for (int q = 0; q < nc; ++q) {
      if (R.S.c[q]) bulk_prefetch_l2(R.S.c[q] + tile, sb);
      const bool heun = (SCHEME == SCHEME_NS_HEUN || SCHEME == SCHEME_EULER_HEUN);
      if (heun && stage == STAGE_HEUN_CORR && R.K1.c[q]) bulk_prefetch_l2(R.K1.c[q] + tile, sb);
      if (SCHEME == SCHEME_BOUS_RK4 && R.X0.c[q]) bulk_prefetch_l2(R.X0.c[q] + tile, sb);
      if (R.SC.c[q] && (heun || stage == STAGE_RK4)) bulk_prefetch_l2(R.SC.c[q] + tile, sb);
      if (!heun && stage == STAGE_RK4) {
        if (R.K1.c[q]) bulk_prefetch_l2(R.K1.c[q] + tile, sb);
        if (R.K2.c[q]) bulk_prefetch_l2(R.K2.c[q] + tile, sb);
        if (R.K3.c[q]) bulk_prefetch_l2(R.K3.c[q] + tile, sb);
      }
    }
  }
  for (int i = tid; i < N; i += nth) s_tw[i] = tw[i];
  if (!tile_wait(&s_bar, &s_ok, status)) return;
  // three fields: both halves transform (fields 2 and 1, then 0), the second
  // half in an exchange area of its own; more fields: the first half alone
  const int tg = tid / (W * F::G), tl = (tid % (W * F::G)) / W;  // group, lane group in it
  if (tg < TG) {
#pragma unroll 1
    for (int r = 0; r < (NO + TG - 1) / TG; ++r) {
      const int f = NO - 1 - r * TG - tg;
      if (f >= 0) {
        cpx<T> v[F::E];
#pragma unroll
        for (int e = 0; e < F::E; ++e) v[e] = s_in[(f * N + F::in_index(tl, e)) * W + c];
        const NamedSync gs{1 + tg, W * F::G};
        cpx<T>* exb = (tg == 0) ? (ALIAS ? s_in + f * N * W : s_ex) : s_ex + (ALIAS ? 0 : W * SX);
        if (ALIAS && tg == 0) gs();  // every input read before the exchange reuses them
        F::run(v, tl, s_tw, exb + c * SX, gs);
#pragma unroll
        for (int e = 0; e < F::E; ++e) {
          const int ikz = row_to_box(F::out_index(tl, e), K, N);
          if (ikz >= 0) s_in[(f * N + R0 + ikz) * W + c] = v[e];
        }
      }
      // a round's exchange runs into the previous round's tile
      if (TG > 1) NamedSync{1 + TG, TG * W * F::G}();
    }
  }
  __syncthreads();
  for (int idx = tid; idx < Y * W; idx += nth) {
    const int ikz = idx / W, cc = idx % W, ikx = xt * W + cc;
    if (ikx >= Box<N>::X) continue;
    const long ik = tile + idx;
    const int iy = iky - K, iz = ikz - K;
    const T kx = (T)ikx * g.alpha, ky = (T)iy, kz = (T)iz;
    const cpx<T> U = s_in[(0 * N + R0 + ikz) * W + cc];
    const cpx<T> V = s_in[(1 * N + R0 + ikz) * W + cc];
    const cpx<T> Wv = s_in[(2 * N + R0 + ikz) * W + cc];
    const cpx<T> RKv = (NO > 3) ? s_in[(3 * N + R0 + ikz) * W + cc] : czero<T>();
    if (SCHEME == SCHEME_RAW) {  // outputs 0-3 to K1, 4-5 to K2
      const T LL = keep_mode<T>(ikx, iy, iz, Box<N>::K, g.alpha) ? (T)1 : (T)0;
#pragma unroll
      for (int q = 0; q < NO; ++q) {
        const cpx<T> a = s_in[(q * N + R0 + ikz) * W + cc];
        cpx<T>* o = (q < 4) ? R.K1.c[q] : R.K2.c[q - 4];
        o[ik] = cpx<T>{LL * a.x, LL * a.y};
      }
      continue;
    }
    // curl of F(-(u x w)) as preStep/corStep form it (3D_NavierStokes/src/kernels.h:327-334)
    scheme_point<T, SCHEME>(g, R, p, stage, ik, ikx, iy, iz, ky * Wv.y - kz * V.y,
                            kz * V.x - ky * Wv.x, kz * U.y - kx * Wv.y, kx * Wv.x - kz * U.x,
                            kx * V.y - ky * U.y, ky * U.x - kx * V.x, RKv);
  }
}

// ---------------------------------------------------------------------------
// global energetics in FP64: sum over kept modes of |w|^2 / max(k^2, 0.001)
// (energy) and |w|^2 (enstrophy), as computeStats forms them
// (3D_NavierStokes/src/functions.h:139-152), plus |rho|^2 for a fourth
// component.  One partial per block, summed by energetics_final in a fixed
// order so that the result does not depend on scheduling.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) energetics_partial(Geom3<T> g, Fields4<T> S, int nc,
                                                          double* __restrict__ part) {
  const int W = kTileW;
  const long total = (long)g.XP * g.Y * g.Y;
  double e = 0.0, z = 0.0, r = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    long q = i / W;
    const int ikz = (int)(q % g.Y); q /= g.Y;
    const int iky = (int)(q % g.Y);
    const int ikx = (int)(q / g.Y) * W + w;
    if (ikx >= g.X || !keep_mode<T>(ikx, iky - g.K, ikz - g.K, g.K, g.alpha)) continue;
    const double kx = (double)ikx * (double)g.alpha, ky = iky - g.K, kz = ikz - g.K;
    double wk = kx * kx + ky * ky + kz * kz;
    wk = wk > 0.001 ? wk : 0.001;
    double v = 0.0;
    for (int c = 0; c < 3; ++c) {
      const cpx<T> a = S.c[c][i];
      v += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
    }
    z += v;
    e += v / wk;
    if (nc > 3) {
      const cpx<T> a = S.c[3][i];
      r += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
    }
  }
  __shared__ double s[3][256];
  s[0][threadIdx.x] = e; s[1][threadIdx.x] = z; s[2][threadIdx.x] = r;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[blockIdx.x * 3 + threadIdx.x] = s[threadIdx.x][0];
}

static __global__ void energetics_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  if (threadIdx.x < 3) {
    double a = 0.0;
    for (int b = 0; b < nblk; ++b) a += part[b * 3 + threadIdx.x];
    out[threadIdx.x] = a;
  }
}

// Boussinesq fluxes (3D_Boussinesq/src/functions.h:288-362): per block the
// partial sums of Re(conj(b) rho), b = v sin(theta) + w cos(theta), and of
// Re zeta at (0, kf, 0); summed by bflux_final in a fixed order
template <typename T>
__global__ void __launch_bounds__(256) bflux_partial(Geom3<T> g, Fields4<T> S, double sinth,
                                                     double costh, double kf,
                                                     double* __restrict__ part) {
  const int W = kTileW;
  const long total = (long)g.XP * g.Y * g.Y;
  double f = 0.0, zf = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    long q = i / W;
    const int ikz = (int)(q % g.Y); q /= g.Y;
    const int iky = (int)(q % g.Y);
    const int ikx = (int)(q / g.Y) * W + w;
    if (ikx >= g.X || !keep_mode<T>(ikx, iky - g.K, ikz - g.K, g.K, g.alpha)) continue;
    const double kx = (double)ikx * (double)g.alpha, ky = iky - g.K, kz = ikz - g.K;
    double wk = kx * kx + ky * ky + kz * kz;
    wk = wk > 0.001 ? wk : 0.001;
    const cpx<T> xa = S.c[0][i], ea = S.c[1][i], za = S.c[2][i], ra = S.c[3][i];
    const double xr = xa.x, xc = xa.y, er = ea.x, ec = ea.y, zr = za.x, zc = za.y;
    const double vr = (kz * xc - kx * zc) / wk, vc = (kx * zr - kz * xr) / wk;
    const double wr = (kx * ec - ky * xc) / wk, wc = (ky * xr - kx * er) / wk;
    const double br = vr * sinth + wr * costh, bc = vc * sinth + wc * costh;
    f += br * (double)ra.x + bc * (double)ra.y;
    if (ikx == 0 && ky == kf && kz == 0.0) zf += zr;
  }
  __shared__ double s[2][256];
  s[0][threadIdx.x] = f; s[1][threadIdx.x] = zf;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int k = 0; k < 2; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 2) part[blockIdx.x * 2 + threadIdx.x] = s[threadIdx.x][0];
}

static __global__ void bflux_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  if (threadIdx.x < 2) {
    double a = 0.0;
    for (int b = 0; b < nblk; ++b) a += part[b * 2 + threadIdx.x];
    out[threadIdx.x] = a;
  }
}

// ---------------------------------------------------------------------------
// layout conversion between the reference's FP64 boxes and the tile layout
// ---------------------------------------------------------------------------
template <typename T>
__global__ void box_from_ref(Geom3<T> g, const double2* __restrict__ src, cpx<T>* __restrict__ dst,
                             cpx<T>* __restrict__ low = nullptr) {
  const int W = kTileW;
  const long total = (long)g.XP * g.Y * g.Y;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    long r = i / W;
    const int ikz = (int)(r % g.Y); r /= g.Y;
    const int iky = (int)(r % g.Y);
    const int xt = (int)(r / g.Y);
    const int ikx = xt * W + w;
    cpx<T> v = czero<T>(), lo = czero<T>();
    if (ikx < g.X) {
      const double2 s = src[((long)ikz * g.Y + iky) * g.X + ikx];
      v = cpx<T>{(T)s.x, (T)s.y};
      lo = cpx<T>{(T)(s.x - (double)v.x), (T)(s.y - (double)v.y)};
    }
    dst[i] = v;
    if (low) low[i] = lo;
  }
}

template <typename T>
__global__ void box_to_ref(Geom3<T> g, const cpx<T>* __restrict__ src, double2* __restrict__ dst,
                           const cpx<T>* __restrict__ low = nullptr) {
  const int W = kTileW;
  const long total = (long)g.Y * g.Y * g.X;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int ikx = (int)(i % g.X);
    const long r = i / g.X;
    const int iky = (int)(r % g.Y), ikz = (int)(r / g.Y);
    const long j = (((long)(ikx / W) * g.Y + iky) * g.Y + ikz) * W + (ikx % W);
    const cpx<T> s = src[j];
    double2 v = make_double2((double)s.x, (double)s.y);
    if (low) {
      const cpx<T> c = low[j];
      v.x += (double)c.x;
      v.y += (double)c.y;
    }
    dst[i] = v;
  }
}

// The same two conversions on the kept modes only, for host boxes in
// page-locked memory that the kernels address directly: the upload reads the
// kept modes (and stores zero for every other mode of the state), the download
// writes the kept modes and leaves the other entries of the host box alone.
template <typename T>
__global__ void box_from_ref_kept(Geom3<T> g, const double2* __restrict__ src,
                                  cpx<T>* __restrict__ dst, cpx<T>* __restrict__ low) {
  const int W = kTileW;
  const long total = (long)g.XP * g.Y * g.Y;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    long r = i / W;
    const int ikz = (int)(r % g.Y); r /= g.Y;
    const int iky = (int)(r % g.Y);
    const int xt = (int)(r / g.Y);
    const int ikx = xt * W + w;
    cpx<T> v = czero<T>(), lo = czero<T>();
    if (ikx < g.X && keep_mode<T>(ikx, iky - g.K, ikz - g.K, g.K, g.alpha)) {
      const double2 s = src[((long)ikz * g.Y + iky) * g.X + ikx];
      v = cpx<T>{(T)s.x, (T)s.y};
      lo = cpx<T>{(T)(s.x - (double)v.x), (T)(s.y - (double)v.y)};
    }
    dst[i] = v;
    if (low) low[i] = lo;
  }
}

template <typename T>
__global__ void box_to_ref_kept(Geom3<T> g, const cpx<T>* __restrict__ src, double2* __restrict__ dst,
                                const cpx<T>* __restrict__ low) {
  const int W = kTileW;
  const long total = (long)g.Y * g.Y * g.X;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int ikx = (int)(i % g.X);
    const long r = i / g.X;
    const int iky = (int)(r % g.Y), ikz = (int)(r / g.Y);
    if (!keep_mode<T>(ikx, iky - g.K, ikz - g.K, g.K, g.alpha)) continue;
    const long j = (((long)(ikx / W) * g.Y + iky) * g.Y + ikz) * W + (ikx % W);
    const cpx<T> s = src[j];
    double2 v = make_double2((double)s.x, (double)s.y);
    if (low) {
      const cpx<T> c = low[j];
      v.x += (double)c.x;
      v.y += (double)c.y;
    }
    dst[i] = v;
  }
}

// running mean squares (the DNS's avgVelocity, 3D_NavierStokes/src/kernels.h:70-81)
template <typename T>
__global__ void rms_acc(const T* __restrict__ u, double* __restrict__ rms, long n, double count) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double v = (double)u[i];
    rms[i] = (rms[i] * count + v * v) / (count + 1.0);
  }
}

template <typename T>
__global__ void real_to_double(const T* __restrict__ src, double* __restrict__ dst, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

template <typename T>
__global__ void copy_fields(Fields4<T> src, Fields4<T> dst, int nc, long len) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x)
    for (int q = 0; q < nc; ++q) dst.c[q][i] = src.c[q][i];
}


// ---------------------------------------------------------------------------
// tangent-linear and adjoint of the RK4/CN step (SCHEME_NS_RK4)
//
// With E the inverse transform of a stored half spectrum (Hermitian
// completion), F = (1/N^3) FFT restricted to the kept modes, B = i k x / k^2
// (Biot-Savart), C = i k x (curl), the right-hand side is
//   N(w) = C F(E(B w) x E(w)),
// bilinear in w, so N'(w) d = C F(E(B d) x E(w)) + C F(E(B w) x E(d)).  Under
// the real inner product of the stored coefficients E^T = 2 N^3 F and
// F^T = E / (2 N^3), B and C are self-adjoint, and a.(b x c) = b.(c x a), so
//   N'(w)^T l = B F(E(w) x E(C l)) + F(E(C l) x E(B w)).
// Every term is one bilinear product P(a, b) = F(-(E(a) x E(b))) of the five
// passes (pass A in pair mode, pass E in raw mode); the kernels below combine
// the products and apply the stage arithmetic of scheme_point's RK4 branch.
// ---------------------------------------------------------------------------
template <typename T>
struct TileMode {
  bool ok, keep;
  T kx, ky, kz, wk;
};

// mode of element i of a tile-major box [xt][iky][ikz][W]
template <typename T>
__device__ __forceinline__ TileMode<T> tile_mode(const Geom3<T>& g, long i) {
  TileMode<T> m;
  const int W = kTileW;
  const int w = (int)(i % W);
  long q = i / W;
  const int ikz = (int)(q % g.Y); q /= g.Y;
  const int iky = (int)(q % g.Y);
  const int ikx = (int)(q / g.Y) * W + w;
  m.ok = ikx < g.X;
  m.keep = m.ok && keep_mode<T>(ikx, iky - g.K, ikz - g.K, g.K, g.alpha);
  m.kx = (T)ikx * g.alpha; m.ky = (T)(iky - g.K); m.kz = (T)(ikz - g.K);
  m.wk = m.kx * m.kx + m.ky * m.ky + m.kz * m.kz;
  return m;
}

template <typename T>
__device__ __forceinline__ void load3(const Fields4<T>& F, long i, cpx<T> (&x)[3]) {
  x[0] = F.c[0][i]; x[1] = F.c[1][i]; x[2] = F.c[2][i];
}

// out = -LL C (Pa + Pb)                       (tangent right-hand side)
// out = -LL (B Pa + Pb)                       (adjoint right-hand side)
template <typename T>
__global__ void lin_combine(Geom3<T> g, int adjoint, Fields4<T> Pa, Fields4<T> Pb, Fields4<T> out,
                            long len) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x) {
    const TileMode<T> m = tile_mode(g, i);
    cpx<T> a[3], b[3], r[3];
    load3(Pa, i, a);
    load3(Pb, i, b);
    if (!adjoint) {
      cpx<T> s[3];
      for (int c = 0; c < 3; ++c) s[c] = cpx<T>{a[c].x + b[c].x, a[c].y + b[c].y};
      for (int c = 0; c < 3; ++c) r[c] = spec_op<T>(OP_CURL, c, s, m.kx, m.ky, m.kz, (T)0);
    } else {
      const T wki = wkinv(m.wk);
      for (int c = 0; c < 3; ++c) {
        const cpx<T> ba = spec_op<T>(OP_BS, c, a, m.kx, m.ky, m.kz, wki);
        r[c] = cpx<T>{ba.x + b[c].x, ba.y + b[c].y};
      }
    }
    const T LL = m.keep ? (T)-1 : (T)0;
    for (int c = 0; c < 3; ++c) out.c[c][i] = cpx<T>{LL * r[c].x, LL * r[c].y};
  }
}

// CN factor of an RK stage, (1 - q nk)/(1 + q nk) = 1 - e
template <typename T>
__device__ __forceinline__ T stage_e(T q, T nk) { return (T)2 * q * nk / ((T)1 + q * nk); }

// component c's viscous factor nu k^2 dt (the density's divided by Sc)
template <typename T>
__device__ __forceinline__ T comp_nk(T nk, int c, T sc) { return c == 3 ? nk / sc : nk; }

// tangent stage: K = dt LL n, Z = (1 - e)(D + fr K)
template <typename T>
__global__ void tan_stage(Geom3<T> g, T dt, T nu, T q, T fr, Fields4<T> n, Fields4<T> D,
                          Fields4<T> Kout, Fields4<T> Zout, long len, int nc, T sc) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x) {
    const TileMode<T> m = tile_mode(g, i);
    const T LL = m.keep ? (T)1 : (T)0;
    for (int c = 0; c < nc; ++c) {
      const T e = stage_e(q, comp_nk(dt * nu * m.wk, c, sc));
      const cpx<T> nn = n.c[c][i], d = D.c[c][i];
      const cpx<T> k = cpx<T>{dt * LL * nn.x, dt * LL * nn.y};
      const cpx<T> v = cpx<T>{d.x + fr * k.x, d.y + fr * k.y};
      Kout.c[c][i] = k;
      Zout.c[c][i] = cpx<T>{v.x - e * v.x, v.y - e * v.y};
    }
  }
}

// divergence removal of scheme_point's final stage, o - k (k.o) / k^2
template <typename T, int M>
__device__ __forceinline__ void remove_div(const TileMode<T>& m, cpx<T> (&o)[M]) {
  const T wki = wkinv(m.wk);
  const T pr = (m.kx * o[0].x + m.ky * o[1].x + m.kz * o[2].x) * wki;
  const T pi = (m.kx * o[0].y + m.ky * o[1].y + m.kz * o[2].y) * wki;
  o[0] = cpx<T>{o[0].x - m.kx * pr, o[0].y - m.kx * pi};
  o[1] = cpx<T>{o[1].x - m.ky * pr, o[1].y - m.ky * pi};
  o[2] = cpx<T>{o[2].x - m.kz * pr, o[2].y - m.kz * pi};
}

// tangent final stage:
// D' = Pdiv LL [(1 - eS) D + (1 - eI)(K1/6 + dt n/6 + (K2 + K3)/3)]; DX' = the
// same before the divergence removal (the tangent of the stage input the next
// step starts from: the forward step hands its final stage on unprojected)
template <typename T>
__global__ void tan_final(Geom3<T> g, T dt, T nu, Fields4<T> n, Fields4<T> K1, Fields4<T> K2,
                          Fields4<T> K3, Fields4<T> D, Fields4<T> DX, long len, int nc, T sc) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x) {
    const TileMode<T> m = tile_mode(g, i);
    const T LL = m.keep ? (T)1 : (T)0;
    const T sixth = (T)(1.0 / 6.0), third = (T)(1.0 / 3.0);
    cpx<T> o[4];
    for (int c = 0; c < nc; ++c) {
      const T nk = comp_nk(dt * nu * m.wk, c, sc), hn = (T)0.5 * nk;
      const T eS = nk / ((T)1 + hn), eI = hn / ((T)1 + hn);
      const cpx<T> d = D.c[c][i], a = K1.c[c][i], b = K2.c[c][i], k3 = K3.c[c][i], nn = n.c[c][i];
      const T ix = sixth * (a.x + dt * nn.x) + third * (b.x + k3.x);
      const T iy = sixth * (a.y + dt * nn.y) + third * (b.y + k3.y);
      o[c] = cpx<T>{LL * ((d.x - eS * d.x) + (ix - eI * ix)), LL * ((d.y - eS * d.y) + (iy - eI * iy))};
    }
    for (int c = 0; c < nc; ++c) DX.c[c][i] = o[c];
    remove_div(m, o);
    for (int c = 0; c < nc; ++c) D.c[c][i] = o[c];
  }
}

// adjoint of the final stage: a = LL Pdiv L', Lz = (1 - eS) a, b = (1 - eI) a,
// Lk1 = b/6, Lk2 = Lk3 = b/3, Ln = dt b/6
template <typename T>
__global__ void adj_final(Geom3<T> g, T dt, T nu, Fields4<T> Lin, Fields4<T> Lz, Fields4<T> Lk1,
                          Fields4<T> Lk2, Fields4<T> Lk3, Fields4<T> Ln, long len, int nc, T sc) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x) {
    const TileMode<T> m = tile_mode(g, i);
    const T LL = m.keep ? (T)1 : (T)0;
    cpx<T> a[4];
    for (int c = 0; c < nc; ++c) a[c] = Lin.c[c][i];
    remove_div(m, a);
    for (int c = 0; c < nc; ++c) {
      const T nk = comp_nk(dt * nu * m.wk, c, sc), hn = (T)0.5 * nk;
      const T eS = nk / ((T)1 + hn), eI = hn / ((T)1 + hn);
      const cpx<T> x = cpx<T>{LL * a[c].x, LL * a[c].y};
      const cpx<T> b = cpx<T>{x.x - eI * x.x, x.y - eI * x.y};
      Lz.c[c][i] = cpx<T>{x.x - eS * x.x, x.y - eS * x.y};
      Lk1.c[c][i] = cpx<T>{b.x / (T)6, b.y / (T)6};
      Lk2.c[c][i] = cpx<T>{b.x / (T)3, b.y / (T)3};
      Lk3.c[c][i] = cpx<T>{b.x / (T)3, b.y / (T)3};
      Ln.c[c][i] = cpx<T>{dt * b.x / (T)6, dt * b.y / (T)6};
    }
  }
}

// adjoint of an RK stage Z = (1 - e)(D + fr K) given Ls, the adjoint of Z:
// Lz += (1 - e) Ls, Lk += fr (1 - e) Ls, and Ln = dt LL Lk, the input of the
// adjoint right-hand side of the stage that produced K
template <typename T>
__global__ void adj_stage(Geom3<T> g, T dt, T nu, T q, T fr, Fields4<T> Ls, Fields4<T> Lz,
                          Fields4<T> Lk, Fields4<T> Ln, long len, int nc, T sc) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x) {
    const TileMode<T> m = tile_mode(g, i);
    const T LL = m.keep ? (T)1 : (T)0;
    for (int c = 0; c < nc; ++c) {
      const T e = stage_e(q, comp_nk(dt * nu * m.wk, c, sc));
      const cpx<T> l = Ls.c[c][i];
      const cpx<T> dl = cpx<T>{l.x - e * l.x, l.y - e * l.y};
      const cpx<T> z = Lz.c[c][i], k = Lk.c[c][i];
      Lz.c[c][i] = cpx<T>{z.x + dl.x, z.y + dl.y};
      const cpx<T> kn = cpx<T>{k.x + fr * dl.x, k.y + fr * dl.y};
      Lk.c[c][i] = kn;
      Ln.c[c][i] = cpx<T>{dt * LL * kn.x, dt * LL * kn.y};
    }
  }
}

// y = b y + a x  (nc components)
template <typename T>
__global__ void lin_axpby(Fields4<T> y, T b, T a, Fields4<T> x, long len, int nc) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x)
    for (int c = 0; c < nc; ++c) {
      const cpx<T> u = y.c[c][i], v = x.c[c][i];
      y.c[c][i] = cpx<T>{b * u.x + a * v.x, b * u.y + a * v.y};
    }
}

// out = z + a x  (nc components)
template <typename T>
__global__ void lin_shift(Fields4<T> out, Fields4<T> z, T a, Fields4<T> x, long len, int nc) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x)
    for (int c = 0; c < nc; ++c) {
      const cpx<T> u = z.c[c][i], v = x.c[c][i];
      out.c[c][i] = cpx<T>{u.x + a * v.x, u.y + a * v.y};
    }
}

// partial sums of |x|^2 (nc components), one per block
template <typename T>
__global__ void __launch_bounds__(256) lin_norm2(Fields4<T> x, long len, int nc, double* part) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x)
    for (int c = 0; c < nc; ++c) {
      const cpx<T> v = x.c[c][i];
      s += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
    }
  __shared__ double r[256];
  r[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) r[threadIdx.x] += r[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = r[0];
}

// Boussinesq adjoint right-hand side from the products
//   PA = F(-(E(w) x E(C lw))), PB = F(-(E(C lw) x E(B w))),
//   SA = [F(psi i k rho) (3), F(psi u_x)], SB = [F(psi u_y), F(psi u_z)], psi = E(l_rho):
// l_w' = -B (PA + F(psi grad rho) - e l_rho) - PB,    e = (0, cos th, sin th)
// l_rho' = conj(b) . l_w + i k . F(psi u),            b = Ri i (-(ky sin th - kz cos th), kx sin th, -kx cos th)
// (buoyancy and stratification of scheme_point's Boussinesq branch, transposed)
template <typename T>
__global__ void bous_adj_combine(Geom3<T> g, T ri, T sinth, T costh, Fields4<T> PA, Fields4<T> PB,
                                 Fields4<T> SA, Fields4<T> SB, Fields4<T> X, Fields4<T> out, long len) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
       i += (long)gridDim.x * blockDim.x) {
    const TileMode<T> m = tile_mode(g, i);
    const T LL = m.keep ? (T)1 : (T)0;
    const T wki = wkinv(m.wk);
    const cpx<T> lr = X.c[3][i];
    cpx<T> v[3];
    for (int c = 0; c < 3; ++c) {
      const cpx<T> a = PA.c[c][i], sg = SA.c[c][i];
      v[c] = cpx<T>{a.x + sg.x, a.y + sg.y};
    }
    v[1] = cpx<T>{v[1].x - costh * lr.x, v[1].y - costh * lr.y};
    v[2] = cpx<T>{v[2].x - sinth * lr.x, v[2].y - sinth * lr.y};
    for (int c = 0; c < 3; ++c) {
      const cpx<T> bw = spec_op<T>(OP_BS, c, v, m.kx, m.ky, m.kz, wki), pb = PB.c[c][i];
      out.c[c][i] = cpx<T>{-LL * (bw.x + pb.x), -LL * (bw.y + pb.y)};
    }
    // conj(i beta) l = beta (l.y, -l.x);  i k u = (-k u.y, k u.x)
    const T beta[3] = {-ri * (m.ky * sinth - m.kz * costh), ri * m.kx * sinth, -ri * m.kx * costh};
    const cpx<T> su[3] = {SA.c[3][i], SB.c[0][i], SB.c[1][i]};
    const T kk[3] = {m.kx, m.ky, m.kz};
    T rx = 0, ry = 0;
    for (int c = 0; c < 3; ++c) {
      const cpx<T> l = X.c[c][i];
      rx += beta[c] * l.y - kk[c] * su[c].y;
      ry += -beta[c] * l.x + kk[c] * su[c].x;
    }
    out.c[3][i] = cpx<T>{LL * rx, LL * ry};
  }
}

// ---------------------------------------------------------------------------
// host engine
// ---------------------------------------------------------------------------
template <typename T>
struct Engine3D final : Engine3DBase {
  Geom3<T> g{};
  int scheme = 0;
  int nc = 3;    // state components
  int nfi = 6;   // fields transformed to physical space
  int nfo = 3;   // fields transformed back
  long box = 0;  // complex words per component
  StepParams<T> prm{};
  cudaStream_t stream = 0;
  int first_rhs = 1;     // mask velocity on the first evaluation after an upload
  cpx<T>* pool = nullptr;
  cpx<T>* tw = nullptr;
  T* dump = nullptr;     // physical fields of the last step (Heun schemes)
  // dump_mode bit 0: the fields the step starts from (the predictor's input)
  // instead of the predicted state's (the corrector's input); bit 1: the
  // velocity beside the vorticity (six fields)
  int dump_mode = 0;
  double* d_rms = nullptr;  // running mean squares of u, v, w (FP64, 3 n^3)
  Regs<T> R{};
  cpx<T>* B1 = nullptr;
  cpx<T>* B2 = nullptr;
  double2* stage_h = nullptr;  // device FP64 staging box
  int* d_status = nullptr;     // device error flag of the bounded waits
  double* d_energ = nullptr;   // energetics partial sums
  unsigned long long* d_umax = nullptr;  // max |u| of the x-pass (bits of a non-negative double)
  double* d_flux = nullptr;    // buoyancy-flux partial sums
  // linearised step (tangent / adjoint), allocated on first use
  cpx<T>* lin = nullptr;
  Fields4<T> Zb[4]{};          // base stage states z, z1, z2, z3
  Fields4<T> LA{}, LN{}, LS{}, LZ{}, LK1{}, LK2{}, LK3{}, PA{}, PB{}, LD{}, LT{};
  // LX: the stage input X0 kept across a Boussinesq tangent right-hand side
  // (which evaluates the engine's own right-hand side through X0); LDX: the
  // tangent of X0 after a tangent step, valid while lin_dx is set
  Fields4<T> LX{}, LDX{};
  bool lin_dx = false;
  Fields4<T> SA{}, SB{};       // Boussinesq adjoint products: psi (i k rho) | psi u
  int c_variant = 0;           // x-pass variant chosen by the autotuner
  // pass A on packed f32x2 transforms (FP32 engine; chosen by the autotuner
  // when its shared memory fits) and the autotuner's timings (scalar, packed)
  bool a_pk = false, a_pk_ok = false;
  float a_ms[2] = {-1.f, -1.f};
  int c_resident[16] = {1, 1, 1, 1};  // resident blocks of each x-pass variant
  float c_ms[16] = {};                 // autotuner timings (ms per launch)
  long launches = 0;
  // optional per-pass timing with CUDA events recorded between the passes
  bool profiling = false;
  // programmatic dependent launch of the passes of a right-hand side (each
  // pass's blocks launch and set up while the previous pass drains), PSG_PDL:
  // 0 off, 1 every pass, 2 (default) every pass but the x-pass.  The x-pass is
  // a single wave of resident blocks sized to fill the SMs; launched early, its
  // blocks land beside the y-inverse's last ones, and with the smaller block
  // variants the step loses more than the overlap gains.  Off while the
  // per-pass events are recorded.
  int pdl = 2;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_tag;
  size_t ev_used = 0;

  void mark(int tag) {
    if (!profiling) return;
    if (ev_used == ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
    cudaEventRecord(ev_pool[ev_used], stream);
    ev_tag.push_back(tag);
    ++ev_used;
  }
  int profile(int enable) override {
    profiling = enable != 0;
    ev_used = 0;
    ev_tag.clear();
    return PSG_OK;
  }
  int profile_read(double* ms, long* counts) override {
    for (int k = 0; k < 5; ++k) { ms[k] = 0.0; counts[k] = 0; }
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    for (size_t i = 1; i < ev_used; ++i) {
      const int t = ev_tag[i];
      if (t < 0) continue;
      float v = 0.f;
      PSG_CUDA_TRY(cudaEventElapsedTime(&v, ev_pool[i - 1], ev_pool[i]));
      ms[t] += v;
      counts[t] += 1;
    }
    return PSG_OK;
  }

  // dynamic shared memory of each pass (must match the kernels' carve-up)
  // pass A runs three groups of W x G threads for the nine Boussinesq fields
  // (three rounds, none idle) and two for the six Navier-Stokes fields
  int groups_a() const { return nc == 4 ? 3 : 2; }
  size_t smem_a() const { return smem_a_nc(nc, groups_a()); }
  // passes B and D: one area for the staged tile and then the exchange; twiddles
  size_t smem_b() const {
    return sizeof(cpx<T>) * (std::max<size_t>((size_t)g.Y * kTileW, (size_t)kTileW * col_stride()) + g.n);
  }
  // x-pass variants: bit 0 twice the rows per block (256/G instead of 128/G),
  // bit 3 half of them (64/G; not with bit 0), bit 1 two copy buffers per
  // warp, bit 2 (FP32) packed f32x2 transforms, two lines each
  static constexpr int kCVariants = 16;
  static int c_rows_x2(int v) { return (v & 8) ? 1 : (v & 1) ? 4 : 2; }  // rows in units of 64/G
  static int c_stages(int v) { return (v & 2) ? 2 : 1; }
  static bool c_packed(int v) { return (v & 4) != 0; }
  static bool c_valid(int v) { return !((v & 8) && (v & 1)) && (!c_packed(v) || sizeof(T) == 4); }
  size_t smem_c_v(int v) const {
    const size_t L = (size_t)(64 / fft_g()) * c_rows_x2(v);
    return sizeof(cpx<T>) * ((size_t)c_stages(v) * nfi * L * g.XP + 2 * g.n + L * row_stride());
  }
  size_t smem_d() const {
    return sizeof(cpx<T>) * (std::max<size_t>((size_t)g.n * kTileW, (size_t)kTileW * col_stride()) + g.n);
  }
  size_t smem_e() const { return smem_e_no(nfo); }
  int col_stride() const {
    switch (g.n) {
      case 16: return ColStride<LineFFT<16, 1, T>::SMEM>::value;
      case 32: return ColStride<LineFFT<32, 1, T>::SMEM>::value;
      case 64: return ColStride<LineFFT<64, 1, T>::SMEM>::value;
      case 128: return ColStride<LineFFT<128, 1, T>::SMEM>::value;
      default: return ColStride<LineFFT<256, 1, T>::SMEM>::value;
    }
  }
  int row_stride() const {
    switch (g.n) {
      case 16: return RowOps<T, 16>::SX;
      case 32: return RowOps<T, 32>::SX;
      case 64: return RowOps<T, 64>::SX;
      case 128: return RowOps<T, 128>::SX;
      default: return RowOps<T, 256>::SX;
    }
  }
  int fft_g() const {
    switch (g.n) {
      case 16: return LineFFT<16, 1, T>::G;
      case 32: return LineFFT<32, 1, T>::G;
      case 64: return LineFFT<64, 1, T>::G;
      case 128: return LineFFT<128, 1, T>::G;
      default: return LineFFT<256, 1, T>::G;
    }
  }
  int fft_smem() const {
    switch (g.n) {
      case 16: return LineFFT<16, 1, T>::SMEM;
      case 32: return LineFFT<32, 1, T>::SMEM;
      case 64: return LineFFT<64, 1, T>::SMEM;
      case 128: return LineFFT<128, 1, T>::SMEM;
      default: return LineFFT<256, 1, T>::SMEM;
    }
  }

  int init(int n, double alpha, int scheme_) override {
    if (!(n == 16 || n == 32 || n == 64 || n == 128 || n == 256)) {
      psg_set_error("3D grid size %d unsupported (powers of two 16..256)", n);
      return PSG_ERR_UNSUPPORTED;
    }
    g.n = n; g.K = n / 3; g.X = g.K + 1; g.Y = 2 * g.K + 1;
    g.XP = (g.X + kTileW - 1) / kTileW * kTileW;
    g.alpha = (T)alpha;
    scheme = scheme_;
    if (const char* e = getenv("PSG_PDL")) pdl = atoi(e);
    if (pdl < 0 || pdl > 2) pdl = 2;
    const bool bous = (scheme == SCHEME_BOUS_RK4);
    nc = bous ? 4 : 3;
    nfi = bous ? 9 : 6;
    nfo = bous ? 4 : 3;
    box = (long)g.Y * g.Y * g.XP;
    const int nregs = (scheme == SCHEME_NS_HEUN || scheme == SCHEME_EULER_HEUN) ? 2 : 5;
    const long b1 = (long)nfi * n * g.Y * g.XP;
    const long b3 = (long)nfo * n * n * g.XP;
    const long b2 = (long)nfi * n * n * g.XP;
    // B1 also holds the x-pass output of the linearised Boussinesq step's
    // scalar products (6 fields)
    const long b3lin = (bous ? 6L : 3L) * n * n * g.XP;
    long nb1 = b1 > b3 ? b1 : b3;
    if (b3lin > nb1) nb1 = b3lin;
    // the FP32 engine carries the rounding error of its state updates
    const int ncomp_regs = std::is_same<T, float>::value ? 1 : 0;
    const long total = (long)(nregs + ncomp_regs) * nc * box + nb1 + b2 + 2 * n;
    PSG_CUDA_TRY(cudaMalloc(&pool, sizeof(cpx<T>) * total));
    PSG_CUDA_TRY(cudaMemset(pool, 0, sizeof(cpx<T>) * total));
    cpx<T>* p = pool;
    Fields4<T>* regs[5] = {&R.S, &R.K1, &R.X0, &R.K2, &R.K3};
    for (int r = 0; r < 5; ++r)
      for (int q = 0; q < 4; ++q) regs[r]->c[q] = nullptr;
    for (int q = 0; q < 4; ++q) R.SC.c[q] = nullptr;
    for (int r = 0; r < nregs; ++r)
      for (int q = 0; q < nc; ++q) { regs[r]->c[q] = p; p += box; }
    if (ncomp_regs)
      for (int q = 0; q < nc; ++q) { R.SC.c[q] = p; p += box; }
    B1 = p; p += nb1;
    B2 = p; p += b2;
    tw = p; p += 2 * n;
    // twiddle tables: the plain plan (column passes, inverse x rows) and the
    // swapped plan (forward x rows)
    std::vector<cpx<T>> h(2 * n);
    switch (n) {
      case 16: LineFFT<16, 1, T>::host_table(h.data()); LineFFT<16, 1, T, true>::host_table(h.data() + n); break;
      case 32: LineFFT<32, 1, T>::host_table(h.data()); LineFFT<32, 1, T, true>::host_table(h.data() + n); break;
      case 64: LineFFT<64, 1, T>::host_table(h.data()); LineFFT<64, 1, T, true>::host_table(h.data() + n); break;
      case 128: LineFFT<128, 1, T>::host_table(h.data()); LineFFT<128, 1, T, true>::host_table(h.data() + n); break;
      default: LineFFT<256, 1, T>::host_table(h.data()); LineFFT<256, 1, T, true>::host_table(h.data() + n); break;
    }
    PSG_CUDA_TRY(cudaMemcpy(tw, h.data(), sizeof(cpx<T>) * 2 * n, cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMalloc(&stage_h, sizeof(double2) * (long)g.Y * g.Y * g.X));
    PSG_CUDA_TRY(cudaMalloc(&d_status, sizeof(int)));
    PSG_CUDA_TRY(cudaMemset(d_status, 0, sizeof(int)));
    if (scheme == SCHEME_NS_HEUN || scheme == SCHEME_EULER_HEUN)
      PSG_CUDA_TRY(cudaMalloc(&dump, sizeof(T) * 3L * n * n * n));
    if (int rc = set_smem_limits()) return rc;
    return autotune();
  }

  ~Engine3D() override {
    release();
    for (auto e : ev_pool) cudaEventDestroy(e);
  }
  void release() {
    if (pool) cudaFree(pool);
    if (stage_h) cudaFree(stage_h);
    if (dump) cudaFree(dump);
    if (d_status) cudaFree(d_status);
    if (d_energ) cudaFree(d_energ);
    if (d_umax) cudaFree(d_umax);
    if (d_flux) cudaFree(d_flux);
    if (d_rms) cudaFree(d_rms);
    d_rms = nullptr;
    if (lin) cudaFree(lin);
    lin = nullptr;
    d_energ = nullptr; d_umax = nullptr; d_flux = nullptr;
    pool = nullptr; stage_h = nullptr; dump = nullptr; d_status = nullptr;
  }

  template <int N>
  int set_smem_limits_n() {
    int dev = 0, big = 0;
    PSG_CUDA_TRY(cudaGetDevice(&dev));
    PSG_CUDA_TRY(cudaDeviceGetAttribute(&big, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    big -= 1024;  // static shared memory of the kernels (mbarrier, flags)
    const size_t need[5] = {smem_a(), smem_b(), smem_c_v(0), smem_d(), smem_e()};
    for (size_t x : need)
      if (x > (size_t)big) {
        psg_set_error("3D grid %d needs %zu bytes of shared memory per block, device allows %d",
                      g.n, x, big);
        return PSG_ERR_UNSUPPORTED;
      }
#define PSG_SMEM(kern) PSG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, big))
    PSG_SMEM((pass_a<T, N, 3, 6>));
    PSG_SMEM((pass_a<T, N, 4, 9, 0, 3>));
    if constexpr (sizeof(T) == 4) {
      a_pk_ok = smem_a_pk_n<N>(nc) <= (size_t)big;
      if (a_pk_ok) {
        PSG_SMEM((pass_a_pk<N, 3, 6>));
        PSG_SMEM((pass_a_pk<N, 4, 9>));
      }
    }
    PSG_SMEM((pass_b<T, N>));
    for (int v = 0; v < kCVariants; ++v) {
      if (!c_valid(v)) continue;
      for (int nf : {6, 9, 7}) {
        const void* k = c_kernel_nf<N>(v, nf);
        if (k) PSG_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
      }
    }
    PSG_SMEM((pass_d<T, N>));
    PSG_SMEM((pass_e<T, N, 3, SCHEME_NS_HEUN>));
    PSG_SMEM((pass_e<T, N, 3, SCHEME_EULER_HEUN>));
    PSG_SMEM((pass_e<T, N, 3, SCHEME_NS_RK4>));
    PSG_SMEM((pass_e<T, N, 4, SCHEME_BOUS_RK4>));
#undef PSG_SMEM
    int nsm = 0;
    PSG_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (int v = 0; v < kCVariants; ++v) {
      int occ = 0;
      const void* k = c_valid(v) ? c_kernel<N>(v) : nullptr;
      if (k && smem_c_v(v) <= (size_t)big)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, c_threads<N>(v), smem_c_v(v));
      c_resident[v] = nsm * occ;  // 0: variant does not fit (or is not built)
    }
    return PSG_OK;
  }

  template <int N>
  static int c_threads(int v) { return 64 * c_rows_x2(v); }

  // the kernel of variant v for nf fields (nullptr: not built; the packed
  // form takes the forward fields only, the adjoint's products (7) run the
  // scalar kernel of the same shape)
  template <int N, int L, int ST>
  static const void* c_fn(int nf, bool pk) {
    if constexpr (sizeof(T) == 4) {
      if (pk && nf != 7)
        return nf == 9 ? (const void*)pass_c<T, N, 9, L, ST, 1> : (const void*)pass_c<T, N, 6, L, ST, 1>;
    }
    if (pk && sizeof(T) != 4) return nullptr;
    return nf == 9 ? (const void*)pass_c<T, N, 9, L, ST> :
           nf == 7 ? (const void*)pass_c<T, N, 7, L, ST> : (const void*)pass_c<T, N, 6, L, ST>;
  }
  template <int N>
  static const void* c_kernel_nf(int v, int nf) {
    constexpr int L0 = 64 / LineFFT<N, 1, T>::G;
    const bool pk = c_packed(v);
    const int rows = c_rows_x2(v), st = c_stages(v);
    if (rows == 1) return st == 1 ? c_fn<N, L0, 1>(nf, pk) : c_fn<N, L0, 2>(nf, pk);
    if (rows == 2) return st == 1 ? c_fn<N, 2 * L0, 1>(nf, pk) : c_fn<N, 2 * L0, 2>(nf, pk);
    return st == 1 ? c_fn<N, 4 * L0, 1>(nf, pk) : c_fn<N, 4 * L0, 2>(nf, pk);
  }
  template <int N>
  const void* c_kernel(int v) const {
    return c_kernel_nf<N>(v, scheme == SCHEME_BOUS_RK4 ? 9 : 6);
  }
  // launch on the engine's stream; dep: with the programmatic-serialisation
  // attribute, for a pass whose predecessor on the stream is another pass
  // kernel (both wait and trigger through pdl_wait / pdl_trigger)
  template <typename... P, typename... A>
  int launch_k(bool dep, void (*k)(P...), dim3 grid, dim3 blk, size_t smem, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = blk;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    if (dep && pdl && !profiling) {
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
    }
    PSG_CUDA_TRY(cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...));
    return PSG_OK;
  }

  // nf: fields the x-pass reads (6: -(u x w); 9: + u.grad rho; 7: the
  // Boussinesq adjoint's scalar products); 0: the engine's own
  template <int N>
  int launch_c(int v, T scale, T* dp, int nf = 0, unsigned long long* um = nullptr,
               bool dep = false) {
    constexpr int L0 = 64 / LineFFT<N, 1, T>::G;
    constexpr int RPW = 32 / LineFFT<N, 1, T>::G;  // rows per warp tile
    const int wpb = L0 * c_rows_x2(v) / RPW;       // warps per block
    const int nwt = (N * N) / RPW;
    const int nblk = (nwt + wpb - 1) / wpb;
    const int grid = nblk < c_resident[v] ? nblk : c_resident[v];
    const size_t sm = smem_c_v(v);
    const int th = c_threads<N>(v);
    if (!nf) nf = (scheme == SCHEME_BOUS_RK4) ? 9 : 6;
    const void* k = c_kernel_nf<N>(v, nf);
    if (!k) { psg_set_error("x-pass variant %d is not built", v); return PSG_ERR_ARG; }
    Geom3<T> gg = g;
    const cpx<T>* in = B2;
    cpx<T>* out = B1;
    const cpx<T>* twp = tw;
    int* st = d_status;
    int nw = nwt;
    unsigned long long* u = um;
    int dnf = (dp && (dump_mode & 2)) ? 6 : 3;
    void* args[] = {&gg, &in, &out, &twp, &scale, &dp, &st, &nw, &u, &dnf};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(th);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    if (dep && pdl && !profiling) {
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
    }
    PSG_CUDA_TRY(cudaLaunchKernelExC(&cfg, k, args));
    return PSG_OK;
  }

  // Autotuner: time every x-pass variant that fits on this device (one warm-up
  // and three timed launches on the engine's own scratch buffers) and keep the
  // fastest.  The transforms' cost does not depend on the data.
  template <int N>
  int autotune_n() {
    // PSG_XPASS_VARIANT=0..15 pins the choice (reproducible profiling runs)
    if (const char* pin = getenv("PSG_XPASS_VARIANT")) {
      const int v = atoi(pin);
      if (v >= 0 && v < kCVariants && c_resident[v] > 0) {
        c_variant = v;
        for (int k = 0; k < kCVariants; ++k) c_ms[k] = -1.f;
        return PSG_OK;
      }
    }
    cudaEvent_t a, b;
    PSG_CUDA_TRY(cudaEventCreate(&a));
    PSG_CUDA_TRY(cudaEventCreate(&b));
    const T scale = (T)1 / ((T)N * (T)N * (T)N);
    float best = 1e30f;
    int pick = 0;
    for (int v = 0; v < kCVariants; ++v) {
      c_ms[v] = -1.f;
      if (c_resident[v] <= 0) continue;
      launch_c<N>(v, scale, nullptr);
      cudaEventRecord(a, stream);
      for (int r = 0; r < 3; ++r) launch_c<N>(v, scale, nullptr);
      cudaEventRecord(b, stream);
      cudaError_t e = cudaEventSynchronize(b);
      if (e != cudaSuccess) { cudaEventDestroy(a); cudaEventDestroy(b); PSG_CUDA_TRY(e); }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      c_ms[v] = ms / 3.f;
      if (c_ms[v] < best) { best = c_ms[v]; pick = v; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    c_variant = pick;
    PSG_CUDA_TRY(cudaGetLastError());
    return check_status();
  }
  // pass A, FP32: scalar or packed transforms, timed the same way
  // (PSG_PASSA_PACKED=0/1 pins the choice)
  template <int N>
  int autotune_a_n() {
    a_ms[0] = a_ms[1] = -1.f;
    a_pk = false;
    if (sizeof(T) != 4 || !a_pk_ok) return PSG_OK;
    if (const char* pin = getenv("PSG_PASSA_PACKED")) {
      a_pk = atoi(pin) != 0;
      return PSG_OK;
    }
    cudaEvent_t a, b;
    PSG_CUDA_TRY(cudaEventCreate(&a));
    PSG_CUDA_TRY(cudaEventCreate(&b));
    for (int pk = 0; pk < 2; ++pk) {
      int rc = launch_a<N>(false, pk != 0, stage_input(), 0);
      cudaEventRecord(a, stream);
      for (int r = 0; r < 3 && !rc; ++r) rc = launch_a<N>(false, pk != 0, stage_input(), 0);
      cudaEventRecord(b, stream);
      cudaError_t e = cudaEventSynchronize(b);
      if (rc || e != cudaSuccess) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (rc) return rc;
        PSG_CUDA_TRY(e);
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      a_ms[pk] = ms / 3.f;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    a_pk = a_ms[1] < a_ms[0];
    PSG_CUDA_TRY(cudaGetLastError());
    return check_status();
  }
  int autotune() override {
    int rc;
    switch (g.n) {
      case 16: rc = autotune_n<16>(); return rc ? rc : autotune_a_n<16>();
      case 32: rc = autotune_n<32>(); return rc ? rc : autotune_a_n<32>();
      case 64: rc = autotune_n<64>(); return rc ? rc : autotune_a_n<64>();
      case 128: rc = autotune_n<128>(); return rc ? rc : autotune_a_n<128>();
      default: rc = autotune_n<256>(); return rc ? rc : autotune_a_n<256>();
    }
  }
  int tuning_a(int* packed, float* ms) override {
    if (packed) *packed = a_pk ? 1 : 0;
    if (ms) { ms[0] = a_ms[0]; ms[1] = a_ms[1]; }
    return PSG_OK;
  }
  int tuning(int* variant, float* ms) override {
    if (variant) *variant = c_variant;
    if (ms)
      for (int v = 0; v < kCVariants; ++v) ms[v] = c_ms[v];
    return PSG_OK;
  }
  int set_smem_limits() {
    switch (g.n) {
      case 16: return set_smem_limits_n<16>();
      case 32: return set_smem_limits_n<32>();
      case 64: return set_smem_limits_n<64>();
      case 128: return set_smem_limits_n<128>();
      default: return set_smem_limits_n<256>();
    }
  }

  int sync() override { return check_status(); }

  // device-side error flag (bounded waits); checked at every synchronisation
  int check_status() {
    int h = 0;
    PSG_CUDA_TRY(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h) {
      psg_set_error("a kernel gave up waiting for its tile copy (status 0x%x)", h);
      cudaMemsetAsync(d_status, 0, sizeof(int), stream);
      return PSG_ERR_CUDA;
    }
    return PSG_OK;
  }

  Fields4<T> stage_input() const {
    if (scheme == SCHEME_NS_HEUN || scheme == SCHEME_EULER_HEUN) return R.S;
    return R.X0;
  }

  // one right-hand-side evaluation followed by the stage update
  // pass A of the step's right-hand side, scalar or on packed transforms
  template <int N>
  int launch_a(bool chain, bool packed, Fields4<T> in, int mv) {
    constexpr int G = LineFFT<N, 1, T>::G;
    const int XT = g.XP / kTileW;
    const bool bous = (scheme == SCHEME_BOUS_RK4);
    if constexpr (sizeof(T) == 4) {
      if (packed && a_pk_ok) {
        if (bous)
          return launch_k(chain, pass_a_pk<N, 4, 9>, dim3(XT, g.Y), dim3(kTileW * G), smem_a_pk_n<N>(4),
                          g, in, B1, tw, mv, d_status);
        return launch_k(chain, pass_a_pk<N, 3, 6>, dim3(XT, g.Y), dim3(kTileW * G), smem_a_pk_n<N>(3), g,
                        in, B1, tw, mv, d_status);
      }
    }
    const Fields4<T> none{};
    if (bous)
      return launch_k(chain, pass_a<T, N, 4, 9, 0, 3>, dim3(XT, g.Y), dim3(3 * kTileW * G), smem_a(), g,
                      in, B1, tw, mv, d_status, none, 0);
    return launch_k(chain, pass_a<T, N, 3, 6>, dim3(XT, g.Y), dim3(2 * kTileW * G), smem_a(), g, in, B1,
                    tw, mv, d_status, none, 0);
  }

  // chain: the stream's last operation is the pass E of the previous
  // right-hand side (so that pass A may launch programmatically after it)
  template <int N>
  int rhs_n(int stage, bool want_dump, bool want_umax = false, bool chain = false) {
    using FG = LineFFT<N, 1, T>;
    const int G = FG::G;
    const dim3 blk(kTileW * G);
    const int XT = g.XP / kTileW;
    Fields4<T> in = stage_input();
    const int mv = first_rhs;
    first_rhs = 0;
    mark(-1);
    const dim3 blk2(2 * kTileW * G);
    int rc = launch_a<N>(chain, a_pk, in, mv);
    if (rc) return rc;
    mark(0);
    if ((rc = launch_k(true, pass_b<T, N>, dim3(XT, N, nfi), blk, smem_b(), g, B1, B2, tw, d_status)))
      return rc;
    mark(1);
    const T scale = (T)1 / ((T)N * (T)N * (T)N);
    T* dp = want_dump ? dump : nullptr;
    if (want_umax) PSG_CUDA_TRY(cudaMemsetAsync(d_umax, 0, sizeof(unsigned long long), stream));
    // after the memset the x-pass is an ordinary launch
    if ((rc = launch_c<N>(c_variant, scale, dp, 0, want_umax ? d_umax : nullptr,
                          !want_umax && pdl != 2)))
      return rc;
    mark(2);
    if ((rc = launch_k(true, pass_d<T, N>, dim3(XT, N, nfo), blk, smem_d(), g, B1, B2, tw, d_status)))
      return rc;
    mark(3);
    const dim3 ge(XT, g.Y);
    switch (scheme) {
      case SCHEME_NS_HEUN:
        rc = launch_k(true, pass_e<T, N, 3, SCHEME_NS_HEUN>, ge, blk2, smem_e(), g, B2, tw, R, prm,
                      stage, d_status);
        break;
      case SCHEME_EULER_HEUN:
        rc = launch_k(true, pass_e<T, N, 3, SCHEME_EULER_HEUN>, ge, blk2, smem_e(), g, B2, tw, R, prm,
                      stage, d_status);
        break;
      case SCHEME_NS_RK4:
        rc = launch_k(true, pass_e<T, N, 3, SCHEME_NS_RK4>, ge, blk2, smem_e(), g, B2, tw, R, prm,
                      stage, d_status);
        break;
      default:
        rc = launch_k(true, pass_e<T, N, 4, SCHEME_BOUS_RK4>, ge, blk2, smem_e(), g, B2, tw, R, prm,
                      stage, d_status);
    }
    if (rc) return rc;
    mark(4);
    launches += 5;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  int rhs(int stage, bool want_dump = false, bool want_umax = false, bool chain = false) {
    switch (g.n) {
      case 16: return rhs_n<16>(stage, want_dump, want_umax, chain);
      case 32: return rhs_n<32>(stage, want_dump, want_umax, chain);
      case 64: return rhs_n<64>(stage, want_dump, want_umax, chain);
      case 128: return rhs_n<128>(stage, want_dump, want_umax, chain);
      default: return rhs_n<256>(stage, want_dump, want_umax, chain);
    }
  }

  // one full time step of length dt; dump: keep the physical vorticity of the
  // predictor (Heun schemes).  chain: the previous step's last pass is the
  // stream's last operation (steps() back to back)
  int step(T dt, bool want_dump = false, bool chain = false) {
    prm.dt = dt;
    lin_dx = false;
    int rc;
    if (scheme == SCHEME_NS_HEUN || scheme == SCHEME_EULER_HEUN) {
      if ((rc = rhs(STAGE_HEUN_PRED, want_dump && (dump_mode & 1), false, chain))) return rc;
      return rhs(STAGE_HEUN_CORR, want_dump && !(dump_mode & 1), false, true);
    }
    if ((rc = rhs(STAGE_RK1, false, false, chain))) return rc;
    if ((rc = rhs(STAGE_RK2, false, false, true))) return rc;
    if ((rc = rhs(STAGE_RK3, false, false, true))) return rc;
    return rhs(STAGE_RK4, false, false, true);
  }

  // host FP64 boxes (reference layout) -> device state; RK4 schemes also set
  // the stage state X0 = S as the reference's setVelocity does.
  int upload(const double* const* comps) override {
    const long nref = (long)g.Y * g.Y * g.X;
    for (int q = 0; q < nc; ++q) {
      PSG_CUDA_TRY(cudaMemcpyAsync(stage_h, comps[q], sizeof(double2) * nref,
                                   cudaMemcpyHostToDevice, stream));
      box_from_ref<T><<<592, 256, 0, stream>>>(g, stage_h, R.S.c[q], R.SC.c[q]);
      ++launches;
    }
    if (R.X0.c[0]) {
      copy_fields<T><<<592, 256, 0, stream>>>(R.S, R.X0, nc, box);
      ++launches;
    }
    first_rhs = 1;
    lin_dx = false;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  int download(double* const* comps) override { return download_from(comps, nullptr); }

  // the kept modes only, read from / written to page-locked host memory by the
  // conversion kernels themselves (no staging copy; the other entries of the
  // host boxes are neither read nor written)
  static const void* host_mapped(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
  }
  int upload_kept(const double* const* comps) override {
    const void* dp[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < nc; ++q)
      if (!(dp[q] = host_mapped(comps[q]))) {
        psg_set_error("kept-mode upload needs page-locked host memory");
        return PSG_ERR_UNSUPPORTED;
      }
    for (int q = 0; q < nc; ++q) {
      box_from_ref_kept<T><<<592, 256, 0, stream>>>(g, (const double2*)dp[q], R.S.c[q], R.SC.c[q]);
      ++launches;
    }
    if (R.X0.c[0]) {
      copy_fields<T><<<592, 256, 0, stream>>>(R.S, R.X0, nc, box);
      ++launches;
    }
    first_rhs = 1;
    lin_dx = false;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }
  int download_kept(double* const* comps) override {
    void* dp[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < nc; ++q)
      if (!(dp[q] = (void*)host_mapped(comps[q]))) {
        psg_set_error("kept-mode download needs page-locked host memory");
        return PSG_ERR_UNSUPPORTED;
      }
    if (int rc = check_status()) return rc;
    for (int q = 0; q < nc; ++q) {
      box_to_ref_kept<T><<<592, 256, 0, stream>>>(g, R.S.c[q], (double2*)dp[q], R.SC.c[q]);
      ++launches;
    }
    PSG_CUDA_TRY(cudaGetLastError());
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }

  // device FP64 boxes (reference layout) <-> state, ordered on the engine's
  // stream, no host synchronisation
  int upload_device(const void* const* comps) override {
    for (int q = 0; q < nc; ++q) {
      box_from_ref<T><<<592, 256, 0, stream>>>(g, (const double2*)comps[q], R.S.c[q], R.SC.c[q]);
      ++launches;
    }
    if (R.X0.c[0]) {
      copy_fields<T><<<592, 256, 0, stream>>>(R.S, R.X0, nc, box);
      ++launches;
    }
    first_rhs = 1;
    lin_dx = false;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }
  int download_device(void* const* comps) override {
    for (int q = 0; q < nc; ++q) {
      box_to_ref<T><<<592, 256, 0, stream>>>(g, R.S.c[q], (double2*)comps[q], R.SC.c[q]);
      ++launches;
    }
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  // ---------------------------------------------------------------- linearised step
  // pass A: staged tile [ncin][Y][W], twiddles, ng exchange groups, 1/k^2 table
  // packed pass A: staged tile, twiddles, one exchange of 16-byte words with
  // pass_a_pk's row stride, 1/k^2 table
  template <int N>
  size_t smem_a_pk_n(int ncin) const {
    constexpr int S = LineFFT<N, 1, float>::SMEM;
    constexpr int SX = S + ((1 - S % 8) + 8) % 8;
    return sizeof(cpx<float>) * ((size_t)ncin * g.Y * kTileW + g.n) + 16 * (size_t)kTileW * SX +
           sizeof(float) * g.Y * kTileW;
  }
  size_t smem_a_nc(int ncin, int ng = 2) const {
    return sizeof(cpx<T>) * ((size_t)ncin * g.Y * kTileW + g.n + (size_t)ng * kTileW * col_stride()) +
           sizeof(T) * g.Y * kTileW;
  }
  // pass E: the NO input tiles, then (exchange inside the tiles) the overrun
  // of the last field's exchange, or a separate exchange area; twiddles; the
  // second transform group's exchange area
  size_t smem_e_no(int no) const {
    const long exw = (long)kTileW * col_stride(), tilew = (long)g.n * kTileW;
    const long over = exw > tilew ? exw - tilew : 0;
    const bool alias = over <= (long)(g.n - g.Y) * kTileW;
    const int tg = (no == 3) ? 2 : 1;  // transform groups (one exchange area each)
    return sizeof(cpx<T>) * ((size_t)no * tilew + g.n + (alias ? over + (tg - 1) * exw : tg * exw));
  }
  size_t smem_pair() const { return smem_a_nc(6); }

  template <int N>
  int lin_attrs() {
    int dev = 0, big = 0;
    PSG_CUDA_TRY(cudaGetDevice(&dev));
    PSG_CUDA_TRY(cudaDeviceGetAttribute(&big, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    big -= 1024;
    const bool bous = (scheme == SCHEME_BOUS_RK4);
    const size_t need = std::max(std::max(smem_pair(), smem_e_no(3)),
                                 bous ? std::max(smem_a_nc(5), smem_e_no(6)) : (size_t)0);
    if (need > (size_t)big) {
      psg_set_error("linearised step at grid %d needs %zu bytes of shared memory per block", g.n,
                    need);
      return PSG_ERR_UNSUPPORTED;
    }
    PSG_CUDA_TRY(cudaFuncSetAttribute(pass_a<T, N, 6, 6, 1>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    PSG_CUDA_TRY(cudaFuncSetAttribute(pass_e<T, N, 3, SCHEME_RAW>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    if (bous) {
      PSG_CUDA_TRY(cudaFuncSetAttribute(pass_a<T, N, 5, 7, 2>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, big));
      PSG_CUDA_TRY(cudaFuncSetAttribute(pass_e<T, N, 6, SCHEME_RAW>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, big));
      // the x-pass kernels of the adjoint's products (7 fields) got their
      // shared-memory limit with the engine's own (set_smem_limits_n)
    }
    return PSG_OK;
  }

  int lin_init() {
    if (lin) return PSG_OK;
    if (scheme != SCHEME_NS_RK4 && scheme != SCHEME_BOUS_RK4) {
      psg_set_error("tangent and adjoint steps are defined for the RK4/CN schemes");
      return PSG_ERR_UNSUPPORTED;
    }
    int rc;
    switch (g.n) {
      case 16: rc = lin_attrs<16>(); break;
      case 32: rc = lin_attrs<32>(); break;
      case 64: rc = lin_attrs<64>(); break;
      case 128: rc = lin_attrs<128>(); break;
      default: rc = lin_attrs<256>(); break;
    }
    if (rc) return rc;
    // state-shaped registers (nc components) and product outputs (3, or 4 + 2)
    constexpr int kState = 15;
    Fields4<T>* st[kState] = {&Zb[0], &Zb[1], &Zb[2], &Zb[3], &LA, &LN, &LS,
                              &LZ, &LK1, &LK2, &LK3, &LD, &LT, &LX, &LDX};
    const long words = ((long)kState * nc + 3 + 3 + (nc > 3 ? 6 : 0)) * box;
    PSG_CUDA_TRY(cudaMalloc(&lin, sizeof(cpx<T>) * words));
    PSG_CUDA_TRY(cudaMemsetAsync(lin, 0, sizeof(cpx<T>) * words, stream));
    cpx<T>* p = lin;
    auto carve = [&](Fields4<T>& f, int k) {
      for (int q = 0; q < 4; ++q) f.c[q] = nullptr;
      for (int q = 0; q < k; ++q) { f.c[q] = p; p += box; }
    };
    for (Fields4<T>* f : st) carve(*f, nc);
    carve(PA, 3);
    carve(PB, 3);
    if (nc > 3) { carve(SA, 4); carve(SB, 2); }
    return PSG_OK;
  }

  // out = P(a, b) = F(-(E(op_a a) x E(op_b b))), a in pass C's u slots, b in its w slots
  template <int N>
  int bilinear_n(Fields4<T> b, int op_b, Fields4<T> a, int op_a, Fields4<T> out) {
    using FG = LineFFT<N, 1, T>;
    const dim3 blk(kTileW * FG::G), blk2(2 * kTileW * FG::G);
    const int XT = g.XP / kTileW;
    pass_a<T, N, 6, 6, 1><<<dim3(XT, g.Y), blk2, smem_pair(), stream>>>(
        g, b, B1, tw, 0, d_status, a, op_b | (op_a << 4));
    pass_b<T, N><<<dim3(XT, N, 6), blk, smem_b(), stream>>>(g, B1, B2, tw, d_status);
    launch_c<N>(c_variant, (T)1 / ((T)N * (T)N * (T)N), nullptr, 6);
    pass_d<T, N><<<dim3(XT, N, 3), blk, smem_d(), stream>>>(g, B1, B2, tw, d_status);
    Regs<T> Rr{};
    Rr.K1 = out;
    pass_e<T, N, 3, SCHEME_RAW><<<dim3(XT, g.Y), blk2, smem_e_no(3), stream>>>(g, B2, tw, Rr, prm, 0,
                                                                          d_status);
    launches += 5;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }
  // SA, SB <- the Boussinesq adjoint's scalar products of psi = E(x_rho) with
  // E(i k z_rho) and E(B z_w)
  template <int N>
  int scale_products_n(Fields4<T> z, Fields4<T> x) {
    using FG = LineFFT<N, 1, T>;
    const dim3 blk(kTileW * FG::G), blk2(2 * kTileW * FG::G);
    const int XT = g.XP / kTileW;
    Fields4<T> psi{};
    psi.c[0] = x.c[3];
    pass_a<T, N, 5, 7, 2><<<dim3(XT, g.Y), blk2, smem_a_nc(5), stream>>>(g, z, B1, tw, 0, d_status,
                                                                         psi, 0);
    pass_b<T, N><<<dim3(XT, N, 7), blk, smem_b(), stream>>>(g, B1, B2, tw, d_status);
    launch_c<N>(c_variant, (T)1 / ((T)N * (T)N * (T)N), nullptr, 7);
    pass_d<T, N><<<dim3(XT, N, 6), blk, smem_d(), stream>>>(g, B1, B2, tw, d_status);
    Regs<T> Rr{};
    Rr.K1 = SA;
    Rr.K2 = SB;
    pass_e<T, N, 6, SCHEME_RAW><<<dim3(XT, g.Y), blk2, smem_e_no(6), stream>>>(g, B2, tw, Rr, prm, 0,
                                                                              d_status);
    launches += 5;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }
  int scale_products(Fields4<T> z, Fields4<T> x) {
    switch (g.n) {
      case 16: return scale_products_n<16>(z, x);
      case 32: return scale_products_n<32>(z, x);
      case 64: return scale_products_n<64>(z, x);
      case 128: return scale_products_n<128>(z, x);
      default: return scale_products_n<256>(z, x);
    }
  }

  double norm2(Fields4<T> x) {
    constexpr int kBlk = 296;
    if (!d_energ && cudaMalloc(&d_energ, sizeof(double) * (3 * kBlk + 3)) != cudaSuccess) return -1.0;
    lin_norm2<T><<<kBlk, 256, 0, stream>>>(x, box, nc, d_energ);
    ++launches;
    double h[kBlk];
    if (cudaMemcpyAsync(h, d_energ, sizeof(double) * kBlk, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return -1.0;
    double t = 0.0;
    for (int b = 0; b < kBlk; ++b) t += h[b];
    return t;
  }

  int bilinear(Fields4<T> b, int op_b, Fields4<T> a, int op_a, Fields4<T> out) {
    switch (g.n) {
      case 16: return bilinear_n<16>(b, op_b, a, op_a, out);
      case 32: return bilinear_n<32>(b, op_b, a, op_a, out);
      case 64: return bilinear_n<64>(b, op_b, a, op_a, out);
      case 128: return bilinear_n<128>(b, op_b, a, op_a, out);
      default: return bilinear_n<256>(b, op_b, a, op_a, out);
    }
  }

  // out = N'(z) x (tangent) or N'(z)^T x (adjoint)
  int lin_rhs(int adjoint, Fields4<T> z, Fields4<T> x, Fields4<T> out) {
    int rc;
    if (scheme == SCHEME_BOUS_RK4) return lin_rhs_bous(adjoint, z, x, out);
    if (!adjoint) {
      if ((rc = bilinear(z, OP_ID, x, OP_BS, PA))) return rc;  // F(-(E(B x) x E(z)))
      if ((rc = bilinear(x, OP_ID, z, OP_BS, PB))) return rc;  // F(-(E(B z) x E(x)))
    } else {
      if ((rc = bilinear(x, OP_CURL, z, OP_ID, PA))) return rc;  // F(-(E(z) x E(C x)))
      if ((rc = bilinear(z, OP_BS, x, OP_CURL, PB))) return rc;  // F(-(E(C x) x E(B z)))
    }
    lin_combine<T><<<592, 256, 0, stream>>>(g, adjoint, PA, PB, out, box);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  // Boussinesq: the tangent as the central difference of the engine's own
  // right-hand side (exact up to round-off: the terms are quadratic and
  // linear), D(z + s x) - D(z - s x) over 2 s with s = |z| / |x|; the adjoint
  // from the cross products and the scalar products, transposed by hand
  int lin_rhs_bous(int adjoint, Fields4<T> z, Fields4<T> x, Fields4<T> out) {
    int rc;
    if (!adjoint) {
      const double nx = norm2(x), nz = norm2(z);
      if (nx < 0.0 || nz < 0.0) { psg_set_error("norm reduction failed"); return PSG_ERR_CUDA; }
      if (nx == 0.0) {
        lin_axpby<T><<<592, 256, 0, stream>>>(out, (T)0, (T)0, x, box, nc);
        ++launches;
        return PSG_OK;
      }
      const T sc = (T)(nz > 0.0 ? sqrt(nz / nx) : 1.0);
      const int saved_first = first_rhs;
      first_rhs = 0;
      copy_fields<T><<<592, 256, 0, stream>>>(R.X0, LX, nc, box);
      lin_shift<T><<<592, 256, 0, stream>>>(R.X0, z, sc, x, box, nc);
      ++launches;
      if ((rc = rhs(STAGE_DERIV))) return rc;
      copy_fields<T><<<592, 256, 0, stream>>>(R.K1, LT, nc, box);
      lin_shift<T><<<592, 256, 0, stream>>>(R.X0, z, -sc, x, box, nc);
      launches += 2;
      if ((rc = rhs(STAGE_DERIV))) return rc;
      first_rhs = saved_first;
      copy_fields<T><<<592, 256, 0, stream>>>(LT, out, nc, box);
      lin_axpby<T><<<592, 256, 0, stream>>>(out, (T)(0.5) / sc, (T)(-0.5) / sc, R.K1, box, nc);
      copy_fields<T><<<592, 256, 0, stream>>>(LX, R.X0, nc, box);
      launches += 4;
      PSG_CUDA_TRY(cudaGetLastError());
      return PSG_OK;
    }
    if ((rc = bilinear(x, OP_CURL, z, OP_ID, PA))) return rc;  // F(-(E(z) x E(C x)))
    if ((rc = bilinear(z, OP_BS, x, OP_CURL, PB))) return rc;  // F(-(E(C x) x E(B z)))
    if ((rc = scale_products(z, x))) return rc;
    bous_adj_combine<T><<<592, 256, 0, stream>>>(g, prm.ri, prm.sinth, prm.costh, PA, PB, SA, SB,
                                                 x, out, box);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  // one forward step from S with X0 = S, keeping the four stage states
  // the base step as step() takes it: from the stage input X0 (the state after
  // an upload, the previous step's final stage before its divergence removal
  // otherwise), stage inputs kept in Zb; afterwards S and X0 are what step()
  // leaves
  int base_stages(T dt) {
    prm.dt = dt;
    copy_fields<T><<<592, 256, 0, stream>>>(R.X0, Zb[0], nc, box);
    launches += 1;
    const int stg[3] = {STAGE_RK1, STAGE_RK2, STAGE_RK3};
    for (int s = 0; s < 3; ++s) {
      if (int rc = rhs(stg[s])) return rc;
      copy_fields<T><<<592, 256, 0, stream>>>(R.X0, Zb[s + 1], nc, box);
      ++launches;
    }
    return rhs(STAGE_RK4);
  }

  // (D, DX) <- the tangent of one step at (S, X0) applied to the tangent D of
  // the state and DX of the stage input; S, X0 <- the step.  DXout receives the
  // tangent of the new stage input (may alias DX, read only by the first
  // stage).
  int tangent_step_t(T dt, Fields4<T> D, Fields4<T> DX, Fields4<T> DXout) {
    int rc;
    if ((rc = base_stages(dt))) return rc;
    const T nu = prm.nu;
    const T qs[3] = {(T)0.25, (T)0.25, (T)0.5}, frs[3] = {(T)0.5, (T)0.5, (T)1};
    Fields4<T> Ks[3] = {LK1, LK2, LK3};
    Fields4<T> in = DX;
    const T sc = prm.sc;
    for (int s = 0; s < 3; ++s) {
      if ((rc = lin_rhs(0, Zb[s], in, LN))) return rc;
      tan_stage<T><<<592, 256, 0, stream>>>(g, dt, nu, qs[s], frs[s], LN, D, Ks[s], LA, box, nc, sc);
      ++launches;
      in = LA;
    }
    if ((rc = lin_rhs(0, Zb[3], LA, LN))) return rc;
    tan_final<T><<<592, 256, 0, stream>>>(g, dt, nu, LN, LK1, LK2, LK3, D, DXout, box, nc, sc);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  // L <- dPhi(S)^T L, S <- Phi(S)
  int adjoint_step_t(T dt, Fields4<T> L) {
    int rc;
    if ((rc = base_stages(dt))) return rc;
    const T nu = prm.nu;
    const T sc = prm.sc;
    adj_final<T><<<592, 256, 0, stream>>>(g, dt, nu, L, LZ, LK1, LK2, LK3, LN, box, nc, sc);
    ++launches;
    const T qs[3] = {(T)0.5, (T)0.25, (T)0.25}, frs[3] = {(T)1, (T)0.5, (T)0.5};
    Fields4<T> Ks[3] = {LK3, LK2, LK1};
    for (int s = 0; s < 3; ++s) {
      if ((rc = lin_rhs(1, Zb[3 - s], LN, LS))) return rc;
      adj_stage<T><<<592, 256, 0, stream>>>(g, dt, nu, qs[s], frs[s], LS, LZ, Ks[s], LN, box, nc, sc);
      ++launches;
    }
    if ((rc = lin_rhs(1, Zb[0], LN, LS))) return rc;
    lin_axpby<T><<<592, 256, 0, stream>>>(LZ, (T)1, (T)1, LS, box, nc);
    copy_fields<T><<<592, 256, 0, stream>>>(LZ, L, nc, box);
    launches += 2;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  // mode 0: tangent step, 1: adjoint step, 2: tangent right-hand side N'(S) x,
  // 3: adjoint right-hand side N'(S)^T x.  in / out: device FP64 boxes in the
  // reference layout (3 components), ordered on the engine's stream.
  int linear(int mode, double dt, const void* const* in, void* const* out) override {
    int rc;
    if ((rc = lin_init())) return rc;
    for (int q = 0; q < nc; ++q)
      box_from_ref<T><<<592, 256, 0, stream>>>(g, (const double2*)in[q], LD.c[q], nullptr);
    launches += nc;
    Fields4<T> res = LD;
    switch (mode) {
      case 0:
        // a tangent step that follows another on the same trajectory starts
        // from the previous one's stage-input tangent; after an upload or a
        // plain step, from the state's
        rc = tangent_step_t((T)dt, LD, lin_dx ? LDX : LD, LDX);
        lin_dx = true;
        break;
      case 1: rc = adjoint_step_t((T)dt, LD); lin_dx = false; break;
      case 2: rc = lin_rhs(0, R.S, LD, LS); res = LS; break;
      case 3: rc = lin_rhs(1, R.S, LD, LS); res = LS; break;
      default: psg_set_error("linear mode %d unknown", mode); return PSG_ERR_ARG;
    }
    if (rc) return rc;
    for (int q = 0; q < nc; ++q)
      box_to_ref<T><<<592, 256, 0, stream>>>(g, res.c[q], (double2*)out[q], nullptr);
    launches += nc;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  int set_forcing_form(int form) override {
    if (form != 0 && form != 1) { psg_set_error("forcing form %d unknown", form); return PSG_ERR_ARG; }
    prm.fform = form;
    return PSG_OK;
  }

  int energetics(double* out) override {
    constexpr int kBlk = 296;
    if (!d_energ) PSG_CUDA_TRY(cudaMalloc(&d_energ, sizeof(double) * (3 * kBlk + 3)));
    energetics_partial<T><<<kBlk, 256, 0, stream>>>(g, R.S, nc, d_energ);
    energetics_final<<<1, 32, 0, stream>>>(d_energ, kBlk, d_energ + 3 * kBlk);
    launches += 2;
    PSG_CUDA_TRY(cudaGetLastError());
    PSG_CUDA_TRY(cudaMemcpyAsync(out, d_energ + 3 * kBlk, sizeof(double) * 3,
                                 cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return check_status();
  }
  // max |u| over the grid of the physical x-velocity of the state the next
  // step starts from (its first right-hand side's input); the evaluation
  // leaves the state, the stage registers a step uses and the first-step
  // velocity masking as they were
  int max_velocity(double* out) override {
    if (scheme != SCHEME_BOUS_RK4 && scheme != SCHEME_NS_RK4) {
      psg_set_error("max velocity is provided for the RK4 schemes");
      return PSG_ERR_UNSUPPORTED;
    }
    if (!d_umax) PSG_CUDA_TRY(cudaMalloc(&d_umax, sizeof(unsigned long long)));
    const int keep = first_rhs;
    int rc = rhs(STAGE_DERIV, false, true);
    first_rhs = keep;
    if (rc) return rc;
    unsigned long long bits = 0;
    PSG_CUDA_TRY(cudaMemcpyAsync(&bits, d_umax, sizeof bits, cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    memcpy(out, &bits, sizeof(double));
    return check_status();
  }

  // Boussinesq fluxes of the state, FP64 sums over the kept modes as the DNS's
  // computeStats forms them (3D_Boussinesq/src/functions.h:288-362):
  // out[0] = sum Re(conj(b) rho), b = v sin(theta) + w cos(theta) with the
  // spectral velocity (v, w) = (i k x w / max(k^2, 0.001))_{y,z};
  // out[1] = Re zeta at (kx, ky, kz) = (0, kf, 0) (0 when that mode is not kept)
  int buoyancy_flux(double* out) override {
    if (scheme != SCHEME_BOUS_RK4) {
      psg_set_error("buoyancy flux is defined for the Boussinesq scheme");
      return PSG_ERR_UNSUPPORTED;
    }
    constexpr int kBlk = 296;
    if (!d_flux) PSG_CUDA_TRY(cudaMalloc(&d_flux, sizeof(double) * (2 * kBlk + 2)));
    bflux_partial<T><<<kBlk, 256, 0, stream>>>(g, R.S, (double)prm.sinth, (double)prm.costh,
                                                (double)prm.kf, d_flux);
    bflux_final<<<1, 32, 0, stream>>>(d_flux, kBlk, d_flux + 2 * kBlk);
    launches += 2;
    PSG_CUDA_TRY(cudaGetLastError());
    PSG_CUDA_TRY(cudaMemcpyAsync(out, d_flux + 2 * kBlk, sizeof(double) * 2,
                                 cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return check_status();
  }

  int download_stage(double* const* comps) override {
    if (!R.X0.c[0]) { psg_set_error("scheme keeps no stage state"); return PSG_ERR_STATE; }
    return download_from(comps, &R.X0);
  }
  int timederiv(double* const* out) override {
    if (scheme != SCHEME_BOUS_RK4 && scheme != SCHEME_NS_RK4) {
      psg_set_error("time derivative is defined for the RK4 schemes");
      return PSG_ERR_UNSUPPORTED;
    }
    int rc = rhs(STAGE_DERIV);
    if (rc) return rc;
    return download_from(out, &R.K1);
  }
  int set_params(double nu, double ampfor, double kf, double ri, double sc, double theta) override {
    prm.nu = (T)nu; prm.ampfor = (T)ampfor; prm.kf = (T)kf; prm.ri = (T)ri; prm.sc = (T)sc;
    prm.sinth = (T)sin(theta); prm.costh = (T)cos(theta);
    return PSG_OK;
  }
  void set_stream(cudaStream_t s) override { stream = s; }
  cudaStream_t get_stream() const override { return stream; }
  long launch_count() const override { return launches; }
  int steps(double dt, int nsteps, int dump_last) override {
    for (int s = 0; s < nsteps; ++s) {
      int rc = step((T)dt, dump_last && s == nsteps - 1, s > 0);
      if (rc) return rc;
    }
    return PSG_OK;
  }
  int layout(int* xp, void** comps) override {
    if (xp) *xp = g.XP;
    if (comps)
      for (int q = 0; q < 4; ++q) comps[q] = (void*)R.S.c[q];
    return PSG_OK;
  }
  int phys(double* const* out) override {
    if (!dump) { psg_set_error("scheme keeps no physical fields"); return PSG_ERR_STATE; }
    return download_phys(out);
  }
  int set_dump_mode(int mode) override {
    if (!dump) { psg_set_error("scheme keeps no physical fields"); return PSG_ERR_STATE; }
    if (mode < 0 || mode > 3) { psg_set_error("dump mode %d unknown", mode); return PSG_ERR_ARG; }
    if ((mode & 2) && !(dump_mode & 2)) {
      cudaFree(dump);
      dump = nullptr;
      PSG_CUDA_TRY(cudaMalloc(&dump, sizeof(T) * 6L * g.n * g.n * g.n));
    }
    dump_mode = mode;
    return PSG_OK;
  }
  int phys_velocity(double* const* out) override {
    if (!dump || !(dump_mode & 2)) {
      psg_set_error("the velocity is kept in dump mode 2 or 3");
      return PSG_ERR_STATE;
    }
    const long nr = (long)g.n * g.n * g.n;
    T* keep = dump;
    dump = keep + 3 * nr;
    const int rc = download_phys(out);
    dump = keep;
    return rc;
  }
  // running mean squares of the kept velocity: rms = (rms count + u^2)/(count + 1)
  int rms_accumulate(double count) override {
    if (!dump || !(dump_mode & 2)) {
      psg_set_error("the velocity is kept in dump mode 2 or 3");
      return PSG_ERR_STATE;
    }
    const long nr = (long)g.n * g.n * g.n;
    if (!d_rms) {
      PSG_CUDA_TRY(cudaMalloc(&d_rms, sizeof(double) * 3 * nr));
      PSG_CUDA_TRY(cudaMemsetAsync(d_rms, 0, sizeof(double) * 3 * nr, stream));
    }
    rms_acc<T><<<592, 256, 0, stream>>>(dump + 3 * nr, d_rms, 3 * nr, count);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }
  int rms_download(double* const* out) override {
    if (!d_rms) { psg_set_error("no mean squares accumulated"); return PSG_ERR_STATE; }
    const long nr = (long)g.n * g.n * g.n;
    for (int q = 0; q < 3; ++q)
      PSG_CUDA_TRY(cudaMemcpyAsync(out[q], d_rms + q * nr, sizeof(double) * nr,
                                   cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return check_status();
  }
  int download_from(double* const* comps, const Fields4<T>* src) {
    if (int rc = check_status()) return rc;
    const long nref = (long)g.Y * g.Y * g.X;
    const Fields4<T>& F = src ? *src : R.S;
    for (int q = 0; q < nc; ++q) {
      box_to_ref<T><<<592, 256, 0, stream>>>(g, F.c[q], stage_h, src ? nullptr : R.SC.c[q]);
      ++launches;
      PSG_CUDA_TRY(cudaMemcpyAsync(comps[q], stage_h, sizeof(double2) * nref,
                                   cudaMemcpyDeviceToHost, stream));
    }
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }

  int download_phys(double* const* out) {
    const long nr = (long)g.n * g.n * g.n;
    double* tmp = nullptr;
    PSG_CUDA_TRY(cudaMalloc(&tmp, sizeof(double) * nr));
    for (int q = 0; q < 3; ++q) {
      real_to_double<T><<<592, 256, 0, stream>>>(dump + q * nr, tmp, nr);
      ++launches;
      cudaError_t e = cudaMemcpyAsync(out[q], tmp, sizeof(double) * nr, cudaMemcpyDeviceToHost, stream);
      if (e != cudaSuccess) { cudaFree(tmp); PSG_CUDA_TRY(e); }
    }
    cudaError_t e = cudaStreamSynchronize(stream);
    cudaFree(tmp);
    PSG_CUDA_TRY(e);
    return PSG_OK;
  }
};

}  // namespace psg

