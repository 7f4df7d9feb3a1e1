// psg_fft2.cuh -- two FP32 line transforms at once on Blackwell's packed
// f32x2 arithmetic (add/sub/mul/fma.rn.f32x2, sm_100a).
//
// A `Pk` holds the same element of two lines side by side: re = (a.re, b.re),
// im = (a.im, b.im).  Both lines go through the identical butterfly network
// and twiddles, so every complex operation of LineFFT<N, SIGN, float> becomes
// one packed instruction per component for the two lines together.  The
// trivial factor +-i folds into the butterfly's subtraction (operands swapped,
// no instruction); the decomposition, register distribution and exchange
// layout are LineFFT's, so a packed transform can replace two scalar ones
// wherever their inputs and outputs sit in the same registers.
#pragma once

#include "psg_fft.cuh"

namespace psg {

struct Pk {
  float2 re, im;
};

__device__ __forceinline__ unsigned long long p_in(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 p_out(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(p_in(a)), "l"(p_in(b)));
  return p_out(d);
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(p_in(a)), "l"(p_in(b)));
  return p_out(d);
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(p_in(a)), "l"(p_in(b)));
  return p_out(d);
}
// a * b + c
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(p_in(a)), "l"(p_in(b)), "l"(p_in(c)));
  return p_out(d);
}
__device__ __forceinline__ float2 psplat(float c) { return make_float2(c, c); }

// d * w for w = (c, s): re = d.re c - d.im s, im = d.re s + d.im c
__device__ __forceinline__ Pk pcmul(Pk d, float c, float s) {
  return Pk{pfma(d.im, psplat(-s), pmul(d.re, psplat(c))), pfma(d.re, psplat(s), pmul(d.im, psplat(c)))};
}

// (a - b) * exp(SIGN * 2 pi i m / 32), 0 <= m < 16
template <int SIGN>
__device__ __forceinline__ Pk pdiff_tw32(Pk a, Pk b, int m) {
  if (m == 0) return Pk{psub(a.re, b.re), psub(a.im, b.im)};
  if (m == 8) {
    // SIGN * i (a - b)
    return SIGN < 0 ? Pk{psub(a.im, b.im), psub(b.re, a.re)} : Pk{psub(b.im, a.im), psub(a.re, b.re)};
  }
  const Pk d{psub(a.re, b.re), psub(a.im, b.im)};
  return pcmul(d, Omega32<float>::c(m), (float)SIGN * Omega32<float>::s(m));
}

// packed counterpart of dft<R, SIGN, float>: the same butterflies and output order
template <int R, int SIGN>
__device__ __forceinline__ void pdft(Pk (&v)[R]) {
  static_assert(R == 1 || R == 2 || R == 4 || R == 8 || R == 16 || R == 32, "radix");
#pragma unroll
  for (int len = R; len >= 2; len >>= 1) {
    const int half = len >> 1;
#pragma unroll
    for (int s = 0; s < R; s += len) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        const Pk a = v[s + j], b = v[s + j + half];
        v[s + j] = Pk{padd(a.re, b.re), padd(a.im, b.im)};
        v[s + j + half] = pdiff_tw32<SIGN>(a, b, j * (32 / len));
      }
    }
  }
  Pk t[R];
#pragma unroll
  for (int i = 0; i < R; ++i) t[i] = v[i];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    int r = 0;
#pragma unroll
    for (int b = 1, q = R >> 1; b < R; b <<= 1, q >>= 1)
      if (i & b) r |= q;
    v[r] = t[i];
  }
}

// Two lines through LineFFT<N, SIGN, float, SWAP>'s plan at once.  tw: that
// plan's table (N entries (cos, sin) of exp(-2 pi i n1 k2 / N)); ex: SMEM
// entries of 16 bytes (the two lines' complex values side by side).
template <int N, int SIGN, bool SWAP = false>
struct LineFFT2 {
  using P = LineFFT<N, SIGN, float, SWAP>;
  static constexpr int R1 = P::R1, R2 = P::R2, G = P::G, E = P::E, A = P::A, B = P::B;
  static constexpr int SMEM = P::SMEM;

  template <typename Sync>
  static __device__ __forceinline__ void run(Pk (&v)[E], int g, const cpx<float>* tw, float4* ex,
                                             Sync sync) {
#pragma unroll
    for (int a = 0; a < A; ++a) {
      Pk w[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = v[a * R2 + n2];
      pdft<R2, SIGN>(w);
      const int n1 = g + G * a;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const cpx<float> t = tw[k2 * R1 + n1];
        const Pk x = (k2 == 0) ? w[k2] : pcmul(w[k2], t.x, SIGN > 0 ? -t.y : t.y);
        ex[k2 * (R1 + 1) + n1] = make_float4(x.re.x, x.re.y, x.im.x, x.im.y);
      }
    }
    sync();
#pragma unroll
    for (int b = 0; b < B; ++b) {
      Pk w[R1];
      const int k2 = g + G * b;
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) {
        const float4 q = ex[k2 * (R1 + 1) + n1];
        w[n1] = Pk{make_float2(q.x, q.y), make_float2(q.z, q.w)};
      }
      pdft<R1, SIGN>(w);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) v[b * R1 + k1] = w[k1];
    }
    sync();
  }

  // The same transform with an exchange buffer of 8-byte entries (SMEM of
  // them, the size a scalar transform uses): the real and the imaginary
  // parts cross it one after the other.
  template <typename Sync>
  static __device__ __forceinline__ void run(Pk (&v)[E], int g, const cpx<float>* tw, float2* ex,
                                             Sync sync) {
#pragma unroll
    for (int a = 0; a < A; ++a) {
      Pk w[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = v[a * R2 + n2];
      pdft<R2, SIGN>(w);
      const int n1 = g + G * a;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const cpx<float> t = tw[k2 * R1 + n1];
        v[a * R2 + k2] = (k2 == 0) ? w[k2] : pcmul(w[k2], t.x, SIGN > 0 ? -t.y : t.y);
      }
    }
#pragma unroll
    for (int part = 0; part < 2; ++part) {
#pragma unroll
      for (int a = 0; a < A; ++a) {
        const int n1 = g + G * a;
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2)
          ex[k2 * (R1 + 1) + n1] = part == 0 ? v[a * R2 + k2].re : v[a * R2 + k2].im;
      }
      sync();
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int k2 = g + G * b;
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) {
          if (part == 0) v[b * R1 + n1].re = ex[k2 * (R1 + 1) + n1];
          else v[b * R1 + n1].im = ex[k2 * (R1 + 1) + n1];
        }
      }
      sync();
    }
#pragma unroll
    for (int b = 0; b < B; ++b) {
      Pk w[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) w[n1] = v[b * R1 + n1];
      pdft<R1, SIGN>(w);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) v[b * R1 + k1] = w[k1];
    }
  }
};

}  // namespace psg
