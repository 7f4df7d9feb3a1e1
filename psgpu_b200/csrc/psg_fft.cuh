// psg_fft.cuh -- register/shared-memory FFT building blocks for sm_100a.
//
// A line of N = R1*R2 points is transformed by G = min(R1,R2) cooperating
// threads with the four-step decomposition
//   n = n1 + R1*n2,  k = k2 + R2*k1,
//   X[k2 + R2 k1] = sum_n1 w_R1^{n1 k1} [ w_N^{n1 k2} sum_n2 x[n1 + R1 n2] w_R2^{n2 k2} ].
// Step 1 (R2-point DFTs) and step 2 (R1-point DFTs) run in registers; the
// only data exchange is one padded shared-memory transpose between them.
// Thread g of a line holds, on input, x[g + G*a + R1*n2] (a < R1/G, n2 < R2)
// and, on output, X[g + G*b + R2*k1] (b < R2/G, k1 < R1).
//
// Sign convention: SIGN = -1 is the forward transform (e^{-i}), SIGN = +1 the
// unnormalised inverse, matching cuFFT's D2Z / Z2D pair.
#pragma once
#include <math.h>

#include "psg_common.cuh"

namespace psg {

// cos / sin of 2*pi*m/32, m = 0..15 (exact decimal expansions of the constants)
template <typename T>
struct Omega32 {
  static __device__ __forceinline__ T c(int m) {
    constexpr double tab[16] = {
        1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
        0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
        0.19509032201612826785, 0.0, -0.19509032201612826785, -0.38268343236508977173,
        -0.55557023301960222474, -0.70710678118654752440, -0.83146961230254523708,
        -0.92387953251128675613, -0.98078528040323044913};
    return (T)tab[m];
  }
  static __device__ __forceinline__ T s(int m) {
    constexpr double tab[16] = {
        0.0, 0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
        0.70710678118654752440, 0.83146961230254523708, 0.92387953251128675613,
        0.98078528040323044913, 1.0, 0.98078528040323044913, 0.92387953251128675613,
        0.83146961230254523708, 0.70710678118654752440, 0.55557023301960222474,
        0.38268343236508977173, 0.19509032201612826785};
    return (T)tab[m];
  }
};

// multiply c by w_32^{m} = exp(SIGN * 2 pi i m / 32), 0 <= m < 16; trivial
// factors are folded once the caller's loops are unrolled.
template <int SIGN, typename T>
__device__ __forceinline__ cpx<T> tw32(cpx<T> c, int m) {
  if (m == 0) return c;
  if (m == 8) {  // exp(SIGN * i pi/2) = SIGN * i
    return SIGN < 0 ? cpx<T>{c.y, -c.x} : cpx<T>{-c.y, c.x};
  }
  const T wr = Omega32<T>::c(m);
  const T wi = (T)SIGN * Omega32<T>::s(m);
  return cpx<T>{c.x * wr - c.y * wi, c.x * wi + c.y * wr};
}

// In-register R-point DFT (R = 2,4,8,16,32), radix-2 decimation in frequency
// followed by a compile-time bit-reversal permutation.
template <int R, int SIGN, typename T>
__device__ __forceinline__ void dft(cpx<T> (&v)[R]) {
  static_assert(R == 1 || R == 2 || R == 4 || R == 8 || R == 16 || R == 32, "radix");
#pragma unroll
  for (int len = R; len >= 2; len >>= 1) {
    const int half = len >> 1;
#pragma unroll
    for (int s = 0; s < R; s += len) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        cpx<T> a = v[s + j], b = v[s + j + half];
        v[s + j] = cpx<T>{a.x + b.x, a.y + b.y};
        v[s + j + half] = tw32<SIGN>(cpx<T>{a.x - b.x, a.y - b.y}, j * (32 / len));
      }
    }
  }
  // undo the bit reversal
  cpx<T> t[R];
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

// Factorisation of a line length.
template <int N>
struct Plan;
template <> struct Plan<16>  { static constexpr int R1 = 4,  R2 = 4;  };
template <> struct Plan<32>  { static constexpr int R1 = 8,  R2 = 4;  };
template <> struct Plan<64>  { static constexpr int R1 = 8,  R2 = 8;  };
template <> struct Plan<128> { static constexpr int R1 = 16, R2 = 8;  };
template <> struct Plan<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Plan<512> { static constexpr int R1 = 32, R2 = 16; };

// SWAP exchanges the two radices.  The output distribution of a plan is the
// input distribution of its swapped plan, so a transform that consumes the
// registers another transform produced (the x-pass: C2R -> product -> R2C)
// must use the swapped factorisation.
template <int N, int SIGN, typename T, bool SWAP = false>
struct LineFFT {
  static constexpr int R1 = SWAP ? Plan<N>::R2 : Plan<N>::R1;
  static constexpr int R2 = SWAP ? Plan<N>::R1 : Plan<N>::R2;
  static constexpr int G = R1 < R2 ? R1 : R2;   // threads per line
  static constexpr int E = N / G;               // elements per thread
  static constexpr int A = R1 / G;              // step-1 DFTs per thread
  static constexpr int B = R2 / G;              // step-2 DFTs per thread
  // complex words of exchange space per line, enough for either orientation
  static constexpr int SMEM = (R2 * (R1 + 1) > R1 * (R2 + 1)) ? R2 * (R1 + 1) : R1 * (R2 + 1);

  // input position of register e (e = a*R2 + n2) for thread g
  static __device__ __forceinline__ int in_index(int g, int e) {
    const int a = e / R2, n2 = e % R2;
    return g + G * a + R1 * n2;
  }
  // output frequency of register e (e = b*R1 + k1) for thread g
  static __device__ __forceinline__ int out_index(int g, int e) {
    const int b = e / R1, k1 = e % R1;
    return g + G * b + R2 * k1;
  }

  // Twiddle table of this plan: TW[k2 * R1 + n1] = exp(-2 pi i n1 k2 / N), so
  // that the R1 threads of a step-1 read for one k2 hit consecutive words.
  static void host_table(cpx<T>* out) {
    for (int k2 = 0; k2 < R2; ++k2)
      for (int n1 = 0; n1 < R1; ++n1) {
        const double a = -2.0 * 3.14159265358979323846 * (double)(n1 * k2) / (double)N;
        out[k2 * R1 + n1] = cpx<T>{(T)cos(a), (T)sin(a)};
      }
  }

  // Full transform.  tw: this plan's table (host_table layout, N entries).
  // ex: this line's exchange buffer (SMEM complex words).  SYNC is a
  // callable that synchronises every thread that shares `ex` between the
  // shared-memory write and read (a warp or the whole block).
  template <typename Sync>
  static __device__ __forceinline__ void run(cpx<T> (&v)[E], int g, const cpx<T>* tw,
                                             cpx<T>* ex, Sync sync) {
    // step 1: A DFTs of size R2
#pragma unroll
    for (int a = 0; a < A; ++a) {
      cpx<T> w[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = v[a * R2 + n2];
      dft<R2, SIGN>(w);
      const int n1 = g + G * a;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        cpx<T> t = tw[k2 * R1 + n1];
        if (SIGN > 0) t.y = -t.y;
        ex[k2 * (R1 + 1) + n1] = cmul(w[k2], t);
      }
    }
    sync();
#pragma unroll
    for (int b = 0; b < B; ++b) {
      cpx<T> w[R1];
      const int k2 = g + G * b;
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) w[n1] = ex[k2 * (R1 + 1) + n1];
      dft<R1, SIGN>(w);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) v[b * R1 + k1] = w[k1];
    }
    sync();  // `ex` may be rewritten by the next call
  }
};

}  // namespace psg
