// psg_api.cu -- error reporting and library information of the C API.
#include <stdarg.h>
#include <stdio.h>
#include <math.h>
#include <string.h>

#include "psg_common.cuh"
#include "psgpu_internal.h"

static thread_local char g_err[1024];

extern "C" void psg_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

extern "C" const char* psg_last_error(void) { return g_err; }

extern "C" void psg_clear_error(void) { g_err[0] = 0; }

extern "C" int psg_version(void) { return PSG_VERSION; }

// ---------------------------------------------------------------------------
// building-block check: the line FFT of psg_fft.cuh applied to `nlines`
// contiguous lines of n complex doubles (one warp-level thread group per
// line).  Used by the unit tests; unnormalised, sign -1 forward / +1 inverse.
// ---------------------------------------------------------------------------
#include "psg_fft.cuh"
#include "psg_tma.cuh"

namespace {
template <int N, int SIGN, bool SWAP>
__global__ void linefft_kernel(const psg::cpx<double>* in, psg::cpx<double>* out,
                               const psg::cpx<double>* tw, int nlines) {
  using F = psg::LineFFT<N, SIGN, double, SWAP>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  psg::cpx<double>* s_tw = reinterpret_cast<psg::cpx<double>*>(smem_raw);
  psg::cpx<double>* s_ex = s_tw + N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s_tw[i] = tw[i];
  __syncthreads();
  const int gpb = blockDim.x / F::G;
  const int grp = threadIdx.x / F::G, g = threadIdx.x % F::G;
  const int line = blockIdx.x * gpb + grp;
  const bool live = line < nlines;
  psg::cpx<double> v[F::E];
#pragma unroll
  for (int e = 0; e < F::E; ++e)
    v[e] = live ? in[(long)line * N + F::in_index(g, e)] : psg::czero<double>();
  F::run(v, g, s_tw, s_ex + grp * F::SMEM, psg::WarpSync());
  if (live) {
#pragma unroll
    for (int e = 0; e < F::E; ++e) out[(long)line * N + F::out_index(g, e)] = v[e];
  }
}

template <int N, int SIGN, bool SWAP>
int launch_linefft(const double* in, double* out, int nlines) {
  using F = psg::LineFFT<N, SIGN, double, SWAP>;
  const long len = (long)nlines * N;
  psg::cpx<double>*d_in = nullptr, *d_out = nullptr, *d_tw = nullptr;
  psg::cpx<double> h_tw[N];
  F::host_table(h_tw);
  int rc = PSG_OK;
  const int threads = 128;
  const int gpb = threads / F::G;
  const size_t smem = sizeof(psg::cpx<double>) * (N + gpb * F::SMEM);
  if (cudaMalloc(&d_in, sizeof(psg::cpx<double>) * len) != cudaSuccess ||
      cudaMalloc(&d_out, sizeof(psg::cpx<double>) * len) != cudaSuccess ||
      cudaMalloc(&d_tw, sizeof(psg::cpx<double>) * N) != cudaSuccess) {
    psg_set_error("cudaMalloc failed");
    rc = PSG_ERR_CUDA;
  }
  if (rc == PSG_OK) {
    cudaMemcpy(d_in, in, sizeof(psg::cpx<double>) * len, cudaMemcpyHostToDevice);
    cudaMemcpy(d_tw, h_tw, sizeof(psg::cpx<double>) * N, cudaMemcpyHostToDevice);
    cudaFuncSetAttribute(linefft_kernel<N, SIGN, SWAP>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    linefft_kernel<N, SIGN, SWAP><<<(nlines + gpb - 1) / gpb, threads, smem>>>(d_in, d_out, d_tw, nlines);
    cudaError_t e = cudaMemcpy(out, d_out, sizeof(psg::cpx<double>) * len, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { psg_set_error("%s", cudaGetErrorString(e)); rc = PSG_ERR_CUDA; }
  }
  cudaFree(d_in); cudaFree(d_out); cudaFree(d_tw);
  return rc;
}
}  // namespace

extern "C" int psg_debug_linefft(int n, int sign, int swap, const double* in, double* out,
                                 int nlines) {
  if (!in || !out || nlines <= 0 || (sign != 1 && sign != -1)) {
    psg_set_error("bad arguments");
    return PSG_ERR_ARG;
  }
#define PSG_LF(NN)                                                                   \
  case NN:                                                                           \
    if (swap)                                                                        \
      return sign < 0 ? launch_linefft<NN, -1, true>(in, out, nlines)                \
                      : launch_linefft<NN, 1, true>(in, out, nlines);                \
    return sign < 0 ? launch_linefft<NN, -1, false>(in, out, nlines)                 \
                    : launch_linefft<NN, 1, false>(in, out, nlines);
  switch (n) {
    PSG_LF(16) PSG_LF(32) PSG_LF(64) PSG_LF(128) PSG_LF(256) PSG_LF(512)
    default:
      psg_set_error("line length %d unsupported", n);
      return PSG_ERR_UNSUPPORTED;
  }
#undef PSG_LF
}

// ---------------------------------------------------------------------------
// The bounded-wait path, exercised: a block arms an mbarrier for a transfer
// that is never issued and waits `polls` times; the wait runs out, the kernel
// records PSG_DEV_TIMEOUT in the status word and returns (no copy is in flight,
// so nothing outlives the block).  The host reads the status as the engines do.
// ---------------------------------------------------------------------------
namespace {
__global__ void wait_nothing(int polls, int* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    psg::mbar_init(&bar, 1);
    psg::mbar_expect_tx(&bar, 16);  // 16 bytes that never arrive
    psg::mbar_wait_polls(&bar, 0, polls, status);
  }
}
}  // namespace

extern "C" int psg_debug_wait_timeout(int polls, int* status_out) {
  if (polls < 1 || polls > (1 << 20) || !status_out) {
    psg_set_error("bad arguments");
    return PSG_ERR_ARG;
  }
  int* d = nullptr;
  PSG_CUDA_TRY(cudaMalloc(&d, sizeof(int)));
  cudaError_t e = cudaMemset(d, 0, sizeof(int));
  if (e == cudaSuccess) {
    wait_nothing<<<1, 32>>>(polls, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(status_out, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  PSG_CUDA_TRY(e);
  return PSG_OK;
}
