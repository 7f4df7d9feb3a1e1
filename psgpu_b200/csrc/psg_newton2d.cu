// psg_newton2d.cu -- batched Newton-GMRES-hookstep search for unstable periodic
// orbits of 2D Kolmogorov flow.
//
// Restates the reference's UPO solver (2D_NavierStokes/src_RK4/src_gmres/
// main.F90:688-1823): Newton on F(z,T,s) = shift_s(Phi_T(z)) - z with the two
// extra unknowns period T and shift s and the two orthogonality rows <dz/dt, .>
// and <dz/ds, .>; GMRES with modified Gram-Schmidt on the augmented Krylov
// vectors; SVD of the Hessenberg matrix; the hookstep trust region with the
// bisection on mu and the halve/double logic of the reference.  Differences in
// form, not in algorithm:
//   * all guesses advance in lock step and every integration of a phase (one
//     per GMRES iteration, one per hookstep trial) is a single persistent
//     launch over the guesses;
//   * Jv is the exact tangent of the discrete step (integrated with the base,
//     psg_tan2d.cuh) in FP64 or in FP32, or the reference's forward
//     difference (eps = 1e-7, FP64: a difference quotient of FP32
//     integrations would be rounding noise).  Phi_T, the residual, dz/dt, the
//     Arnoldi vectors and the hookstep are FP64 in every mode;
//   * the Arnoldi orthogonalisation runs on the GPU in FP64, one block per
//     guess; the small Hessenberg SVD runs on the host (one-sided Jacobi).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <vector>

#include "psg_tan2d_run.cuh"

namespace psg {

PSG_TAN2D_EXTERN(double)
PSG_TAN2D_EXTERN(float)

using C2 = cpx<double>;

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// per-guess descriptor of the vector kernels
struct VecJob {
  const C2* a;
  const C2* b;
  const C2* c;
  C2* out;
  double ca, cb, cc;   // coefficients
  double sx, sy;       // shift
  int rsym;
};

__device__ __forceinline__ bool keep_ik(int ik, int K, int X) {
  return keep2(ik % X, ik / X - K, K);
}

// out = ca a + cb b + cc c on kept modes, 0 elsewhere (b, c may be null)
__global__ void vec_lincomb(const VecJob* jobs, int K, int X, int nkt) {
  const VecJob J = jobs[blockIdx.y];
  for (int ik = blockIdx.x * blockDim.x + threadIdx.x; ik < nkt; ik += gridDim.x * blockDim.x) {
    C2 r = czero<double>();
    if (keep_ik(ik, K, X)) {
      const C2 a = J.a[ik];
      r = C2{J.ca * a.x, J.ca * a.y};
      if (J.b) { const C2 b = J.b[ik]; r.x += J.cb * b.x; r.y += J.cb * b.y; }
      if (J.c) { const C2 c = J.c[ik]; r.x += J.cc * c.x; r.y += J.cc * c.y; }
    }
    J.out[ik] = r;
  }
}

// out = exp(-i kx sx) exp(-i ky sy) * (rsym ? conj(a(kx,-ky)) : a(kx,ky)) on kept
// modes (src_gmres/main.F90:718-731)
__global__ void vec_shift(const VecJob* jobs, int K, int X, int nkt) {
  const VecJob J = jobs[blockIdx.y];
  for (int ik = blockIdx.x * blockDim.x + threadIdx.x; ik < nkt; ik += gridDim.x * blockDim.x) {
    const int ikx = ik % X, iky = ik / X;
    C2 r = czero<double>();
    if (keep_ik(ik, K, X)) {
      C2 a = J.rsym ? J.a[(2 * K - iky) * X + ikx] : J.a[ik];
      if (J.rsym) a.y = -a.y;
      const double ph = -(double)ikx * J.sx - (double)(iky - K) * J.sy;
      double s, c;
      sincos(ph, &s, &c);
      r = C2{c * a.x - s * a.y, c * a.y + s * a.x};
    }
    J.out[ik] = r;
  }
}

// out = -i kx a on kept modes (dZ/dS, src_gmres/main.F90:825-832)
__global__ void vec_dkx(const VecJob* jobs, int K, int X, int nkt) {
  const VecJob J = jobs[blockIdx.y];
  for (int ik = blockIdx.x * blockDim.x + threadIdx.x; ik < nkt; ik += gridDim.x * blockDim.x) {
    C2 r = czero<double>();
    if (keep_ik(ik, K, X)) {
      const C2 a = J.a[ik];
      const double kx = (double)(ik % X);
      r = C2{kx * a.y, -kx * a.x};
    }
    J.out[ik] = r;
  }
}

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) red[0] = s;
  }
  __syncthreads();
  s = red[0];
  __syncthreads();
  return s;
}

// real inner products Re sum_kept conj(a) b for every guess (one block each)
struct DotJob {
  const C2* a;
  const C2* b;
  double* out;
};
__global__ void __launch_bounds__(256) vec_dot(const DotJob* jobs, int K, int X, int nkt) {
  __shared__ double red[32];
  const DotJob J = jobs[blockIdx.x];
  double s = 0.0;
  for (int ik = threadIdx.x; ik < nkt; ik += blockDim.x)
    if (keep_ik(ik, K, X)) {
      const C2 a = J.a[ik], b = J.b[ik];
      s += a.x * b.x + a.y * b.y;
    }
  s = block_sum(s, red);
  if (threadIdx.x == 0) *J.out = s;
}

// Modified Gram-Schmidt of the augmented vector (v, vN1, vN2, vN3) against
// (q_j, qN1_j, qN2_j, qN3_j), j < m, then H[m+1,m] and q_{m+1}
// (src_gmres/main.F90:1130-1155; the third row is arc-length continuation's,
// zero otherwise).  One block per guess, FP64.
struct MgsJob {
  C2* v;
  C2* const* q;     // device array of m+1 basis pointers (q[m] receives the new vector)
  const double* qn; // host-mirrored extra rows: qN1[j], qN2[j], qN3[j] (3*(m+1))
  double vn1, vn2, vn3;  // extra rows of v
  int m;            // number of basis vectors to orthogonalise against
  double* H;        // out: H[0..m] of column m (m+1 entries) + vN1, vN2, vN3 of q_{m+1}
};
__global__ void __launch_bounds__(256) mgs_kernel(const MgsJob* jobs, int K, int X, int nkt) {
  __shared__ double red[32];
  const MgsJob J = jobs[blockIdx.x];
  double vn1 = J.vn1, vn2 = J.vn2, vn3 = J.vn3;
  for (int j = 0; j < J.m; ++j) {
    const C2* qj = J.q[j];
    double s = 0.0;
    for (int ik = threadIdx.x; ik < nkt; ik += blockDim.x)
      if (keep_ik(ik, K, X)) {
        const C2 a = qj[ik], b = J.v[ik];
        s += a.x * b.x + a.y * b.y;
      }
    double h = block_sum(s, red) + J.qn[3 * j] * vn1 + J.qn[3 * j + 1] * vn2 + J.qn[3 * j + 2] * vn3;
    for (int ik = threadIdx.x; ik < nkt; ik += blockDim.x)
      if (keep_ik(ik, K, X)) {
        const C2 a = qj[ik];
        C2 b = J.v[ik];
        b.x -= h * a.x;
        b.y -= h * a.y;
        J.v[ik] = b;
      }
    vn1 -= h * J.qn[3 * j];
    vn2 -= h * J.qn[3 * j + 1];
    vn3 -= h * J.qn[3 * j + 2];
    if (threadIdx.x == 0) J.H[j] = h;
    __syncthreads();
  }
  double s = 0.0;
  for (int ik = threadIdx.x; ik < nkt; ik += blockDim.x)
    if (keep_ik(ik, K, X)) {
      const C2 b = J.v[ik];
      s += b.x * b.x + b.y * b.y;
    }
  const double hn = sqrt(block_sum(s, red) + vn1 * vn1 + vn2 * vn2 + vn3 * vn3);
  C2* qn = J.q[J.m];
  for (int ik = threadIdx.x; ik < nkt; ik += blockDim.x)
    qn[ik] = keep_ik(ik, K, X) ? C2{J.v[ik].x / hn, J.v[ik].y / hn} : czero<double>();
  if (threadIdx.x == 0) {
    J.H[J.m] = hn;
    J.H[J.m + 1] = vn1 / hn;
    J.H[J.m + 2] = vn2 / hn;
    J.H[J.m + 3] = vn3 / hn;
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

// thin SVD of the (r x c) column-major matrix A (r >= c) by one-sided Jacobi:
// A = U diag(S) V^T with U (r x c), V (c x c)
static void jacobi_svd(int r, int c, const std::vector<double>& A, std::vector<double>& U,
                       std::vector<double>& S, std::vector<double>& V) {
  U = A;
  V.assign((size_t)c * c, 0.0);
  for (int i = 0; i < c; ++i) V[(size_t)i * c + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < c - 1; ++p)
      for (int q = p + 1; q < c; ++q) {
        double a = 0, b = 0, d = 0;
        for (int i = 0; i < r; ++i) {
          const double x = U[(size_t)p * r + i], y = U[(size_t)q * r + i];
          a += x * x; b += y * y; d += x * y;
        }
        if (fabs(d) <= 1e-300) continue;
        off = std::max(off, fabs(d) / sqrt(a * b));
        const double zeta = (b - a) / (2.0 * d);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int i = 0; i < r; ++i) {
          const double x = U[(size_t)p * r + i], y = U[(size_t)q * r + i];
          U[(size_t)p * r + i] = cs * x - sn * y;
          U[(size_t)q * r + i] = sn * x + cs * y;
        }
        for (int i = 0; i < c; ++i) {
          const double x = V[(size_t)p * c + i], y = V[(size_t)q * c + i];
          V[(size_t)p * c + i] = cs * x - sn * y;
          V[(size_t)q * c + i] = sn * x + cs * y;
        }
      }
    if (off < 1e-15) break;
  }
  S.assign(c, 0.0);
  for (int j = 0; j < c; ++j) {
    double nrm = 0;
    for (int i = 0; i < r; ++i) nrm += U[(size_t)j * r + i] * U[(size_t)j * r + i];
    nrm = sqrt(nrm);
    S[j] = nrm;
    if (nrm > 0)
      for (int i = 0; i < r; ++i) U[(size_t)j * r + i] /= nrm;
  }
}

enum UpoStatus : int {
  UPO_ACTIVE = 0,
  UPO_CONVERGED = 1,
  UPO_GMRES_FAILED = 2,
  UPO_HOOK_FAILED = 3,
  UPO_STALLED = 4,
  UPO_TSTEP_FAILED = 5,
  UPO_PERIOD_TOO_SMALL = 6,
  UPO_NEWTON_FAILED = 7,
};

struct Guess {
  // device vectors (nkt complex each)
  C2 *z, *zn, *znshift, *fn, *dzdt, *dzndt, *dzds, *dznds, *v, *diff, *jdiff, *zplus, *zplus2,
      *zn_trial, *zn2, *fnplus, *fnplus2, *scratch;
  // arc-length continuation: the branch tangent dZ/dr, the last converged state
  // Zr2 and shift(dPhi_T/dnu) (exact Jv), device vectors
  C2 *dzrdr, *zr2, *dphidnu;
  bool arc = false;
  double dTrdr = 0, dSrdr = 0, dv2rdr = 0, Tr2 = 0, Sr2 = 0, v2r2 = 0, ndelta = 0;
  double c0 = 0;     // <dZ/dr, Zr2>
  double narc = 0, narcplus = 0, narcplus2 = 0, v2plus = 0, v2plus2 = 0, dV = 0;
  std::vector<C2*> q;  // Krylov basis
  InstTan2D<double> inst;  // integration buffers
  InstTan2D<float> inst32;  // FP32 integration buffers (exact Jv in FP32)
  // host state
  double T = 0, sx = 0, sy = 0, nu = 0, dt0 = 0, dt_true = 0;
  // viscosity TIMEDERIV sees: the reference keeps one NU array, set last by
  // the previous hookstep trial (v2plus), not reset when the trial is
  // reverted (src_gmres/main.F90:1458-1470, 816-821)
  double nu_rhs = 0;
  int rsym = 0;
  double delta = 0.1;
  double normfn = 0, normz = 1, ner = 0, ner_old = 0;
  int ner_count = 0;
  int status = UPO_ACTIVE;
  int newton = 0, gmres = 0, hook = 0;
  std::vector<double> qn;  // qN1, qN2, qN3 per basis vector
  std::vector<double> H;   // (kmax+1) x kmax column-major
  int m = 0;               // GMRES iterations done in this Newton step
  bool gmres_done = false;
  // hookstep
  std::vector<double> U, S, Vt, P;
  double mu = 0, normb = 0;
  double Tplus = 0, Splus = 0, Tplus2 = 0, Splus2 = 0;
  double nfpred = 0, nfplus = 0, nfplus2 = 0;
  double dT = 0, dS = 0;
  bool halve = false, dbl = false, hook_done = false;
  int ihook = 0;
  // one record per Newton step: newton index, GMRES iterations, hookstep
  // trials, Delta after the step, mu of the last trial, T, shift, residual,
  // |F|, time step in use, viscosity
  std::vector<std::array<double, 11>> trace;
};

struct Upo2D {
  // jv_mode 0: exact tangent (FP64), 1: forward difference, 2: exact tangent in FP32
  int ng = 0, n = 0, K = 0, X = 0, Y = 0, nkt = 0, kmax = 0, jv_mode = 0;
  double eps = 1e-7, gmtol = 1e-3;
  std::vector<Guess> G;
  C2* pool = nullptr;
  cpx<float>* pool32 = nullptr;
  IntPlan<double> plan64;
  IntPlan<float> plan32;
  CvtJob* d_cvt = nullptr;
  VecJob* d_vec = nullptr;
  DotJob* d_dot = nullptr;
  MgsJob* d_mgs = nullptr;
  double* d_scalars = nullptr;  // per-guess scalar outputs
  C2** d_qptr = nullptr;
  double* d_qn = nullptr;
  double* d_H = nullptr;
  int* d_next = nullptr;
  cudaStream_t stream = 0;
  long launches = 0, integrations = 0;
  // phase timing (psg_upo2d_profile): seconds in the batched integrations by
  // kind (exact Jv FP64, exact Jv FP32, Phi_T, dz/dt), in the host SVDs, and in
  // solve() as a whole; the stream is synchronised around each integration
  // while it is on
  bool prof = false;
  double t_int[4] = {0, 0, 0, 0}, t_svd = 0, t_solve = 0;
  // blocks per instance (a cluster) when the batch leaves room: at most this many
  int cluster_max = 4;
  // side streams and events of integrations split over several launches
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[3] = {nullptr, nullptr, nullptr};

  ~Upo2D() {
    if (pool) cudaFree(pool);
    if (pool32) cudaFree(pool32);
    if (d_cvt) cudaFree(d_cvt);
    plan64.release();
    plan32.release();
    if (d_vec) cudaFree(d_vec);
    if (d_dot) cudaFree(d_dot);
    if (d_mgs) cudaFree(d_mgs);
    if (d_scalars) cudaFree(d_scalars);
    if (d_qptr) cudaFree(d_qptr);
    if (d_qn) cudaFree(d_qn);
    if (d_H) cudaFree(d_H);
    if (d_next) cudaFree(d_next);
    for (int k = 0; k < 3; ++k) {
      if (side[k]) cudaStreamDestroy(side[k]);
      if (ev_join[k]) cudaEventDestroy(ev_join[k]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
  }

  int init(int ng_, int n_, int kmax_, int jv_mode_) {
    ng = ng_; n = n_; kmax = kmax_; jv_mode = jv_mode_;
    if (!(n == 16 || n == 32 || n == 64 || n == 128 || n == 256)) {
      psg_set_error("UPO grid %d unsupported", n);
      return PSG_ERR_UNSUPPORTED;
    }
    if (kmax < 1 || kmax > 500 || ng < 1) { psg_set_error("bad UPO sizes"); return PSG_ERR_ARG; }
    K = n / 3; X = K + 1; Y = 2 * K + 1; nkt = X * Y;
    const long nvec = 21 + (kmax + 1) + 10;
    const long work = 6L * n * X;
    const long per = nvec * nkt + work;
    const long twl = 2L * n;
    PSG_CUDA_TRY(cudaMalloc(&pool, sizeof(C2) * (per * ng + twl)));
    PSG_CUDA_TRY(cudaMemset(pool, 0, sizeof(C2) * (per * ng + twl)));
    G.resize(ng);
    for (int g = 0; g < ng; ++g) {
      C2* p = pool + per * g;
      Guess& U_ = G[g];
      C2** v[] = {&U_.z, &U_.zn, &U_.znshift, &U_.fn, &U_.dzdt, &U_.dzndt, &U_.dzds, &U_.dznds,
                  &U_.v, &U_.diff, &U_.jdiff, &U_.zplus, &U_.zplus2, &U_.zn_trial, &U_.zn2,
                  &U_.fnplus, &U_.fnplus2, &U_.scratch, &U_.dzrdr, &U_.zr2, &U_.dphidnu};
      for (auto pp : v) { *pp = p; p += nkt; }
      U_.q.resize(kmax + 1);
      for (int j = 0; j <= kmax; ++j) { U_.q[j] = p; p += nkt; }
      InstTan2D<double>& I = U_.inst;
      I.n = n;
      I.Z = p; p += nkt; I.Z0 = p; p += nkt; I.Z1 = p; p += nkt; I.Z2 = p; p += nkt; I.Z3 = p; p += nkt;
      I.D = p; p += nkt; I.D0 = p; p += nkt; I.D1 = p; p += nkt; I.D2 = p; p += nkt; I.D3 = p; p += nkt;
      I.work = p; p += work;
      U_.qn.assign(3 * (kmax + 1), 0.0);
      U_.H.assign((size_t)(kmax + 1) * kmax, 0.0);
    }
    if (int rc = plan64.init(n, ng, pool + per * ng)) return rc;
    if (jv_mode == 2) {
      // FP32 base + tangent buffers and twiddles for the Krylov products
      const long per32 = 10L * nkt + work;
      PSG_CUDA_TRY(cudaMalloc(&pool32, sizeof(cpx<float>) * (per32 * ng + twl)));
      PSG_CUDA_TRY(cudaMemset(pool32, 0, sizeof(cpx<float>) * (per32 * ng + twl)));
      for (int g = 0; g < ng; ++g) {
        cpx<float>* p = pool32 + per32 * g;
        InstTan2D<float>& I = G[g].inst32;
        I.n = n;
        I.Z = p; p += nkt; I.Z0 = p; p += nkt; I.Z1 = p; p += nkt; I.Z2 = p; p += nkt; I.Z3 = p; p += nkt;
        I.D = p; p += nkt; I.D0 = p; p += nkt; I.D1 = p; p += nkt; I.D2 = p; p += nkt; I.D3 = p; p += nkt;
        I.work = p;
      }
      if (int rc = plan32.init(n, ng, pool32 + per32 * ng)) return rc;
    }
    PSG_CUDA_TRY(cudaMalloc(&d_cvt, sizeof(CvtJob) * 2 * ng));
    PSG_CUDA_TRY(cudaMalloc(&d_vec, sizeof(VecJob) * ng));
    PSG_CUDA_TRY(cudaMalloc(&d_dot, sizeof(DotJob) * ng * 4));
    PSG_CUDA_TRY(cudaMalloc(&d_mgs, sizeof(MgsJob) * ng));
    PSG_CUDA_TRY(cudaMalloc(&d_scalars, sizeof(double) * ng * 4));
    PSG_CUDA_TRY(cudaMalloc(&d_qptr, sizeof(C2*) * ng * (kmax + 1)));
    PSG_CUDA_TRY(cudaMalloc(&d_qn, sizeof(double) * ng * 3 * (kmax + 1)));
    PSG_CUDA_TRY(cudaMalloc(&d_H, sizeof(double) * ng * (kmax + 4)));
    PSG_CUDA_TRY(cudaMalloc(&d_next, sizeof(int)));
    std::vector<C2*> qp((size_t)ng * (kmax + 1));
    for (int g = 0; g < ng; ++g)
      for (int j = 0; j <= kmax; ++j) qp[(size_t)g * (kmax + 1) + j] = G[g].q[j];
    PSG_CUDA_TRY(cudaMemcpy(d_qptr, qp.data(), sizeof(C2*) * qp.size(), cudaMemcpyHostToDevice));
    // PSG_UPO_CLUSTER: the largest cluster an integration may use (1, 2 or 4)
    if (const char* e = getenv("PSG_UPO_CLUSTER")) cluster_max = atoi(e);
    return PSG_OK;
  }

  // ----- batched integration: for every guess in `who`, integrate from z_in
  // (and, mode 0, the perturbation d_in) over its period T with its time step
  struct IntReq {
    int g;
    const C2* z_in;
    const C2* d_in;
    double T;
    int mode;
    double nu = -1.0;  // viscosity of this integration (< 0: the guess's)
  };
  int integrate(const std::vector<IntReq>& reqs) {
    if (reqs.empty()) return PSG_OK;
    // the Krylov products (mode 0) of jv_mode 2 integrate base and tangent in
    // FP32; every other integration (Phi_T, dz/dt, FP64 tangents) in FP64
    bool fp32 = jv_mode == 2;
    for (const IntReq& r : reqs) fp32 = fp32 && r.mode == 0;
    std::chrono::steady_clock::time_point t0;
    if (prof) {
      PSG_CUDA_TRY(cudaStreamSynchronize(stream));
      t0 = std::chrono::steady_clock::now();
    }
    const int rc = fp32 ? integrate_t<float>(reqs, plan32) : integrate_t<double>(reqs, plan64);
    if (prof && !rc) {
      PSG_CUDA_TRY(cudaStreamSynchronize(stream));
      const int kind = reqs[0].mode == 0 ? (fp32 ? 1 : 0) : reqs[0].mode == 1 ? 2 : 3;
      t_int[kind] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return rc;
  }

  InstTan2D<double>& inst_of(Guess& U_, double*) { return U_.inst; }
  InstTan2D<float>& inst_of(Guess& U_, float*) { return U_.inst32; }

  int convert(const std::vector<CvtJob>& jobs, bool to32) {
    if (jobs.empty()) return PSG_OK;
    PSG_CUDA_TRY(cudaMemcpyAsync(d_cvt, jobs.data(), sizeof(CvtJob) * jobs.size(),
                                 cudaMemcpyHostToDevice, stream));
    if (to32) cvt_launch<float>(d_cvt, (int)jobs.size(), nkt, stream);
    else cvt_launch<double>(d_cvt, (int)jobs.size(), nkt, stream);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  template <typename T>
  int integrate_t(const std::vector<IntReq>& reqs, IntPlan<T>& plan) {
    constexpr bool is32 = sizeof(T) == 4;
    std::vector<InstTan2D<T>> h;
    std::vector<CvtJob> in_jobs, out_jobs;
    for (const IntReq& r : reqs) {
      Guess& U_ = G[r.g];
      InstTan2D<T> I = inst_of(U_, (T*)nullptr);
      I.mode = r.mode;
      I.nu = (T)(r.nu >= 0.0 ? r.nu : U_.nu);
      if (r.mode == 2) {
        I.nsteps = 0;
        I.dt = 0;
      } else {
        // NSTOP = INT(T/DELT); DELT = T/NSTOP (src_gmres/main.F90:697-699)
        int ns = (int)(r.T / U_.dt_true);
        if (ns < 1) ns = 1;
        I.nsteps = ns;
        I.dt = (T)(r.T / (double)ns);
      }
      if (is32) {
        // inputs rounded to FP32; outputs widened back into the FP64 buffers
        in_jobs.push_back(CvtJob{r.z_in, I.Z});
        in_jobs.push_back(CvtJob{r.d_in, I.D});
        out_jobs.push_back(CvtJob{I.Z, U_.inst.Z});
        out_jobs.push_back(CvtJob{I.D, U_.inst.D});
      } else {
        PSG_CUDA_TRY(cudaMemcpyAsync(I.Z, r.z_in, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream));
        if (r.mode == 0)
          PSG_CUDA_TRY(cudaMemcpyAsync(I.D, r.d_in, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream));
      }
      h.push_back(I);
    }
    if (is32)
      if (int rc = convert(in_jobs, true)) return rc;
    // blocks per guess: every guess starts with one; while blocks are left
    // (the resident capacity of the device at the integrator's registers), the
    // guess that would finish last moves to a cluster of two, then four.
    // Relative speeds of one, two and four blocks on one guess (FP64 tangent
    // at 128^2): 1, 1.67, 2.34.
    const int ni = (int)h.size();
    const int grid_cap = plan.grid_cap;
    std::vector<int> cs(ni, 1);
    auto speed = [](int c) { return c == 4 ? 2.34 : c == 2 ? 1.67 : 1.0; };
    auto work = [&](int i) { return (double)h[i].nsteps * (h[i].mode == 0 ? 5 : 3); };
    if (cluster_max >= 2 && ni <= grid_cap) {
      int used = ni;
      for (;;) {
        int worst = 0;
        for (int i = 1; i < ni; ++i)
          if (work(i) / speed(cs[i]) > work(worst) / speed(cs[worst])) worst = i;
        const int up = cs[worst] == 1 ? 2 : 4;
        if (cs[worst] == 4 || up > cluster_max || used + up - cs[worst] > grid_cap) break;
        used += up - cs[worst];
        cs[worst] = up;
      }
    }
    // groups of four, two and one block(s), each longest first
    std::vector<int> idx(ni);
    for (int i = 0; i < ni; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
      return cs[a] != cs[b] ? cs[a] > cs[b] : work(a) > work(b);
    });
    std::vector<InstTan2D<T>> hs(ni);
    int cnt[3] = {0, 0, 0};  // four, two, one
    for (int i = 0; i < ni; ++i) {
      hs[i] = h[idx[i]];
      ++cnt[cs[idx[i]] == 4 ? 0 : cs[idx[i]] == 2 ? 1 : 2];
    }
    PSG_CUDA_TRY(cudaMemcpyAsync(plan.d_inst, hs.data(), sizeof(InstTan2D<T>) * ni,
                                 cudaMemcpyHostToDevice, stream));
    PSG_CUDA_TRY(cudaMemsetAsync(d_next, 0, sizeof(int), stream));
    const int ngroups = (cnt[0] > 0) + (cnt[1] > 0) + (cnt[2] > 0);
    if (ngroups > 1 && !side[0]) {
      for (int k = 0; k < 3; ++k) {
        PSG_CUDA_TRY(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
        PSG_CUDA_TRY(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
      }
      PSG_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    }
    // one group: on the engine's stream; more: each on a stream of its own,
    // all after the copies above and before anything queued later
    if (ngroups > 1) PSG_CUDA_TRY(cudaEventRecord(ev_fork, stream));
    int off = 0;
    const int csz[3] = {4, 2, 1};
    for (int k = 0; k < 3; ++k) {
      if (!cnt[k]) continue;
      cudaStream_t st = stream;
      if (ngroups > 1) {
        st = side[k];
        PSG_CUDA_TRY(cudaStreamWaitEvent(st, ev_fork, 0));
      }
      const int m = cnt[k];
      tan2d_launch<T>(n, csz[k], m, std::min<int>(m, grid_cap), plan.smem, st, plan.d_inst + off,
                      d_next, plan.tw);
      PSG_CUDA_TRY(cudaGetLastError());
      if (ngroups > 1) {
        PSG_CUDA_TRY(cudaEventRecord(ev_join[k], st));
        PSG_CUDA_TRY(cudaStreamWaitEvent(stream, ev_join[k], 0));
      }
      ++launches;
      off += m;
    }
    if (is32)
      if (int rc = convert(out_jobs, false)) return rc;
    integrations += (long)ni;
    return PSG_OK;
  }

  int vec_launch(void (*k)(const VecJob*, int, int, int), const std::vector<VecJob>& jobs) {
    if (jobs.empty()) return PSG_OK;
    PSG_CUDA_TRY(cudaMemcpyAsync(d_vec, jobs.data(), sizeof(VecJob) * jobs.size(),
                                 cudaMemcpyHostToDevice, stream));
    k<<<dim3((nkt + 255) / 256, (unsigned)jobs.size()), 256, 0, stream>>>(d_vec, K, X, nkt);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  // dots[i] = <a_i, b_i> (synchronous)
  int dots(const std::vector<std::pair<const C2*, const C2*>>& ab, std::vector<double>& out) {
    out.assign(ab.size(), 0.0);
    if (ab.empty()) return PSG_OK;
    std::vector<DotJob> j(ab.size());
    for (size_t i = 0; i < ab.size(); ++i) j[i] = DotJob{ab[i].first, ab[i].second, d_scalars + i};
    if (ab.size() > (size_t)ng * 4) { psg_set_error("too many dot products"); return PSG_ERR_ARG; }
    PSG_CUDA_TRY(cudaMemcpyAsync(d_dot, j.data(), sizeof(DotJob) * j.size(), cudaMemcpyHostToDevice, stream));
    vec_dot<<<(unsigned)j.size(), 256, 0, stream>>>(d_dot, K, X, nkt);
    ++launches;
    PSG_CUDA_TRY(cudaMemcpyAsync(out.data(), d_scalars, sizeof(double) * ab.size(),
                                 cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }

  int shift(const std::vector<int>& who, C2* Guess::*out, const C2* Guess::*in, double Guess::*sx) {
    std::vector<VecJob> jobs;
    for (int g : who) {
      VecJob J{};
      J.a = G[g].*in; J.out = G[g].*out; J.sx = G[g].*sx; J.sy = G[g].sy; J.rsym = G[g].rsym;
      jobs.push_back(J);
    }
    return vec_launch(vec_shift, jobs);
  }
  int shift_ptr(const std::vector<int>& who, const std::vector<const C2*>& in,
                const std::vector<C2*>& out, const std::vector<double>& sx) {
    std::vector<VecJob> jobs;
    for (size_t i = 0; i < who.size(); ++i) {
      VecJob J{};
      J.a = in[i]; J.out = out[i]; J.sx = sx[i]; J.sy = G[who[i]].sy; J.rsym = G[who[i]].rsym;
      jobs.push_back(J);
    }
    return vec_launch(vec_shift, jobs);
  }
  int lincomb(const std::vector<VecJob>& jobs) { return vec_launch(vec_lincomb, jobs); }

  static VecJob lc(C2* out, const C2* a, double ca, const C2* b = nullptr, double cb = 0,
                   const C2* c = nullptr, double cc = 0) {
    VecJob J{};
    J.out = out; J.a = a; J.ca = ca; J.b = b; J.cb = cb; J.c = c; J.cc = cc;
    return J;
  }

  int copy_out(const std::vector<int>& who, C2* Guess::*dst, bool from_D) {
    for (int g : who)
      PSG_CUDA_TRY(cudaMemcpyAsync(G[g].*dst, from_D ? G[g].inst.D : G[g].inst.Z, sizeof(C2) * nkt,
                                   cudaMemcpyDeviceToDevice, stream));
    return PSG_OK;
  }

  // J q for every guess in `who` (q from the pointer list), written to `out`:
  // shift(dPhi_T(z) q) - q + dZN/dS q_s + dZN/dt q_T (src_gmres/main.F90:1100-1116),
  // and with arc-length continuation + shift(dPhi_T/dnu) q_v: the forward
  // difference perturbs the viscosity with the state (main.F90:1050-1063), the
  // exact form adds the derivative formed once per Newton step
  int apply_j(const std::vector<int>& who, const std::vector<const C2*>& q,
              const std::vector<double>& qs, const std::vector<double>& qt,
              const std::vector<double>& qv, C2* Guess::*out) {
    std::vector<IntReq> reqs;
    std::vector<VecJob> jobs;
    if (jv_mode != 1) {
      for (size_t i = 0; i < who.size(); ++i)
        reqs.push_back(IntReq{who[i], G[who[i]].z, q[i], G[who[i]].T, 0});
      if (int rc = integrate(reqs)) return rc;
      std::vector<const C2*> src;
      std::vector<C2*> dst;
      std::vector<double> sx;
      for (int g : who) { src.push_back(G[g].inst.D); dst.push_back(G[g].*out); sx.push_back(G[g].sx); }
      if (int rc = shift_ptr(who, src, dst, sx)) return rc;
    } else {
      // forward difference with eps = 1e-7 (src_gmres/main.F90:1048-1108)
      for (size_t i = 0; i < who.size(); ++i) jobs.push_back(lc(G[who[i]].scratch, G[who[i]].z, 1.0, q[i], eps));
      if (int rc = lincomb(jobs)) return rc;
      for (size_t i = 0; i < who.size(); ++i) {
        const Guess& U_ = G[who[i]];
        reqs.push_back(IntReq{who[i], U_.scratch, nullptr, U_.T, 1,
                              U_.arc ? U_.nu + eps * qv[i] : -1.0});
      }
      if (int rc = integrate(reqs)) return rc;
      jobs.clear();
      for (int g : who) jobs.push_back(lc(G[g].scratch, G[g].inst.Z, 1.0 / eps, G[g].zn, -1.0 / eps));
      if (int rc = lincomb(jobs)) return rc;
      std::vector<const C2*> src;
      std::vector<C2*> dst;
      std::vector<double> sx;
      for (int g : who) { src.push_back(G[g].scratch); dst.push_back(G[g].*out); sx.push_back(G[g].sx); }
      if (int rc = shift_ptr(who, src, dst, sx)) return rc;
    }
    jobs.clear();
    for (size_t i = 0; i < who.size(); ++i)
      jobs.push_back(lc(G[who[i]].*out, G[who[i]].*out, 1.0, q[i], -1.0, G[who[i]].dznds, qs[i]));
    if (int rc = lincomb(jobs)) return rc;
    jobs.clear();
    for (size_t i = 0; i < who.size(); ++i) {
      const Guess& U_ = G[who[i]];
      const bool dnu = U_.arc && jv_mode != 1;
      jobs.push_back(lc(U_.*out, U_.*out, 1.0, U_.dzndt, qt[i], dnu ? U_.dphidnu : nullptr,
                        dnu ? qv[i] : 0.0));
    }
    return lincomb(jobs);
  }

  // F = shift(Phi_T(z)) - z, norms and residual for the guesses in `who`
  int residual(const std::vector<int>& who) {
    std::vector<IntReq> reqs;
    for (int g : who) reqs.push_back(IntReq{g, G[g].z, nullptr, G[g].T, 1});
    if (int rc = integrate(reqs)) return rc;
    if (int rc = copy_out(who, &Guess::zn, false)) return rc;
    if (int rc = shift(who, &Guess::znshift, (const C2* Guess::*)&Guess::zn, &Guess::sx)) return rc;
    std::vector<VecJob> jobs;
    for (int g : who) jobs.push_back(lc(G[g].fn, G[g].znshift, 1.0, G[g].z, -1.0));
    if (int rc = lincomb(jobs)) return rc;
    std::vector<std::pair<const C2*, const C2*>> ab;
    for (int g : who) { ab.push_back({G[g].zn, G[g].zn}); ab.push_back({G[g].fn, G[g].fn}); }
    std::vector<double> d;
    if (int rc = dots(ab, d)) return rc;
    for (size_t i = 0; i < who.size(); ++i) {
      Guess& U_ = G[who[i]];
      U_.normz = sqrt(d[2 * i]);
      U_.normfn = sqrt(d[2 * i + 1]);
      U_.ner = U_.normfn / U_.normz;
    }
    return PSG_OK;
  }

  // x(mu) = P S / (mu + S^2), its norm
  static double xnorm(const Guess& U_, int m, double mu, std::vector<double>& x) {
    x.assign(m, 0.0);
    double s = 0;
    for (int j = 0; j < m; ++j) {
      x[j] = (mu == 0.0) ? U_.P[j] / U_.S[j] : U_.P[j] * U_.S[j] / (mu + U_.S[j] * U_.S[j]);
      s += x[j] * x[j];
    }
    return sqrt(s);
  }

  // mu so that delta/sqrt2 < |x| < sqrt2 delta (src_gmres/main.F90:1283-1335);
  // returns the step y = V x in the Krylov basis
  static void hook_step(Guess& U_, int m, std::vector<double>& y) {
    const double root2 = sqrt(2.0);
    std::vector<double> x;
    double nx = xnorm(U_, m, 0.0, x);
    U_.mu = 0.0;
    if (nx > root2 * U_.delta) {
      double mu1 = 0.0, mu2 = *std::max_element(U_.S.begin(), U_.S.begin() + m);
      nx = xnorm(U_, m, mu2, x);
      for (int it = 0; it < 2000 && !(nx < U_.delta); ++it) {
        mu1 = mu2;
        mu2 = 2.0 * mu2;
        nx = xnorm(U_, m, mu2, x);
      }
      double mid = mu2;
      for (int it = 0; it < 2000 && !(nx < root2 * U_.delta && nx > U_.delta / root2); ++it) {
        mid = 0.5 * (mu2 + mu1);
        nx = xnorm(U_, m, mid, x);
        if (nx > U_.delta) mu1 = mid;
        else mu2 = mid;
      }
      U_.mu = mid;
    }
    y.assign(m, 0.0);
    for (int i = 0; i < m; ++i) {
      double a = 0;
      for (int j = 0; j < m; ++j) a += U_.Vt[(size_t)j * m + i] * x[j];
      y[i] = a;
    }
  }

  int solve(int max_newton, double tol) {
    std::vector<int> act;
    for (int g = 0; g < ng; ++g)
      if (G[g].status == UPO_ACTIVE) act.push_back(g);
    if (int rc = residual(act)) return rc;
    for (int g : act)
      if (G[g].ner <= tol) G[g].status = UPO_CONVERGED;
    std::vector<C2*> qdev;
    for (int it = 0; it < max_newton; ++it) {
      act.clear();
      for (int g = 0; g < ng; ++g)
        if (G[g].status == UPO_ACTIVE) act.push_back(g);
      if (act.empty()) break;
      std::vector<VecJob> jobs;
      for (int g : act) {
        Guess& U_ = G[g];
        U_.newton += 1;
        // |b| with the arc-length residual as one more row (main.F90:802-815)
        U_.normb = U_.arc ? sqrt(U_.normfn * U_.normfn + U_.narc * U_.narc) : U_.normfn;
        U_.m = 0;
        U_.gmres_done = false;
        std::fill(U_.H.begin(), U_.H.end(), 0.0);
        std::fill(U_.qn.begin(), U_.qn.end(), 0.0);
        if (U_.arc) U_.qn[2] = -U_.narc / U_.normb;
        jobs.push_back(lc(U_.q[0], U_.fn, -1.0 / U_.normb));
      }
      if (int rc = lincomb(jobs)) return rc;
      // exact Jv with continuation: shift(dPhi_T/dnu) by a central difference in
      // nu (step 1e-5 nu: truncation and round-off both near 1e-10 relative)
      if (jv_mode != 1) {
        std::vector<int> an;
        for (int g : act)
          if (G[g].arc) an.push_back(g);
        if (!an.empty()) {
          std::vector<IntReq> reqs;
          for (int g : an) reqs.push_back(IntReq{g, G[g].z, nullptr, G[g].T, 1, G[g].nu * (1.0 + 1e-5)});
          if (int rc = integrate(reqs)) return rc;
          if (int rc = copy_out(an, &Guess::dphidnu, false)) return rc;
          reqs.clear();
          for (int g : an) reqs.push_back(IntReq{g, G[g].z, nullptr, G[g].T, 1, G[g].nu * (1.0 - 1e-5)});
          if (int rc = integrate(reqs)) return rc;
          std::vector<VecJob> dj;
          for (int g : an)
            dj.push_back(lc(G[g].scratch, G[g].dphidnu, 0.5e5 / G[g].nu, G[g].inst.Z, -0.5e5 / G[g].nu));
          if (int rc = lincomb(dj)) return rc;
          std::vector<const C2*> src;
          std::vector<C2*> dst;
          std::vector<double> sx;
          for (int g : an) { src.push_back(G[g].scratch); dst.push_back(G[g].dphidnu); sx.push_back(G[g].sx); }
          if (int rc = shift_ptr(an, src, dst, sx)) return rc;
        }
      }
      // dZN/dt and dz/dt (TIMEDERIV), dZN/dS and dz/dS
      {
        std::vector<IntReq> reqs;
        for (int g : act) reqs.push_back(IntReq{g, G[g].znshift, nullptr, 0.0, 2, G[g].nu_rhs});
        if (int rc = integrate(reqs)) return rc;
        if (int rc = copy_out(act, &Guess::dzndt, true)) return rc;
        reqs.clear();
        for (int g : act) reqs.push_back(IntReq{g, G[g].z, nullptr, 0.0, 2, G[g].nu_rhs});
        if (int rc = integrate(reqs)) return rc;
        if (int rc = copy_out(act, &Guess::dzdt, true)) return rc;
        std::vector<VecJob> dj;
        for (int g : act) { VecJob J{}; J.a = G[g].znshift; J.out = G[g].dznds; dj.push_back(J); }
        if (int rc = vec_launch(vec_dkx, dj)) return rc;
        dj.clear();
        for (int g : act) { VecJob J{}; J.a = G[g].z; J.out = G[g].dzds; dj.push_back(J); }
        if (int rc = vec_launch(vec_dkx, dj)) return rc;
      }
      // ------------------------------------------------------------- GMRES
      for (int k = 0; k < kmax; ++k) {
        std::vector<int> ga;
        for (int g : act)
          if (!G[g].gmres_done) ga.push_back(g);
        if (ga.empty()) break;
        std::vector<const C2*> q;
        std::vector<double> qs, qt, qv;
        for (int g : ga) {
          q.push_back(G[g].q[k]);
          qt.push_back(G[g].qn[3 * k]);
          qs.push_back(G[g].qn[3 * k + 1]);
          qv.push_back(G[g].qn[3 * k + 2]);
        }
        if (int rc = apply_j(ga, q, qs, qt, qv, &Guess::v)) return rc;
        std::vector<std::pair<const C2*, const C2*>> ab;
        for (int g : ga) {
          ab.push_back({G[g].dzdt, G[g].q[k]});
          ab.push_back({G[g].dzds, G[g].q[k]});
          ab.push_back({G[g].dzrdr, G[g].q[k]});
        }
        std::vector<double> vn;
        if (int rc = dots(ab, vn)) return rc;
        std::vector<MgsJob> mj;
        std::vector<double> qnh;
        for (size_t i = 0; i < ga.size(); ++i) {
          const int g = ga[i];
          MgsJob J{};
          J.v = G[g].v;
          J.q = d_qptr + (size_t)g * (kmax + 1);
          J.qn = d_qn + (size_t)i * 3 * (kmax + 1);
          J.vn1 = vn[3 * i];
          J.vn2 = vn[3 * i + 1];
          // the arc-length row (main.F90:1123-1126)
          const Guess& U_ = G[g];
          J.vn3 = U_.arc ? vn[3 * i + 2] + U_.dTrdr * U_.qn[3 * k] + U_.dSrdr * U_.qn[3 * k + 1] +
                               U_.dv2rdr * U_.qn[3 * k + 2]
                         : 0.0;
          J.m = k + 1;
          J.H = d_H + (size_t)i * (kmax + 4);
          mj.push_back(J);
          qnh.insert(qnh.end(), G[g].qn.begin(), G[g].qn.end());
        }
        PSG_CUDA_TRY(cudaMemcpyAsync(d_qn, qnh.data(), sizeof(double) * qnh.size(), cudaMemcpyHostToDevice, stream));
        PSG_CUDA_TRY(cudaMemcpyAsync(d_mgs, mj.data(), sizeof(MgsJob) * mj.size(), cudaMemcpyHostToDevice, stream));
        // MgsJob.q points at the basis pointer array: q[0..k] existing, q[k+1] new
        mgs_kernel<<<(unsigned)mj.size(), 256, 0, stream>>>(d_mgs, K, X, nkt);
        ++launches;
        std::vector<double> hh(ga.size() * (kmax + 4));
        PSG_CUDA_TRY(cudaMemcpyAsync(hh.data(), d_H, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, stream));
        PSG_CUDA_TRY(cudaStreamSynchronize(stream));
        PSG_CUDA_TRY(cudaGetLastError());
        for (size_t i = 0; i < ga.size(); ++i) {
          Guess& U_ = G[ga[i]];
          const double* h = hh.data() + i * (kmax + 4);
          const int rows = kmax + 1;
          for (int j = 0; j <= k + 1; ++j) U_.H[(size_t)k * rows + j] = h[j];
          U_.qn[3 * (k + 1)] = h[k + 2];
          U_.qn[3 * (k + 1) + 1] = h[k + 3];
          U_.qn[3 * (k + 1) + 2] = h[k + 4];
          // SVD of H(1:k+2, 1:k+1) and the GMRES residual (src_gmres/main.F90:1161-1228)
          const int r = k + 2, c = k + 1;
          std::vector<double> A((size_t)r * c);
          for (int cc = 0; cc < c; ++cc)
            for (int rr = 0; rr < r; ++rr) A[(size_t)cc * r + rr] = U_.H[(size_t)cc * rows + rr];
          std::vector<double> Um, Sm, Vm;
          const auto ts0 = std::chrono::steady_clock::now();
          jacobi_svd(r, c, A, Um, Sm, Vm);
          if (prof) t_svd += std::chrono::duration<double>(std::chrono::steady_clock::now() - ts0).count();
          U_.P.assign(c, 0.0);
          for (int j = 0; j < c; ++j) U_.P[j] = U_.normb * Um[(size_t)j * r + 0];
          U_.S = Sm;
          U_.Vt.assign((size_t)c * c, 0.0);
          for (int a = 0; a < c; ++a)
            for (int b = 0; b < c; ++b) U_.Vt[(size_t)a * c + b] = Vm[(size_t)a * c + b];
          // GMR = | H y - |b| e1 | / |b| with y = V x, x = P / S
          std::vector<double> y(c, 0.0), hy(r, 0.0);
          for (int ii = 0; ii < c; ++ii) {
            double a = 0;
            for (int j = 0; j < c; ++j) a += Vm[(size_t)j * c + ii] * (Sm[j] > 0 ? U_.P[j] / Sm[j] : 0.0);
            y[ii] = a;
          }
          for (int rr = 0; rr < r; ++rr) {
            double a = 0;
            for (int cc = 0; cc < c; ++cc) a += U_.H[(size_t)cc * rows + rr] * y[cc];
            hy[rr] = a;
          }
          hy[0] -= U_.normb;
          double gmr = 0;
          for (double t : hy) gmr += t * t;
          gmr = sqrt(gmr) / U_.normb;
          if (gmr <= gmtol || k + 1 == kmax) {
            U_.m = k + 1;
            U_.gmres_done = true;
            U_.gmres += k + 1;
            if (gmr > gmtol) {
              U_.status = UPO_GMRES_FAILED;
              U_.trace.push_back({(double)U_.newton, (double)(k + 1), 0.0, U_.delta, 0.0, U_.T,
                                  U_.sx, U_.ner, U_.normfn, U_.dt_true, U_.nu});
            }
          }
        }
      }
      // ------------------------------------------------------------- hookstep
      std::vector<int> ha;
      for (int g : act)
        if (G[g].status == UPO_ACTIVE) {
          G[g].ihook = 0; G[g].halve = false; G[g].dbl = false; G[g].hook_done = false;
          ha.push_back(g);
        }
      for (int round = 0; round < 64; ++round) {
        std::vector<int> hr;
        for (int g : ha)
          if (!G[g].hook_done) hr.push_back(g);
        if (hr.empty()) break;
        std::vector<int> live;
        for (int g : hr) {
          Guess& U_ = G[g];
          U_.ihook += 1;
          if (U_.ihook > 50) { U_.status = UPO_HOOK_FAILED; U_.hook_done = true; continue; }
          live.push_back(g);
        }
        if (live.empty()) break;
        // step y in the Krylov basis; DIFF = Q y, DIFFT, DIFFS
        std::vector<double> coef((size_t)live.size() * (kmax + 1), 0.0);
        std::vector<VecJob> jobs2;
        for (size_t i = 0; i < live.size(); ++i) {
          Guess& U_ = G[live[i]];
          std::vector<double> y;
          hook_step(U_, U_.m, y);
          U_.dT = 0; U_.dS = 0; U_.dV = 0;
          for (int j = 0; j < U_.m; ++j) {
            U_.dT += U_.qn[3 * j] * y[j];
            U_.dS += U_.qn[3 * j + 1] * y[j];
            U_.dV += U_.qn[3 * j + 2] * y[j];
          }
          // diff = sum_j y_j q_j, accumulated three basis vectors per launch
          for (int j = 0; j < U_.m; ++j) coef[i * (kmax + 1) + j] = y[j];
        }
        for (int j = 0; j < kmax; ++j) {
          jobs2.clear();
          bool any = false;
          for (size_t i = 0; i < live.size(); ++i) {
            Guess& U_ = G[live[i]];
            if (j >= U_.m) continue;
            any = true;
            const double cj = coef[i * (kmax + 1) + j];
            jobs2.push_back(j == 0 ? lc(U_.diff, U_.q[0], cj) : lc(U_.diff, U_.diff, 1.0, U_.q[j], cj));
          }
          if (!any) break;
          if (int rc = lincomb(jobs2)) return rc;
        }
        // J DIFF and the predicted residual
        std::vector<const C2*> dq;
        std::vector<double> qs, qt, qv;
        for (int g : live) {
          dq.push_back(G[g].diff);
          qs.push_back(G[g].dS);
          qt.push_back(G[g].dT);
          qv.push_back(G[g].dV);
        }
        if (int rc = apply_j(live, dq, qs, qt, qv, &Guess::jdiff)) return rc;
        jobs2.clear();
        for (int g : live) jobs2.push_back(lc(G[g].scratch, G[g].fn, 1.0, G[g].jdiff, 1.0));
        if (int rc = lincomb(jobs2)) return rc;
        // trial: z + DIFF over T + DIFFT with shift s + DIFFS
        jobs2.clear();
        for (int g : live) jobs2.push_back(lc(G[g].zplus, G[g].z, 1.0, G[g].diff, 1.0));
        if (int rc = lincomb(jobs2)) return rc;
        std::vector<IntReq> reqs;
        for (int g : live) {
          G[g].Tplus = G[g].T + G[g].dT;
          G[g].Splus = G[g].sx + G[g].dS;
          G[g].v2plus = G[g].nu + (G[g].arc ? G[g].dV : 0.0);
          G[g].nu_rhs = G[g].v2plus;
          reqs.push_back(IntReq{g, G[g].zplus, nullptr, G[g].Tplus, 1, G[g].v2plus});
        }
        if (int rc = integrate(reqs)) return rc;
        if (int rc = copy_out(live, &Guess::zn_trial, false)) return rc;
        {
          std::vector<const C2*> src;
          std::vector<C2*> dst;
          std::vector<double> sx;
          for (int g : live) { src.push_back(G[g].zn_trial); dst.push_back(G[g].fnplus); sx.push_back(G[g].Splus); }
          if (int rc = shift_ptr(live, src, dst, sx)) return rc;
        }
        jobs2.clear();
        for (int g : live) jobs2.push_back(lc(G[g].fnplus, G[g].fnplus, 1.0, G[g].zplus, -1.0));
        if (int rc = lincomb(jobs2)) return rc;
        std::vector<std::pair<const C2*, const C2*>> ab;
        for (int g : live) {
          ab.push_back({G[g].scratch, G[g].scratch});
          ab.push_back({G[g].fnplus, G[g].fnplus});
          ab.push_back({G[g].dzrdr, G[g].zplus});
        }
        std::vector<double> d;
        if (int rc = dots(ab, d)) return rc;
        // accept / retry logic (src_gmres/main.F90:1523-1622)
        for (size_t i = 0; i < live.size(); ++i) {
          Guess& U_ = G[live[i]];
          U_.nfpred = sqrt(d[3 * i]);
          U_.nfplus = sqrt(d[3 * i + 1]);
          // |b| of the trial and of the prediction with const = 0, with the
          // arc-length residual when continuing (main.F90:1420-1480)
          double normb_pred = U_.normfn, normb_plus = U_.nfplus;
          if (U_.arc) {
            U_.narcplus = d[3 * i + 2] - U_.c0 + U_.dSrdr * (U_.Splus - U_.Sr2) +
                          U_.dv2rdr * (U_.v2plus - U_.v2r2) - U_.ndelta +
                          U_.dTrdr * (U_.Tplus - U_.Tr2);
            normb_pred = sqrt(U_.normfn * U_.normfn + U_.narc * U_.narc);
            normb_plus = sqrt(U_.nfplus * U_.nfplus + U_.narcplus * U_.narcplus);
          }
          auto save = [&]() {
            cudaMemcpyAsync(U_.zplus2, U_.zplus, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
            cudaMemcpyAsync(U_.zn2, U_.zn_trial, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
            cudaMemcpyAsync(U_.fnplus2, U_.fnplus, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
            U_.Tplus2 = U_.Tplus; U_.Splus2 = U_.Splus; U_.nfplus2 = U_.nfplus;
            U_.v2plus2 = U_.v2plus; U_.narcplus2 = U_.narcplus;
          };
          auto revert = [&]() {
            cudaMemcpyAsync(U_.zplus, U_.zplus2, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
            cudaMemcpyAsync(U_.zn_trial, U_.zn2, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
            cudaMemcpyAsync(U_.fnplus, U_.fnplus2, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
            U_.Tplus = U_.Tplus2; U_.Splus = U_.Splus2; U_.nfplus = U_.nfplus2;
            U_.v2plus = U_.v2plus2; U_.narcplus = U_.narcplus2;
          };
          if (U_.nfplus != U_.nfplus || U_.nfpred != U_.nfpred) {
            U_.delta *= 0.5; U_.halve = true;
            continue;
          }
          if (normb_plus >= normb_pred) {
            if (U_.dbl) { revert(); U_.delta *= 0.5; U_.hook_done = true; continue; }
            U_.delta *= 0.5; U_.halve = true;
          } else {
            if (U_.halve) { U_.hook_done = true; continue; }
            if (U_.dbl && U_.nfplus > U_.nfplus2) { revert(); U_.delta *= 0.5; U_.hook_done = true; continue; }
            if (U_.mu == 0.0) { U_.hook_done = true; }
            else if (fabs(U_.nfpred - U_.nfplus) < 0.1 * fabs(U_.nfplus - U_.normfn)) {
              U_.delta *= 2.0; U_.dbl = true; save();
            } else if (U_.nfplus < U_.nfpred) {
              U_.delta *= 2.0; U_.dbl = true; save();
            } else {
              U_.hook_done = true;
            }
          }
        }
      }
      // ------------------------------------------------------------- update
      std::vector<int> up, redo;
      for (int g : ha) {
        Guess& U_ = G[g];
        U_.hook += U_.ihook;
        const bool blown = U_.nfpred != U_.nfpred || U_.nfplus != U_.nfplus;
        if (blown) {
          // a trial integration blew up: halve the time step and redo the
          // Newton step from the same z, T, s (src_gmres/main.F90:1636-1665)
          U_.trace.push_back({(double)U_.newton, (double)U_.m, (double)U_.ihook, U_.delta, U_.mu,
                              U_.T, U_.sx, U_.ner, U_.normfn, U_.dt_true, U_.nu});
          if (U_.dt_true < 0.1 * U_.dt0) {
            U_.status = UPO_TSTEP_FAILED;
          } else {
            U_.dt_true *= 0.5;
            U_.status = UPO_ACTIVE;
            redo.push_back(g);
          }
          continue;
        }
        if (U_.status != UPO_ACTIVE) {
          U_.trace.push_back({(double)U_.newton, (double)U_.m, (double)U_.ihook, U_.delta, U_.mu,
                              U_.T, U_.sx, U_.ner, U_.normfn, U_.dt_true, U_.nu});
          continue;
        }
        up.push_back(g);
        cudaMemcpyAsync(U_.zn, U_.zn_trial, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(U_.z, U_.zplus, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(U_.fn, U_.fnplus, sizeof(C2) * nkt, cudaMemcpyDeviceToDevice, stream);
        U_.T = U_.Tplus;
        U_.sx = U_.Splus;
        U_.normfn = U_.nfplus;
        if (U_.arc) {
          U_.nu = U_.v2plus;
          U_.narc = U_.narcplus;
        }
      }
      // the shifted final state of a redone step is rebuilt from the old Phi_T(z)
      if (int rc = shift(redo, &Guess::znshift, (const C2* Guess::*)&Guess::zn, &Guess::sx)) return rc;
      if (int rc = shift(up, &Guess::znshift, (const C2* Guess::*)&Guess::zn, &Guess::sx)) return rc;
      std::vector<std::pair<const C2*, const C2*>> ab;
      for (int g : up) ab.push_back({G[g].zn, G[g].zn});
      std::vector<double> d;
      if (int rc = dots(ab, d)) return rc;
      for (size_t i = 0; i < up.size(); ++i) {
        Guess& U_ = G[up[i]];
        U_.normz = sqrt(d[i]);
        const double ner = U_.normfn / U_.normz;
        U_.trace.push_back({(double)U_.newton, (double)U_.m, (double)U_.ihook, U_.delta, U_.mu,
                            U_.T, U_.sx, ner, U_.normfn, U_.dt_true, U_.nu});
        if (ner != ner) { U_.status = UPO_TSTEP_FAILED; continue; }
        // stall detection before the convergence test, as the reference
        // orders them (src_gmres/main.F90:1752-1804)
        const double rel = fabs((ner - U_.ner_old) / ner);
        bool stalled = false;
        if (rel < 0.001) {
          stalled = ++U_.ner_count > 3;
        } else {
          U_.ner_count = 0;
        }
        U_.ner_old = ner;
        U_.ner = ner;
        if (stalled) U_.status = UPO_STALLED;
        else if (ner <= tol) U_.status = UPO_CONVERGED;
        else if (U_.T < 0.1) U_.status = UPO_PERIOD_TOO_SMALL;
        else if (U_.newton >= max_newton) U_.status = UPO_NEWTON_FAILED;
      }
      for (int g : redo)
        if (G[g].newton >= max_newton) G[g].status = UPO_NEWTON_FAILED;
    }
    for (int g = 0; g < ng; ++g)
      if (G[g].status == UPO_ACTIVE) G[g].status = UPO_NEWTON_FAILED;
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }
};

}  // namespace psg

using namespace psg;

struct psg_upo2d {
  Upo2D* u = nullptr;
};

#define PSG_U2(h)                                                                  \
  do {                                                                             \
    if (!(h) || !(h)->u) { psg_set_error("null UPO handle"); return PSG_ERR_ARG; } \
  } while (0)

extern "C" int psg_upo2d_create(psg_upo2d** out, int nguess, int n, int kmax, int jv_mode) {
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  *out = nullptr;
  if (jv_mode < 0 || jv_mode > 2) {
    psg_set_error("jv_mode: 0 exact tangent, 1 finite difference, 2 exact tangent in FP32");
    return PSG_ERR_ARG;
  }
  psg_upo2d* h = new psg_upo2d();
  h->u = new Upo2D();
  int rc = h->u->init(nguess, n, kmax, jv_mode);
  if (rc) { delete h->u; delete h; return rc; }
  *out = h;
  return PSG_OK;
}

extern "C" void psg_upo2d_destroy(psg_upo2d* h) {
  if (!h) return;
  delete h->u;
  delete h;
}

extern "C" int psg_upo2d_set_guess(psg_upo2d* h, int i, const double* Z, double T, double sx,
                                   double sy, int rsym, double nu, double dt) {
  PSG_U2(h);
  Upo2D& U = *h->u;
  if (i < 0 || i >= U.ng || !Z || T <= 0 || dt <= 0) { psg_set_error("bad guess"); return PSG_ERR_ARG; }
  Guess& g = U.G[i];
  std::vector<C2> z((size_t)U.nkt);
  const int K = U.K, X = U.X;
  for (int ik = 0; ik < U.nkt; ++ik) {
    const int ikx = ik % X, ky = ik / X - K;
    const bool keep = !(ikx == 0 && ky <= 0) && 4 * (ikx * ikx + ky * ky) <= (2 * K - 1) * (2 * K - 1);
    z[ik] = keep ? C2{Z[2 * ik], Z[2 * ik + 1]} : C2{0.0, 0.0};
  }
  PSG_CUDA_TRY(cudaMemcpy(g.z, z.data(), sizeof(C2) * U.nkt, cudaMemcpyHostToDevice));
  g.T = T; g.sx = sx; g.sy = sy; g.rsym = rsym; g.nu = nu; g.nu_rhs = nu; g.dt0 = dt; g.dt_true = dt;
  // a guess period from a run with this time step is taken as exact
  // (src_gmres/main.F90:688-695)
  if (fabs(T - nearbyint(T / dt) * dt) < 1e-10) g.T = nearbyint(T / dt) * dt;
  g.delta = 0.1; g.status = UPO_ACTIVE; g.newton = g.gmres = g.hook = 0;
  g.ner_old = 0; g.ner_count = 0;
  g.trace.clear();
  g.arc = false;
  return PSG_OK;
}

extern "C" int psg_upo2d_solve(psg_upo2d* h, int max_newton, double tol, double gmres_tol) {
  PSG_U2(h);
  h->u->gmtol = gmres_tol;
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = h->u->solve(max_newton, tol);
  if (h->u->prof) {
    cudaStreamSynchronize(h->u->stream);
    h->u->t_solve += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return rc;
}

extern "C" int psg_upo2d_get(psg_upo2d* h, int i, double* Z, double* vals, int* info) {
  PSG_U2(h);
  Upo2D& U = *h->u;
  if (i < 0 || i >= U.ng) { psg_set_error("guess %d out of range", i); return PSG_ERR_ARG; }
  Guess& g = U.G[i];
  if (Z) PSG_CUDA_TRY(cudaMemcpy(Z, g.z, sizeof(C2) * U.nkt, cudaMemcpyDeviceToHost));
  if (vals) { vals[0] = g.T; vals[1] = g.sx; vals[2] = g.sy; vals[3] = g.ner; }
  if (info) { info[0] = g.status; info[1] = g.newton; info[2] = g.gmres; info[3] = g.hook; }
  return PSG_OK;
}

// building blocks at guess i: Phi_T(z) (mode 1), the tangent dPhi_T(z) q
// (mode 0, q in/out) or dz/dt (mode 2); all unshifted
extern "C" int psg_upo2d_apply(psg_upo2d* h, int i, int mode, double* Zout, double* q) {
  PSG_U2(h);
  Upo2D& U = *h->u;
  if (i < 0 || i >= U.ng || mode < 0 || mode > 2) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  Guess& g = U.G[i];
  if (mode == 0) {
    if (!q) { psg_set_error("null perturbation"); return PSG_ERR_ARG; }
    PSG_CUDA_TRY(cudaMemcpy(g.scratch, q, sizeof(C2) * U.nkt, cudaMemcpyHostToDevice));
  }
  std::vector<Upo2D::IntReq> r{Upo2D::IntReq{i, g.z, g.scratch, g.T, mode}};
  if (int rc = U.integrate(r)) return rc;
  PSG_CUDA_TRY(cudaStreamSynchronize(U.stream));
  if (Zout && mode != 2) PSG_CUDA_TRY(cudaMemcpy(Zout, g.inst.Z, sizeof(C2) * U.nkt, cudaMemcpyDeviceToHost));
  if (mode == 0) PSG_CUDA_TRY(cudaMemcpy(q, g.inst.D, sizeof(C2) * U.nkt, cudaMemcpyDeviceToHost));
  if (mode == 2 && Zout) PSG_CUDA_TRY(cudaMemcpy(Zout, g.inst.D, sizeof(C2) * U.nkt, cudaMemcpyDeviceToHost));
  return PSG_OK;
}

// Arc-length continuation of guess i (src_gmres/main.F90:408-640): the
// viscosity becomes an unknown, with the pseudo-arclength row
// <dZ/dr, z - Zr2> + dT/dr (T - Tr2) + dS/dr (s - Sr2) + dv2/dr (nu - v2r2) = ndelta
// (dZrdr, Zr2: complex128 boxes, reference layout).  Call after
// psg_upo2d_set_guess, which puts the prediction in place and clears this.
extern "C" int psg_upo2d_set_arc(psg_upo2d* h, int i, const double* dZrdr, const double* Zr2,
                                 double dTrdr, double dSrdr, double dv2rdr, double Tr2,
                                 double Sr2, double v2r2, double ndelta) {
  PSG_U2(h);
  Upo2D& U = *h->u;
  if (i < 0 || i >= U.ng || !dZrdr || !Zr2) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  Guess& g = U.G[i];
  std::vector<C2> a((size_t)U.nkt), b((size_t)U.nkt);
  const int K = U.K, X = U.X;
  for (int ik = 0; ik < U.nkt; ++ik) {
    const int ikx = ik % X, ky = ik / X - K;
    const bool keep = !(ikx == 0 && ky <= 0) && 4 * (ikx * ikx + ky * ky) <= (2 * K - 1) * (2 * K - 1);
    a[ik] = keep ? C2{dZrdr[2 * ik], dZrdr[2 * ik + 1]} : C2{0.0, 0.0};
    b[ik] = keep ? C2{Zr2[2 * ik], Zr2[2 * ik + 1]} : C2{0.0, 0.0};
  }
  PSG_CUDA_TRY(cudaMemcpy(g.dzrdr, a.data(), sizeof(C2) * U.nkt, cudaMemcpyHostToDevice));
  PSG_CUDA_TRY(cudaMemcpy(g.zr2, b.data(), sizeof(C2) * U.nkt, cudaMemcpyHostToDevice));
  std::vector<double> d;
  if (int rc = U.dots({{g.dzrdr, g.zr2}, {g.dzrdr, g.z}}, d)) return rc;
  g.dTrdr = dTrdr; g.dSrdr = dSrdr; g.dv2rdr = dv2rdr;
  g.Tr2 = Tr2; g.Sr2 = Sr2; g.v2r2 = v2r2; g.ndelta = ndelta;
  g.c0 = d[0];
  // the initial arc-length residual (main.F90:633-640)
  g.narc = d[1] - g.c0 + dSrdr * (g.sx - Sr2) + dv2rdr * (g.nu - v2r2) - ndelta + dTrdr * (g.T - Tr2);
  g.arc = true;
  return PSG_OK;
}

// the current viscosity of guess i (the continuation parameter)
extern "C" int psg_upo2d_get_nu(psg_upo2d* h, int i, double* nu) {
  PSG_U2(h);
  if (i < 0 || i >= h->u->ng || !nu) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  *nu = h->u->G[i].nu;
  return PSG_OK;
}

// the per-Newton-step record k of guess i (rec[11]; see Guess::trace)
extern "C" int psg_upo2d_trace(psg_upo2d* h, int i, int k, double* rec) {
  PSG_U2(h);
  Upo2D& U = *h->u;
  if (i < 0 || i >= U.ng || !rec) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  const Guess& g = U.G[i];
  if (k < 0 || k >= (int)g.trace.size()) {
    psg_set_error("guess %d has %d trace records", i, (int)g.trace.size());
    return PSG_ERR_ARG;
  }
  for (int j = 0; j < 11; ++j) rec[j] = g.trace[k][j];
  return PSG_OK;
}

extern "C" int psg_upo2d_trace_count(psg_upo2d* h, int i) {
  if (!h || !h->u || i < 0 || i >= h->u->ng) return -1;
  return (int)h->u->G[i].trace.size();
}

extern "C" long psg_upo2d_integrations(psg_upo2d* h) { return (h && h->u) ? h->u->integrations : -1; }
extern "C" long psg_upo2d_launches(psg_upo2d* h) { return (h && h->u) ? h->u->launches : -1; }

// phase timing of the solver: enable (1) clears the counters and synchronises
// around every batched integration from then on; 0 turns it off
extern "C" int psg_upo2d_profile(psg_upo2d* h, int enable) {
  PSG_U2(h);
  Upo2D& U = *h->u;
  U.prof = enable != 0;
  if (U.prof) {
    for (double& t : U.t_int) t = 0;
    U.t_svd = U.t_solve = 0;
  }
  return PSG_OK;
}

// out[6] = {seconds in solve, exact-Jv integrations FP64, exact-Jv FP32,
// Phi_T integrations (residuals, trials, forward differences), dz/dt, host SVDs}
extern "C" int psg_upo2d_profile_read(psg_upo2d* h, double* out) {
  PSG_U2(h);
  if (!out) { psg_set_error("bad arguments"); return PSG_ERR_ARG; }
  const Upo2D& U = *h->u;
  out[0] = U.t_solve;
  for (int k = 0; k < 4; ++k) out[1 + k] = U.t_int[k];
  out[5] = U.t_svd;
  return PSG_OK;
}
