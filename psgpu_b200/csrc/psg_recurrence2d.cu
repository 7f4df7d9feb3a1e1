// psg_recurrence2d.cu -- near-recurrence search for UPO guesses of 2D
// Kolmogorov runs on the GPU, batched over the runs of an ensemble.
//
// Restates the 2D DNS's recurrence check (2D_NavierStokes/src_RK4/
// functions.h:105-309: computeZdash and recurrence_check) for many runs at
// once.  Every NOUT steps each run's newest state is compared, under every
// trial translation of an NSHIFTX x NSHIFTY grid, with the earlier states of
// its ring of storeSize states over the modes of a low-wavenumber box
// (0 <= kx < W, -W <= ky < W: 2 W^2 modes); the reference's selection logic
// (first turning point in the period, minimum over periods, entering and
// leaving the residual threshold, the skip of odd periods beyond 20) runs on
// the host per run over the residuals, in the reference's order.
//
// The 2D DNS's own set-up file (its init.h, which fixes NSHIFTX, NSHIFTY, the
// box and the ring size) is not in the reference tree; the box, the shift
// grids (2 pi i / (NSHIFTX alpha), 2 pi j / NSHIFTY) and freq2 = 2 NOUT dt
// follow the 3D build's set-up (3D_NavierStokes/src/init.h:182-213), which
// the 2D recurrence_check mirrors line for line.
//
// Device work per check: the shifted copies of every run's newest box (one
// launch), then one block per (run, earlier state) that forms the residual of
// every shift and keeps the smallest in the reference's loop order (y outer,
// x inner, strict <): a residual and a shift index per pair come back to the
// host, not the whole residual table.  The rings of full states (FP64) stay on
// the device.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "psg_common.cuh"
#include "psgpu_internal.h"

namespace psg {

// ring slot `slot` of every run from its state (FP32 or FP64 boxes), the
// comparison box and its norm over the kept modes; one block per run
template <typename S>
__global__ void rec2d_put(const S* const* __restrict__ states, int nkt, int slot, int store,
                          const int* __restrict__ inorm, const unsigned char* __restrict__ ll,
                          int nnorm, double2* __restrict__ ring_full,
                          double2* __restrict__ ring_sub, double* __restrict__ norms) {
  const int r = blockIdx.x;
  const S* src = states[r];
  double2* full = ring_full + ((size_t)r * store + slot) * nkt;
  for (int i = threadIdx.x; i < nkt; i += blockDim.x)
    full[i] = make_double2((double)src[2 * i], (double)src[2 * i + 1]);
  __syncthreads();
  __shared__ double red[256];
  double s = 0.0;
  double2* sub = ring_sub + ((size_t)r * store + slot) * nnorm;
  for (int i = threadIdx.x; i < nnorm; i += blockDim.x) {
    const int ik = inorm[i];
    const double2 z = full[ik];
    sub[i] = z;
    if (ll[ik]) s += z.x * z.x + z.y * z.y;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) norms[(size_t)r * store + slot] = red[0];
}

// shifted copies of every run's newest box: z exp(-i (kx sx + ky sy))
// (computeZdash, functions.h:105-129), shift s = ix + nsx * iy
__global__ void rec2d_dash(const double2* __restrict__ ring_sub, int store, int slot,
                           const double* __restrict__ kxy, const double* __restrict__ shifts,
                           int nsx, int nnorm, double2* __restrict__ dash) {
  const int s = blockIdx.y, r = blockIdx.z, nshift = gridDim.y;
  const int isx = s % nsx, isy = s / nsx;
  const double sx = shifts[isx], sy = shifts[nsx + isy];
  const double2* sub = ring_sub + ((size_t)r * store + slot) * nnorm;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnorm; i += gridDim.x * blockDim.x) {
    const double sh = kxy[i] * sx + kxy[nnorm + i] * sy;
    double sn, cs;
    sincos(sh, &sn, &cs);
    const double2 z = sub[i];
    dash[((size_t)r * nshift + s) * nnorm + i] = make_double2(cs * z.x + sn * z.y, cs * z.y - sn * z.x);
  }
}

// for every run and earlier slot: the smallest residual over the shifts,
// sqrt((-2 <dash_s, old> + |dash_s|^2 + |old|^2) / |newest|^2), and its shift
// (the first in the order y outer, x inner); one block per (slot, run)
__global__ void __launch_bounds__(256) rec2d_resid(const double2* __restrict__ dash,
                                                   const double2* __restrict__ ring_sub,
                                                   const int* __restrict__ cand,
                                                   const double* __restrict__ norms, int store,
                                                   int newest, int nnorm, int nshift,
                                                   double* __restrict__ res,
                                                   int* __restrict__ arg) {
  const int ci = blockIdx.x, r = blockIdx.y, ncand = gridDim.x;
  const int slot = cand[ci];
  const double2* o = ring_sub + ((size_t)r * store + slot) * nnorm;
  const double no = norms[(size_t)r * store + slot], nn = norms[(size_t)r * store + newest];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
  double best = 10000.0;
  int bs = nshift;
  for (int s = warp; s < nshift; s += nw) {
    const double2* d = dash + ((size_t)r * nshift + s) * nnorm;
    double cross = 0.0, nd = 0.0;
    for (int i = lane; i < nnorm; i += 32) {
      const double2 x = d[i], y = o[i];
      cross += x.x * y.x + x.y * y.y;
      nd += x.x * x.x + x.y * x.y;
    }
    for (int off = 16; off > 0; off >>= 1) {
      cross += __shfl_down_sync(0xffffffffu, cross, off);
      nd += __shfl_down_sync(0xffffffffu, nd, off);
    }
    if (lane == 0) {
      const double v = sqrt((-2.0 * cross + nd + no) / nn);
      if (v < best) { best = v; bs = s; }  // s increases: the first minimum is kept
    }
  }
  __shared__ double wb[32];
  __shared__ int ws[32];
  if (lane == 0) { wb[warp] = best; ws[warp] = bs; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 10000.0;
    int a = nshift;
    for (int w = 0; w < nw; ++w)
      if (wb[w] < b || (wb[w] == b && ws[w] < a)) { b = wb[w]; a = ws[w]; }
    res[(size_t)r * ncand + ci] = b;
    arg[(size_t)r * ncand + ci] = a;
  }
}

struct Rec2D {
  int nrun = 0, n = 0, K = 0, X = 0, Y = 0, store = 0, nw = 0, nnorm = 0, nsx = 0, nsy = 0;
  long nkt = 0;
  double alpha = 1.0, thresh = 0.0, delt = 0.0, tstart = 0.0, freq2 = 0.0;
  int nout = 1;
  std::vector<double> v2;
  cudaStream_t stream = 0;
  double2* ring_full = nullptr;  // [run][store][nkt]
  double2* ring_sub = nullptr;   // [run][store][nnorm]
  double2* dash = nullptr;       // [run][nshift][nnorm]
  double* d_norms = nullptr;     // [run][store]
  double* d_kxy = nullptr;       // [2][nnorm]
  double* d_shifts = nullptr;
  int* d_inorm = nullptr;
  unsigned char* d_ll = nullptr;
  int* d_cand = nullptr;
  double* d_res = nullptr;       // [run][cand]
  int* d_arg = nullptr;
  const void** d_states = nullptr;
  long launches = 0;
  std::vector<double> shiftx, shifty;
  // the reference's bookkeeping: the ring indices are shared (all runs store
  // in lock step); the selection state is per run
  int nStore = 0, nCopy = 0, iStart = 0;
  struct Sel {
    int recOut = 0, minStoreOuter = 0;
    double minResOuter = 0.0, minTimeOuter = 0.0, recPeriod = 0.0;
    double minSxOuter = 0.0, minSyOuter = 0.0;
  };
  std::vector<Sel> sel;
  struct Guess2 {
    double meta[7];  // run, start time, v2, period, shift x, shift y, residual
    std::vector<double2> z;
  };
  std::vector<Guess2> guesses;

  ~Rec2D() {
    void* ps[] = {ring_full, ring_sub, dash, d_norms, d_kxy, d_shifts, d_inorm, d_ll, d_cand,
                  d_res, d_arg, (void*)d_states};
    for (void* p : ps)
      if (p) cudaFree(p);
  }

  int init(int nrun_, int n_, double alpha_, int store_, int nw_, int nsx_, int nsy_, double th,
           int nout_, double delt_, double tstart_, const double* v2_) {
    nrun = nrun_; n = n_; K = n / 3; X = K + 1; Y = 2 * K + 1; nkt = (long)X * Y;
    store = store_; nw = nw_; nsx = nsx_; nsy = nsy_;
    alpha = alpha_; thresh = th; nout = nout_; delt = delt_; tstart = tstart_;
    if (nrun < 1 || n < 8 || store < 2 || nw < 1 || nw > K || nsx < 1 || nsy < 1 || nout < 1 ||
        nsx * nsy > 4096 || !v2_) {
      psg_set_error("2D recurrence: bad sizes");
      return PSG_ERR_ARG;
    }
    v2.assign(v2_, v2_ + nrun);
    freq2 = 2 * nout * delt;
    nnorm = 2 * nw * nw;
    std::vector<int> inorm(nnorm);
    std::vector<double> kxy(2 * (size_t)nnorm);
    for (int iy = 0; iy < 2 * nw; ++iy)
      for (int ix = 0; ix < nw; ++ix) {
        const int i = iy * nw + ix, iky = K - nw + iy;
        inorm[i] = iky * X + ix;
        kxy[i] = ix * alpha;
        kxy[nnorm + i] = iky - K;
      }
    std::vector<unsigned char> ll(nkt);
    for (int iky = 0; iky < Y; ++iky)
      for (int ikx = 0; ikx < X; ++ikx) {
        const double kx = ikx * alpha, ky = iky - K;
        ll[(long)iky * X + ikx] = !(kx == 0.0 && ky <= 0.0) && sqrt(kx * kx + ky * ky) <= K - 0.5;
      }
    const double twopi = 4.0 * asin(1.0);
    for (int i = 0; i < nsx; ++i) shiftx.push_back(twopi * i / (nsx * alpha));
    for (int i = 0; i < nsy; ++i) shifty.push_back(twopi * i / nsy);
    std::vector<double> sh(shiftx);
    sh.insert(sh.end(), shifty.begin(), shifty.end());
    sel.assign(nrun, Sel());
    const size_t nshift = (size_t)nsx * nsy;
    PSG_CUDA_TRY(cudaMalloc(&ring_full, sizeof(double2) * (size_t)nrun * store * nkt));
    PSG_CUDA_TRY(cudaMalloc(&ring_sub, sizeof(double2) * (size_t)nrun * store * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&dash, sizeof(double2) * (size_t)nrun * nshift * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&d_norms, sizeof(double) * (size_t)nrun * store));
    PSG_CUDA_TRY(cudaMalloc(&d_kxy, sizeof(double) * 2 * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&d_shifts, sizeof(double) * sh.size()));
    PSG_CUDA_TRY(cudaMalloc(&d_inorm, sizeof(int) * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&d_ll, nkt));
    PSG_CUDA_TRY(cudaMalloc(&d_cand, sizeof(int) * store));
    PSG_CUDA_TRY(cudaMalloc(&d_res, sizeof(double) * (size_t)nrun * store));
    PSG_CUDA_TRY(cudaMalloc(&d_arg, sizeof(int) * (size_t)nrun * store));
    PSG_CUDA_TRY(cudaMalloc(&d_states, sizeof(void*) * nrun));
    PSG_CUDA_TRY(cudaMemset(d_norms, 0, sizeof(double) * (size_t)nrun * store));
    PSG_CUDA_TRY(cudaMemcpy(d_kxy, kxy.data(), sizeof(double) * kxy.size(), cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMemcpy(d_shifts, sh.data(), sizeof(double) * sh.size(), cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMemcpy(d_inorm, inorm.data(), sizeof(int) * nnorm, cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMemcpy(d_ll, ll.data(), nkt, cudaMemcpyHostToDevice));
    return PSG_OK;
  }

  // every run's state (device boxes of `precision`) into ring slot `slot`
  int put(int slot, const void* const* st, int precision) {
    PSG_CUDA_TRY(cudaMemcpyAsync(d_states, st, sizeof(void*) * nrun, cudaMemcpyHostToDevice, stream));
    if (precision == 64)
      rec2d_put<double><<<nrun, 256, 0, stream>>>((const double* const*)d_states, (int)nkt, slot,
                                                  store, d_inorm, d_ll, nnorm, ring_full,
                                                  ring_sub, d_norms);
    else
      rec2d_put<float><<<nrun, 256, 0, stream>>>((const float* const*)d_states, (int)nkt, slot,
                                                 store, d_inorm, d_ll, nnorm, ring_full,
                                                 ring_sub, d_norms);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    return PSG_OK;
  }

  int start(const void* const* st, int precision) {
    nStore = 0; nCopy = 0; iStart = 0;
    sel.assign(nrun, Sel());
    return put(0, st, precision);
  }

  // recurrence_check (functions.h:194-309) of every run's newest state
  int check(int nt, int* emitted) {
    const double tme = tstart + (nt - nout) * delt;
    struct Cand { int icount, slot; double period; };
    std::vector<Cand> cand;
    for (int icount = nStore - 1; icount >= 1; --icount) {
      const double period = ((nStore - icount) * nout) * delt;
      int slot = icount + iStart;
      slot -= (int)floor((double)slot / store) * store;
      if (period > 20.0 && fabs(period - freq2 * floor(period / freq2 + 0.5)) > 0.0001) continue;
      cand.push_back(Cand{icount, slot, period});
    }
    const int nc = (int)cand.size(), nshift = nsx * nsy;
    std::vector<double> res((size_t)nrun * nc);
    std::vector<int> arg((size_t)nrun * nc);
    if (nc > 0) {
      std::vector<int> slots;
      for (const Cand& c : cand) slots.push_back(c.slot);
      PSG_CUDA_TRY(cudaMemcpyAsync(d_cand, slots.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, stream));
      rec2d_dash<<<dim3((nnorm + 127) / 128, nshift, nrun), 128, 0, stream>>>(
          ring_sub, store, nCopy, d_kxy, d_shifts, nsx, nnorm, dash);
      rec2d_resid<<<dim3(nc, nrun), 256, 0, stream>>>(dash, ring_sub, d_cand, d_norms, store,
                                                       nCopy, nnorm, nshift, d_res, d_arg);
      launches += 2;
      PSG_CUDA_TRY(cudaGetLastError());
      PSG_CUDA_TRY(cudaMemcpyAsync(res.data(), d_res, sizeof(double) * res.size(),
                                   cudaMemcpyDeviceToHost, stream));
      PSG_CUDA_TRY(cudaMemcpyAsync(arg.data(), d_arg, sizeof(int) * arg.size(),
                                   cudaMemcpyDeviceToHost, stream));
      PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    *emitted = 0;
    for (int r = 0; r < nrun; ++r) {
      Sel& S = sel[r];
      double minResInner = 10000.0, minPeriod = 10000.0, rs = 0.0;
      int minPflag = 1, minStoreInner = 0, minCountInner = 0;
      double minSxInner = 0.0, minSyInner = 0.0;
      for (int ci = 0; ci < nc; ++ci) {
        const double resPrev = rs;
        rs = res[(size_t)r * nc + ci];
        const int s = arg[(size_t)r * nc + ci];
        const double sx = s < nshift ? shiftx[s % nsx] : 0.0, sy = s < nshift ? shifty[s / nsx] : 0.0;
        if (rs > resPrev && minPflag == 1) minPeriod = cand[ci].period;
        else minPflag = 0;
        if (rs < minResInner && cand[ci].period > minPeriod) {
          minResInner = rs;
          minStoreInner = cand[ci].slot;
          minCountInner = nStore - cand[ci].icount;
          minSxInner = sx; minSyInner = sy;
        }
      }
      if (minResInner < thresh && S.recOut == 0) {
        S.minResOuter = thresh;
        S.recOut = 1;
      }
      if (minResInner < S.minResOuter && S.recOut == 1) {
        S.minResOuter = minResInner;
        S.minStoreOuter = minStoreInner;
        S.minTimeOuter = tme + minCountInner * nout * delt;
        S.minSxOuter = minSxInner; S.minSyOuter = minSyInner;
        S.recPeriod = (minCountInner * nout) * delt;
      }
      if (minResInner > thresh && S.recOut == 1) {
        S.recOut = 0;
        Guess2 g;
        const double m[7] = {(double)r, S.minTimeOuter, v2[r], S.recPeriod, S.minSxOuter,
                             S.minSyOuter, S.minResOuter};
        memcpy(g.meta, m, sizeof m);
        g.z.resize(nkt);
        PSG_CUDA_TRY(cudaMemcpy(g.z.data(), ring_full + ((size_t)r * store + S.minStoreOuter) * nkt,
                                sizeof(double2) * nkt, cudaMemcpyDeviceToHost));
        guesses.push_back(std::move(g));
        ++*emitted;
      }
    }
    return PSG_OK;
  }

  // one output interval (the ring bookkeeping of the DNS loop): check, advance, store
  int add(int nt, const void* const* st, int precision, int* emitted) {
    *emitted = 0;
    if (nStore >= 1)
      if (int rc = check(nt, emitted)) return rc;
    ++nStore;
    if (nStore >= store) {
      nStore = store;
      ++nCopy;
      nCopy -= (nCopy / store) * store;
      iStart = nCopy;
    } else {
      nCopy = nStore;
    }
    return put(nCopy, st, precision);
  }
};

}  // namespace psg

using namespace psg;

struct psg_rec2d {
  Rec2D r;
};

extern "C" int psg_rec2d_create(psg_rec2d** h, int nrun, int n, double alpha, int store_size,
                                int norm_width, int nshift_x, int nshift_y, double threshold,
                                int nout, double dt, double tstart, const double* v2) {
  if (!h) { psg_set_error("null handle"); return PSG_ERR_ARG; }
  *h = nullptr;
  psg_rec2d* p = new psg_rec2d();
  int rc = p->r.init(nrun, n, alpha, store_size, norm_width, nshift_x, nshift_y, threshold, nout,
                     dt, tstart, v2);
  if (rc) { delete p; return rc; }
  *h = p;
  return PSG_OK;
}

extern "C" void psg_rec2d_destroy(psg_rec2d* h) { delete h; }

extern "C" int psg_rec2d_set_stream(psg_rec2d* h, void* s) {
  if (!h) { psg_set_error("null handle"); return PSG_ERR_ARG; }
  h->r.stream = (cudaStream_t)s;
  return PSG_OK;
}

static int rec2d_prec_ok(int precision) {
  if (precision != 32 && precision != 64) {
    psg_set_error("2D recurrence: precision must be 32 or 64");
    return 0;
  }
  return 1;
}

extern "C" int psg_rec2d_start(psg_rec2d* h, void* const* states, int precision) {
  if (!h || !states) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  if (!rec2d_prec_ok(precision)) return PSG_ERR_ARG;
  return h->r.start((const void* const*)states, precision);
}

extern "C" int psg_rec2d_add(psg_rec2d* h, int nt, void* const* states, int precision,
                             int* emitted) {
  if (!h || !states || !emitted) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  if (!rec2d_prec_ok(precision)) return PSG_ERR_ARG;
  return h->r.add(nt, (const void* const*)states, precision, emitted);
}

extern "C" int psg_rec2d_count(psg_rec2d* h) { return h ? (int)h->r.guesses.size() : -1; }

extern "C" int psg_rec2d_guess(psg_rec2d* h, int k, double* meta, double* Z) {
  if (!h || !meta) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  if (k < 0 || k >= (int)h->r.guesses.size()) {
    psg_set_error("guess %d of %d", k, (int)h->r.guesses.size());
    return PSG_ERR_ARG;
  }
  const Rec2D::Guess2& g = h->r.guesses[k];
  memcpy(meta, g.meta, sizeof(g.meta));
  if (Z) memcpy(Z, g.z.data(), sizeof(double2) * g.z.size());
  return PSG_OK;
}

extern "C" long psg_rec2d_launches(psg_rec2d* h) { return h ? h->r.launches : -1; }
