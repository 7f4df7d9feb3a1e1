// psg_recurrence.cu -- near-recurrence search for UPO guesses on the GPU.
//
// Restates the 3D DNS's recurrence check (3D_NavierStokes/src/functions.h:
// 111-389, set up in init.h:182-213, driven from cuda.cu:116-138): every NOUT
// steps the newest stored state is compared, under every trial shift of a
// grid of NSHIFTX x NSHIFTY x NSHIFTZ translations, with the earlier states of
// a ring of storeSize; the comparison uses the modes of a low-wavenumber box
// (|kx| < W, |ky|, |kz| < W around the origin, 4 W^3 modes).  The residuals of
// all (earlier state, shift) pairs are one kernel launch; the reference's
// selection logic (first turning point in the period, minimum over periods,
// entering and leaving the threshold) runs on the host over those residuals,
// in the reference's order.  The ring of full states stays on the device.
//
// The Boussinesq DNS's variant (3D_Boussinesq/src/functions.h:189-205,
// 416-616, driven from out_high.h:5-40) carries the density as a fourth
// field: its residual weights the density terms by Ri, normalises by the sum
// of both states' norms, skips periods below 0.5, and takes the norm over
// the whole box without the mask, with Ri on the real part of the density
// only (computeNorm, functions.h:202, as written).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "psg_common.cuh"
#include "psgpu_internal.h"

typedef struct psg_ns3d psg_ns3d;

namespace psg {

// the comparison box of the newest state and its norm: the Navier-Stokes
// form sums the three vorticity components over the kept modes
// (3D_NavierStokes/src/functions.h:111-126); the Boussinesq form (nc = 4)
// sums over the whole box with ri * Re(rho)^2 + Im(rho)^2 for the density
// (3D_Boussinesq/src/functions.h:189-205)
__global__ void rec_gather(const double2* __restrict__ full, long nkt, int nc, double ri,
                           const int* __restrict__ inorm, const unsigned char* __restrict__ ll,
                           int nnorm, double2* __restrict__ sub, double* __restrict__ norm) {
  __shared__ double r[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < nnorm; i += blockDim.x) {
    const int ik = inorm[i];
    double v = 0.0;
    for (int q = 0; q < nc; ++q) {
      const double2 x = full[q * nkt + ik];
      sub[q * nnorm + i] = x;
      v += (q == 3) ? ri * x.x * x.x + x.y * x.y : x.x * x.x + x.y * x.y;
    }
    if (nc == 4 || ll[ik]) s += v;
  }
  r[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) r[threadIdx.x] += r[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *norm = r[0];
}

// shifted copies of the newest state's box: z exp(-i (kx sx + ky sy + kz sz))
// (computeZdash, functions.h:212-249), shift s fastest in x, then z, then y
__global__ void rec_dash(const double2* __restrict__ sub, const double* __restrict__ kxyz,
                         const double* __restrict__ shifts, int nsx, int nsy, int nsz, int nnorm,
                         int nc, double2* __restrict__ dash) {
  const int s = blockIdx.y;
  const int isx = s % nsx, isz = (s / nsx) % nsz, isy = s / (nsx * nsz);
  const double sx = shifts[isx], sy = shifts[nsx + isy], sz = shifts[nsx + nsy + isz];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnorm; i += gridDim.x * blockDim.x) {
    const double sh = kxyz[i] * sx + kxyz[nnorm + i] * sy + kxyz[2 * nnorm + i] * sz;
    double sn, cs;
    sincos(sh, &sn, &cs);
    for (int q = 0; q < nc; ++q) {
      const double2 z = sub[q * nnorm + i];
      dash[((long)s * nc + q) * nnorm + i] = make_double2(cs * z.x + sn * z.y, cs * z.y - sn * z.x);
    }
  }
}

// res2[c][s] = -2 <dash_s, old_c> + |dash_s|^2 + norm(old_c), the density
// terms (fourth field) weighted by ri
__global__ void rec_resid(const double2* __restrict__ dash, const double2* __restrict__ ring,
                          const int* __restrict__ cand, const double* __restrict__ norms,
                          int nnorm, int nshift, int nc, double ri, double* __restrict__ res2) {
  const int s = blockIdx.x, ci = blockIdx.y;
  const int slot = cand[ci];
  const double2* d = dash + (long)s * nc * nnorm;
  const double2* o = ring + (long)slot * nc * nnorm;
  double cross = 0.0, nd = 0.0;
  for (int i = threadIdx.x; i < nc * nnorm; i += blockDim.x) {
    const double2 x = d[i], y = o[i];
    const double w = (i >= 3 * nnorm) ? ri : 1.0;
    cross += w * (x.x * y.x + x.y * y.y);
    nd += w * (x.x * x.x + x.y * x.y);
  }
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = cross;
  r2[threadIdx.x] = nd;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      r1[threadIdx.x] += r1[threadIdx.x + h];
      r2[threadIdx.x] += r2[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) res2[(long)ci * nshift + s] = -2.0 * r1[0] + r2[0] + norms[slot];
}

struct Rec3D {
  int n = 0, K = 0, X = 0, Y = 0, store = 0, nw = 0, nnorm = 0, nsx = 0, nsy = 0, nsz = 0;
  int nc = 3;       // 3: Navier-Stokes; 4: Boussinesq (density as the fourth field)
  double ri = 0.0;  // Boussinesq weight of the density terms
  long nkt = 0;
  double alpha = 1.0, thresh = 0.0, delt = 0.0, tstart = 0.0, v2 = 0.0, freq2 = 0.0;
  int nout = 1;
  cudaStream_t stream = 0;
  // device
  double2* ring_full = nullptr;  // [store][nc][nkt]
  double2* ring_sub = nullptr;   // [store][nc][nnorm]
  double2* dash = nullptr;       // [nshift][nc][nnorm]
  double* d_norms = nullptr;     // [store]
  double* d_kxyz = nullptr;      // [3][nnorm]
  double* d_shifts = nullptr;
  int* d_inorm = nullptr;
  unsigned char* d_ll = nullptr;
  int* d_cand = nullptr;
  double* d_res2 = nullptr;
  double2* staging = nullptr;    // a state taken from an engine
  long launches = 0;
  // host state of the reference's bookkeeping (cuda.cu:116-138, functions.h globals)
  std::vector<double> shiftx, shifty, shiftz, norms;
  int nStore = 0, nCopy = 0, iStart = 0, recOut = 0, minStoreOuter = 0, guesses = 0;
  double minResOuter = 0.0, minTimeOuter = 0.0, recPeriod = 0.0;
  double minSxInner = 0.0, minSyInner = 0.0, minSzInner = 0.0;
  double minSxOuter = 0.0, minSyOuter = 0.0, minSzOuter = 0.0;
  // the last emitted guess
  int have_guess = 0;
  double gmeta[7] = {0};
  int gslot = 0;

  ~Rec3D() {
    void* ps[] = {ring_full, ring_sub, dash, d_norms, d_kxyz, d_shifts, d_inorm, d_ll, d_cand, d_res2,
                  staging};
    for (void* p : ps)
      if (p) cudaFree(p);
  }

  int init(int n_, double alpha_, int store_, int nw_, int nsx_, int nsy_, int nsz_, double th,
           int nout_, double delt_, double tstart_, double v2_, int nc_ = 3, double ri_ = 0.0) {
    nc = nc_; ri = ri_;
    n = n_; K = n / 3; X = K + 1; Y = 2 * K + 1; nkt = (long)X * Y * Y;
    store = store_; nw = nw_; nsx = nsx_; nsy = nsy_; nsz = nsz_;
    alpha = alpha_; thresh = th; nout = nout_; delt = delt_; tstart = tstart_; v2 = v2_;
    if (n < 8 || store < 2 || nw < 1 || nw > K || nw > X || nsx < 1 || nsy < 1 || nsz < 1 ||
        nout < 1) {
      psg_set_error("recurrence: bad sizes");
      return PSG_ERR_ARG;
    }
    freq2 = 2 * nout * delt;  // init.h:19
    nnorm = 4 * nw * nw * nw;
    // index box of init.h:184-191 (centred on KTZ in y and z)
    std::vector<int> inorm(nnorm);
    std::vector<double> kxyz(3 * (size_t)nnorm);
    for (int iz = 0; iz < 2 * nw; ++iz)
      for (int iy = 0; iy < 2 * nw; ++iy)
        for (int ix = 0; ix < nw; ++ix) {
          const int i = (iz * 2 * nw + iy) * nw + ix;
          const int ikz = K - nw + iz, iky = K - nw + iy;
          inorm[i] = (ikz * Y + iky) * X + ix;
          kxyz[i] = ix * alpha;
          kxyz[nnorm + i] = iky - K;
          kxyz[2 * nnorm + i] = ikz - K;
        }
    std::vector<unsigned char> ll(nkt);
    for (int ikz = 0; ikz < Y; ++ikz)
      for (int iky = 0; iky < Y; ++iky)
        for (int ikx = 0; ikx < X; ++ikx) {
          const double kx = ikx * alpha, ky = iky - K, kz = ikz - K;
          bool keep = !(kx == 0.0 && ky < 0.0) && !(kx == 0.0 && ky == 0.0 && kz <= 0.0) &&
                      sqrt(kx * kx + ky * ky + kz * kz) <= K - 0.5;
          ll[((long)ikz * Y + iky) * X + ikx] = keep;
        }
    // trial shifts (init.h:202-210)
    const double twopi = 4.0 * asin(1.0);
    for (int i = 0; i < nsx; ++i) shiftx.push_back(twopi * i / (nsx * alpha));
    for (int i = 0; i < nsy; ++i) shifty.push_back(twopi * i / nsy);
    for (int i = 0; i < nsz; ++i) shiftz.push_back(twopi * i / nsz);
    std::vector<double> sh(shiftx);
    sh.insert(sh.end(), shifty.begin(), shifty.end());
    sh.insert(sh.end(), shiftz.begin(), shiftz.end());
    norms.assign(store, 0.0);
    const int nshift = nsx * nsy * nsz;
    PSG_CUDA_TRY(cudaMalloc(&ring_full, sizeof(double2) * (size_t)store * nc * nkt));
    PSG_CUDA_TRY(cudaMalloc(&ring_sub, sizeof(double2) * (size_t)store * nc * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&dash, sizeof(double2) * (size_t)nshift * nc * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&d_norms, sizeof(double) * store));
    PSG_CUDA_TRY(cudaMalloc(&d_kxyz, sizeof(double) * 3 * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&d_shifts, sizeof(double) * sh.size()));
    PSG_CUDA_TRY(cudaMalloc(&d_inorm, sizeof(int) * nnorm));
    PSG_CUDA_TRY(cudaMalloc(&d_ll, nkt));
    PSG_CUDA_TRY(cudaMalloc(&d_cand, sizeof(int) * store));
    PSG_CUDA_TRY(cudaMalloc(&d_res2, sizeof(double) * (size_t)store * nshift));
    PSG_CUDA_TRY(cudaMemset(d_norms, 0, sizeof(double) * store));
    PSG_CUDA_TRY(cudaMemcpy(d_kxyz, kxyz.data(), sizeof(double) * 3 * nnorm, cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMemcpy(d_shifts, sh.data(), sizeof(double) * sh.size(), cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMemcpy(d_inorm, inorm.data(), sizeof(int) * nnorm, cudaMemcpyHostToDevice));
    PSG_CUDA_TRY(cudaMemcpy(d_ll, ll.data(), nkt, cudaMemcpyHostToDevice));
    return PSG_OK;
  }

  // copy a state (nc device FP64 boxes) into ring slot `slot` and its box
  int put(int slot, const void* const* st) {
    for (int q = 0; q < nc; ++q)
      PSG_CUDA_TRY(cudaMemcpyAsync(ring_full + ((size_t)slot * nc + q) * nkt, st[q],
                                   sizeof(double2) * nkt, cudaMemcpyDeviceToDevice, stream));
    const double2* base = ring_full + (size_t)slot * nc * nkt;
    rec_gather<<<1, 256, 0, stream>>>(base, nkt, nc, ri, d_inorm, d_ll, nnorm,
                                      ring_sub + (size_t)slot * nc * nnorm, d_norms + slot);
    ++launches;
    PSG_CUDA_TRY(cudaGetLastError());
    PSG_CUDA_TRY(cudaMemcpyAsync(&norms[slot], d_norms + slot, sizeof(double),
                                 cudaMemcpyDeviceToHost, stream));
    PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    return PSG_OK;
  }

  // the initial state into slot 0 (init.h:171-176, 211-212)
  int start(const void* const* st) {
    nStore = 0; nCopy = 0; iStart = 0; recOut = 0; minResOuter = 0.0; have_guess = 0;
    return put(0, st);
  }

  // recurrence_check (functions.h:251-389) of the newest stored state
  int check(int nt, int* emitted) {
    const double tme = tstart + (nt - nout) * delt;
    struct Cand { int icount, slot; double period; };
    std::vector<Cand> cand;
    for (int icount = nStore - 1; icount >= 1; --icount) {
      const double period = ((nStore - icount) * nout) * delt;
      int slot = icount + iStart;
      slot -= (int)floor((double)slot / store) * store;
      if (nc == 4 && period < 0.5) continue;  // 3D_Boussinesq/src/functions.h:513
      if (period > 20.0 && fabs(period - freq2 * floor(period / freq2 + 0.5)) > 0.0001) continue;
      cand.push_back(Cand{icount, slot, period});
    }
    const int nshift = nsx * nsy * nsz;
    std::vector<double> res2((size_t)cand.size() * nshift);
    if (!cand.empty()) {
      std::vector<int> slots;
      for (const Cand& c : cand) slots.push_back(c.slot);
      PSG_CUDA_TRY(cudaMemcpyAsync(d_cand, slots.data(), sizeof(int) * slots.size(),
                                   cudaMemcpyHostToDevice, stream));
      rec_dash<<<dim3((nnorm + 255) / 256, nshift), 256, 0, stream>>>(
          ring_sub + (size_t)nCopy * nc * nnorm, d_kxyz, d_shifts, nsx, nsy, nsz, nnorm, nc, dash);
      rec_resid<<<dim3(nshift, (unsigned)cand.size()), 256, 0, stream>>>(
          dash, ring_sub, d_cand, d_norms, nnorm, nshift, nc, ri, d_res2);
      launches += 2;
      PSG_CUDA_TRY(cudaGetLastError());
      PSG_CUDA_TRY(cudaMemcpyAsync(res2.data(), d_res2, sizeof(double) * res2.size(),
                                   cudaMemcpyDeviceToHost, stream));
      PSG_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    double minResInner = 10000.0, minPeriod = 10000.0, res = 0.0;
    int minPflag = 1, minStoreInner = 0, minCountInner = 0;
    for (size_t ci = 0; ci < cand.size(); ++ci) {
      const double resPrev = res;
      res = 10000.0;
      double sx = 0, sy = 0, sz = 0;
      // shifts in the reference's loop order: y outer, then z, then x
      for (int iy = 0; iy < nsy; ++iy)
        for (int iz = 0; iz < nsz; ++iz)
          for (int ix = 0; ix < nsx; ++ix) {
            const int s = ix + nsx * (iz + nsz * iy);
            // Boussinesq: normalised by both states' norms (functions.h:546)
            const double den = nc == 4 ? norms[cand[ci].slot] + norms[nCopy] : norms[nCopy];
            const double r = sqrt(res2[ci * nshift + s] / den);
            if (r < res) { res = r; sx = shiftx[ix]; sy = shifty[iy]; sz = shiftz[iz]; }
          }
      if (res > resPrev && minPflag == 1) minPeriod = cand[ci].period;
      else minPflag = 0;
      if (res < minResInner && cand[ci].period > minPeriod) {
        minResInner = res;
        minStoreInner = cand[ci].slot;
        minCountInner = nStore - cand[ci].icount;
        minSxInner = sx; minSyInner = sy; minSzInner = sz;
      }
    }
    *emitted = 0;
    if (minResInner < thresh && recOut == 0) {
      minResOuter = thresh;
      recOut = 1;
    }
    if (minResInner < minResOuter && recOut == 1) {
      minResOuter = minResInner;
      minStoreOuter = minStoreInner;
      minTimeOuter = tme + minCountInner * nout * delt;
      minSxOuter = minSxInner; minSyOuter = minSyInner; minSzOuter = minSzInner;
      recPeriod = (minCountInner * nout) * delt;
    }
    if (minResInner > thresh && recOut == 1) {
      recOut = 0;
      const double m[7] = {minTimeOuter, v2, recPeriod, minSxOuter, minSyOuter, minSzOuter,
                           minResOuter};
      memcpy(gmeta, m, sizeof m);
      gslot = minStoreOuter;
      have_guess = 1;
      ++guesses;
      *emitted = 1;
    }
    return PSG_OK;
  }

  // one output interval (cuda.cu:116-138): check, advance the ring, store
  int add(int nt, const void* const* st, int* emitted) {
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
    return put(nCopy, st);
  }
};

}  // namespace psg

using namespace psg;

struct psg_rec3d {
  Rec3D r;
};

extern "C" int psg_rec3d_create(psg_rec3d** h, int n, double alpha, int store_size, int norm_width,
                                int nshift_x, int nshift_y, int nshift_z, double threshold,
                                int nout, double dt, double tstart, double v2) {
  if (!h) { psg_set_error("null handle"); return PSG_ERR_ARG; }
  *h = nullptr;
  psg_rec3d* p = new psg_rec3d();
  int rc = p->r.init(n, alpha, store_size, norm_width, nshift_x, nshift_y, nshift_z, threshold,
                     nout, dt, tstart, v2);
  if (rc) { delete p; return rc; }
  *h = p;
  return PSG_OK;
}

// the Boussinesq DNS's variant: states of four fields (xii, eta, zet, rho)
extern "C" int psg_rec3d_create_bous(psg_rec3d** h, int n, double alpha, int store_size,
                                     int norm_width, int nshift_x, int nshift_y, int nshift_z,
                                     double threshold, int nout, double dt, double tstart,
                                     double v2, double ri) {
  if (!h) { psg_set_error("null handle"); return PSG_ERR_ARG; }
  *h = nullptr;
  psg_rec3d* p = new psg_rec3d();
  int rc = p->r.init(n, alpha, store_size, norm_width, nshift_x, nshift_y, nshift_z, threshold,
                     nout, dt, tstart, v2, 4, ri);
  if (rc) { delete p; return rc; }
  *h = p;
  return PSG_OK;
}

extern "C" void psg_rec3d_destroy(psg_rec3d* h) { delete h; }

extern "C" int psg_rec3d_set_stream(psg_rec3d* h, void* s) {
  if (!h) { psg_set_error("null handle"); return PSG_ERR_ARG; }
  h->r.stream = (cudaStream_t)s;
  return PSG_OK;
}

extern "C" int psg_rec3d_start(psg_rec3d* h, void* const* state) {
  if (!h || !state) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  return h->r.start((const void* const*)state);
}

extern "C" int psg_rec3d_add(psg_rec3d* h, int nt, void* const* state, int* emitted) {
  if (!h || !state || !emitted) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  return h->r.add(nt, (const void* const*)state, emitted);
}

extern "C" int psg_rec3d_guess(psg_rec3d* h, double* meta, double* xii, double* eta, double* zet) {
  if (!h || !meta) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  if (!h->r.have_guess) { psg_set_error("no guess emitted yet"); return PSG_ERR_STATE; }
  memcpy(meta, h->r.gmeta, sizeof(h->r.gmeta));
  double* out[3] = {xii, eta, zet};
  for (int q = 0; q < 3; ++q)
    if (out[q]) {
      cudaError_t e = cudaMemcpy(out[q], h->r.ring_full + ((size_t)h->r.gslot * h->r.nc + q) * h->r.nkt,
                                 sizeof(double2) * h->r.nkt, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { psg_set_error("guess copy: %s", cudaGetErrorString(e)); return PSG_ERR_CUDA; }
    }
  return PSG_OK;
}

// the density of the last guess (Boussinesq variant)
extern "C" int psg_rec3d_guess_rho(psg_rec3d* h, double* rho) {
  if (!h || !rho) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  if (h->r.nc != 4) { psg_set_error("not the Boussinesq variant"); return PSG_ERR_STATE; }
  if (!h->r.have_guess) { psg_set_error("no guess emitted yet"); return PSG_ERR_STATE; }
  cudaError_t e = cudaMemcpy(rho, h->r.ring_full + ((size_t)h->r.gslot * 4 + 3) * h->r.nkt,
                             sizeof(double2) * h->r.nkt, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { psg_set_error("guess copy: %s", cudaGetErrorString(e)); return PSG_ERR_CUDA; }
  return PSG_OK;
}

// the same, taking the state from a 3D engine (FP64 boxes staged on the device)
extern "C" int psg_ns3d_download_device(psg_ns3d* h, void* const* comps);

static int engine_state(psg_rec3d* h, psg_ns3d* eng, void** ptrs) {
  Rec3D& r = h->r;
  if (!r.staging) PSG_CUDA_TRY(cudaMalloc(&r.staging, sizeof(double2) * 4 * r.nkt));
  for (int q = 0; q < 4; ++q) ptrs[q] = r.staging + q * r.nkt;
  if (int rc = psg_ns3d_download_device(eng, ptrs)) return rc;
  PSG_CUDA_TRY(cudaDeviceSynchronize());
  return PSG_OK;
}

extern "C" int psg_rec3d_start_engine(psg_rec3d* h, psg_ns3d* eng) {
  if (!h || !eng) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  void* p[4];
  if (int rc = engine_state(h, eng, p)) return rc;
  return h->r.start((const void* const*)p);
}

extern "C" int psg_rec3d_add_engine(psg_rec3d* h, int nt, psg_ns3d* eng, int* emitted) {
  if (!h || !eng || !emitted) { psg_set_error("null argument"); return PSG_ERR_ARG; }
  void* p[4];
  if (int rc = engine_state(h, eng, p)) return rc;
  return h->r.add(nt, (const void* const*)p, emitted);
}

extern "C" int psg_rec3d_count(psg_rec3d* h) { return h ? h->r.guesses : -1; }
extern "C" long psg_rec3d_launches(psg_rec3d* h) { return h ? h->r.launches : -1; }
