// psg_dropin3d.cu -- reference-compatible timestep_cuda_ entry points (3D).
//
// Compiled once per flavour (-DPSG_FLAVOUR_NS3D / _NS3D_NEWTON / _EULER3D /
// _BOUS3D / _BOUS3D_DNS) into
// libpsg_<flavour>.so, because every flavour exports the same Fortran-mangled
// symbol.  The argument lists are the reference's, all by pointer; the state
// arrays are overwritten in place exactly as the reference does.  Unlike the
// reference, device buffers persist between calls (one cached engine per grid
// size), so a call costs one upload, the steps and one download.
//
// Precision: FP64 storage and transforms, the reference's, unless
// PSG_PRECISION=32 in the environment selects the FP32 engine.  A failure
// prints one line to stderr and fills the state arrays with NaN: the
// reference has no error channel, and its Newton drivers detect a failed
// integration by the NaN it leaves (2D_NavierStokes/src_RK4/src_gmres/
// main.F90:1527-1534); an unchanged state would read as Phi_T(z) = z.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include <cuda_runtime.h>

#include "../../include/psgpu.h"
#include "../../include/psgpu_ref_abi.h"
#include "psgpu_internal.h"

namespace {

struct Cached {
  psg_ns3d* h = nullptr;
  int n = 0, scheme = -1, precision = 0;
};
Cached g_cache;

int env_precision() {
  const char* s = getenv("PSG_PRECISION");
  if (s && (!strcmp(s, "32") || !strcmp(s, "fp32"))) return 32;
  return 64;
}

void report(const char* where) {
  fprintf(stderr, "psgpu_b200 %s: %s\n", where, psg_last_error());
}

// the caller's state arrays as NaN (nkt complex entries each), when nkt is sane
void fill_nan(double2* const* comps, int ncomp, long nkt) {
  if (nkt <= 0 || nkt > (1L << 31)) return;
  for (int c = 0; c < ncomp; ++c) {
    if (!comps[c]) continue;
    for (long i = 0; i < nkt; ++i) comps[c][i].x = comps[c][i].y = NAN;
  }
}

[[maybe_unused]] long box_nkt(int n) {
  const long K = n / 3;
  return (K + 1) * (2 * K + 1) * (2 * K + 1);
}

psg_ns3d* engine(int n, int scheme) {
  const int prec = env_precision();
  if (g_cache.h && g_cache.n == n && g_cache.scheme == scheme && g_cache.precision == prec)
    return g_cache.h;
  if (g_cache.h) psg_ns3d_destroy(g_cache.h);
  g_cache = Cached();
  psg_ns3d* h = nullptr;
  if (psg_ns3d_create(&h, n, 1.0, scheme, prec) != PSG_OK) return nullptr;
  g_cache.h = h; g_cache.n = n; g_cache.scheme = scheme; g_cache.precision = prec;
  return h;
}

// the sizes the drivers pass must describe a cubic 2/3-truncated box
bool check_sizes(const char* who, int IKTX, int IKTY, int IKTZ, int KTZ, int NKT, int NX,
                 int NY, int NZ, double alpha) {
  const int K = NY / 3;
  if (NX != NY || NY != NZ || alpha != 1.0 || IKTX != K + 1 || IKTY != 2 * K + 1 ||
      IKTZ != 2 * K + 1 || KTZ != K || NKT != IKTX * IKTY * IKTZ) {
    fprintf(stderr,
            "psgpu_b200 %s: unsupported sizes NX=%d NY=%d NZ=%d IKTX=%d IKTY=%d IKTZ=%d KTZ=%d "
            "NKT=%d alpha=%g (cubic 2/3-truncated boxes only)\n",
            who, NX, NY, NZ, IKTX, IKTY, IKTZ, KTZ, NKT, alpha);
    return false;
  }
  return true;
}

#if defined(PSG_FLAVOUR_BOUS3D)
// Runs [begin, end) of the reference box (in doubles, ikx fastest) that hold
// modes outside the kept set: |k| > N/3 - 1/2, and the kx = 0 half-plane's
// duplicates (ky < 0, or ky = 0 and kz <= 0) (3D_NavierStokes/src/init.F90:
// 38-57).  Built once per grid size.
const std::vector<long>& nonkept_runs(int n) {
  static int cached_n = 0;
  static std::vector<long> runs;
  if (cached_n == n) return runs;
  runs.clear();
  const int K = n / 3, X = K + 1, Y = 2 * K + 1;
  const double lim = (K - 0.5) * (K - 0.5);
  long i = 0, start = -1;
  for (int ikz = 0; ikz < Y; ++ikz)
    for (int iky = 0; iky < Y; ++iky)
      for (int ikx = 0; ikx < X; ++ikx, ++i) {
        const int ky = iky - K, kz = ikz - K;
        const bool keep = !(ikx == 0 && ky < 0) && !(ikx == 0 && ky == 0 && kz <= 0) &&
                          !((double)ikx * ikx + (double)ky * ky + (double)kz * kz > lim);
        if (!keep && start < 0) start = i;
        if (keep && start >= 0) {
          runs.push_back(2 * start);
          runs.push_back(2 * i);
          start = -1;
        }
      }
  if (start >= 0) {
    runs.push_back(2 * start);
    runs.push_back(2 * i);
  }
  cached_n = n;
  return runs;
}

bool nonkept_zero(const double* a, int n) {
  const std::vector<long>& r = nonkept_runs(n);
  for (size_t k = 0; k < r.size(); k += 2)
    for (long i = r[k]; i < r[k + 1]; ++i)
      if (a[i] != 0.0) return false;
  return true;
}

// Upload, steps() and download of an in-place call.  When the state arrays are
// page-locked and every entry outside the kept modes is zero, only the kept
// modes cross the host link (the conversion kernels read and write the host
// arrays directly; the zero check runs on the host while the device steps).
// Otherwise, or with PSG_DROPIN_FULL_COPY=1, the whole boxes are copied; both
// paths return the same state.
template <typename Steps>
int advance(psg_ns3d* h, double2* const* state, int nc, int n, Steps steps) {
  const double* in[4] = {nullptr, nullptr, nullptr, nullptr};
  double* out[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int q = 0; q < nc; ++q) {
    in[q] = (const double*)state[q];
    out[q] = (double*)state[q];
  }
  const char* full = getenv("PSG_DROPIN_FULL_COPY");
  if (!(full && atoi(full) == 1) && psg_ns3d_upload_kept(h, in) == PSG_OK) {
    if (int rc = steps()) return rc;
    bool zero = true;
    for (int q = 0; q < nc && zero; ++q) zero = nonkept_zero(in[q], n);
    if (zero) return psg_ns3d_download_kept(h, out);
    // a non-kept entry was set: once more from the whole box
    if (int rc = psg_ns3d_sync(h)) return rc;
  }
  if (int rc = psg_ns3d_upload(h, in)) return rc;
  if (int rc = steps()) return rc;
  return psg_ns3d_download(h, out);
}
#endif

#if defined(PSG_FLAVOUR_BOUS3D_DNS)
// one guess of the recurrence search in the reference's records
// (3D_Boussinesq/src/functions.h:592-609): UPO_ZK.out gets start time, v2,
// period, shifts x, y, z, residual and the four fields; UPOinfo_ts.dat a line
int write_guess(psg_rec3d* rec, FILE* zk, FILE* info, long nkt, int izkout) {
  double meta[7];
  std::vector<double> f(4 * 2 * (size_t)nkt);
  double* p = f.data();
  if (psg_rec3d_guess(rec, meta, p, p + 2 * nkt, p + 4 * nkt) ||
      psg_rec3d_guess_rho(rec, p + 6 * nkt))
    return 1;
  fwrite(meta, sizeof(double), 7, zk);
  fwrite(p, sizeof(double), f.size(), zk);
  fflush(zk);
  fprintf(info, "%d %e %e %e %e %e %e \n", izkout, meta[0], meta[2], meta[3], meta[4], meta[5],
          meta[6]);
  fflush(info);
  return 0;
}
#endif

}  // namespace

#if defined(PSG_FLAVOUR_NS3D)

extern "C" void timestep_cuda_(double2* xii, double2* eta, double2* zet, double* xir, double* etr,
                               double* ztr, double* nuzn, double* nu1, double* kx, double* ky,
                               double* kz, double* Time, double* TSTART, double* AMPFOR,
                               double* DELT, double* ResThresh, double* KFY, double* V2,
                               double* alpha, int* ikF, int* ikN, int* LC, int* IKTX, int* IKTY,
                               int* IKTZ, int* KTZ, int* NKT, int* NX, int* NY, int* NZ,
                               int* NSTOP, int* NOUT, int* NOUTV, int* statsFLAG, int* RecFLAG,
                               int* RANK) {
  (void)nuzn; (void)nu1; (void)kx; (void)ky; (void)kz; (void)ResThresh; (void)ikF; (void)ikN;
  (void)LC; (void)NOUT; (void)NOUTV; (void)statsFLAG; (void)RecFLAG; (void)RANK;
  double2* state[3] = {xii, eta, zet};
  if (!check_sizes("timestep_cuda_", *IKTX, *IKTY, *IKTZ, *KTZ, *NKT, *NX, *NY, *NZ, *alpha)) {
    fill_nan(state, 3, *NKT);
    return;
  }
  psg_ns3d* h = engine(*NX, PSG_SCHEME_NS_HEUN);
  const double* in[3] = {(const double*)xii, (const double*)eta, (const double*)zet};
  double* out[3] = {(double*)xii, (double*)eta, (double*)zet};
  double* phys[3] = {xir, etr, ztr};
  if (!h || psg_ns3d_set_params(h, *V2, *AMPFOR, *KFY, 0.0, 1.0, 0.0) ||
      psg_ns3d_upload(h, in) || psg_ns3d_step(h, *DELT, *NSTOP, 1) || psg_ns3d_download(h, out) ||
      (*NSTOP > 0 && psg_ns3d_download_phys(h, phys))) {
    report("timestep_cuda_");
    fill_nan(state, 3, *NKT);
    return;
  }
  if (*NSTOP > 0) *Time = *TSTART + (double)(*NSTOP) * (*DELT);
}

#elif defined(PSG_FLAVOUR_NS3D_NEWTON)

// The Newton-solver build's step (3D_NavierStokes/src_gmres/cuda.cu:10-176):
// 18 arguments and no sizes -- the reference fixes the grid at compile time
// in its kernels.h (128^3 as shipped).  The grid here is 128 unless
// PSG_NEWTON_N in the environment names another supported size.
extern "C" void timestep_cuda_(double2* xii, double2* eta, double2* zet, double* nuzn, double* nu1,
                               double* kx, double* ky, double* kz, double* Time, double* TSTART,
                               double* AMPFOR, double* DELT, int* KFY, double* V2, int* ikF,
                               int* ikN, int* LC, int* NSTOP) {
  (void)nuzn; (void)nu1; (void)kx; (void)ky; (void)kz; (void)ikF; (void)ikN; (void)LC;
  int n = 128;
  if (const char* e = getenv("PSG_NEWTON_N")) n = atoi(e);
  double2* state[3] = {xii, eta, zet};
  psg_ns3d* h = engine(n, PSG_SCHEME_NS_HEUN);
  const double* in[3] = {(const double*)xii, (const double*)eta, (const double*)zet};
  double* out[3] = {(double*)xii, (double*)eta, (double*)zet};
  if (!h || psg_ns3d_set_forcing_form(h, PSG_FORCING_NEWTON) ||
      psg_ns3d_set_params(h, *V2, *AMPFOR, (double)*KFY, 0.0, 1.0, 0.0) ||
      psg_ns3d_upload(h, in) || psg_ns3d_step(h, *DELT, *NSTOP, 0) || psg_ns3d_download(h, out)) {
    report("timestep_cuda_");
    // the caller's arrays hold the box of the compiled-in grid
    fill_nan(state, 3, box_nkt(n));
    return;
  }
  if (*NSTOP > 0) *Time = *TSTART + (double)(*NSTOP) * (*DELT);
}

#elif defined(PSG_FLAVOUR_EULER3D)

extern "C" void timestep_cuda_(double2* xii, double2* eta, double2* zet, double* xir, double* etr,
                               double* ztr, double* kx, double* ky, double* kz, double* Time,
                               double* TSTART, double* DELT, double* alpha, int* ikF, int* ikN,
                               int* LC, int* IKTX, int* IKTY, int* IKTZ, int* KTZ, int* NKT,
                               int* NX, int* NY, int* NZ, int* NSTOP, int* NOUT, int* NOUTV,
                               int* statsFLAG) {
  (void)kx; (void)ky; (void)kz; (void)ikF; (void)ikN; (void)LC; (void)NOUT; (void)NOUTV;
  (void)statsFLAG;
  double2* state[3] = {xii, eta, zet};
  if (!check_sizes("timestep_cuda_", *IKTX, *IKTY, *IKTZ, *KTZ, *NKT, *NX, *NY, *NZ, *alpha)) {
    fill_nan(state, 3, *NKT);
    return;
  }
  psg_ns3d* h = engine(*NX, PSG_SCHEME_EULER_HEUN);
  const double* in[3] = {(const double*)xii, (const double*)eta, (const double*)zet};
  double* out[3] = {(double*)xii, (double*)eta, (double*)zet};
  double* phys[3] = {xir, etr, ztr};
  if (!h || psg_ns3d_set_params(h, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0) || psg_ns3d_upload(h, in) ||
      psg_ns3d_step(h, *DELT, *NSTOP, 1) || psg_ns3d_download(h, out) ||
      (*NSTOP > 0 && psg_ns3d_download_phys(h, phys))) {
    report("timestep_cuda_");
    fill_nan(state, 3, *NKT);
    return;
  }
  if (*NSTOP > 0) *Time = *TSTART + (double)(*NSTOP) * (*DELT);
}

#elif defined(PSG_FLAVOUR_BOUS3D)

// Integration from TSTART to Tstep with the reference's loop: full steps while
// Tstep - t > dt, then one step of the remaining length
// (3D_Boussinesq/src/src_gmres/cuda.cu:187-250).  *Time advances by dt per full step.
extern "C" void timestep_cuda_(double2* xii, double2* eta, double2* zet, double2* rho, double* kx,
                               double* ky, double* kz, double* Time, double* TSTART,
                               double* Tstep, double* AMPFOR, double* DELT, double* ResThresh,
                               double* KFY, double* V2, double* Ri, double* Sc, double* Theta,
                               double* alpha, double* Dtarget, int* ikF, int* ikN, int* LC,
                               int* IKTX, int* IKTY, int* IKTZ, int* KTZ, int* NKT, int* NX,
                               int* NY, int* NZ, int* NOUT, int* NOUTV, int* statsFLAG,
                               int* RecFLAG, int* adaptFLAG, int* RANK) {
  (void)kx; (void)ky; (void)kz; (void)ResThresh; (void)Dtarget; (void)ikF; (void)ikN; (void)LC;
  (void)NOUT; (void)NOUTV; (void)statsFLAG; (void)RecFLAG; (void)adaptFLAG; (void)RANK;
  double2* state[4] = {xii, eta, zet, rho};
  if (!check_sizes("timestep_cuda_", *IKTX, *IKTY, *IKTZ, *KTZ, *NKT, *NX, *NY, *NZ, *alpha)) {
    fill_nan(state, 4, *NKT);
    return;
  }
  psg_ns3d* h = engine(*NX, PSG_SCHEME_BOUS_RK4);
  const double delt = *DELT;
  double tme = *TSTART;
  int nfull = 0;
  while (*Tstep - tme > delt) {
    ++nfull;
    tme += delt;
  }
  auto steps = [&]() -> int {
    if (int rc = psg_ns3d_step(h, delt, nfull, 0)) return rc;
    return tme != *Tstep ? psg_ns3d_step(h, *Tstep - tme, 1, 0) : PSG_OK;
  };
  if (!h || psg_ns3d_set_params(h, *V2, *AMPFOR, *KFY, *Ri, *Sc, *Theta) ||
      advance(h, state, 4, *NX, steps)) {
    report("timestep_cuda_");
    fill_nan(state, 4, *NKT);
    return;
  }
  for (int i = 0; i < nfull; ++i) *Time = *Time + delt;
}

// dz/dt at the given state; the state arrays receive the derivative
// (3D_Boussinesq/src/src_gmres/cuda.cu:319-533).
extern "C" void timederiv_cuda_(double2* xii, double2* eta, double2* zet, double2* rho, double* kx,
                                double* ky, double* kz, double* Time, double* TSTART,
                                double* Tstep, double* AMPFOR, double* DELT, double* ResThresh,
                                double* KFY, double* V2, double* Ri, double* Sc, double* Theta,
                                double* alpha, double* Dtarget, int* ikF, int* ikN, int* LC,
                                int* IKTX, int* IKTY, int* IKTZ, int* KTZ, int* NKT, int* NX,
                                int* NY, int* NZ, int* NOUT, int* NOUTV, int* statsFLAG,
                                int* RecFLAG, int* adaptFLAG, int* RANK) {
  (void)kx; (void)ky; (void)kz; (void)Time; (void)TSTART; (void)Tstep; (void)DELT;
  (void)ResThresh; (void)Dtarget; (void)ikF; (void)ikN; (void)LC; (void)NOUT; (void)NOUTV;
  (void)statsFLAG; (void)RecFLAG; (void)adaptFLAG; (void)RANK;
  double2* state[4] = {xii, eta, zet, rho};
  if (!check_sizes("timederiv_cuda_", *IKTX, *IKTY, *IKTZ, *KTZ, *NKT, *NX, *NY, *NZ, *alpha)) {
    fill_nan(state, 4, *NKT);
    return;
  }
  psg_ns3d* h = engine(*NX, PSG_SCHEME_BOUS_RK4);
  const double* in[4] = {(const double*)xii, (const double*)eta, (const double*)zet, (const double*)rho};
  double* out[4] = {(double*)xii, (double*)eta, (double*)zet, (double*)rho};
  if (!h || psg_ns3d_set_params(h, *V2, *AMPFOR, *KFY, *Ri, *Sc, *Theta) ||
      psg_ns3d_upload(h, in) || psg_ns3d_timederiv(h, out)) {
    report("timederiv_cuda_");
    fill_nan(state, 4, *NKT);
  }
}

#elif defined(PSG_FLAVOUR_BOUS3D_DNS)

// The Boussinesq DNS build's step (3D_Boussinesq/src/cuda.cu:21-117): the
// same 38 arguments as the Newton-solver build, a different loop.
//   * the step: delt = Tstep/nStop when nStop*DELT != Tstep (nStop = Tstep/DELT
//     in floating point), else DELT (init.h:23-29); steps while tme <= Tstep;
//   * an output time is one that the previous step crossed: a multiple of
//     Tout = NOUT*delt in (tme - delt + small, tme + small], small = 1e-10
//     (out_low.h:8-9);
//   * at output times with statsFLAG != 0 and adaptFLAG = 1, before the step:
//     delt = max(C/|Umax|, deltp), C = 2 pi/NX, deltp the initial delt,
//     Umax = max |u| of the physical x-velocity (out_low.h:11-16);
//   * at output times with statsFLAG = 1 (or 2 past t = 50), after the step,
//     the forcing throttle ampfor *= (Dtarget - bflux)/input from the state's
//     buoyancy flux bflux = Ri sum Re(conj(v sin(theta) + w cos(theta)) rho) and
//     energy input input = -ampfor Re zeta(0, kf, 0)/kf (functions.h:288-369);
//   * with Dtarget != 0 the device forcing amplitude is set to the host's
//     ampfor after every step (cuda.cu:104-106).  The host copy starts as
//     -AMPFOR (init.h:18) while the device starts from AMPFOR (init.h:138), so
//     from the first step on the forcing acts with the host's sign, as it
//     does in the reference.
//   * RecFLAG = 1: the recurrence search for UPO guesses at output times, the
//     DNS's Boussinesq variant (4 fields, storeSize 500, normWidth 8, 64 x 1 x 1
//     trial shifts: 3D_Boussinesq/src/kernels.h:12-16, functions.h:416-616),
//     with the initial state stored first (init.h:268-296); guesses go to
//     JOB<RANK>/UPO_ZK.out and JOB<RANK>/UPOinfo_ts.dat in the reference's
//     record layout.  The periods are counted in the initial delt.  The
//     reference's check also assigns the loop's time variable,
//     tme = tstart + (NT - nOut) delt (functions.h:501), which sets the loop
//     back NOUT steps at the first check and so runs NOUT more steps; the same
//     assignment is made here.
// The DNS's other diagnostic files (stats.dat, engy.dat, spectra, RiG, pdfs,
// raw volumes) are not written.
extern "C" void timestep_cuda_(double2* xii, double2* eta, double2* zet, double2* rho, double* kx,
                               double* ky, double* kz, double* Time, double* TSTART,
                               double* Tstep, double* AMPFOR, double* DELT, double* ResThresh,
                               double* KFY, double* V2, double* Ri, double* Sc, double* Theta,
                               double* alpha, double* Dtarget, int* ikF, int* ikN, int* LC,
                               int* IKTX, int* IKTY, int* IKTZ, int* KTZ, int* NKT, int* NX,
                               int* NY, int* NZ, int* NOUT, int* NOUTV, int* statsFLAG,
                               int* RecFLAG, int* adaptFLAG, int* RANK) {
  (void)kx; (void)ky; (void)kz; (void)ikF; (void)ikN; (void)LC; (void)NOUTV;
  double2* state[4] = {xii, eta, zet, rho};
  if (!check_sizes("timestep_cuda_", *IKTX, *IKTY, *IKTZ, *KTZ, *NKT, *NX, *NY, *NZ, *alpha) ||
      *NOUT < 1) {
    fill_nan(state, 4, *NKT);
    return;
  }
  psg_ns3d* h = engine(*NX, PSG_SCHEME_BOUS_RK4);
  const double* in[4] = {(const double*)xii, (const double*)eta, (const double*)zet, (const double*)rho};
  double* out[4] = {(double*)xii, (double*)eta, (double*)zet, (double*)rho};
  const double small = 1e-10, twopi = 4.0 * asin(1.0);
  const double nstop = *Tstep / *DELT;
  double delt = (nstop * *DELT != *Tstep) ? *Tstep / nstop : *DELT;
  const double C = twopi / *NX, Tout = *NOUT * delt, deltp = delt;
  double tme = *TSTART;
  double ampfor = -*AMPFOR;       // host copy
  double dev_ampfor = *AMPFOR;    // device copy
  const double dtarget = *Dtarget, kfy = *KFY, ri = *Ri;
  auto fail = [&]() {
    report("timestep_cuda_");
    fill_nan(state, 4, *NKT);
  };
  if (!h || psg_ns3d_set_params(h, *V2, dev_ampfor, kfy, ri, *Sc, *Theta) ||
      psg_ns3d_upload(h, in)) {
    fail();
    return;
  }
  psg_rec3d* rec = nullptr;
  FILE* upozk = nullptr;
  FILE* upoinfo = nullptr;
  int izkout = 0, rec_outputs = 0;
  auto close_rec = [&]() {
    if (rec) psg_rec3d_destroy(rec);
    if (upozk) fclose(upozk);
    if (upoinfo) fclose(upoinfo);
    rec = nullptr; upozk = upoinfo = nullptr;
  };
  if (*RecFLAG == 1) {
    char fn[64];
    snprintf(fn, sizeof fn, "JOB%1d/UPO_ZK.out", *RANK);
    upozk = fopen(fn, "wb");
    snprintf(fn, sizeof fn, "JOB%1d/UPOinfo_ts.dat", *RANK);
    upoinfo = fopen(fn, "w");
    if (upoinfo)
      fprintf(upoinfo, "Guess No : Start time : guess Period : guess Shift x: guess Shift y: guess Residual \n");
    if (!upozk || !upoinfo ||
        psg_rec3d_create_bous(&rec, *NX, *alpha, 500, 8, 64, 1, 1, *ResThresh, *NOUT, delt, tme,
                              *V2, ri) ||
        psg_rec3d_start_engine(rec, h)) {
      if (!upozk || !upoinfo) psg_set_error("cannot open JOB%d/UPO_ZK.out or UPOinfo_ts.dat", *RANK);
      close_rec();
      fail();
      return;
    }
  }
  int timestep = 0;
  while (tme <= *Tstep) {
    ++timestep;
    const double tcrit = Tout * (double)(int)((tme + small) / Tout);
    const double tcheck = (tme - delt - tcrit + small) * (tme + small - tcrit);
    if (tcheck < 0.0 && *statsFLAG != 0 && *adaptFLAG == 1) {
      double umax = 0.0;
      if (psg_ns3d_max_velocity(h, &umax)) { fail(); return; }
      delt = fmax(C / fabs(umax), deltp);
    }
    if (psg_ns3d_step(h, delt, 1, 0)) { fail(); return; }
    *Time = *Time + delt;
    tme += delt;
    if (tcheck < 0.0 && (*RecFLAG == 1 || *statsFLAG != 0) && timestep != 0) {
      if (rec) {
        int emitted = 0;
        const bool checks = rec_outputs++ > 0;  // the first output only stores
        if (psg_rec3d_add_engine(rec, timestep, h, &emitted)) { close_rec(); fail(); return; }
        if (emitted && write_guess(rec, upozk, upoinfo, *NKT, ++izkout)) {
          close_rec();
          fail();
          return;
        }
        if (checks) tme = *TSTART + (timestep - *NOUT) * delt;
      }
      if (*statsFLAG == 1 || (*statsFLAG == 2 && tme > 50.0)) {
        double fl[2];
        if (psg_ns3d_buoyancy_flux(h, fl)) { close_rec(); fail(); return; }
        const double bflux = ri * fl[0];
        const double input = -ampfor * fl[1] / kfy;
        if (dtarget != 0.0) ampfor = ampfor * (dtarget - bflux) / input;
      }
    }
    if (*Dtarget != 0 && dev_ampfor != ampfor) {
      dev_ampfor = ampfor;
      if (psg_ns3d_set_params(h, *V2, dev_ampfor, kfy, ri, *Sc, *Theta)) { close_rec(); fail(); return; }
    }
  }
  close_rec();
  if (psg_ns3d_download(h, out)) fail();
}

#else
#error "define PSG_FLAVOUR_NS3D, PSG_FLAVOUR_EULER3D or PSG_FLAVOUR_BOUS3D"
#endif

// set_gpu_: the Navier-Stokes and Euler builds only report the current device
// (3D_NavierStokes/src/functions.h:3-20); the Boussinesq build selects device
// *go (3D_Boussinesq/src/functions.h:9-28).
extern "C" void set_gpu_(int* go) {
  int count = 0, dev = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    printf("cutil error: no devices supporting CUDA\n");
    exit(-1);
  }
#if defined(PSG_FLAVOUR_BOUS3D) || defined(PSG_FLAVOUR_BOUS3D_DNS)
  dev = *go;
  cudaSetDevice(dev);
#else
  (void)go;
  cudaGetDevice(&dev);
#endif
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  printf("\n Using CUDA device %d: %s\n\n", dev, prop.name);
}
