/* psg_host.c -- host-side pieces of psgpu's drivers (include/psgpu_host.h).
 *
 * Plain C, no GPU: the parameter file, the drivers' random-number generator
 * and random starts, Fortran sequential-record I/O, restart files and the
 * 3D DNS statistics lines.  Each function cites the Fortran or CUDA host code
 * whose behaviour it restates. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "psgpu_host.h"

void psg_set_error(const char* fmt, ...);

static int set_err(const char* msg) {
  psg_set_error("%s", msg);
  return -1;
}

/* ------------------------------------------------------------ parameters */

static int next_line(FILE* f, char* buf, size_t cap) {
  if (!fgets(buf, (int)cap, f)) return -1;
  size_t n = strlen(buf);
  while (n && (buf[n - 1] == '\n' || buf[n - 1] == '\r')) buf[--n] = 0;
  return 0;
}

/* the text after `label` on the next line (read_label, parameters.F90:43-59) */
static const char* labelled(FILE* f, const char* label, char* buf, size_t cap) {
  if (next_line(f, buf, cap)) {
    psg_set_error("params: missing line for label '%s'", label);
    return NULL;
  }
  size_t n = strlen(label);
  if (strncmp(buf, label, n) != 0) {
    psg_set_error("params: bad label, expected '%s' in '%s'", label, buf);
    return NULL;
  }
  return buf + n;
}

/* Fortran Iw input: the first w columns, blanks ignored */
static int field_int(const char* s, int w, int* v) {
  char t[64];
  int k = 0;
  for (int i = 0; i < w && s[i]; ++i)
    if (s[i] != ' ') t[k++] = s[i];
  t[k] = 0;
  if (!k) { *v = 0; return 0; }
  char* end;
  long x = strtol(t, &end, 10);
  if (*end) return -1;
  *v = (int)x;
  return 0;
}

/* Fortran Fw.d input: the first w columns; without a decimal point the last
 * d digits are the fraction (F12.4 reads "50" as 0.0050); D exponents allowed */
static int field_float(const char* s, int w, int d, double* v) {
  char t[64];
  int k = 0, point = 0;
  for (int i = 0; i < w && s[i]; ++i) {
    char c = s[i];
    if (c == ' ') continue;
    if (c == 'd' || c == 'D') c = 'e';
    if (c == '.' || c == 'e' || c == 'E') point = 1;
    t[k++] = c;
  }
  t[k] = 0;
  if (!k) { *v = 0.0; return 0; }
  char* end;
  double x = strtod(t, &end);
  if (*end) return -1;
  *v = point ? x : x / pow(10.0, d);
  return 0;
}

static void copy_string(char* dst, const char* src) {
  size_t n = strlen(src);
  while (n && src[n - 1] == ' ') --n;
  if (n > 255) n = 255;
  memcpy(dst, src, n);
  dst[n] = 0;
}

int psg_read_params3d(const char* path, psg_params3d* p) {
  FILE* f = fopen(path, "r");
  if (!f) { psg_set_error("params: cannot open %s", path); return -1; }
  memset(p, 0, sizeof(*p));
  char buf[512];
  const char* r;
  int bad = 0;
#define PI_(label, dst) \
  if (!bad) { r = labelled(f, label, buf, sizeof buf); bad = !r || field_int(r, 10, &(dst)); }
#define PF_(label, dst) \
  if (!bad) { r = labelled(f, label, buf, sizeof buf); bad = !r || field_float(r, 12, 4, &(dst)); }
#define PS_(label, dst) \
  if (!bad) { r = labelled(f, label, buf, sizeof buf); bad = !r; if (r) copy_string(dst, r); }
  /* order of params_read_txt, 3D_NavierStokes/src/parameters.F90:139-155 */
  PI_("ISEED = ", p->iseed);
  PI_("IREST = ", p->irest);
  PS_("infile = ", p->infile);
  PS_("infile type = ", p->infile_type);
  PI_("KF = ", p->kf);
  PF_("Re = ", p->re);
  PF_("TSTEP = ", p->tstep);
  PF_("ResidualThreshold = ", p->residual_threshold);
  PF_("outfreq1 = ", p->outfreq1);
  PF_("outfreq2 = ", p->outfreq2);
  PF_("DELT = ", p->delt);
  PF_("AMPV = ", p->ampv);
  PI_("STATSFLAG = ", p->statsflag);
  PI_("RCFLAG = ", p->rcflag);
  PI_("UPOflag = ", p->upoflag);
  PI_("ISTOP = ", p->istop);
#undef PI_
#undef PF_
#undef PS_
  fclose(f);
  if (bad) {
    if (r) psg_set_error("params: unreadable value in '%s'", buf);
    return -1;
  }
  /* params_update, parameters.F90:28-40 (INT() truncates toward zero) */
  p->v2 = 1.0 / p->re;
  p->ampfor = -0.25 * p->kf * p->kf;
  p->nstop = (int)(p->tstep / p->delt);
  p->nout = (int)(p->outfreq1 / p->delt);
  p->noutv = (int)(p->outfreq2 / p->delt);
  /* main.F90:45-46 */
  if (p->nout == 0) p->nout = 1;
  if (p->noutv == 0) p->noutv = 1;
  return 0;
}

/* ------------------------------------------------------- random numbers */

void psg_ranno_init(psg_ranno_state* s) { memset(s, 0, sizeof(*s)); }

/* ran1 (3D_NavierStokes/src/init.F90:260-285): minimal standard generator,
 * x <- 16807 x mod (2^31 - 1) by Schrage's method, shuffled through a
 * 32-entry table; reseeds whenever called with a non-positive argument. */
static double ran1(psg_ranno_state* s, int* idum) {
  const int ia = 16807, im = 2147483647, iq = 127773, ir = 2836, ntab = 32;
  const int ndiv = 1 + (im - 1) / ntab;
  const double am = 1.0 / im, eps = 1.2e-7, rnmx = 1.0 - eps;
  int k, j;
  if (*idum <= 0 || s->iy == 0) {
    *idum = (-*idum > 1) ? -*idum : 1;
    for (j = ntab + 8; j >= 1; --j) {
      k = *idum / iq;
      *idum = ia * (*idum - k * iq) - ir * k;
      if (*idum < 0) *idum += im;
      if (j <= ntab) s->iv[j - 1] = *idum;
    }
    s->iy = s->iv[0];
  }
  k = *idum / iq;
  *idum = ia * (*idum - k * iq) - ir * k;
  if (*idum < 0) *idum += im;
  j = 1 + s->iy / ndiv;
  s->iy = s->iv[j - 1];
  s->iv[j - 1] = *idum;
  const double r = am * s->iy;
  return r < rnmx ? r : rnmx;
}

/* ranno (init.F90:236-257): seed with i != 0, else draw with the next seed
 * of the counter (junk - 1), as (ran1 - 1/2) * 2 pi */
double psg_ranno(psg_ranno_state* s, int i) {
  const double twopi = 4.0 * asin(1.0);
  if (i != 0) {
    if (i > 0) i = -i;
    s->junk = i;
    return (ran1(s, &i) - 0.5) * twopi;
  }
  s->junk -= 1;
  int ihold = s->junk;
  return (ran1(s, &ihold) - 0.5) * twopi;
}

/* ------------------------------------------------- initial conditions */

/* the storage mask of init.F90:38-57 (3D) */
static int keep3(double kx, double ky, double kz, int K) {
  const double wk = sqrt(kx * kx + ky * ky + kz * kz);
  if (kx < 0.0) return 0;
  if (kx == 0.0 && ky < 0.0) return 0;
  if (kx == 0.0 && ky == 0.0 && kz <= 0.0) return 0;
  if (wk > (double)K - 0.5) return 0;
  return 1;
}

int psg_ic_random3d(int n, int iseed, double ampv, double* xii, double* eta, double* zet) {
  if (n < 4 || (n % 2)) { psg_set_error("ic3d: bad grid %d", n); return -1; }
  const int K = n / 3, X = K + 1, Y = 2 * K + 1;
  const long nkt = (long)X * Y * Y;
  memset(xii, 0, sizeof(double) * 2 * nkt);
  memset(eta, 0, sizeof(double) * 2 * nkt);
  memset(zet, 0, sizeof(double) * 2 * nkt);
  psg_ranno_state s;
  psg_ranno_init(&s);
  psg_ranno(&s, iseed);  /* TIME = RANNO(ISEED), main.F90:43 */
  double enstro = 0.0;
  for (int ikx = 0; ikx < X; ++ikx)
    for (int iky = 0; iky < Y; ++iky)
      for (int ikz = 0; ikz < Y; ++ikz) {
        const long ik = ((long)ikz * Y + iky) * X + ikx;
        const double kx = ikx, ky = iky - K, kz = ikz - K;
        const double wk = sqrt(kx * kx + ky * ky + kz * kz);
        if (!keep3(kx, ky, kz, K)) continue;
        const double ek = (wk > 2.5 && wk <= 9.5) ? 1.0 : 0.0;
        double ph = psg_ranno(&s, 0);
        xii[2 * ik] = ek * cos(ph); xii[2 * ik + 1] = ek * sin(ph);
        ph = psg_ranno(&s, 0);
        eta[2 * ik] = ek * cos(ph); eta[2 * ik + 1] = ek * sin(ph);
        ph = psg_ranno(&s, 0);
        zet[2 * ik] = ek * cos(ph); zet[2 * ik + 1] = ek * sin(ph);
        const double r1 = xii[2 * ik] * xii[2 * ik] + eta[2 * ik] * eta[2 * ik] +
                          zet[2 * ik] * zet[2 * ik];
        const double r2 = xii[2 * ik + 1] * xii[2 * ik + 1] + eta[2 * ik + 1] * eta[2 * ik + 1] +
                          zet[2 * ik + 1] * zet[2 * ik + 1];
        enstro = enstro + r1 + r2;
      }
  enstro *= 2.0;
  const double sc = sqrt(ampv / enstro);
  for (long ik = 0; ik < 2 * nkt; ++ik) { xii[ik] *= sc; eta[ik] *= sc; zet[ik] *= sc; }
  return 0;
}

int psg_ic_random2d(int n, int iseed, double ampv, double* Z) {
  if (n < 4 || (n % 2)) { psg_set_error("ic2d: bad grid %d", n); return -1; }
  const int K = n / 3, X = K + 1, Y = 2 * K + 1;
  memset(Z, 0, sizeof(double) * 2 * (long)X * Y);
  psg_ranno_state s;
  psg_ranno_init(&s);
  psg_ranno(&s, iseed);
  double enstro = 0.0;
  for (int ikx = 0; ikx < X; ++ikx)
    for (int iky = 0; iky < Y; ++iky) {
      const double kx = ikx, ky = iky - K;
      const double wk = sqrt(kx * kx + ky * ky);
      /* mask of 2D_NavierStokes/src_RK4/src_gmres/init.F90:30-36 */
      if (kx < 0.0 || (kx == 0.0 && ky <= 0.0) || wk > (double)K - 0.5) continue;
      double ek = (wk > 2.5 && wk <= 9.5) ? 1.0 / wk : 0.0;
      if (kx < 0.1) ek = 0.0;
      const double vk = wk * wk * ek;
      const double ph = psg_ranno(&s, 0);
      const double a = sqrt(vk / wk);
      const long ik = (long)iky * X + ikx;
      Z[2 * ik] = a * cos(ph);
      Z[2 * ik + 1] = a * sin(ph);
      enstro = enstro + Z[2 * ik] * Z[2 * ik] + Z[2 * ik + 1] * Z[2 * ik + 1];
    }
  enstro *= 2.0;
  const double sc = sqrt(ampv / enstro);
  for (long ik = 0; ik < 2L * X * Y; ++ik) Z[ik] *= sc;
  return 0;
}

/* ------------------------------------------- Fortran sequential records */

int psg_frec_write(FILE* f, const void* const* parts, const size_t* sizes, int nparts) {
  size_t tot = 0;
  for (int i = 0; i < nparts; ++i) tot += sizes[i];
  if (tot > 0x7fffffffu) { psg_set_error("record of %zu bytes too long", tot); return -1; }
  const int32_t m = (int32_t)tot;
  if (fwrite(&m, 4, 1, f) != 1) return -1;
  for (int i = 0; i < nparts; ++i)
    if (sizes[i] && fwrite(parts[i], 1, sizes[i], f) != sizes[i]) return -1;
  if (fwrite(&m, 4, 1, f) != 1) return -1;
  return 0;
}

int psg_frec_read(FILE* f, void* buf, size_t cap, size_t* len) {
  int32_t a, b;
  if (fread(&a, 4, 1, f) != 1) return -1;
  if (a < 0 || (size_t)a > cap) { psg_set_error("record of %d bytes exceeds %zu", a, cap); return -1; }
  if (a && fread(buf, 1, (size_t)a, f) != (size_t)a) return -1;
  if (fread(&b, 4, 1, f) != 1 || b != a) { psg_set_error("record markers differ"); return -1; }
  if (len) *len = (size_t)a;
  return 0;
}

int psg_read_state3d(const char* path, const char* type, int irest, int n, double* meta,
                     double* xii, double* eta, double* zet) {
  const int K = n / 3, X = K + 1, Y = 2 * K + 1;
  const size_t nkt = (size_t)X * Y * Y, fb = 16 * nkt;
  FILE* f = fopen(path, "rb");
  if (!f) { psg_set_error("restart: cannot open %s", path); return -1; }
  int rc = -1;
  for (int q = 0; q < 7; ++q) meta[q] = 0.0;
  double* parts[3] = {xii, eta, zet};
  if (!strcmp(type, "A") || !strcmp(type, "B")) {
    for (int r = 0; r < irest; ++r) {
      int ok = fread(meta, 8, 7, f) == 7;
      for (int q = 0; q < 3 && ok; ++q) ok = fread(parts[q], 1, fb, f) == fb;
      if (!ok) { psg_set_error("restart: record %d missing", r + 1); goto done; }
    }
    rc = 0;
  } else if (!strcmp(type, "C") || !strcmp(type, "D")) {
    const int withmeta = !strcmp(type, "D");
    if (withmeta) {
      int32_t hdr[4];
      size_t len;
      if (psg_frec_read(f, hdr, sizeof hdr, &len) || len != sizeof hdr) goto done;
      if (hdr[1] != X || hdr[2] != Y || hdr[3] != Y) {
        psg_set_error("restart: file grid %d x %d x %d, this grid %d x %d x %d (changing the "
                      "resolution is not supported)", hdr[1], hdr[2], hdr[3], X, Y, Y);
        goto done;
      }
    }
    const size_t cap = 56 + 3 * fb;
    unsigned char* buf = (unsigned char*)malloc(cap);
    if (!buf) goto done;
    for (int r = 0; r < irest; ++r) {
      size_t len = 0;
      if (psg_frec_read(f, buf, cap, &len) || len != (withmeta ? 56 : 0) + 3 * fb) {
        free(buf);
        psg_set_error("restart: record %d missing or of the wrong size", r + 1);
        goto done;
      }
    }
    size_t o = 0;
    if (withmeta) { memcpy(meta, buf, 56); o = 56; }
    for (int q = 0; q < 3; ++q) memcpy(parts[q], buf + o + q * fb, fb);
    free(buf);
    rc = 0;
  } else {
    psg_set_error("restart: infile type '%s' unknown", type);
  }
done:
  if (rc == 0 && irest < 1) { psg_set_error("restart: record number %d", irest); rc = -1; }
  fclose(f);
  return rc;
}

int psg_write_state3d_header(FILE* f, int count, int n) {
  const int K = n / 3;
  const int32_t hdr[4] = {count, K + 1, 2 * K + 1, 2 * K + 1};
  const void* parts[1] = {hdr};
  const size_t sizes[1] = {sizeof hdr};
  return psg_frec_write(f, parts, sizes, 1);
}

int psg_write_state3d_record(FILE* f, int n, const double* meta, const double* xii,
                             const double* eta, const double* zet) {
  const int K = n / 3;
  const size_t fb = 16 * (size_t)(K + 1) * (2 * K + 1) * (2 * K + 1);
  const void* parts[4] = {meta, xii, eta, zet};
  const size_t sizes[4] = {56, fb, fb, fb};
  return psg_frec_write(f, parts, sizes, 4);
}

/* ----------------------------------------------------------- statistics */

struct psg_stats3d {
  int n, K, X, Y, kf;
  long nkt;
  double v2, ampfor, count;
  double* avg[3];  /* running time averages of the state (XIItavg, ...) */
  /* histories by statistics index NT/NOUT - 1 (energy, dissipation, input),
   * their extrema (from 0: the reference's globals start at zero, kernels.h:24)
   * and running averages */
  double* hist[3];
  long nhist, index;
  double lo[3], hi[3], mean[3];
};

psg_stats3d* psg_stats3d_create(int n, double v2, double ampfor, int kf) {
  psg_stats3d* s = (psg_stats3d*)calloc(1, sizeof(*s));
  if (!s) return NULL;
  s->n = n; s->K = n / 3; s->X = s->K + 1; s->Y = 2 * s->K + 1; s->kf = kf;
  s->nkt = (long)s->X * s->Y * s->Y;
  s->v2 = v2; s->ampfor = ampfor;
  s->index = -1;
  for (int q = 0; q < 3; ++q) {
    s->avg[q] = (double*)calloc(2 * s->nkt, sizeof(double));
    if (!s->avg[q]) { psg_stats3d_destroy(s); return NULL; }
  }
  return s;
}

void psg_stats3d_destroy(psg_stats3d* s) {
  if (!s) return;
  for (int q = 0; q < 3; ++q) { free(s->avg[q]); free(s->hist[q]); }
  free(s);
}

double psg_stats3d_count(const psg_stats3d* s) { return s ? s->count : 0.0; }

int psg_stats3d_mean(const psg_stats3d* s, double* xii, double* eta, double* zet) {
  double* out[3] = {xii, eta, zet};
  for (int q = 0; q < 3; ++q) {
    if (!out[q]) return set_err("null output");
    memcpy(out[q], s->avg[q], sizeof(double) * 2 * s->nkt);
  }
  return 0;
}

static double sq(double x) { return x * x; }

/* computeStats (3D_NavierStokes/src/functions.h:128-209) */
int psg_stats3d_add(psg_stats3d* s, double t, const double* xii, const double* eta,
                    const double* zet, FILE* stats, FILE* engy) {
  double energy = 0.0, diss = 0.0, input = 0.0, eturb = 0.0, dturb = 0.0;
  double XIa = 0.0, ETa = 0.0, ZTa = 0.0, Ua = 0.0, Va = 0.0, Wa = 0.0;
  const double kfy = (double)s->kf, c = s->count;
  for (int ikz = 0; ikz < s->Y; ++ikz)
    for (int iky = 0; iky < s->Y; ++iky)
      for (int ikx = 0; ikx < s->X; ++ikx) {
        const long i = ((long)ikz * s->Y + iky) * s->X + ikx;
        const double kx = ikx, ky = iky - s->K, kz = ikz - s->K;
        if (!keep3(kx, ky, kz, s->K)) continue;
        double wk = kx * kx + ky * ky + kz * kz;
        wk = wk > 0.001 ? wk : 0.001;
        const double xr = xii[2 * i], xm = xii[2 * i + 1], er = eta[2 * i], em = eta[2 * i + 1];
        const double zr = zet[2 * i], zm = zet[2 * i + 1];
        const double VZX = xr * xr + xm * xm, VZY = er * er + em * em, VZZ = zr * zr + zm * zm;
        double VZ = VZX + VZY + VZZ;
        diss += VZ;
        energy += VZ / wk;
        XIa += VZX; ETa += VZY; ZTa += VZZ;
        Ua += sq((ky * zm - kz * em) / wk) + sq((kz * er - ky * zr) / wk);
        Va += sq((kz * xm - kx * zm) / wk) + sq((kx * zr - kz * xr) / wk);
        Wa += sq((kx * em - ky * xm) / wk) + sq((ky * xr - kx * er) / wk);
        double* a[3] = {s->avg[0], s->avg[1], s->avg[2]};
        const double* v[3] = {xii, eta, zet};
        for (int q = 0; q < 3; ++q)
          for (int p = 0; p < 2; ++p) a[q][2 * i + p] = (a[q][2 * i + p] * c + v[q][2 * i + p]) / (c + 1.0);
        VZ = sq(a[0][2 * i]) + sq(a[0][2 * i + 1]) + sq(a[1][2 * i]) + sq(a[1][2 * i + 1]) +
             sq(a[2][2 * i]) + sq(a[2][2 * i + 1]);
        eturb += VZ / wk;
        dturb += VZ;
        if (kx == 0.0 && ky == kfy && kz == kfy) input += s->ampfor * xr;
        if (kx == 0.0 && ky == kfy && kz == -kfy) input -= s->ampfor * xr;
      }
  input *= s->v2 * kfy * kfy;
  diss *= s->v2 * s->v2 * 8.0 * kfy * kfy;
  dturb *= s->v2 * 16.0 * kfy * kfy;
  const double val[3] = {energy, diss, input};
  for (int q = 0; q < 3; ++q) {
    s->lo[q] = val[q] < s->lo[q] ? val[q] : s->lo[q];
    s->hi[q] = val[q] > s->hi[q] ? val[q] : s->hi[q];
    s->mean[q] = (s->mean[q] * c + val[q]) / (c + 1.0);
  }
  if (s->index >= 0) {
    if (s->index >= s->nhist) {
      const long m = s->index + 64;
      for (int q = 0; q < 3; ++q) {
        double* h = (double*)realloc(s->hist[q], sizeof(double) * m);
        if (!h) return set_err("out of host memory");
        for (long i = s->nhist; i < m; ++i) h[i] = 0.0;
        s->hist[q] = h;
      }
      s->nhist = m;
    }
    for (int q = 0; q < 3; ++q) s->hist[q][s->index] = val[q];
  }
  s->count += 1.0;
  if (stats) { fprintf(stats, "%e %e %e %e %e %e \n", t, energy, eturb, diss, dturb, input); fflush(stats); }
  if (engy) { fprintf(engy, "%e %e %e %e %e %e %e \n", t, Ua, Va, Wa, XIa, ETa, ZTa); fflush(engy); }
  return 0;
}

/* the same, storing the history at index nt/nout - 1 as computeStats does
 * (functions.h:197-200); nt: the step index NT of the reference's loop */
int psg_stats3d_add_at(psg_stats3d* s, int nt, int nout, double t, const double* xii,
                       const double* eta, const double* zet, FILE* stats, FILE* engy) {
  if (nout < 1) return set_err("NOUT must be >= 1");
  s->index = nt / nout - 1;
  const int rc = psg_stats3d_add(s, t, xii, eta, zet, stats, engy);
  s->index = -1;
  return rc;
}

/* The end-of-run statistics of the DNS (3D_NavierStokes/src/finalise.h:19-166,
 * statsFLAG = 1, NSTOP > 1), after the last psg_stats3d_add_at of the final state:
 * uvw = the physical velocity of the time-averaged state (psg_stats3d_mean),
 * ms = the running mean squares of the physical velocity (u^2, v^2, w^2).
 * avgs: five records (time, n^3 doubles): U, V, W, mean v^2, mean u^2 - U^2.
 * means: per (z, y) (z outer), y, z and the x averages of U, V, mean u^2 - U^2
 * and mean v^2.  pdfs (when the dissipation spans more than 1e-3): 100 bins of
 * energy, dissipation and input over the first NSTOP/NOUT histories, bin j
 * holding the values with int((x - min)/dx) + 1 = j (a value in bin 100, the
 * top one, falls outside the array in the reference and is not counted here).
 * Prints the averages and extrema as the reference does. */
int psg_stats3d_finish(psg_stats3d* s, int nstop, int nout, double time,
                       const double* const* uvw, const double* const* ms, FILE* avgs,
                       FILE* means, FILE* pdfs) {
  const int n = s->n;
  const long nr = (long)n * n * n, ny = n, nz = n, nx = n;
  const double twopi = 8.0 * atan(1.0);
  double* prof[4];
  for (int q = 0; q < 4; ++q) {
    prof[q] = (double*)calloc(ny * nz, sizeof(double));
    if (!prof[q]) { for (int p = 0; p < q; ++p) free(prof[p]); return set_err("out of host memory"); }
  }
  double* uvar = (double*)malloc(sizeof(double) * nr);
  if (!uvar) { for (int q = 0; q < 4; ++q) free(prof[q]); return set_err("out of host memory"); }
  for (long i = 0; i < nr; ++i) uvar[i] = ms[0][i] - uvw[0][i] * uvw[0][i];
  const double* rec[5] = {uvw[0], uvw[1], uvw[2], ms[1], uvar};
  int rc = 0;
  for (int r = 0; r < 5 && !rc; ++r)
    if (avgs && (fwrite(&time, sizeof(double), 1, avgs) != 1 ||
                 fwrite(rec[r], sizeof(double), nr, avgs) != (size_t)nr))
      rc = set_err("writing avgs failed");
  /* x averages: U, V, u variance, v mean square */
  const double* src[4] = {uvw[0], uvw[1], uvar, ms[1]};
  for (long iz = 0; iz < nz && !rc; ++iz)
    for (long iy = 0; iy < ny; ++iy) {
      const long ik = iz * ny + iy;
      for (int q = 0; q < 4; ++q) {
        double a = 0.0;
        for (long ix = 0; ix < nx; ++ix) a += src[q][(ny * iz + iy) * nx + ix];
        prof[q][ik] = a / (double)nx;
      }
      if (means)
        fprintf(means, "%.15e %.15e %.15e %.15e %.15e %.15e \n", iy * twopi / (double)ny,
                iz * twopi / (double)nz, prof[0][ik], prof[1][ik], prof[2][ik], prof[3][ik]);
    }
  printf("AVERAGE STATS *****\n");
  printf("energy = %e,  eturb = %e \n", s->mean[0], 0.0);
  printf("dissipation = %e,  dturb = %e \n", s->mean[1], 0.0);
  printf("input E = %e \n", s->mean[2]);
  printf("max/min dissipation %e, %e \n ", s->hi[1], s->lo[1]);
  printf("max/min energy %e, %e \n", s->hi[0], s->lo[0]);
  printf("max/min input %e, %e \n", s->hi[2], s->lo[2]);
  const long nstats = nstop / nout + 1;
  if (!rc && s->hi[1] - s->lo[1] > 0.001) {
    enum { NBIN = 100 };
    const double correct = 1.0000001;
    long cnt[3][NBIN + 1] = {{0}};
    double dx[3];
    for (int q = 0; q < 3; ++q) dx[q] = (s->hi[q] * correct - s->lo[q]) / (double)NBIN;
    for (long t = 0; t < nstats - 1; ++t)
      for (int q = 0; q < 3; ++q) {
        const double x = t < s->nhist ? s->hist[q][t] : 0.0;
        const long j = (long)((x - s->lo[q]) / dx[q]) + 1;
        if (j >= 0 && j <= NBIN) ++cnt[q][j];
      }
    const double norm = (double)(nstats - 1);
    for (int ib = 0; ib < NBIN && pdfs; ++ib)
      fprintf(pdfs, "%.15e %.15e %.15e %.15e %.15e %.15e \n", s->lo[0] + (ib - 0.5) * dx[0],
              cnt[0][ib] / (norm * dx[0]), s->lo[1] + (ib - 0.5) * dx[1], cnt[1][ib] / (norm * dx[1]),
              s->lo[2] + (ib - 0.5) * dx[2], cnt[2][ib] / (norm * dx[2]));
  }
  for (int q = 0; q < 4; ++q) free(prof[q]);
  free(uvar);
  return rc;
}
