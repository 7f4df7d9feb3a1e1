/*
 * psg_oracle.c -- FP64 CPU restatement of psgpu's pseudospectral step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * psg_oracle.h.  Each function cites the reference lines it restates; the
 * reference paths are relative to the psgpu project root.
 *
 * The FFT is a project-written iterative radix-2 transform (complex double),
 * applied line by line; the 3D and 2D real transforms follow cuFFT's
 * conventions: C2R is unnormalised with e^{+i k x}, R2C uses e^{-i k x}, and
 * the reference normalises R2C output by 1/(NX*NY*NZ) afterwards.
 */
#include "psg_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* radix-2 FFT                                                              */
/* ------------------------------------------------------------------------ */

#define ORC_MAXLOG 12
static cplx *g_tw[ORC_MAXLOG + 1];   /* g_tw[l][j] = exp(-2 pi i j / 2^l), j < 2^(l-1) */

static int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return ((1 << l) == n) ? l : -1;
}

static void tw_init(int n) {
  int L = ilog2i(n);
  for (int l = 1; l <= L; ++l) {
    if (g_tw[l]) continue;
    int m = 1 << l;
    cplx *t = (cplx *)malloc(sizeof(cplx) * (m / 2));
    for (int j = 0; j < m / 2; ++j) {
      double a = -2.0 * M_PI * (double)j / (double)m;
      t[j] = cos(a) + I * sin(a);
    }
    g_tw[l] = t;
  }
}

/* In-place FFT of a contiguous line.  sign=-1 forward (e^{-i}), +1 inverse. */
static void fft_line(cplx *x, int n, int sign) {
  int L = ilog2i(n);
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { cplx t = x[i]; x[i] = x[j]; x[j] = t; }
  }
  for (int l = 1; l <= L; ++l) {
    int m = 1 << l, h = m >> 1;
    const cplx *tw = g_tw[l];
    for (int s = 0; s < n; s += m) {
      for (int j = 0; j < h; ++j) {
        cplx w = (sign < 0) ? tw[j] : conj(tw[j]);
        cplx a = x[s + j], b = x[s + j + h] * w;
        x[s + j] = a + b;
        x[s + j + h] = a - b;
      }
    }
  }
}

/* FFT along a strided axis: `count` lines, line i starts at base[i*lstride],
 * elements spaced by estride. */
static void fft_strided(cplx *base, int n, long estride, long count,
                        long (*line_off)(long, const long *), const long *ctx,
                        int sign) {
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp for schedule(static)
    for (long i = 0; i < count; ++i) {
      cplx *p = base + line_off(i, ctx);
      for (int e = 0; e < n; ++e) buf[e] = p[(long)e * estride];
      fft_line(buf, n, sign);
      for (int e = 0; e < n; ++e) p[(long)e * estride] = buf[e];
    }
    free(buf);
  }
}

/* ------------------------------------------------------------------------ */
/* layouts                                                                  */
/* ------------------------------------------------------------------------ */

int orc_nkt2d(int n) { int k = n / 3; return (k + 1) * (2 * k + 1); }
int orc_nkt3d(int n) { int k = n / 3; return (k + 1) * (2 * k + 1) * (2 * k + 1); }

/* 2D_NavierStokes/src_RK4/src_gmres/init.F90:25-39 (mask) and
 * main.F90:328-335 (wavenumbers).  kx fastest: ik = iky*IKTX + ikx. */
void orc_layout2d(int n, double alpha, double *kx, double *ky, int *LL) {
  int K = n / 3, X = K + 1, Y = 2 * K + 1;
  for (int iy = 0; iy < Y; ++iy)
    for (int ix = 0; ix < X; ++ix) {
      int ik = iy * X + ix;
      double KX = ix * alpha, KY = iy - K;
      double wk = sqrt(KX * KX + KY * KY);
      int keep = 1;
      if (KX < 0) keep = 0;
      if (KX == 0 && KY <= 0) keep = 0;
      if (wk > (double)K - 0.5) keep = 0;
      kx[ik] = KX; ky[ik] = KY; LL[ik] = keep;
    }
}

/* 3D_NavierStokes/src/init.F90:25-57.  ik = (ikz*IKTY + iky)*IKTX + ikx. */
void orc_layout3d(int n, double alpha, double *kx, double *ky, double *kz, int *LL) {
  int K = n / 3, X = K + 1, Y = 2 * K + 1, Z = 2 * K + 1;
  for (int iz = 0; iz < Z; ++iz)
    for (int iy = 0; iy < Y; ++iy)
      for (int ix = 0; ix < X; ++ix) {
        int ik = (iz * Y + iy) * X + ix;
        double KX = ix * alpha, KY = iy - K, KZ = iz - K;
        double wk = sqrt(KX * KX + KY * KY + KZ * KZ);
        int keep = 1;
        if (KX < 0) keep = 0;
        if (KX == 0 && KY < 0) keep = 0;
        if (KX == 0 && KY == 0 && KZ <= 0) keep = 0;
        if (wk > (double)K - 0.5) keep = 0;
        kx[ik] = KX; ky[ik] = KY; kz[ik] = KZ; LL[ik] = keep;
      }
}

/* 2D_NavierStokes/src_RK4/src_gmres/main.F90:292-325 */
void orc_ikf2d(int n, int *ikF) {
  int K = n / 3, X = K + 1, nx2 = n / 2 + 1;
  for (int iy = 0; iy < n; ++iy)
    for (int ix = 0; ix < nx2; ++ix) {
      int v = -1;
      if (ix < X) {
        if (iy <= K) v = ix + X * (iy + K);
        else if (iy >= n - K) v = ix + X * (iy + K - n);
      }
      ikF[iy * nx2 + ix] = v;
    }
}

void orc_ikn2d(int n, int *ikN) {
  int K = n / 3, X = K + 1, Y = 2 * K + 1, nx2 = n / 2 + 1;
  for (int iy = 0; iy < Y; ++iy)
    for (int ix = 0; ix < X; ++ix) {
      int row = (iy < K) ? (n + iy - K) : (iy - K);
      ikN[iy * X + ix] = row * nx2 + ix;
    }
}

/* 3D_NavierStokes/src/main.F90:100-156 */
void orc_ikf3d(int n, int *ikF) {
  int K = n / 3, X = K + 1, Y = 2 * K + 1, nx2 = n / 2 + 1;
  for (int iz = 0; iz < n; ++iz)
    for (int iy = 0; iy < n; ++iy)
      for (int ix = 0; ix < nx2; ++ix) {
        int v = -1;
        int yy = -1, zz = -1;
        if (iy <= K) yy = iy + K; else if (iy >= n - K) yy = iy + K - n;
        if (iz <= K) zz = iz + K; else if (iz >= n - K) zz = iz + K - n;
        if (ix < X && yy >= 0 && zz >= 0) v = ix + X * (yy + Y * zz);
        ikF[((long)iz * n + iy) * nx2 + ix] = v;
      }
}

/* 3D_NavierStokes/src/main.F90:158-199 */
void orc_ikn3d(int n, int *ikN) {
  int K = n / 3, X = K + 1, Y = 2 * K + 1, nx2 = n / 2 + 1;
  for (int iz = 0; iz < Y; ++iz)
    for (int iy = 0; iy < Y; ++iy)
      for (int ix = 0; ix < X; ++ix) {
        int zz = (iz < K) ? (n + iz - K) : (iz - K);
        int yy = (iy < K) ? (n + iy - K) : (iy - K);
        ikN[(iz * Y + iy) * X + ix] = (zz * n + yy) * nx2 + ix;
      }
}

/* ------------------------------------------------------------------------ */
/* transform plumbing                                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
  int n, K, X, Y, nx2;
  long nkt, n2, nr;
  int *ikF, *ikN;
  double *kx, *ky, *kz;
  int *LL;
  int dim;
} geom_t;

static int geom_init(geom_t *g, int dim, int n, double alpha) {
  if (n < 8 || ilog2i(n) < 0 || (1 << ilog2i(n)) != n || ilog2i(n) > ORC_MAXLOG) return -1;
  tw_init(n);
  g->dim = dim; g->n = n; g->K = n / 3; g->X = g->K + 1; g->Y = 2 * g->K + 1;
  g->nx2 = n / 2 + 1;
  if (dim == 2) {
    g->nkt = orc_nkt2d(n); g->n2 = (long)g->nx2 * n; g->nr = (long)n * n;
  } else {
    g->nkt = orc_nkt3d(n); g->n2 = (long)g->nx2 * n * n; g->nr = (long)n * n * n;
  }
  g->ikF = (int *)malloc(sizeof(int) * g->n2);
  g->ikN = (int *)malloc(sizeof(int) * g->nkt);
  g->kx = (double *)malloc(sizeof(double) * g->nkt);
  g->ky = (double *)malloc(sizeof(double) * g->nkt);
  g->kz = (double *)calloc(g->nkt, sizeof(double));
  g->LL = (int *)malloc(sizeof(int) * g->nkt);
  if (dim == 2) {
    orc_ikf2d(n, g->ikF); orc_ikn2d(n, g->ikN); orc_layout2d(n, alpha, g->kx, g->ky, g->LL);
  } else {
    orc_ikf3d(n, g->ikF); orc_ikn3d(n, g->ikN); orc_layout3d(n, alpha, g->kx, g->ky, g->kz, g->LL);
  }
  return 0;
}

static void geom_free(geom_t *g) {
  free(g->ikF); free(g->ikN); free(g->kx); free(g->ky); free(g->kz); free(g->LL);
}

static long off_zline(long i, const long *c) {  /* c: nx2, n -> line (x,y) along z */
  long nx2 = c[0], n = c[1];
  long y = i / nx2, x = i % nx2;
  return y * nx2 + x;
  (void)n;
}
static long off_yline(long i, const long *c) {  /* lines along y: (x,z) */
  long nx2 = c[0], n = c[1];
  long z = i / nx2, x = i % nx2;
  return z * n * nx2 + x;
}

/* cufftExecZ2D on the padded half spectrum F (destroyed) -> real r.
 * 3D: plan3d(NZ,NY,NX); 2D: plan2d(NY,NX). */
static void c2r(const geom_t *g, cplx *F, double *r) {
  int n = g->n, nx2 = g->nx2;
  long ctx[2] = {nx2, n};
  if (g->dim == 3) {
    fft_strided(F, n, (long)nx2 * n, (long)nx2 * n, off_zline, ctx, +1);
    fft_strided(F, n, nx2, (long)nx2 * n, off_yline, ctx, +1);
  } else {
    fft_strided(F, n, nx2, nx2, off_zline, ctx, +1);  /* lines along y: (x) */
  }
  long rows = g->nr / n;
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp for schedule(static)
    for (long row = 0; row < rows; ++row) {
      const cplx *s = F + row * nx2;
      buf[0] = s[0];
      for (int k = 1; k < n / 2; ++k) { buf[k] = s[k]; buf[n - k] = conj(s[k]); }
      buf[n / 2] = s[n / 2];
      /* C2R uses only the real parts of the self-conjugate bins */
      buf[0] = creal(buf[0]);
      buf[n / 2] = creal(buf[n / 2]);
      fft_line(buf, n, +1);
      double *d = r + row * n;
      for (int x = 0; x < n; ++x) d[x] = creal(buf[x]);
    }
    free(buf);
  }
}

/* cufftExecD2Z: real r -> padded half spectrum F */
static void r2c(const geom_t *g, const double *r, cplx *F) {
  int n = g->n, nx2 = g->nx2;
  long rows = g->nr / n;
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp for schedule(static)
    for (long row = 0; row < rows; ++row) {
      const double *s = r + row * n;
      for (int x = 0; x < n; ++x) buf[x] = s[x];
      fft_line(buf, n, -1);
      cplx *d = F + row * nx2;
      for (int k = 0; k < nx2; ++k) d[k] = buf[k];
    }
    free(buf);
  }
  long ctx[2] = {nx2, n};
  if (g->dim == 3) {
    fft_strided(F, n, nx2, (long)nx2 * n, off_yline, ctx, -1);
    fft_strided(F, n, (long)nx2 * n, (long)nx2 * n, off_zline, ctx, -1);
  } else {
    fft_strided(F, n, nx2, nx2, off_zline, ctx, -1);
  }
}

/* setFFN: gather the truncated box into the zero-padded half spectrum
 * (3D_NavierStokes/src/kernels.h:51-68). If kk is non-NULL, fold in the
 * gradient multiply i*kk as setFFK does (3D_Boussinesq/src/kernels.h:75-93). */
static void pad(const geom_t *g, const cplx *V, const double *kk, cplx *F) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < g->n2; ++i) {
    int s = g->ikF[i];
    if (s < 0) F[i] = 0;
    else F[i] = kk ? (I * kk[s]) * V[s] : V[s];
  }
}

/* normFF1: gather kept modes from the R2C output and scale by 1/nr
 * (3D_NavierStokes/src/kernels.h:266-277) */
static void gather(const geom_t *g, const cplx *F, cplx *V) {
  double in = 1.0 / (double)g->nr;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < g->nkt; ++i) V[i] = F[g->ikN[i]] * in;
}

/* 3D conj: copy, filling the kx=0 plane's lower half with conjugates of
 * the mirrored upper half and zeroing k=0 (3D_NavierStokes/src/kernels.h:113-163). */
static void conj3d(const geom_t *g, const cplx *Z, cplx *T) {
  int X = g->X, Y = g->Y, K = g->K;
#pragma omp parallel for schedule(static)
  for (long ik = 0; ik < g->nkt; ++ik) {
    if (g->kx[ik] == 0.0) {
      int ikt = (int)(ik / X);
      int ikz = ikt / Y, iky = ikt - ikz * Y;
      if (iky == K) {
        if (ikz == K) T[ik] = 0;
        else if (ikz < K) T[ik] = conj(Z[((Y - 1 - ikz) * Y + iky) * X]);
        else T[ik] = Z[ik];
      } else if (iky < K) {
        T[ik] = conj(Z[((Y - 1 - ikz) * Y + (Y - 1 - iky)) * X]);
      } else {
        T[ik] = Z[ik];
      }
    } else {
      T[ik] = Z[ik];
    }
  }
}

/* 2D conj, in place (2D_NavierStokes/src_RK4/kernels.h:82-96) */
static void conj2d(const geom_t *g, cplx *Z) {
  int X = g->X, Y = g->Y;
  for (long ik = 0; ik < g->nkt; ++ik)
    if (g->kx[ik] == 0.0 && g->ky[ik] < 0.0) {
      int iky = (int)(ik / X);
      Z[ik] = conj(Z[(long)(Y - iky - 1) * X]);
    }
}

/* ------------------------------------------------------------------------ */
/* 2D Navier-Stokes                                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
  geom_t g;
  cplx *Z0, *UK, *VK, *NZK, *F;
  double *ZR, *UR, *VR, *NZR;
} ns2d_t;

/* KR_FFT_ALL + multReal + RK_FFT of the 2D step
 * (2D_NavierStokes/src_RK4/functions.h:33-57,137-149; kernels.h:187-201):
 * NZK[0:nkt] = F(v w)/nr, NZK[nkt:2nkt] = F(u w)/nr. */
static void ns2d_convol(ns2d_t *s) {
  geom_t *g = &s->g;
  conj2d(g, s->Z0); pad(g, s->Z0, NULL, s->F); c2r(g, s->F, s->ZR);
  conj2d(g, s->UK); pad(g, s->UK, NULL, s->F); c2r(g, s->F, s->UR);
  conj2d(g, s->VK); pad(g, s->VK, NULL, s->F); c2r(g, s->F, s->VR);
  for (long i = 0; i < g->nr; ++i) {
    s->NZR[i] = s->VR[i] * s->ZR[i];
    s->NZR[g->nr + i] = s->UR[i] * s->ZR[i];
  }
  r2c(g, s->NZR, s->F); gather(g, s->F, s->NZK);
  r2c(g, s->NZR + g->nr, s->F); gather(g, s->F, s->NZK + g->nkt);
}

static void vel2d(double kx, double ky, cplx z, cplx *u, cplx *v) {
  double wk = kx * kx + ky * ky;
  double wki = 1.0 / (wk > 0.001 ? wk : 0.001);
  *u = (-ky * cimag(z) * wki) + I * (ky * creal(z) * wki);
  *v = (kx * cimag(z) * wki) + I * (-kx * creal(z) * wki);
}

/* curl/divergence finish + hard-coded forcing of Step1/Step2/Step
 * (2D_NavierStokes/src_RK4/kernels.h:260-266) */
static cplx ns2d_nl(const ns2d_t *s, long ik) {
  double kx = s->g.kx[ik], ky = s->g.ky[ik];
  cplx a = s->NZK[ik], b = s->NZK[ik + s->g.nkt];
  double re = kx * cimag(b) + ky * cimag(a);
  double im = -kx * creal(b) - ky * creal(a);
  if (kx == 0.0 && fabs(ky) == 4.0) re -= 2.0;
  return re + I * im;
}

int orc_ns2d_timestep(double *Zd, int n, double alpha, double nu, double dt,
                      int nstop, double *time) {
  ns2d_t s;
  if (geom_init(&s.g, 2, n, alpha)) return -1;
  geom_t *g = &s.g;
  long nkt = g->nkt;
  cplx *Z = (cplx *)Zd;
  cplx *Z1 = (cplx *)calloc(nkt, sizeof(cplx)), *Z2 = (cplx *)calloc(nkt, sizeof(cplx));
  cplx *Z3 = (cplx *)calloc(nkt, sizeof(cplx));
  s.Z0 = (cplx *)calloc(nkt, sizeof(cplx)); s.UK = (cplx *)calloc(nkt, sizeof(cplx));
  s.VK = (cplx *)calloc(nkt, sizeof(cplx)); s.NZK = (cplx *)calloc(2 * nkt, sizeof(cplx));
  s.F = (cplx *)calloc(g->n2, sizeof(cplx));
  s.ZR = (double *)malloc(sizeof(double) * g->nr); s.UR = (double *)malloc(sizeof(double) * g->nr);
  s.VR = (double *)malloc(sizeof(double) * g->nr); s.NZR = (double *)malloc(sizeof(double) * 2 * g->nr);

  /* setVelocity (kernels.h:112-147) */
  for (long ik = 0; ik < nkt; ++ik) {
    if (g->LL[ik]) { vel2d(g->kx[ik], g->ky[ik], Z[ik], &s.UK[ik], &s.VK[ik]); s.Z0[ik] = Z[ik]; }
    else { s.UK[ik] = 0; s.VK[ik] = 0; s.Z0[ik] = 0; }
  }
  *time = 0.0;
  for (int nt = 0; nt < nstop; ++nt) {
    /* stages 1..3: Step1, Step1, Step2 (kernels.h:247-370) */
    cplx *kreg[3] = {Z1, Z2, Z3};
    double frac[3] = {0.5, 0.5, 1.0};
    for (int st = 0; st < 3; ++st) {
      ns2d_convol(&s);
      for (long ik = 0; ik < nkt; ++ik) {
        if (g->LL[ik]) {
          cplx d = dt * ns2d_nl(&s, ik);
          kreg[st][ik] = d;
          s.Z0[ik] = Z[ik] + frac[st] * d;
          vel2d(g->kx[ik], g->ky[ik], s.Z0[ik], &s.UK[ik], &s.VK[ik]);
        } else {
          s.UK[ik] = 0; s.VK[ik] = 0; Z[ik] = 0;
        }
      }
    }
    /* final stage: Step (kernels.h:373-435) */
    ns2d_convol(&s);
    for (long ik = 0; ik < nkt; ++ik) {
      if (g->LL[ik]) {
        double kx = g->kx[ik], ky = g->ky[ik], wk = kx * kx + ky * ky;
        double damp1 = 1 - 0.5 * dt * nu * wk;
        double damp2 = 1. / (1 + 0.5 * dt * nu * wk);
        cplx d = dt * ns2d_nl(&s, ik);
        double zr = damp2 * (damp1 * creal(Z[ik]) +
                             (creal(Z1[ik]) + 2 * creal(Z2[ik]) + 2 * creal(Z3[ik]) + creal(d)) / 6.);
        double zi = damp2 * (damp1 * cimag(Z[ik]) +
                             (cimag(Z1[ik]) + 2 * cimag(Z2[ik]) + 2 * cimag(Z3[ik]) + cimag(d)) / 6.);
        Z[ik] = zr + I * zi;
        s.Z0[ik] = Z[ik];
        vel2d(kx, ky, s.Z0[ik], &s.UK[ik], &s.VK[ik]);
      } else {
        s.UK[ik] = 0; s.VK[ik] = 0; Z[ik] = 0;
      }
    }
    *time += dt;
  }
  free(Z1); free(Z2); free(Z3); free(s.Z0); free(s.UK); free(s.VK); free(s.NZK);
  free(s.F); free(s.ZR); free(s.UR); free(s.VR); free(s.NZR);
  geom_free(g);
  return 0;
}

/* 2D_NavierStokes/src_RK4/src_gmres/timederiv.F90:2-32 with CONVOL
 * (convol.F90:2-64) and the driver's NU (init.F90:191-192). */
int orc_ns2d_timederiv(const double *Zd, double *dZd, int n, double alpha, double nu) {
  ns2d_t s;
  if (geom_init(&s.g, 2, n, alpha)) return -1;
  geom_t *g = &s.g;
  long nkt = g->nkt;
  const cplx *Zin = (const cplx *)Zd;
  cplx *dZ = (cplx *)dZd;
  s.Z0 = (cplx *)calloc(nkt, sizeof(cplx)); s.UK = (cplx *)calloc(nkt, sizeof(cplx));
  s.VK = (cplx *)calloc(nkt, sizeof(cplx)); s.NZK = (cplx *)calloc(2 * nkt, sizeof(cplx));
  s.F = (cplx *)calloc(g->n2, sizeof(cplx));
  s.ZR = (double *)malloc(sizeof(double) * g->nr); s.UR = (double *)malloc(sizeof(double) * g->nr);
  s.VR = (double *)malloc(sizeof(double) * g->nr); s.NZR = (double *)malloc(sizeof(double) * 2 * g->nr);
  for (long ik = 0; ik < nkt; ++ik) {
    /* CONVOL: UK = L*i*ky*Z/wk, VK = -L*i*kx*Z/wk */
    s.Z0[ik] = Zin[ik];
    if (g->LL[ik]) vel2d(g->kx[ik], g->ky[ik], Zin[ik], &s.UK[ik], &s.VK[ik]);
    else { s.UK[ik] = 0; s.VK[ik] = 0; }
  }
  ns2d_convol(&s);
  for (long ik = 0; ik < nkt; ++ik) {
    if (!g->LL[ik]) { dZ[ik] = 0; continue; }
    double kx = g->kx[ik], ky = g->ky[ik];
    double wk = sqrt(kx * kx + ky * ky);
    double NU = pow(10.0, log10(nu) + 2.0 * log10(wk));
    cplx nl = ns2d_nl(&s, ik);
    dZ[ik] = -NU * Zin[ik] + nl;
  }
  free(s.Z0); free(s.UK); free(s.VK); free(s.NZK); free(s.F);
  free(s.ZR); free(s.UR); free(s.VR); free(s.NZR);
  geom_free(g);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* 3D common: velocity, transforms of the vorticity system                  */
/* ------------------------------------------------------------------------ */

/* u = i k x w / k^2 with the reference's component formulas
 * (3D_NavierStokes/src/kernels.h:194-201); wki already masked or not by caller */
static inline void vel3d(double kx, double ky, double kz, double wki,
                         cplx xi, cplx et, cplx zt, cplx *u, cplx *v, cplx *w) {
  double xiX = creal(xi), xiY = cimag(xi), etX = creal(et), etY = cimag(et);
  double ztX = creal(zt), ztY = cimag(zt);
  *u = (-(ky * ztY - kz * etY) * wki) + I * (-(kz * etX - ky * ztX) * wki);
  *v = (-(kz * xiY - kx * ztY) * wki) + I * (-(kx * ztX - kz * xiX) * wki);
  *w = (-(kx * etY - ky * xiY) * wki) + I * (-(ky * xiX - kx * etX) * wki);
}

static inline double wkinv(double wk) { return 1.0 / (wk > 0.001 ? wk : 0.001); }

typedef struct {
  geom_t g;
  cplx *T, *F;
  double *R[10];    /* xir etr ztr UR VR WR (+ rx ry rz) */
} work3d_t;

static int work3d_init(work3d_t *w, int n, double alpha, int nreal) {
  if (geom_init(&w->g, 3, n, alpha)) return -1;
  w->T = (cplx *)malloc(sizeof(cplx) * w->g.nkt);
  w->F = (cplx *)malloc(sizeof(cplx) * w->g.n2);
  for (int i = 0; i < 10; ++i) w->R[i] = NULL;
  for (int i = 0; i < nreal; ++i) w->R[i] = (double *)malloc(sizeof(double) * w->g.nr);
  return 0;
}
static void work3d_free(work3d_t *w) {
  free(w->T); free(w->F);
  for (int i = 0; i < 10; ++i) free(w->R[i]);
  geom_free(&w->g);
}

/* KR_FFT_ALL for the 6 vorticity/velocity fields
 * (3D_NavierStokes/src/functions.h:26-75): conj -> setFFN -> Z2D. */
static void kr_fft_all(work3d_t *w, cplx *const in[6]) {
  for (int f = 0; f < 6; ++f) {
    conj3d(&w->g, in[f], w->T);
    pad(&w->g, w->T, NULL, w->F);
    c2r(&w->g, w->F, w->R[f]);
  }
}

/* multReal: U,V,W <- -(u x w) (3D_NavierStokes/src/kernels.h:281-306) */
static void mult_real(work3d_t *w) {
  double *X = w->R[0], *E = w->R[1], *Zt = w->R[2], *U = w->R[3], *V = w->R[4], *W = w->R[5];
#pragma omp parallel for schedule(static)
  for (long i = 0; i < w->g.nr; ++i) {
    double TU = U[i], TV = V[i], TW = W[i], TX = X[i], TE = E[i], TZ = Zt[i];
    double NX = TV * TZ - TW * TE, NY = TW * TX - TU * TZ, NZ = TU * TE - TV * TX;
    U[i] = -NX; V[i] = -NY; W[i] = -NZ;
  }
}

/* RK_FFT: D2Z -> normFF1 for 3 fields (3D_NavierStokes/src/functions.h:79-108) */
static void rk_fft(work3d_t *w, double *const r[], cplx *const out[], int nf) {
  for (int f = 0; f < nf; ++f) {
    r2c(&w->g, r[f], w->F);
    gather(&w->g, w->F, out[f]);
  }
}

/* N(w) spectral: UK,VK,WK hold F(-(u x w))/nr; return the curl as the
 * reference's preStep/corStep forms it (kernels.h:327-334). */
static inline void curl3d(double kx, double ky, double kz, cplx U, cplx V, cplx W,
                          cplx *nx, cplx *ny, cplx *nz) {
  double UKX = creal(U), UKY = cimag(U), VKX = creal(V), VKY = cimag(V);
  double WKX = creal(W), WKY = cimag(W);
  *nx = (ky * WKY - kz * VKY) + I * (kz * VKX - ky * WKX);
  *ny = (kz * UKY - kx * WKY) + I * (kx * WKX - kz * UKX);
  *nz = (kx * VKY - ky * UKY) + I * (ky * UKX - kx * VKX);
}

/* ------------------------------------------------------------------------ */
/* 3D Navier-Stokes (DNS build) and Euler: Heun with/without CN             */
/* ------------------------------------------------------------------------ */

/* forcing of the Heun/CN flavours: form 0 as the DNS build applies it
 * (3D_NavierStokes/src/kernels.h:342-343, 419-420), form 1 as the
 * Newton-solver build does (3D_NavierStokes/src_gmres/kernels.h:234-238, 320-324) */
static void heun_force(int form, double kx, double ky, double kz, double kfy, double ampfor,
                       cplx *nx, cplx *ny, cplx *nz) {
  if (form == 0) {
    if (kx == 0.0 && kz == kfy && ky == kfy) *nx += ampfor;
    if (kx == 0.0 && kz == -kfy && ky == kfy) *nx -= ampfor;
  } else {
    if (kx == 0.0 && kz == kfy && ky == kfy) { *ny += I * ampfor; *nz -= I * ampfor; }
    if (kx == 0.0 && kz == -kfy && ky == kfy) { *ny += I * ampfor; *nz += I * ampfor; }
  }
}

static int heun3d(int euler, int fform, double *xid, double *etd, double *ztd, double *phys,
                  const double *nuzn, const double *nu1, int n, double alpha,
                  double ampfor, double kfy, double dt, int nstop, double tstart,
                  double *time) {
  work3d_t w;
  if (work3d_init(&w, n, alpha, 6)) return -1;
  geom_t *g = &w.g;
  long nkt = g->nkt;
  cplx *xi = (cplx *)xid, *et = (cplx *)etd, *zt = (cplx *)ztd;
  cplx *U = (cplx *)malloc(sizeof(cplx) * nkt), *V = (cplx *)malloc(sizeof(cplx) * nkt);
  cplx *W = (cplx *)malloc(sizeof(cplx) * nkt);
  cplx *RX = (cplx *)calloc(nkt, sizeof(cplx)), *RY = (cplx *)calloc(nkt, sizeof(cplx));
  cplx *RZ = (cplx *)calloc(nkt, sizeof(cplx));
  cplx *fields[6] = {xi, et, zt, U, V, W};
  double *rr[3] = {w.R[3], w.R[4], w.R[5]};
  cplx *uk[3] = {U, V, W};

  /* setVelocity (kernels.h:168-205): masked wki */
  for (long ik = 0; ik < nkt; ++ik) {
    double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
    double wki = g->LL[ik] ? wkinv(kx * kx + ky * ky + kz * kz) : 0.0;
    vel3d(kx, ky, kz, wki, xi[ik], et[ik], zt[ik], &U[ik], &V[ik], &W[ik]);
  }
  for (int nt = 0; nt < nstop; ++nt) {
    kr_fft_all(&w, fields);
    mult_real(&w);
    rk_fft(&w, rr, uk, 3);
    /* preStep (NS: kernels.h:309-386; Euler: 3D_Euler/src/kernels.h:296-366) */
#pragma omp parallel for schedule(static)
    for (long ik = 0; ik < nkt; ++ik) {
      double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
      double wki = wkinv(kx * kx + ky * ky + kz * kz);
      cplx nx, ny, nz;
      curl3d(kx, ky, kz, U[ik], V[ik], W[ik], &nx, &ny, &nz);
      if (!euler) {
        heun_force(fform, kx, ky, kz, kfy, ampfor, &nx, &ny, &nz);
        double NUZN = nuzn[ik], NU1 = g->LL[ik] * nu1[ik];
        RX[ik] = nx; RY[ik] = ny; RZ[ik] = nz;
        nx = NU1 * (creal(xi[ik]) * NUZN + creal(nx)) + I * (NU1 * (NUZN * cimag(xi[ik]) + cimag(nx)));
        ny = NU1 * (creal(et[ik]) * NUZN + creal(ny)) + I * (NU1 * (NUZN * cimag(et[ik]) + cimag(ny)));
        nz = NU1 * (creal(zt[ik]) * NUZN + creal(nz)) + I * (NU1 * (NUZN * cimag(zt[ik]) + cimag(nz)));
      } else {
        double L = g->LL[ik];
        RX[ik] = L * nx; RY[ik] = L * ny; RZ[ik] = L * nz;
        nx = xi[ik] + dt * nx; ny = et[ik] + dt * ny; nz = zt[ik] + dt * nz;
      }
      vel3d(kx, ky, kz, wki, nx, ny, nz, &U[ik], &V[ik], &W[ik]);
      xi[ik] = nx; et[ik] = ny; zt[ik] = nz;
    }
    kr_fft_all(&w, fields);
    if (phys && nt == nstop - 1) {
      memcpy(phys, w.R[0], sizeof(double) * g->nr);
      memcpy(phys + g->nr, w.R[1], sizeof(double) * g->nr);
      memcpy(phys + 2 * g->nr, w.R[2], sizeof(double) * g->nr);
    }
    mult_real(&w);
    rk_fft(&w, rr, uk, 3);
    *time = tstart + (nt + 1) * dt;
    /* corStep (NS: kernels.h:389-464; Euler: 3D_Euler/src/kernels.h:369-439) */
#pragma omp parallel for schedule(static)
    for (long ik = 0; ik < nkt; ++ik) {
      double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
      double wki = wkinv(kx * kx + ky * ky + kz * kz);
      cplx nx, ny, nz;
      curl3d(kx, ky, kz, U[ik], V[ik], W[ik], &nx, &ny, &nz);
      double L = g->LL[ik];
      double NU2;
      if (!euler) {
        NU2 = 0.5 * nu1[ik];
        heun_force(fform, kx, ky, kz, kfy, ampfor, &nx, &ny, &nz);
      } else {
        NU2 = 0.5 * dt;
      }
      nx = L * (creal(xi[ik]) + NU2 * (creal(nx) - creal(RX[ik]))) +
           I * (L * (cimag(xi[ik]) + NU2 * (cimag(nx) - cimag(RX[ik]))));
      ny = L * (creal(et[ik]) + NU2 * (creal(ny) - creal(RY[ik]))) +
           I * (L * (cimag(et[ik]) + NU2 * (cimag(ny) - cimag(RY[ik]))));
      nz = L * (creal(zt[ik]) + NU2 * (creal(nz) - creal(RZ[ik]))) +
           I * (L * (cimag(zt[ik]) + NU2 * (cimag(nz) - cimag(RZ[ik]))));
      vel3d(kx, ky, kz, wki, nx, ny, nz, &U[ik], &V[ik], &W[ik]);
      xi[ik] = nx; et[ik] = ny; zt[ik] = nz;
      RX[ik] = 0; RY[ik] = 0; RZ[ik] = 0;
    }
  }
  free(U); free(V); free(W); free(RX); free(RY); free(RZ);
  work3d_free(&w);
  return 0;
}

int orc_ns3d_timestep(double *xii, double *eta, double *zet, double *phys,
                      const double *nuzn, const double *nu1, int n, double alpha,
                      double ampfor, double kfy, double dt, int nstop,
                      double tstart, double *time) {
  return heun3d(0, 0, xii, eta, zet, phys, nuzn, nu1, n, alpha, ampfor, kfy, dt,
                nstop, tstart, time);
}

/* the Newton-solver build's step (3D_NavierStokes/src_gmres/cuda.cu:10-176):
 * the same Heun/CN scheme with its own forcing form */
int orc_ns3d_newton_timestep(double *xii, double *eta, double *zet, const double *nuzn,
                             const double *nu1, int n, double alpha, double ampfor, double kfy,
                             double dt, int nstop, double tstart, double *time) {
  return heun3d(0, 1, xii, eta, zet, NULL, nuzn, nu1, n, alpha, ampfor, kfy, dt, nstop,
                tstart, time);
}

int orc_euler3d_timestep(double *xii, double *eta, double *zet, double *phys,
                         int n, double alpha, double dt, int nstop,
                         double tstart, double *time) {
  return heun3d(1, 0, xii, eta, zet, phys, NULL, NULL, n, alpha, 0.0, 0.0, dt,
                nstop, tstart, time);
}

/* ------------------------------------------------------------------------ */
/* 3D Boussinesq RK4/CN                                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
  work3d_t w;
  cplx *U, *V, *W, *RK;   /* spectral velocity, then F(-(u x w)), F(u.grad rho) */
  double nu, ri, sc, sinth, costh, ampfor, kfy;
} bous_t;

/* KR_FFT_ALL (3D_Boussinesq/src/functions.h:60-125) + multReal (kernels.h:298-328)
 * + RK_FFT (functions.h:129-165) applied to the stage state (x0,e0,z0,r0). */
static void bous_rhs_transforms(bous_t *b, cplx *x0, cplx *e0, cplx *z0, cplx *r0) {
  work3d_t *w = &b->w;
  geom_t *g = &w->g;
  cplx *f6[6] = {x0, e0, z0, b->U, b->V, b->W};
  kr_fft_all(w, f6);
  conj3d(g, r0, w->T);
  pad(g, w->T, g->kx, w->F); c2r(g, w->F, w->R[6]);
  pad(g, w->T, g->ky, w->F); c2r(g, w->F, w->R[7]);
  pad(g, w->T, g->kz, w->F); c2r(g, w->F, w->R[8]);
  double *X = w->R[0], *E = w->R[1], *Zt = w->R[2], *Ur = w->R[3], *Vr = w->R[4], *Wr = w->R[5];
  double *rx = w->R[6], *ry = w->R[7], *rz = w->R[8];
#pragma omp parallel for schedule(static)
  for (long i = 0; i < g->nr; ++i) {
    double TU = Ur[i], TV = Vr[i], TW = Wr[i], TX = X[i], TE = E[i], TZ = Zt[i];
    double NX = TV * TZ - TW * TE, NY = TW * TX - TU * TZ, NZ = TU * TE - TV * TX;
    Ur[i] = -NX; Vr[i] = -NY; Wr[i] = -NZ;
    rx[i] = TU * rx[i] + TV * ry[i] + TW * rz[i];
  }
  double *rr[4] = {Ur, Vr, Wr, rx};
  cplx *out[4] = {b->U, b->V, b->W, b->RK};
  rk_fft(w, rr, out, 4);
}

/* the spectral right-hand side of Step1/Step2/Step/RHS (kernels.h:340-384):
 * curl + buoyancy (masked by LC when masked != 0), density rhs, forcing. */
static void bous_point_rhs(const bous_t *b, long ik, int masked, const cplx *x0,
                           const cplx *e0, const cplx *z0, const cplx *r0,
                           cplx *nx, cplx *ny, cplx *nz, cplx *nr) {
  const geom_t *g = &b->w.g;
  double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
  double wk = kx * kx + ky * ky + kz * kz, wki = wkinv(wk);
  double ROX = creal(r0[ik]), ROY = cimag(r0[ik]);
  double rXR = -kx * ROY, rXC = kx * ROX, rYR = -ky * ROY, rYC = ky * ROX;
  double rZR = -kz * ROY, rZC = kz * ROX;
  double LC = masked ? g->LL[ik] : 1.0;
  double UKX = creal(b->U[ik]), UKY = cimag(b->U[ik]), VKX = creal(b->V[ik]);
  double VKY = cimag(b->V[ik]), WKX = creal(b->W[ik]), WKY = cimag(b->W[ik]);
  double ri = b->ri, S = b->sinth, C = b->costh;
  double xiX = LC * (ky * WKY - kz * VKY - ri * (rYR * S - rZR * C));
  double xiY = LC * (kz * VKX - ky * WKX - ri * (rYC * S - rZC * C));
  double etX = LC * (kz * UKY - kx * WKY + ri * rXR * S);
  double etY = LC * (kx * WKX - kz * UKX + ri * rXC * S);
  double ztX = LC * (kx * VKY - ky * UKY - ri * rXR * C);
  double ztY = LC * (ky * UKX - kx * VKX - ri * rXC * C);
  double rr = -LC * (creal(b->RK[ik]) + (kz * cimag(x0[ik]) - kx * cimag(z0[ik])) * wki * C +
                     (kx * cimag(e0[ik]) - ky * cimag(x0[ik])) * wki * S);
  double ri_ = -LC * (cimag(b->RK[ik]) + (kx * creal(z0[ik]) - kz * creal(x0[ik])) * wki * C +
                      (ky * creal(x0[ik]) - kx * creal(e0[ik])) * wki * S);
  if (kx == 0.0 && kz == 0.0 && ky == b->kfy) ztX += b->ampfor;
  *nx = xiX + I * xiY; *ny = etX + I * etY; *nz = ztX + I * ztY; *nr = rr + I * ri_;
}

static void bous_velocity(bous_t *b, const cplx *x0, const cplx *e0, const cplx *z0) {
  geom_t *g = &b->w.g;
#pragma omp parallel for schedule(static)
  for (long ik = 0; ik < g->nkt; ++ik) {
    double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
    double wki = wkinv(kx * kx + ky * ky + kz * kz);
    vel3d(kx, ky, kz, wki, x0[ik], e0[ik], z0[ik], &b->U[ik], &b->V[ik], &b->W[ik]);
  }
}

static int bous_init(bous_t *b, int n, double alpha, double ampfor, double kfy,
                     double nu, double ri, double sc, double theta) {
  if (work3d_init(&b->w, n, alpha, 9)) return -1;
  long nkt = b->w.g.nkt;
  b->U = (cplx *)calloc(nkt, sizeof(cplx)); b->V = (cplx *)calloc(nkt, sizeof(cplx));
  b->W = (cplx *)calloc(nkt, sizeof(cplx)); b->RK = (cplx *)calloc(nkt, sizeof(cplx));
  b->nu = nu; b->ri = ri; b->sc = sc; b->sinth = sin(theta); b->costh = cos(theta);
  b->ampfor = ampfor; b->kfy = kfy;
  return 0;
}
static void bous_free(bous_t *b) {
  free(b->U); free(b->V); free(b->W); free(b->RK);
  work3d_free(&b->w);
}

/* one RK4/CN step of length dt (cuda.cu:192-211 / kernels.h Step1,Step1,Step2,Step) */
static void bous_step(bous_t *b, double dt, cplx *st[4], cplx *s0[4], cplx *k1[4],
                      cplx *k2[4], cplx *k3[4]) {
  geom_t *g = &b->w.g;
  long nkt = g->nkt;
  double nu = b->nu, sc = b->sc;
  cplx **kr[3] = {k1, k2, k3};
  for (int stage = 0; stage < 3; ++stage) {
    bous_rhs_transforms(b, s0[0], s0[1], s0[2], s0[3]);
    double q = (stage == 2) ? 0.5 : 0.25;  /* damp factor: 1/4 dt (Step1), 1/2 dt (Step2) */
    double fr = (stage == 2) ? 1.0 : 0.5;
#pragma omp parallel for schedule(static)
    for (long ik = 0; ik < nkt; ++ik) {
      cplx r[4];
      bous_point_rhs(b, ik, 1, s0[0], s0[1], s0[2], s0[3], &r[0], &r[1], &r[2], &r[3]);
      double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
      double wk = kx * kx + ky * ky + kz * kz;
      double d1 = (1. - q * dt * nu * wk) / (1. + q * dt * nu * wk);
      double d2 = (1. - q * dt * nu * wk / sc) / (1. + q * dt * nu * wk / sc);
      for (int c = 0; c < 4; ++c) {
        kr[stage][c][ik] = dt * r[c];
        double d = (c < 3) ? d1 : d2;
        s0[c][ik] = d * (st[c][ik] + fr * dt * r[c]);
      }
    }
    bous_velocity(b, s0[0], s0[1], s0[2]);
  }
  bous_rhs_transforms(b, s0[0], s0[1], s0[2], s0[3]);
#pragma omp parallel for schedule(static)
  for (long ik = 0; ik < nkt; ++ik) {
    cplx r[4];
    bous_point_rhs(b, ik, 0, s0[0], s0[1], s0[2], s0[3], &r[0], &r[1], &r[2], &r[3]);
    double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
    double wk = kx * kx + ky * ky + kz * kz, wki = wkinv(wk);
    double LC = g->LL[ik];
    double d1 = 1. - 0.5 * dt * nu * wk, d2 = 1. - 0.5 * dt * nu * wk / sc;
    for (int c = 0; c < 4; ++c) {
      double d = (c < 3) ? d1 : d2;
      double den = (c < 3) ? (1. + 0.5 * dt * nu * wk) : (1. + 0.5 * dt * nu * wk / sc);
      double re = LC * (d * creal(st[c][ik]) + (1.0 / 6.0) * (creal(k1[c][ik]) + dt * creal(r[c])) +
                        (1.0 / 3.0) * (creal(k2[c][ik]) + creal(k3[c][ik]))) / den;
      double im = LC * (d * cimag(st[c][ik]) + (1.0 / 6.0) * (cimag(k1[c][ik]) + dt * cimag(r[c])) +
                        (1.0 / 3.0) * (cimag(k2[c][ik]) + cimag(k3[c][ik]))) / den;
      st[c][ik] = re + I * im;
      s0[c][ik] = st[c][ik];
    }
    /* remove the divergence of the vorticity (kernels.h:597-606) */
    double phiR = (kx * cimag(st[0][ik]) + ky * cimag(st[1][ik]) + kz * cimag(st[2][ik])) * wki;
    double phiC = -(kx * creal(st[0][ik]) + ky * creal(st[1][ik]) + kz * creal(st[2][ik])) * wki;
    st[0][ik] -= (-kx * phiC) + I * (kx * phiR);
    st[1][ik] -= (-ky * phiC) + I * (ky * phiR);
    st[2][ik] -= (-kz * phiC) + I * (kz * phiR);
  }
  bous_velocity(b, s0[0], s0[1], s0[2]);
}

int orc_bous3d_timestep(double *xii, double *eta, double *zet, double *rho, int n,
                        double alpha, double ampfor, double kfy, double nu, double ri,
                        double sc, double theta, double dt, double tstart, double tend,
                        double *time) {
  bous_t b;
  if (bous_init(&b, n, alpha, ampfor, kfy, nu, ri, sc, theta)) return -1;
  long nkt = b.w.g.nkt;
  cplx *st[4] = {(cplx *)xii, (cplx *)eta, (cplx *)zet, (cplx *)rho};
  cplx *s0[4], *k1[4], *k2[4], *k3[4];
  for (int c = 0; c < 4; ++c) {
    s0[c] = (cplx *)malloc(sizeof(cplx) * nkt);
    k1[c] = (cplx *)calloc(nkt, sizeof(cplx));
    k2[c] = (cplx *)calloc(nkt, sizeof(cplx));
    k3[c] = (cplx *)calloc(nkt, sizeof(cplx));
    memcpy(s0[c], st[c], sizeof(cplx) * nkt);   /* setVelocity copies x0 = xii ... */
  }
  bous_velocity(&b, s0[0], s0[1], s0[2]);
  /* setVelocity masks wki by LL (kernels.h:216-217) */
  {
    geom_t *g = &b.w.g;
    for (long ik = 0; ik < nkt; ++ik)
      if (!g->LL[ik]) { b.U[ik] = 0; b.V[ik] = 0; b.W[ik] = 0; }
  }
  double tme = tstart;
  int steps = 0;
  while (tend - tme > dt) {  /* src_gmres/cuda.cu:187 */
    ++steps;
    bous_step(&b, dt, st, s0, k1, k2, k3);
    *time += dt;
    tme += dt;
  }
  if (tme != tend) {          /* src_gmres/cuda.cu:218-249 */
    double d = tend - tme;
    bous_step(&b, d, st, s0, k1, k2, k3);
  }
  for (int c = 0; c < 4; ++c) { free(s0[c]); free(k1[c]); free(k2[c]); free(k3[c]); }
  bous_free(&b);
  return steps;
}

/* timederiv_cuda_ (3D_Boussinesq/src/src_gmres/cuda.cu:319-533 with RHS
 * kernels.h:624-692): x0.. = z, one transform set, dz/dt out. */
int orc_bous3d_timederiv(const double *xii, const double *eta, const double *zet,
                         const double *rho, double *dxii, double *deta, double *dzet,
                         double *drho, int n, double alpha, double ampfor, double kfy,
                         double nu, double ri, double sc, double theta) {
  bous_t b;
  if (bous_init(&b, n, alpha, ampfor, kfy, nu, ri, sc, theta)) return -1;
  geom_t *g = &b.w.g;
  long nkt = g->nkt;
  cplx *s0[4];
  const double *in[4] = {xii, eta, zet, rho};
  cplx *out[4] = {(cplx *)dxii, (cplx *)deta, (cplx *)dzet, (cplx *)drho};
  for (int c = 0; c < 4; ++c) {
    s0[c] = (cplx *)malloc(sizeof(cplx) * nkt);
    memcpy(s0[c], in[c], sizeof(cplx) * nkt);
  }
  for (long ik = 0; ik < nkt; ++ik) {
    double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
    double wki = g->LL[ik] ? wkinv(kx * kx + ky * ky + kz * kz) : 0.0;
    vel3d(kx, ky, kz, wki, s0[0][ik], s0[1][ik], s0[2][ik], &b.U[ik], &b.V[ik], &b.W[ik]);
  }
  bous_rhs_transforms(&b, s0[0], s0[1], s0[2], s0[3]);
  for (long ik = 0; ik < nkt; ++ik) {
    cplx r[4];
    bous_point_rhs(&b, ik, 1, s0[0], s0[1], s0[2], s0[3], &r[0], &r[1], &r[2], &r[3]);
    double kx = g->kx[ik], ky = g->ky[ik], kz = g->kz[ik];
    double wk = kx * kx + ky * ky + kz * kz;
    double d1 = -nu * wk, d2 = -nu * wk / sc;
    for (int c = 0; c < 4; ++c) out[c][ik] = ((c < 3) ? d1 : d2) * s0[c][ik] + r[c];
  }
  for (int c = 0; c < 4; ++c) free(s0[c]);
  bous_free(&b);
  return 0;
}

double orc_energy3d(const double *xii, const double *eta, const double *zet, int n,
                    double alpha) {
  geom_t g;
  if (geom_init(&g, 3, n, alpha)) return -1.0;
  const cplx *a = (const cplx *)xii, *b = (const cplx *)eta, *c = (const cplx *)zet;
  double e = 0.0;
  for (long ik = 0; ik < g.nkt; ++ik) {
    if (!g.LL[ik]) continue;
    double wk = g.kx[ik] * g.kx[ik] + g.ky[ik] * g.ky[ik] + g.kz[ik] * g.kz[ik];
    double vz = creal(a[ik] * conj(a[ik])) + creal(b[ik] * conj(b[ik])) + creal(c[ik] * conj(c[ik]));
    e += vz / (wk > 0.001 ? wk : 0.001);
  }
  geom_free(&g);
  return e;
}
