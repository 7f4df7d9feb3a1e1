/*
 * psgpu_host.h -- host-side pieces of psgpu's drivers, restated in C so that a
 * driver can be written without the Fortran front end: the parameter file,
 * the seeded initial conditions (and their random-number generator), the
 * Fortran sequential-record files the drivers read and write, and the
 * statistics lines of the 3D DNS.  All of it lives in libpsgpu.so; none of it
 * touches the GPU.  psg_dns3 (psgpu_b200/host/psg_dns3.c) is a 3D
 * Navier-Stokes DNS driver built on these and on psg_ns3d_*.
 */
#ifndef PSGPU_HOST_H
#define PSGPU_HOST_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ parameters */
/* The 3D Navier-Stokes params.txt, read in the order and with the labels of
 * 3D_NavierStokes/src/parameters.F90:136-157 ("ISEED = ", ..., "ISTOP = "),
 * and the derived values of params_update (parameters.F90:28-40). */
typedef struct {
  int iseed, irest;
  char infile[256], infile_type[256];
  int kf;
  double re, tstep, residual_threshold, outfreq1, outfreq2, delt, ampv;
  int statsflag, rcflag, upoflag, istop;
  /* derived */
  double v2, ampfor;
  int nstop, nout, noutv;
} psg_params3d;

/* 0 on success; -1 (and a message in psg_last_error) when the file is
 * missing or a label does not match */
int psg_read_params3d(const char* path, psg_params3d* p);

/* ------------------------------------------------------- random numbers */
/* The drivers' generator: ranno(i) over ran1, the minimal-standard
 * multiplicative congruential generator (a = 16807, m = 2^31 - 1, Schrage's
 * factorisation) with a 32-entry Bays-Durham shuffle, as
 * 3D_NavierStokes/src/init.F90:236-292 states it.  ranno(seed != 0) seeds
 * it; ranno(0) draws the next phase, uniform in (-pi, pi). */
typedef struct {
  int junk, iy;
  int iv[32];
} psg_ranno_state;

void psg_ranno_init(psg_ranno_state* s);
double psg_ranno(psg_ranno_state* s, int i);

/* ------------------------------------------------- initial conditions */
/* 3D Navier-Stokes random start (3D_NavierStokes/src/init.F90:151-230):
 * unit-modulus vorticity components with random phases on the kept modes
 * 2.5 < |k| <= 9.5 (three draws per kept mode, kx outermost, kz innermost),
 * scaled so that 2 sum |w|^2 = ampv.  Seeds the generator with iseed first,
 * as the driver's TIME = RANNO(ISEED) does.  Boxes: IKTZ*IKTY*IKTX complex
 * (interleaved double pairs), kx fastest. */
int psg_ic_random3d(int n, int iseed, double ampv, double* xii, double* eta, double* zet);
/* 2D random start (2D_NavierStokes/src_RK4/src_gmres/init.F90:146-213):
 * unit modulus on 2.5 < |k| <= 9.5 with kx >= 1, one draw per kept mode,
 * 2 sum |Z|^2 = ampv; box IKTY*IKTX complex. */
int psg_ic_random2d(int n, int iseed, double ampv, double* Z);

/* ------------------------------------------- Fortran sequential records */
/* One record: a 4-byte length marker, the payload (the concatenation of the
 * given parts), the marker again (gfortran's default sequential layout). */
int psg_frec_write(FILE* f, const void* const* parts, const size_t* sizes, int nparts);
/* Reads one record into buf (at most cap bytes); *len = its payload size.
 * 0 on success, -1 at end of file or on a malformed / oversized record. */
int psg_frec_read(FILE* f, void* buf, size_t cap, size_t* len);

/* The state files the 3D drivers restart from (3D_NavierStokes/src/init.F90:66-140):
 * type "A"/"B": stream records (time, v2 or a dummy, period, shift x/y/z,
 * residual, xii, eta, zet); "C": sequential records of (xii, eta, zet);
 * "D": sequential, a header record (count, IKTX, IKTY, IKTZ) then records as
 * "A".  Reads the irest-th record (1-based) of a file of the same grid;
 * meta[7] = time, v2, period, shiftx, shifty, shiftz, residual (zeros for
 * "C").  0 on success. */
int psg_read_state3d(const char* path, const char* type, int irest, int n, double* meta,
                     double* xii, double* eta, double* zet);
/* Writes a type "D" file: the header record, then one record per state. */
int psg_write_state3d_header(FILE* f, int count, int n);
int psg_write_state3d_record(FILE* f, int n, const double* meta, const double* xii,
                             const double* eta, const double* zet);

/* ----------------------------------------------------------- statistics */
/* The 3D DNS statistics (3D_NavierStokes/src/functions.h:128-209): per call
 * one stats.dat line "t energy eturb diss dturb input" and one engy.dat line
 * "t Ua Va Wa XIa ETa ZTa", with the running time averages of the state
 * behind eturb / dturb kept in the accumulator. */
typedef struct psg_stats3d psg_stats3d;
psg_stats3d* psg_stats3d_create(int n, double v2, double ampfor, int kf);
void psg_stats3d_destroy(psg_stats3d* s);
int psg_stats3d_add(psg_stats3d* s, double t, const double* xii, const double* eta,
                    const double* zet, FILE* stats, FILE* engy);
/* the same, keeping the energy, dissipation and input at history index
 * nt/nout - 1 (nt: the step index of the reference's loop, functions.h:197-200) */
int psg_stats3d_add_at(psg_stats3d* s, int nt, int nout, double t, const double* xii,
                       const double* eta, const double* zet, FILE* stats, FILE* engy);
/* the number of statistics added so far (the reference's tavgCount) */
double psg_stats3d_count(const psg_stats3d* s);
/* the running time average of the state (XIItavg, ETAtavg, ZETtavg), reference layout */
int psg_stats3d_mean(const psg_stats3d* s, double* xii, double* eta, double* zet);
/* the DNS's end-of-run statistics (3D_NavierStokes/src/finalise.h:19-166): avgs
 * (five records: time, n^3 doubles of U, V, W of the time average, mean v^2, mean
 * u^2 - U^2), means (y, z and x averages of U, V, u variance and mean v^2 per
 * (z, y)) and pdfs (100 bins of energy, dissipation and input); uvw: the
 * physical velocity of psg_stats3d_mean's state, ms: the running mean squares
 * of the physical velocity (psg_ns3d_rms_download); any FILE may be NULL */
int psg_stats3d_finish(psg_stats3d* s, int nstop, int nout, double time,
                       const double* const* uvw, const double* const* ms, FILE* avgs,
                       FILE* means, FILE* pdfs);

#ifdef __cplusplus
}
#endif
#endif
