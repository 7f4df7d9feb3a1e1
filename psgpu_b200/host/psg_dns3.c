/* psg_dns3 -- 3D Navier-Stokes DNS driver on psgpu_b200, in place of the
 * reference's Fortran front end (3D_NavierStokes/src/main.F90).
 *
 *   psg_dns3 [-n N] [-d JOBDIR] [-p 32|64]
 *
 * Reads JOBDIR/params.txt (JOBDIR defaults to JOB<rank>, the rank taken from
 * the MPI launcher's environment, as main.F90:38 names it), builds the random
 * start (or reads the restart file named there), integrates NSTOP Heun /
 * Crank-Nicolson steps with the DNS forcing, writes JOBDIR/stats.dat and
 * JOBDIR/engy.dat every NOUT steps as the reference's statistics do
 * (3D_NavierStokes/src/cuda.cu:116-140), with RCFLAG = 1 the recurrence
 * search's UPO_ZK.out / UPOinfo_ts.dat, every NOUTV steps (NT = 0, NOUTV, ...,
 * when NSTOP > 1) the physical vorticity of the state before step NT as raw
 * FP64 volumes JOBDIR/xii%03d.raw, eta%03d.raw, zet%03d.raw, x fastest
 * (3D_NavierStokes/src/cuda.cu:72-93), and JOBDIR/Zk.out: main.F90's header
 * record (1, IKTX, IKTY, IKTZ) followed by the final state as a type "D"
 * restart record.  With STATSFLAG = 1 it also keeps the running mean squares
 * of the physical velocity (every NOUT steps, kernels.h:70-81) and at the end
 * writes avgs.dat, means.dat and pdfs.dat (finalise.h:19-166).  The grid is
 * compile-time in the reference (global_params.F90, 128^3); here it is -n
 * (default 128). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "psgpu.h"
#include "psgpu_host.h"

static int env_rank(void) {
  const char* names[] = {"OMPI_COMM_WORLD_RANK", "PMI_RANK", "RANK"};
  for (int i = 0; i < 3; ++i) {
    const char* v = getenv(names[i]);
    if (v) return atoi(v);
  }
  return 0;
}

static double now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

#define FAIL(...) do { fprintf(stderr, "psg_dns3: " __VA_ARGS__); fprintf(stderr, "\n"); return 1; } while (0)

int main(int argc, char** argv) {
  int n = 128, prec = 32;
  char dir[512];
  snprintf(dir, sizeof dir, "JOB%d", env_rank());
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "-n") && i + 1 < argc) n = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-d") && i + 1 < argc) snprintf(dir, sizeof dir, "%s", argv[++i]);
    else if (!strcmp(argv[i], "-p") && i + 1 < argc) prec = atoi(argv[++i]);
    else FAIL("usage: psg_dns3 [-n N] [-d JOBDIR] [-p 32|64]");
  }
  char path[1024];
  psg_params3d P;
  snprintf(path, sizeof path, "%s/params.txt", dir);
  if (psg_read_params3d(path, &P)) FAIL("%s", psg_last_error());
  const int K = n / 3;
  const long nkt = (long)(K + 1) * (2 * K + 1) * (2 * K + 1);
  double* st[3];
  for (int q = 0; q < 3; ++q)
    if (!(st[q] = (double*)calloc(2 * nkt, sizeof(double)))) FAIL("out of host memory");
  double meta[7] = {0};
  if (P.irest == 0) {
    if (psg_ic_random3d(n, P.iseed, P.ampv, st[0], st[1], st[2])) FAIL("%s", psg_last_error());
  } else {
    snprintf(path, sizeof path, "%s/%s", dir, P.infile);
    if (psg_read_state3d(path, P.infile_type, P.irest, n, meta, st[0], st[1], st[2]))
      FAIL("%s", psg_last_error());
    if (P.infile_type[0] == 'A' || P.infile_type[0] == 'D') P.v2 = meta[1];
  }
  if (P.upoflag == 1) P.tstep = meta[2];  /* main.F90:68-77 */
  P.nstop = (int)(P.tstep / P.delt);
  printf("        Re= %g\n          NSTOP= %d\n          NOUT= %d\n          NOUTV= %d\n",
         1.0 / P.v2, P.nstop, P.nout, P.noutv);

  psg_ns3d* h = NULL;
  if (psg_ns3d_create(&h, n, 1.0, PSG_SCHEME_NS_HEUN, prec) ||
      psg_ns3d_set_params(h, P.v2, P.ampfor, (double)P.kf, 0.0, 1.0, 0.0))
    FAIL("%s", psg_last_error());
  const double* in[3] = {st[0], st[1], st[2]};
  double* out[3] = {st[0], st[1], st[2]};
  if (psg_ns3d_upload(h, in)) FAIL("%s", psg_last_error());

  FILE *fs = NULL, *fe = NULL, *fu = NULL, *fi = NULL, *fa = NULL, *fm = NULL, *fp = NULL;
  psg_stats3d* S = NULL;
  psg_rec3d* rec = NULL;
  if (P.rcflag == 1) {
    /* recurrence search (init.h:182-213): UPO guesses into UPO_ZK.out (a type A
     * stream) and UPOinfo_ts.dat */
    if (psg_rec3d_create(&rec, n, 1.0, 500, 8, 30, 2, 2, P.residual_threshold, P.nout, P.delt,
                         0.0, P.v2) ||
        psg_rec3d_start_engine(rec, h))
      FAIL("%s", psg_last_error());
    snprintf(path, sizeof path, "%s/UPO_ZK.out", dir);
    fu = fopen(path, "wb");
    snprintf(path, sizeof path, "%s/UPOinfo_ts.dat", dir);
    fi = fopen(path, "w");
    if (!fu || !fi) FAIL("cannot open the recurrence files in %s", dir);
    fprintf(fi, "Guess No : Start time : guess Period : guess Shift x: guess Shift y: guess Residual \n");
  }
  if (P.statsflag) {
    /* the statistics files of init.h:114-133 */
    static const char* names[5] = {"stats.dat", "engy.dat", "avgs.dat", "means.dat", "pdfs.dat"};
    FILE** fl[5] = {&fs, &fe, &fa, &fm, &fp};
    for (int k = 0; k < 5; ++k) {
      snprintf(path, sizeof path, "%s/%s", dir, names[k]);
      *fl[k] = fopen(path, k == 2 ? "wb" : "w");
      if (!*fl[k]) FAIL("cannot open %s", path);
    }
    S = psg_stats3d_create(n, P.v2, P.ampfor, P.kf);
    if (!S) FAIL("out of host memory");
  }
  const long nr = (long)n * n * n;
  /* the fields a step starts from are kept (the raw volumes and the mean
   * squares hold those of the state before step NT, cuda.cu:68-93); the
   * velocity too when statistics are on */
  if (psg_ns3d_dump_mode(h, 1 | (S ? 2 : 0))) FAIL("%s", psg_last_error());
  const double t0 = now();
  int done = 0;
  double* vol[3] = {NULL, NULL, NULL};
  int nvol = 0;
  const int want_vol = P.noutv > 0 && P.nstop > 1;
  if (want_vol)
    for (int q = 0; q < 3; ++q)
      if (!(vol[q] = (double*)malloc(sizeof(double) * nr))) FAIL("out of host memory");
  int izkout = 0;
  /* events at the step index NT of the reference's loop (NT = 0 .. NSTOP-1): a raw
   * volume of the state before step NT (NT a multiple of NOUTV), the mean squares
   * of its velocity (statistics on, NT a multiple of NOUT), then after the step
   * the recurrence check and the statistics of the new state (NT a multiple of
   * NOUT, NT > 0) */
  int next_vol = want_vol ? 0 : P.nstop;
  int next_out = (S || rec) ? 0 : P.nstop;
  for (;;) {
    const int NT = next_vol < next_out ? next_vol : next_out;
    if (NT >= P.nstop) break;
    const int is_vol = NT == next_vol, is_out = NT == next_out;
    const int want_dump = is_vol || (is_out && S);
    if (NT + 1 > done && psg_ns3d_step(h, P.delt, NT + 1 - done, want_dump))
      FAIL("%s", psg_last_error());
    done = NT + 1;
    if (is_vol) {
      static const char* names[3] = {"xii", "eta", "zet"};
      if (psg_ns3d_download_phys(h, vol)) FAIL("%s", psg_last_error());
      ++nvol;
      for (int q = 0; q < 3; ++q) {
        snprintf(path, sizeof path, "%s/%s%03d.raw", dir, names[q], nvol);
        FILE* fv = fopen(path, "wb");
        if (!fv || fwrite(vol[q], sizeof(double), nr, fv) != (size_t)nr) FAIL("cannot write %s", path);
        fclose(fv);
      }
      next_vol += P.noutv;
    }
    if (!is_out) continue;
    next_out += P.nout;
    if (S && psg_ns3d_rms_accumulate(h, psg_stats3d_count(S))) FAIL("%s", psg_last_error());
    if (NT == 0) continue;
    const double tme = done * P.delt;
    if (rec) {
      int emitted = 0;
      if (psg_rec3d_add_engine(rec, NT, h, &emitted)) FAIL("%s", psg_last_error());
      if (emitted) {
        double meta[7];
        if (psg_rec3d_guess(rec, meta, st[0], st[1], st[2])) FAIL("%s", psg_last_error());
        fwrite(meta, sizeof(double), 7, fu);
        for (int q = 0; q < 3; ++q) fwrite(st[q], 2 * sizeof(double), nkt, fu);
        ++izkout;
        fprintf(fi, "%d %e %e %e %e %e %e \n", izkout, meta[0], meta[2], meta[3], meta[4], meta[5],
                meta[6]);
        fflush(fu);
        fflush(fi);
      }
    }
    if (S && !(P.statsflag == 2 && tme <= 500.0)) {
      if (psg_ns3d_download(h, out)) FAIL("%s", psg_last_error());
      if (psg_stats3d_add_at(S, NT, P.nout, tme, st[0], st[1], st[2], fs, fe))
        FAIL("%s", psg_last_error());
    }
  }
  if (done < P.nstop && psg_ns3d_step(h, P.delt, P.nstop - done, 0)) FAIL("%s", psg_last_error());
  if (psg_ns3d_download(h, out)) FAIL("%s", psg_last_error());
  const double el = now() - t0;

  snprintf(path, sizeof path, "%s/Zk.out", dir);
  FILE* fz = fopen(path, "wb");
  if (!fz) FAIL("cannot write %s", path);
  const double fin[7] = {P.nstop * P.delt, P.v2, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (psg_write_state3d_header(fz, 1, n) || psg_write_state3d_record(fz, n, fin, st[0], st[1], st[2]))
    FAIL("writing %s failed", path);
  fclose(fz);
  if (S && P.statsflag == 1 && P.nstop > 1) {
    /* finalise.h:19-166: the statistics of the final state, then the mean
     * profiles of the time average and the pdfs */
    const double tend = P.nstop * P.delt;
    if (psg_stats3d_add_at(S, P.nstop + 1, P.nout, tend, st[0], st[1], st[2], fs, fe))
      FAIL("%s", psg_last_error());
    double* fld[6];
    for (int q = 0; q < 6; ++q)
      if (!(fld[q] = (double*)malloc(sizeof(double) * nr))) FAIL("out of host memory");
    if (psg_stats3d_mean(S, st[0], st[1], st[2]) || psg_ns3d_upload(h, in) ||
        psg_ns3d_step(h, P.delt, 1, 1) || psg_ns3d_download_phys_velocity(h, fld) ||
        psg_ns3d_rms_download(h, fld + 3))
      FAIL("%s", psg_last_error());
    if (psg_stats3d_finish(S, P.nstop, P.nout, tend, (const double* const*)fld,
                           (const double* const*)(fld + 3), fa, fm, fp))
      FAIL("%s", psg_last_error());
    for (int q = 0; q < 6; ++q) free(fld[q]);
  }
  if (fa) fclose(fa);
  if (fm) fclose(fm);
  if (fp) fclose(fp);
  if (fs) fclose(fs);
  if (fe) fclose(fe);
  if (fu) fclose(fu);
  if (fi) fclose(fi);
  psg_rec3d_destroy(rec);
  psg_stats3d_destroy(S);
  psg_ns3d_destroy(h);
  for (int q = 0; q < 3; ++q) free(vol[q]);
  printf("time stepping done: %d steps in %.3f s (%.1f steps/s)\n", P.nstop, el,
         el > 0 ? P.nstop / el : 0.0);
  for (int q = 0; q < 3; ++q) free(st[q]);
  return 0;
}
