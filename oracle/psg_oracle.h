/*
 * psg_oracle.h -- FP64 CPU restatement of psgpu's pseudospectral time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * The product (psgpu_b200) never links or calls it.
 *
 * Every routine restates the reference algorithm step by step (cited per
 * function in psg_oracle.c) with a project-written radix-2 FFT in place of
 * cuFFT.  Layouts are the reference's: the truncated spectral box is stored
 * Fortran-order with kx fastest, ik = (ikz*IKTY + iky)*IKTX + ikx, and the
 * padded FFT arrays follow cufftPlan3d(NZ,NY,NX) (x fastest, NX/2+1 complex).
 *
 * Parity pin: the oracle is checked against golden vectors produced by the
 * reference's own CUDA timestep_cuda_ (built from its sources into oracle/_ref
 * and run on a B200); see tests/golden/make_golden.py.
 */
#ifndef PSG_ORACLE_H
#define PSG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- layout helpers (2D_NavierStokes/src_RK4/src_gmres/init.F90:25-39,
 *      main.F90:292-335; 3D_NavierStokes/src/init.F90:25-64, main.F90:100-199) */
int  orc_nkt2d(int n);
int  orc_nkt3d(int n);
void orc_layout2d(int n, double alpha, double *kx, double *ky, int *LL);
void orc_layout3d(int n, double alpha, double *kx, double *ky, double *kz, int *LL);
void orc_ikf2d(int n, int *ikF);      /* length (n/2+1)*n   */
void orc_ikn2d(int n, int *ikN);      /* length nkt2d        */
void orc_ikf3d(int n, int *ikF);      /* length (n/2+1)*n*n */
void orc_ikn3d(int n, int *ikN);      /* length nkt3d        */

/* ---- 2D vorticity RK4 + final Crank-Nicolson factor
 *      (2D_NavierStokes/src_RK4/src_gmres/cuda.cu:16-83, kernels.h:112-435).
 *      Z: complex128 interleaved [IKTY][IKTX], overwritten.  *time is reset to
 *      0 and advanced by dt per step, as the reference does.              */
int orc_ns2d_timestep(double *Z, int n, double alpha, double nu, double dt,
                      int nstop, double *time);

/* dZ/dt = -nu k^2 Z + N(Z) + forcing, the CPU TIMEDERIV of the Newton solver
 * (2D_NavierStokes/src_RK4/src_gmres/timederiv.F90:2-32, convol.F90:2-64).
 * nuk2 is NU(ikx,iky) = 10**(log10(v2)+2 log10|k|) as the driver builds it. */
int orc_ns2d_timederiv(const double *Z, double *dZ, int n, double alpha, double nu);

/* ---- 3D Navier-Stokes Heun predictor-corrector with Crank-Nicolson viscosity
 *      (3D_NavierStokes/src/cuda.cu:18-151, kernels.h:113-464).  State xii,eta,zet
 *      complex128 [IKTZ][IKTY][IKTX] overwritten; phys (may be NULL) receives the
 *      three physical vorticity fields of the last predictor transform, n^3 each. */
int orc_ns3d_newton_timestep(double *xii, double *eta, double *zet, const double *nuzn,
                             const double *nu1, int n, double alpha, double ampfor, double kfy,
                             double dt, int nstop, double tstart, double *time);
int orc_ns3d_timestep(double *xii, double *eta, double *zet, double *phys,
                      const double *nuzn, const double *nu1,
                      int n, double alpha, double ampfor, double kfy,
                      double dt, int nstop, double tstart, double *time);

/* ---- 3D Euler Heun (3D_Euler/src/cuda.cu:17-123, kernels.h:296-439). */
int orc_euler3d_timestep(double *xii, double *eta, double *zet, double *phys,
                         int n, double alpha, double dt, int nstop,
                         double tstart, double *time);

/* ---- 3D Boussinesq RK4 with per-stage CN factors, GMRES build semantics
 *      (3D_Boussinesq/src/src_gmres/cuda.cu:12-314, kernels.h:331-621).
 *      Integrates from tstart to tend with the reference's loop
 *      while(tend - t > dt) plus one adjusted final step.  Returns the number
 *      of full steps taken (the adjusted step not counted).               */
int orc_bous3d_timestep(double *xii, double *eta, double *zet, double *rho,
                        int n, double alpha, double ampfor, double kfy,
                        double nu, double ri, double sc, double theta,
                        double dt, double tstart, double tend, double *time);

/* dz/dt of the Boussinesq system (3D_Boussinesq/src/src_gmres/cuda.cu:319-533,
 * kernels.h:624-692); outputs into dxii..drho. */
int orc_bous3d_timederiv(const double *xii, const double *eta, const double *zet,
                         const double *rho, double *dxii, double *deta,
                         double *dzet, double *drho, int n, double alpha,
                         double ampfor, double kfy, double nu, double ri,
                         double sc, double theta);

/* ---- diagnostics over the kept modes (FP64 sums) */
double orc_energy3d(const double *xii, const double *eta, const double *zet, int n, double alpha);

int  orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
