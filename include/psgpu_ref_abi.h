/*
 * psgpu_ref_abi.h -- the reference-compatible entry points of the drop-in
 * libraries libpsg_ns2d.so, libpsg_ns3d.so, libpsg_ns3d_newton.so,
 * libpsg_euler3d.so, libpsg_bous3d.so.
 *
 * psgpu's Fortran drivers call one C-ABI function per flavour with every
 * argument by pointer (Fortran by-reference ABI, no hidden lengths).  Each
 * drop-in library exports the same symbol names with the same argument
 * lists, so a driver links against it unchanged.  Every flavour exports
 * timestep_cuda_, hence one library per flavour; define exactly one of
 * PSG_ABI_NS2D, PSG_ABI_NS3D, PSG_ABI_EULER3D, PSG_ABI_BOUS3D, PSG_ABI_BOUS3D_DNS before including
 * this header to get that flavour's prototypes (PSG_ABI_NS3D_NEWTON for the
 * Newton-solver build's 3D step).
 *
 * double2 is CUDA's vector type (two doubles: real, imaginary).
 */
#ifndef PSGPU_REF_ABI_H
#define PSGPU_REF_ABI_H

#ifdef __CUDACC__
#include <vector_types.h>
#else
typedef struct { double x, y; } double2;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces set_gpu_ of every flavour (3D_NavierStokes/src/functions.h:3-20,
 * 2D_NavierStokes/src_RK4/functions.h:13-29, 3D_Boussinesq/src/functions.h:9-28). */
void set_gpu_(int* go);

#if defined(PSG_ABI_NS2D) || defined(PSG_FLAVOUR_NS2D)
/* 2D vorticity RK4 with a final Crank-Nicolson viscous factor; replaces
 * 2D_NavierStokes/src_RK4/src_gmres/cuda.cu:16-34 (called from
 * src_gmres/main.F90:708-710, 1076-1078, 1387-1389, 1483-1485). */
void timestep_cuda_(double2* Z, double* ZR, double* kx, double* ky, double* Time,
                    double* TSTART, double* TNEWT, double* DELT, double* alpha, double* V2,
                    int* ikF, int* ikN, int* IKTX, int* IKTY, int* KTY, int* NX, int* NY,
                    int* NSTOP, int* LC);
#endif

#if defined(PSG_ABI_NS3D) || defined(PSG_FLAVOUR_NS3D)
/* 3D Navier-Stokes Heun / Crank-Nicolson; replaces 3D_NavierStokes/src/cuda.cu:18-54
 * (called from 3D_NavierStokes/src/main.F90:203-204). */
void timestep_cuda_(double2* xii, double2* eta, double2* zet, double* xir, double* etr,
                    double* ztr, double* nuzn, double* nu1, double* kx, double* ky, double* kz,
                    double* Time, double* TSTART, double* AMPFOR, double* DELT,
                    double* ResThresh, double* KFY, double* V2, double* alpha, int* ikF,
                    int* ikN, int* LC, int* IKTX, int* IKTY, int* IKTZ, int* KTZ, int* NKT,
                    int* NX, int* NY, int* NZ, int* NSTOP, int* NOUT, int* NOUTV,
                    int* statsFLAG, int* RecFLAG, int* RANK);
#endif

#if defined(PSG_ABI_NS3D_NEWTON) || defined(PSG_FLAVOUR_NS3D_NEWTON)
/* 3D Navier-Stokes Heun / Crank-Nicolson as the Newton-solver build steps it
 * (its own forcing form, no outputs besides the state); replaces
 * 3D_NavierStokes/src_gmres/cuda.cu:10-28.  The reference fixes the grid in
 * its kernels.h (128^3); libpsg_ns3d_newton.so uses 128 unless PSG_NEWTON_N is
 * set in the environment. */
void timestep_cuda_(double2* xii, double2* eta, double2* zet, double* nuzn, double* nu1,
                    double* kx, double* ky, double* kz, double* Time, double* TSTART,
                    double* AMPFOR, double* DELT, int* KFY, double* V2, int* ikF, int* ikN,
                    int* LC, int* NSTOP);
#endif

#if defined(PSG_ABI_EULER3D) || defined(PSG_FLAVOUR_EULER3D)
/* 3D Euler Heun; replaces 3D_Euler/src/cuda.cu:17-44. */
void timestep_cuda_(double2* xii, double2* eta, double2* zet, double* xir, double* etr,
                    double* ztr, double* kx, double* ky, double* kz, double* Time,
                    double* TSTART, double* DELT, double* alpha, int* ikF, int* ikN, int* LC,
                    int* IKTX, int* IKTY, int* IKTZ, int* KTZ, int* NKT, int* NX, int* NY,
                    int* NZ, int* NSTOP, int* NOUT, int* NOUTV, int* statsFLAG);
#endif

#if defined(PSG_ABI_BOUS3D_DNS) || defined(PSG_FLAVOUR_BOUS3D_DNS)
/* 3D Boussinesq RK4/CN as its DNS build steps it (libpsg_bous3d_dns.so):
 * steps while t <= Tstep, the CFL-adaptive time step (adaptFLAG = 1) and the
 * forcing throttle towards Dtarget at output times; replaces
 * 3D_Boussinesq/src/cuda.cu:21-117 (called from src/main.F90:224-226). */
void timestep_cuda_(double2* xii, double2* eta, double2* zet, double2* rho, double* kx,
                    double* ky, double* kz, double* Time, double* TSTART, double* Tstep,
                    double* AMPFOR, double* DELT, double* ResThresh, double* KFY, double* V2,
                    double* Ri, double* Sc, double* Theta, double* alpha, double* Dtarget,
                    int* ikF, int* ikN, int* LC, int* IKTX, int* IKTY, int* IKTZ, int* KTZ,
                    int* NKT, int* NX, int* NY, int* NZ, int* NOUT, int* NOUTV,
                    int* statsFLAG, int* RecFLAG, int* adaptFLAG, int* RANK);
#endif

#if defined(PSG_ABI_BOUS3D) || defined(PSG_FLAVOUR_BOUS3D)
/* 3D Boussinesq RK4 with per-stage Crank-Nicolson factors as the Newton
 * solver's build steps it (libpsg_bous3d.so: full steps while Tstep - t > dt,
 * then one shorter step); replaces 3D_Boussinesq/src/src_gmres/cuda.cu:12-49. */
void timestep_cuda_(double2* xii, double2* eta, double2* zet, double2* rho, double* kx,
                    double* ky, double* kz, double* Time, double* TSTART, double* Tstep,
                    double* AMPFOR, double* DELT, double* ResThresh, double* KFY, double* V2,
                    double* Ri, double* Sc, double* Theta, double* alpha, double* Dtarget,
                    int* ikF, int* ikN, int* LC, int* IKTX, int* IKTY, int* IKTZ, int* KTZ,
                    int* NKT, int* NX, int* NY, int* NZ, int* NOUT, int* NOUTV,
                    int* statsFLAG, int* RecFLAG, int* adaptFLAG, int* RANK);
/* dz/dt; replaces 3D_Boussinesq/src/src_gmres/cuda.cu:319-356. */
void timederiv_cuda_(double2* xii, double2* eta, double2* zet, double2* rho, double* kx,
                     double* ky, double* kz, double* Time, double* TSTART, double* Tstep,
                     double* AMPFOR, double* DELT, double* ResThresh, double* KFY, double* V2,
                     double* Ri, double* Sc, double* Theta, double* alpha, double* Dtarget,
                     int* ikF, int* ikN, int* LC, int* IKTX, int* IKTY, int* IKTZ, int* KTZ,
                     int* NKT, int* NX, int* NY, int* NZ, int* NOUT, int* NOUTV,
                     int* statsFLAG, int* RecFLAG, int* adaptFLAG, int* RANK);
#endif

#ifdef __cplusplus
}
#endif
#endif
