/*
 * psgpu.h -- re-entrant C API of psgpu_b200 (libpsgpu.so).
 *
 * The reference (psgpu) exposes one non-re-entrant Fortran-ABI entry point
 * per flavour, timestep_cuda_, that allocates, plans, copies, integrates and
 * frees on every call (declared in psgpu_ref_abi.h, exported by the drop-in
 * libraries).  This API is the persistent form of the same step: a handle
 * owns device buffers and an explicit stream; the state stays resident in HBM
 * between calls; every function returns a status (PSG_OK = 0) and
 * psg_last_error() describes the last failure of the calling thread.
 *
 * Host state arrays use the reference's layout: complex128 interleaved boxes,
 * kx fastest, ik = (ikz*IKTY + iky)*IKTX + ikx (3D) or iky*IKTX + ikx (2D),
 * IKTX = N/3+1, IKTY = IKTZ = 2*(N/3)+1.
 */
#ifndef PSGPU_H
#define PSGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PSG_VERSION 100

#define PSG_OK 0
#define PSG_ERR_ARG 1
#define PSG_ERR_CUDA 2
#define PSG_ERR_UNSUPPORTED 3
#define PSG_ERR_STATE 4

/* time schemes of the 3D engine */
#define PSG_SCHEME_NS_HEUN 0   /* 3D_NavierStokes/src/kernels.h:309-464 (Heun + CN)      */
#define PSG_SCHEME_EULER_HEUN 1 /* 3D_Euler/src/kernels.h:296-439 (Heun, inviscid)      */
#define PSG_SCHEME_NS_RK4 2    /* 3D_Boussinesq/src/kernels.h:331-621 with Ri = 0, no rho */
#define PSG_SCHEME_BOUS_RK4 3  /* 3D_Boussinesq/src/kernels.h:331-621 (RK4 + CN stages)  */

const char* psg_last_error(void);
void psg_clear_error(void);
int psg_version(void);
/* building-block check: the library's line FFT on nlines contiguous lines of n
 * complex doubles (in -> out), unnormalised, sign -1 forward / +1 inverse;
 * swap selects the transposed factorisation used after another transform */
/* Runs one block whose bounded mbarrier wait cannot succeed (a transfer that
 * is never issued), `polls` polls long (1..2^20); *status is the status word
 * the kernel leaves: PSG_DEVICE_TIMEOUT when the wait ran out.  The engines'
 * waits end the same way (2^22 polls) and their sync calls report it. */
#define PSG_DEVICE_TIMEOUT 0x7e01
int psg_debug_wait_timeout(int polls, int* status);
int psg_debug_linefft(int n, int sign, int swap, const double* in, double* out, int nlines);

/* ---------------------------------------------------------------- 3D */
typedef struct psg_ns3d psg_ns3d;

/* n: grid points per direction (16..512, power of two); alpha must be 1;
 * precision: 32 (FP32 storage and transforms) or 64. */
int psg_ns3d_create(psg_ns3d** h, int n, double alpha, int scheme, int precision);
void psg_ns3d_destroy(psg_ns3d* h);
/* nu = 1/Re; ampfor/kf: forcing as the reference's d_AMPFOR/d_KFY; ri, sc,
 * theta (radians): Boussinesq parameters (ignored by the other schemes). */
/* Heun/CN forcing of the 3D Navier-Stokes scheme: PSG_FORCING_DNS adds
 * +-ampfor to Re xi at (0, kf, +-kf) (3D_NavierStokes/src/kernels.h:342-343);
 * PSG_FORCING_NEWTON adds to Im eta and Im zeta at (0, kf, +-kf) as the
 * Newton-solver build does (3D_NavierStokes/src_gmres/kernels.h:234-238) */
#define PSG_FORCING_DNS 0
#define PSG_FORCING_NEWTON 1
int psg_ns3d_set_forcing_form(psg_ns3d* h, int form);
int psg_ns3d_set_params(psg_ns3d* h, double nu, double ampfor, double kf, double ri,
                        double sc, double theta);
int psg_ns3d_set_stream(psg_ns3d* h, void* cuda_stream);
/* comps[0..2] = xii, eta, zet (+ comps[3] = rho for the Boussinesq scheme) */
int psg_ns3d_upload(psg_ns3d* h, const double* const* comps);
int psg_ns3d_download(psg_ns3d* h, double* const* comps);
/* RK4 schemes: the stage state x0 (vorticity before the divergence clean-up) */
int psg_ns3d_download_stage(psg_ns3d* h, double* const* comps);
/* The state to / from page-locked host arrays in the reference layout, kept
 * modes only: the conversion kernels read / write the host memory directly and
 * leave its other entries alone (the upload sets the engine's other modes to
 * zero).  PSG_ERR_UNSUPPORTED for pageable memory.  The drop-ins use them for
 * in-place calls on page-locked arrays whose non-kept entries are zero. */
int psg_ns3d_upload_kept(psg_ns3d* h, const double* const* comps);
int psg_ns3d_download_kept(psg_ns3d* h, double* const* comps);
/* nsteps steps of length dt, enqueued on the handle's stream.  dump_last:
 * keep the physical vorticity of the last predictor (Heun schemes) */
int psg_ns3d_step(psg_ns3d* h, double dt, int nsteps, int dump_last);
/* dz/dt at the uploaded state (RK4 schemes), written to out[0..nc-1] */
int psg_ns3d_timederiv(psg_ns3d* h, double* const* out);
/* physical fields kept by dump_last: out[0..2], n^3 doubles each, x fastest */
int psg_ns3d_download_phys(psg_ns3d* h, double* const* out);
/* Heun schemes: what dump_last keeps.  mode bit 0 clear (default): the
 * physical vorticity the last step's corrector starts from (the predicted
 * state, what the DNS returns in xir/etr/ztr, 3D_NavierStokes/src/finalise.h:
 * 9-11); set: the physical fields of the state the last step started from (what
 * the DNS's raw volumes and mean squares take, cuda.cu:68-93).  Bit 1: the
 * velocity u, v, w as well (psg_ns3d_download_phys_velocity). */
int psg_ns3d_dump_mode(psg_ns3d* h, int mode);
int psg_ns3d_download_phys_velocity(psg_ns3d* h, double* const* out);
/* running mean squares of the kept velocity on the device (FP64):
 * rms = (rms count + u^2) / (count + 1), the DNS's avgVelocity
 * (3D_NavierStokes/src/kernels.h:70-81); psg_ns3d_rms_download: out[0..2] */
int psg_ns3d_rms_accumulate(psg_ns3d* h, double count);
int psg_ns3d_rms_download(psg_ns3d* h, double* const* out);
int psg_ns3d_sync(psg_ns3d* h);
long psg_ns3d_launches(psg_ns3d* h);
/* device state pointers and padded row length (complex words) */
int psg_ns3d_layout(psg_ns3d* h, int* xp, void** comps);
/* per-pass timing: enable(1) resets and records CUDA events between the five
 * passes of every right-hand side; read returns total ms and launch counts of
 * passes A..E (z-inverse, y-inverse, x, y-forward, z-forward + update) */
int psg_ns3d_profile(psg_ns3d* h, int enable);
int psg_ns3d_profile_read(psg_ns3d* h, double* ms, long* counts);
/* re-run the set-up autotuner (x-pass rows per block, buffers per warp and, in FP32,
 * packed f32x2 transforms; timed on this device); variant receives the choice (0..15:
 * bit 0 twice the rows, bit 3 half of them, bit 1 two buffers, bit 2 packed), ms[16]
 * the timing of each variant (-1: does not fit, or not built: bits 0 and 3 together,
 * packed in FP64) */
int psg_ns3d_autotune(psg_ns3d* h, int* variant, float* ms);
/* the autotuner's current choice and timings, without re-running it
 * (PSG_XPASS_VARIANT=0..15 in the environment pins the choice at set-up) */
int psg_ns3d_tuning(psg_ns3d* h, int* variant, float* ms);
/* the autotuner's pass-A choice (FP32 engines): *packed = 1 when the z-inverse
 * transforms two fields per packed f32x2 instruction, 0 for the scalar kernel;
 * ms[2] its timings (scalar, packed; -1: not timed: FP64, or the packed
 * kernel's shared memory does not fit).  PSG_PASSA_PACKED=0/1 pins it. */
int psg_ns3d_tuning_a(psg_ns3d* h, int* packed, float* ms);
/* the state from / to device arrays: FP64 complex boxes in the reference
 * layout (IKTX*IKTY*IKTZ double2 per component), ordered on the engine's
 * stream without a host synchronisation */
int psg_ns3d_upload_device(psg_ns3d* h, void* const* comps);
int psg_ns3d_download_device(psg_ns3d* h, void* const* comps);
/* global sums over the kept modes, accumulated in FP64 on the device:
 * out[0] = sum |w|^2 / max(k^2, 0.001) (the reference's energy,
 * 3D_NavierStokes/src/functions.h:139-152), out[1] = sum |w|^2 (enstrophy),
 * out[2] = sum |rho|^2 (Boussinesq; 0 otherwise) */
int psg_ns3d_energetics(psg_ns3d* h, double* out);
/* max |u| over the grid of the physical x-velocity of the state the next step
 * starts from, reduced on the device (RK4 schemes; the Boussinesq DNS's CFL
 * input, 3D_Boussinesq/src/out_low.h:14).  One right-hand-side evaluation;
 * the state is unchanged. */
int psg_ns3d_max_velocity(psg_ns3d* h, double* umax);
/* Boussinesq scheme: FP64 sums over the kept modes of the state, as the DNS's
 * computeStats forms them (3D_Boussinesq/src/functions.h:288-362): out[0] =
 * sum Re(conj(b) rho) with b = v sin(theta) + w cos(theta) from the spectral
 * velocity (the buoyancy flux before the factor Ri), out[1] = Re zeta at
 * (kx, ky, kz) = (0, kf, 0), the forced mode (0 when it is not kept) */
int psg_ns3d_buoyancy_flux(psg_ns3d* h, double* out);

/* Tangent-linear and adjoint of the RK4/CN step (PSG_SCHEME_NS_RK4, and
 * PSG_SCHEME_BOUS_RK4 with the density as a fourth component), exact to
 * round-off for the discrete step (one RK4/CN step with the stage state
 * reset to the state, as after an upload).  in / out: 3 (4) device arrays
 * each, FP64 complex boxes in the reference layout; in == out is allowed.
 *   PSG_LIN_TANGENT_STEP   out = dPhi_dt(S) in,     then S = Phi_dt(S)
 *   PSG_LIN_ADJOINT_STEP   out = dPhi_dt(S)^T in,   then S = Phi_dt(S)
 *   PSG_LIN_TANGENT_RHS    out = N'(S) in           (S unchanged, dt unused)
 *   PSG_LIN_ADJOINT_RHS    out = N'(S)^T in
 * where N is the right-hand side without viscosity (N(w) = curl F(u x w);
 * Boussinesq: also buoyancy, -F(u.grad rho) and the stratification term) and
 * the transpose is taken in the real inner product of the stored
 * coefficients. */
#define PSG_LIN_TANGENT_STEP 0
#define PSG_LIN_ADJOINT_STEP 1
#define PSG_LIN_TANGENT_RHS 2
#define PSG_LIN_ADJOINT_RHS 3
int psg_ns3d_linear(psg_ns3d* h, int mode, double dt, void* const* in, void* const* out);

/* ---------------------------------------------------------------- 2D */
/* A batch of independent 2D Kolmogorov-flow instances (sizes 16..256, any
 * mix) integrated by one persistent launch: one thread block per instance,
 * largest first.  The scheme is the reference's 2D RK4 step with the final
 * Crank-Nicolson viscous factor and the forcing -2 at (kx,ky) = (0,+-4)
 * (2D_NavierStokes/src_RK4/kernels.h:112-435).  The single-instance drop-in
 * libpsg_ns2d.so is a batch of one. */
typedef struct psg_batch2d psg_batch2d;

int psg_batch2d_create(psg_batch2d** h, int ninst, const int* sizes, int precision);
void psg_batch2d_destroy(psg_batch2d* h);
int psg_batch2d_set_stream(psg_batch2d* h, void* cuda_stream);
/* Z: complex128 box [2K+1][K+1] of instance i (reference layout) */
int psg_batch2d_upload(psg_batch2d* h, int i, const double* Z);
int psg_batch2d_download(psg_batch2d* h, int i, double* Z);
/* enqueue nsteps[i] steps of length dt[i] with viscosity nu[i] for every
 * instance, in one kernel launch on the handle's stream */
int psg_batch2d_run(psg_batch2d* h, const double* nu, const double* dt, const int* nsteps);
/* psg_batch2d_run in two parts: set the per-instance parameters (waits for the
 * small host-to-device copy), then launch the integration as one CUDA graph
 * (reset of the work counter + the persistent kernel), which later launches
 * replay without host work; the graph is captured on first launch */
int psg_batch2d_set_params(psg_batch2d* h, const double* nu, const double* dt, const int* nsteps);
int psg_batch2d_launch(psg_batch2d* h);
/* time the persistent kernel at 128, 256 and 512 threads per block on the
 * current parameters (2-step runs, states restored afterwards) and keep the
 * fastest, then (FP32) pick each grid size's transform schedule, scalar or
 * packed, the same way; variant 0/1/2, ms[3] per run (-1: does not fit) */
int psg_batch2d_autotune(psg_batch2d* h, int* variant, float* ms);
int psg_batch2d_tuning(psg_batch2d* h, int* variant, float* ms);
/* the transform schedule psg_batch2d_autotune chose per grid size (n = 16, 32,
 * 64, 128, 256): packed[5] = 1 where the size runs its transforms two lines per
 * packed f32x2 instruction (FP32 batches), ms[10] the timing of the batch with
 * that size scalar / packed (-1: size absent, or FP64) */
int psg_batch2d_schedule(psg_batch2d* h, int* packed, float* ms);
/* pin the schedule (packed[5] as above); PSG_ERR_UNSUPPORTED for packed sizes in
 * an FP64 batch */
int psg_batch2d_set_schedule(psg_batch2d* h, const int* packed);
int psg_batch2d_sync(psg_batch2d* h);
long psg_batch2d_launches(psg_batch2d* h);
/* device pointer of instance i's state (complex of the batch precision, [2K+1][K+1]).
 * The FP32 batch keeps, right after the state, an array of the same shape with
 * the rounding error its updates carry (state value = Z + Zlow); a caller that
 * writes Z directly must zero that array too (or use psg_batch2d_upload). */
int psg_batch2d_device_state(psg_batch2d* h, int i, void** Z);

/* ------------------------------------------------------- recurrence search */
/* Near-recurrence search for UPO guesses, as the 3D DNS does it
 * (3D_NavierStokes/src/functions.h:111-389): a ring of store_size states,
 * each new one compared with the earlier ones under nshift_x * nshift_y *
 * nshift_z trial translations over the 4 W^3 modes of a low-wavenumber box
 * (W = norm_width; the reference uses 500, 8, 30, 2, 2).  States are 3 device
 * FP64 boxes (reference layout).  psg_rec3d_start takes the initial state;
 * psg_rec3d_add the state after step nt (nt = NOUT, 2 NOUT, ...); *emitted is
 * 1 when a guess left the residual threshold, whose data psg_rec3d_guess then
 * returns: meta[7] = start time, v2, period, shift x, y, z, residual, and the
 * state (host arrays, each may be null). */
typedef struct psg_rec3d psg_rec3d;
int psg_rec3d_create(psg_rec3d** h, int n, double alpha, int store_size, int norm_width,
                     int nshift_x, int nshift_y, int nshift_z, double threshold, int nout,
                     double dt, double tstart, double v2);
/* The Boussinesq DNS's variant (3D_Boussinesq/src/functions.h:189-205,
 * 416-616): states of four fields (xii, eta, zet, rho), the density terms
 * weighted by ri, residuals normalised by the sum of both states' norms,
 * periods below 0.5 skipped; psg_rec3d_guess_rho returns the guess's density. */
int psg_rec3d_create_bous(psg_rec3d** h, int n, double alpha, int store_size, int norm_width,
                          int nshift_x, int nshift_y, int nshift_z, double threshold, int nout,
                          double dt, double tstart, double v2, double ri);
int psg_rec3d_guess_rho(psg_rec3d* h, double* rho);
void psg_rec3d_destroy(psg_rec3d* h);
int psg_rec3d_set_stream(psg_rec3d* h, void* cuda_stream);
int psg_rec3d_start(psg_rec3d* h, void* const* state);
int psg_rec3d_add(psg_rec3d* h, int nt, void* const* state, int* emitted);
int psg_rec3d_guess(psg_rec3d* h, double* meta, double* xii, double* eta, double* zet);
/* the same, with the state taken from a 3D engine (its current state) */
int psg_rec3d_start_engine(psg_rec3d* h, psg_ns3d* engine);
int psg_rec3d_add_engine(psg_rec3d* h, int nt, psg_ns3d* engine, int* emitted);
int psg_rec3d_count(psg_rec3d* h);
long psg_rec3d_launches(psg_rec3d* h);

/* Near-recurrence search for UPO guesses of 2D runs, batched over nrun runs of
 * one grid (2D_NavierStokes/src_RK4/functions.h:105-309): per run a ring of
 * store_size states; every output interval each run's newest state is
 * compared with its earlier ones under nshift_x * nshift_y trial
 * translations (2 pi i / (nshift_x alpha), 2 pi j / nshift_y) over the 2 W^2
 * modes of the box 0 <= kx < W, -W <= ky < W (W = norm_width), and the
 * reference's selection logic emits a guess when a run's minimum residual
 * enters and then leaves the threshold.  psg_rec2d_start takes the initial
 * states, psg_rec2d_add the states after step nt (nt = NOUT, 2 NOUT, ...):
 * states[r] is run r's device box (complex of `precision`, [2K+1][K+1], e.g.
 * psg_batch2d_device_state); *emitted counts the guesses this call added.
 * psg_rec2d_guess returns guess k: meta[7] = run, start time, v2, period,
 * shift x, shift y, residual, and its state (complex128 box, may be null). */
typedef struct psg_rec2d psg_rec2d;
int psg_rec2d_create(psg_rec2d** h, int nrun, int n, double alpha, int store_size,
                     int norm_width, int nshift_x, int nshift_y, double threshold, int nout,
                     double dt, double tstart, const double* v2);
void psg_rec2d_destroy(psg_rec2d* h);
int psg_rec2d_set_stream(psg_rec2d* h, void* cuda_stream);
int psg_rec2d_start(psg_rec2d* h, void* const* states, int precision);
int psg_rec2d_add(psg_rec2d* h, int nt, void* const* states, int precision, int* emitted);
int psg_rec2d_count(psg_rec2d* h);
int psg_rec2d_guess(psg_rec2d* h, int k, double* meta, double* Z);
long psg_rec2d_launches(psg_rec2d* h);

/* ---------------------------------------------------------------- UPO search */
/* Batched Newton-GMRES-hookstep search for unstable periodic orbits of 2D
 * Kolmogorov flow (2D_NavierStokes/src_RK4/src_gmres/main.F90:688-1823), all
 * guesses in lock step, on the GPU.  jv_mode 0: exact tangent
 * Jacobian-vector products of the discrete step in FP64; 1: the reference's
 * forward difference (eps = 1e-7) of FP64 integrations; 2: the exact tangent
 * with base and tangent integrated in FP32 (Krylov products only: Phi_T, the
 * residual, dz/dt, Arnoldi and the hookstep stay FP64).  kmax: Krylov
 * dimension (GMRESMAX). */
typedef struct psg_upo2d psg_upo2d;

#define PSG_UPO_ACTIVE 0
#define PSG_UPO_CONVERGED 1
#define PSG_UPO_GMRES_FAILED 2
#define PSG_UPO_HOOK_FAILED 3
#define PSG_UPO_STALLED 4
#define PSG_UPO_TSTEP_FAILED 5
#define PSG_UPO_PERIOD_TOO_SMALL 6
#define PSG_UPO_NEWTON_FAILED 7

int psg_upo2d_create(psg_upo2d** h, int nguess, int n, int kmax, int jv_mode);
void psg_upo2d_destroy(psg_upo2d* h);
/* guess i: state Z (complex128 box [2K+1][K+1]), period T, shifts (sx, sy),
 * shift-reflect flag (RsymFLAG), viscosity nu = 1/Re, time step dt (TRUEDELT) */
int psg_upo2d_set_guess(psg_upo2d* h, int i, const double* Z, double T, double sx, double sy,
                        int rsym, double nu, double dt);
/* Newton iterations until |F|/|Phi_T(z)| <= tol (NETOL) for every guess or
 * max_newton; gmres_tol: GMTOL */
int psg_upo2d_solve(psg_upo2d* h, int max_newton, double tol, double gmres_tol);
/* vals[4] = {T, sx, sy, residual}; info[4] = {status, newton, gmres, hookstep} */
int psg_upo2d_get(psg_upo2d* h, int i, double* Z, double* vals, int* info);
/* building blocks at guess i (unshifted): mode 1 Phi_T(z) -> Zout; mode 0 also
 * the tangent dPhi_T(z) q (q in/out); mode 2 dz/dt -> Zout */
int psg_upo2d_apply(psg_upo2d* h, int i, int mode, double* Zout, double* q);
/* per-Newton-step record k of guess i, rec[11] = {Newton index, GMRES
 * iterations of the step, hookstep trials, Delta after the step, mu of the
 * last trial, T, shift x, residual |F|/|Phi_T(z)|, |F|, time step, nu}; the
 * quantities the reference prints per step (src_gmres/main.F90:1225-1760) */
int psg_upo2d_trace(psg_upo2d* h, int i, int k, double* rec);
/* Arc-length continuation of guess i in the viscosity (src_gmres/main.F90:
 * 408-640, 799-1823 with arclcFLAG): nu becomes an unknown with the
 * pseudo-arclength row <dZ/dr, z - Zr2> + dT/dr (T - Tr2) + dS/dr (s - Sr2)
 * + dnu/dr (nu - nu_r2) = ndelta; dZrdr and Zr2 are complex128 boxes.  Call
 * after psg_upo2d_set_guess (the predicted z, T, s, nu), which clears it;
 * psg_upo2d_get_nu returns the current nu of a guess. */
int psg_upo2d_set_arc(psg_upo2d* h, int i, const double* dZrdr, const double* Zr2, double dTrdr,
                      double dSrdr, double dv2rdr, double Tr2, double Sr2, double v2r2,
                      double ndelta);
int psg_upo2d_get_nu(psg_upo2d* h, int i, double* nu);
int psg_upo2d_trace_count(psg_upo2d* h, int i);
long psg_upo2d_integrations(psg_upo2d* h);
long psg_upo2d_launches(psg_upo2d* h);
/* Phase timing of psg_upo2d_solve.  psg_upo2d_profile(h, 1) clears the counters
 * and synchronises the stream around every batched integration from then on
 * (0 turns it off); psg_upo2d_profile_read fills out[6] = {seconds in solve,
 * exact-Jv integrations in FP64, exact-Jv integrations in FP32, Phi_T
 * integrations (residuals, hookstep trials, forward differences), dz/dt, host
 * SVDs of the Hessenberg matrices}. */
int psg_upo2d_profile(psg_upo2d* h, int enable);
int psg_upo2d_profile_read(psg_upo2d* h, double* out);

/* Allocation-free 2D step.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory when they step: a plugin
 * inside a host runtime that owns all GPU memory, code running while a CUDA
 * graph is being captured, or an embedded driver with a fixed memory budget.
 * It integrates nsteps RK4/CN steps of one 2D instance (the same kernel body
 * as psg_batch2d_run) with all scratch -- stage registers, row buffers and
 * twiddles -- in a 512 KiB array compiled into the library, which every GPU
 * that loads the library holds until the process exits.  Limits: n in
 * {16, 32, 64, 128}; larger grids are rejected with PSG_ERR_UNSUPPORTED.
 *
 * z_in, z_out: device pointers owned by the caller to the complex state in the
 * reference layout [2K+1][K+1] (float2 for precision 32, double2 for 64);
 * z_in == z_out is allowed.  The work is enqueued on `stream` (NULL: the
 * default stream).  The first call on a device looks up the array's address
 * and writes the twiddle tables (a synchronous copy), so make that first call
 * before any stream capture: a first call on a capturing stream is refused
 * with PSG_ERR_UNSUPPORTED.  The set-up is remembered for the life of the
 * process; calls after cudaDeviceReset are not supported.  Every call uses the
 * same array and leaves its last contents there (no call relies on them: each
 * scratch word is written, or cleared on the call's stream, before it is
 * read), so calls that overlap on the GPU -- e.g. on two streams at once --
 * race; serialise them on one stream.
 *
 * Precision 32 carries the rounding error of each state update in the array,
 * as psg_batch2d_run's FP32 engine does, starting from zero at every call (the
 * state is exactly the caller's FP32 input); the carried remainder is dropped
 * when the call returns, so a long FP32 run split over many calls rounds once
 * per call more than one long call. */
int psg_ns2d_step_noalloc(int n, int precision, double nu, double dt, int nsteps,
                          const void* z_in, void* z_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
