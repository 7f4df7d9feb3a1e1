// psg_ns3d.cuh -- the 3D pseudospectral right-hand side as five fused passes.
//
// State layout in HBM (per component, complex T): the reference's truncated
// box (kx fastest, 3D_NavierStokes/src/init.F90:25-36) cut into tiles of W = 8
// adjacent kx columns, S[xt][iky][ikz][W], ikz, iky in [0, 2K], xt in
// [0, XP / W) with XP = IKTX rounded up to W (padding columns hold zeros), so
// that the z-line tile of one (xt, iky) is one contiguous chunk.
//
// One evaluation of N(w) = curl(u x w) (plus buoyancy / density advection for
// the Boussinesq system) is
//   A  z-inverse  : stage state -> {w, u = i k x w / k^2 (, i k rho)}   [f][z][ky][kx]
//   B  y-inverse  :                                                      [f][z][y][kx]
//   C  x-pass     : C2R -> -(u x w) (, u.grad rho) -> R2C, scaled 1/N^3   [g][z][y][kx]
//   D  y-forward  :                                                      [g][z][ky][kx]
//   E  z-forward  : + curl, forcing, buoyancy and the time-scheme update  -> state
// Passes A, B, D and E transform tiles of W adjacent kx columns along a
// strided axis; pass C transforms whole x rows, one row per thread group.
// Truncated modes are never loaded in the inverse direction and never
// produced in the forward direction.
#pragma once
#include "psg_common.cuh"
#include "psg_fft.cuh"

namespace psg {

enum Scheme3D : int {
  SCHEME_NS_HEUN = 0,     // 3D_NavierStokes/src/kernels.h:309-464
  SCHEME_EULER_HEUN = 1,  // 3D_Euler/src/kernels.h:296-439
  SCHEME_NS_RK4 = 2,      // 3D_Boussinesq/src/kernels.h:331-621 without density
  SCHEME_BOUS_RK4 = 3,    // 3D_Boussinesq/src/kernels.h:331-621
  SCHEME_RAW = 4,         // pass E writes the masked transform itself (bilinear products)
};

// stage codes of pass E
enum StageCode : int {
  STAGE_HEUN_PRED = 0,
  STAGE_HEUN_CORR = 1,
  STAGE_RK1 = 2,
  STAGE_RK2 = 3,
  STAGE_RK3 = 4,
  STAGE_RK4 = 5,
  STAGE_DERIV = 6,  // dz/dt into K1 (3D_Boussinesq/src/kernels.h:624-692)
};

template <typename T>
struct Geom3 {
  int n, K, X, Y, XP;
  T alpha;
};

template <typename T>
struct StepParams {
  T dt;      // step length
  T nu;      // viscosity (1/Re)
  T ampfor;  // forcing amplitude (the reference's d_AMPFOR)
  T kf;      // forcing wavenumber
  int fform; // Heun/CN forcing: 0 as the DNS build applies it, 1 as the Newton-solver build
  T ri, sc, sinth, costh;  // Boussinesq parameters
};

template <typename T>
struct Fields4 {
  cpx<T>* c[4];
};

// precision-independent interface of the 3D engine (psg_ns3d_impl.cuh)
struct Engine3DBase {
  virtual ~Engine3DBase() {}
  virtual int init(int n, double alpha, int scheme) = 0;
  virtual int set_params(double nu, double ampfor, double kf, double ri, double sc, double theta) = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  virtual cudaStream_t get_stream() const = 0;
  virtual int upload(const double* const* comps) = 0;
  virtual int download(double* const* comps) = 0;
  virtual int download_stage(double* const* comps) = 0;
  virtual int upload_device(const void* const* comps) = 0;
  virtual int download_device(void* const* comps) = 0;
  virtual int upload_kept(const double* const* comps) = 0;
  virtual int download_kept(double* const* comps) = 0;
  virtual int energetics(double* out) = 0;
  virtual int max_velocity(double* out) = 0;
  virtual int buoyancy_flux(double* out) = 0;
  virtual int set_forcing_form(int form) = 0;
  virtual int linear(int mode, double dt, const void* const* in, void* const* out) = 0;
  virtual int steps(double dt, int nsteps, int dump_last) = 0;
  virtual int timederiv(double* const* out) = 0;
  virtual int phys(double* const* out) = 0;
  virtual int set_dump_mode(int mode) = 0;
  virtual int phys_velocity(double* const* out) = 0;
  virtual int rms_accumulate(double count) = 0;
  virtual int rms_download(double* const* out) = 0;
  virtual int layout(int* xp, void** comps) = 0;
  virtual long launch_count() const = 0;
  virtual int sync() = 0;  // wait for the stream and check the device error flag
  // x-pass autotuner: run at set-up; report the chosen variant and timings
  virtual int autotune() = 0;
  virtual int tuning(int* variant, float* ms) = 0;
  virtual int tuning_a(int* packed, float* ms) = 0;
  // per-pass timing (A, B, C, D, E) with CUDA events between the launches
  virtual int profile(int enable) = 0;
  virtual int profile_read(double* ms, long* counts) = 0;
};

Engine3DBase* make_engine3d_f32();
Engine3DBase* make_engine3d_f64();

}  // namespace psg
