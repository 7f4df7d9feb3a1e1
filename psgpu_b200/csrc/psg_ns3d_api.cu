// psg_ns3d_api.cu -- C API of the 3D engine (include/psgpu.h).
#include "psg_ns3d.cuh"
#include "psgpu_internal.h"

using namespace psg;

struct psg_ns3d {
  Engine3DBase* e = nullptr;
};

#define PSG_CHECK_HANDLE(h)                                 \
  do {                                                      \
    if (!(h) || !(h)->e) {                                  \
      psg_set_error("null or destroyed psg_ns3d handle");   \
      return PSG_ERR_ARG;                                   \
    }                                                       \
  } while (0)

extern "C" int psg_ns3d_create(psg_ns3d** out, int n, double alpha, int scheme, int precision) {
  if (!out) { psg_set_error("null output handle"); return PSG_ERR_ARG; }
  *out = nullptr;
  if (scheme < 0 || scheme > 3) { psg_set_error("unknown scheme %d", scheme); return PSG_ERR_ARG; }
  if (precision != 32 && precision != 64) { psg_set_error("precision must be 32 or 64"); return PSG_ERR_ARG; }
  if (alpha != 1.0) {
    psg_set_error("aspect ratio alpha=%g unsupported: the box must be cubic", alpha);
    return PSG_ERR_UNSUPPORTED;
  }
  psg_ns3d* h = new psg_ns3d();
  h->e = (precision == 64) ? make_engine3d_f64() : make_engine3d_f32();
  int rc = h->e->init(n, alpha, scheme);
  if (rc) { delete h->e; delete h; return rc; }
  *out = h;
  return PSG_OK;
}

extern "C" void psg_ns3d_destroy(psg_ns3d* h) {
  if (!h) return;
  delete h->e;
  delete h;
}

extern "C" int psg_ns3d_set_params(psg_ns3d* h, double nu, double ampfor, double kf, double ri,
                                   double sc, double theta) {
  PSG_CHECK_HANDLE(h);
  return h->e->set_params(nu, ampfor, kf, ri, sc, theta);
}

extern "C" int psg_ns3d_set_stream(psg_ns3d* h, void* stream) {
  PSG_CHECK_HANDLE(h);
  h->e->set_stream((cudaStream_t)stream);
  return PSG_OK;
}

extern "C" int psg_ns3d_upload(psg_ns3d* h, const double* const* comps) {
  PSG_CHECK_HANDLE(h);
  if (!comps) { psg_set_error("null state"); return PSG_ERR_ARG; }
  return h->e->upload(comps);
}

extern "C" int psg_ns3d_download(psg_ns3d* h, double* const* comps) {
  PSG_CHECK_HANDLE(h);
  if (!comps) { psg_set_error("null state"); return PSG_ERR_ARG; }
  return h->e->download(comps);
}

extern "C" int psg_ns3d_download_stage(psg_ns3d* h, double* const* comps) {
  PSG_CHECK_HANDLE(h);
  if (!comps) { psg_set_error("null state"); return PSG_ERR_ARG; }
  return h->e->download_stage(comps);
}

extern "C" int psg_ns3d_step(psg_ns3d* h, double dt, int nsteps, int dump_last) {
  PSG_CHECK_HANDLE(h);
  if (nsteps < 0) { psg_set_error("negative step count"); return PSG_ERR_ARG; }
  return h->e->steps(dt, nsteps, dump_last);
}

extern "C" int psg_ns3d_timederiv(psg_ns3d* h, double* const* out) {
  PSG_CHECK_HANDLE(h);
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->timederiv(out);
}

extern "C" int psg_ns3d_download_phys(psg_ns3d* h, double* const* out) {
  PSG_CHECK_HANDLE(h);
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->phys(out);
}

extern "C" int psg_ns3d_dump_mode(psg_ns3d* h, int mode) {
  PSG_CHECK_HANDLE(h);
  return h->e->set_dump_mode(mode);
}

extern "C" int psg_ns3d_download_phys_velocity(psg_ns3d* h, double* const* out) {
  PSG_CHECK_HANDLE(h);
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->phys_velocity(out);
}

extern "C" int psg_ns3d_rms_accumulate(psg_ns3d* h, double count) {
  PSG_CHECK_HANDLE(h);
  if (count < 0) { psg_set_error("count must be >= 0"); return PSG_ERR_ARG; }
  return h->e->rms_accumulate(count);
}

extern "C" int psg_ns3d_rms_download(psg_ns3d* h, double* const* out) {
  PSG_CHECK_HANDLE(h);
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->rms_download(out);
}

extern "C" int psg_ns3d_sync(psg_ns3d* h) {
  PSG_CHECK_HANDLE(h);
  return h->e->sync();
}

extern "C" long psg_ns3d_launches(psg_ns3d* h) {
  if (!h || !h->e) return -1;
  return h->e->launch_count();
}

extern "C" int psg_ns3d_layout(psg_ns3d* h, int* xp, void** comps) {
  PSG_CHECK_HANDLE(h);
  return h->e->layout(xp, comps);
}

extern "C" int psg_ns3d_profile(psg_ns3d* h, int enable) {
  PSG_CHECK_HANDLE(h);
  return h->e->profile(enable);
}

extern "C" int psg_ns3d_profile_read(psg_ns3d* h, double* ms, long* counts) {
  PSG_CHECK_HANDLE(h);
  if (!ms || !counts) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->profile_read(ms, counts);
}

extern "C" int psg_ns3d_autotune(psg_ns3d* h, int* variant, float* ms) {
  PSG_CHECK_HANDLE(h);
  int rc = h->e->autotune();
  if (rc) return rc;
  return h->e->tuning(variant, ms);
}

extern "C" int psg_ns3d_tuning(psg_ns3d* h, int* variant, float* ms) {
  PSG_CHECK_HANDLE(h);
  return h->e->tuning(variant, ms);
}

extern "C" int psg_ns3d_tuning_a(psg_ns3d* h, int* packed, float* ms) {
  PSG_CHECK_HANDLE(h);
  return h->e->tuning_a(packed, ms);
}

extern "C" int psg_ns3d_upload_kept(psg_ns3d* h, const double* const* comps) {
  PSG_CHECK_HANDLE(h);
  if (!comps) { psg_set_error("null state"); return PSG_ERR_ARG; }
  return h->e->upload_kept(comps);
}

extern "C" int psg_ns3d_download_kept(psg_ns3d* h, double* const* comps) {
  PSG_CHECK_HANDLE(h);
  if (!comps) { psg_set_error("null state"); return PSG_ERR_ARG; }
  return h->e->download_kept(comps);
}

extern "C" int psg_ns3d_upload_device(psg_ns3d* h, void* const* comps) {
  PSG_CHECK_HANDLE(h);
  return h->e->upload_device((const void* const*)comps);
}

extern "C" int psg_ns3d_download_device(psg_ns3d* h, void* const* comps) {
  PSG_CHECK_HANDLE(h);
  return h->e->download_device(comps);
}

extern "C" int psg_ns3d_energetics(psg_ns3d* h, double* out) {
  PSG_CHECK_HANDLE(h);
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->energetics(out);
}

extern "C" int psg_ns3d_max_velocity(psg_ns3d* h, double* umax) {
  PSG_CHECK_HANDLE(h);
  if (!umax) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->max_velocity(umax);
}

extern "C" int psg_ns3d_buoyancy_flux(psg_ns3d* h, double* out) {
  PSG_CHECK_HANDLE(h);
  if (!out) { psg_set_error("null output"); return PSG_ERR_ARG; }
  return h->e->buoyancy_flux(out);
}

extern "C" int psg_ns3d_linear(psg_ns3d* h, int mode, double dt, void* const* in, void* const* out) {
  PSG_CHECK_HANDLE(h);
  if (!in || !out) { psg_set_error("null vector"); return PSG_ERR_ARG; }
  return h->e->linear(mode, dt, (const void* const*)in, out);
}

extern "C" int psg_ns3d_set_forcing_form(psg_ns3d* h, int form) {
  PSG_CHECK_HANDLE(h);
  return h->e->set_forcing_form(form);
}
