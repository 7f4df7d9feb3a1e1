// psg_tan2d_f32.cu -- the FP32 instantiations of the 2D base + tangent
// integrator kernels of the UPO search (psg_tan2d_run.cuh).
#include "psg_tan2d_run.cuh"

namespace psg {
PSG_TAN2D_INSTANTIATE(float)
}  // namespace psg
