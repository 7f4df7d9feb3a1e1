// psgpu_internal.h -- host-side declarations shared by the CUDA translation units.
#pragma once
#include "../../include/psgpu.h"

#ifdef __cplusplus
extern "C" {
#endif
void psg_set_error(const char* fmt, ...);
#ifdef __cplusplus
}
#endif
