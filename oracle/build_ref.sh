#!/usr/bin/env bash
# Compiles the reference's own CUDA time steps, unmodified, from the read-only
# reference tree into oracle/_ref/ (git-ignored; the .so files travel to the GPU
# box).  Test infrastructure only: these libraries are the "plain form" the
# product is checked and timed against.  Nothing here copies reference sources.
#
#   REF=/path/to/psgpu ./oracle/build_ref.sh
#
# One shared object per flavour, because every flavour exports the same
# Fortran-mangled symbol timestep_cuda_.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${REF:-/root/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
ARCH="${ARCH:--gencode arch=compute_100a,code=sm_100a}"
if [ ! -d "$REF" ]; then
  echo "reference tree $REF not found; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
build() {  # name source-dir cuda.cu [extra flags]
  local name="$1" dir="$2" src="$3" extra="${4:-}"
  local tgt="$OUT/libref_${name}.so"
  if [ -f "$tgt" ] && [ "$tgt" -nt "$REF/$src" ]; then return 0; fi
  # The reference's makefiles use -O3 --use_fast_math (3D_NavierStokes/src/makefile:5).
  "$NVCC" -O3 --use_fast_math $ARCH -Xcompiler -fPIC -shared -w \
      $extra -I"$REF/$dir" -I"$HERE/ref_shim" -o "$tgt" "$REF/$src" -lcufft
  echo "built $tgt"
}
build ns2d     2D_NavierStokes/src_RK4           2D_NavierStokes/src_RK4/src_gmres/cuda.cu &
build ns3d     3D_NavierStokes/src               3D_NavierStokes/src/cuda.cu &
build euler3d  3D_Euler/src                      3D_Euler/src/cuda.cu &
build bous3d   3D_Boussinesq/src                 3D_Boussinesq/src/src_gmres/cuda.cu &
# the Boussinesq DNS build: adaptive time step and forcing throttle; writes its
# diagnostics under JOB<rank>/ of the working directory
build bous3d_dns 3D_Boussinesq/src               3D_Boussinesq/src/cuda.cu &
# the 3D NS Newton-solver step (18 arguments, grid fixed at 128^3 by its kernels.h)
build ns3d_gmres 3D_NavierStokes/src_gmres       3D_NavierStokes/src_gmres/cuda.cu &
# The 3D NS DNS build formats "JOB0/xii001.raw" (16 bytes) into a 14-byte
# buffer at NT=0 whenever NSTOP > 1 (3D_NavierStokes/src/init.h:106 vs
# cuda.cu:74).  glibc's fortified sprintf aborts there, and a build with the
# check turned off crashed on the host at N=256; callers therefore drive this
# build one step per call (NSTOP = 1), which skips the volume dump.
wait
