"""In-tree build of the CUDA layer for sm_100a.

    python -m psgpu_b200.build          # or psgpu_b200.build.build()

Produces (git-ignored, shipped with the tree):
  psgpu_b200/lib/libpsgpu.so          engines + re-entrant C API (include/psgpu.h)
  psgpu_b200/lib/libpsg_<flavour>.so  reference-compatible timestep_cuda_ drop-ins
                                      (include/psgpu_ref_abi.h), linked to libpsgpu.so
  psgpu_b200/bin/psg_dns3             3D Navier-Stokes DNS driver (include/psgpu_host.h)
Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BIN = os.path.join(HERE, "bin")
CC = os.environ.get("CC", "gcc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--ptxas-options=-O3", f"-I{INCLUDE}", f"-I{CSRC}"]

# translation units of libpsgpu.so
CORE = ["psg_api.cu", "psg_ns3d_api.cu", "psg_ns3d_f32.cu", "psg_ns3d_f64.cu",
        "psg_ns2d.cu", "psg_newton2d.cu", "psg_tan2d_f64.cu", "psg_tan2d_f32.cu",
        "psg_recurrence.cu", "psg_recurrence2d.cu"]
# host-side C of libpsgpu.so (parameter files, random starts, record I/O)
HOST_SRC = ["psg_host.c"]
# driver programs: name -> source (linked to libpsgpu.so)
DRIVERS = {"psg_dns3": "psg_dns3.c"}
# drop-in libraries: name -> (source, macro)
DROPINS = {
    "ns3d": ("psg_dropin3d.cu", "PSG_FLAVOUR_NS3D"),
    "ns3d_newton": ("psg_dropin3d.cu", "PSG_FLAVOUR_NS3D_NEWTON"),
    "euler3d": ("psg_dropin3d.cu", "PSG_FLAVOUR_EULER3D"),
    "bous3d": ("psg_dropin3d.cu", "PSG_FLAVOUR_BOUS3D"),
    "bous3d_dns": ("psg_dropin3d.cu", "PSG_FLAVOUR_BOUS3D_DNS"),
    "ns2d": ("psg_dropin2d.cu", "PSG_FLAVOUR_NS2D"),
}


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs += glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "host", "*.h"))
    hs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources) or _headers() > t


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def _compile(src, obj, defines=()):
    srcp = os.path.join(CSRC, src)
    if not _stale(obj, [srcp]):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *[f"-D{d}" for d in defines], "-c", srcp, "-o", obj]
    _run(cmd)
    return obj


def _compile_c(src, obj):
    srcp = os.path.join(HOST, src)
    if not _stale(obj, [srcp]):
        return obj
    _run([CC, "-std=c11", "-O2", "-fPIC", "-Wall", "-D_POSIX_C_SOURCE=200809L", f"-I{INCLUDE}",
          "-c", srcp, "-o", obj])
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    jobs = []
    core = [s for s in CORE if os.path.exists(os.path.join(CSRC, s))]
    dropins = {k: v for k, v in DROPINS.items() if os.path.exists(os.path.join(CSRC, v[0]))}
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for s in core:
            jobs.append(ex.submit(_compile, s, os.path.join(OBJ, s.replace(".cu", ".o"))))
        for name, (s, macro) in dropins.items():
            jobs.append(ex.submit(_compile, s, os.path.join(OBJ, f"dropin_{name}.o"), (macro,)))
        for s in HOST_SRC:
            jobs.append(ex.submit(_compile_c, s, os.path.join(OBJ, s.replace(".c", ".o"))))
        for j in jobs:
            j.result()
    core_objs = [os.path.join(OBJ, s.replace(".cu", ".o")) for s in core]
    core_objs += [os.path.join(OBJ, s.replace(".c", ".o")) for s in HOST_SRC]
    libcore = os.path.join(LIB, "libpsgpu.so")
    if _stale(libcore, core_objs):
        _run([NVCC, *ARCH, "-shared", "-o", libcore, *core_objs, "-lcudart"])
    for name in dropins:
        obj = os.path.join(OBJ, f"dropin_{name}.o")
        out = os.path.join(LIB, f"libpsg_{name}.so")
        if _stale(out, [obj, libcore]):
            _run([NVCC, *ARCH, "-shared", "-o", out, obj, f"-L{LIB}", "-lpsgpu", "-lcudart",
                  "-Xlinker", "-rpath,$ORIGIN"])
    for name, src in DRIVERS.items():
        srcp = os.path.join(HOST, src)
        out = os.path.join(BIN, name)
        if _stale(out, [srcp, libcore]):
            _run([CC, "-std=c11", "-O2", "-Wall", "-D_POSIX_C_SOURCE=200809L", f"-I{INCLUDE}", srcp,
                  "-o", out, f"-L{LIB}", "-lpsgpu", "-Wl,-rpath,$ORIGIN/../lib", "-lm"])
    if verbose:
        print("built", libcore)
    return libcore


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
