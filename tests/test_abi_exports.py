"""The C-ABI libraries load without a GPU and export every symbol that
include/*.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "psgpu_b200", "lib")


def _declared(header, guard=None):
    src = open(os.path.join(ROOT, "include", header)).read()
    if guard:
        blocks = re.findall(r"#if defined\((\w+)\)[^\n]*\n(.*?)#endif", src, re.S)
        src = "\n".join(b for g, b in blocks if g == guard)
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(psg_\w+|timestep_cuda_|timederiv_cuda_|set_gpu_)\s*\(", src)))


def _load(name):
    path = os.path.join(LIB, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built")
    return ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)


def test_core_exports_every_declared_symbol():
    L = _load("libpsgpu.so")
    names = _declared("psgpu.h")
    assert len(names) > 20
    for s in names:
        assert hasattr(L, s), s


@pytest.mark.parametrize("flavour,guard", [("ns2d", "PSG_ABI_NS2D"), ("ns3d", "PSG_ABI_NS3D"),
                                           ("ns3d_newton", "PSG_ABI_NS3D_NEWTON"),
                                           ("euler3d", "PSG_ABI_EULER3D"),
                                           ("bous3d", "PSG_ABI_BOUS3D"),
                                           ("bous3d_dns", "PSG_ABI_BOUS3D_DNS")])
def test_dropin_exports(flavour, guard):
    _load("libpsgpu.so")
    L = _load(f"libpsg_{flavour}.so")
    names = _declared("psgpu_ref_abi.h", guard) + ["set_gpu_"]
    assert "timestep_cuda_" in names
    for s in names:
        assert hasattr(L, s), s


def test_error_channel_without_gpu():
    L = _load("libpsgpu.so")
    L.psg_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p()
    # an unsupported grid size fails on argument checks before any device call
    rc = L.psg_ns3d_create(ctypes.byref(h), ctypes.c_int(48), ctypes.c_double(1.0),
                           ctypes.c_int(2), ctypes.c_int(32))
    assert rc != 0
    assert b"unsupported" in L.psg_last_error()
