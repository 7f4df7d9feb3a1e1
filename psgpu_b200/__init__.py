"""psgpu_b200 -- B200-native pseudospectral time step for periodic-box flows.

Python host side of the CUDA layer (``psgpu_b200/lib/libpsgpu.so``).  The
library is required: there is no CPU fallback, and every entry point raises
if the shared object is missing or a CUDA call fails.

The reference-compatible ``timestep_cuda_`` entry points live in the drop-in
libraries ``lib/libpsg_<flavour>.so`` and are driven through
:class:`psgpu_b200.abi.TimestepLibrary`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .fields import Grid2D, Grid3D  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")
CORE = os.path.join(LIBDIR, "libpsgpu.so")

SCHEME_NS_HEUN = 0
SCHEME_EULER_HEUN = 1
SCHEME_NS_RK4 = 2
SCHEME_BOUS_RK4 = 3

_lib = None


class PsgError(RuntimeError):
    pass


def dropin_path(flavour: str) -> str:
    p = os.path.join(LIBDIR, f"libpsg_{flavour}.so")
    if not os.path.exists(p):
        raise PsgError(f"drop-in library {p} is not built (run python -m psgpu_b200.build)")
    return p


def lib():
    """Load libpsgpu.so (raises PsgError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(CORE):
        raise PsgError(f"{CORE} is not built; run `python -m psgpu_b200.build`")
    L = C.CDLL(CORE, mode=C.RTLD_GLOBAL)
    vp, ip, d, i = C.c_void_p, C.c_int, C.c_double, C.c_int
    pp = C.POINTER(C.c_void_p)
    L.psg_last_error.restype = C.c_char_p
    L.psg_version.restype = i
    L.psg_debug_linefft.argtypes = [i, i, i, C.POINTER(C.c_double), C.POINTER(C.c_double), i]
    L.psg_ns3d_create.argtypes = [C.POINTER(vp), i, d, i, i]
    L.psg_ns3d_destroy.argtypes = [vp]
    L.psg_ns3d_destroy.restype = None
    L.psg_ns3d_set_params.argtypes = [vp, d, d, d, d, d, d]
    L.psg_ns3d_set_stream.argtypes = [vp, vp]
    L.psg_ns3d_upload.argtypes = [vp, pp]
    L.psg_ns3d_download.argtypes = [vp, pp]
    L.psg_ns3d_download_stage.argtypes = [vp, pp]
    L.psg_ns3d_step.argtypes = [vp, d, i, i]
    L.psg_ns3d_timederiv.argtypes = [vp, pp]
    L.psg_ns3d_download_phys.argtypes = [vp, pp]
    L.psg_ns3d_dump_mode.argtypes = [vp, i]
    L.psg_ns3d_download_phys_velocity.argtypes = [vp, pp]
    L.psg_ns3d_rms_accumulate.argtypes = [vp, C.c_double]
    L.psg_ns3d_rms_download.argtypes = [vp, pp]
    L.psg_ns3d_sync.argtypes = [vp]
    L.psg_ns3d_launches.argtypes = [vp]
    L.psg_ns3d_launches.restype = C.c_long
    L.psg_ns3d_layout.argtypes = [vp, C.POINTER(ip), pp]
    L.psg_ns3d_profile.argtypes = [vp, i]
    L.psg_ns3d_autotune.argtypes = [vp, C.POINTER(i), C.POINTER(C.c_float)]
    L.psg_ns3d_tuning.argtypes = [vp, C.POINTER(i), C.POINTER(C.c_float)]
    L.psg_ns3d_profile_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_long)]
    L.psg_ns3d_upload_device.argtypes = [vp, C.POINTER(vp)]
    L.psg_ns3d_download_device.argtypes = [vp, C.POINTER(vp)]
    L.psg_ns3d_energetics.argtypes = [vp, C.POINTER(C.c_double)]
    L.psg_ns3d_linear.argtypes = [vp, i, d, C.POINTER(vp), C.POINTER(vp)]
    _declare_2d(L)
    _lib = L
    return L


def _declare_2d(L):
    vp, i = C.c_void_p, C.c_int
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    L.psg_batch2d_create.argtypes = [C.POINTER(vp), i, ip, i]
    L.psg_batch2d_destroy.argtypes = [vp]
    L.psg_batch2d_destroy.restype = None
    L.psg_batch2d_set_stream.argtypes = [vp, vp]
    L.psg_batch2d_upload.argtypes = [vp, i, dp]
    L.psg_batch2d_download.argtypes = [vp, i, dp]
    L.psg_batch2d_run.argtypes = [vp, dp, dp, ip]
    L.psg_batch2d_set_params.argtypes = [vp, dp, dp, ip]
    L.psg_batch2d_launch.argtypes = [vp]
    L.psg_batch2d_autotune.argtypes = [vp, ip, C.POINTER(C.c_float)]
    L.psg_batch2d_tuning.argtypes = [vp, ip, C.POINTER(C.c_float)]
    L.psg_batch2d_schedule.argtypes = [vp, ip, C.POINTER(C.c_float)]
    L.psg_batch2d_set_schedule.argtypes = [vp, ip]
    L.psg_batch2d_sync.argtypes = [vp]
    L.psg_batch2d_launches.argtypes = [vp]
    L.psg_batch2d_launches.restype = C.c_long
    L.psg_batch2d_device_state.argtypes = [vp, i, C.POINTER(vp)]
    L.psg_ns2d_step_noalloc.argtypes = [i, i, C.c_double, C.c_double, i, vp, vp, vp]
    d = C.c_double
    L.psg_rec3d_create.argtypes = [C.POINTER(vp), i, d, i, i, i, i, i, d, i, d, d, d]
    L.psg_rec3d_destroy.argtypes = [vp]
    L.psg_rec3d_destroy.restype = None
    L.psg_rec3d_start.argtypes = [vp, C.POINTER(vp)]
    L.psg_rec3d_add.argtypes = [vp, i, C.POINTER(vp), C.POINTER(i)]
    L.psg_rec3d_guess.argtypes = [vp, dp, dp, dp, dp]
    L.psg_rec3d_count.argtypes = [vp]
    L.psg_rec3d_create_bous.argtypes = [C.POINTER(vp), i, d, i, i, i, i, i, d, i, d, d, d, d]
    L.psg_rec3d_guess_rho.argtypes = [vp, dp]
    L.psg_rec2d_create.argtypes = [C.POINTER(vp), i, i, d, i, i, i, i, d, i, d, d, dp]
    L.psg_rec2d_destroy.argtypes = [vp]
    L.psg_rec2d_destroy.restype = None
    L.psg_rec2d_set_stream.argtypes = [vp, vp]
    L.psg_rec2d_start.argtypes = [vp, C.POINTER(vp), i]
    L.psg_rec2d_add.argtypes = [vp, i, C.POINTER(vp), i, C.POINTER(i)]
    L.psg_rec2d_count.argtypes = [vp]
    L.psg_rec2d_guess.argtypes = [vp, i, dp, dp]
    L.psg_rec2d_launches.argtypes = [vp]
    L.psg_rec2d_launches.restype = C.c_long
    L.psg_upo2d_create.argtypes = [C.POINTER(vp), i, i, i, i]
    L.psg_upo2d_destroy.argtypes = [vp]
    L.psg_upo2d_destroy.restype = None
    L.psg_upo2d_set_guess.argtypes = [vp, i, dp, C.c_double, C.c_double, C.c_double, i, C.c_double, C.c_double]
    L.psg_upo2d_solve.argtypes = [vp, i, C.c_double, C.c_double]
    L.psg_upo2d_get.argtypes = [vp, i, dp, dp, ip]
    L.psg_upo2d_apply.argtypes = [vp, i, i, dp, dp]
    L.psg_upo2d_integrations.argtypes = [vp]
    L.psg_upo2d_integrations.restype = C.c_long
    L.psg_upo2d_trace.argtypes = [vp, i, i, dp]
    L.psg_upo2d_trace_count.argtypes = [vp, i]
    L.psg_upo2d_launches.argtypes = [vp]
    L.psg_upo2d_launches.restype = C.c_long
    L.psg_upo2d_set_arc.argtypes = [vp, i, dp, dp] + [C.c_double] * 7
    L.psg_upo2d_profile.argtypes = [vp, i]
    L.psg_upo2d_profile_read.argtypes = [vp, dp]
    L.psg_upo2d_get_nu.argtypes = [vp, i, dp]


def _check(rc):
    if rc != 0:
        raise PsgError(lib().psg_last_error().decode(errors="replace"))


def _ptrs(arrays):
    arr = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    return C.cast(arr, C.POINTER(C.c_void_p))


class NS3D:
    """Persistent 3D instance: device buffers and state stay in HBM across calls.

    scheme: SCHEME_NS_HEUN (3D NS DNS build), SCHEME_EULER_HEUN, SCHEME_NS_RK4
    (the Boussinesq RK4/CN scheme without density), SCHEME_BOUS_RK4.
    precision: 32 or 64.
    """

    def __init__(self, n: int, scheme: int = SCHEME_NS_RK4, precision: int = 32,
                 nu: float = 0.0, ampfor: float = 0.0, kf: float = 4.0, ri: float = 0.0,
                 sc: float = 1.0, theta: float = 0.0):
        L = lib()
        h = C.c_void_p()
        _check(L.psg_ns3d_create(C.byref(h), n, 1.0, scheme, precision))
        self._h = h
        self.n = n
        self.grid = Grid3D(n)
        self.scheme = scheme
        self.precision = precision
        self.ncomp = 4 if scheme == SCHEME_BOUS_RK4 else 3
        self.set_params(nu, ampfor, kf, ri, sc, theta)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().psg_ns3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, nu, ampfor=0.0, kf=4.0, ri=0.0, sc=1.0, theta=0.0):
        _check(lib().psg_ns3d_set_params(self._h, nu, ampfor, kf, ri, sc, theta))

    def set_stream(self, stream_ptr: int):
        _check(lib().psg_ns3d_set_stream(self._h, C.c_void_p(stream_ptr)))

    def upload(self, *comps):
        if len(comps) != self.ncomp:
            raise ValueError(f"expected {self.ncomp} components")
        arrs = [np.ascontiguousarray(c, dtype=np.complex128).reshape(-1) for c in comps]
        for a in arrs:
            if a.size != self.grid.nkt:
                raise ValueError("component size does not match the grid")
        _check(lib().psg_ns3d_upload(self._h, _ptrs(arrs)))

    def download(self, stage: bool = False):
        out = [np.zeros(self.grid.shape, np.complex128) for _ in range(self.ncomp)]
        fn = lib().psg_ns3d_download_stage if stage else lib().psg_ns3d_download
        _check(fn(self._h, _ptrs(out)))
        return tuple(out)

    def step(self, dt: float, nsteps: int = 1, dump_last: bool = False):
        _check(lib().psg_ns3d_step(self._h, dt, nsteps, int(dump_last)))

    def timederiv(self):
        out = [np.zeros(self.grid.shape, np.complex128) for _ in range(self.ncomp)]
        _check(lib().psg_ns3d_timederiv(self._h, _ptrs(out)))
        return tuple(out)

    def physical(self):
        n = self.n
        out = [np.zeros(n * n * n) for _ in range(3)]
        _check(lib().psg_ns3d_download_phys(self._h, _ptrs(out)))
        return np.stack([o.reshape(n, n, n) for o in out])

    def dump_mode(self, start_of_step: bool = False, velocity: bool = False):
        """Heun schemes: what step(..., dump_last=True) keeps: the physical
        vorticity of the predicted state (default) or of the state the step
        starts from, and optionally the velocity too (physical_velocity)."""
        _check(lib().psg_ns3d_dump_mode(self._h, int(start_of_step) | (2 * int(velocity))))

    def physical_velocity(self):
        n = self.n
        out = [np.zeros(n * n * n) for _ in range(3)]
        _check(lib().psg_ns3d_download_phys_velocity(self._h, _ptrs(out)))
        return np.stack([o.reshape(n, n, n) for o in out])

    def rms_accumulate(self, count: float):
        """mean squares of the kept velocity: ms = (ms count + u^2) / (count + 1)"""
        _check(lib().psg_ns3d_rms_accumulate(self._h, float(count)))

    def rms(self):
        n = self.n
        out = [np.zeros(n * n * n) for _ in range(3)]
        _check(lib().psg_ns3d_rms_download(self._h, _ptrs(out)))
        return np.stack([o.reshape(n, n, n) for o in out])

    def sync(self):
        _check(lib().psg_ns3d_sync(self._h))

    def energetics(self):
        """(energy, enstrophy, density variance): FP64 sums over the kept modes of
        |w|^2/k^2, |w|^2 and |rho|^2 (the reference's computeStats sums)."""
        out = (C.c_double * 3)()
        _check(lib().psg_ns3d_energetics(self._h, out))
        return out[0], out[1], out[2]

    def upload_device(self, ptrs):
        """state from device FP64 complex boxes (reference layout), one pointer per
        component; ordered on the engine's stream"""
        if len(ptrs) != self.ncomp:
            raise ValueError(f"expected {self.ncomp} components")
        arr = (C.c_void_p * self.ncomp)(*[int(p) for p in ptrs])
        _check(lib().psg_ns3d_upload_device(self._h, arr))

    LIN_TANGENT_STEP, LIN_ADJOINT_STEP, LIN_TANGENT_RHS, LIN_ADJOINT_RHS = 0, 1, 2, 3

    def linear(self, mode: int, x, dt: float = 0.0, out=None):
        """Tangent / adjoint step or right-hand side (see psg_ns3d_linear) applied to
        x, a torch CUDA complex128 tensor of shape (ncomp, IKTZ, IKTY, IKTX) in the
        reference layout (ncomp = 3, or 4 with the density); returns `out` (a new
        tensor unless given).  Ordered on the engine's stream (set_stream) -- the
        caller synchronises."""
        import torch
        nc = self.ncomp
        if x.dtype != torch.complex128 or not x.is_cuda or x.shape[0] != nc:
            raise ValueError(f"x must be a CUDA complex128 tensor of {nc} components")
        x = x.contiguous()
        if out is None:
            out = torch.empty_like(x)
        ip = (C.c_void_p * nc)(*[x[q].data_ptr() for q in range(nc)])
        op = (C.c_void_p * nc)(*[out[q].data_ptr() for q in range(nc)])
        _check(lib().psg_ns3d_linear(self._h, mode, dt, ip, op))
        return out

    def download_device(self, ptrs):
        if len(ptrs) != self.ncomp:
            raise ValueError(f"expected {self.ncomp} components")
        arr = (C.c_void_p * self.ncomp)(*[int(p) for p in ptrs])
        _check(lib().psg_ns3d_download_device(self._h, arr))

    @property
    def launches(self) -> int:
        return int(lib().psg_ns3d_launches(self._h))

    PASSES = ("z-inverse", "y-inverse", "x-pass", "y-forward", "z-forward+update")

    def profile(self, enable: bool = True):
        _check(lib().psg_ns3d_profile(self._h, int(enable)))

    def profile_read(self):
        ms = (C.c_double * 5)()
        cnt = (C.c_long * 5)()
        _check(lib().psg_ns3d_profile_read(self._h, ms, cnt))
        return {p: (ms[i], cnt[i]) for i, p in enumerate(self.PASSES)}

    def autotune(self, rerun: bool = True):
        """x-pass autotuner: (chosen variant, ms per launch of each variant)"""
        v = C.c_int()
        ms = (C.c_float * 16)()
        fn = lib().psg_ns3d_autotune if rerun else lib().psg_ns3d_tuning
        _check(fn(self._h, C.byref(v), ms))
        return v.value, list(ms)

    def pass_a_tuning(self):
        """pass-A choice of the autotuner: (packed f32x2 transforms or not,
        (ms scalar, ms packed) per launch; -1 where not timed)"""
        pk = C.c_int()
        ms = (C.c_float * 2)()
        _check(lib().psg_ns3d_tuning_a(self._h, C.byref(pk), ms))
        return bool(pk.value), (ms[0], ms[1])

    def device_state(self):
        xp = C.c_int()
        ptrs = (C.c_void_p * 4)()
        _check(lib().psg_ns3d_layout(self._h, C.byref(xp), C.cast(ptrs, C.POINTER(C.c_void_p))))
        return xp.value, [ptrs[i] for i in range(self.ncomp)]


class Batch2D:
    """Independent 2D Kolmogorov-flow instances of mixed sizes, integrated by one
    persistent kernel launch (one thread block per instance)."""

    def __init__(self, sizes, precision: int = 32):
        L = lib()
        self.sizes = [int(s) for s in sizes]
        arr = (C.c_int * len(self.sizes))(*self.sizes)
        h = C.c_void_p()
        _check(L.psg_batch2d_create(C.byref(h), len(self.sizes), arr, precision))
        self._h = h
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().psg_batch2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.sizes)

    def set_stream(self, stream_ptr: int):
        _check(lib().psg_batch2d_set_stream(self._h, C.c_void_p(stream_ptr)))

    def upload(self, i: int, Z):
        g = Grid2D(self.sizes[i])
        a = np.ascontiguousarray(Z, dtype=np.complex128).reshape(-1)
        if a.size != g.nkt:
            raise ValueError("state size does not match the instance grid")
        _check(lib().psg_batch2d_upload(self._h, i, a.ctypes.data_as(C.POINTER(C.c_double))))

    def download(self, i: int):
        g = Grid2D(self.sizes[i])
        a = np.zeros(g.shape, np.complex128)
        _check(lib().psg_batch2d_download(self._h, i, a.ctypes.data_as(C.POINTER(C.c_double))))
        return a

    def device_state(self, i: int) -> int:
        """device address of instance i's state (complex of the batch precision)"""
        p = C.c_void_p()
        _check(lib().psg_batch2d_device_state(self._h, i, C.byref(p)))
        return p.value

    def _params(self, nu, dt, nsteps):
        m = len(self.sizes)
        nu = np.broadcast_to(np.asarray(nu, np.float64), (m,)).copy()
        dt = np.broadcast_to(np.asarray(dt, np.float64), (m,)).copy()
        ns = np.broadcast_to(np.asarray(nsteps, np.int32), (m,)).copy()
        return (nu, dt, ns), (nu.ctypes.data_as(C.POINTER(C.c_double)),
                              dt.ctypes.data_as(C.POINTER(C.c_double)),
                              ns.ctypes.data_as(C.POINTER(C.c_int)))

    def run(self, nu, dt, nsteps):
        """integrate every instance i by nsteps[i] steps of dt[i] at viscosity nu[i]"""
        keep, args = self._params(nu, dt, nsteps)
        _check(lib().psg_batch2d_run(self._h, *args))

    def set_params(self, nu, dt, nsteps):
        keep, args = self._params(nu, dt, nsteps)
        _check(lib().psg_batch2d_set_params(self._h, *args))

    def launch(self):
        """one integration with the current parameters, as a replayed CUDA graph"""
        _check(lib().psg_batch2d_launch(self._h))

    def autotune(self):
        """block size of the persistent kernel: (variant, ms per 2-step run for 128,
        256, 512 threads)"""
        v = C.c_int()
        ms = (C.c_float * 3)()
        _check(lib().psg_batch2d_autotune(self._h, C.byref(v), ms))
        return v.value, list(ms)

    def schedule(self):
        """transform schedule per grid size {16, 32, 64, 128, 256}: (packed or
        not, (ms scalar, ms packed) of the batch); set by autotune()"""
        pk = (C.c_int * 5)()
        ms = (C.c_float * 10)()
        _check(lib().psg_batch2d_schedule(self._h, pk, ms))
        return {16 << q: (bool(pk[q]), (ms[2 * q], ms[2 * q + 1])) for q in range(5)}

    def set_schedule(self, packed):
        """pin the transform schedule: packed = a set of grid sizes (or a dict
        size -> bool) that run packed f32x2 transforms"""
        sel = {k for k, v in packed.items() if v} if isinstance(packed, dict) else set(packed)
        pk = (C.c_int * 5)(*[int((16 << q) in sel) for q in range(5)])
        _check(lib().psg_batch2d_set_schedule(self._h, pk))

    def sync(self):
        _check(lib().psg_batch2d_sync(self._h))

    @property
    def launches(self) -> int:
        return int(lib().psg_batch2d_launches(self._h))


class Recurrence3D:
    """Near-recurrence search over a ring of stored 3D states (the DNS's UPO guess
    generator), residuals on the GPU.  States are torch CUDA complex128 tensors
    of shape (3, IKTZ, IKTY, IKTX) in the reference layout; with ri given, the
    Boussinesq DNS's variant on four fields (xii, eta, zet, rho)."""

    def __init__(self, n, nout, dt, threshold, store_size=500, norm_width=8, nshift=(30, 2, 2),
                 alpha=1.0, tstart=0.0, v2=0.0, ri=None):
        h = C.c_void_p()
        if ri is None:
            _check(lib().psg_rec3d_create(C.byref(h), n, alpha, store_size, norm_width, nshift[0],
                                          nshift[1], nshift[2], threshold, nout, dt, tstart, v2))
            self.nc = 3
        else:
            _check(lib().psg_rec3d_create_bous(C.byref(h), n, alpha, store_size, norm_width,
                                               nshift[0], nshift[1], nshift[2], threshold, nout,
                                               dt, tstart, v2, ri))
            self.nc = 4
        self._h = h
        self.grid = Grid3D(n)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().psg_rec3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptrs(self, t):
        if t.shape[0] != self.nc:
            raise ValueError(f"expected {self.nc} fields")
        return (C.c_void_p * self.nc)(*[t[q].data_ptr() for q in range(self.nc)])

    def start(self, state):
        _check(lib().psg_rec3d_start(self._h, self._ptrs(state.contiguous())))

    def add(self, nt, state) -> bool:
        e = C.c_int()
        _check(lib().psg_rec3d_add(self._h, int(nt), self._ptrs(state.contiguous()), C.byref(e)))
        return bool(e.value)

    def guess(self):
        meta = np.zeros(7)
        out = [np.zeros(self.grid.shape, np.complex128) for _ in range(3)]
        dp = C.POINTER(C.c_double)
        _check(lib().psg_rec3d_guess(self._h, meta.ctypes.data_as(dp),
                                     *[o.ctypes.data_as(dp) for o in out]))
        if self.nc == 4:
            rho = np.zeros(self.grid.shape, np.complex128)
            _check(lib().psg_rec3d_guess_rho(self._h, rho.ctypes.data_as(dp)))
            out.append(rho)
        keys = ("time", "v2", "period", "shift_x", "shift_y", "shift_z", "residual")
        return dict(zip(keys, meta.tolist())), tuple(out)

    @property
    def count(self) -> int:
        return int(lib().psg_rec3d_count(self._h))


class Recurrence2D:
    """Near-recurrence search over rings of stored 2D states, batched over the
    runs of an ensemble (the 2D DNS's UPO guess generator), residuals on the
    GPU.  States are device boxes, one per run: torch CUDA tensors or the
    instances of a Batch2D of one grid size."""

    def __init__(self, nrun, n, nout, dt, threshold, v2, store_size=500, norm_width=8,
                 nshift=(32, 4), alpha=1.0, tstart=0.0):
        h = C.c_void_p()
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(v2, np.float64), (nrun,)))
        _check(lib().psg_rec2d_create(C.byref(h), nrun, n, alpha, store_size, norm_width,
                                      nshift[0], nshift[1], threshold, nout, dt, tstart,
                                      v.ctypes.data_as(C.POINTER(C.c_double))))
        self._h = h
        self.nrun = nrun
        self.grid = Grid2D(n)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().psg_rec2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptrs(self, states):
        if isinstance(states, Batch2D):
            ptrs = [states.device_state(i) for i in range(self.nrun)]
            return (C.c_void_p * self.nrun)(*ptrs), states.precision
        prec = 64 if states[0].dtype in (getattr(__import__("torch"), "complex128"),) else 32
        return (C.c_void_p * self.nrun)(*[t.data_ptr() for t in states]), prec

    def start(self, states):
        p, prec = self._ptrs(states)
        _check(lib().psg_rec2d_start(self._h, p, prec))

    def add(self, nt, states) -> int:
        """the states after step nt; returns the number of guesses emitted"""
        p, prec = self._ptrs(states)
        e = C.c_int()
        _check(lib().psg_rec2d_add(self._h, int(nt), p, prec, C.byref(e)))
        return int(e.value)

    @property
    def count(self) -> int:
        return int(lib().psg_rec2d_count(self._h))

    def guess(self, k):
        meta = np.zeros(7)
        Z = np.zeros(self.grid.shape, np.complex128)
        dp = C.POINTER(C.c_double)
        _check(lib().psg_rec2d_guess(self._h, k, meta.ctypes.data_as(dp), Z.ctypes.data_as(dp)))
        keys = ("run", "time", "v2", "period", "shift_x", "shift_y", "residual")
        d = dict(zip(keys, meta.tolist()))
        d["run"] = int(d["run"])
        return d, Z


UPO_STATUS = {0: "ACTIVE", 1: "CONVERGED", 2: "GMRES FAILED", 3: "H-STEP FAILED", 4: "NEWTON STALLED",
              5: "T-STEP FAILED", 6: "PERIOD TOO SMALL", 7: "NEWTON FAILED"}


class UPO2D:
    """Batched Newton-GMRES-hookstep search for periodic orbits of 2D Kolmogorov
    flow (all guesses of one grid size, FP64 integrations on the GPU)."""

    def __init__(self, nguess: int, n: int, kmax: int = 60, exact_jv: bool = True,
                 jv_precision: int = 64):
        """exact_jv: Krylov products from the exact tangent (jv_precision 64: FP64,
        32: base and tangent integrated in FP32) or, when False, the reference's
        FP64 forward difference.  Phi_T, residuals, Arnoldi and the hookstep are
        FP64 in every form."""
        if jv_precision not in (32, 64):
            raise ValueError("jv_precision must be 32 or 64")
        mode = (0 if jv_precision == 64 else 2) if exact_jv else 1
        h = C.c_void_p()
        _check(lib().psg_upo2d_create(C.byref(h), nguess, n, kmax, mode))
        self._h = h
        self.n = n
        self.grid = Grid2D(n)
        self.nguess = nguess

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().psg_upo2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_guess(self, i, Z, T, sx=0.0, sy=0.0, rsym=0, nu=1 / 40, dt=0.005):
        a = np.ascontiguousarray(Z, np.complex128).reshape(-1)
        _check(lib().psg_upo2d_set_guess(self._h, i, a.ctypes.data_as(C.POINTER(C.c_double)),
                                         T, sx, sy, rsym, nu, dt))

    def solve(self, max_newton=30, tol=1e-10, gmres_tol=1e-3):
        _check(lib().psg_upo2d_solve(self._h, max_newton, tol, gmres_tol))

    def get(self, i):
        Z = np.zeros(self.grid.shape, np.complex128)
        vals = np.zeros(4)
        info = np.zeros(4, np.int32)
        _check(lib().psg_upo2d_get(self._h, i, Z.ctypes.data_as(C.POINTER(C.c_double)),
                                   vals.ctypes.data_as(C.POINTER(C.c_double)),
                                   info.ctypes.data_as(C.POINTER(C.c_int))))
        return {"Z": Z, "T": vals[0], "sx": vals[1], "sy": vals[2], "residual": vals[3],
                "status": UPO_STATUS[int(info[0])], "newton": int(info[1]),
                "gmres": int(info[2]), "hookstep": int(info[3])}

    def set_arc(self, i, dZrdr, Zr2, dTrdr, dSrdr, dv2rdr, Tr2, Sr2, v2r2, ndelta):
        """Make guess i a pseudo-arclength corrector: nu becomes one more
        unknown and <dZrdr, z - Zr2> + dTrdr (T - Tr2) + dSrdr (sx - Sr2)
        + dv2rdr (nu - v2r2) = ndelta one more equation (call after set_guess)."""
        dz = np.ascontiguousarray(dZrdr, np.complex128).reshape(-1)
        z2 = np.ascontiguousarray(Zr2, np.complex128).reshape(-1)
        if dz.size != self.grid.nkt or z2.size != self.grid.nkt:
            raise ValueError("arc fields must have the grid's size")
        _check(lib().psg_upo2d_set_arc(self._h, i, dz.ctypes.data_as(C.POINTER(C.c_double)),
                                       z2.ctypes.data_as(C.POINTER(C.c_double)), dTrdr, dSrdr,
                                       dv2rdr, Tr2, Sr2, v2r2, ndelta))

    def nu(self, i):
        v = C.c_double()
        _check(lib().psg_upo2d_get_nu(self._h, i, C.byref(v)))
        return v.value

    def apply(self, i, mode, q=None):
        Z = np.zeros(self.grid.shape, np.complex128)
        qq = None
        if q is not None:
            qq = np.ascontiguousarray(q, np.complex128).copy()
        _check(lib().psg_upo2d_apply(self._h, i, mode, Z.ctypes.data_as(C.POINTER(C.c_double)),
                                     qq.ctypes.data_as(C.POINTER(C.c_double)) if qq is not None else None))
        return Z, qq

    def trace(self, i):
        """Per-Newton-step records of guess i: dicts with the Newton index, GMRES
        iterations and hookstep trials of the step, Delta after it, mu of its last
        trial, T, shift, residual |F|/|Phi_T(z)|, |F|, the time step in use and
        nu (which arc-length continuation moves)."""
        out = []
        rec = np.zeros(11)
        for k in range(int(lib().psg_upo2d_trace_count(self._h, i))):
            _check(lib().psg_upo2d_trace(self._h, i, k, rec.ctypes.data_as(C.POINTER(C.c_double))))
            out.append({"newton": int(rec[0]), "gmres": int(rec[1]), "hook": int(rec[2]),
                        "delta": rec[3], "mu": rec[4], "T": rec[5], "sx": rec[6],
                        "ner": rec[7], "normfn": rec[8], "dt": rec[9], "nu": rec[10]})
        return out

    @property
    def integrations(self):
        return int(lib().psg_upo2d_integrations(self._h))

    def profile(self, enable: bool = True):
        """phase timing of solve() (synchronises around every batched integration)"""
        _check(lib().psg_upo2d_profile(self._h, int(enable)))

    def profile_read(self):
        out = np.zeros(6)
        _check(lib().psg_upo2d_profile_read(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return dict(zip(("solve", "jv_exact64", "jv_exact32", "phi", "dzdt", "host_svd"),
                        out.tolist()))
