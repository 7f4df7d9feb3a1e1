"""Benchmark: 3D Navier-Stokes 256^3 RK4/CN steps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (per GPU): the Taylor-Green vortex u = (sin x cos y cos z,
-cos x sin y cos z, 0) on [0, 2pi]^3 plus a seeded divergence-free
perturbation of amplitude 1e-3 on |k| <= 4, nu = 1/1600, dt = 1e-3, 256^3 grid,
2/3 dealiasing, RK4 with per-stage Crank-Nicolson factors (the reference's RK4
scheme, 3D_Boussinesq/src/kernels.h:331-621, at Ri = 0).  Data are synthetic
(seeded initial field).  A step is one full RK4 step (four right-hand sides).

* ``value``: steps/s with the state resident in HBM (FP32 storage and
  transforms, vorticity only), all ranks' steps / max-over-ranks device time.
* ``e2e``: the same metric through the reference-facing C ABI
  (libpsg_bous3d.so ``timestep_cuda_``, Ri = 0, FP64 host arrays in pinned
  memory) with the host<->device copies of every call inside the timed region,
  10 steps per call.
* ``--impl reference``: the reference's own CUDA step built from its sources
  (oracle/_ref/libref_bous3d.so, FP64 cuFFT), driven by the same calls.
* ``cpu_baseline``: the FP64 CPU oracle (C + OpenMP on all host threads) on a
  bounded sample of the same workload (one RK4 step of the same scheme).
* ``roofline``: the dominant pass (largest share of the step's device time),
  its algorithmic HBM bytes per launch over its average CUDA-event duration,
  against the measured copy bandwidth in MEASURED_PEAKS.json.
* ``fp64_engine``: device steps/s of the same workload on the FP64 engine (the
  reference's precision), Navier-Stokes RK4/CN and Boussinesq at Ri = 0.

The device working set (state, stage registers, transform buffers: ~0.8 GB)
is far larger than the 126 MB L2, so every pass streams from HBM; no L2 flush
is needed between steps.  Multi-GPU runs are independent replicas (a single
256^3 field is not split across GPUs), scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
NU = 1.0 / 1600.0
DT = 1e-3
STEPS_PER_CALL = 10
METRIC = "3D NS 256^3 RK4/CN steps/s (Taylor-Green, FP32, 1 B200 per replica)"


# ---------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=10.0):
        """block until nvidia-smi has produced its first sample"""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(n, word=8, nc=3, nfi=6):
    """HBM bytes of one right-hand side per pass, complex words of `word` bytes,
    counting only kept modes (IKTX = n/3+1 columns, IKTY = IKTZ = 2(n/3)+1 rows)
    and one read plus one write per pass; pass A also reads the nc stage-state
    components, pass E writes/reads the scheme registers (counted per stage in
    stage_bytes).  nc state components, nfi fields through the x-pass (3, 6
    for Navier-Stokes; 4, 9 for Boussinesq)."""
    K = n // 3
    X, Y = K + 1, 2 * K + 1
    a = (nc * X * Y * Y + nfi * X * Y * n) * word
    b = (nfi * X * Y * n + nfi * X * n * n) * word
    c = (nfi * X * n * n + nc * X * n * n) * word
    d = (nc * X * n * n + nc * X * Y * n) * word
    e = (nc * X * Y * n) * word
    return [a, b, c, d, e]


def stage_bytes(n, stage, word=8, nc=3, carried=True):
    """state/register traffic of pass E for RK4 stage 0..3 (nc components each):
    stages 0-2 read S and write K_s and X0; the final stage reads S, K1, K2, K3
    (and the carried rounding error of the FP32 state) and writes S, X0 (and
    that error)."""
    K = n // 3
    nkt = (K + 1) * (2 * K + 1) ** 2
    arrays = 3 if stage < 3 else (8 if carried else 6)
    return arrays * nc * nkt * word


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, dist):
    import torch
    import psgpu_b200 as P
    from psgpu_b200.abi import TimestepLibrary
    from psgpu_b200.fields import taylor_green3d

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    xi, et, zt = taylor_green3d(N, 1234 + rank, amp=1e-3)
    eng = P.NS3D(N, P.SCHEME_NS_RK4, precision=32, nu=NU)
    stream = torch.cuda.current_stream(dev)
    eng.set_stream(stream.cuda_stream)
    eng.upload(xi, et, zt)
    tune = eng.autotune(rerun=False)
    tune_a = eng.pass_a_tuning()
    for _ in range(args.warmup):
        eng.step(DT, 1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(dev.index)
    clk.start()
    clk.wait_first()
    l0 = eng.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.step(DT, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = eng.launches - l0
    clocks = clk.stop()
    # per-pass shares of the step: a further segment with CUDA events between
    # the passes (each event ends the programmatic overlap of two passes, so
    # the timed region above runs without them)
    eng.profile(True)
    eng.step(DT, min(args.steps, 20))
    prof = eng.profile_read()
    eng.profile(False)
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.steps / (ms / 1e3)

    # roofline of the dominant pass
    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes(N, 8)
    per_step_stage = sum(stage_bytes(N, s) for s in range(4)) / 4.0
    shares = {}
    tot = sum(v[0] for v in prof.values())
    roof = None
    for i, (name, (pms, cnt)) in enumerate(prof.items()):
        shares[name] = round(pms / tot, 4) if tot else None
    dom_i = max(range(5), key=lambda i: list(prof.values())[i][0])
    dom_name = list(prof.keys())[dom_i]
    dom_ms, dom_cnt = list(prof.values())[dom_i]
    dom_bytes = alg[dom_i] + (per_step_stage if dom_i == 4 else 0)
    achieved = dom_bytes / (dom_ms / dom_cnt / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        with open(tf) as f:
            traffic = json.load(f).get(dom_name)
    roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1),
            "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "algorithmic_bytes": int(dom_bytes), "avg_launch_ms": round(dom_ms / dom_cnt, 5),
            "launches_timed": int(dom_cnt),
            "timed_by": "CUDA events on the engine's stream between the passes, over a segment of "
                        "min(steps, 20) steps after the headline's timed region",
            "pass_share": shares}
    step_bytes = 4 * sum(alg) + sum(stage_bytes(N, s) for s in range(4))
    whole = {"algorithmic_bytes_per_step": int(step_bytes),
             "achieved_GBps": round(step_bytes / (ms / args.steps / 1e3) / 1e9, 1)}
    whole["frac"] = round(whole["achieved_GBps"] / peak, 4)

    # e2e through the reference-facing C ABI with host buffers
    e2e = None if args.no_e2e else run_e2e(args, dev, dist, world, rank)
    fp64_e2e = None if args.no_e2e else run_e2e(args, dev, dist, world, rank, precision=64)
    eng.close()
    ref_steady = reference_steady() if (world == 1 and not args.no_ref) else None

    same_prec = run_fp64(args, dev, stream) if world == 1 and not args.no_fp64 else None
    upo = run_upo(args) if (world == 1 and not args.no_upo) else None
    ens = None if args.no_ensemble else run_ensemble2d(args, rank, world, dist, dev)
    single2d = run_ns2d_single(args) if (world == 1 and not args.no_ensemble) else None

    out = None
    if rank == 0:
        cpu = cpu_baseline() if world == 1 and not args.no_cpu else None
        if N != 256:
            out_note = f"profiling grid {N}^3, not the benchmark configuration"
        else:
            out_note = None
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "3D NS 256^3 Taylor-Green, RK4/CN (Boussinesq scheme, Ri=0), "
                                   "nu=1/1600, dt=1e-3, 2/3 dealias",
                       "grid": N, "replicas": world, "parallelism": f"replicas{world}",
                       "l2": "working set ~0.8 GB per replica >> 126 MB L2; no flush"},
            "e2e": e2e, "roofline": roof, "whole_step": whole, "cpu_baseline": cpu, "upo": upo,
            "ensemble2d": ens, "ns2d_single": single2d, "fp64_engine": same_prec,
            "fp64_e2e": fp64_e2e,
            "reference_steady_ms_per_step": ref_steady["steady_ms_per_step"] if ref_steady else None,
            "reference_steady": ref_steady,
            "clocks": clocks, "gpu_launches": int(launches),
            "pass_a_autotune": {"packed": tune_a[0], "ms_per_launch": [round(x, 4) for x in tune_a[1]],
                                "choices": "scalar, packed f32x2 (two fields per instruction)"},
            "launch": "passes chained by programmatic dependent launch, the x-pass excepted "
                      "(each pass's blocks start and stage their tables while the previous pass "
                      "drains; PSG_PDL=" + os.environ.get("PSG_PDL", "2") + ")",
            "x_pass_autotune": {"variant": tune[0], "ms_per_launch": [round(x, 4) for x in tune[1]],
                                "variants": "bit 0: 256/G rows per block (else 128/G), bit 3: "
                                            "64/G rows, bit 1: two copy buffers per warp, bit 2: "
                                            "packed f32x2 transforms (FP32); -1: not built or "
                                            "does not fit"},
        }
        if out_note:
            out["note"] = out_note
    return out


def pass_table(args, nsteps=10):
    """Per-pass live timings (CUDA events at the engine's pass boundaries,
    psg_ns3d_profile_read) at args.grid^3 for the Navier-Stokes and
    Boussinesq RK4/CN engines in FP32 and FP64, after 3 warm-up steps: average
    launch time, algorithmic bytes (algorithmic_bytes / stage_bytes, the final
    stage's registers averaged over the four stages) and the achieved fraction
    of the measured HBM copy bandwidth.  Every pass input at 256^3 exceeds
    the 126 MB L2."""
    import torch
    import psgpu_b200 as P
    from psgpu_b200.fields import taylor_green3d

    torch.cuda.set_device(0)
    n = args.grid
    peak, kind = measured_peaks()
    xi, et, zt = taylor_green3d(n, 1234, amp=1e-3)
    out = {"grid": n, "steps": nsteps, "peak_GBps": peak, "peak_kind": kind, "engines": {}}
    for name, scheme, prec in (("ns_rk4_fp32", P.SCHEME_NS_RK4, 32),
                               ("ns_rk4_fp64", P.SCHEME_NS_RK4, 64),
                               ("bous_fp32", P.SCHEME_BOUS_RK4, 32),
                               ("bous_fp64", P.SCHEME_BOUS_RK4, 64)):
        bous = scheme == P.SCHEME_BOUS_RK4
        eng = P.NS3D(n, scheme, precision=prec, nu=NU, ri=1.0 if bous else 0.0)
        eng.upload(*((xi, et, zt, 0.01 * xi) if bous else (xi, et, zt)))
        eng.step(DT, 3)
        eng.sync()
        eng.profile(True)
        eng.step(DT, nsteps)
        eng.sync()
        prof = eng.profile_read()
        eng.profile(False)
        nc, nfi = (4, 9) if bous else (3, 6)
        word = 8 if prec == 32 else 16
        alg = algorithmic_bytes(n, word, nc, nfi)
        stage = sum(stage_bytes(n, s, word, nc, carried=(prec == 32)) for s in range(4)) / 4.0
        rows = {}
        for i, (pname, (ms, cnt)) in enumerate(prof.items()):
            b = alg[i] + (stage if i == 4 else 0)
            t = ms / cnt / 1e3
            rows[pname] = {"avg_launch_us": round(t * 1e6, 2), "algorithmic_MB": round(b / 1e6, 1),
                           "achieved_GBps": round(b / t / 1e9, 1),
                           "frac": round(b / t / 1e9 / peak, 4)}
        tot_ms = sum(v[0] for v in prof.values())
        step_b = 4 * sum(alg) + sum(stage_bytes(n, s, word, nc, carried=(prec == 32))
                                    for s in range(4))
        out["engines"][name] = {"passes": rows, "xpass_variant": eng.autotune(rerun=False),
                                "ms_per_step_passes": round(tot_ms / nsteps, 4),
                                "step_frac": round(step_b / (tot_ms / nsteps / 1e3) / 1e9 / peak, 4)}
        eng.close()
    return out


def run_fp64(args, dev, stream, nsteps=20):
    """The same workload on the FP64 engine (the reference's precision), device
    steps/s for the Navier-Stokes RK4/CN scheme and the Boussinesq scheme at
    Ri = 0 that the reference arm runs."""
    import torch
    import psgpu_b200 as P
    from psgpu_b200.fields import taylor_green3d

    xi, et, zt = taylor_green3d(N, 1234, amp=1e-3)
    out = {}
    for name, scheme, comps in (("ns_rk4", P.SCHEME_NS_RK4, (xi, et, zt)),
                                ("boussinesq_ri0", P.SCHEME_BOUS_RK4,
                                 (xi, et, zt, np.zeros_like(xi)))):
        eng = P.NS3D(N, scheme, precision=64, nu=NU)
        eng.set_stream(stream.cuda_stream)
        eng.upload(*comps)
        eng.step(DT, 3)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step(DT, nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        eng.close()
        out[name + "_steps_per_s"] = round(nsteps / (e0.elapsed_time(e1) / 1e3), 2)
    out["steps"] = nsteps
    return out


class quiet_stdout:
    """Send what native code writes to file descriptor 1 (the reference's
    progress lines) to stderr, so that stdout carries only the JSON line."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        self._libc = ctypes.CDLL(None)
        self._libc.fflush(None)
        self._saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        return False


def ref2d_step_ms(steps, n=None):
    """ms per step of the reference's 2D timestep_cuda_ (n^2, default 128^2, one
    call of `steps` steps including its per-call set-up), in a fresh process"""
    cmd = [sys.executable, os.path.abspath(__file__), "--ref2d-probe", str(steps)]
    if n:
        cmd += ["--grid2d", str(n)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    for line in reversed(r.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)["ms_per_step"]
    raise RuntimeError("reference 2D probe failed: " + r.stderr[-400:])


def run_ref2d_probe(steps, n=None):
    import torch
    from psgpu_b200.abi import TimestepLibrary
    from psgpu_b200.fields import kolmogorov_ic2d

    torch.cuda.set_device(0)
    n = n or UPO_N
    lib = TimestepLibrary(os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so"), "ns2d")
    Z = kolmogorov_ic2d(n, 4242)
    with quiet_stdout():
        lib.ns2d(Z, n, UPO_NU, UPO_DT, 10)
        t0 = time.perf_counter()
        lib.ns2d(Z, n, UPO_NU, UPO_DT, steps)
        sec = time.perf_counter() - t0
    return {"ms_per_step": 1e3 * sec / steps, "steps": steps, "n": n}


# ------------------------------------------------------ UPO Newton iterations
UPO_N, UPO_NU, UPO_DT, UPO_GUESSES, UPO_KMAX = 128, 1.0 / 40.0, 0.005, 64, 60


def upo_guesses(G=UPO_GUESSES, search=400.0, seed=5000):
    """64 guesses from turbulent 2D Kolmogorov states, Re = 40, 128^2: 64 seeded
    runs (modes 1 <= |k| <= 8, enstrophy 1) spun up for 500 time units in one
    persistent FP32 launch, then continued for `search` time units under the
    GPU recurrence search (every 0.1 time units, a ring of 20 time units,
    32 x 4 trial shifts over the 2 x 8^2 lowest modes, threshold 0.4).  Of the
    emitted guesses those with periods in [5, 20] are kept, lowest residual
    first; runs that emitted none (or too few overall) contribute their last
    state with a period drawn uniformly in [5, 20]."""
    import psgpu_b200 as P
    from psgpu_b200.fields import kolmogorov_ic2d

    n, nu, dt = UPO_N, UPO_NU, UPO_DT
    b = P.Batch2D([n] * G, precision=32)
    for i in range(G):
        b.upload(i, kolmogorov_ic2d(n, seed + i))
    t0 = time.perf_counter()
    b.run([nu] * G, [dt] * G, [int(round(500.0 / dt))] * G)
    b.sync()
    spin_s = time.perf_counter() - t0
    nout = 20
    rec = P.Recurrence2D(G, n, nout, dt, 0.4, nu, store_size=int(round(20.0 / (nout * dt))) + 1,
                         norm_width=8, nshift=(32, 4), tstart=500.0)
    t0 = time.perf_counter()
    rec.start(b)
    nchk = int(round(search / (nout * dt)))
    for k in range(1, nchk + 1):
        b.run(nu, dt, nout)
        rec.add(k * nout, b)
    b.sync()
    search_s = time.perf_counter() - t0
    found = [rec.guess(k) for k in range(rec.count)]
    found = [g for g in found if 5.0 <= g[0]["period"] <= 20.0]
    found.sort(key=lambda g: g[0]["residual"])
    guesses = [(Z, m["period"], m["shift_x"], m["shift_y"], m["residual"]) for m, Z in found[:G]]
    nrec = len(guesses)
    rng = np.random.default_rng(77)
    i = 0
    while len(guesses) < G:
        guesses.append((b.download(i % G), float(rng.uniform(5.0, 20.0)), 0.0, 0.0, None))
        i += 1
    b.close()
    rec.close()
    return guesses, {"spinup_seconds": round(spin_s, 2), "search_seconds": round(search_s, 2),
                     "recurrence_guesses": nrec, "search_time_units": search,
                     "median_recurrence_residual":
                         float(np.median([g[4] for g in guesses[:nrec]])) if nrec else None}


def solve_upo(guesses, form, max_newton):
    """one batched Newton-GMRES-hookstep solve of all guesses; form: exact32,
    exact64 or fd"""
    import torch
    import psgpu_b200 as P

    n, nu, dt = UPO_N, UPO_NU, UPO_DT
    G = len(guesses)
    u = P.UPO2D(G, n, kmax=UPO_KMAX, exact_jv=form != "fd",
                jv_precision=32 if form == "exact32" else 64)
    for i, (Z, T, sx, sy, _) in enumerate(guesses):
        u.set_guess(i, Z, T=float(T), sx=float(sx), sy=float(sy), nu=nu, dt=dt)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    u.solve(max_newton=max_newton, tol=1e-10, gmres_tol=1e-3)
    sec = time.perf_counter() - t0
    info = [u.get(i) for i in range(G)]
    u.close()
    newton = sum(x["newton"] for x in info)
    conv = sum(x["status"] == "CONVERGED" for x in info)
    res = np.array([x["residual"] for x in info])
    status = {}
    for x in info:
        status[x["status"]] = status.get(x["status"], 0) + 1
    return {"newton_iters_per_s": round(newton / sec, 4), "newton_iters": newton,
            "gmres_iters": sum(x["gmres"] for x in info), "seconds": round(sec, 2),
            "converged": int(conv),
            "seconds_per_converged_orbit": round(sec / conv, 2) if conv else None,
            "converged_periods": sorted(round(x["T"], 5) for x in info
                                        if x["status"] == "CONVERGED"),
            "median_rel_residual": float(np.median(res)),
            "min_rel_residual": float(res.min()), "statuses": status}


def plain_upo(guess, max_newton=1):
    """The reference's plain form, run: its Newton-GMRES-hookstep (the FP64
    restatement oracle/newton2d.py, one guess at a time, forward-difference Jv
    with eps = 1e-7, DGESDD) with every integration one call of the reference's
    own 2D timestep_cuda_ (oracle/_ref/libref_ns2d.so, FP64 cuFFT, allocations
    and plans per call) and TIMEDERIV on the host; the host's linear algebra
    is included, as in the reference's driver."""
    from oracle import pyoracle as O
    from oracle.newton2d import Newton2D
    from psgpu_b200.abi import TimestepLibrary

    path = os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so")
    if not os.path.exists(path):
        return None
    n, nu, dt = UPO_N, UPO_NU, UPO_DT
    lib = TimestepLibrary(path, "ns2d")

    def phi(z, t, truedelt):
        ns = int(t / truedelt)
        return lib.ns2d(z, n, nu, t / ns, ns)[0]

    def rhs(z):
        return O.ns2d_timederiv(z, n, nu)

    Z, T, sx, sy, _ = guess
    solver = Newton2D(n, phi, rhs, gmresmax=UPO_KMAX)
    with quiet_stdout():
        t0 = time.perf_counter()
        r = solver.solve(Z, float(T), float(sx), float(sy), 0, dt, max_newton=max_newton)
        sec = time.perf_counter() - t0
    return {"newton_iters_per_s": round(r.newton / sec, 6), "newton_iters": r.newton,
            "gmres_iters": r.gmres, "integrations": r.integrations, "seconds": round(sec, 2),
            "period": round(float(T), 4), "rel_residual": r.ner, "status": r.status,
            "how": "one guess, the reference's Newton-GMRES-hookstep restated in FP64 on the "
                   "host with every integration a call of the reference's own 2D "
                   "timestep_cuda_ (FP64 cuFFT), run, not costed"}


def run_upo(args):
    """Batched Newton-GMRES-hookstep on 2D Kolmogorov flow, Re = 40, 128^2,
    Krylov dimension 60, FP64 residuals, Arnoldi and hookstep, target 1e-10:
    the 64 recurrence-derived guesses of upo_guesses() solved in the chosen
    form (exact tangent Jv integrated in FP32), with the FP64 forward
    difference of the same solver beside it, and the reference's plain form
    (one guess at a time, one reference timestep_cuda_ call per integration)
    run on the shortest-period guess; then the --upo-converge shortest-period
    guesses solved in both forms for up to --upo-converge-newton iterations,
    with the orbits converged to 1e-10 and the seconds per converged orbit."""
    guesses, out = upo_guesses()
    out["workload"] = ("2D Kolmogorov Re=40 128^2, 64 guesses from turbulent states after a "
                       "500 time-unit spin-up, periods in [5,20] from the recurrence search, "
                       "Krylov 60, FP64 residual/Arnoldi/hookstep, tol 1e-10")
    out["newton_per_guess_max"] = args.upo_newton
    forms = ("exact32", "fd") if not args.upo_all_forms else ("exact32", "exact64", "fd")
    for form in forms:
        out[{"exact32": "exact_jv", "exact64": "exact_jv_fp64", "fd": "fd_jv"}[form]] = \
            solve_upo(guesses, form, args.upo_newton)
    if not args.no_upo_plain:
        short = min(guesses, key=lambda g: g[1])
        plain = plain_upo(short)
        if plain:
            out["plain_reference"] = plain
            out["exact_vs_plain"] = round(out["exact_jv"]["newton_iters_per_s"] /
                                          plain["newton_iters_per_s"], 1)
    out["exact_vs_fd"] = round(out["exact_jv"]["newton_iters_per_s"] /
                               out["fd_jv"]["newton_iters_per_s"], 3)
    if args.upo_converge:
        # to convergence within the default run's time: the shortest-period
        # guesses, up to `upo_converge_newton` Newton iterations each
        short = sorted(guesses, key=lambda g: g[1])[:args.upo_converge]
        conv = {"guesses": len(short), "newton_per_guess_max": args.upo_converge_newton,
                "periods": [round(float(g[1]), 3) for g in short]}
        for form in ("exact32", "fd"):
            conv[{"exact32": "exact_jv", "fd": "fd_jv"}[form]] = \
                solve_upo(short, form, args.upo_converge_newton)
        out["to_convergence"] = conv
    return out


# --------------------------------------------- 2D Kolmogorov flow, one instance
def run_ns2d_single(args):
    """2D Kolmogorov flow, 128^2, nu = 1/40, dt = 0.005, 2000 RK4/CN steps, FP64,
    seeded initial vorticity (modes 1 <= |k| <= 8, amplitude ~ 1/|k|, enstrophy
    1): through the 2D drop-in timestep_cuda_ (host arrays in and out inside the
    timed region), beside the reference's own 2D step (timed on a 200-step call
    in a separate process) and the oracle's host step on a 50-step sample."""
    import psgpu_b200 as P
    from oracle import pyoracle as O
    from psgpu_b200.abi import TimestepLibrary
    from psgpu_b200.fields import kolmogorov_ic2d

    n, nu, dt, steps = 128, 1.0 / 40.0, 0.005, 2000
    Z0 = kolmogorov_ic2d(n, 77)
    os.environ["PSG_PRECISION"] = "64"
    lib = TimestepLibrary(P.dropin_path("ns2d"), "ns2d")
    lib.ns2d(Z0.copy(), n, nu, dt, 10)
    t0 = time.perf_counter()
    Z, _ = lib.ns2d(Z0.copy(), n, nu, dt, steps)
    ours = time.perf_counter() - t0
    os.environ["PSG_PRECISION"] = "32"
    out = {"workload": "2D Kolmogorov 128^2, nu=1/40, dt=0.005, 2000 RK4/CN steps, FP64",
           "steps_per_s": round(steps / ours, 1), "api": "timestep_cuda_ (2D ABI), e2e",
           "finite": bool(np.isfinite(Z).all())}
    path = os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so")
    if os.path.exists(path):
        ms = ref2d_step_ms(200, n)
        out["reference_steps_per_s"] = round(1e3 / ms, 1)
    t0 = time.perf_counter()
    O.ns2d_timestep(Z0.copy(), n, nu, dt, 50)
    out["cpu_port_steps_per_s"] = round(50 / (time.perf_counter() - t0), 1)
    out["cpu_cores"] = O.num_threads()
    return out


# ------------------------------------------------------------ 2D ensemble
def run_ensemble2d(args, rank=0, world=1, dist=None, dev=None):
    """512 independent 2D Kolmogorov runs in one persistent launch replayed as a
    CUDA graph: sizes uniform over {64^2, 128^2, 256^2}, Re uniform in [20, 100],
    forcing wavenumber 4, seeded initial vorticity (modes 1 <= |k| <= 8, phases
    uniform, amplitude ~ 1/|k|, enstrophy 1), dt = 0.005, 1000 steps each, FP32;
    block size picked by the autotuner.  Instance-steps per second on the device
    and end to end (initial states uploaded from the host and final states
    downloaded inside the timed region), beside the reference's 2D step run one
    instance at a time (its ms/step per size measured on a 200-step call).
    With N ranks the 512 instances are split by cost (psgpu_b200.replicas) and
    the time is the slowest rank's (strong scaling: the total work is fixed)."""
    import torch
    import psgpu_b200 as P
    from psgpu_b200.fields import kolmogorov_ic2d
    from psgpu_b200.replicas import cost2d, max_over_ranks, shard

    M, steps = 512, 1000
    rng = np.random.default_rng(2048)
    sizes_all = rng.choice([64, 128, 256], M)
    nu_all = 1.0 / rng.uniform(20.0, 100.0, M)
    mine = shard([cost2d(int(n)) for n in sizes_all], world)[rank]
    sizes = [int(sizes_all[i]) for i in mine]
    nu = nu_all[mine]
    ics = [kolmogorov_ic2d(int(sizes_all[i]), 9000 + i) for i in mine]
    m = len(mine)
    b = P.Batch2D(sizes, precision=32)
    for i in range(m):
        b.upload(i, ics[i])
    b.set_params(nu, 0.005, steps)
    tune = b.autotune()
    sched = b.schedule()
    stream = torch.cuda.current_stream()
    b.set_stream(stream.cuda_stream)
    b.launch()  # warm-up: captures the graph
    b.sync()
    for i in range(m):
        b.upload(i, ics[i])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    l0 = b.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.launch()
    e1.record(stream)
    torch.cuda.synchronize()
    dev_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, dev)
    launches = b.launches - l0
    # end to end: upload every initial state, integrate, download every result
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(m):
        b.upload(i, ics[i])
    b.launch()
    outs = [b.download(i) for i in range(m)]
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    finite = all(np.isfinite(o).all() for o in outs)
    b.close()
    if rank != 0:
        return None
    out = {"workload": "512 x 2D Kolmogorov, sizes U{64,128,256}^2, Re U[20,100], kf=4, "
                       "dt=0.005, 1000 steps, FP32, one persistent launch (CUDA graph) per GPU",
           "instance_steps_per_s": round(M * steps / dev_s, 1), "seconds": round(dev_s, 4),
           "e2e_instance_steps_per_s": round(M * steps / e2e_s, 1), "e2e_seconds": round(e2e_s, 3),
           "scaling": "strong", "ranks": world, "gpu_launches": launches, "finite": bool(finite),
           "block_autotune": {"variant": tune[0], "ms_per_2_steps": [round(x, 4) for x in tune[1]],
                              "threads": [128, 256, 512]},
           "transform_schedule": {str(n): {"packed": pk, "ms_scalar_packed": [round(x, 4) for x in ms]}
                                  for n, (pk, ms) in sched.items() if ms[0] >= 0}}
    flops = ensemble_flops([int(n) for n in sizes_all], steps)
    peak = fp32_simt_peak(dev if dev is not None else torch.cuda.current_device())
    out["flop_rate"] = {"achieved_tflops": round(flops / dev_s / 1e12, 3),
                        "peak_tflops": round(peak / 1e12, 2), "frac": round(flops / dev_s / peak, 4),
                        "peak_kind": "nominal FP32 SIMT (SMs x 128 lanes x 2 x max SM clock)",
                        "flops": "nominal FFT flops: a real N x N transform 2.5 N^2 log2 N^2, five "
                                 "per right-hand side, four per RK4 step (the truncated modes the "
                                 "kernel skips are counted)"}
    path = os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so")
    if os.path.exists(path) and world == 1:
        out["plain_reference"] = ensemble_plain(sizes_all, nu_all, path)
    return out


def ensemble_flops(sizes, steps):
    """Nominal FFT flops of `steps` RK4/CN steps of 2D instances of the given
    grid sizes: a real N x N transform counted as 2.5 N^2 log2(N^2) (the
    5 n log2 n convention for a complex length-n transform), five per
    right-hand side (w, u, v inverse; the two products forward), four
    right-hand sides per step."""
    per_step = sum(4 * 5 * 2.5 * n * n * math.log2(n * n) for n in sizes)
    return per_step * steps


def fp32_simt_peak(dev):
    """Nominal FP32 SIMT rate of the device in FLOP/s: SMs x 128 FP32 lanes x
    2 (fused multiply-add) x the maximum SM clock recorded in the peaks file
    (1965 MHz without one)."""
    import torch
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = 1965.0
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            mhz = float(json.load(f).get("sm_max_mhz", mhz))
    return nsm * 128 * 2 * mhz * 1e6


def ensemble_plain(sizes_all, nu_all, path, per_size=4, steps=200):
    """The reference's plain form of the ensemble, run on a stated subset: the
    first `per_size` instances of each grid size (their own initial states and
    viscosities), one reference 2D timestep_cuda_ call of `steps` steps each,
    one instance at a time, host arrays in and out (its set-up per call
    included).  The subset holds equal numbers of each size, as the
    ensemble's uniform size draw does on average."""
    from psgpu_b200.abi import TimestepLibrary
    from psgpu_b200.fields import kolmogorov_ic2d

    lib = TimestepLibrary(path, "ns2d")
    pick = []
    for sz in (64, 128, 256):
        pick += [i for i in range(len(sizes_all)) if int(sizes_all[i]) == sz][:per_size]
    with quiet_stdout():
        lib.ns2d(kolmogorov_ic2d(64, 1), 64, 1 / 40, 0.005, 2)  # first-call costs
        t0 = time.perf_counter()
        for i in pick:
            n = int(sizes_all[i])
            lib.ns2d(kolmogorov_ic2d(n, 9000 + i), n, float(nu_all[i]), 0.005, steps)
        sec = time.perf_counter() - t0
    return {"instance_steps_per_s": round(len(pick) * steps / sec, 2), "instances": len(pick),
            "steps_each": steps, "seconds": round(sec, 2),
            "how": f"the reference's 2D timestep_cuda_ run on {per_size} instances of each size "
                   f"of the ensemble, {steps} steps each, one call per instance"}


def run_e2e(args, dev, dist, world, rank, precision=32):
    """The bench workload through the Boussinesq drop-in timestep_cuda_ with FP64
    host arrays: precision 32 is the FP32 engine (PSG_PRECISION=32); 64 is the
    drop-in's default, the reference's precision."""
    import psgpu_b200 as P
    from psgpu_b200.abi import TimestepLibrary

    if precision == 32:
        os.environ["PSG_PRECISION"] = "32"
    else:
        os.environ.pop("PSG_PRECISION", None)
    try:
        lib = TimestepLibrary(P.dropin_path("bous3d"), "bous3d")
        out = time_abi_calls(lib, args, dev, dist, world, rank, ours=True)
    finally:
        os.environ.pop("PSG_PRECISION", None)
    out["precision"] = f"fp{precision}"
    return out


def reference_steady(steps=200, short=10):
    """The reference's Boussinesq timestep_cuda_ on the bench workload, its
    per-call set-up separated from its steady time per step: one call of
    `short` steps and one of `short + steps`, both timed end to end (each call
    allocates, plans, copies, steps and frees); steady = difference / steps,
    set-up = short call - short * steady."""
    import torch
    from psgpu_b200.abi import TimestepLibrary
    from psgpu_b200.fields import Grid3D, taylor_green3d

    path = os.path.join(ROOT, "oracle", "_ref", "libref_bous3d.so")
    if not os.path.exists(path):
        return None
    lib = TimestepLibrary(path, "bous3d")
    g = Grid3D(N)
    xi, et, zt = taylor_green3d(N, 1234, amp=1e-3)
    comps0 = [np.ascontiguousarray(a, np.complex128) for a in (xi, et, zt, np.zeros_like(xi))]

    def call(nsteps):
        comps = [a.copy() for a in comps0]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lib.bous3d_inplace(comps, N, NU, DT, (nsteps + 0.5) * DT)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, rk4_evaluations(0.0, (nsteps + 0.5) * DT, DT)

    with quiet_stdout():
        call(short)  # first-call costs (context, cuFFT library load)
        t_s, n_s = call(short)
        t_l, n_l = call(short + steps)
    steady = (t_l - t_s) / (n_l - n_s)
    return {"steady_ms_per_step": round(1e3 * steady, 4),
            "setup_ms_per_call": round(1e3 * (t_s - n_s * steady), 2),
            "short_call_steps": n_s, "long_call_steps": n_l,
            "how": "reference timestep_cuda_ (3D_Boussinesq/src/src_gmres/cuda.cu, FP64 cuFFT), "
                   "a short and a long call on the same 256^3 workload, host arrays"}


def time_abi_calls(lib, args, dev, dist, world, rank, ours):
    """K steps in calls of STEPS_PER_CALL through timestep_cuda_ with pinned host
    arrays; the copies in and out of every call are inside the timed region."""
    import torch
    from psgpu_b200.fields import Grid3D, taylor_green3d

    g = Grid3D(N)
    xi, et, zt = taylor_green3d(N, 1234 + rank, amp=1e-3)
    comps = []
    for a in (xi, et, zt, np.zeros_like(xi)):
        t = torch.empty(g.nkt * 2, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = a.view(np.float64).ravel()
        comps.append(t.numpy().view(np.complex128).reshape(g.shape))
    calls = max(1, args.steps // STEPS_PER_CALL)
    wcalls = max(1, args.warmup // STEPS_PER_CALL)
    tend = STEPS_PER_CALL * DT
    per_call = rk4_evaluations(0.0, tend, DT)

    def call():
        lib.bous3d_inplace(comps, N, NU, DT, tend)

    for _ in range(wcalls):
        call()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(calls):
        call()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    if dist:
        t = torch.tensor([sec], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
    steps = calls * per_call
    # the drop-in moves the kept modes of in-place page-locked arrays whose other
    # entries are zero (the Taylor-Green state's are), the whole box otherwise
    m = g.mask()
    kept = ours and all(not np.any(c[~m]) for c in comps)
    nbytes = 4 * (int(m.sum()) if kept else g.nkt) * 16
    return {"value": round(world * steps / sec, 3), "unit": "steps/s",
            "h2d_bytes_per_step": int(nbytes / per_call) if ours else 0,
            "d2h_bytes_per_step": int(nbytes / per_call) if ours else 0,
            "steps_per_call": per_call, "calls": calls,
            "transfer": ("kept modes only, read and written in the page-locked host arrays by "
                         "the conversion kernels" if kept else "whole box"),
            "api": "timestep_cuda_ (3D Boussinesq ABI, Ri=0, FP64 host arrays)"}


def rk4_evaluations(tstart, tend, dt):
    """RK4 steps one Boussinesq call takes: full steps while tend - t > dt, then
    one adjusted step if t != tend (3D_Boussinesq/src/src_gmres/cuda.cu:187-250)."""
    t, n = tstart, 0
    while tend - t > dt:
        n += 1
        t += dt
    return n + (1 if t != tend else 0)


def cpu_baseline():
    """One RK4/CN step of the same workload on the host cores, FP64 oracle."""
    from oracle import pyoracle as O
    from psgpu_b200.fields import taylor_green3d

    xi, et, zt = taylor_green3d(N, 1234, amp=1e-3)
    t0 = time.perf_counter()
    O.bous3d_timestep(xi, et, zt, np.zeros_like(xi), N, NU, DT, 2 * DT)
    sec = time.perf_counter() - t0
    nsteps = rk4_evaluations(0.0, 2 * DT, DT)
    return {"value": round(nsteps / sec, 5), "unit": "steps/s", "cores": O.num_threads(),
            "kind": "port",
            "sample": f"{nsteps} RK4/CN steps of the 256^3 Taylor-Green workload, FP64, "
                      "Boussinesq scheme at Ri=0 (density carried), oracle C code"}


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank, world, dist):
    import torch
    from psgpu_b200.abi import TimestepLibrary

    path = os.path.join(ROOT, "oracle", "_ref", "libref_bous3d.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_bous3d.so not built"}
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lib = TimestepLibrary(path, "bous3d")
    clk = ClockSampler(dev.index)
    clk.start()
    clk.wait_first()
    with quiet_stdout():
        e2e = time_abi_calls(lib, args, dev, dist, world, rank, ours=False)
    clocks = clk.stop()
    if rank != 0:
        return None
    v = e2e["value"]
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * world / v, 4) if v else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "3D NS 256^3 Taylor-Green, RK4/CN (Boussinesq scheme, Ri=0), "
                               "nu=1/1600, dt=1e-3, 2/3 dealias",
                   "grid": N, "replicas": world, "parallelism": f"replicas{world}",
                   "implementation": "reference timestep_cuda_ (3D_Boussinesq/src/src_gmres/"
                                     "cuda.cu) built unmodified for sm_100a, FP64 cuFFT"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": None, "unit": "steps/s", "cores": 0, "kind": "reference",
                         "sample": "the reference has no host implementation of this step; "
                                   "this arm runs its CUDA step on the GPU, "
                                   f"{e2e['steps_per_call']} steps per call"},
        "clocks": clocks,
    }


# ------------------------------------------------------------ accuracy study
def run_accuracy(args):
    """FP32 against FP64 on the bench workload: energy / enstrophy / dissipation
    histories every step and the final vorticity after `args.accuracy` steps;
    with the reference build present, both are also compared with the
    reference's own FP64 step on the same initial state."""
    import torch
    import psgpu_b200 as P
    from psgpu_b200.abi import TimestepLibrary
    from psgpu_b200.fields import Grid3D, taylor_green3d

    torch.cuda.set_device(0)
    nsteps = args.accuracy
    xi, et, zt = taylor_green3d(N, 1234, amp=1e-3)
    hist = {}
    final = {}
    for prec in (64, 32):
        eng = P.NS3D(N, P.SCHEME_NS_RK4, precision=prec, nu=NU)
        eng.upload(xi, et, zt)
        h = np.zeros((nsteps + 1, 2))
        h[0] = eng.energetics()[:2]
        for s in range(nsteps):
            eng.step(DT, 1)
            h[s + 1] = eng.energetics()[:2]
        hist[prec] = h
        final[prec] = np.stack(eng.download())
        eng.close()

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    def rel2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    h32, h64 = hist[32], hist[64]
    out = {
        "mode": "accuracy", "workload": "3D NS 256^3 Taylor-Green + 1e-3 perturbation, RK4/CN, "
        "nu=1/1600, dt=1e-3", "steps": nsteps,
        "energy_def": "sum over kept modes |w|^2/k^2 (reference computeStats)",
        "enstrophy_def": "sum over kept modes |w|^2; dissipation = 2 nu * enstrophy",
        "fp32_vs_fp64": {
            "energy_max_rel": float(np.max(np.abs(h32[:, 0] - h64[:, 0]) / h64[:, 0])),
            "enstrophy_max_rel": float(np.max(np.abs(h32[:, 1] - h64[:, 1]) / h64[:, 1])),
            "dissipation_max_rel": float(np.max(np.abs(h32[:, 1] - h64[:, 1]) / h64[:, 1])),
            "vorticity_maxnorm_rel": rel(final[32], final[64]),
            "vorticity_l2_rel": rel2(final[32], final[64]),
        },
        "energy_start_end": [float(h64[0, 0]), float(h64[-1, 0])],
        "enstrophy_start_end": [float(h64[0, 1]), float(h64[-1, 1])],
    }
    # energy budget of the unforced truncated system, dE/dt = -2 nu Z (the
    # dealiased nonlinear term only moves energy between modes): per step, the
    # change of E against the trapezoid -nu dt (Z_n + Z_n+1), relative to the
    # change; over the run, E_end - E_0 against the sum of the trapezoids
    g = Grid3D(N)
    kx, ky, kz = g.wavenumbers()
    kmag = np.sqrt(kx * kx + ky * ky + kz * kz)

    def budget(h):
        dE = h[1:, 0] - h[:-1, 0]
        loss = NU * DT * (h[1:, 1] + h[:-1, 1])
        return {"per_step_max_rel": float(np.max(np.abs(dE + loss) / np.abs(dE))),
                "whole_run_rel": float(abs(dE.sum() + loss.sum()) / abs(dE.sum()))}

    def divergence(w):
        d = np.abs(kx * w[0] + ky * w[1] + kz * w[2])
        return float(d.max() / np.max(kmag * np.sqrt(np.sum(np.abs(w) ** 2, axis=0))))

    out["energy_budget"] = {"definition": "dE + nu dt (Z_n + Z_n+1) relative to dE, E = sum |w|^2/k^2, "
                                          "Z = sum |w|^2 over the kept modes",
                            "fp64": budget(h64), "fp32": budget(h32)}
    out["divergence"] = {"definition": "max |k . w| / max |k| |w| of the final state",
                         "fp64": divergence(final[64]), "fp32": divergence(final[32])}
    path = os.path.join(ROOT, "oracle", "_ref", "libref_bous3d.so")
    if os.path.exists(path) and not args.no_ref:
        lib = TimestepLibrary(path, "bous3d")
        comps = [a.copy() for a in (xi, et, zt, np.zeros_like(xi))]
        t0 = time.perf_counter()
        with quiet_stdout():
            lib.bous3d_inplace(comps, N, NU, DT, nsteps * DT)
        ref = np.stack(comps[:3])
        out["reference_fp64_seconds"] = round(time.perf_counter() - t0, 2)
        out["reference_steps"] = rk4_evaluations(0.0, nsteps * DT, DT)
        out["fp64_vs_reference"] = {"vorticity_maxnorm_rel": rel(final[64], ref),
                                    "vorticity_l2_rel": rel2(final[64], ref)}
        out["fp32_vs_reference"] = {"vorticity_maxnorm_rel": rel(final[32], ref),
                                    "vorticity_l2_rel": rel2(final[32], ref)}
    return out


# --------------------------------------------- gradient through a 3D trajectory
def run_adjoint(args):
    """Gradient of the terminal kinetic energy with respect to the divergence-free
    initial velocity, 3D Navier-Stokes 128^3 (seeded random field, shell
    spectrum ~ k^4 exp(-2 (k/4)^2), energy 0.5), nu = 1/400, dt = 5e-3, 400
    RK4/CN steps, checkpoints every 20 steps: time per gradient (FP32 and FP64
    engines), agreement of the FP64 adjoint with central differences on 16
    seeded directions, and of the FP32 gradient with the FP64 one."""
    import torch
    import psgpu_b200 as P
    from psgpu_b200.adjoint import Spectral3D, trajectory

    torch.cuda.set_device(0)
    n, nu, dt, steps, every = 128, 1.0 / 400.0, 5e-3, args.adjoint, 20
    sp = Spectral3D(n)
    u0 = sp.random_velocity(2024, energy=0.5)

    def loss(u, eng):
        return sp.energy(sp.velocity(trajectory(sp.curl(u), eng, dt, steps, every)))

    out = {"mode": "adjoint", "workload": f"3D NS {n}^3, nu=1/400, dt=5e-3, {steps} RK4/CN steps, "
           f"checkpoints every {every}; L = terminal mean kinetic energy; gradient w.r.t. u0"}
    grads = {}
    for prec in (64, 32):
        eng = P.NS3D(n, P.SCHEME_NS_RK4, precision=prec, nu=nu)
        u = u0.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L = loss(u, eng)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        L.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        grads[prec] = u.grad.detach().clone()
        out[f"fp{prec}"] = {"loss": float(L.detach()), "forward_s": round(t1 - t0, 3),
                            "backward_s": round(t2 - t1, 3),
                            "gradient_s": round(t2 - t0, 3)}
        if prec == 64:
            eng64 = eng
    g64 = grads[64]
    out["fp32_vs_fp64_gradient_maxnorm_rel"] = float((grads[32] - g64).abs().max() / g64.abs().max())
    eps = 1e-4
    errs, nerrs = [], []
    with torch.no_grad():
        for d in range(args.adjoint_dirs):
            v = sp.random_velocity(7000 + d, energy=1.0)
            lp = float(loss(u0 + eps * v, eng64))
            lm = float(loss(u0 - eps * v, eng64))
            fd = (lp - lm) / (2 * eps)
            ad = float((g64.real * v.real + g64.imag * v.imag).sum())
            errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
            scale = float(g64.abs().pow(2).sum().sqrt() * v.abs().pow(2).sum().sqrt())
            nerrs.append(abs(ad - fd) / scale)
    # Boussinesq variant: N = 1 (Ri = 1), Pr = 1 (Sc = 1), gravity along z
    rng = np.random.default_rng(2025)
    r0 = torch.tensor((rng.standard_normal(sp.grid.shape) + 1j * rng.standard_normal(sp.grid.shape))
                      * sp.grid.mask() * 1e-3, dtype=torch.complex128, device="cuda")
    beng = P.NS3D(n, P.SCHEME_BOUS_RK4, precision=64, nu=nu, ri=1.0, sc=1.0, theta=np.pi / 2)

    def bloss(u, r):
        s0 = torch.cat([sp.curl(u), r[None]], 0)
        return sp.energy(sp.velocity(trajectory(s0, beng, dt, steps, every)[:3]))

    u = u0.clone().requires_grad_(True)
    r = r0.clone().requires_grad_(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = bloss(u, r)
    L.backward()
    torch.cuda.synchronize()
    bsec = time.perf_counter() - t0
    berrs, bnerrs = [], []
    with torch.no_grad():
        for d in range(min(4, args.adjoint_dirs)):
            vu = sp.random_velocity(8000 + d, energy=1.0)
            vr = torch.tensor(np.random.default_rng(8100 + d).standard_normal(sp.grid.shape) *
                              sp.grid.mask() * 1e-2, dtype=torch.complex128, device="cuda")
            fd = (float(bloss(u0 + eps * vu, r0 + eps * vr)) -
                  float(bloss(u0 - eps * vu, r0 - eps * vr))) / (2 * eps)
            ad = float((u.grad.real * vu.real + u.grad.imag * vu.imag).sum() +
                       (r.grad.real * vr.real + r.grad.imag * vr.imag).sum())
            berrs.append(abs(ad - fd) / max(abs(fd), 1e-300))
            gn = float((u.grad.abs().pow(2).sum() + r.grad.abs().pow(2).sum()).sqrt())
            vn = float((vu.abs().pow(2).sum() + vr.abs().pow(2).sum()).sqrt())
            bnerrs.append(abs(ad - fd) / (gn * vn))
    out["boussinesq"] = {"workload": "Ri=1, Sc=1, gravity along z, rho0 seeded 1e-3; "
                                     "L = terminal kinetic energy; gradient w.r.t. (u0, rho0)",
                         "fp64_gradient_s": round(bsec, 3), "loss": float(L.detach()),
                         "fd_directions": len(berrs),
                         "fp64_adjoint_vs_central_fd_max_rel": float(max(berrs)) if berrs else None,
                         "fp64_adjoint_vs_central_fd_max_normalised":
                             float(max(bnerrs)) if bnerrs else None}
    out["fd_directions"] = args.adjoint_dirs
    out["fd_eps"] = eps
    out["fp64_adjoint_vs_central_fd_max_rel"] = float(max(errs)) if errs else None
    out["fp64_adjoint_vs_central_fd_median_rel"] = float(np.median(errs)) if errs else None
    out["fp64_adjoint_vs_central_fd_max_normalised"] = float(max(nerrs)) if nerrs else None
    out["normalisation"] = "rel: |<g,v> - fd| / |fd|; normalised: |<g,v> - fd| / (|g| |v|)"
    return out


# ------------------------------------------------------------ profiling cases
PROFILE_CASES = ("ns3d_rk4_fp32", "ns3d_rk4_fp64", "bous3d_fp32", "bous3d_fp64", "ns2d_batch",
                 "upo_tangent64", "upo_tangent32", "adjoint3d", "rec2d")


def run_profile_case(name, grid):
    """One small workload per hot-kernel family, for ncu captures (inputs larger
    than L2 where the family allows, a handful of launches after a warm-up):
    ns3d_rk4_* / bous3d_*: two RK4/CN steps at `grid`^3 (default 128) after one
    warm-up step; ns2d_batch: 148 instances of 128^2, 20 steps; upo_tangent*:
    one Newton step of 64 guesses at 128^2, T = 1, Krylov dimension 1;
    adjoint3d: one adjoint step at 64^3; rec2d: 60 checks of the 2D
    recurrence search over 64 runs at 128^2."""
    import torch
    import psgpu_b200 as P
    from psgpu_b200.fields import kolmogorov_ic2d, random_vorticity3d, taylor_green3d

    torch.cuda.set_device(0)
    n = grid or 128
    if name.startswith("ns3d_rk4") or name.startswith("bous3d"):
        prec = 64 if name.endswith("fp64") else 32
        bous = name.startswith("bous3d")
        xi, et, zt = taylor_green3d(n, 1234, amp=1e-3)
        eng = P.NS3D(n, P.SCHEME_BOUS_RK4 if bous else P.SCHEME_NS_RK4, precision=prec, nu=NU,
                     ri=1.0 if bous else 0.0)
        eng.upload(*((xi, et, zt, 0.01 * xi) if bous else (xi, et, zt)))
        eng.step(DT, 1)
        eng.sync()
        eng.step(DT, 2)
        eng.sync()
        eng.close()
    elif name == "ns2d_batch":
        b = P.Batch2D([128] * 148, precision=32)
        for i in range(148):
            b.upload(i, kolmogorov_ic2d(128, i))
        b.run(UPO_NU, UPO_DT, 2)
        b.sync()
        b.run(UPO_NU, UPO_DT, 20)
        b.sync()
        b.close()
    elif name.startswith("upo_tangent"):
        # one Newton step of 64 guesses (T = 1, 200 steps): the residual's Phi_T
        # launches, two dz/dt launches, then the Krylov products (base +
        # tangent) of the first GMRES iteration, each one to three launches
        prec = 32 if name.endswith("32") else 64
        G = 64
        u = P.UPO2D(G, 128, kmax=1, exact_jv=True, jv_precision=prec)
        for i in range(G):
            u.set_guess(i, kolmogorov_ic2d(128, i), T=1.0, nu=UPO_NU, dt=UPO_DT)
        u.solve(max_newton=1, tol=1e-10, gmres_tol=1e-3)
        u.close()
    elif name == "adjoint3d":
        nn = grid or 64
        eng = P.NS3D(nn, P.SCHEME_NS_RK4, precision=64, nu=1 / 400)
        xi, et, zt = random_vorticity3d(nn, 3, solenoidal=True)
        eng.upload(xi, et, zt)
        lam = torch.from_numpy(np.stack([xi, et, zt])).cuda()
        for _ in range(2):
            lam = eng.linear(eng.LIN_ADJOINT_STEP, lam, dt=5e-3)
        eng.sync()
        eng.close()
    elif name == "rec2d":
        G = 64
        b = P.Batch2D([128] * G, precision=32)
        for i in range(G):
            b.upload(i, kolmogorov_ic2d(128, i))
        rec = P.Recurrence2D(G, 128, 20, UPO_DT, 0.4, UPO_NU, store_size=201, norm_width=8,
                             nshift=(32, 4))
        rec.start(b)
        for k in range(1, 61):
            b.run(UPO_NU, UPO_DT, 20)
            rec.add(20 * k, b)
        b.sync()
        rec.close()
        b.close()
    else:
        raise SystemExit(f"unknown profile case {name}; one of {PROFILE_CASES}")
    torch.cuda.synchronize()
    return {"profile_case": name, "ok": True}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the C-ABI end-to-end leg")
    ap.add_argument("--grid", type=int, default=256,
                    help="grid size (256 is the benchmark; smaller grids are for profiling)")
    ap.add_argument("--no-upo", action="store_true", help="skip the UPO Newton leg")
    ap.add_argument("--upo-newton", type=int, default=3,
                    help="largest number of Newton iterations per guess in the UPO leg")
    ap.add_argument("--upo-converge", type=int, default=8, metavar="G",
                    help="also solve the G shortest-period guesses to convergence (0: skip)")
    ap.add_argument("--upo-converge-newton", type=int, default=12,
                    help="Newton iterations per guess of the to-convergence sub-leg")
    ap.add_argument("--upo-all-forms", action="store_true",
                    help="also solve with the FP64 exact tangent")
    ap.add_argument("--no-upo-plain", action="store_true",
                    help="skip the run of the reference's plain UPO form")
    ap.add_argument("--pass-table", action="store_true",
                    help="per-pass live timings and roofline fractions of the 3D engines, then exit")
    ap.add_argument("--profile-case", default="", choices=("",) + PROFILE_CASES,
                    help="run one small fixed workload of a kernel family (for ncu) and exit")
    ap.add_argument("--upo-only", action="store_true",
                    help="run the UPO leg alone and print its JSON")
    ap.add_argument("--accuracy", type=int, default=0, metavar="STEPS",
                    help="run the FP32-vs-FP64 accuracy study over STEPS steps instead")
    ap.add_argument("--adjoint", type=int, default=0, metavar="STEPS",
                    help="run the 128^3 gradient study over STEPS steps instead")
    ap.add_argument("--adjoint-dirs", type=int, default=16,
                    help="finite-difference directions of the gradient study")
    ap.add_argument("--ref2d-probe", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--grid2d", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 2D ensemble leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-engine leg")
    ap.add_argument("--no-ref", action="store_true",
                    help="accuracy study without the reference FP64 run")
    args = ap.parse_args()
    global N
    N = args.grid
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.ref2d_probe:
        print(json.dumps(run_ref2d_probe(args.ref2d_probe, args.grid2d or None)), flush=True)
        return
    if args.accuracy:
        if rank == 0:
            print(json.dumps(run_accuracy(args)), flush=True)
        return
    if args.adjoint:
        if rank == 0:
            print(json.dumps(run_adjoint(args)), flush=True)
        return
    if args.profile_case:
        print(json.dumps(run_profile_case(args.profile_case, args.grid if args.grid != 256 else 0)),
              flush=True)
        return
    if args.pass_table:
        if rank == 0:
            print(json.dumps(pass_table(args)), flush=True)
        return
    if args.upo_only:
        if rank == 0:
            import torch
            torch.cuda.set_device(0)
            print(json.dumps(run_upo(args)), flush=True)
        return
    if args.impl == "reference":
        # rank 0 alone times the reference; the other ranks exit without work
        if rank != 0:
            return
        out = run_reference(args, 0, 1, None)
        if out is not None:
            out["n_gpus"] = world
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        out = run_ours(args, rank, world, dist)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
