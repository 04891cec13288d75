#!/usr/bin/env python
"""Headline benchmark: 256^3 Swift-Hohenberg steps/s on one B200 (FP32 path,
with the FP64 path timed beside it), in the configuration the metric is quoted
on: the Neumann (REDFT10/REDFT01) solver of cosNoAdvMorph at 256^3,
eps=-0.75, beta=2, gamma=1, q0=1, dx=2 pi/8, dt=0.05, hyperboloid initial
condition 0.5 cos(q0 s) + 1e-3 U(-1,1) (seeded synthetic input).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload neumann256|periodic256|periodic128|batch64]

A step is one time step of every domain the job integrates.  With N GPUs each
rank integrates its own domain (replicas only: the path does not shard), and
``value`` is the total steps of all ranks divided by the slowest rank's
device time.  One JSON line is printed by rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256³ SH steps/s: FP32 vs FP64 GPU @ψ rel err≤1e-5; adjoint/forward time ratio"
L2_BYTES = 126 * 2 ** 20

WORKLOADS = {
    # name: (boundary, n, batch, precision, ic)
    "neumann256": ("neumann", 256, 1, "fp32", "hyperboloid"),
    "periodic256": ("periodic", 256, 1, "fp32", "noise"),
    "periodic128": ("periodic", 128, 1, "fp64", "noise"),
    "batch64": ("periodic", 64, 64, "fp32", "noise"),
}


def make_ic(kind, n, batch, dx, seed=0):
    from smectic3d_b200 import ic
    if kind == "hyperboloid":
        a = ic.hyperboloid(n, dx, seed=seed)
    else:
        a = ic.noise(n, seed) if batch == 1 else ic.noise_batch(n, range(seed, seed + batch))
    return a


def params_for(workload, precision=None):
    import numpy as np
    import smectic3d_b200 as S
    bnd, n, batch, prec, _ = WORKLOADS[workload]
    kw = {}
    if batch > 1:
        kw["eps_per_replica"] = tuple(np.linspace(-0.9, -0.5, batch))
    return S.Params(n=n, batch=batch, boundary=bnd, precision=precision or prec, dt=0.05, eps=-0.75, **kw)


def workload_label(workload):
    bnd, n, batch, _, ick = WORKLOADS[workload]
    return f"{workload}: {bnd} {n}^3 x{batch}, {ick} IC, dt=0.05, eps=-0.75, beta=2, gamma=1, q0=1, dx=2pi/8"


def algorithmic_bytes(boundary, n, batch, precision):
    """Bytes one launch of each pass must move (read its inputs once, write
    its outputs once): pencil reads N-partial + W, writes W + psi-partial;
    plane reads the psi-partial, writes the N-partial."""
    s = 4 if precision == "fp32" else 8
    if boundary == "periodic":
        field = 2 * s * n * n * (n // 2 + 1)     # H: half spectrum
    else:
        field = s * n ** 3                        # R: real field
    return {"pencil": 4 * field * batch, "plane": 2 * field * batch, "field": field * batch}


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and throttle reasons sampled every 10 ms by an NVML thread
    while the timed region runs (read-only NVML queries); the GPU is found
    by its UUID so CUDA_VISIBLE_DEVICES remapping does not matter."""
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, cuda_index, period=0.01):
        import threading
        self.cuda_index = cuda_index
        self.period = period
        self.samples = []          # (t, sm_mhz, reasons bitmask)
        self.window = None
        self.smax = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _run(self, nv, h):
        get_r = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.samples.append((time.perf_counter(), nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), get_r(h)))
            except Exception:
                pass
            self._stop.wait(self.period)

    def start(self):
        import threading
        try:
            nv, h = self._handle()
            self.smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            return
        self._nvml = nv
        self._thread = threading.Thread(target=self._run, args=(nv, h), daemon=True)
        self._thread.start()
        t0 = time.perf_counter()
        while not self.samples and time.perf_counter() - t0 < 2.0:
            time.sleep(0.002)

    def begin(self):
        self.window = [time.perf_counter(), None]

    def end(self):
        if self.window:
            self.window[1] = time.perf_counter()

    def stop(self):
        if self._thread is None:
            return None
        self._stop.set()
        self._thread.join(timeout=2)
        lo, hi = self.window if self.window and self.window[1] else (-math.inf, math.inf)
        rows = [s for s in self.samples if lo <= s[0] <= hi]
        if not rows:   # region shorter than the period: the samples either side
            before = [s for s in self.samples if s[0] < lo][-1:]
            after = [s for s in self.samples if s[0] > hi][:1]
            rows = before + after
        if not rows:
            return None
        reasons = sorted({k for _, _, m in rows for k, bit in self.REASONS.items() if m & bit})
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": self.smax, "reasons": reasons,
                "samples": len(rows), "source": "nvml, 10 ms"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_record(kernel_key):
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    return json.load(open(path)).get(kernel_key)


def max_over_ranks(x, torch, dist, device="cuda"):
    """Largest value of x over all ranks (the job time is the slowest rank's)."""
    if dist is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, ms_per_rank, torch, dist, device="cuda"):
    """Whole-job throughput: units of every rank over the slowest rank's time."""
    world = dist.get_world_size() if dist is not None else 1
    ms = max_over_ranks(ms_per_rank, torch, dist, device)
    return world * units_per_rank / (ms / 1e3), ms


def timed_steps(solver, k, torch, dist, clocks=None):
    ext = torch.cuda.ExternalStream(solver.stream)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    solver.synchronize()
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.begin()
    start.record(ext)
    solver.step_async(k)
    end.record(ext)
    end.synchronize()
    if clocks is not None:
        clocks.end()
    solver.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    return max_over_ranks(start.elapsed_time(end), torch, dist)


def rank_inputs(workload, rank):
    """Parameters and initial state of one rank: every rank integrates its own
    domain (replicas only), seeded by its rank."""
    _, n, batch, _, ick = WORKLOADS[workload]
    p = params_for(workload)
    return p, make_ic(ick, n, batch, p.dx, seed=rank)


def run_ours(args, rank, world, local_rank, dist):
    import numpy as np
    import torch

    import smectic3d_b200 as S

    torch.cuda.set_device(local_rank)
    bnd, n, batch, prec, ick = WORKLOADS[args.workload]
    p32, psi0 = rank_inputs(args.workload, rank)
    k, w = args.steps, args.warmup

    # ---- device-resident timing of the headline precision -----------------
    s32 = S.Solver(p32)
    s32.set_psi(psi0)
    s32.step(w)
    s32.prepare()  # the replayed step graph is instantiated before the timed region
    l0 = s32.kernel_launches
    clocks = ClockSampler(local_rank)
    clocks.start()
    ms = timed_steps(s32, k, torch, dist, clocks)
    clk = clocks.stop()
    launches = s32.kernel_launches - l0
    value = world * k / (ms / 1e3)

    # ---- the other precision (ratio and accuracy of the FP32 path) ---------
    other = "fp64" if prec == "fp32" else "fp32"
    s64 = S.Solver(params_for(args.workload, other))
    s64.set_psi(psi0)
    s64.step(w)
    s64.prepare()
    ms64 = timed_steps(s64, k, torch, dist)
    a32 = s32.get_psi()
    a64 = s64.get_psi()
    rel_err = float(np.linalg.norm(a32 - a64) / max(np.linalg.norm(a64 if prec == "fp32" else a32), 1e-300))
    s64.close()
    # FP32 fields with the CNAB2 update in FP64 (the long-run option)
    u64 = None
    if prec == "fp32":
        su = S.Solver(params_for(args.workload, "fp32_u64"))
        su.set_psi(psi0)
        su.step(w)
        su.prepare()
        msu = timed_steps(su, k, torch, dist)
        au = su.get_psi()
        su.close()
        u64 = {"precision": "fp32_u64", "value": world * k / (msu / 1e3), "ms_per_step": msu / k,
               "rel_err_vs_fp64": float(np.linalg.norm(au - a64) / np.linalg.norm(a64)), "after_steps": w + k}

    # ---- accuracy of the FP32 path after 100 steps (the 1e-5 accuracy bound),
    # on the workload's IC and on the non-decaying reference-amplitude lamellae
    acc100, energy_rel = {}, {}
    for label, ic0 in (("workload_ic", psi0),
                       ("lamellae_amp1.3", S.ic.undulated_lamellae(n, p32.dx, amp=1.3, seed=rank)
                        if batch == 1 else None)):
        if ic0 is None:
            continue
        outs, ens = {}, {}
        for pr in ("fp32", "fp64"):
            with S.Solver(params_for(args.workload, pr)) as sv:
                sv.set_psi(ic0)
                sv.step(100)
                outs[pr] = sv.get_psi()
                ens[pr] = np.asarray(sv.energy(), dtype=np.float64)
        acc100[label] = float(np.linalg.norm(outs["fp32"] - outs["fp64"]) / np.linalg.norm(outs["fp64"]))
        # energy of the FP32 state (FP64 sums) against the FP64 state's
        energy_rel[label] = float(np.max(np.abs(ens["fp32"] - ens["fp64"]) / np.abs(ens["fp64"])))

    # ---- per-pass device times (roofline of the dominant kernel) -----------
    nprof = max(10, min(200, k // 10))
    ms_pencil, ms_plane = s32.profile_steps(nprof)
    residency = s32.residency()
    s32.close()
    ab = algorithmic_bytes(bnd, n, batch, prec)
    per = {"pencil": ms_pencil / nprof, "plane": ms_plane / nprof}
    dom = max(per, key=per.get)
    peak, peak_kind = peaks()
    achieved = ab[dom] / (per[dom] / 1e3) / 1e9
    tr = traffic_record(f"{dom}/{args.workload}/{prec}")

    # ---- end to end through the public API with host buffers ---------------
    pe = params_for(args.workload)
    pe.l1_interval = 100
    se = S.Solver(pe)
    nbytes = psi0.size * 8
    hp_in, hp_out = C.c_void_p(), C.c_void_p()
    S.load_library().sh_host_alloc(nbytes, C.byref(hp_in))
    S.load_library().sh_host_alloc(nbytes, C.byref(hp_out))
    host_in = np.ctypeslib.as_array((C.c_double * psi0.size).from_address(hp_in.value)).reshape(psi0.shape)
    host_out = np.ctypeslib.as_array((C.c_double * psi0.size).from_address(hp_out.value)).reshape(psi0.shape)
    host_in[...] = psi0
    se.run(host_in, w, host_out)  # warm
    se.prepare()  # the step graph (replayed between the L1 monitor's steps) is instantiated before timing
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    se.run(host_in, k, host_out)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0, torch, dist)
    se.close()
    S.load_library().sh_host_free(hp_in)
    S.load_library().sh_host_free(hp_out)
    e2e = {"value": world * k / e2e_s, "unit": "steps/s",
           "h2d_bytes_per_step": nbytes / k, "d2h_bytes_per_step": (nbytes + 8 * batch * (k // 100) + 4) / k,
           "api": "smectic3d_b200.Solver.run -> sh_run (pinned host psi in, K steps with the L1 monitor every 100, psi out)"}

    adj = adjoint_ratio(args, torch) if args.adjoint_steps > 0 else None
    others = other_configs(torch) if (world == 1 and args.other_configs) else None
    comparator = cufft_comparator(torch) if (world == 1 and args.other_configs) else None

    if rank != 0:
        return None
    cpu = cpu_baseline(args.workload, budget_s=args.cpu_seconds) if world == 1 else None
    field_mb = ab["field"] / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": k, "warmup": w,
        "ms_per_step": ms / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if prec == "fp32" else "f64", "data": "synthetic",
        "config": bench_config(args),
        "precision": prec, "parallelism": f"replicas x{world}",
        "l2": f"inputs larger than L2: working set {3 * field_mb:.0f} MB > 126 MB, no flush",
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": ab[dom], "avg_launch_ms": per[dom],
                     "traffic": (tr["bytes_per_launch"] if tr else None),
                     "step_frac": (ab["pencil"] + ab["plane"]) / (ms / k / 1e3) / 1e9 / peak,
                     "pass_ms": per, "residency": residency},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk,
        "other_precision": {"precision": other, "value": world * k / (ms64 / 1e3), "ms_per_step": ms64 / k,
                            "speedup_fp32_over_fp64": (ms64 / ms) if prec == "fp32" else (ms / ms64),
                            "rel_err_fp32_vs_fp64": rel_err, "after_steps": w + k,
                            "rel_err_fp32_vs_fp64_after_100_steps": acc100,
                            "energy_rel_err_fp32_vs_fp64_after_100_steps": energy_rel},
        "fp32_fp64_update": u64,
        "adjoint_forward_ratio": adj["backward_over_forward"] if adj else None,
        "adjoint": adj,
        "other_configs": others,
        "cufft_comparator": comparator,
    }
    return line


def adjoint_ratio(args, torch):
    """Differentiation workload: 128^3 periodic, FP32 forward, FP64 gradient
    accumulation, dt=0.05, checkpoints every 50 steps, L = 1/2 ||psi_T - target||^2
    with target 0.5 cos(1.05 z), psi0 = 1.328 cos(z) + U(-0.1, 0.1).  Device-timed
    (CUDA events on the solver's stream): T plain forward steps; the forward sweep
    that keeps the checkpoints (sh_adjoint_forward, what the autograd forward runs);
    the backward sweep (sh_adjoint_backward: recompute from the checkpoints and the
    reverse steps).  total_over_forward = (forward sweep + backward) / plain forward,
    the cost of forward plus backward through torch.autograd."""
    import numpy as np
    import smectic3d_b200 as S
    n, k = 128, 50
    t_steps = args.adjoint_steps
    p = S.Params(n=n, precision="fp32", dt=0.05, eps=-0.75)
    # lamellae of the reference amplitude along z, slightly off the target wavenumber, plus noise
    z = np.arange(n) * p.dx
    psi0 = 1.328 * np.cos(z)[None, None, :] + S.ic.noise(n, 0)
    target = 0.5 * np.broadcast_to(np.cos(1.05 * np.arange(n) * p.dx)[None, None, :], (n, n, n))
    with S.Solver(p) as s:
        ext = torch.cuda.ExternalStream(s.stream)

        def timed(fn):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.synchronize()
            e0.record(ext)
            fn()
            e1.record(ext)
            e1.synchronize()
            return e0.elapsed_time(e1)

        s.set_psi(psi0)
        s.step(5)
        s.prepare()
        s.set_psi(psi0)
        t_fwd = timed(lambda: s.step_async(t_steps))
        lam = s.get_psi() - target
        s.adjoint_forward(psi0, t_steps, k)  # warm: kernels and the adjoint's buffers
        s.adjoint_backward(lam)
        t_fck = timed(lambda: s.adjoint_forward(psi0, t_steps, k))
        out = {}
        t_bwd = timed(lambda: out.update(g=s.adjoint_backward(lam)))
        ge, gq, _ = out["g"]
        # one segment of T steps: the forward sweep keeps every state (2 fields per
        # step in HBM, 17 GB at 128^3 FP32, T = 1000) and the backward recomputes nothing
        s.adjoint_forward(psi0, t_steps, t_steps)
        s.adjoint_backward(lam)
        t_fall = timed(lambda: s.adjoint_forward(psi0, t_steps, t_steps))
        t_ball = timed(lambda: out.update(g2=s.adjoint_backward(lam)))
    return {"workload": f"periodic {n}^3 fp32, dt=0.05, T={t_steps}, checkpoints every {k}",
            "timing": "CUDA events on the solver stream",
            "forward_ms_per_step": t_fwd / t_steps, "forward_with_checkpoints_ms_per_step": t_fck / t_steps,
            "backward_ms_per_step": t_bwd / t_steps,
            "backward_over_forward": t_bwd / t_fwd, "total_over_forward": (t_fck + t_bwd) / t_fwd,
            "all_states_kept": {"ckpt_every": t_steps, "backward_over_forward": t_ball / t_fwd,
                                "total_over_forward": (t_fall + t_ball) / t_fwd,
                                # the checkpointed run takes each segment's first state through an
                                # extra transform: the gradients agree to FP32 rounding
                                "grad_rel_diff": max(abs(out["g2"][0][0] - ge[0]) / abs(ge[0]),
                                                     abs(out["g2"][1][0] - gq[0]) / abs(gq[0]))},
            "grad_eps": float(ge[0]), "grad_q0": float(gq[0])}


def other_configs(torch, steps=200):
    """Device-timed steps/s of the other synthetic configurations (seeded inputs):
    C1 periodic 128^3 FP64; C3 periodic 256^3 FP32 with Stokes advection, dt=0.02,
    undulated lamellae, the surfTrack pass every 10 steps (host-timed, since each
    pass returns its surface to the host); C4 64 replicas x 64^3 FP32 with
    eps_r = linspace(-0.9, -0.5, 64).  Each reports steps/s and the HBM roofline
    fraction of its algorithmic bytes per step, counting every transform's input
    read and output written once: periodic 2R + 4H, advected 8R + 12H."""
    import numpy as np
    import smectic3d_b200 as S
    peak, _ = peaks()
    out = {}

    def model_bytes(n, batch, prec, advect):
        s_ = 4 if prec == "fp32" else 8
        r_, h_ = s_ * n ** 3, 2 * s_ * n * n * (n // 2 + 1)
        return batch * ((8 * r_ + 12 * h_) if advect else (2 * r_ + 4 * h_))

    # C1 and C4: plain steps, CUDA events on the solver stream
    for name, p, psi in (
            ("C1 periodic 128^3 fp64", S.Params(n=128, precision="fp64", dt=0.05, eps=-0.75), S.ic.noise(128, 0)),
            ("C4 64 x 64^3 fp32", S.Params(n=64, batch=64, precision="fp32", dt=0.05, eps=-0.75,
                                           eps_per_replica=tuple(np.linspace(-0.9, -0.5, 64))),
             S.ic.noise_batch(64, range(64)))):
        with S.Solver(p) as s:
            s.set_psi(psi)
            s.step(10)
            s.prepare()
            ms = timed_steps(s, steps, torch, None)
        rate = steps / (ms / 1e3)
        b = model_bytes(p.n, p.batch, p.precision, False)
        out[name] = {"steps_per_s": rate, "us_per_step": 1e3 * ms / steps,
                     "roofline_frac": b * rate / (peak * 1e9)}
    # C3: advected, surfTrack every 10 steps
    n = 256
    p = S.Params(n=n, precision="fp32", dt=0.02, eps=-0.75, advection=True)
    with S.Solver(p) as s:
        s.set_psi(S.ic.undulated_lamellae(n, p.dx, seed=0))
        s.step(3)
        s.surface_step()  # the first surface pass allocates its buffers: set-up, not timed
        s.synchronize()
        nblk = max(1, steps // 20)
        t0 = time.perf_counter()
        found = 0
        for _ in range(nblk):
            z, _vn, _hh, _kk = s.surface_step()
            found = int((z >= 0).sum())
            s.step(9)
        s.synchronize()
        t1 = time.perf_counter()
        rate = 10 * nblk / (t1 - t0)
        s.step(3)
        s.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ext = torch.cuda.ExternalStream(s.stream)
        ev0.record(ext)
        s.step_async(20)
        ev1.record(ext)
        ev1.synchronize()
        plain = 20 / (ev0.elapsed_time(ev1) / 1e3)
    b = model_bytes(n, 1, "fp32", True)
    out["C3 advected 256^3 fp32 + surfTrack/10"] = {
        "steps_per_s": rate, "us_per_step": 1e6 / rate, "steps_per_s_without_surface": plain,
        "roofline_frac": b * plain / (peak * 1e9), "surface_columns_found": found,
        "timing": "host clock around 10-step blocks (each surface pass returns to the host)"}
    return out


def cufft_comparator(torch, steps=100):
    """Context only: the plain periodic CNAB2 step at 256^3 FP32 written with
    torch.fft (cuFFT) and elementwise torch ops, unfused, beside this library's
    own periodic 256^3 FP32 step.  Same algorithm (W-state CNAB2, quintic N);
    both timed with CUDA events over ``steps`` steps."""
    import numpy as np
    import smectic3d_b200 as S
    n, dt, eps, beta, gamma = 256, 0.05, -0.75, 2.0, 1.0
    p = S.Params(n=n, precision="fp32", dt=dt, eps=eps)
    dev = torch.device("cuda")
    k = torch.fft.fftfreq(n, d=p.dx / (2 * np.pi), device=dev, dtype=torch.float32)
    kz = torch.fft.rfftfreq(n, d=p.dx / (2 * np.pi), device=dev, dtype=torch.float32)
    q2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    a_lin = eps - (q2 - 1.0) ** 2
    c1, inv_c2 = 1 + 0.5 * dt * a_lin, 1.0 / (1 - 0.5 * dt * a_lin)
    psi = torch.tensor(S.ic.noise(n, 0), dtype=torch.float32, device=dev)
    nl = lambda x: beta * x ** 3 - gamma * x ** 5
    w = c1 * torch.fft.rfftn(psi) - 0.5 * dt * torch.fft.rfftn(nl(psi))

    def step(psi, w):
        nh = torch.fft.rfftn(nl(psi))
        ph = (w + 1.5 * dt * nh) * inv_c2
        return torch.fft.irfftn(ph, s=(n, n, n)), c1 * ph - 0.5 * dt * nh

    for _ in range(5):
        psi, w = step(psi, w)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        psi, w = step(psi, w)
    e1.record()
    e1.synchronize()
    torch_rate = steps / (e0.elapsed_time(e1) / 1e3)
    with S.Solver(p) as s:
        s.set_psi(S.ic.noise(n, 0))
        s.step(10)
        s.prepare()
        ours = steps / (timed_steps(s, steps, torch, None) / 1e3)
    return {"what": "plain periodic CNAB2 step, 256^3 FP32: torch.fft (cuFFT) + torch elementwise, unfused, "
                    "against this library's fused passes",
            "torch_fft_steps_per_s": torch_rate, "ours_steps_per_s": ours, "ours_over_torch_fft": ours / torch_rate}


# ---------------------------------------------------------------------------
# CPU legs: the oracle port (the reference itself needs FFTW-MPI + MPI)
# ---------------------------------------------------------------------------
def _oracle_solver(workload):
    from oracle import sh_oracle as O
    bnd, n, batch, _, ick = WORKLOADS[workload]
    p = params_for(workload)
    op = O.Params(n=n, dx=p.dx, dt=p.dt, eps=p.eps, beta=p.beta, gamma=p.gamma, alpha=p.alpha, q0=p.q0)
    psi0 = make_ic(ick, n, 1, p.dx)
    cls = O.PeriodicOracle if bnd == "periodic" else O.NeumannOracle
    return cls(psi0, op), batch


def cpu_baseline(workload, budget_s=20.0, max_steps=None):
    orc, batch = _oracle_solver(workload)
    orc.step()  # warm
    t0 = time.perf_counter()
    steps = 0
    while True:
        orc.step()
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps and steps >= max_steps):
            break
    n = orc.n
    # a step of the workload advances all `batch` domains: one oracle domain-step is 1/batch of it
    return {"value": steps / el / batch, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{steps} oracle steps of one {n}^3 FP64 domain (SciPy pocketfft, workers={os.cpu_count()}) "
                      f"in {el:.1f} s" + (f", scaled by 1/{batch} domains" if batch > 1 else "")}


def run_reference(args, rank, budget_s=180.0):
    """The reference arm: the oracle port (the reference itself needs FFTW-MPI
    + MPI, absent here) on all host cores, W untimed warm-up steps, then K
    timed steps, or as many as fit ``budget_s`` when K steps would not."""
    if rank != 0:
        return None
    w = args.warmup
    orc, batch = _oracle_solver(args.workload)
    t0 = time.perf_counter()
    for _ in range(w):
        orc.step()
    per_step = (time.perf_counter() - t0) / max(w, 1)
    k = args.steps if per_step * args.steps <= budget_s else max(1, int(budget_s / per_step))
    t0 = time.perf_counter()
    for _ in range(k):
        orc.step()
    el = time.perf_counter() - t0
    v = k / el / batch
    bnd, n, _, prec, _ = WORKLOADS[args.workload]
    sample = (f"{k} timed steps after {w} warm-up steps of one {n}^3 FP64 domain, oracle port on SciPy pocketfft "
              f"with workers={os.cpu_count()}")
    if k < args.steps:
        sample += f" ({args.steps} requested; {k} fit the {budget_s:.0f} s budget)"
    sample += "; the reference needs FFTW-MPI + MPI, absent here"
    cb = {"value": v, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port", "sample": sample}
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": k,
            "warmup": w, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": bench_config(args), "precision": "fp64 (CPU oracle port)",
            "parallelism": f"{os.cpu_count()} host threads",
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}


def bench_config(args) -> dict:
    """The workload both arms measure (the same dict in the GPU line and the reference line)."""
    return {"workload": workload_label(args.workload)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="neumann256", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--adjoint-steps", type=int, default=1000, help="steps of the adjoint ratio (0 = skip)")
    ap.add_argument("--no-other-configs", dest="other_configs", action="store_false",
                    help="skip the C1 / C3 / C4 measurements reported beside the headline")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(local_rank)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    try:
        line = run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
