#!/usr/bin/env python
"""Throughput of the conserved semi-implicit PFC step on B200.

Workload: 3D PFC on a 512^3 grid in FP32 -- random liquid psi0 = -0.18 +
U(-0.05, 0.05) (numpy PCG64, seed 2024 + rank), eps = 0.3, dt = 0.25, dx = pi/4, no
noise -- the grid and precision the headline metric is quoted on.  A step is one
conserved semi-implicit step of the whole field (inverse FFT, cubic term, forward
FFT, propagator).  The 539 MB state is larger than L2 (126 MB), so no L2 flush is
needed between steps.

Arms
  default            this library's fused stepper (pfc_step through the C ABI)
  --impl reference   the reference's own stock cuFFT step (copy, C2R, psi3_split,
                     R2C, update_eom; cuda/kernels/eom.hpp etc.), compiled from the
                     reference sources into oracle/_ref by oracle/Makefile

Multi-GPU (torchrun, one process per GPU): every rank advances its own field
(replicas only, no data-path collective); timing is the max over ranks and `value`
counts the steps of all ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mcstar-libs_b200"))

import numpy as np  # noqa: E402
import torch  # noqa: E402

WL = dict(nx=512, ny=512, nz=512, dx=math.pi / 4, dt=0.25, eps=0.3, psi0=-0.18, amp=0.05, seed=2024)
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=512, help="grid side (the headline workload is 512)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="pfc512", choices=["pfc512", "ensemble", "lowpass", "peaks"],
                    help="pfc512: the headline 512^3 field (default); ensemble: 64 mixed-size replicas; "
                         "lowpass: the 2D amplitude low-pass with its LOWPASS dump (4096^2 unless --size); "
                         "peaks: peak finding and bond order on the headline field after 200 steps")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples (200 ms) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [ln.split(",") for ln in open(self.path).read().splitlines() if ln.strip()]
        os.unlink(self.path)
        mhz, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [v.strip() for v in r]
            try:
                mhz.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except (ValueError, IndexError):
                continue
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        if not mhz:
            return None
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(mhz)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel, size):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(p))
        e = d[kernel]
        return float(e["dram_bytes_per_launch"]) * (size / float(e.get("size", size))) ** 3
    except (OSError, KeyError, ValueError):
        return None


X_KERNELS = {0: "k_xrow", 1: "k_xpair", 2: "k_xlane"}


def kernel_table(prof, S, steps, x_kernel=0, y_kernel=0):
    """Per-kernel device time of the timed region (the library's CUDA-event brackets on
    its stream) with the algorithmic HBM bytes of one launch, S = bytes of one
    half-spectrum field: every pass reads each input field once and writes each output
    field once."""
    t = {}

    def add(name, fam, bytes_per_launch):
        calls = prof["calls"][fam]
        if calls:
            t[name] = {"ms_total": prof["ms"][fam], "launches": calls, "ms_per_launch": prof["ms"][fam] / calls,
                       "bytes_per_launch": bytes_per_launch}

    if prof["xy_mode"] == 2 and prof["calls"][3]:
        # y-inverse and y-forward between the tiled layouts (the TMA kernel k_ybulk, or
        # k_ycol3); the last step's y-forward into the standard layout is k_ycol3
        y3 = prof.get("y_variant") in (6, 7, 8)
        add(("k_ybulk" if y_kernel == 1 else "k_ycol3") if y3 else "k_ycol", 3, 2.0 * S)
        add(X_KERNELS.get(x_kernel, "k_xrow"), 4, 2.0 * S)  # C2R, cubic term, R2C of every row, in place
    elif prof["xy_mode"] == 2:
        add("k_ycol+k_xrow+k_ycol (z slabs)", 1, 6.0 * S)
    elif prof["xy_mode"] == 1:
        add("k_plane_xy", 1, 2.0 * S)
    else:
        add("k_cols+k_rows_nonlin+k_cols", 1, 6.0 * S)
    if prof["z_mode"] in (2, 4, 5):
        # psi^ and B read, psi^' and A' written; the last step of a run writes psi^' only
        name = {4: "k_zbulk", 2: "k_zcarry", 5: "k_zprop (psi^ carried)"}[prof["z_mode"]]
        add(name, 2, (4.0 * (steps - 1) + 3.0) / steps * S)
    else:
        name = "k_zprop" if prof["z_mode"] == 0 else ("k_zcol3" if prof.get("z_variant") == 6 else "k_zcol")
        add(name, 2, 3.0 * S)
    return t


def initial_field(shape, seed):
    from mcstar_b200 import liquid_random
    return liquid_random(shape, WL["psi0"], WL["amp"], seed)


def cpu_baseline(n, steps_budget_s=20.0):
    """The oracle (numpy/scipy restatement of the reference's step) in FP32 on the host
    cores, a bounded number of steps of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pfc_oracle as O
    cores = len(os.sched_getaffinity(0))
    shape = (n, n, n)
    psi = initial_field(shape, WL["seed"]).astype(np.float32)
    lens = tuple(v * WL["dx"] for v in shape)
    k = O.r2c(psi, workers=cores)
    t0 = time.perf_counter()
    k = O.step(k, 1, WL["dt"], WL["eps"], lens, shape, workers=cores, dtype=np.float32)
    t1 = time.perf_counter()
    extra = int(max(0, min(4, steps_budget_s / max(t1 - t0, 1e-3) - 1)))
    if extra:
        k = O.step(k, extra, WL["dt"], WL["eps"], lens, shape, workers=cores, dtype=np.float32)
    t2 = time.perf_counter()
    nsteps = 1 + extra
    return {"value": nsteps / (t2 - t0), "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{nsteps} step(s) of the {n}^3 fp32 workload, oracle/pfc_oracle.py with scipy.fft "
                      f"workers={cores}"}


# ---------------------------------------------------------------------------------------
def dist_setup(args):
    from mcstar_b200 import dist
    ws, rank, local = dist.env_world()
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if ws > 1:
        dist.init("nccl", timeout_s=300)
    return ws, rank, local


def barrier(ws):
    from mcstar_b200 import dist
    dist.barrier(ws)


def max_over_ranks(ws, v):
    from mcstar_b200 import dist
    return dist.reduce_scalars(ws, [v], "max")[0]


def run_ensemble(args, ws, rank, local):
    """The batched workload: 48 2D + 16 3D FP32 fields of mixed sizes, eps, psi0, seeds,
    noise T = 1e-3, one graph launch per step on each GPU (members dealt out by cost);
    against the same members stepped one at a time through pfc_step."""
    from mcstar_b200 import Ensemble, Stepper, ensemble_members, partition
    members = ensemble_members(seed=4)
    mine = partition(members, ws)[rank]
    ens = Ensemble([members[i] for i in mine], steps_per_graph=1)
    ens.run(args.warmup)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    e0.record()
    ens.run(args.steps)
    e1.record()
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    ms = max_over_ranks(ws, e0.elapsed_time(e1))
    cells = sum(int(np.prod(m["shape"])) for m in members)
    value = cells * args.steps / (ms / 1e3) / 1e9
    out = {
        "metric": "ensemble Gcell-upd/s (48 2D + 16 3D mixed-size fp32 replicas, one graph launch per step)",
        "value": round(value, 2), "unit": "Gcell-upd/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic: seeded random liquids (numpy PCG64)",
        "config": {"workload": "ensemble of 64 replicas", "members": len(members), "members_this_rank": len(mine),
                   "steps_per_graph": 1, "noise_T": 1e-3, "parallelism": f"members dealt by cost over {ws} GPU(s)"},
        "clocks": clk,
    }
    if ws == 1:
        # the same members one after another, each through pfc_step
        seq_ms = 0.0
        for m in members:
            st = Stepper(m["shape"], m["dx"], m["dt"], m["eps"], dtype=np.float32, namp=m["namp"], seed=m["seed"])
            st.set_real(initial_field(m["shape"], m["seed"]))
            st.step(2)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            st.step(args.steps)
            b.record()
            torch.cuda.synchronize()
            seq_ms += a.elapsed_time(b)
        out["sequential"] = {"value": round(cells * args.steps / (seq_ms / 1e3) / 1e9, 2), "unit": "Gcell-upd/s",
                             "ms_per_step": round(seq_ms / args.steps, 4)}
    return out


LP = dict(n=4096, dx=0.8, dps=2.0, seed=11)


def run_lowpass(args, ws, rank, local):
    """The 2D amplitude low-pass (calc_amplitude_lowpass: high-pass, square, low-pass, the
    gzip LOWPASS dump, amplitude) on an n^2 FP32 field, n = 4096 unless --size is given;
    each call restores the input spectrum first (one device copy).  N GPUs run replicas."""
    from mcstar_b200 import get_context
    n = LP["n"] if args.size == 512 else args.size
    shape = (n, n, 1)
    lens, hh = (n * LP["dx"], n * LP["dx"], 1.0), (LP["dx"], LP["dx"], 1.0)
    ctx = get_context(shape, np.float32)
    x = np.arange(n) * LP["dx"]
    psi = (0.3 * np.cos(2 * math.pi * (n // 8) / lens[0] * x)[None, :] +
           0.05 * np.random.default_rng(LP["seed"]).standard_normal((n, n))).astype(np.float32)
    real = ctx.empty_state()
    real[: n * n].copy_(torch.from_numpy(psi.ravel()))
    spec0, spec, aux, g = ctx.empty_state(), ctx.empty_state(), ctx.empty_state(), ctx.empty_state()
    ctx.r2c(real, spec0)
    ctx.gaussian_init(g, lens, hh, LP["dps"])
    path = os.path.join(tempfile.mkdtemp(prefix="lowpass_"), f"rank{rank}.gz")

    def call(dump):
        spec.copy_(spec0)
        ctx.amplitude_lowpass(spec, aux, g, lens, path if dump else None)

    for _ in range(args.warmup):
        call(True)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    barrier(ws)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call(True)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    clk = clocks.stop()
    barrier(ws)
    ms = max_over_ranks(ws, ms)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        call(False)
    e1.record()
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1)
    return {
        "metric": f"2D amplitude low-pass calls/s at {n}^2 fp32 (calc_amplitude_lowpass with its LOWPASS dump)",
        "value": round(ws * args.steps / (ms / 1e3), 2), "unit": "calls/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: a stripe pattern with seeded noise (numpy PCG64)",
        "config": {"workload": f"amplitude-lowpass {n}^2 fp32", "grid": [n, n], "dx": LP["dx"],
                   "divs_per_sigma": LP["dps"], "parallelism": f"{ws} replica(s)",
                   "timing": "host clock around synchronised calls (each call ends with the dump's D2H and "
                             "gzip write); device_only: CUDA events, no dump"},
        "device_only": {"ms_per_call": round(dev_ms / args.steps, 4),
                        "kernels_per_call": "kmult, C2R (2 passes), norm+square, R2C (2 passes), kmult, "
                                            "C2R (2 passes), norm"},
        "clocks": clk,
    }


def run_reference_lowpass(args):
    name = os.path.join(ROOT, "oracle", "_ref", "libref_lowpass_f32.so")
    if not torch.cuda.is_available():
        return {"impl": "reference", "unavailable": "no CUDA device: the reference's low-pass is CUDA/cuFFT code"}
    if not os.path.exists(name):
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_lowpass_f32.so not built (make -C oracle)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pfc_oracle as O
    L = ctypes.CDLL(name)
    I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L.refl32_time_amplitude_lowpass.argtypes = [I, I, P, P, D, D, ctypes.c_char_p, I, I]
    L.refl32_time_amplitude_lowpass.restype = D
    n = LP["n"] if args.size == 512 else args.size
    lens, hh = (n * LP["dx"], n * LP["dx"], 1.0), (LP["dx"], LP["dx"], 1.0)
    x = np.arange(n) * LP["dx"]
    psi = (0.3 * np.cos(2 * math.pi * (n // 8) / lens[0] * x)[None, :] +
           0.05 * np.random.default_rng(LP["seed"]).standard_normal((n, n))).astype(np.float32)
    spec = np.ascontiguousarray(O.r2c(psi[None]).astype(np.complex64))
    g = np.ascontiguousarray(O.gaussian_init((n, n, 1), lens, hh, LP["dps"], np.float32))
    path = os.path.join(tempfile.mkdtemp(prefix="lowpass_ref_"), "ref.gz")
    clocks = Clocks(0)
    clocks.start()
    ms = L.refl32_time_amplitude_lowpass(n, n, spec.ctypes.data, g.ctypes.data, lens[0], lens[1],
                                         path.encode(), args.warmup, args.steps)
    clk = clocks.stop()
    value = args.steps / (ms / 1e3)
    return {
        "impl": "reference",
        "metric": f"2D amplitude low-pass calls/s at {n}^2 fp32 (calc_amplitude_lowpass with its LOWPASS dump)",
        "value": round(value, 2), "unit": "calls/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: a stripe pattern with seeded noise (numpy PCG64)",
        "config": {"workload": f"amplitude-lowpass {n}^2 fp32", "grid": [n, n], "dx": LP["dx"],
                   "divs_per_sigma": LP["dps"], "parallelism": "single GPU"},
        "cpu_baseline": {"value": round(value, 2), "unit": "calls/s", "cores": 1, "kind": "reference",
                         "sample": "the reference's calc_amplitude_lowpass (lowpass.hpp:78-93, cuFFT plans made "
                                   "once, oracle/_ref) on the GPU, driven by one host thread"},
        "e2e": {"value": round(value, 2), "unit": "calls/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk,
    }


def run_peaks(args, ws, rank, local):
    """Peak finding (26-neighbour strict maxima, sorted records) on the 512^3 FP32 field of
    the headline workload after 200 steps, and bond order (q4, q6, q8, w4, w6, ...) on its
    peaks: CUDA-event device time per call.  Roofline of the peak finder: it reads the field
    once (4 N bytes) and writes one bit per cell and a 16-byte record per peak."""
    from mcstar_b200 import Stepper
    n = args.size
    shape = (n, n, n)
    st = Stepper(shape, WL["dx"], WL["dt"], WL["eps"], dtype=np.float32)
    st.set_real(initial_field(shape, WL["seed"] + rank))
    st.step(200)
    field = st.real_device().contiguous().clone()
    ctx = st.ctx
    ths = -1.0
    cnt, rec = ctx.findpeaks(field, ths)
    for _ in range(args.warmup):
        ctx.findpeaks(field, ths, out=rec, capacity=cnt)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        ctx.findpeaks(field, ths, out=rec, capacity=cnt)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ws, e0.elapsed_time(e1) / args.steps)
    rlim = 10.0
    ctx.bond_order(rec, cnt, st.hh, ths, st.lens[0], rlim)  # warm-up (grows the scratch)
    torch.cuda.synchronize()
    nb = max(1, args.steps // 4)
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    for _ in range(nb):
        rows = ctx.bond_order(rec, cnt, st.hh, ths, st.lens[0], rlim)
    b1.record()
    torch.cuda.synchronize()
    ms_bond = b0.elapsed_time(b1) / nb
    peak, peak_kind = measured_peak()
    alg = 4.0 * n ** 3
    achieved = alg / (ms / 1e3) / 1e9
    return {
        "metric": f"peak-finding calls/s on the {n}^3 fp32 headline field (26-neighbour strict maxima, sorted)",
        "value": round(ws * 1e3 / ms, 2), "unit": "calls/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: the headline random liquid after 200 steps (numpy PCG64 seed)",
        "config": {"workload": f"findpeaks {n}^3 fp32 + bond order of its peaks", "grid": [n, n, n],
                   "ths": ths, "peaks": int(cnt), "bond_rlim": rlim, "l2": "field (537 MB) larger than L2"},
        "roofline": {"bound": "hbm", "kernel": "findpeaks (mark, count, scan, emit)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes": alg, "peak_kind": f"{peak_kind} copy bandwidth"},
        "bond_order": {"ms_per_call": round(ms_bond, 4), "atoms": int(cnt), "rows": int(rows.shape[0])},
        "clocks": clk,
    }


def run_b200(args, ws, rank, local):
    from mcstar_b200 import Stepper
    n = args.size
    shape = (n, n, n)
    st = Stepper(shape, WL["dx"], WL["dt"], WL["eps"], dtype=np.float32)
    st.set_real(initial_field(shape, WL["seed"] + rank))
    ctx = st.ctx
    S = ctx.state_bytes
    # untimed warm-up
    st.step(args.warmup)
    torch.cuda.synchronize()
    # ---- device-resident timed region --------------------------------------------------
    clocks = Clocks(local)
    ctx.profile_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    e0.record()
    st.step(args.steps)
    e1.record()
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    prof = ctx.profile_read()
    ctx.profile_enable(False)
    ms_max = max_over_ranks(ws, ms)
    # ---- end to end through the public API with host buffers ----------------------------------
    host_in = torch.empty_like(st.kpsi, device="cpu").pin_memory()
    host_in.copy_(st.kpsi)
    host_out = torch.empty_like(host_in).pin_memory()
    torch.cuda.synchronize()
    barrier(ws)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    st.step_host(host_in, host_out, args.steps)  # pfc_step_host: copy in, K steps, copy out
    e3.record()
    torch.cuda.synchronize()
    barrier(ws)
    ms_e2e = max_over_ranks(ws, e2.elapsed_time(e3))
    if not np.isfinite(host_out.numpy()[:2]).all():
        raise RuntimeError("non-finite state")

    steps_total = ws * args.steps
    value = steps_total / (ms_max / 1e3)
    cells = n ** 3
    # ---- roofline of the dominant kernel family -------------------------------------------------
    peak, peak_kind = measured_peak()
    kern = kernel_table(prof, S, args.steps, ctx.options.get("x_kernel", 0), ctx.options.get("y_kernel", 0))
    dom = max(kern, key=lambda k: kern[k]["ms_total"])
    d = kern[dom]
    achieved = d["bytes_per_launch"] / (d["ms_per_launch"] / 1e3) / 1e9
    step_bytes = sum(k["bytes_per_launch"] * k["launches"] for k in kern.values()) / args.steps
    # the step's fraction of the roofline with the minimum traffic a step can have (two
    # read+write passes of the half spectrum, 4 S bytes), beside the traffic of this design
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)", "unit": "GB/s",
            "frac": round(achieved / peak, 4), "algorithmic_bytes_per_launch": d["bytes_per_launch"],
            "ms_per_launch": round(d["ms_per_launch"], 5),
            "traffic": ncu_traffic(dom, n),
            "step_bytes_alg": step_bytes,
            "step_frac": round(step_bytes * (value / ws) / 1e9 / peak, 4),
            "step_frac_4S": round(4.0 * S * (value / ws) / 1e9 / peak, 4),
            "kernels": {k: {"ms_per_launch": round(v["ms_per_launch"], 5), "launches": v["launches"],
                            "share": round(v["ms_total"] / max(1e-9, prof["ms"][1] + prof["ms"][2]), 4),
                            "alg_bytes_per_launch": v["bytes_per_launch"],
                            "frac": round(v["bytes_per_launch"] / (v["ms_per_launch"] / 1e3) / 1e9 / peak, 4)}
                        for k, v in kern.items()},
            "entry_exit_ms_per_run": round(prof["ms"][0], 5)}
    out = {
        "metric": "PFC steps/s (Gcell-upd/s in gcell_upd_per_s) at 512^3 fp32",
        "value": round(value, 2), "unit": "steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded random liquid psi0=-0.18+U(-0.05,0.05) (numpy PCG64)",
        "config": {"workload": f"pfc3d-conserved-semi-implicit {n}^3 fp32 liquid", "grid": [n, n, n],
                   "dx": WL["dx"], "dt": WL["dt"], "eps": WL["eps"], "noise": False,
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "state (539 MB at 512^3) larger than L2; no flush"},
        "gcell_upd_per_s": round(value * cells / 1e9, 2),
        "e2e": {"value": round(steps_total / (ms_e2e / 1e3), 2), "unit": "steps/s",
                "h2d_bytes_per_step": S / args.steps, "d2h_bytes_per_step": S / args.steps,
                "note": "per K-step run, one C-ABI call (pfc_step_host): the initial half spectrum from "
                        "pinned host memory, K steps, the final half spectrum back to pinned host memory; "
                        "the copy in runs by ky chunks overlapped with the entry pass"},
        "gpu_launches": prof["launches"],
        "roofline": roof,
        "clocks": clk,
    }
    return out


def run_reference(args):
    name = os.path.join(ROOT, "oracle", "_ref", "libref_pfc_f32.so")
    if not torch.cuda.is_available():
        return {"impl": "reference", "unavailable": "no CUDA device: the reference's step is CUDA/cuFFT code"}
    if not os.path.exists(name):
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_pfc_f32.so not built (make -C oracle)"}
    L = ctypes.CDLL(name)
    P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    L.ref32_create.argtypes = [I, I, I, ctypes.c_ulonglong]
    L.ref32_create.restype = P
    L.ref32_destroy.argtypes = [P]
    L.ref32_r2c.argtypes = [P, P, P]
    L.ref32_set_kpsi.argtypes = [P, P]
    L.ref32_step.argtypes = [P, I, D, D, D, D, D, D, D, I]
    for f in (L.ref32_time_steps, L.ref32_time_e2e):
        f.argtypes = [P, I, D, D, D, D, D, D, D, I]
        f.restype = ctypes.c_float
    n = args.size
    shape = (n, n, n)
    lens = tuple(v * WL["dx"] for v in shape)
    psi = initial_field(shape, WL["seed"]).astype(np.float32)
    h = L.ref32_create(n, n, n, 1234)
    k = np.zeros((n, n, n // 2 + 1), dtype=np.complex64)
    L.ref32_r2c(h, psi.ctypes.data, k.ctypes.data)
    L.ref32_set_kpsi(h, k.ctypes.data)
    L.ref32_step(h, args.warmup, 0.0, WL["dt"], WL["eps"], *lens, 0.0, 0)
    clocks = Clocks(0)
    clocks.start()
    ms = L.ref32_time_steps(h, args.steps, 0.0, WL["dt"], WL["eps"], *lens, 0.0, 0)
    clk = clocks.stop()
    ms_e2e = L.ref32_time_e2e(h, args.steps, 0.0, WL["dt"], WL["eps"], *lens, 0.0, 0)
    L.ref32_destroy(h)
    S = (n // 2 + 1) * n * n * 8
    value = args.steps / (ms / 1e3)
    return {
        "impl": "reference",
        "metric": "PFC steps/s (Gcell-upd/s in gcell_upd_per_s) at 512^3 fp32",
        "value": round(value, 2), "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: seeded random liquid psi0=-0.18+U(-0.05,0.05) (numpy PCG64)",
        "config": {"workload": f"pfc3d-conserved-semi-implicit {n}^3 fp32 liquid", "grid": [n, n, n],
                   "dx": WL["dx"], "dt": WL["dt"], "eps": WL["eps"], "noise": False,
                   "parallelism": "single GPU", "l2": "state larger than L2; no flush"},
        "gcell_upd_per_s": round(value * n ** 3 / 1e9, 2),
        "e2e": {"value": round(args.steps / (ms_e2e / 1e3), 2), "unit": "steps/s",
                "h2d_bytes_per_step": S / args.steps, "d2h_bytes_per_step": S / args.steps},
        "cpu_baseline": {"value": round(value, 2), "unit": "steps/s", "cores": 1, "kind": "reference",
                         "sample": "the reference has no CPU implementation of the step: this arm runs its "
                                   "cuFFT path (oracle/_ref) on the GPU, driven by one host thread"},
        "clocks": clk,
    }


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    from mcstar_b200 import dist
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference_lowpass(args) if args.workload == "lowpass" else run_reference(args)))
        dist.shutdown(ws)
        return
    if args.workload == "ensemble":
        out = run_ensemble(args, ws, rank, local)
    elif args.workload == "lowpass":
        out = run_lowpass(args, ws, rank, local)
    elif args.workload == "peaks":
        out = run_peaks(args, ws, rank, local)
    else:
        out = run_b200(args, ws, rank, local)
        if rank == 0 and ws == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args.size)
    if rank == 0:
        print(json.dumps(out))
    dist.shutdown(ws)


if __name__ == "__main__":
    main()
