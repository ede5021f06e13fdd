"""Precision study: the FP32 stepper (FP64 k = 0 mode, FP64 energy sums) against an FP64
run of the same step from the same initial field.

Reports the field's relative L2 error, the free-energy error, the drift of the mean
density (psi^(k=0) / N) of both runs, and whether the peak lists agree.  Run as
``python -m mcstar_b200.precision [--n 512 --steps 1000]``; prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from .kernels import records_to_host
from .stepper import Stepper, liquid_random


def precision_study(n=512, steps=1000, dt=0.25, eps=0.3, psi0=-0.18, amp=0.05, seed=2024, dx=math.pi / 4,
                    chunk=100, ths=0.0):
    shape = (n, n, n)
    psi = liquid_random(shape, psi0, amp, seed)
    runs = {}
    for dtype in (np.float64, np.float32):
        st = Stepper(shape, dx, dt, eps, dtype=dtype)
        st.set_real(psi)
        runs[np.dtype(dtype).name] = st
    s64, s32 = runs["float64"], runs["float32"]
    k0_64, k0_32 = s64.kpsi[:2].double().cpu().numpy(), s32.kpsi[:2].double().cpu().numpy()
    history = []
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        m = min(chunk, steps - done)
        s64.step(m)
        s32.step(m)
        done += m
        history.append({"step": done, "F64": s64.free_energy(), "F32": s32.free_energy()})
    elapsed = time.perf_counter() - t0
    r64 = s64.real_device().clone()
    r32 = s32.real_device().double()
    rel_l2 = float(torch.linalg.vector_norm(r32 - r64) / torch.linalg.vector_norm(r64))
    n64, rec64 = s64.peaks(ths)
    n32, rec32 = s32.peaks(ths)
    p64 = records_to_host(rec64, np.float64)
    p32 = records_to_host(rec32, np.float32)
    set64 = {(int(a), int(b), int(c)) for a, b, c in zip(p64["i0"], p64["i1"], p64["i2"])}
    set32 = {(int(a), int(b), int(c)) for a, b, c in zip(p32["i0"], p32["i1"], p32["i2"])}
    k1_64, k1_32 = s64.kpsi[:2].double().cpu().numpy(), s32.kpsi[:2].double().cpu().numpy()
    F64, F32 = history[-1]["F64"], history[-1]["F32"]
    return {
        "grid": n, "steps": steps, "dt": dt, "eps": eps, "psi0": psi0, "amp": amp, "seed": seed,
        "field_rel_l2_fp32_vs_fp64": rel_l2,
        "free_energy_rel_err": abs(F32 - F64) / abs(F64),
        "free_energy_fp64": F64,
        "mean_density_drift_fp32": float(abs(k1_32[0] - k0_32[0]) / abs(k0_32[0])),
        "mean_density_drift_fp64": float(abs(k1_64[0] - k0_64[0]) / abs(k0_64[0])),
        "peaks_fp64": n64, "peaks_fp32": n32, "peaks_identical": set64 == set32,
        "peaks_symmetric_difference": len(set64 ^ set32),
        "history": history, "wall_s": elapsed,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--chunk", type=int, default=100)
    a = ap.parse_args()
    print(json.dumps(precision_study(n=a.n, steps=a.steps, chunk=a.chunk)))


if __name__ == "__main__":
    main()
