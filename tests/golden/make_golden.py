"""Generates the golden fixtures of tests/golden from the reference itself.

Bond order: point sets (grid indices + field) are analysed by the UNMODIFIED reference
``bond_order_analysis`` (bond-order-analysis/bond-order.cpp), compiled where it lies by
``make -C oracle`` into oracle/_ref/libbondorder_ref.so; its text table is stored next
to the inputs.  Run from the repository root after ``make -C oracle``:

    python tests/golden/make_golden.py

The fixtures are small (a few hundred atoms each) and committed; the tests never run
the reference.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pfc_oracle as O  # noqa: E402


def lattice(kind, n, a, jitter, rng):
    basis = {"bcc": [(0, 0, 0), (0.5, 0.5, 0.5)],
             "fcc": [(0, 0, 0), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5)],
             "sc": [(0, 0, 0)]}[kind]
    pts = []
    for i in range(0, n, a):
        for j in range(0, n, a):
            for k in range(0, n, a):
                for b in basis:
                    pts.append((i + int(b[0] * a), j + int(b[1] * a), k + int(b[2] * a)))
    pts = np.array(pts)
    if jitter:
        pts = pts + rng.integers(-jitter, jitter + 1, size=pts.shape)
    return pts % n


def cases():
    rng = np.random.default_rng(20240601)
    out = []
    pts = lattice("bcc", 64, 8, 1, rng)
    out.append(("bcc_jitter_f32", pts, rng.uniform(0.0, 1.0, len(pts)), np.float32,
                dict(h=np.pi / 4, ths=0.1, n=64, rlim=8.0)))
    pts = lattice("fcc", 48, 12, 0, rng)
    out.append(("fcc_perfect_f32", pts, np.ones(len(pts)), np.float32, dict(h=1.0, ths=-1e6, n=48, rlim=9.0)))
    pts = lattice("sc", 40, 8, 0, rng)
    out.append(("sc_poles_f64", pts, rng.uniform(0.5, 1.0, len(pts)), np.float64, dict(h=0.5, ths=0.0, n=40, rlim=4.2)))
    pts = rng.integers(0, 32, size=(220, 3))
    pts = np.unique(pts, axis=0)
    out.append(("random_f32", pts, rng.uniform(-1.0, 1.0, len(pts)), np.float32, dict(h=0.5, ths=-0.2, n=32, rlim=4.0)))
    pts = lattice("bcc", 48, 12, 2, rng)
    out.append(("bcc_wide_f64", pts, rng.uniform(0.0, 1.0, len(pts)), np.float64, dict(h=0.75, ths=0.05, n=48, rlim=13.0)))
    return out


def main():
    so = os.path.join(ROOT, "oracle", "_ref", "libbondorder_ref.so")
    lib = ctypes.CDLL(so)
    for fn in (lib.ref_bond_order_f32, lib.ref_bond_order_f64):
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 6 + [ctypes.c_char_p]
        fn.restype = ctypes.c_int
    for name, pts, field, dt, p in cases():
        M = np.zeros(len(pts), dtype=O.MAX_DTYPE[dt])
        M["i0"], M["i1"], M["i2"] = pts[:, 0], pts[:, 1], pts[:, 2]
        M["field"] = field.astype(np.float32)
        h = p["h"]
        hf = float(np.float32(h)) if dt == np.float32 else float(h)
        box = p["n"] * hf
        txt = os.path.join(HERE, f"bond_{name}.txt")
        fn = lib.ref_bond_order_f32 if dt == np.float32 else lib.ref_bond_order_f64
        rc = fn(M.ctypes.data, len(M), hf, hf, hf, p["ths"], box, p["rlim"], txt.encode())
        assert rc == 0
        np.savez(os.path.join(HERE, f"bond_{name}.npz"), idx=pts.astype(np.int32), field=M["field"],
                 dtype=np.dtype(dt).name, h=hf, ths=p["ths"], box=box, rlim=p["rlim"])
        print(name, len(M), "atoms ->", txt)


if __name__ == "__main__":
    main()
