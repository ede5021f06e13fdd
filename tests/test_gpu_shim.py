"""A host program written against the mcstar-libs source API (tests/shim/driver_step.cu,
built on the mcstar-libs-named headers of include/mcstar and libpfc_b200) runs the
reference drivers' per-step loop -- copy psi^, C2R, psi3_split(norm), R2C,
[fill_kspace], update_eom -- then the free energy, the peak list and the bond-order
table.  Every output is checked against the oracle's restatement of the same calls."""
import math
import os
import subprocess

import numpy as np
import pytest

import pfc_oracle as O
from conftest import build_shim_driver

pytestmark = pytest.mark.gpu

_BUILT = {}


def _driver(flt, tmp_path_factory, name="driver_step.cu"):
    key = (flt, name)
    if key not in _BUILT:
        from conftest import ROOT
        d = tmp_path_factory.mktemp("drv_" + flt)
        rc, out = build_shim_driver(flt, d / "driver", os.path.join(ROOT, "tests", "shim", name))
        assert rc == 0, out[-3000:]
        _BUILT[key] = str(d / "driver")
    return _BUILT[key]


def _run(drv, shape, dx, steps, dt, eps, namp, seed, psi, outdir):
    inp = os.path.join(outdir, "in.npy")
    np.save(inp, psi if shape[2] > 1 else psi[0])
    args = [drv, *(str(v) for v in shape), repr(dx), str(steps), repr(dt), repr(eps), repr(namp), str(seed), inp,
            str(outdir)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    F = float(next(ln.split()[1] for ln in r.stdout.splitlines() if ln.startswith("F ")))
    k = np.load(os.path.join(outdir, "kpsi.npy"))
    return k.reshape(O.cmpl_shape(shape)), F


def _lens(shape, dx):
    return (shape[0] * dx, shape[1] * dx, shape[2] * dx if shape[2] > 1 else 1.0)


def _oracle_loop(psi, shape, dx, steps, dt, eps, namp, seed, dtype):
    ctype = np.complex64 if dtype == np.float32 else np.complex128
    lens = _lens(shape, dx)
    kpsi = O.r2c(psi.astype(dtype)).astype(ctype)
    for t in range(steps):
        real = O.c2r(kpsi, shape).astype(dtype)
        knl = O.r2c(O.psi3_split(real, None, 0.0, norm=True).astype(dtype)).astype(ctype)
        kn = O.fill_kspace(shape, seed, t, dtype=dtype) if namp else None
        kpsi = O.update_eom(kpsi, knl, kn, namp, dt, eps, lens, shape, C=1.0, ref_float_sqrt=True).astype(ctype)
    return kpsi


def _bcc(n, a_cells, psi0=-0.2, amp=0.2):
    """One-mode bcc, sum of cos(q.r) over the six <110>/sqrt(2) directions (|q| = 1), with
    lattice constant a_cells grid cells (dx = 2 pi sqrt(2) / a_cells)."""
    dx = 2 * math.pi * math.sqrt(2) / a_cells
    r = np.arange(n) * dx
    z, y, x = np.meshgrid(r, r, r, indexing="ij")
    s = 1 / math.sqrt(2)
    acc = np.zeros_like(x)
    for q in [(s, s, 0), (s, -s, 0), (s, 0, s), (s, 0, -s), (0, s, s), (0, s, -s)]:
        acc += np.cos(q[0] * x + q[1] * y + q[2] * z)
    return psi0 + amp * acc, dx


def _peaks_txt(path, dx):
    text = open(path).read().split()
    rows = np.array([float(v) for v in text]).reshape(-1, 4)
    return np.rint(rows[:, :3] / dx).astype(int), rows[:, 3]


CASES = [  # (name, shape, precision, namp, steps)
    ("bcc-f32", (32, 32, 32), "float", 0.0, 4),
    # 8192 maxima: more atoms than a bond-order scratch starts with (it grows in the call)
    ("bcc-many-f32", (64, 64, 64), "float", 0.0, 2),
    ("liquid-f64", (32, 32, 32), "double", 0.0, 3),
    ("liquid-2d-f64", (64, 64, 1), "double", 0.0, 5),
    ("noise-f32", (32, 32, 32), "float", 0.02, 3),
]


@pytest.mark.parametrize("name,shape,flt,namp,steps", CASES, ids=[c[0] for c in CASES])
def test_reference_style_driver_matches_oracle(name, shape, flt, namp, steps, tmp_path, tmp_path_factory):
    dtype = np.float32 if flt == "float" else np.float64
    drv = _driver(flt, tmp_path_factory)
    nx, ny, nz = shape
    a_cells = 16 if name == "bcc-f32" else 4
    if name.startswith("bcc"):
        psi, dx = _bcc(nx, a_cells)
    else:
        # 3D liquids stay below the peak threshold (empty peak list and table); the 2D
        # liquid has mean 0 and so plenty of peaks
        dx = math.pi / 4
        psi = (-0.2 if nz > 1 else 0.0) + 0.1 * np.random.default_rng(4).uniform(-1, 1, (nz, ny, nx))
    psi = psi.astype(dtype)
    dt, eps, seed = 0.5, 0.3, 9
    got, F = _run(drv, shape, dx, steps, dt, eps, namp, seed, psi, tmp_path)
    want = _oracle_loop(psi, shape, dx, steps, dt, eps, namp, seed, dtype)
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol

    # free energy of the driver's final state through the same path (eom.hpp:88-141)
    lens = _lens(shape, dx)
    F_want = O.free_energy(got.astype(np.complex128), eps, lens, (dx, dx, dx), shape)
    assert abs(F - F_want) <= 2e-6 * abs(F_want) + 1e-9

    # peaks of the driver's final field, in increasing linear index
    field = O.norm(O.c2r(got.astype(np.complex128), shape))
    idx, val = _peaks_txt(os.path.join(tmp_path, "peaks.txt"), dx)
    if nz > 1:
        widx, wval = O.findpeaks3d(field, 0.0)
    else:
        widx, wval = O.findpeaks2d(field[0], 0.0)
    assert np.array_equal(idx, widx)
    assert np.allclose(val, wval, atol=1e-5)
    if name.startswith("bcc"):
        assert len(idx) == 2 * (nx // a_cells) ** 3  # conventional cells of 2 sites

    if nz > 1:
        table = O.parse_bond_table(open(os.path.join(tmp_path, "bond.txt")).read())
        ref, _ = O.bond_order(idx, val, (dx, dx, dx), 0.0, nx * dx, 8.3)
        for col, v in table.items():
            assert np.allclose(v, np.asarray(ref[col], dtype=np.float64), atol=2e-6), col
        if name.startswith("bcc"):
            assert len(table["nb"]) == len(idx)
            assert np.all(table["nb"] == 8) and np.allclose(table["q6"], 0.628539, atol=1e-4)


@pytest.mark.parametrize("flt", ["double", "float"])
def test_relaxation_driver_matches_oracle(flt, tmp_path, tmp_path_factory):
    """tests/shim/driver_relax.cu: exponential conserved steps (eom-exp.hpp) then the
    non-conserved relaxation (el.hpp) until the largest mode change drops below 1e-3."""
    dtype = np.float32 if flt == "float" else np.float64
    drv = _driver(flt, tmp_path_factory, "driver_relax.cu")
    shape, dx, steps, dt, eps = (32, 32, 16), math.pi / 4, 5, 0.5, 0.3
    nx, ny, nz = shape
    psi = (-0.2 + 0.05 * np.random.default_rng(21).uniform(-1, 1, (nz, ny, nx))).astype(dtype)
    inp = os.path.join(tmp_path, "in.npy")
    np.save(inp, psi)
    r = subprocess.run([drv, str(nx), str(ny), str(nz), repr(dx), str(steps), repr(dt), repr(eps), inp, str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    iters = int(next(ln.split()[1] for ln in r.stdout.splitlines() if ln.startswith("iters ")))
    lens = _lens(shape, dx)
    kop = O.init_eom_op(shape, lens, dt, eps)
    k = O.r2c(psi.astype(np.float64))

    def knl_of(k):
        return O.r2c(O.psi3_split(O.c2r(k, shape), None, 0.0, norm=True))

    for _ in range(steps):
        k = O.update_eom_exp(kop, k, knl_of(k), None, 0.0, eps, lens, shape)
    got = np.load(os.path.join(tmp_path, "kpsi_exp.npy")).reshape(O.cmpl_shape(shape))
    # the operator is exp(-L dt) in single precision (the reference's expf) in both
    # precisions; CUDA's expf and numpy's float32 exp differ by up to a float ulp
    tol = 1e-4 if dtype == np.float32 else 1e-7
    assert np.linalg.norm(got - k) / np.linalg.norm(k) < tol
    for _ in range(min(iters + 1, 200)):
        k, _change = O.update_el(k, knl_of(k), dt, eps, lens, shape)
    got = np.load(os.path.join(tmp_path, "kpsi_el.npy")).reshape(O.cmpl_shape(shape))
    assert np.linalg.norm(got - k) / np.linalg.norm(k) < tol


@pytest.mark.parametrize("flt", ["double", "float"])
def test_lowpass_driver_matches_oracle(flt, tmp_path, tmp_path_factory):
    """tests/shim/driver_lowpass.cu: R2C, the Gaussian filter (gaussian.hpp) and
    calc_amplitude_lowpass (lowpass.hpp): the amplitude field and the LOWPASS dump."""
    import gzip
    dtype = np.float32 if flt == "float" else np.float64
    drv = _driver(flt, tmp_path_factory, "driver_lowpass.cu")
    nx, ny, dx, dps = 96, 64, 0.8, 2.0
    shape = (nx, ny, 1)
    x = np.arange(nx) * dx
    psi = (0.3 * np.cos(2 * math.pi * 12 / (nx * dx) * x)[None, None, :] +
           0.05 * np.random.default_rng(8).standard_normal((1, ny, nx))).astype(dtype)
    inp = os.path.join(tmp_path, "in.npy")
    np.save(inp, psi)
    r = subprocess.run([drv, str(nx), str(ny), repr(dx), repr(dps), inp, str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lens, hh = (nx * dx, ny * dx, 1.0), (dx, dx, 1.0)
    g = O.gaussian_init(shape, lens, hh, dps, dtype)
    amp, low = O.amplitude_lowpass(O.r2c(psi.astype(np.float64)), g, shape)
    got = np.load(os.path.join(tmp_path, "amplitude.npy")).reshape(amp.shape)
    tol = 2e-5 if dtype == np.float32 else 1e-11
    assert np.linalg.norm(got - amp) / np.linalg.norm(amp) < tol
    text = gzip.decompress(open(os.path.join(tmp_path, "lowpass.gz"), "rb").read())
    assert text.startswith(b"LOWPASS\n")
    assert text.count(b"\n") > 4
