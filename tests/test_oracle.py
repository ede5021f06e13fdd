"""CPU tests of the oracle: pinned against the reference's golden vectors and against
known answers derived from the reference's mathematics."""
import glob
import math
import os

import numpy as np
import pytest

import pfc_oracle as O
from conftest import GOLDEN


# ---- Philox4x32-10 known answers (Random123 kat_vectors) ---------------------------------
@pytest.mark.parametrize("ctr,key,want", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_kat(ctr, key, want):
    got = O.philox4x32_10(*ctr, *key)
    assert tuple(int(v) for v in got) == want


# ---- bond order against the reference library's own output ------------------------------------
def _golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "bond_*.npz")))


@pytest.mark.parametrize("path", _golden_cases(), ids=lambda p: os.path.basename(p)[5:-4])
def test_bond_order_oracle_vs_reference(path):
    g = np.load(path)
    ref = O.parse_bond_table(open(path[:-4] + ".txt").read())
    h = float(g["h"])
    res, _ = O.bond_order(g["idx"], g["field"], (h, h, h), float(g["ths"]), float(g["box"]), float(g["rlim"]))
    assert len(res["x"]) == len(ref["x"])
    for c in O.BOND_COLUMNS[:13]:
        # the reference prints %.6f.  Its closed-form Y_8 (bond-order.cpp:163-175) divides
        # ((1+x)/(1-x))^m by a polynomial with cancellation, which loses up to ~5e-5 in q8
        # for neighbours with 1 - |cos theta| ~ 2e-3 (scipy and this oracle agree to 1e-15).
        tol = 1e-4 if c in ("q8", "q8b") else 1.5e-6
        np.testing.assert_allclose(res[c], ref[c], atol=tol, rtol=0, err_msg=c)


def test_bond_order_fcc_known_values():
    g = np.load(os.path.join(GOLDEN, "bond_fcc_perfect_f32.npz"))
    h = float(g["h"])
    res, _ = O.bond_order(g["idx"], g["field"], (h, h, h), float(g["ths"]), float(g["box"]), float(g["rlim"]))
    # perfect fcc, 12 neighbours: q4 = 0.19094, q6 = 0.57452, w4 = -0.15932, w6 = -0.01316
    assert np.all(res["nb"] == 12)
    np.testing.assert_allclose(res["q4"], 0.190941, atol=2e-6)
    np.testing.assert_allclose(res["q6"], 0.574524, atol=2e-6)
    np.testing.assert_allclose(res["w4"], -0.159317, atol=2e-6)
    np.testing.assert_allclose(res["w6"], -0.013161, atol=2e-6)


def test_wigner3j_racah():
    w = O.wigner3j_lll(4)
    assert len(w) == 61
    # sum over m of (l l l; m -m 0)^2 (2l+1) ... orthogonality: sum_{m1,m2} (3j)^2 = 1/(2l+1) per m3
    for l in (4, 6):
        w = O.wigner3j_lll(l)
        for m3 in range(-l, l + 1):
            s = sum(v * v for (a, b, c), v in w.items() if c == m3)
            assert abs(s * (2 * l + 1) - 1.0) < 1e-12


def test_ylm_matches_scipy_outside_pole_band():
    from scipy.special import sph_harm_y
    rng = np.random.default_rng(3)
    th = rng.uniform(0.1, np.pi - 0.1, 200)
    ph = rng.uniform(-np.pi, np.pi, 200)
    for l in (4, 6, 8):
        y = O.ylm_all(l, np.cos(th), ph)
        ys = np.array([sph_harm_y(l, m, th, ph) for m in range(-l, l + 1)])
        assert np.max(np.abs(y - ys)) < 1e-12


# ---- FFT: numpy is the reference's own FFT oracle (cufft_unittest/my_unit_test.py) ----------------
def test_r2c_c2r_roundtrip_scaling():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((6, 10, 15))
    X = O.r2c(x)
    assert X.shape == (6, 10, 8)
    y = O.c2r(X, (15, 10, 6))
    np.testing.assert_allclose(y / x.size, x, atol=1e-14)


# ---- step: known answers from the reference's mathematics ------------------------------------
def test_uniform_state_is_fixed_point_and_k0_invariant():
    shape = (16, 12, 10)
    lens = tuple(n * math.pi / 4 for n in shape)
    psi = np.full((10, 12, 16), -0.2)
    k = O.r2c(psi)
    k1 = O.step(k, 3, 0.5, 0.3, lens, shape)
    np.testing.assert_allclose(k1, k, atol=1e-12)
    rng = np.random.default_rng(1)
    k = O.r2c(-0.2 + 0.05 * rng.standard_normal((10, 12, 16)))
    k1 = O.step(k, 5, 0.5, 0.3, lens, shape, namp=0.1, seed=7)
    assert k1[0, 0, 0] == k[0, 0, 0]  # k = 0: k^2 = 0 and |k| = 0 zero both update terms


def test_single_mode_linear_amplification():
    # psi = psi0 + d cos(q x): per step the mode grows by (1 - dt q^2 (3 psi0^2 - C)) / D(q) to O(d^2)
    nx, ny, nz = 32, 4, 4
    dx = math.pi / 4
    lens = (nx * dx, ny * dx, nz * dx)
    psi0, d, dt, eps = -0.25, 1e-7, 0.1, 0.3
    x = np.arange(nx) * dx
    q = 2 * math.pi * 3 / lens[0]
    psi = psi0 + d * np.cos(q * x)[None, None, :] * np.ones((nz, ny, 1))
    k = O.r2c(psi)
    k1 = O.step(k, 1, dt, eps, lens, (nx, ny, nz))
    growth = (k1[0, 0, 3] / k[0, 0, 3]).real
    q2 = q * q
    want = (1 - dt * q2 * (3 * psi0 ** 2 - 1)) / (1 + dt * q2 * ((1 - q2) ** 2 + 1 - eps))
    assert abs(growth - want) < 1e-6


def test_free_energy_of_uniform_state():
    # F / V = 1/2 (1 - eps) psi0^2 + 1/4 psi0^4   (common/pfc.hpp:4-5 without the -mu psi0 term)
    shape = (8, 8, 8)
    dx = 0.7
    lens = tuple(n * dx for n in shape)
    psi0, eps = -0.3, 0.25
    k = O.r2c(np.full((8, 8, 8), psi0))
    F = O.free_energy(k, eps, lens, (dx, dx, dx), shape)
    V = np.prod(lens)
    assert abs(F / V - (0.5 * (1 - eps) * psi0 ** 2 + 0.25 * psi0 ** 4)) < 1e-14


# ---- noise -------------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(16, 12, 10), (15, 9, 7), (32, 32, 1)])
def test_kspace_noise_hermitian_and_moments(shape):
    nx, ny, nz = shape
    xi = O.fill_kspace(shape, 11, 3, dtype=np.float64)
    # Hermitian on the i0 = 0 (and nx/2) planes
    planes = [0] + ([nx // 2] if nx % 2 == 0 else [])
    for i0 in planes:
        p = xi[:, :, i0]
        mirror = p[(-np.arange(nz)) % nz][:, (-np.arange(ny)) % ny]
        np.testing.assert_array_equal(p, np.conj(mirror))
    assert abs(np.mean(np.abs(xi) ** 2) - 1.0) < 0.1
    # C2R of Hermitian noise is real white noise with variance N per cell
    r = O.c2r(xi, shape) / math.sqrt(nx * ny * nz)
    assert abs(r.var() - 1.0) < 0.15


def test_peaks_on_gaussian_lattice():
    n = 24
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    sites = [(4, 5, 6), (16, 5, 6), (10, 17, 20), (0, 0, 23)]
    f = np.zeros((n, n, n))
    for (a, b, c) in sites:
        dxx = (x - a + n / 2) % n - n / 2
        dyy = (y - b + n / 2) % n - n / 2
        dzz = (z - c + n / 2) % n - n / 2
        f += np.exp(-(dxx ** 2 + dyy ** 2 + dzz ** 2) / 4.0)
    idx, val = O.findpeaks3d(f, 0.5)
    got = sorted(map(tuple, idx.tolist()))
    assert got == sorted(sites)


def test_fused_forms_of_the_polynomial_and_hpfc_updates_equal_their_kernel_mirrors():
    """The oracle's propagate() forms of kernel_update_eom_py and kernel_update_eom_hpfcnoise
    (the stabilisation constant C in place of the reference's 1) equal its direct mirrors of
    the two kernels at C = 1, with and without noise."""
    rng = np.random.default_rng(0)
    shape, lens = (32, 16, 8), (32 * 0.78, 16 * 0.78, 8 * 0.78)
    k = O.r2c(rng.standard_normal(shape[::-1]))
    n = O.r2c(rng.standard_normal(shape[::-1]))
    xi = O.fill_kspace(shape, 3, 1, np.float64)
    # (the mirrors take sqrt(N) and |k| in single precision, as the reference's sqrtf)
    for noise, namp, tol in ((None, 0.0, 1e-12), (xi, 0.02, 1e-6)):
        a, _ = O.propagate(k, n, noise, namp, 0.5, 0.3, lens, shape, 1.0, "conserved_poly")
        b = O.update_eom_py(k, n, noise, namp, 0.5, 0.3, lens, shape)
        assert np.abs(a - b).max() <= tol * np.abs(b).max()
    s2, l2 = (64, 48, 1), (64 * 0.5, 48 * 0.5, 0.5)
    k = O.r2c(rng.standard_normal(s2[::-1]))
    n = O.r2c(rng.standard_normal(s2[::-1]))
    f = [O.fill_kspace(s2, 3, 1, np.float64, domain=O.HPFC_DOMAIN + i) for i in (1, 2, 3)]
    a, _ = O.propagate(k, n, tuple(f), 0.01, 0.5, 0.3, l2, s2, 1.0, "conserved_hpfc")
    b = O.update_eom_hpfcnoise(k, n, *f, 0.01, 0.5, 0.3, l2, s2)
    assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
    assert not np.allclose(f[0], f[1])  # three independent streams
