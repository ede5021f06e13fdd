"""CPU oracle for the conserved semi-implicit PFC step -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy (FP64 unless a dtype is passed), the arithmetic of
the reference's hot path so that the CUDA implementation can be checked against it.
It is imported only by tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline
leg of ``bench.py``; the product path never calls it.

What each function restates (reference paths relative to the mcstar-libs root):

* ``kgrid``              -- ``K()`` and ``L_L2()``, cuda/kernels/common.hpp:18-28
* ``update_eom``         -- ``kernel_update_eom``, cuda/kernels/eom.hpp:60-72
* ``update_eom_with_fen``-- ``kernel_update_eom_with_fen``, eom.hpp:88-102
* ``psi3_split``         -- ``kernel_psi3_split(_pot)``, cuda/kernels/psi3_split.hpp:1-26
* ``norm``               -- ``kernel_norm``, cuda/kernels/norm.hpp:1-10
* ``calc_fen``           -- ``kernel_calc_fen``/``call_kernel_calc_fen``, eom.hpp:111-141
* ``r2c``/``c2r``        -- ``FFT::CufftPlan::execute`` (unnormalised cuFFT R2C / C2R),
                            cuda/cufft_wrapper.hpp:50-86; numpy's rfftn is the oracle the
                            reference's own test uses (cufft_unittest/my_unit_test.py:138)
* ``findpeaks3d/2d``     -- ``kernel_findpeaks`` (findpeaks.hpp:7-29) and
                            ``kernel_findpeaks_2d`` (findpeaks_2d.hpp:7-27), returned
                            sorted by linear index (the reference's order is atomic-racy)
* ``bond_order``         -- ``bond_order_analysis`` and helpers,
                            bond-order-analysis/bond-order.cpp:53-349
* ``step``               -- the driver loop of one conserved step (copy, C2R,
                            psi3_split(norm), R2C, [noise], update_eom), or with the
                            updates of eom-exp.hpp, el.hpp, el-exp.hpp (``propagate``)
* ``fill_kspace``        -- the k-space noise contract of ``NoiseHostApi::fill_kspace``
                            (cuda/noise.hpp:7-142): complex normal modes with
                            E|xi|^2 = 1, Hermitian pairs on the i0 = 0 and i0 = nx/2
                            planes, self-conjugate modes real with unit variance.  The
                            reference draws them from cuRAND XORWOW, which this build
                            replaces by counter-based Philox4x32-10 (Salmon et al., SC'11)
                            keyed by the canonical member of each +-k pair; the random
                            stream itself therefore differs by design and parity with the
                            reference is statistical, while parity between this oracle and
                            the CUDA kernels is value-for-value.

* ``gaussian_init``, ``kmult``, ``amplitude_lowpass``, ``lowpass_text`` -- the 2D
                            spectral low-pass (cuda/kernels/gaussian.hpp:23-67,
                            cuda/kernels/lowpass.hpp:1-93) and its LOWPASS dump format

Pinning: the FFT against numpy at the reference's own tolerances, the bond-order
restatement against the compiled reference library (tests/golden, oracle/Makefile),
and the step against the reference's cuFFT path on a GPU (oracle/_ref).
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

TWO_PI_REF = 6.283185307179586232  # the literal the reference uses in K(), common.hpp:28


# ----------------------------------------------------------------------------------
# grids and FFTs
# ----------------------------------------------------------------------------------
def cmpl_shape(shape_xyz):
    nx, ny, nz = shape_xyz
    return (nz, ny, nx // 2 + 1)


def real_shape(shape_xyz):
    nx, ny, nz = shape_xyz
    return (nz, ny, nx)


def wavenumbers(n, length, half=False, dtype=np.float64):
    """K(i, n, len) = (i < n/2+1 ? i : i-n) * 2pi / len  (common.hpp:27-28)."""
    m = n // 2 + 1 if half else n
    i = np.arange(m)
    sgn = np.where(i < n // 2 + 1, i, i - n).astype(dtype)
    return sgn * dtype(TWO_PI_REF) / dtype(length)


def kgrid(shape_xyz, lens, dtype=np.float64):
    """Returns k^2 on the half-spectrum grid, numpy shape (nz, ny, nx//2+1)."""
    nx, ny, nz = shape_xyz
    k0 = wavenumbers(nx, lens[0], half=True, dtype=dtype)
    k1 = wavenumbers(ny, lens[1], dtype=dtype)
    k2 = wavenumbers(nz, lens[2], dtype=dtype)
    return (k0[None, None, :] ** 2 + k1[None, :, None] ** 2 + k2[:, None, None] ** 2).astype(dtype)


def _fft_mod(workers):
    if workers is None:
        return np.fft, {}
    import scipy.fft as sfft
    return sfft, {"workers": workers}


def r2c(real, workers=None):
    """Unnormalised forward R2C over all axes; numpy shape (nz, ny, nx) -> (nz, ny, nx//2+1)."""
    mod, kw = _fft_mod(workers)
    out = mod.rfftn(real, **kw)
    return out.astype(np.complex64) if real.dtype == np.float32 else out


def c2r(cmpl, shape_xyz, workers=None):
    """Unnormalised backward C2R: a round trip r2c -> c2r multiplies by N
    (cufft_unittest/my_unit_test.py:95)."""
    mod, kw = _fft_mod(workers)
    rs = real_shape(shape_xyz)
    n = rs[0] * rs[1] * rs[2]
    out = mod.irfftn(cmpl, s=rs, axes=tuple(range(len(rs))), **kw) * n
    return out.astype(np.float32) if cmpl.dtype == np.complex64 else out


# ----------------------------------------------------------------------------------
# pointwise kernels
# ----------------------------------------------------------------------------------
def update_eom(kpsi, knl, knoise, namp, dt, eps, lens, shape_xyz, C=1.0, ref_float_sqrt=True):
    """psi^ <- (psi^ - dt k^2 N^ + dt namp sqrt(N) |k| xi^) / (1 + dt k^2 ((1-k^2)^2 + C - eps)).

    C = 1 is the reference (eom.hpp:62-71: denom = 1 - dt((2-eps)(-k^2) + 2k^4 - k^6));
    C is the stabilisation constant of the split, matching psi3_split's  - C psi.
    ref_float_sqrt: the reference takes sqrt(N) and |k| with sqrtf (eom.hpp:62,68), i.e. in
    single precision even for double fields; False evaluates both in full precision.
    """
    nx, ny, nz = shape_xyz
    k2 = kgrid(shape_xyz, lens)
    dopx = -k2
    dopy = k2 * k2
    if ref_float_sqrt:
        k = np.sqrt(k2.astype(np.float32)).astype(np.float64)
        namp_eff = namp * float(np.sqrt(np.float32(nx * ny * nz)))
    else:
        k = np.sqrt(k2)
        namp_eff = namp * math.sqrt(nx * ny * nz)
    denom = 1.0 - dt * ((1.0 + C - eps) * dopx + 2.0 * dopy + dopx * dopy)
    num = kpsi.astype(np.complex128) + dt * dopx * knl
    if knoise is not None:
        num = num + dt * namp_eff * k * knoise
    return num / denom


def lop(shape_xyz, lens, eps):
    """L^ = (2 - eps) + 2(-k^2) + k^4 = (1-k^2)^2 + 1 - eps (eom.hpp:97)."""
    k2 = kgrid(shape_xyz, lens)
    return (2.0 - eps) - 2.0 * k2 + k2 * k2


def update_eom_with_fen(kpsi, knl, knoise, namp, dt, eps, lens, shape_xyz, C=1.0):
    """Returns (updated psi^, L^ psi^_old) -- eom.hpp:88-102 overwrites knoise with the latter."""
    new = update_eom(kpsi, knl, knoise, namp, dt, eps, lens, shape_xyz, C=C)
    return new, lop(shape_xyz, lens, eps) * kpsi


def psi3_split(arr, pot=None, mu=0.0, norm=False, C=1.0):
    """(m psi)^3 - C (m psi) - mu (+ pot), m = 1/N when norm (psi3_split.hpp:1-26)."""
    mul = 1.0 / arr.size if norm else 1.0
    t = arr * mul
    out = t * t * t - C * t - mu
    if pot is not None:
        out = out + pot
    return out


def norm(arr):
    """arr / N (norm.hpp:1-3)."""
    return arr / arr.size


def calc_fen(psi, lpsi, hh):
    """f = 1/2 psi (Lpsi - psi + 1/2 psi^3); returns (sum(f) * hx hy hz, f) -- eom.hpp:111-141.
    The sum here is exact-order FP64 (math.fsum); the reference accumulates float atomics."""
    f = 0.5 * psi * (lpsi - psi + 0.5 * psi * psi * psi)
    total = math.fsum(np.asarray(f, dtype=np.float64).ravel().tolist()) if f.size <= 1 << 22 \
        else float(np.sum(f.astype(np.float64)))
    return total * hh[0] * hh[1] * hh[2], f


def free_energy(kpsi, eps, lens, hh, shape_xyz):
    """F of the state psi^ through the reference's path (eom.hpp:88-141 at dt = 0)."""
    lpsi = norm(c2r(lop(shape_xyz, lens, eps) * kpsi, shape_xyz))
    psi = norm(c2r(kpsi, shape_xyz))
    return calc_fen(psi, lpsi, hh)[0]


# ----------------------------------------------------------------------------------
# the reference's other propagators (FP64 restatements; exp and sqrt in single
# precision where the reference calls expf / sqrtf)
# ----------------------------------------------------------------------------------
def _f32(fn, x):
    return fn(np.asarray(x, dtype=np.float64).astype(np.float32)).astype(np.float64)


def _dops(shape_xyz, lens):
    k2 = kgrid(shape_xyz, lens)
    return -k2, k2 * k2


def init_eom_op(shape_xyz, lens, dt, eps):
    """kernel_init_eom_op (eom-exp.hpp:3-10): kop = exp(-L dt) + i (exp(-L dt) - 1)/L,
    L = -dop.x ((2 - eps) + 2 dop.x + dop.y); -dt where L = 0 (the 0/0 at k = 0)."""
    dx, dy = _dops(shape_xyz, lens)
    lin = -dx * ((2.0 - eps) + 2.0 * dx + dy)
    e = _f32(np.exp, -lin * dt)
    with np.errstate(invalid="ignore", divide="ignore"):
        second = (e - 1.0) / lin
    return e + 1j * np.where(np.isnan(second), -dt, second)


def update_eom_exp(kop, kpsi, knl, knoise, namp, eps, lens, shape_xyz, with_fen=False):
    """kernel_update_eom(_with_fen) of eom-exp.hpp:18-60: kop.x psi^ - dop.x kop.y N^ -
    namp sqrt(N) |k| kop.y xi^; with_fen also returns L^ psi^_old."""
    nx, ny, nz = shape_xyz
    dx, dy = _dops(shape_xyz, lens)
    k = _f32(np.sqrt, -dx)
    ne = namp * float(np.sqrt(np.float32(nx * ny * nz)))
    a, b = kop.real, kop.imag
    new = kpsi * a - dx * knl * b
    if knoise is not None:
        new = new - ne * k * knoise * b
    if with_fen:
        return new, ((2.0 - eps) + 2.0 * dx + dy) * kpsi
    return new


def update_el(kpsi, knl, dt, eps, lens, shape_xyz):
    """kernel_update_el (el.hpp:3-25): (psi^ - dt N^)/(1 + dt((2 - eps) + 2 dop.x + dop.y)),
    and max_k |psi^' - psi^| (call_kernel_update_el, el.hpp:26-45)."""
    dx, dy = _dops(shape_xyz, lens)
    new = (kpsi - dt * knl) / (1.0 + dt * ((2.0 - eps) + 2.0 * dx + dy))
    return new, float(np.max(np.abs(kpsi - new)))


def init_el_op(shape_xyz, lens, dt, eps):
    """kernel_init_el_op (el-exp.hpp:3-9): exp(-L dt) + i (exp(-L dt) - 1)/L, L = (2-eps) + 2 dop.x + dop.y."""
    dx, dy = _dops(shape_xyz, lens)
    lin = (2.0 - eps) + 2.0 * dx + dy
    e = _f32(np.exp, -lin * dt)
    return e + 1j * (e - 1.0) / lin


def update_el_exp(kop, kpsi, knl):
    """kernel_update_el of el-exp.hpp:17-40: kop.x psi^ + kop.y N^, and the largest change."""
    new = kpsi * kop.real + knl * kop.imag
    return new, float(np.max(np.abs(kpsi - new)))


PY_COEFFS = (-57.94636917114257, 164.4074088310241, -181.1481995196213, 100.6942650417575,
             -30.20985042718309, 4.678065276755401, -0.293423255328944)  # c0, c2, ..., c12 (eom.hpp:143-149)


def update_eom_py(kpsi, knl, knoise, namp, dt, eps, lens, shape_xyz):
    """kernel_update_eom_py (eom.hpp:151-176): denominator 1 - dt dop.x (1 - eps - P(k^2))."""
    nx, ny, nz = shape_xyz
    dx, _ = _dops(shape_xyz, lens)
    k2 = -dx
    p = np.full_like(k2, PY_COEFFS[-1])
    for c in PY_COEFFS[-2::-1]:
        p = p * k2 + c
    denom = 1.0 - dt * dx * (1.0 - eps - p)
    ne = namp * float(np.sqrt(np.float32(nx * ny * nz)))
    num = kpsi + dt * dx * knl
    if knoise is not None:
        num = num + dt * ne * _f32(np.sqrt, k2) * knoise
    return num / denom


def update_eom_hpfcnoise(kpsi, knl, n1, n2, n3, namp, dt, eps, lens, shape_xyz, dtype=np.float64):
    """kernel_update_eom_hpfcnoise (eom.hpp:16-44), 2D: the noise
    (c1 kx^2 + c2 ky^2) xi1 + (c2 kx^2 + c1 ky^2) xi2 + 2 kx ky xi3 for |k| <= 0.25, kappa = 4/3,
    c2 = sqrt(1 + kappa/2 + sqrt(1 + kappa)), c1 = kappa / (2 c2): kappa and the sums in the
    field's precision (dtype), both square roots in single precision (sqrtf)."""
    nx, ny, nz = shape_xyz
    t = np.dtype(dtype).type
    kappa = t(4.0) / t(3.0)
    inner = t(np.sqrt(np.float32(t(1.0) + kappa)))
    c2 = t(np.sqrt(np.float32(t(1.0) + kappa / t(2.0) + inner)))
    c1 = float(kappa / c2 / t(2.0))
    c2 = float(c2)
    k0 = wavenumbers(nx, lens[0], half=True)[None, None, :]
    k1 = wavenumbers(ny, lens[1])[None, :, None]
    dx, dy = _dops(shape_xyz, lens)
    k = _f32(np.sqrt, -dx)
    denom = 1.0 - dt * ((2.0 - eps) * dx + 2.0 * dy + dx * dy)
    noise = (c1 * k0 * k0 + c2 * k1 * k1) * n1 + (c2 * k0 * k0 + c1 * k1 * k1) * n2 + 2.0 * k0 * k1 * n3
    noise = np.where(k <= 0.25, noise, 0.0)
    ne = namp * float(np.sqrt(np.float32(nx * ny * nz)))
    return (kpsi + dt * dx * knl + dt * ne * noise) / denom


# ----------------------------------------------------------------------------------
# reverse mode of the step (no reference counterpart; pinned by finite differences of
# step() in the tests)
# ----------------------------------------------------------------------------------
def half_weights(shape_xyz):
    """w_k on the half spectrum: 2 for 0 < i0 < nx/2 (the mode and its mirror), else 1."""
    nx, ny, nz = shape_xyz
    i0 = np.arange(nx // 2 + 1)
    w = np.where((i0 == 0) | ((nx % 2 == 0) & (i0 == nx // 2)), 1.0, 2.0)
    return np.broadcast_to(w[None, None, :], cmpl_shape(shape_xyz))


def sf_loss(kpsi, s_target, shape_xyz):
    """L = sum over the full spectrum of (|psi^|^2/N - s)^2 and lam_T = dL/dpsi_T =
    (4/N) C2R(r psi^), r = |psi^|^2/N - s (unnormalised C2R)."""
    n = float(np.prod(shape_xyz))
    k = kpsi.astype(np.complex128)
    r = (k.real ** 2 + k.imag ** 2) / n - s_target
    loss = float(np.sum(half_weights(shape_xyz) * r * r))
    return loss, c2r((4.0 / n) * r * k, shape_xyz)


def adjoint_step(kpsi_n, kpsi_np1, lam, dt, eps, lens, shape_xyz, C=1.0):
    """lam_n = M lam_{n+1} - (3 psi_n^2 - C) K lam_{n+1}, M = F^-1 D^-1 F,
    K = F^-1 (dt k^2 / D) F, and this step's dL/deps = (1/N) sum_k w_k
    Re(conj(lam^_{n+1}) (dt k^2 / D) psi^_{n+1}); D as in update_eom."""
    n = float(np.prod(shape_xyz))
    k2 = kgrid(shape_xyz, lens)
    D = 1.0 + dt * k2 * (C - eps + (1.0 - k2) ** 2)
    kf = dt * k2 / D
    lh = r2c(lam.astype(np.float64))
    deps = float(np.sum(half_weights(shape_xyz) * np.real(np.conj(lh) * kf * kpsi_np1))) / n
    A = c2r(lh / D, shape_xyz) / n
    B = c2r(kf * lh, shape_xyz) / n
    psi = c2r(kpsi_n.astype(np.complex128), shape_xyz) / n
    return A - (3.0 * psi * psi - C) * B, deps


def sf_loss_grads(psi_init, nsteps, s_target, dt, eps, lens, shape_xyz, C=1.0, mu=0.0):
    """(L, dL/dpsi_init, dL/deps) of nsteps of step() in FP64, storing every state."""
    states = [r2c(psi_init.astype(np.float64))]
    for _ in range(nsteps):
        states.append(step(states[-1], 1, dt, eps, lens, shape_xyz, mu=mu, C=C))
    loss, lam = sf_loss(states[-1], s_target, shape_xyz)
    deps = 0.0
    for t in range(nsteps - 1, -1, -1):
        lam, d = adjoint_step(states[t], states[t + 1], lam, dt, eps, lens, shape_xyz, C=C)
        deps += d
    return loss, lam, deps


# ----------------------------------------------------------------------------------
# Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as
# 1, 2, 3", SC'11) -- vectorised over numpy uint64 lanes holding 32-bit words.
# ----------------------------------------------------------------------------------
PHILOX_M0 = 0xD2511F53
PHILOX_M1 = 0xCD9E8D57
PHILOX_W0 = 0x9E3779B9
PHILOX_W1 = 0xBB67AE85
MASK32 = 0xFFFFFFFF


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32 with 10 rounds; inputs are arrays/ints of 32-bit words."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint64) & MASK32 for c in (c0, c1, c2, c3))
    k0 = np.asarray(k0, dtype=np.uint64) & MASK32
    k1 = np.asarray(k1, dtype=np.uint64) & MASK32
    m0 = np.uint64(PHILOX_M0)
    m1 = np.uint64(PHILOX_M1)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(PHILOX_W0)) & MASK32
            k1 = (k1 + np.uint64(PHILOX_W1)) & MASK32
        p0 = m0 * c0
        p1 = m1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK32, lo1, (hi0 ^ c3 ^ k1) & MASK32, lo0
    return c0, c1, c2, c3


def _u01_f32(r):
    """(2*(r>>9)+1) * 2^-24: exact in float32, strictly inside (0, 1)."""
    return ((r >> np.uint64(9)) * np.uint64(2) + np.uint64(1)).astype(np.float64) * 2.0 ** -24


def _u01_f64(hi, lo):
    """(2*((hi:lo)>>12)+1) * 2^-53: exact in float64, strictly inside (0, 1)."""
    v = ((hi << np.uint64(32)) | lo) >> np.uint64(12)
    return (v * np.uint64(2) + np.uint64(1)).astype(np.float64) * 2.0 ** -53


KSPACE_DOMAIN = 0x0          # key word-1 xor for k-space noise
REAL_DOMAIN = 0x52454131     # key word-1 xor for real-space noise ("REA1")
HPFC_DOMAIN = 0x48504600     # + 1, 2, 3: the three k-space fields of the anisotropic 2D noise


def _normals(idx, seed, counter, domain, f64):
    seed = int(seed)
    counter = int(counter)
    idx = np.asarray(idx, dtype=np.uint64)
    r0, r1, r2, r3 = philox4x32_10(idx & MASK32, idx >> np.uint64(32),
                                   counter & MASK32, (counter >> 32) & MASK32,
                                   seed & MASK32, ((seed >> 32) & MASK32) ^ domain)
    if f64:
        u1, u2 = _u01_f64(r0, r1), _u01_f64(r2, r3)
    else:
        u1, u2 = _u01_f32(r0), _u01_f32(r1)
    rad = np.sqrt(-2.0 * np.log(u1))
    return rad * np.cos(2.0 * np.pi * u2), rad * np.sin(2.0 * np.pi * u2)


def fill_kspace(shape_xyz, seed, counter, dtype=np.float32, domain=KSPACE_DOMAIN):
    """Hermitian-consistent complex normal k-space noise, E|xi|^2 = 1 (see module doc);
    domain: the key word-1 xor of the stream."""
    nx, ny, nz = shape_xyz
    nxh = nx // 2 + 1
    f64 = np.dtype(dtype) == np.float64
    i2, i1, i0 = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nxh), indexing="ij")
    lin = ((i2 * ny + i1) * nxh + i0).astype(np.int64)
    on_plane = (i0 == 0) | ((nx % 2 == 0) & (i0 == nx // 2))
    partner = ((((nz - i2) % nz) * ny + (ny - i1) % ny) * nxh + i0).astype(np.int64)
    canon = np.where(on_plane, np.minimum(lin, partner), lin)
    conj = on_plane & (lin > partner)
    selfc = on_plane & (lin == partner)
    g1, g2 = _normals(canon.ravel(), seed, counter, domain, f64)
    g1 = g1.reshape(lin.shape)
    g2 = g2.reshape(lin.shape)
    s = 1.0 / math.sqrt(2.0)
    re = np.where(selfc, g1, g1 * s)
    im = np.where(selfc, 0.0, np.where(conj, -g2 * s, g2 * s))
    out = re + 1j * im
    return out.astype(np.complex128 if f64 else np.complex64)


def fill_real(n, sigma, seed, counter, dtype=np.float32):
    """Real-space normal noise N(0, sigma^2) -- the contract of NoiseHostApi::fill (noise.hpp:108)."""
    f64 = np.dtype(dtype) == np.float64
    g1, _ = _normals(np.arange(n, dtype=np.uint64), seed, counter, REAL_DOMAIN, f64)
    return (g1 * sigma).astype(dtype)


# ----------------------------------------------------------------------------------
# the step
# ----------------------------------------------------------------------------------
def py_poly(k2):
    """The degree-6 polynomial in k^2 of kernel_update_eom_py (eom.hpp:143-149), Horner."""
    d = np.full_like(k2, PY_COEFFS[-1])
    for ci in PY_COEFFS[-2::-1]:
        d = d * k2 + ci
    return d


def hpfc_noise(fields, shape_xyz, lens):
    """The anisotropic 2D noise of kernel_update_eom_hpfcnoise (eom.hpp:16-58) from three
    k-space fields: (c1 kx^2 + c2 ky^2) xi1 + (c2 kx^2 + c1 ky^2) xi2 + 2 kx ky xi3, zero
    for |k| > 1/4; kappa = 4/3, c2 = sqrt(1 + kappa/2 + sqrt(1 + kappa)), c1 = kappa/(2 c2)."""
    nx, ny, nz = shape_xyz
    kappa = 4.0 / 3.0
    c2 = math.sqrt(1.0 + kappa / 2.0 + math.sqrt(1.0 + kappa))
    c1 = kappa / c2 / 2.0
    k0 = wavenumbers(nx, lens[0], half=True)[None, None, :]
    k1 = wavenumbers(ny, lens[1])[None, :, None]
    a, b, c = (f.astype(np.complex128) for f in fields)
    out = (c1 * k0 ** 2 + c2 * k1 ** 2) * a + (c2 * k0 ** 2 + c1 * k1 ** 2) * b + 2.0 * k0 * k1 * c
    return np.where(np.sqrt(kgrid(shape_xyz, lens)) <= 0.25, out, 0.0)


def propagate(kpsi, knl, knoise, namp, dt, eps, lens, shape_xyz, C, propagator):
    """One update of the fused stepper's other propagators, in full precision (the fused
    kernels evaluate exp in the field's precision), with the stabilisation C
    (deps = 1 + C - eps; C = 1 is the reference's split):
      "conserved_exp"  eom-exp.hpp:3-60   psi^' = E psi^ - dop.x Q N^ - namp sqrt(N) |k| Q xi^,
                       L = -dop.x (deps + 2 dop.x + dop.y), E = exp(-L dt), Q = (E-1)/L (-dt at L = 0)
      "relax"          el.hpp:3-25         psi^' = (psi^ - dt N^) / (1 + dt (deps + 2 dop.x + dop.y))
      "relax_exp"      el-exp.hpp:3-40     psi^' = E psi^ + Q N^, L = deps + 2 dop.x + dop.y
      "conserved_poly" eom.hpp:143-180     psi^' = (psi^ + dt dop.x N^ + dt namp sqrt(N) |k| xi^)
                       / (1 - dt dop.x (C - eps - P(k^2)))
      "conserved_hpfc" eom.hpp:16-58       the conserved update with the anisotropic noise of
                       hpfc_noise (knoise: its three fields) in place of |k| xi^
    Returns (psi^', max_k |psi^' - psi^|)."""
    dx, dy = _dops(shape_xyz, lens)
    deps = 1.0 + C - eps
    if propagator == "conserved_exp":
        lin = -dx * (deps + 2.0 * dx + dy)
        e = np.exp(-lin * dt)
        with np.errstate(invalid="ignore", divide="ignore"):
            q = (e - 1.0) / lin
        q = np.where(np.isnan(q), -dt, q)
        new = e * kpsi - dx * q * knl
        if knoise is not None:
            nx, ny, nz = shape_xyz
            new = new - namp * np.sqrt(float(nx * ny * nz)) * np.sqrt(-dx) * q * knoise
    elif propagator == "relax":
        new = (kpsi - dt * knl) / (1.0 + dt * (deps + 2.0 * dx + dy))
    elif propagator == "relax_exp":
        lin = deps + 2.0 * dx + dy
        e = np.exp(-lin * dt)
        with np.errstate(invalid="ignore", divide="ignore"):
            q = (e - 1.0) / lin
        new = e * kpsi + np.where(np.isnan(q), -dt, q) * knl
    elif propagator == "conserved_poly":
        denom = 1.0 - dt * dx * (deps - 1.0 - py_poly(-dx))
        new = kpsi + dt * dx * knl
        if knoise is not None:
            nx, ny, nz = shape_xyz
            new = new + dt * namp * np.sqrt(float(nx * ny * nz)) * np.sqrt(-dx) * knoise
        new = new / denom
    elif propagator == "conserved_hpfc":
        denom = 1.0 - dt * (deps * dx + 2.0 * dy + dx * dy)
        new = kpsi + dt * dx * knl
        if knoise is not None:
            nx, ny, nz = shape_xyz
            new = new + dt * namp * np.sqrt(float(nx * ny * nz)) * hpfc_noise(knoise, shape_xyz, lens)
        new = new / denom
    else:
        raise ValueError(propagator)
    return new, float(np.max(np.abs(new - kpsi)))


def step(kpsi, nsteps, dt, eps, lens, shape_xyz, mu=0.0, C=1.0, namp=0.0,
         seed=0, counter0=0, workers=None, dtype=np.float64, noise_dtype=None, ref_float_sqrt=False,
         propagator="conserved", return_max_change=False):
    """nsteps steps of the driver loop of the reference (copy, C2R, psi3_split(norm=True),
    R2C, [fill_kspace], update): the conserved semi-implicit update (eom.hpp:60-72) or,
    with `propagator`, one of the updates of ``propagate``.  noise_dtype selects the
    precision of the Philox draw (that of the field being compared); the fused stepper
    evaluates sqrt(N) and |k| in full precision, hence ref_float_sqrt=False by default
    here.  return_max_change: also return the last step's max_k |psi^' - psi^|."""
    real_t = np.dtype(dtype)
    cmpl_t = np.complex128 if real_t == np.float64 else np.complex64
    noise_t = real_t if noise_dtype is None else np.dtype(noise_dtype)
    kpsi = kpsi.astype(cmpl_t)
    change = 0.0
    for t in range(nsteps):
        psi = c2r(kpsi, shape_xyz, workers=workers).astype(real_t)
        nl = psi3_split(psi, None, mu, norm=True, C=C).astype(real_t)
        knl = r2c(nl, workers=workers).astype(cmpl_t)
        knoise = None
        if namp != 0.0 and propagator == "conserved_hpfc":
            knoise = tuple(fill_kspace(shape_xyz, seed, counter0 + t, dtype=noise_t, domain=HPFC_DOMAIN + i)
                           for i in (1, 2, 3))
        elif namp != 0.0:
            knoise = fill_kspace(shape_xyz, seed, counter0 + t, dtype=noise_t)
        if propagator == "conserved":
            new = update_eom(kpsi, knl, knoise, namp, dt, eps, lens, shape_xyz, C=C, ref_float_sqrt=ref_float_sqrt)
        else:
            new, change = propagate(kpsi.astype(np.complex128), knl.astype(np.complex128), knoise, namp, dt, eps,
                                    lens, shape_xyz, C, propagator)
        kpsi = new.astype(cmpl_t)
    return (kpsi, change) if return_max_change else kpsi


# ----------------------------------------------------------------------------------
# peaks
# ----------------------------------------------------------------------------------
MAX_DTYPE = {
    np.float32: np.dtype([("i0", "<f4"), ("i1", "<f4"), ("i2", "<f4"), ("field", "<f4")]),
    np.float64: np.dtype([("i0", "<f8"), ("i1", "<f8"), ("i2", "<f8"), ("field", "<f4")], align=True),
}


def _peaks(psi, ths, offsets):
    peak = np.ones(psi.shape, dtype=bool)
    for off in offsets:
        peak &= psi > np.roll(psi, shift=tuple(-o for o in off), axis=tuple(range(psi.ndim)))
    peak &= psi >= ths
    return peak


def findpeaks3d(psi, ths):
    """Strict 26-neighbour periodic local maxima with psi >= ths (findpeaks.hpp:7-29).
    psi has numpy shape (nz, ny, nx); returns (i0, i1, i2, field) rows sorted by linear index."""
    offs = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1) if (a, b, c) != (0, 0, 0)]
    mask = _peaks(psi, ths, offs)
    i2, i1, i0 = np.nonzero(mask)
    return np.stack([i0, i1, i2], axis=1), psi[mask]


def findpeaks2d(psi, ths):
    """Strict 8-neighbour periodic local maxima (findpeaks_2d.hpp:7-27); psi shape (ny, nx)."""
    offs = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1) if (a, b) != (0, 0)]
    mask = _peaks(psi, ths, offs)
    i1, i0 = np.nonzero(mask)
    return np.stack([i0, i1, np.zeros_like(i0)], axis=1), psi[mask]


# ----------------------------------------------------------------------------------
# Steinhardt bond order (bond-order-analysis/bond-order.cpp)
# ----------------------------------------------------------------------------------
def min_image(d1, w):
    """get_diff (bond-order.cpp:53-64): among d, d-w, d+w the smallest |.|, with the
    reference's tie order (d before d+w only if strictly smaller, etc.)."""
    d2 = d1 - w
    d3 = d1 + w
    a1, a2, a3 = np.abs(d1), np.abs(d2), np.abs(d3)
    return np.where(a1 < a2, np.where(a1 < a3, d1, d3), np.where(a2 < a3, d2, d3))


def _fact(n):
    return math.factorial(n)


def assoc_legendre_norm(l, x):
    """Normalised associated Legendre functions with Condon-Shortley phase,
    N_lm P_l^m(x) for m = 0..l, N_lm = sqrt((2l+1)/(4pi) (l-m)!/(l+m)!), evaluated by
    the standard upward recurrences in m and l (the published stable method)."""
    x = np.asarray(x, dtype=np.float64)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    out = []
    for m in range(l + 1):
        # P_m^m = (-1)^m (2m-1)!! s^m, normalised
        pmm = np.ones_like(x)
        fact = 1.0
        for _ in range(m):
            pmm = -pmm * fact * s
            fact += 2.0
        if l == m:
            p = pmm
        else:
            pmmp1 = x * (2 * m + 1) * pmm
            if l == m + 1:
                p = pmmp1
            else:
                pll = None
                for ll in range(m + 2, l + 1):
                    pll = (x * (2 * ll - 1) * pmmp1 - (ll + m - 1) * pmm) / (ll - m)
                    pmm, pmmp1 = pmmp1, pll
                p = pll
        nlm = math.sqrt((2 * l + 1) / (4 * math.pi) * _fact(l - m) / _fact(l + m))
        out.append(nlm * p)
    return out


POLE_BAND = 1e-3  # bond-order.cpp:123-133: Y_lm is set to 0 for m>0 (m<0) when |1-x| (|1+x|) < 1e-3


def ylm_all(l, cos_theta, phi):
    """Y_l^m(theta, phi), m = -l..l, shape (2l+1, n); Y_l^{-m} = (-1)^m conj(Y_l^m).
    Includes the reference's pole band (prefF in bond-order.cpp:123-133)."""
    x = np.asarray(cos_theta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    plm = assoc_legendre_norm(l, x)
    res = np.zeros((2 * l + 1,) + x.shape, dtype=np.complex128)
    north = np.abs(1.0 - x) < POLE_BAND
    south = np.abs(1.0 + x) < POLE_BAND
    for m in range(l + 1):
        ypos = plm[m] * np.exp(1j * m * phi)
        if m == 0:
            res[l] = ypos
            continue
        yneg = (-1) ** m * np.conj(ypos)
        res[l + m] = np.where(north, 0.0, ypos)
        res[l - m] = np.where(south, 0.0, yneg)
    return res


def wigner3j_lll(l):
    """All (l l l; m1 m2 m3) with m1+m2+m3 = 0 from the Racah formula, exact rationals
    under the square root, returned as {(m1, m2, m3): float}."""
    def tri(a, b, c):
        return Fraction(_fact(a + b - c) * _fact(a - b + c) * _fact(-a + b + c), _fact(a + b + c + 1))

    out = {}
    for m1 in range(-l, l + 1):
        for m2 in range(-l, l + 1):
            m3 = -m1 - m2
            if abs(m3) > l:
                continue
            j1 = j2 = j3 = l
            pref2 = tri(j1, j2, j3) * _fact(j1 + m1) * _fact(j1 - m1) * _fact(j2 + m2) * _fact(j2 - m2) \
                * _fact(j3 + m3) * _fact(j3 - m3)
            kmin = max(0, j2 - j3 - m1, j1 - j3 + m2)
            kmax = min(j1 + j2 - j3, j1 - m1, j2 + m2)
            ssum = Fraction(0)
            for k in range(kmin, kmax + 1):
                den = _fact(k) * _fact(j1 + j2 - j3 - k) * _fact(j1 - m1 - k) * _fact(j2 + m2 - k) \
                    * _fact(j3 - j2 + m1 + k) * _fact(j3 - j1 - m2 + k)
                ssum += Fraction((-1) ** k, den)
            sign = (-1) ** (j1 - j2 - m3)
            out[(m1, m2, m3)] = float(sign * math.sqrt(pref2) * ssum)
    return out


def _wl(qlm, l, w3j):
    """w_l = sum_{m1+m2+m3=0} (l l l; m1 m2 m3) q_m1 q_m2 q_m3 / (sum |q_m|^2)^(3/2)."""
    csum = np.zeros(qlm.shape[1:], dtype=np.complex128)
    for (m1, m2, m3), w in w3j.items():
        csum += w * qlm[m1 + l] * qlm[m2 + l] * qlm[m3 + l]
    ss = np.sum(np.abs(qlm) ** 2, axis=0)
    return csum.real / np.sqrt(ss ** 3)


def _ql(qlm, l):
    return np.sqrt(4.0 * math.pi / (2 * l + 1) * np.sum(np.abs(qlm) ** 2, axis=0))


BOND_COLUMNS = ("x", "y", "z", "nb", "xi", "q4", "q6", "q8", "w4", "q4b", "q6b", "q8b", "w4b", "w6")


def bond_order(idx, field, h, ths, boxsize, rlim):
    """Restatement of bond_order_analysis (bond-order.cpp:289-349) plus w6 (not in the
    reference).  idx: (P, 3) integer grid indices (i0, i1, i2); field: (P,).
    Returns a dict of per-atom columns (atoms with at least one neighbour, in input
    order) -- the rows the reference prints -- and the neighbour lists."""
    keep = np.asarray(field) > ths
    pos = np.asarray(idx, dtype=np.float64)[keep] * np.asarray(h, dtype=np.float64)[None, :]
    p = pos.shape[0]
    nbrs, cts, phis = [], [], []
    for i in range(p):
        d = min_image(pos[:, :] - pos[i][None, :], boxsize)
        r = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        sel = (r <= rlim)
        sel[i] = False
        j = np.nonzero(sel)[0]
        nbrs.append(j)
        cts.append(d[j, 2] / r[j])
        phis.append(np.arctan2(d[j, 1], d[j, 0]))
    nb = np.array([len(j) for j in nbrs], dtype=np.int64)
    q = {}
    for l in (4, 6, 8):
        ql = np.zeros((2 * l + 1, p), dtype=np.complex128)
        for i in range(p):
            if nb[i] > 0:
                ql[:, i] = ylm_all(l, cts[i], phis[i]).sum(axis=1) / nb[i]
        q[l] = ql
    w4j = wigner3j_lll(4)
    w6j = wigner3j_lll(6)
    res = {c: np.zeros(p) for c in BOND_COLUMNS}
    res["x"], res["y"], res["z"] = pos[:, 0], pos[:, 1], pos[:, 2]
    res["nb"] = nb
    with np.errstate(invalid="ignore", divide="ignore"):
        for l, name in ((4, "q4"), (6, "q6"), (8, "q8")):
            res[name] = _ql(q[l], l)
        res["w4"] = _wl(q[4], 4, w4j)
        res["w6"] = _wl(q[6], 6, w6j)
        xi = np.zeros(p, dtype=np.int64)
        qbar = {l: np.zeros_like(q[l]) for l in (4, 6, 8)}
        w4b = np.zeros(p)
        for i in range(p):
            if nb[i] == 0:
                continue
            for l in (4, 6, 8):
                qbar[l][:, i] = (q[l][:, i] + q[l][:, nbrs[i]].sum(axis=1)) / (1.0 + nb[i])
            # w4b as the reference computes it (bond-order.cpp:205-219): the average is
            # overwritten by the last neighbour's q4m, then divided by Nb.
            last = q[4][:, nbrs[i][-1]] / float(nb[i])
            w4b[i] = _wl(last[:, None], 4, w4j)[0]
            n6i = np.sqrt(np.sum(np.abs(q[6][:, i]) ** 2))
            dots = (q[6][:, i][:, None] * np.conj(q[6][:, nbrs[i]])).sum(axis=0).real
            n6j = np.sqrt(np.sum(np.abs(q[6][:, nbrs[i]]) ** 2, axis=0))
            xi[i] = int(np.sum(dots / (n6i * n6j) > 0.7))
        res["q4b"], res["q6b"], res["q8b"] = _ql(qbar[4], 4), _ql(qbar[6], 6), _ql(qbar[8], 8)
        res["w4b"] = w4b
        res["xi"] = xi
    has = nb > 0
    return {c: np.asarray(v)[has] for c, v in res.items()}, [nbrs[i] for i in range(p) if has[i]]


def format_bond_table(res):
    """The reference's text table (bond-order.cpp:333-338) for the first 13 columns."""
    lines = ["# x y z #nb xi q4 q6 q8 w4 q4b q6b q8b w4b"]
    for r in range(len(res["nb"])):
        lines.append("%.6f\t%.6f\t%.6f\t%d\t%d\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f" % (
            res["x"][r], res["y"][r], res["z"][r], res["nb"][r], res["xi"][r], res["q4"][r],
            res["q6"][r], res["q8"][r], res["w4"][r], res["q4b"][r], res["q6b"][r], res["q8b"][r],
            res["w4b"][r]))
    return "\n".join(lines) + "\n"


def parse_bond_table(text):
    rows = [ln.split() for ln in text.splitlines() if ln and not ln.startswith("#")]
    arr = np.array([[float(v) for v in r] for r in rows]) if rows else np.zeros((0, 13))
    return {c: arr[:, i] for i, c in enumerate(BOND_COLUMNS[:13])}


# ----------------------------------------------------------------------------------
# spectral low-pass post-processing of 2D fields (cuda/kernels/gaussian.hpp,
# cuda/kernels/lowpass.hpp)
# ----------------------------------------------------------------------------------
def gaussian_init(shape_xyz, lens, hh, divs_per_sigma, dtype=np.float64):
    """``kernel_gaussian_init`` (gaussian.hpp:23-33): g = e + i (1 - e) with
    e = exp(-1/2 sum_a (1.1 d h_a K_a)^2), evaluated in ``dtype`` (the reference's Float)."""
    nx, ny, nz = shape_xyz
    f = dtype
    s = [f(1.1) * f(divs_per_sigma) * f(h) for h in hh]
    a = s[0] * wavenumbers(nx, lens[0], half=True, dtype=f)
    b = s[1] * wavenumbers(ny, lens[1], dtype=f)
    c = s[2] * wavenumbers(nz, lens[2], dtype=f)
    q = (a[None, None, :] * a[None, None, :] + b[None, :, None] * b[None, :, None]) + c[:, None, None] * c[:, None, None]
    e = np.exp(f(-0.5) * q.astype(f)).astype(f)
    out = np.empty(e.shape, dtype=np.complex64 if f == np.float32 else np.complex128)
    out.real, out.imag = e, f(1) - e
    return out


def kmult(karr, kgauss, imag=False):
    """``kernel_kmult_real`` / ``_imag`` (gaussian.hpp:41-67; lowpass.hpp:1-35): the
    complex field times the real or imaginary part of kgauss."""
    return karr * (kgauss.imag if imag else kgauss.real)


def amplitude_lowpass(kpsi, kgauss, shape_xyz):
    """``calc_amplitude_lowpass`` (lowpass.hpp:78-93) in FP64: high-pass, C2R, normalise,
    square, R2C, low-pass (the spectrum the LOWPASS dump writes), C2R, normalise.
    Returns (amplitude field, numpy shape (ny, nx) for a 2D grid; low-passed spectrum)."""
    rs = real_shape(shape_xyz)
    n = rs[0] * rs[1] * rs[2]
    k = np.asarray(kpsi, dtype=np.complex128) * np.asarray(kgauss.imag, dtype=np.float64)
    a = c2r(k, shape_xyz) / n
    low = r2c(a * a) * np.asarray(kgauss.real, dtype=np.float64)
    return c2r(low, shape_xyz) / n, low


def lowpass_text(spectrum, nx, ny, lx, ly, dtype=np.float32):
    """The LOWPASS dump of ``write_lowpass_2d`` (lowpass.hpp:54-77) before compression:
    "LOWPASS\\n<len>\\n", a protocol-0 pickle of {n0, n1, l0, l1} of that length, then
    "i0 i1 re im\\n" for every mode with re^2 + im^2 > 1e-6 (evaluated in ``dtype``), i0 in
    the outer loop, values in iostream's default format (%g, 6 significant digits)."""
    f = dtype
    pickle = "(S'n0'\nI%d\nS'n1'\nI%d\nS'l0'\nF%f\nS'l1'\nF%f\nd.\n" % (nx, ny, float(f(lx)), float(f(ly)))
    out = ["LOWPASS\n%d\n" % len(pickle), pickle]
    sp = np.asarray(spectrum).reshape(ny, nx // 2 + 1)
    re = sp.real.astype(f)
    im = sp.imag.astype(f)
    m = (re * re + im * im).astype(f)
    for i0 in range(nx // 2 + 1):
        for i1 in range(ny):
            if float(m[i1, i0]) > 1e-6:
                out.append("%d %d %g %g\n" % (i0, i1, float(re[i1, i0]), float(im[i1, i0])))
    return "".join(out).encode()
