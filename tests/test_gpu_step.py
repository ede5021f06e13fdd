"""Parity of the fused conserved stepper (pfc_step through the C ABI) with the oracle
and with the reference's own cuFFT step (oracle/_ref), plus the known answers derived
from the reference's mathematics."""
import math

import numpy as np
import pytest
import torch

import pfc_oracle as O
from conftest import ref_lib

pytestmark = pytest.mark.gpu

F32, F64 = np.float32, np.float64


def stepper(shape, dtype, dx=math.pi / 4, dt=0.5, eps=0.3, namp=0.0, seed=0, C=1.0, mu=0.0):
    from mcstar_b200 import Stepper
    return Stepper(shape, dx, dt, eps, dtype=dtype, namp=namp, seed=seed, C=C, mu=mu)


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


CASES = [
    ((16, 12, 10), F64, 0.0), ((16, 12, 10), F64, 0.05), ((15, 9, 7), F64, 0.0), ((24, 20, 1), F64, 0.0),
    ((64, 1, 1), F64, 0.0), ((32, 32, 32), F32, 0.0), ((32, 32, 32), F32, 0.02), ((64, 64, 64), F32, 0.0),
    ((128, 128, 128), F32, 0.0), ((256, 256, 1), F64, 0.0), ((48, 40, 30), F32, 0.0),
    # every fused plane-kernel variant (FP32, nx = ny in {64, 128, 256, 512})
    ((64, 64, 16), F32, 0.05), ((128, 128, 8), F32, 0.0), ((256, 256, 12), F32, 0.02), ((512, 512, 6), F32, 0.0),
    ((512, 512, 1), F32, 0.0),
    # every register z-kernel variant (nz in {64, 128, 256, 512}), with and without noise,
    # including a partial last tile of kx columns (nx/2 + 1 = 17)
    ((16, 16, 512), F32, 0.03), ((16, 8, 512), F32, 0.0), ((32, 32, 256), F32, 0.02), ((32, 16, 128), F32, 0.05),
    ((64, 64, 64), F32, 0.02),
    # the kx-tiled carry (register y, x and z passes; partial last tile of one column)
    ((64, 64, 512), F32, 0.02), ((128, 64, 256), F32, 0.0), ((64, 128, 128), F32, 0.03),
    # the 3 2^k and 5 2^k register kernels (radix-3 or radix-5 first stage; x, y, z lengths
    # 96, 160 and 192, mixed), tiled, and 2D fields through their y and x passes
    ((192, 192, 192), F32, 0.02), ((96, 96, 96), F32, 0.0), ((96, 192, 96), F32, 0.03), ((192, 96, 192), F32, 0.0),
    ((192, 192, 1), F32, 0.02), ((96, 96, 64), F32, 0.0), ((160, 160, 160), F32, 0.02), ((160, 96, 192), F32, 0.0),
    ((160, 160, 1), F32, 0.0), ((1024, 1024, 1), F32, 0.02),
]


@pytest.mark.parametrize("shape,dtype,namp", CASES, ids=lambda v: str(v))
def test_step_matches_oracle(shape, dtype, namp):
    nx, ny, nz = shape
    st = stepper(shape, dtype, namp=namp, seed=17)
    psi = O.r2c(np.full((nz, ny, nx), -0.2) + 0.1 * np.random.default_rng(1).uniform(-1, 1, (nz, ny, nx)))
    st.set_kspace(psi.astype(np.complex64 if dtype == F32 else np.complex128))
    nsteps = 6
    st.step(nsteps)
    got = st.kspace()
    want = O.step(psi, nsteps, st.dt, st.eps, st.lens, shape, namp=namp, seed=17, counter0=0, noise_dtype=dtype)
    tol = 2e-6 if dtype == F32 else 1e-12
    assert rel_l2(got, want) < tol


VARIANT_SHAPES = [((64, 64, 64), 0.02), ((128, 128, 16), 0.0), ((32, 16, 128), 0.05), ((256, 256, 8), 0.0),
                  ((512, 512, 4), 0.0), ((16, 16, 512), 0.03), ((16, 8, 512), 0.0), ((64, 64, 512), 0.02),
                  ((128, 64, 512), 0.0), ((512, 64, 64), 0.02), ((512, 128, 64), 0.0), ((128, 512, 64), 0.02),
                  ((48, 40, 30), 0.02), ((96, 80, 1), 0.0)]
OPTIONS = [dict(z_carry=1), dict(z_carry=0), dict(tiled=0), dict(x_kernel=0), dict(x_kernel=1), dict(x_kernel=2),
           dict(x_kernel=2, z_carry=0), dict(z_carry=1, tiled=0), dict(y_kernel=0),
           dict(radix_order=1), dict(radix_order=2), dict(tile_shift=[1, 2, 1, 2]), dict(tile_shift=[3, 3, 4, 3])]


@pytest.mark.parametrize("options", OPTIONS, ids=lambda o: ",".join(f"{k}={v}" for k, v in o.items()))
def test_step_kernel_schedules_match_oracle(options):
    """Every kernel schedule a context can be made with (pfc_options: the z pass carrying
    psi^ or A, the standard or kx-tiled layout, the three x kernels, the general
    passes' radix order and tiles) computes the same step.  Options a shape has no kernel
    for are refused at creation (PFC_ERR_UNSUPPORTED) and skipped."""
    from mcstar_b200 import PfcError, Stepper
    tried = 0
    for shape, namp in VARIANT_SHAPES:
        nx, ny, nz = shape
        try:
            st = Stepper(shape, math.pi / 4, 0.5, 0.3, dtype=F32, namp=namp, seed=5, options=options)
        except PfcError as e:
            assert e.status == 2, (shape, options, e)
            continue
        tried += 1
        rng = np.random.default_rng(3)
        k = O.r2c(-0.2 + 0.1 * rng.uniform(-1, 1, (nz, ny, nx)))
        st.set_kspace(k.astype(np.complex64))
        st.step(4)
        want = O.step(k, 4, 0.5, 0.3, st.lens, shape, namp=namp, seed=5, noise_dtype=F32)
        assert rel_l2(st.kspace(), want) < 2e-6, (shape, options, st.ctx.options)
        st.ctx.close()
    assert tried >= 3


@pytest.mark.parametrize("y_kernel", [0, 1])
@pytest.mark.parametrize("shape,namp", [((128, 512, 64), 0.02), ((64, 512, 512), 0.0), ((64, 512, 512), 0.03),
                                        ((512, 512, 4), 0.0)])
def test_y_pass_kernels_match_oracle(shape, namp, y_kernel):
    """The two y-pass kernels between the kx-tiled layouts (ny = 512): per-thread accesses
    and the TMA form (a bulk copy of the row-tiled block, tensor-map tiles of the z-tiled
    pieces, the partial last kx tile by per-thread accesses), under the A-carrying
    (nz = 64) and the psi^-carrying (nz = 512) schedules; a shape that is not tiled takes
    the option and runs its own passes."""
    from mcstar_b200 import Stepper
    st = Stepper(shape, math.pi / 4, 0.5, 0.3, dtype=F32, namp=namp, seed=9, options=dict(y_kernel=y_kernel))
    assert st.ctx.options["y_kernel"] == y_kernel
    nx, ny, nz = shape
    k = O.r2c(-0.2 + 0.1 * np.random.default_rng(8).uniform(-1, 1, (nz, ny, nx)))
    st.set_kspace(k.astype(np.complex64))
    st.step(3)
    want = O.step(k, 3, 0.5, 0.3, st.lens, shape, namp=namp, seed=9, noise_dtype=F32)
    assert rel_l2(st.kspace(), want) < 2e-6


@pytest.mark.parametrize("shape,dtype,z_mode", [((64, 64, 64), F32, 3), ((64, 64, 512), F32, 4),
                                                 ((512, 512, 4), F32, 5), ((16, 16, 512), F32, 1),
                                                 ((16, 12, 10), F64, 5), ((96, 80, 1), F32, 0),
                                                 ((192, 192, 192), F32, 3), ((96, 96, 96), F32, 5)])
def test_stepper_layout_mode(shape, dtype, z_mode):
    """FP32 grids with register y, x and z passes run kx-tiled: nz = 512 carries psi^ through
    the bulk-copy z pass (z_mode 4), other lengths carry A (3); the register z pass alone
    keeps the standard layout (1); other shapes use the general z pass carrying psi^ (5),
    and 2D fields (no z transforms) its flat form (0)."""
    assert stepper(shape, dtype).ctx.profile_read()["z_mode"] == z_mode


@pytest.mark.parametrize("shape,dtype", [((64, 64, 64), F32), ((32, 32, 32), F32), ((16, 12, 10), F64)],
                         ids=["register-z", "register-z-32", "general-z"])
def test_nonfinite_state_is_reported_and_context_stays_usable(shape, dtype):
    """A NaN planted in psi^ on the host reaches every mode after one transform; the z
    pass's watchdog flags it and pfc_step returns PFC_ERR_NONFINITE.  The next run on a
    clean state works."""
    from mcstar_b200 import PfcError
    from mcstar_b200._lib import PFC_ERR_NONFINITE
    nx, ny, nz = shape
    psi = -0.2 + 0.05 * np.random.default_rng(2).uniform(-1, 1, (nz, ny, nx))
    st = stepper(shape, dtype)
    st.set_real(psi)
    st.kpsi[10] = float("nan")
    with pytest.raises(PfcError) as err:
        st.step(2)
    assert err.value.status == PFC_ERR_NONFINITE
    st.set_real(psi)
    st.step(2)
    want = O.step(O.r2c(psi), 2, st.dt, st.eps, st.lens, shape)
    assert rel_l2(st.kspace(), want) < (2e-6 if dtype == F32 else 1e-12)


def test_step_stabilisation_constant_and_mu():
    shape = (16, 16, 16)
    st = stepper(shape, F64, C=0.0, mu=0.07, dt=0.1)
    rng = np.random.default_rng(4)
    psi = O.r2c(-0.2 + 0.1 * rng.uniform(-1, 1, (16, 16, 16)))
    st.set_kspace(psi)
    st.step(5)
    want = O.step(psi, 5, 0.1, st.eps, st.lens, shape, mu=0.07, C=0.0)
    assert rel_l2(st.kspace(), want) < 1e-12


@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 64, 64)])
def test_k0_mode_bit_invariant_with_noise(shape):
    st = stepper(shape, F32, namp=0.05, seed=3)
    rng = np.random.default_rng(2)
    st.set_real(-0.18 + 0.05 * rng.uniform(-1, 1, shape[::-1]))
    k0 = st.kspace()[0, 0, 0]
    for _ in range(4):
        st.step(25)
        assert st.kspace()[0, 0, 0] == k0


def test_uniform_state_fixed_point():
    shape = (32, 24, 16)
    st = stepper(shape, F64)
    st.set_real(np.full((16, 24, 32), -0.25))
    k = st.kspace()
    st.step(10)
    np.testing.assert_allclose(st.kspace(), k, atol=1e-9)


@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 64, 64)])
def test_resume_is_bit_exact(shape):
    a = stepper(shape, F32, namp=0.05, seed=9)
    b = stepper(shape, F32, namp=0.05, seed=9)
    rng = np.random.default_rng(5)
    psi = -0.2 + 0.05 * rng.uniform(-1, 1, shape[::-1])
    a.set_real(psi)
    b.set_real(psi)
    a.step(10)
    b.step(4)
    b.step(6)
    np.testing.assert_array_equal(a.kspace(), b.kspace())


@pytest.mark.parametrize("shape,nsteps,namp", [((64, 64, 512), 3, 0.05), ((64, 64, 512), 1, 0.0),
                                               ((128, 64, 512), 2, 0.0), ((32, 24, 20), 3, 0.05)])
def test_step_host_equals_device_step(shape, nsteps, namp):
    """pfc_step_host (the field in pinned host memory, copies by ky chunks overlapped with the
    entry pass and the last z pass; in order where the schedule has no chunked passes) gives
    the bits of copy in + pfc_step + copy out, with host_out distinct from or equal to host_in."""
    a = stepper(shape, F32, namp=namp, seed=4)
    b = stepper(shape, F32, namp=namp, seed=4)
    rng = np.random.default_rng(8)
    a.set_real(-0.2 + 0.05 * rng.uniform(-1, 1, shape[::-1]))
    host_in = a.kpsi.cpu().pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    a.step(nsteps)
    want = a.kpsi.cpu()
    b.step_host(host_in, host_out, nsteps)
    assert torch.equal(host_out, want)
    assert torch.equal(b.kpsi.cpu(), want)
    b.kpsi.zero_()
    b.counter = 0
    b.step_host(host_in, host_in, nsteps)  # in place on the host
    assert torch.equal(host_in, want)


@pytest.mark.parametrize("dtype,shape,nsteps", [(F64, (64, 64, 1), 20), (F64, (16, 16, 16), 20),
                                                 (F32, (64, 64, 64), 20), (F64, (36, 30, 20), 10)])
def test_step_vs_reference_cufft(dtype, shape, nsteps):
    ref = ref_lib(dtype)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    nx, ny, nz = shape
    dx, dt, eps = math.pi / 4, 0.5, 0.25
    lens = (nx * dx, ny * dx, nz * dx)
    rng = np.random.default_rng(11)
    psi = -0.25 + 0.01 * rng.uniform(-1, 1, (nz, ny, nx))
    k = O.r2c(psi).astype(np.complex64 if dtype == F32 else np.complex128)
    h = ref["create"](nx, ny, nz, 1)
    ref["set_kpsi"](h, k.ctypes.data)
    ref["step"](h, nsteps, 0.0, dt, eps, *lens, 0.0, 0)
    want = np.zeros_like(k)
    ref["get_kpsi"](h, want.ctypes.data)
    ref["destroy"](h)
    st = stepper(shape, dtype, dx=dx, dt=dt, eps=eps)
    st.set_kspace(k)
    st.step(nsteps)
    tol = 1e-5 if dtype == F32 else 1e-12
    assert rel_l2(st.kspace(), want) < tol


def test_free_energy_and_peaks_of_stepper_match_reference():
    ref = ref_lib(F64)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    from mcstar_b200 import bcc_sphere
    shape = (32, 32, 32)
    dx = math.pi / 4
    psi = bcc_sphere(shape, dx, -0.2, 0.2, 9.0)
    k = O.r2c(psi)
    h = ref["create"](32, 32, 32, 1)
    ref["set_kpsi"](h, k.ctypes.data)
    ref["step"](h, 10, 0.0, 0.5, 0.3, 32 * dx, 32 * dx, 32 * dx, 0.0, 0)
    f_ref = ref["free_energy"](h, 0.3, 32 * dx, 32 * dx, 32 * dx, dx, dx, dx, None)
    ref["destroy"](h)
    st = stepper(shape, F64, dx=dx)
    st.set_kspace(k)
    st.step(10)
    # the reference returns a float summed with float atomics (eom.hpp:126)
    assert abs(st.free_energy() - f_ref) / abs(f_ref) < 1e-5
