"""The fused stepper with the reference's other update kernels in its propagator slot
(pfc_step_prop): exponential time differencing of the conserved equation (eom-exp.hpp),
the non-conserved relaxation (el.hpp) and its exponential form (el-exp.hpp), the
polynomial correlation function (kernel_update_eom_py) and the anisotropic 2D noise
(kernel_update_eom_hpfcnoise) of eom.hpp.  Each is
checked against the oracle's driver loop (C2R, psi3_split, R2C, update) on every kernel
family of the stepper: the general passes (FP64 and odd shapes), the register passes
(standard and kx-tiled layouts), the 512-point z kernels carrying A or psi^ -- and the
relaxations' largest mode change against the oracle's (call_kernel_update_el)."""
import math

import numpy as np
import pytest

import pfc_oracle as O

pytestmark = pytest.mark.gpu

CASES = [((16, 12, 10), np.float64, None), ((24, 20, 1), np.float64, None), ((48, 40, 30), np.float32, None),
         ((64, 64, 64), np.float32, None), ((32, 16, 128), np.float32, None), ((64, 64, 512), np.float32, None),
         ((64, 64, 512), np.float32, dict(z_carry=1)), ((128, 64, 256), np.float32, dict(tiled=0))]


@pytest.mark.parametrize("propagator", ["conserved_exp", "relax", "relax_exp", "conserved_poly"])
@pytest.mark.parametrize("shape,dtype,options", CASES, ids=lambda v: str(v))
def test_fused_propagators_match_oracle(shape, dtype, options, propagator):
    from mcstar_b200 import Stepper
    nx, ny, nz = shape
    namp = 0.03 if propagator in ("conserved_exp", "conserved_poly") else 0.0
    st = Stepper(shape, math.pi / 4, 0.3, 0.3, dtype=dtype, namp=namp, seed=21, mu=0.05, options=options)
    k = O.r2c(-0.2 + 0.1 * np.random.default_rng(2).uniform(-1, 1, (nz, ny, nx)))
    st.set_kspace(k.astype(np.complex64 if dtype == np.float32 else np.complex128))
    change = st.step(5, propagator=propagator)
    want, want_change = O.step(k, 5, 0.3, 0.3, st.lens, shape, mu=0.05, namp=namp, seed=21, noise_dtype=dtype,
                               propagator=propagator, return_max_change=True)
    got = st.kspace()
    tol = 2e-6 if dtype == np.float32 else 1e-12
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol
    if propagator in ("conserved_exp", "conserved_poly"):
        assert change == 0.0
        assert got.flat[0] == k.astype(got.dtype).flat[0]  # the mean density is carried exactly
    else:
        # the relaxation moves the k = 0 mode; its largest change is reported (a float)
        rel = 1e-3 if dtype == np.float32 else 1e-6
        assert want_change > 0 and abs(change - want_change) <= rel * want_change


def test_relaxation_rejects_noise():
    from mcstar_b200 import PfcError, Stepper
    st = Stepper((16, 16, 16), math.pi / 4, 0.3, 0.3, dtype=np.float64, namp=0.1)
    st.set_kspace(O.r2c(np.full((16, 16, 16), -0.2)))
    with pytest.raises(PfcError) as e:
        st.step(1, propagator="relax")
    assert e.value.status == 1


@pytest.mark.parametrize("shape,dtype", [((24, 20, 1), np.float64), ((64, 48, 1), np.float32), ((256, 256, 1), np.float32),
                                         ((96, 80, 1), np.float32)])
def test_fused_hpfc_noise_2d_matches_oracle(shape, dtype):
    """The anisotropic noise of kernel_update_eom_hpfcnoise: three Philox fields weighted by
    the wavevector, cut off above |k| = 1/4 (a box of 64 dx = 16 pi reaches it at |i| = 1
    .. 3), against the oracle's draw of the same fields."""
    from mcstar_b200 import Stepper
    nx, ny, nz = shape
    dx = 4.0 * math.pi / max(nx, ny) * 4  # several modes below |k| = 1/4
    st = Stepper(shape, dx, 0.3, 0.3, dtype=dtype, namp=0.05, seed=8, options=None)
    k = O.r2c(-0.2 + 0.1 * np.random.default_rng(3).uniform(-1, 1, (nz, ny, nx)))
    st.set_kspace(k.astype(np.complex64 if dtype == np.float32 else np.complex128))
    st.step(4, propagator="conserved_hpfc")
    want = O.step(k, 4, 0.3, 0.3, st.lens, shape, namp=0.05, seed=8, noise_dtype=dtype, propagator="conserved_hpfc")
    noiseless = O.step(k, 4, 0.3, 0.3, st.lens, shape, propagator="conserved_hpfc")
    got = st.kspace()
    tol = 2e-6 if dtype == np.float32 else 1e-12
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol
    assert np.linalg.norm(want - noiseless) > 10 * tol * np.linalg.norm(want)  # the noise is there
    assert got.flat[0] == k.astype(got.dtype).flat[0]


def test_hpfc_noise_is_2d_only():
    from mcstar_b200 import PfcError, Stepper
    st = Stepper((16, 16, 16), math.pi / 4, 0.3, 0.3, dtype=np.float32, namp=0.1)
    st.set_kspace(O.r2c(np.full((16, 16, 16), -0.2)).astype(np.complex64))
    with pytest.raises(PfcError) as e:
        st.step(1, propagator="conserved_hpfc")
    assert e.value.status == 1
