"""The headline workload itself: 512^3 FP32, the seeded random liquid psi0 = -0.18 +
U(-0.05, 0.05) (numpy PCG64, seed 2024), eps = 0.3, dt = 0.25, dx = pi/4, no noise -- the
field and parameters the benchmark times.

The FP32 stepper is measured against FP64 (the reference's own FP64 cuFFT path, built from
its sources into oracle/_ref) beside the reference's FP32 cuFFT path on the same steps:
after 1 and 10 steps, where round-off has not yet been amplified by the dynamics, and
after 1000 steps (the precision study: field error, free energy, mean density, peaks).
The liquid at eps = 0.3 is linearly unstable, so round-off of either implementation grows
with time; the FP32 stepper is required to be no less accurate than the reference's FP32
path at every horizon."""
import math

import numpy as np
import pytest

import pfc_oracle as O
from conftest import ref_lib

pytestmark = pytest.mark.gpu

N, DX, DT, EPS = 512, math.pi / 4, 0.25, 0.3
SHAPE = (N, N, N)
LENS = (N * DX,) * 3


def _ref_fields(k0, dtype, checkpoints):
    ref = ref_lib(dtype)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    h = ref["create"](N, N, N, 1)
    kc = np.ascontiguousarray(k0.astype(np.complex64 if dtype == np.float32 else np.complex128))
    ref["set_kpsi"](h, kc.ctypes.data)
    out, done = {}, 0
    for c in checkpoints:
        ref["step"](h, c - done, 0.0, DT, EPS, *LENS, 0.0, 0)
        done = c
        f = np.zeros(SHAPE[::-1], dtype=dtype)
        ref["get_psi"](h, f.ctypes.data)
        out[c] = f
    kend = np.zeros(k0.shape, dtype=kc.dtype)
    ref["get_kpsi"](h, kend.ctypes.data)
    ref["destroy"](h)
    return out, kend


def _mine(k0, checkpoints):
    from mcstar_b200 import Stepper
    st = Stepper(SHAPE, DX, DT, EPS, dtype=np.float32)
    st.set_kspace(k0.astype(np.complex64))
    kk = st.kpsi[:2].double().cpu().numpy().copy()
    out, done = {}, 0
    for c in checkpoints:
        st.step(c - done)
        done = c
        out[c] = st.real()
    assert np.array_equal(st.kpsi[:2].double().cpu().numpy(), kk)  # the mean density, to the bit
    return out, st


def _rel(a, b):
    return float(np.linalg.norm((a.astype(np.float64) - b).ravel()) / np.linalg.norm(b.ravel()))


def test_headline_512_fp32_short_horizon_no_worse_than_reference():
    import os
    from mcstar_b200 import liquid_random
    k0 = np.ascontiguousarray(O.r2c(liquid_random(SHAPE, -0.18, 0.05, 2024), workers=len(os.sched_getaffinity(0))))
    ck = (1, 10)
    truth, _ = _ref_fields(k0, np.float64, ck)
    theirs, _ = _ref_fields(k0, np.float32, ck)
    mine, _ = _mine(k0, ck)
    for c in ck:
        e_mine, e_ref = _rel(mine[c], truth[c]), _rel(theirs[c], truth[c])
        print(f"512^3 fp32 vs fp64 after {c} step(s): this stepper {e_mine:.3e}, reference cuFFT {e_ref:.3e}")
        assert e_mine <= 1.1 * e_ref


def test_headline_512_precision_study_1000_steps():
    import os
    from mcstar_b200 import Stepper, liquid_random, records_to_host
    k0 = np.ascontiguousarray(O.r2c(liquid_random(SHAPE, -0.18, 0.05, 2024), workers=len(os.sched_getaffinity(0))))
    truth, k64 = _ref_fields(k0, np.float64, (1000,))
    theirs, _ = _ref_fields(k0, np.float32, (1000,))
    mine, st = _mine(k0, (1000,))
    e_mine, e_ref = _rel(mine[1000], truth[1000]), _rel(theirs[1000], truth[1000])
    # free energy of both final states through this library (FP64 sums)
    f32 = st.free_energy()
    del st
    ref64 = Stepper(SHAPE, DX, DT, EPS, dtype=np.float64)
    ref64.set_kspace(k64)
    f64 = ref64.free_energy()
    df = abs(f32 - f64) / abs(f64)
    # peak lists of the final fields
    n32, rec = _peaks_of(mine[1000])
    n64, rec64 = _peaks_of(truth[1000])
    nref, recref = _peaks_of(theirs[1000])
    diff_mine = len(rec ^ rec64)
    diff_ref = len(recref ^ rec64)
    print(f"512^3 x 1000: field rel L2 this stepper {e_mine:.3e}, reference cuFFT {e_ref:.3e}; F rel {df:.2e}; "
          f"peaks {n32} / {n64} (fp64), differing {diff_mine} (reference fp32: {diff_ref})")
    assert e_mine <= e_ref
    assert df < 1e-5
    assert diff_mine <= max(1.1 * diff_ref, 10) and abs(n32 - n64) <= 0.001 * n64


def _peaks_of(field):
    idx, _ = O.findpeaks3d(field, -1.0)
    return len(idx), set(map(tuple, idx.tolist()))
