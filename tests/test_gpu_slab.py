"""Slab-decomposed steps through the C ABI (pfc_slab_zinv, pfc_slab_xy, pfc_slab_zpass):
G ranks emulated in one process (the exchanges as device copies; the run has one GPU) step
their slabs, and the assembled half spectrum equals pfc_step on the whole field -- with
conserved noise, whose keys are the whole field's indices."""
import math

import numpy as np
import pytest

import pfc_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,dtype,g,namp", [((32, 32, 32), np.float64, 2, 0.0), ((32, 32, 32), np.float64, 4, 0.03),
                                                ((64, 64, 64), np.float32, 2, 0.02), ((48, 40, 30), np.float64, 2, 0.0),
                                                ((64, 32, 16), np.float32, 4, 0.0)])
def test_emulated_slab_ranks_match_whole_field(shape, dtype, g, namp):
    from mcstar_b200 import Stepper
    from mcstar_b200 import slab as S
    nx, ny, nz = shape
    dx, dt, eps, steps = math.pi / 4, 0.5, 0.3, 4
    ct = np.complex64 if dtype == np.float32 else np.complex128
    k0 = O.r2c(-0.2 + 0.1 * np.random.default_rng(4).uniform(-1, 1, (nz, ny, nx))).astype(ct)
    ranks = [S.SlabRank(shape, r, g, dx, dt, eps, dtype=dtype, mu=0.01, namp=namp, seed=7) for r in range(g)]
    for r in ranks:
        r.set_kspace_slab(k0[:, r.ky0:r.ky0 + r.nys, :])
    S.run_steps(ranks, steps)
    got = np.concatenate([r.kspace_slab() for r in ranks], axis=1)
    st = Stepper(shape, dx, dt, eps, dtype=dtype, mu=0.01, namp=namp, seed=7)
    st.set_kspace(k0)
    st.step(steps)
    want = st.kspace()
    tol = 2e-6 if dtype == np.float32 else 1e-12
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol
    assert got[0, 0, 0] == k0[0, 0, 0]  # the mean density, carried in FP64 by the rank holding ky = 0
