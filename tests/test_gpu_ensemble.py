"""Ensembles (pfc_ensemble_* through the C ABI): every member of a graph-replayed ensemble
matches the same field advanced alone by pfc_step, and the oracle; runs resume."""
import math

import numpy as np
import pytest

import pfc_oracle as O

pytestmark = pytest.mark.gpu


def _members():
    """Members of mixed shapes; several share a shape (and so one batched launch per pass)
    with their own eps, psi0, noise amplitude and seed."""
    mk = lambda shape, eps, psi0, seed, namp: dict(shape=shape, dx=math.pi / 4, dt=0.5, eps=eps, psi0=psi0,
                                                   seed=seed, namp=namp)
    return [mk((64, 64, 1), 0.25, -0.25, 11, 0.03), mk((32, 32, 32), 0.3, -0.2, 12, 0.05),
            mk((48, 40, 30), 0.2, -0.3, 13, 0.0), mk((96, 96, 1), 0.35, -0.18, 14, 0.02),
            mk((64, 64, 64), 0.3, -0.2, 15, 0.0), mk((64, 64, 1), 0.15, -0.3, 16, 0.01),
            mk((64, 64, 1), 0.4, -0.2, 17, 0.05), mk((32, 32, 32), 0.2, -0.25, 18, 0.02),
            mk((48, 40, 30), 0.35, -0.2, 19, 0.0), mk((64, 64, 64), 0.2, -0.3, 20, 0.0),
            mk((64, 64, 64), 0.25, -0.22, 21, 0.02), mk((32, 16, 512), 0.3, -0.2, 22, 0.01),
            mk((32, 16, 512), 0.25, -0.25, 23, 0.02), mk((64, 512, 64), 0.3, -0.2, 24, 0.0),
            mk((64, 512, 64), 0.25, -0.22, 25, 0.02),
            # batched classes through the 3 2^k / 5 2^k register passes: x 192 (tiled, z 64),
            # 2D 160, and 96 beside the general z pass
            mk((192, 64, 64), 0.3, -0.2, 26, 0.02), mk((192, 64, 64), 0.25, -0.25, 27, 0.0),
            mk((160, 160, 1), 0.3, -0.2, 28, 0.03), mk((160, 160, 1), 0.2, -0.3, 29, 0.0),
            mk((96, 96, 24), 0.3, -0.22, 30, 0.02), mk((96, 96, 24), 0.35, -0.2, 31, 0.0)]


@pytest.mark.parametrize("spg", [1, 3])
def test_ensemble_members_match_individual_steps_and_oracle(spg):
    from mcstar_b200 import Ensemble, Stepper
    members = _members()
    ens = Ensemble(members, steps_per_graph=spg)
    k0 = [ens.kspace(i) for i in range(len(members))]
    ens.run(6)
    for i, m in enumerate(members):
        got = ens.kspace(i)
        st = Stepper(m["shape"], m["dx"], m["dt"], m["eps"], dtype=np.float32, namp=m["namp"], seed=m["seed"])
        st.set_kspace(k0[i])
        st.step(6)
        alone = st.kspace()
        assert np.linalg.norm(got - alone) / np.linalg.norm(alone) < 1e-6, i
        want = O.step(k0[i], 6, m["dt"], m["eps"], st.lens, m["shape"], namp=m["namp"], seed=m["seed"],
                      noise_dtype=np.float32)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 2e-6, i
        assert got[0, 0, 0] == k0[i][0, 0, 0]  # conserved mean density


def test_ensemble_resumes_with_fresh_noise():
    from mcstar_b200 import Ensemble
    members = _members()[:2]
    a = Ensemble(members)
    b = Ensemble(members)
    a.run(8)
    b.run(4)
    b.run(4)
    for i in range(len(members)):
        x, y = a.kspace(i), b.kspace(i)
        assert np.linalg.norm(x - y) / np.linalg.norm(x) < 1e-6
