"""The oracle's restatement of the reverse mode (pfc_oracle.adjoint_step / sf_loss), the
checker of the GPU adjoint, pinned against central finite differences of its own
forward step in FP64: dL/deps, dL/dpsi0 and a random directional derivative of the
initial field."""
import math

import numpy as np

import pfc_oracle as O


def test_oracle_adjoint_matches_central_differences():
    shape = (12, 10, 8)
    nx, ny, nz = shape
    dx, dt, eps, steps = math.pi / 4, 0.5, 0.3, 6
    lens = tuple(n * dx for n in shape)
    rng = np.random.default_rng(3)
    psi = -0.2 + 0.1 * rng.uniform(-1, 1, (nz, ny, nx))
    s = np.abs(O.r2c(-0.21 + 0.1 * rng.uniform(-1, 1, (nz, ny, nx)))) ** 2 / (nx * ny * nz)
    loss, lam, deps = O.sf_loss_grads(psi, steps, s, dt, eps, lens, shape)

    def L(p, e):
        return O.sf_loss(O.step(O.r2c(p), steps, dt, e, lens, shape), s, shape)[0]

    h = 1e-5
    assert abs(L(psi, eps) - loss) <= 1e-12 * abs(loss)
    fd_eps = (L(psi, eps + h) - L(psi, eps - h)) / (2 * h)
    fd_psi0 = (L(psi + h, eps) - L(psi - h, eps)) / (2 * h)
    v = rng.standard_normal(psi.shape)
    fd_v = (L(psi + h * v, eps) - L(psi - h * v, eps)) / (2 * h)
    assert abs(deps - fd_eps) <= 1e-5 * abs(fd_eps)
    assert abs(lam.sum() - fd_psi0) <= 1e-5 * abs(fd_psi0)
    assert abs((lam * v).sum() - fd_v) <= 1e-5 * abs(fd_v)


def test_sf_loss_gradient_alone():
    """dL/dpsi_T of the loss itself (no steps) against central differences."""
    shape = (8, 6, 4)
    nx, ny, nz = shape
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((nz, ny, nx))
    s = rng.uniform(0, 1, O.cmpl_shape(shape))
    for i0 in (0, nx // 2):  # s must be even in k: on the self-mirrored planes s(ky, kz) = s(-ky, -kz)
        plane = s[:, :, i0]
        s[:, :, i0] = 0.5 * (plane + plane[(-np.arange(nz)) % nz][:, (-np.arange(ny)) % ny])
    loss, lam = O.sf_loss(O.r2c(psi), s, shape)
    v = rng.standard_normal(psi.shape)
    h = 1e-6
    fd = (O.sf_loss(O.r2c(psi + h * v), s, shape)[0] - O.sf_loss(O.r2c(psi - h * v), s, shape)[0]) / (2 * h)
    assert abs((lam * v).sum() - fd) <= 1e-6 * abs(fd)
