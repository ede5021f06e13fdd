"""The reverse mode on the GPU (pfc_sf_loss, pfc_adjoint_step through
mcstar_b200.AdjointRun): against the oracle's FP64 restatement, against central finite
differences of the GPU forward run in FP64, checkpoint segmentation, the autograd
binding, and the 128^3 differentiable-run workload in FP32 beside FP64."""
import math

import numpy as np
import pytest
import torch

import pfc_oracle as O

pytestmark = pytest.mark.gpu


def _liquid(shape, psi0, seed, amp=0.05):
    nx, ny, nz = shape
    return psi0 + amp * np.random.default_rng(seed).uniform(-1, 1, (nz, ny, nx))


def _target(run, psi, nsteps, eps):
    from mcstar_b200 import structure_factor
    e0 = run.eps
    run.eps = eps
    k = run.forward(torch.from_numpy(psi).to("cuda", run.ctx.torch_dtype), nsteps)
    run.eps = e0
    return structure_factor(run.ctx, k).to(run.ctx.torch_dtype).contiguous()


def test_adjoint_fp64_matches_oracle():
    from mcstar_b200 import AdjointRun
    shape, dx, dt, eps, steps = (16, 12, 10), math.pi / 4, 0.5, 0.3, 8
    lens = tuple(n * dx for n in shape)
    psi = _liquid(shape, -0.2, 1, amp=0.1)
    tgt = _liquid(shape, -0.21, 2, amp=0.1)
    s = np.abs(O.r2c(tgt)) ** 2 / np.prod(shape)
    run = AdjointRun(shape, dx, dt, eps, dtype=np.float64, every=3)
    loss, g, deps, dpsi0 = run.sf_loss_and_grads(torch.from_numpy(psi).cuda(), steps,
                                                 torch.from_numpy(np.ascontiguousarray(s).ravel()).cuda())
    L_w, lam_w, deps_w = O.sf_loss_grads(psi, steps, s, dt, eps, lens, shape)
    assert abs(loss - L_w) <= 1e-11 * abs(L_w)
    g = g.cpu().numpy()
    assert np.linalg.norm(g - lam_w) <= 1e-10 * np.linalg.norm(lam_w)
    assert abs(deps - deps_w) <= 1e-9 * abs(deps_w)
    assert abs(dpsi0 - lam_w.sum()) <= 1e-9 * abs(lam_w.sum())


def test_adjoint_fp64_matches_central_differences():
    from mcstar_b200 import AdjointRun
    shape, dx, dt, eps, steps, h = (32, 32, 32), math.pi / 4, 0.5, 0.3, 40, 1e-4
    psi = _liquid(shape, -0.2, 3)
    run = AdjointRun(shape, dx, dt, eps, dtype=np.float64, every=10)
    s = _target(run, _liquid(shape, -0.21, 4), steps, 0.32)
    p = torch.from_numpy(psi).cuda()
    loss, g, deps, dpsi0 = run.sf_loss_and_grads(p, steps, s)
    g = g.clone()

    def L(pp, e):
        run.eps = e
        lam = run.ctx.empty_state()
        v = run.ctx.sf_loss(run.forward(pp, steps), s, lam)
        run.eps = eps
        return v

    def central(f, hh):
        return (f(hh) - f(-hh)) / (2 * hh)

    def richardson(f):  # (4 D(h/2) - D(h)) / 3: the h^2 term of the central difference cancels
        return (4 * central(f, h / 2) - central(f, h)) / 3, central(f, h)

    v = torch.from_numpy(np.random.default_rng(7).standard_normal(psi.shape)).cuda()
    for adj, f in [(deps, lambda d: L(p, eps + d)), (dpsi0, lambda d: L(p + d, eps)),
                   (float((g * v).sum()), lambda d: L(p + d * v, eps))]:
        rich, fd = richardson(f)
        assert abs(adj - fd) <= 1e-4 * abs(fd)  # h = 1e-4: O(h^2) truncation left
        assert abs(adj - rich) <= 2e-6 * abs(rich)


def test_checkpoint_spacing_does_not_change_gradients():
    from mcstar_b200 import AdjointRun
    shape, dx, dt, eps, steps = (32, 32, 16), math.pi / 4, 0.5, 0.3, 12
    psi = torch.from_numpy(_liquid(shape, -0.2, 5)).to("cuda", torch.float32)
    out = []
    for every in (1, 5, 12):
        run = AdjointRun(shape, dx, dt, eps, dtype=np.float32, every=every, namp=0.01, seed=3)
        s = _target(run, _liquid(shape, -0.21, 6), steps, 0.32)
        loss, g, deps, _ = run.sf_loss_and_grads(psi, steps, s)
        out.append((loss, g.clone(), deps))
    for loss, g, deps in out[1:]:
        assert loss == out[0][0] and deps == out[0][2] and torch.equal(g, out[0][1])


def test_autograd_binding():
    from mcstar_b200 import AdjointRun, SFLoss
    shape, dx, dt, steps = (16, 16, 16), math.pi / 4, 0.5, 10
    run = AdjointRun(shape, dx, dt, 0.3, dtype=np.float64, every=4)
    s = _target(run, _liquid(shape, -0.21, 8), steps, 0.32)
    psi = torch.from_numpy(_liquid(shape, -0.2, 9)).cuda().requires_grad_(True)
    eps = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    L = SFLoss.apply(psi, eps, run, steps, s)
    L.backward()
    loss, g, deps, _ = AdjointRun(shape, dx, dt, 0.3, dtype=np.float64, every=4).sf_loss_and_grads(
        psi.detach(), steps, s)
    assert abs(L.item() - loss) <= 1e-12 * abs(loss)
    assert torch.allclose(psi.grad, g, rtol=0, atol=1e-12 * float(g.abs().max()))
    assert abs(eps.grad.item() - deps) <= 1e-12 * abs(deps)


def test_differentiable_run_128_fp32_beside_fp64():
    """The 128^3 workload: 500 steps, checkpoints every 50, loss on the structure factor
    of a run at eps = 0.32, psi0 = -0.21; gradients at eps = 0.3, psi0 = -0.2.  FP64
    gradients are pinned by a central difference in eps (h = 1e-4); the FP32 gradients
    are checked against the FP64 ones."""
    from mcstar_b200 import AdjointRun
    shape, dx, dt, steps, h = (128, 128, 128), math.pi / 4, 0.5, 500, 1e-4
    res = {}
    for dt_ in (np.float64, np.float32):
        run = AdjointRun(shape, dx, dt, 0.3, dtype=dt_, every=50)
        s = _target(run, _liquid(shape, -0.21, 11).astype(dt_), steps, 0.32)
        p = torch.from_numpy(_liquid(shape, -0.2, 12).astype(dt_)).cuda()
        loss, g, deps, dpsi0 = run.sf_loss_and_grads(p, steps, s)
        res[np.dtype(dt_).name] = (loss, g.double().clone(), deps, dpsi0)
        if dt_ is np.float64:
            def L(e):
                run.eps = e
                lam = run.ctx.empty_state()
                v = run.ctx.sf_loss(run.forward(p, steps), s, lam)
                run.eps = 0.3
                return v
            fd = (L(0.3 + h) - L(0.3 - h)) / (2 * h)
            fd2 = (L(0.3 + h / 2) - L(0.3 - h / 2)) / h
            rich = (4 * fd2 - fd) / 3  # the O(h^2) error of the central difference cancels
            print(f"128^3 x 500 FP64 dL/deps: adjoint {deps:.9e}, central h=1e-4 {fd:.9e}, Richardson {rich:.9e}")
            assert abs(deps - fd) <= 1e-3 * abs(fd)
            assert abs(deps - rich) <= 1e-5 * abs(rich)
    l64, g64, e64, p64 = res["float64"]
    l32, g32, e32, p32 = res["float32"]
    rel_g = float(torch.linalg.vector_norm(g32 - g64) / torch.linalg.vector_norm(g64))
    print(f"128^3 x 500: L {l64:.6e} (fp32 {l32:.6e}); dL/deps {e64:.6e} (fp32 {e32:.6e}); "
          f"dL/dpsi0 {p64:.6e} (fp32 {p32:.6e}); dL/dpsi_init fp32 rel L2 {rel_g:.3e}")
    assert np.isfinite([l32, e32, p32]).all() and math.isfinite(rel_g)
    # FP32 gradients against FP64 (measured about 4e-5, 3e-6 and 2.9e-4)
    assert abs(e32 - e64) <= 2e-4 * abs(e64)
    assert abs(p32 - p64) <= 2e-5 * abs(p64)
    assert rel_g <= 1.5e-3
    assert abs(l32 - l64) <= 1e-3 * abs(l64)
