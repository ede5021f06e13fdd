"""Gradients through a run of the conserved stepper: the reverse mode of pfc_step (no
counterpart in mcstar-libs).

``AdjointRun`` advances psi^ one pfc_step at a time from a real initial field, keeping
a copy of psi^ every ``every`` steps; the structure-factor loss
L = sum_k (|psi^_k(T)|^2 / N - s_k)^2 (full spectrum) seeds lam_T = dL/dpsi_T
(pfc_sf_loss); the adjoint sweep then walks the segments from the last one back,
recomputes each segment's states from its checkpoint (same noise counters, so the same
trajectory) and applies pfc_adjoint_step per step, accumulating dL/deps.  Results:
dL/dpsi_init (the real field lam_0), dL/deps and dL/dpsi0 = sum(lam_0) for the initial
mean density.  Memory: one state per checkpoint plus every+1 states for the segment
being swept.

``SFLoss`` wraps one such run as a torch.autograd.Function of (psi_init, eps).
"""
from __future__ import annotations

import numpy as np
import torch

from .context import get_context


def structure_factor(ctx, kpsi):
    """|psi^_k|^2 / N on the half spectrum, as a device tensor of n_cmpl reals."""
    c = torch.view_as_complex(kpsi.view(-1, 2))
    return (c.real * c.real + c.imag * c.imag) / float(ctx.n_real)


class AdjointRun:
    def __init__(self, shape, dx, dt, eps, dtype=np.float32, C=1.0, mu=0.0, namp=0.0, seed=0, counter=0,
                 every=50):
        self.shape = tuple(int(v) for v in shape)
        self.dtype = np.dtype(dtype)
        self.ctx = get_context(self.shape, self.dtype)
        self.dx = float(dx)
        self.lens = tuple(n * self.dx for n in self.shape)
        self.dt, self.eps, self.C, self.mu = float(dt), float(eps), float(C), float(mu)
        self.namp, self.seed, self.counter = float(namp), int(seed), int(counter)
        self.every = max(1, int(every))
        self.ckpt = {}
        self.nsteps = 0

    def _step(self, kpsi, n):
        self.ctx.step(kpsi, 1, self.dt, self.eps, self.lens, mu=self.mu, C=self.C, namp=self.namp, seed=self.seed,
                      counter=self.counter + n)

    def _state_from_real(self, psi_init):
        """psi_init: device tensor of n_real values (any shape), the context's precision."""
        buf = self.ctx.empty_state()
        buf[: self.ctx.n_real].copy_(psi_init.reshape(-1))
        k = self.ctx.empty_state()
        self.ctx.r2c(buf, k)
        return k

    def forward(self, psi_init, nsteps):
        """psi^ after nsteps from the real field psi_init; keeps the checkpoints."""
        k = self._state_from_real(psi_init)
        self.ckpt = {0: k.clone()}
        for n in range(nsteps):
            self._step(k, n)
            if (n + 1) % self.every == 0 and n + 1 < nsteps:
                self.ckpt[n + 1] = k.clone()
        self.nsteps = int(nsteps)
        return k

    def backward(self, lam):
        """lam: dL/dpsi_T (real field in a state buffer), overwritten with dL/dpsi_0;
        returns dL/deps."""
        ws = self.ctx.adjoint_workspace()
        deps = 0.0
        starts = sorted(self.ckpt)
        ends = starts[1:] + [self.nsteps]
        for s, e in reversed(list(zip(starts, ends))):
            states = [self.ckpt[s]]
            for n in range(s, e):
                k = states[-1].clone()
                self._step(k, n)
                states.append(k)
            for n in reversed(range(s, e)):
                deps += self.ctx.adjoint_step(states[n - s], states[n - s + 1], lam, self.dt, self.eps, self.lens,
                                              C=self.C, workspace=ws)
        return deps

    def sf_loss_and_grads(self, psi_init, nsteps, s_target):
        """(L, dL/dpsi_init as an (nz, ny, nx) view, dL/deps, dL/dpsi0)."""
        kT = self.forward(psi_init, nsteps)
        lam = self.ctx.empty_state()
        loss = self.ctx.sf_loss(kT, s_target, lam)
        deps = self.backward(lam)
        nx, ny, nz = self.shape
        g = lam[: self.ctx.n_real].view(nz, ny, nx)
        return loss, g, deps, float(g.double().sum().item())


class SFLoss(torch.autograd.Function):
    """L(psi_init, eps) of an AdjointRun; the adjoint sweep runs in forward and its
    results are returned by backward."""

    @staticmethod
    def forward(fctx, psi_init, eps, run, nsteps, s_target):
        run.eps = float(eps)
        loss, g, deps, _ = run.sf_loss_and_grads(psi_init.detach(), nsteps, s_target)
        fctx.save_for_backward(g.clone(), torch.tensor(deps, dtype=torch.float64))
        return torch.tensor(loss, dtype=torch.float64, device=psi_init.device)

    @staticmethod
    def backward(fctx, grad_out):
        g, deps = fctx.saved_tensors
        return grad_out.to(g.dtype) * g, (grad_out.cpu() * deps).to(torch.float64), None, None, None
