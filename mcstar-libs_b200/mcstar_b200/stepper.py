"""The fused conserved stepper and the seeded initial conditions of the PFC workloads.

``Stepper`` keeps the state psi^ (half spectrum, reference layout) on the device and
advances it with ``pfc_step``; observables (free energy, peaks, bond order) are
computed from it on the device.  Initial fields are built in FP64 on the host from
numpy's PCG64 (``numpy.random.default_rng(seed)``).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .context import Context, get_context

# The six <110>/sqrt(2) wave vectors of the one-mode bcc ansatz (|q| = 1).
BCC_Q = np.array([[1, 1, 0], [1, -1, 0], [1, 0, 1], [1, 0, -1], [0, 1, 1], [0, 1, -1]], dtype=np.float64) / math.sqrt(2.0)


def namp_from_temperature(T, dt, h=None, dims=3):
    """Noise amplitude ``namp`` of the reference's update (eom.hpp:62,70) for a
    conserved k-space noise of amplitude sqrt(2 dt T) |k| per unit-variance white
    mode: dt * namp = sqrt(2 dt T)  =>  namp = sqrt(2 T / dt).  With a lattice
    spacing h the per-cell variance 2 T dt / h^d gives namp = sqrt(2 T / (dt h^d))."""
    if h is None:
        return math.sqrt(2.0 * T / dt)
    return math.sqrt(2.0 * T / (dt * h ** dims))


def liquid_random(shape, psi0, amp, seed):
    """psi0 + U(-amp, amp), numpy shape (nz, ny, nx), FP64."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    return psi0 + rng.uniform(-amp, amp, size=(nz, ny, nx))


def bcc_sphere(shape, dx, psi0, amp, radius):
    """psi0 + amp * sum cos(q.r) over the six <110>/sqrt(2) vectors inside a sphere of
    the given radius at the box centre; liquid psi0 outside.  FP64, numpy (nz, ny, nx)."""
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz) * dx, np.arange(ny) * dx, np.arange(nx) * dx, indexing="ij")
    cx, cy, cz = nx * dx / 2.0, ny * dx / 2.0, nz * dx / 2.0
    rx, ry, rz = x - cx, y - cy, z - cz
    inside = rx * rx + ry * ry + rz * rz < radius * radius
    s = np.zeros_like(x)
    for q in BCC_Q:
        s += np.cos(q[0] * rx + q[1] * ry + q[2] * rz)
    return np.where(inside, psi0 + amp * s, psi0)


class Stepper:
    """Device state psi^ of one field and the fused step."""

    def __init__(self, shape, dx, dt, eps, dtype=np.float32, mu=0.0, C=1.0, namp=0.0, seed=0, counter=0,
                 options=None):
        self.shape = tuple(int(v) for v in shape)
        self.dtype = np.dtype(dtype)
        # the shared per-shape context, or a context of its own with the given kernel schedules
        self.ctx = get_context(self.shape, self.dtype) if options is None else Context(self.shape, self.dtype, options)
        self.dx = float(dx)
        self.lens = tuple(n * self.dx for n in self.shape)
        self.hh = (self.dx, self.dx, self.dx)
        self.dt, self.eps, self.mu, self.C = float(dt), float(eps), float(mu), float(C)
        self.namp = float(namp)
        self.seed = int(seed)
        self.counter = int(counter)
        self.kpsi = self.ctx.empty_state()
        self._real = self.ctx.empty_state()

    # -- state in and out ----------------------------------------------------------------
    def set_real(self, psi):
        """psi: numpy (nz, ny, nx) real field; stored as its unnormalised R2C."""
        n = self.ctx.n_real
        flat = torch.from_numpy(np.ascontiguousarray(psi, dtype=self.dtype).ravel())
        self._real[:n].copy_(flat)
        self.ctx.r2c(self._real, self.kpsi)

    def real_device(self):
        """psi = C2R(psi^)/N on the device (a view of an internal buffer)."""
        self.ctx.c2r(self.kpsi, self._real)
        nx, ny, nz = self.shape
        v = self._real[: self.ctx.n_real]
        v.mul_(1.0 / self.ctx.n_real)
        return v.view(nz, ny, nx)

    def real(self):
        return self.real_device().cpu().numpy()

    def kspace(self):
        nx, ny, nz = self.shape
        return torch.view_as_complex(self.kpsi.view(-1, 2)).view(nz, ny, nx // 2 + 1).cpu().numpy()

    def set_kspace(self, k):
        self.kpsi.copy_(torch.from_numpy(np.ascontiguousarray(k).view(self.dtype).ravel()))

    # -- dynamics and observables --------------------------------------------------------------
    def step(self, nsteps, propagator="conserved"):
        """Advances nsteps fused steps; returns the last step's largest mode change for the
        relaxation propagators (else 0)."""
        m = self.ctx.step(self.kpsi, nsteps, self.dt, self.eps, self.lens, mu=self.mu, C=self.C, namp=self.namp,
                          seed=self.seed, counter=self.counter, propagator=propagator)
        self.counter += int(nsteps)
        return m

    def step_host(self, host_in, host_out, nsteps):
        """nsteps fused steps of the field held in host memory (pfc_step_host): psi^ from
        host_in through this stepper's device state, the final psi^ into host_out."""
        self.ctx.step_host(host_in, host_out, self.kpsi, nsteps, self.dt, self.eps, self.lens, mu=self.mu, C=self.C,
                           namp=self.namp, seed=self.seed, counter=self.counter)
        self.counter += int(nsteps)

    def free_energy(self):
        return self.ctx.free_energy(self.kpsi, self.eps, self.lens, self.hh)

    def mean_density(self):
        """psi^(k=0) / N, read from the device state."""
        v = self.kpsi[:1].double().item()
        return v / self.ctx.n_real

    def peaks(self, ths):
        """(count, device Maximum<F> records sorted by linear index)."""
        v = self.real_device()
        return self.ctx.findpeaks(v, ths)

    def bond_order(self, ths, rlim):
        n, rec = self.peaks(ths)
        if self.shape[2] == 1:
            raise ValueError("bond order needs a 3D field")
        return self.ctx.bond_order(rec, n, self.hh, ths, self.lens[0], rlim)
