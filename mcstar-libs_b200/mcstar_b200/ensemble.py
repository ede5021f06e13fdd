"""Ensembles of independent PFC fields advanced by one CUDA-graph launch per step.

Each member owns a context (never shared: members run concurrently), its state psi^
and its step parameters.  ``Ensemble.run(n)`` replays a graph that holds one step of
every member on its own branch, so fields of different sizes share the GPU.  Across
GPUs the members are dealt out by cost (``partition``): no data moves between ranks,
only the final scalars are gathered.

``ensemble_members`` builds the batched workload: 48 2D fields with sides drawn from
{128, 192, 256, 384, 512, 768, 1024} and 16 3D fields with sides from
{64, 96, 128, 160, 192}; eps ~ U[0.1, 0.4], psi0 ~ U[-0.35, -0.15], per-member seeds,
conserved noise at T = 1e-3, FP32.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from ._lib import PfcStepParams, check, lib
from .context import Context
from .stepper import liquid_random, namp_from_temperature

SIDES_2D = (128, 192, 256, 384, 512, 768, 1024)
SIDES_3D = (64, 96, 128, 160, 192)


def ensemble_members(seed=4, n2d=48, n3d=16, T=1e-3, dt=0.5, dx=math.pi / 4):
    """The member specifications of the batched workload (dicts)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n2d + n3d):
        if i < n2d:
            s = int(rng.choice(SIDES_2D))
            shape = (s, s, 1)
        else:
            s = int(rng.choice(SIDES_3D))
            shape = (s, s, s)
        out.append(dict(shape=shape, dx=dx, dt=dt, eps=float(rng.uniform(0.1, 0.4)),
                        psi0=float(rng.uniform(-0.35, -0.15)), seed=int(rng.integers(1, 2 ** 31)),
                        namp=namp_from_temperature(T, dt)))
    return out


def member_cost(m):
    n = int(np.prod(m["shape"]))
    return n * math.log2(n)


def partition(members, nranks):
    """Greedy longest-processing-time assignment of members to ranks by N log N cost.
    Returns a list of index lists, one per rank."""
    order = sorted(range(len(members)), key=lambda i: -member_cost(members[i]))
    load = [0.0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += member_cost(members[i])
    return [sorted(p) for p in parts]


class Ensemble:
    """Members on the current device; ``run(n)`` advances all of them by n steps."""

    def __init__(self, members, steps_per_graph=1, dtype=np.float32, amp=0.01):
        self.members = list(members)
        self.steps_per_graph = int(steps_per_graph)
        self.ctxs, self.kpsi, self.params = [], [], []
        for m in self.members:
            ctx = Context(m["shape"], dtype)
            k = ctx.empty_state()
            real = ctx.empty_state()
            psi = liquid_random(m["shape"], m["psi0"], amp, m["seed"]).astype(dtype)
            real[: ctx.n_real].copy_(torch.from_numpy(psi.ravel()))
            ctx.r2c(real, k)
            lens = tuple(n * m["dx"] for n in m["shape"])
            self.ctxs.append(ctx)
            self.kpsi.append(k)
            self.params.append(PfcStepParams(m["dt"], m["eps"], m.get("mu", 0.0), m.get("C", 1.0), m["namp"],
                                             lens[0], lens[1], lens[2], m["seed"], 0))
        n = len(self.members)
        ctx_arr = (ctypes.c_void_p * n)(*[c.handle.value for c in self.ctxs])
        k_arr = (ctypes.c_void_p * n)(*[k.data_ptr() for k in self.kpsi])
        p_arr = (PfcStepParams * n)(*self.params)
        h = ctypes.c_void_p()
        torch.cuda.synchronize()
        check(lib().pfc_ensemble_create(n, ctx_arr, k_arr, p_arr, self.steps_per_graph, ctypes.byref(h)), None,
              "pfc_ensemble_create")
        self._h = h
        self.cells = sum(int(np.prod(m["shape"])) for m in self.members)

    def run(self, nsteps):
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        s = lib().pfc_ensemble_run(self._h, int(nsteps), st)
        if s != 0:
            msg = lib().pfc_ensemble_last_error(self._h).decode()
            from ._lib import PfcError
            raise PfcError(s, msg)

    def kspace(self, i):
        nx, ny, nz = self.members[i]["shape"]
        return torch.view_as_complex(self.kpsi[i].view(-1, 2)).view(nz, ny, nx // 2 + 1).cpu().numpy()

    def close(self):
        if getattr(self, "_h", None):
            lib().pfc_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
