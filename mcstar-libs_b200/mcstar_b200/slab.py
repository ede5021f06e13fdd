"""Slab-decomposed steps of one field spread over several processes (one per GPU).

A field of nx x NY x NZ cells too large for one GPU is split over G ranks.  Between steps
rank r holds the ky-slab of the stepper's carried field A = IFFT_z(psi^)/NZ -- all kz of its
NY / G rows of ky, in a context of shape (nx, NY / G, NZ) -- and inside a step the z-slab of
NZ / G planes, in a context of shape (nx, NY, NZ / G).  One step:

    A (ky-slabs) --all-to-all--> A (z-slabs)            the only two exchanges of a step,
    xy part on the z-slab: B = FFT_xy(cubic(IFFT_xy(A)))  each moving (G - 1) / G of the
    B (z-slabs) --all-to-all--> B (ky-slabs)            field's half spectrum per rank
    z pass on the ky-slab: N^ = FFT_z(B), the update at the field's wavenumbers, A' = IFFT_z(psi^')

through the C ABI (pfc_slab_zinv, pfc_slab_xy, pfc_slab_zpass).  The exchange is NCCL's
all-to-all (or point-to-point sends where the backend lacks all-to-all); ``Emulated`` runs
all ranks in one process with the exchange as device copies, which is how the
decomposition is tested with a single GPU.  The packing of the exchanges (``to_z_chunks``,
``from_z_chunks``, ``to_ky_chunks``, ``from_ky_chunks``) works on any torch tensors, CPU
included.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import PfcStepParams, check, lib
from .context import Context


def split(n, g):
    if n % g:
        raise ValueError(f"{n} does not split into {g} equal slabs")
    return n // g


# -- packing of the exchanges: slab buffers viewed as (z, y, kx, re/im) -------------------------
def to_z_chunks(a_ky, g):
    """ky-slab (NZ, nys, nxh, 2) -> the chunk for each rank's z-slab: planes q NZ/G ... ."""
    nzs = split(a_ky.shape[0], g)
    return [a_ky[q * nzs:(q + 1) * nzs].contiguous() for q in range(g)]


def from_z_chunks(chunks):
    """The chunks rank r received (from rank p: its ky rows of r's planes, (nzs, nys, nxh, 2))
    -> r's z-slab (nzs, NY, nxh, 2), ky rows of rank p at p nys."""
    return torch.cat(chunks, dim=1)


def to_ky_chunks(b_z, g):
    """z-slab (nzs, NY, nxh, 2) -> the chunk for each rank's ky-slab: its rows of these planes."""
    nys = split(b_z.shape[1], g)
    return [b_z[:, q * nys:(q + 1) * nys].contiguous() for q in range(g)]


def from_ky_chunks(chunks):
    """The chunks rank r received (from rank p: r's rows of p's planes) -> r's ky-slab
    (NZ, nys, nxh, 2), planes of rank p at p nzs."""
    return torch.cat(chunks, dim=0)


def exchange(send, group=None):
    """All-to-all of equal-size chunks between the ranks of the default process group:
    recv[p] = the chunk rank p sent to this rank."""
    import torch.distributed as dist
    g = dist.get_world_size(group)
    r = dist.get_rank(group)
    recv = [torch.empty_like(send[0]) for _ in range(g)]
    if dist.get_backend(group) == "nccl":
        dist.all_to_all(recv, send, group=group)
        return recv
    # backends without all-to-all (gloo): paired sends and receives
    ops = []
    for p in range(g):
        if p == r:
            recv[p].copy_(send[p])
        else:
            ops.append(dist.P2POp(dist.isend, send[p], p, group))
            ops.append(dist.P2POp(dist.irecv, recv[p], p, group))
    for w in dist.batch_isend_irecv(ops) if ops else []:
        w.wait()
    return recv


class SlabRank:
    """The slabs and contexts of one rank of a field of `shape` (nx, NY, NZ) over g ranks."""

    def __init__(self, shape, rank, g, dx, dt, eps, dtype=np.float32, mu=0.0, C=1.0, namp=0.0, seed=0):
        nx, ny, nz = (int(v) for v in shape)
        self.shape, self.rank, self.g = (nx, ny, nz), rank, g
        self.nys, self.nzs = split(ny, g), split(nz, g)
        self.nxh = nx // 2 + 1
        self.ky0 = rank * self.nys
        self.ky_ctx = Context((nx, self.nys, nz), dtype)
        self.z_ctx = Context((nx, ny, self.nzs), dtype)
        self.dtype = np.dtype(dtype)
        self.lens = (nx * dx, ny * dx, nz * dx)
        self.dt, self.eps, self.mu, self.C, self.namp, self.seed = dt, eps, mu, C, namp, seed
        self.A = self.ky_ctx.empty_state()   # the carried ky-slab
        self.Az = self.z_ctx.empty_state()
        self.Bz = self.z_ctx.empty_state()
        self.B = self.ky_ctx.empty_state()

    def view_ky(self, t):
        _, _, nz = self.shape
        return t.view(nz, self.nys, self.nxh, 2)

    def view_z(self, t):
        _, ny, _ = self.shape
        return t.view(self.nzs, ny, self.nxh, 2)

    def set_kspace_slab(self, kslab):
        """This rank's ky-slab of the field's half spectrum (numpy (NZ, nys, nxh) complex)."""
        k = self.ky_ctx.empty_state()
        k.copy_(torch.from_numpy(np.ascontiguousarray(kslab).view(self.dtype).ravel()))
        self.ky_ctx._call("pfc_slab_zinv", ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(self.A.data_ptr()),
                          int(self.ky0))

    def params(self, counter):
        return PfcStepParams(float(self.dt), float(self.eps), float(self.mu), float(self.C), float(self.namp),
                             *(float(v) for v in self.lens), int(self.seed), int(counter))

    def xy(self):
        self.z_ctx._call("pfc_slab_xy", ctypes.c_void_p(self.Az.data_ptr()), ctypes.c_void_p(self.Bz.data_ptr()),
                         float(self.C), float(self.mu))

    def zpass(self, counter, last):
        p = self.params(counter)
        self.ky_ctx._call("pfc_slab_zpass", ctypes.c_void_p(self.A.data_ptr()), ctypes.c_void_p(self.B.data_ptr()),
                          ctypes.byref(p), int(self.ky0), int(self.shape[1]), int(bool(last)))

    def kspace_slab(self):
        """After a run: this rank's ky-slab of psi^ (numpy (NZ, nys, nxh) complex)."""
        _, _, nz = self.shape
        ct = np.complex64 if self.dtype == np.float32 else np.complex128
        return self.A.cpu().numpy().view(ct).reshape(nz, self.nys, self.nxh)


def run_steps(ranks, nsteps, counter0=0, exchange_fn=None):
    """nsteps slab steps.  ranks: the SlabRank objects this process drives (all of them when
    emulated; its own one in a multi-process run, with exchange_fn = ``exchange``).  After
    the last step each rank's A holds its ky-slab of psi^."""
    g = ranks[0].g
    for t in range(nsteps):
        last = t == nsteps - 1
        if exchange_fn is None:  # emulated: every rank's chunks are here
            sends = [to_z_chunks(r.view_ky(r.A), g) for r in ranks]
            for q, r in enumerate(ranks):
                r.view_z(r.Az).copy_(from_z_chunks([sends[p][q] for p in range(g)]))
        else:
            r = ranks[0]
            r.view_z(r.Az).copy_(from_z_chunks(exchange_fn(to_z_chunks(r.view_ky(r.A), g))))
        for r in ranks:
            r.xy()
        if exchange_fn is None:
            sends = [to_ky_chunks(r.view_z(r.Bz), g) for r in ranks]
            for q, r in enumerate(ranks):
                r.view_ky(r.B).copy_(from_ky_chunks([sends[p][q] for p in range(g)]))
        else:
            r = ranks[0]
            r.view_ky(r.B).copy_(from_ky_chunks(exchange_fn(to_ky_chunks(r.view_z(r.Bz), g))))
        for r in ranks:
            r.zpass(counter0 + t, last)
