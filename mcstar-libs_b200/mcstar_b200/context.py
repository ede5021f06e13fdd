"""Python face of one pfc_ctx: shape, precision, stream, and thin methods over the C ABI.

Field buffers are torch CUDA tensors owned by the caller (flat, in the reference's
complex-sized allocation, see ``array.GPUArray``); methods pass their device pointers
and the current torch stream to the library.  Results that live on the host (sums,
counts) come back as Python numbers.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np
import torch

from . import _lib
from ._lib import PfcDesc, PfcStepParams, check, lib

_NP = {np.dtype(np.float32): _lib.PFC_F32, np.dtype(np.float64): _lib.PFC_F64}
_TORCH = {_lib.PFC_F32: torch.float32, _lib.PFC_F64: torch.float64}


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """One context per (shape, precision); owns the library's workspaces."""

    def __init__(self, shape, dtype=np.float32, options=None):
        """options: None (the library's choices) or a dict of pfc_options fields (the
        kernel schedules: z_carry, x_kernel, tiled, radix_order, tile_shift, y_kernel), e.g. the
        result of ``tune``."""
        nx, ny, nz = (int(v) for v in shape)
        self.shape = (nx, ny, nz)
        self.np_dtype = np.dtype(dtype)
        if self.np_dtype not in _NP:
            raise ValueError("dtype must be float32 or float64")
        self.code = _NP[self.np_dtype]
        self.torch_dtype = _TORCH[self.code]
        if not torch.cuda.is_available():
            raise RuntimeError("the pfc_b200 kernels need a CUDA device (B200, sm_100a)")
        torch.cuda.init()
        h = ctypes.c_void_p()
        opts = None if options is None else ctypes.byref(_lib.PfcOptions.from_dict(options))
        check(lib().pfc_create_with(ctypes.byref(PfcDesc(nx, ny, nz, self.code)), opts, ctypes.byref(h)), None,
              f"pfc_create{self.shape}")
        self._h = h
        self.nxh = nx // 2 + 1
        self.n_real = nx * ny * nz
        self.n_cmpl = self.nxh * ny * nz
        self.state_bytes = int(lib().pfc_state_bytes(h))

    @property
    def options(self):
        """The kernel schedules in effect (pfc_get_options), as a dict."""
        o = _lib.PfcOptions()
        check(lib().pfc_get_options(self._h, ctypes.byref(o)), self._h, "pfc_get_options")
        return o.to_dict()

    # -- plumbing ---------------------------------------------------------------------
    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().pfc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sync_stream(self):
        s = torch.cuda.current_stream().cuda_stream
        lib().pfc_set_stream(self._h, ctypes.c_void_p(s))

    def _call(self, name, *args):
        self._sync_stream()
        check(getattr(lib(), name)(self._h, *args), self._h, name)

    def empty_state(self):
        """A device buffer of the reference's complex-sized allocation (2*n_cmpl F)."""
        return torch.empty(2 * self.n_cmpl, dtype=self.torch_dtype, device="cuda")

    # -- FFT ----------------------------------------------------------------------------
    def r2c(self, real_in, cmpl_out):
        self._call("pfc_fft_r2c", _ptr(real_in), _ptr(cmpl_out))

    def c2r(self, cmpl_in, real_out):
        self._call("pfc_fft_c2r", _ptr(cmpl_in), _ptr(real_out))

    # -- pointwise ----------------------------------------------------------------------
    def update_eom(self, kpsi, knl, knoise, namp, dt, eps, lens):
        self._call("pfc_update_eom", _ptr(kpsi), _ptr(knl), _ptr(knoise), float(namp), float(dt), float(eps),
                   *(float(v) for v in lens))

    def update_eom_with_fen(self, kpsi, knl, knoise, namp, dt, eps, lens):
        self._call("pfc_update_eom_with_fen", _ptr(kpsi), _ptr(knl), _ptr(knoise), float(namp), float(dt),
                   float(eps), *(float(v) for v in lens))

    def psi3_split(self, arr, pot=None, mu=0.0, norm=False):
        self._call("pfc_psi3_split", _ptr(arr), _ptr(pot), float(mu), int(bool(norm)))

    def norm(self, arr):
        self._call("pfc_norm", _ptr(arr))

    def calc_fen(self, psi, lpsi, hh):
        out = ctypes.c_double()
        self._call("pfc_calc_fen", _ptr(psi), _ptr(lpsi), *(float(v) for v in hh), ctypes.byref(out))
        return out.value

    def noise_kspace(self, arr, seed, counter):
        self._call("pfc_noise_fill_kspace", _ptr(arr), ctypes.c_uint64(seed), ctypes.c_uint64(counter))

    def noise_real(self, arr, sigma, seed, counter):
        self._call("pfc_noise_fill", _ptr(arr), float(sigma), ctypes.c_uint64(seed), ctypes.c_uint64(counter))

    # -- the reference's other propagators (eom-exp.hpp, el.hpp, el-exp.hpp, eom.hpp) -----------
    def init_eom_op(self, kop, dt, eps, lens):
        self._call("pfc_init_eom_op", _ptr(kop), float(dt), float(eps), *(float(v) for v in lens))

    def update_eom_exp(self, kop, kpsi, knl, knoise, namp, eps, lens, with_fen=False):
        name = "pfc_update_eom_exp_with_fen" if with_fen else "pfc_update_eom_exp"
        self._call(name, _ptr(kop), _ptr(kpsi), _ptr(knl), _ptr(knoise), float(namp), float(eps),
                   *(float(v) for v in lens))

    # ---- spectral low-pass post-processing (gaussian.hpp, lowpass.hpp) ----
    def gaussian_init(self, kgauss, lens, hh, divs_per_sigma):
        """kgauss_k = (e, 1 - e), e = exp(-1/2 sum_a (1.1 d h_a K_a)^2)."""
        self._call("pfc_gaussian_init", _ptr(kgauss), *(float(v) for v in lens), *(float(v) for v in hh),
                   float(divs_per_sigma))

    def kmult_real(self, karr, kgauss):
        self._call("pfc_kmult_real", _ptr(karr), _ptr(kgauss))

    def kmult_imag(self, karr, kgauss):
        self._call("pfc_kmult_imag", _ptr(karr), _ptr(kgauss))

    def square(self, arr):
        self._call("pfc_square", _ptr(arr))

    def write_lowpass_2d(self, spectrum, kgauss, lens, path):
        """spectrum *= Re kgauss, then the gzip LOWPASS dump of it to path (2D grids)."""
        self._call("pfc_write_lowpass_2d", _ptr(spectrum), _ptr(kgauss), float(lens[0]), float(lens[1]),
                   os.fsencode(path))

    def amplitude_lowpass(self, spectrum, aux, kgauss, lens, path=None):
        """Local amplitude of a 2D field into aux (calc_amplitude_lowpass); the LOWPASS dump
        to path unless it is None."""
        self._call("pfc_amplitude_lowpass", _ptr(spectrum), _ptr(aux), _ptr(kgauss), float(lens[0]),
                   float(lens[1]), None if path is None else os.fsencode(path))

    def update_el(self, kpsi, knl, dt, eps, lens):
        """Non-conserved relaxation step; returns max_k |psi^'_k - psi^_k|."""
        out = ctypes.c_double()
        self._call("pfc_update_el", _ptr(kpsi), _ptr(knl), float(dt), float(eps), *(float(v) for v in lens),
                   ctypes.byref(out))
        return out.value

    def init_el_op(self, kop, dt, eps, lens):
        self._call("pfc_init_el_op", _ptr(kop), float(dt), float(eps), *(float(v) for v in lens))

    def update_el_exp(self, kop, kpsi, knl):
        out = ctypes.c_double()
        self._call("pfc_update_el_exp", _ptr(kop), _ptr(kpsi), _ptr(knl), ctypes.byref(out))
        return out.value

    def update_eom_py(self, kpsi, knl, knoise, namp, dt, eps, lens):
        self._call("pfc_update_eom_py", _ptr(kpsi), _ptr(knl), _ptr(knoise), float(namp), float(dt), float(eps),
                   *(float(v) for v in lens))

    def update_eom_hpfcnoise(self, kpsi, knl, n1, n2, n3, namp, dt, eps, lens):
        self._call("pfc_update_eom_hpfcnoise", _ptr(kpsi), _ptr(knl), _ptr(n1), _ptr(n2), _ptr(n3), float(namp),
                   float(dt), float(eps), *(float(v) for v in lens))

    # -- analysis -----------------------------------------------------------------------
    def findpeaks(self, psi, ths, out=None, capacity=None):
        """Returns (n_found, records) where records is a device uint8 tensor of
        Maximum<F> structs (16 B for float, 32 B for double), sorted by linear index."""
        rec = 16 if self.code == _lib.PFC_F32 else 32
        if out is None:
            capacity = max(1, self.n_real // 8) if capacity is None else capacity
            out = torch.empty(capacity * rec, dtype=torch.uint8, device="cuda")
        else:
            capacity = out.numel() // rec if capacity is None else capacity
        n = ctypes.c_int()
        self._call("pfc_findpeaks", _ptr(psi), float(ths), _ptr(out), int(capacity), ctypes.byref(n))
        return n.value, out[: n.value * rec]

    def findpeaks_async(self, psi, ths, host_out):
        """Starts a peak search whose records go to host_out (a pinned CPU uint8 tensor of
        Maximum<F> records, e.g. torch.empty(..., dtype=torch.uint8).pin_memory()) while the
        caller keeps stepping; returns at once.  findpeaks_wait() gives the count."""
        rec = 16 if self.code == _lib.PFC_F32 else 32
        self._async_count = torch.zeros(1, dtype=torch.int32).pin_memory()
        self._async_out = host_out
        self._call("pfc_findpeaks_async", _ptr(psi), float(ths), ctypes.c_void_p(host_out.data_ptr()),
                   int(host_out.numel() // rec), ctypes.cast(ctypes.c_void_p(self._async_count.data_ptr()),
                                                             ctypes.POINTER(ctypes.c_int)))

    def findpeaks_wait(self):
        """Waits for the search of findpeaks_async; returns (n_found, records on the host)."""
        rec = 16 if self.code == _lib.PFC_F32 else 32
        n = ctypes.c_int()
        self._call("pfc_findpeaks_wait", ctypes.byref(n))
        return n.value, self._async_out[: n.value * rec]

    def bond_order(self, maxima, n, h, ths, boxsize, rlim, capacity=None):
        capacity = max(1, n) if capacity is None else capacity
        rows = torch.empty(capacity * _lib.PFC_BOND_NCOL, dtype=torch.float64, device="cuda")
        nr = ctypes.c_int()
        self._call("pfc_bond_order", _ptr(maxima), int(n), *(float(v) for v in h), float(ths), float(boxsize),
                   float(rlim), _ptr(rows), int(capacity), ctypes.byref(nr))
        return rows[: nr.value * _lib.PFC_BOND_NCOL].view(nr.value, _lib.PFC_BOND_NCOL)

    def bond_reserve(self, max_atoms, max_pairs):
        """Grows the bond-order scratch up front (pfc_bond_order grows it on demand)."""
        check(lib().pfc_bond_reserve(self._h, int(max_atoms), int(max_pairs)), self._h, "pfc_bond_reserve")

    # -- stepper ------------------------------------------------------------------------
    def step(self, kpsi, nsteps, dt, eps, lens, mu=0.0, C=1.0, namp=0.0, seed=0, counter=0, propagator="conserved"):
        """nsteps fused steps (pfc_step_prop); propagator: "conserved" (eom.hpp),
        "conserved_exp" (eom-exp.hpp), "relax" (el.hpp), "relax_exp" (el-exp.hpp).  Returns
        the last step's largest mode change for the relaxations, else 0."""
        p = PfcStepParams(float(dt), float(eps), float(mu), float(C), float(namp), float(lens[0]),
                          float(lens[1]), float(lens[2]), int(seed), int(counter))
        m = ctypes.c_double(0.0)
        self._call("pfc_step_prop", _ptr(kpsi), int(nsteps), ctypes.byref(p), _lib.PROPAGATORS[propagator],
                   ctypes.byref(m))
        return m.value

    def step_host(self, host_in, host_out, kpsi, nsteps, dt, eps, lens, mu=0.0, C=1.0, namp=0.0, seed=0, counter=0):
        """pfc_step_host: psi^ from host_in (a CPU tensor, pinned for overlap) through the
        device buffer kpsi, nsteps fused steps, the final psi^ into host_out."""
        p = PfcStepParams(float(dt), float(eps), float(mu), float(C), float(namp), float(lens[0]),
                          float(lens[1]), float(lens[2]), int(seed), int(counter))
        self._call("pfc_step_host", ctypes.c_void_p(host_in.data_ptr()), ctypes.c_void_p(host_out.data_ptr()),
                   _ptr(kpsi), int(nsteps), ctypes.byref(p))

    # -- reverse mode --------------------------------------------------------------------
    def adjoint_workspace(self):
        """Device workspace of pfc_adjoint_step (two states)."""
        n = int(lib().pfc_adjoint_workspace_bytes(self._h)) // self.torch_dtype.itemsize
        return torch.empty(n, dtype=self.torch_dtype, device="cuda")

    def sf_loss(self, kpsi, s_target, lam_out):
        """L = sum_k (|psi^_k|^2/N - s_k)^2 over the full spectrum; lam_out <- dL/dpsi (real)."""
        out = ctypes.c_double()
        self._call("pfc_sf_loss", _ptr(kpsi), _ptr(s_target), _ptr(lam_out), ctypes.byref(out))
        return out.value

    def adjoint_step(self, kpsi_n, kpsi_np1, lam, dt, eps, lens, C=1.0, workspace=None, with_eps=True):
        """lam <- dL/dpsi_n from dL/dpsi_{n+1}; returns this step's dL/deps (0 if not with_eps)."""
        p = PfcStepParams(float(dt), float(eps), 0.0, float(C), 0.0, float(lens[0]), float(lens[1]), float(lens[2]),
                          0, 0)
        ws = self.adjoint_workspace() if workspace is None else workspace
        d = ctypes.c_double(0.0)
        self._call("pfc_adjoint_step", _ptr(kpsi_n), _ptr(kpsi_np1), _ptr(lam), ctypes.byref(p), _ptr(ws),
                   ctypes.byref(d) if with_eps else None)
        return d.value

    def profile_enable(self, on=True):
        check(lib().pfc_profile_enable(self._h, int(bool(on))), self._h, "pfc_profile_enable")

    def profile_read(self):
        """{"launches": n, "calls": [5], "ms": [5]} since profile_enable (families:
        0 entry/exit, 1 xy part of a step, 2 z pass, 3 register y passes, 4 register x
        pass; 3 and 4 are also counted inside 1)."""
        self._sync_stream()
        p = _lib.PfcProfile()
        check(lib().pfc_profile_read(self._h, ctypes.byref(p)), self._h, "pfc_profile_read")
        return {"launches": int(p.launches), "calls": [int(v) for v in p.calls], "ms": [float(v) for v in p.ms],
                "xy_variant": int(p.xy_variant), "xy_mode": int(p.xy_mode), "z_mode": int(p.z_mode),
                "z_variant": int(p.z_variant), "y_variant": int(p.y_variant)}

    def free_energy(self, kpsi, eps, lens, hh):
        out = ctypes.c_double()
        self._call("pfc_free_energy", _ptr(kpsi), float(eps), *(float(v) for v in lens), *(float(v) for v in hh),
                   ctypes.byref(out))
        return out.value


_cache = threading.local()


def get_context(shape, dtype):
    """Per-thread cache of contexts keyed by (shape, dtype, device)."""
    d = getattr(_cache, "d", None)
    if d is None:
        d = _cache.d = {}
    key = (tuple(int(v) for v in shape), np.dtype(dtype).str, torch.cuda.current_device())
    ctx = d.get(key)
    if ctx is None:
        ctx = d[key] = Context(shape, dtype)
    return ctx


def tune(shape, dtype=np.float32, cache_path=None):
    """pfc_tune: the fastest kernel schedules for this shape and precision on the current
    device, as (options dict, ms per step).  With a cache_path, results are read from and
    written to that JSON file."""
    nx, ny, nz = (int(v) for v in shape)
    if not torch.cuda.is_available():
        raise RuntimeError("the pfc_b200 kernels need a CUDA device (B200, sm_100a)")
    torch.cuda.init()
    o = _lib.PfcOptions()
    ms = ctypes.c_double(0.0)
    path = None if cache_path is None else os.fsencode(cache_path)
    check(lib().pfc_tune(ctypes.byref(PfcDesc(nx, ny, nz, _NP[np.dtype(dtype)])), path, ctypes.byref(o),
                         ctypes.byref(ms)), None, f"pfc_tune{(nx, ny, nz)}")
    return o.to_dict(), ms.value
