"""Device and pinned-host arrays with the reference's interface
(``Array::GPUArray<F>`` / ``Array::CPUArray<F>``, cuda/array_abstraction.hpp:37-211).

Every array is allocated complex-sized, (nx/2+1)*ny*nz*2 elements of F, so one buffer
serves as a real field F[nz][ny][nx] (first nx*ny*nz elements) or as a half spectrum
{re, im}[nz][ny][nx/2+1] -- exactly the reference's layout (Array::m_bytes, line 53).
Extents are given x-first, ``(nx, ny, nz)`` as the reference's int3.
"""
from __future__ import annotations

import sys

import numpy as np
import torch

_TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}


class AsReal:
    """Save tag: the buffer is written as a real array (array_abstraction.hpp:17)."""


class AsCmpl:
    """Save tag: the buffer is written as a complex half spectrum (array_abstraction.hpp:18)."""


def shape_tr(ext):
    """x-fastest extents -> numpy (C-order) shape (common/technicalities.hpp:16-32)."""
    nx, ny, nz = ext
    if nz == 1 and ny == 1:
        return (nx,)
    if nz == 1:
        return (ny, nx)
    return (nz, ny, nx)


class _Array:
    def __init__(self, ext, dtype):
        ext = tuple(int(v) for v in ext)
        if len(ext) != 3:
            raise ValueError("extent is (nx, ny, nz)")
        if ext[0] < 1 or ext[1] < 1 or ext[2] < 1:
            raise RuntimeError("extent must be >=1 in all dimensions")
        self.dtype = np.dtype(dtype)
        if self.dtype not in _TORCH:
            raise ValueError("float32 or float64 only")
        self.m_ext_real = ext
        self.m_ext_cmpl = (ext[0] // 2 + 1, ext[1], ext[2])
        self.m_dims = 3 if ext[2] != 1 else (2 if ext[1] != 1 else 1)
        self.m_real_elems = ext[0] * ext[1] * ext[2]
        self.m_cmpl_elems = self.m_ext_cmpl[0] * ext[1] * ext[2]
        self.m_bytes = self.m_cmpl_elems * 2 * self.dtype.itemsize

    def real_elems(self):
        return self.m_real_elems

    def cmpl_elems(self):
        return self.m_cmpl_elems

    def real_vext(self):
        return self.m_ext_real

    def cmpl_vext(self):
        return self.m_ext_cmpl

    def real_ext(self, i):
        return self.m_ext_real[i]

    def cmpl_ext(self, i):
        return self.m_ext_cmpl[i]

    def ptr_void(self):
        return self.buf

    def ptr_real(self):
        """Real view, shape (nz, ny, nx)."""
        nx, ny, nz = self.m_ext_real
        return self.buf[: self.m_real_elems].view(nz, ny, nx)

    def ptr_cmpl(self):
        """Complex view, shape (nz, ny, nx/2+1)."""
        nxh, ny, nz = self.m_ext_cmpl
        return torch.view_as_complex(self.buf.view(-1, 2)).view(nz, ny, nxh)

    def _same(self, o):
        assert o.real_vext() == self.m_ext_real, "array dimensions differ"


class GPUArray(_Array):
    """``GPUArray(int3)`` or ``GPUArray(CPUArray&)`` (array_abstraction.hpp:74-96)."""

    def __init__(self, src, dtype=np.float32):
        if isinstance(src, CPUArray):
            super().__init__(src.real_vext(), src.dtype)
        else:
            super().__init__(src, dtype)
        self.buf = torch.empty(2 * self.m_cmpl_elems, dtype=_TORCH[self.dtype], device="cuda")
        if isinstance(src, CPUArray):
            src >> self

    def __rshift__(self, o):
        """``>>``: device-to-device or device-to-host copy of the whole buffer."""
        self._same(o)
        o.buf.copy_(self.buf)

    def __mod__(self, o):
        """``%``: swap the buffers of two device arrays."""
        self._same(o)
        self.buf, o.buf = o.buf, self.buf


class CPUArray(_Array):
    """Pinned host array (array_abstraction.hpp:98-211)."""

    def __init__(self, src, dtype=np.float32):
        if isinstance(src, CPUArray):
            super().__init__(src.real_vext(), src.dtype)
        else:
            super().__init__(src, dtype)
        pin = torch.cuda.is_available()
        self.buf = torch.zeros(2 * self.m_cmpl_elems, dtype=_TORCH[self.dtype], pin_memory=pin)
        if isinstance(src, CPUArray):
            src >> self

    def numpy(self):
        return self.buf.numpy()

    def __rshift__(self, o):
        self._same(o)
        o.buf.copy_(self.buf)

    def __mod__(self, o):
        self._same(o)
        self.buf, o.buf = o.buf, self.buf

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            x, y, z = idx
            idx = (z * self.m_ext_real[1] + y) * self.m_ext_real[0] + x
        return self.buf[idx].item()

    def __setitem__(self, idx, v):
        if isinstance(idx, tuple):
            x, y, z = idx
            idx = (z * self.m_ext_real[1] + y) * self.m_ext_real[0] + x
        self.buf[idx] = v

    def load(self, fn):
        """Fill from a .npy file; the numpy shape must match (array_abstraction.hpp:138-153)."""
        data = np.load(fn)
        sh = data.shape
        ext = {1: (sh[0], 1, 1), 2: (sh[-1], sh[0], 1) if len(sh) == 2 else None,
               3: (sh[-1], sh[1], sh[0]) if len(sh) == 3 else None}.get(len(sh))
        if ext is None:
            raise RuntimeError("shouldn't happen")
        if tuple(ext) != self.m_ext_real:
            raise RuntimeError("*** array dimension mismatch")
        flat = np.ascontiguousarray(data, dtype=self.dtype).ravel()
        self.numpy()[: flat.size] = flat
        sys.stderr.write(f"*** array initialized from file <{fn}>\n")

    def save(self, fn, kind=AsReal):
        """Write the buffer as .npy, real or complex (array_abstraction.hpp:154-180)."""
        a = self.numpy()
        if kind is AsCmpl:
            cplx = a.view(np.complex64 if self.dtype == np.float32 else np.complex128)
            np.save(fn, cplx.reshape(shape_tr(self.m_ext_cmpl)))
        else:
            np.save(fn, a[: self.m_real_elems].reshape(shape_tr(self.m_ext_real)))

    # host pointwise helpers (array_abstraction.hpp:183-210)
    def over(self, closure, cmpl=False, with_index=False):
        a = self.numpy()
        view = a.view(np.complex64 if self.dtype == np.float32 else np.complex128) if cmpl else a[: self.m_real_elems]
        for i in range(view.size):
            r = closure(view[i], i) if with_index else closure(view[i])
            if r is not None:
                view[i] = r

    def _real(self):
        return self.numpy()[: self.m_real_elems]

    def square(self):
        r = self._real()
        r *= r

    def set_to(self, val):
        self._real()[:] = val

    def mult(self, val):
        self._real()[:] *= val

    def add(self, val):
        self._real()[:] += val

    def max(self):
        return float(self._real().max())

    def min(self):
        return float(self._real().min())
