"""The reference's host API on top of libpfc_b200, under the reference's names.

* ``CufftPlan`` / ``R2C`` / ``C2R``         -- FFT::CufftPlan (cuda/cufft_wrapper.hpp:40-86)
* ``NoiseHostApi``                          -- cuda/noise.hpp:93-150
* ``call_kernel_update_eom[_with_fen]``     -- cuda/kernels/eom.hpp:73-109
* ``call_kernel_calc_fen``                  -- eom.hpp:130-141
* ``call_kernel_psi3_split``                -- cuda/kernels/psi3_split.hpp:15-26
* ``call_kernel_norm``                      -- cuda/kernels/norm.hpp:5-10
* ``call_kernel_findpeaks[_2d]``            -- cuda/kernels/findpeaks.hpp:31-63, findpeaks_2d.hpp:29-56
* ``bond_order_analysis``                   -- bond-order-analysis/bond-order.hpp:4
* ``mu`` / ``omega``                        -- common/pfc.hpp:2-7
* ``init_pot_line``                         -- cuda/potentials.hpp:1-20
* ``TimeAcc``                               -- cuda/cutiming.hpp:5-25
* ``Maximum``                               -- common/maximum_struct.hpp:3-6 (numpy dtype)

Each call runs the CUDA kernels of libpfc_b200 through its C ABI; the reference's
cudaThreadSynchronize after every call is kept (calls return with the work done).
Errors raise ``PfcError`` instead of exit(); the reference's silent refusals (a
non-cubic box in findpeaks, a non-2D array in findpeaks_2d) print the same message
and return.
"""
from __future__ import annotations

import math
import sys

import numpy as np
import torch

from ._lib import PFC_BOND_NCOL
from .array import GPUArray, CPUArray
from .context import get_context


class R2C:
    """Plan direction tag (cufft_wrapper.hpp:41)."""


class C2R:
    """Plan direction tag (cufft_wrapper.hpp:42)."""


def _ctx(arr):
    return get_context(arr.real_vext(), arr.dtype)


def _sync():
    torch.cuda.current_stream().synchronize()


class CufftPlan:
    """``CufftPlan<F, R2C|C2R>(int3 shape)``; ``execute(in, out)`` runs the unnormalised
    transform with this library's Stockham FFT (no cuFFT)."""

    def __init__(self, dtype, kind, shape):
        self.dtype = np.dtype(dtype)
        self.kind = kind
        self.m_shape = tuple(int(v) for v in shape)
        self._ctx = get_context(self.m_shape, self.dtype)

    def execute(self, inp, out):
        assert inp.real_vext() == self.m_shape and out.real_vext() == self.m_shape, \
            "array dimensions in plan and execute phase do not match up"
        if self.kind is R2C:
            self._ctx.r2c(inp.buf, out.buf)
        else:
            self._ctx.c2r(inp.buf, out.buf)
        _sync()


class NoiseHostApi:
    """``NoiseHostApi<F>(seed)``: counter-based Philox noise.  Each fill advances an
    internal draw counter, so (seed, draws) identifies the stream position exactly."""

    def __init__(self, dtype=np.float32, seed=1234):
        self.dtype = np.dtype(dtype)
        self.seed = int(seed)
        self.counter = 0

    def fill(self, arr, sigma):
        _ctx(arr).noise_real(arr.buf, sigma, self.seed, self.counter)
        self.counter += 1
        _sync()

    def fill_kspace(self, arr):
        _ctx(arr).noise_kspace(arr.buf, self.seed, self.counter)
        self.counter += 1
        _sync()


def call_kernel_update_eom(arr_kpsi, arr_knonlin, *args):
    """(kpsi, knonlin, knoise, namp, dt, eps, lens) or (kpsi, knonlin, namp, dt, eps, lens)."""
    if isinstance(args[0], GPUArray):
        knoise, namp, dt, eps, lens = args
        kn = knoise.buf
    else:
        namp, dt, eps, lens = args
        kn = None
    _ctx(arr_kpsi).update_eom(arr_kpsi.buf, arr_knonlin.buf, kn, namp, dt, eps, lens)
    _sync()


def call_kernel_update_eom_with_fen(arr_kpsi, arr_knonlin, arr_knoise, namp, dt, eps, lens):
    _ctx(arr_kpsi).update_eom_with_fen(arr_kpsi.buf, arr_knonlin.buf, arr_knoise.buf, namp, dt, eps, lens)
    _sync()


def call_kernel_calc_fen(arr_psi, arr_lpsi, hh):
    """Returns h^3 sum f (FP64 fixed-order sum); lpsi receives the density f."""
    return _ctx(arr_psi).calc_fen(arr_psi.buf, arr_lpsi.buf, hh)


def call_kernel_psi3_split(arr, pot=None, mu=0.0, norm=False):
    _ctx(arr).psi3_split(arr.buf, None if pot is None else pot.buf, mu, norm)
    _sync()


def call_kernel_norm(arr):
    _ctx(arr).norm(arr.buf)
    _sync()


# ---- peaks -------------------------------------------------------------------------------
def maximum_dtype(dtype):
    """numpy dtype of Maximum<F> (common/maximum_struct.hpp:3-6)."""
    f = "<f4" if np.dtype(dtype) == np.float32 else "<f8"
    return np.dtype([("i0", f), ("i1", f), ("i2", f), ("field", "<f4")], align=True)


Maximum = maximum_dtype


def findpeaks_device(arr, ths):
    """(count, device records) of the local maxima of a GPUArray's real field."""
    return _ctx(arr).findpeaks(arr.buf, ths)


def records_to_host(records, dtype):
    md = maximum_dtype(dtype)
    raw = records.cpu().numpy()
    return raw.view(md).copy() if raw.size else np.zeros(0, dtype=md)


def _write_peaks(fn, recs, hh, dtype):
    f = np.float32 if np.dtype(dtype) == np.float32 else np.float64
    h = [f(v) for v in hh]
    try:
        with open(fn, "w") as fp:
            for m in recs:
                x0 = np.float32(f(m["i0"]) * h[0])
                x1 = np.float32(f(m["i1"]) * h[1])
                x2 = np.float32(f(m["i2"]) * h[2])
                fp.write("%f %f %f %f\n" % (x0, x1, x2, m["field"]))
    except OSError:
        print(f"output file <{fn}> cannot be opened for writing")


def call_kernel_findpeaks(inp, peaks_outfn, oorder_outfn, hh, length, ths, rlim):
    if length[0] != length[1] or length[0] != length[2]:
        sys.stderr.write("orientational mapping needs a cube\n")
        return
    n, dev = findpeaks_device(inp, ths)
    sys.stderr.write(f"found {n} maxima\n")
    recs = records_to_host(dev, inp.dtype)
    _write_peaks(peaks_outfn, recs, hh, inp.dtype)
    try:
        fp = open(oorder_outfn, "w")
    except OSError:
        print(f"output file <{oorder_outfn}> cannot be opened for writing")
        return
    with fp:
        f = np.float32 if inp.dtype == np.float32 else np.float64
        rows = _ctx(inp).bond_order(dev, n, [float(f(v)) for v in hh], float(f(ths)), float(f(length[0])),
                                    float(f(rlim))).cpu().numpy()
        write_bond_table(fp, rows)


def call_kernel_findpeaks_2d(inp, peaks_outfn, hh, length, ths):
    nx, ny, nz = inp.real_vext()
    if not (nx > 1 and ny > 1 and nz == 1):
        sys.stderr.write("input not a 2d array\n")
        return
    n, dev = findpeaks_device(inp, ths)
    sys.stderr.write(f"found {n} maxima\n")
    _write_peaks(peaks_outfn, records_to_host(dev, inp.dtype), hh, inp.dtype)


# ---- bond order --------------------------------------------------------------------------
BOND_COLUMNS = ("x", "y", "z", "nb", "xi", "q4", "q6", "q8", "w4", "q4b", "q6b", "q8b", "w4b", "w6")


def write_bond_table(fp, rows):
    """The reference's table (bond-order.cpp:333-338); w6 is not part of it."""
    fp.write("# x y z #nb xi q4 q6 q8 w4 q4b q6b q8b w4b\n")
    for r in rows:
        fp.write("%.6f\t%.6f\t%.6f\t%d\t%d\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\n" % (
            r[0], r[1], r[2], int(r[3]), int(r[4]), r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12]))
    fp.flush()


def bond_order_analysis(maxima, input_len, h0, h1, h2, ths, boxsize, rlim, fp=None, dtype=np.float32):
    """GPU bond order of Maximum records (numpy structured array or device uint8
    records); writes the reference table to fp when given and returns the rows
    (numpy, PFC_BOND_NCOL columns)."""
    if isinstance(maxima, np.ndarray):
        dtype = np.float32 if maxima.dtype["i0"] == np.float32 else np.float64
        dev = torch.from_numpy(np.ascontiguousarray(maxima).view(np.uint8).ravel()).cuda()
    else:
        dev = maxima
    # a context of any shape carries the bond-order workspace, which grows with the input
    ctx = get_context((8, 8, 8), dtype)
    rows = ctx.bond_order(dev, input_len, (h0, h1, h2), ths, boxsize, rlim).cpu().numpy()
    if fp is not None:
        write_bond_table(fp, rows)
    return rows


# ---- common/pfc.hpp, cuda/potentials.hpp, cuda/cutiming.hpp ----------------------------------
def mu(eps, psi0):
    """Liquid chemical potential (1 - eps) psi0 + psi0^3 (common/pfc.hpp:2-3)."""
    return (1.0 - eps) * psi0 + psi0 ** 3


def omega(eps, psi0, fen=None):
    """Grand potential density (common/pfc.hpp:4-7)."""
    if fen is None:
        return 0.5 * (1.0 - eps) * psi0 ** 2 + 0.25 * psi0 ** 4 - mu(eps, psi0) * psi0
    return fen - mu(eps, psi0) * psi0


def sm_square(x, y):
    return (math.cos(x) + math.cos(y) + 2.0) / 4.0


def init_pot_line(arr, l, h, power, sigma, amp):
    """Host initialisation of the 2D line potential (cuda/potentials.hpp:5-20)."""
    nx, ny, nz = arr.real_vext()
    assert nz == 1 and ny > 1 and nx > 1, "array is not 2d"
    f = 2 * math.pi / sigma
    y = np.arange(ny)[:, None] * h[1] - l[1] / 2.0
    x = np.arange(nx)[None, :] * h[0] - l[0] / 2.0
    part1 = 0.5 * (np.tanh(y + sigma / 2) + 1)
    part2 = 0.5 * (np.tanh(-y + sigma / 2) + 1)
    sq = (np.cos(f * x) + np.cos(f * y) + 2.0) / 4.0
    val = amp * sq ** power * part1 * part2
    arr.numpy()[: nx * ny] = val.astype(arr.dtype).ravel()
    print('"init_pot_line" potential initialized')


class TimeAcc:
    """cudaEvent accumulator (cuda/cutiming.hpp:5-25)."""

    def __init__(self):
        self.m_times = 1
        self.m_elapsed_ms = 0.0
        self._a = torch.cuda.Event(enable_timing=True)
        self._b = torch.cuda.Event(enable_timing=True)

    def start(self):
        self._a.record()

    def stop(self, incr=True):
        self._b.record()
        self._b.synchronize()
        if incr:
            self.m_times += 1
        self.m_elapsed_ms += self._a.elapsed_time(self._b)

    def reset(self):
        self.m_times = 1
        self.m_elapsed_ms = 0.0

    def __str__(self):
        return str(self.m_elapsed_ms)
