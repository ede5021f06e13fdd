"""The peak finder for callers that cannot allocate device memory (pfc_findpeaks_static).

Such a caller -- a simulation whose device memory is all reserved by its own pool, or a
driver that must not take the implicit synchronisation of a cudaMalloc -- cannot make a
context, so this entry point takes shape, precision and stream directly and keeps its
scratch in a static device array.  Its output must equal that of the context entry point
(pfc_findpeaks) on the same field, call after call: the static scratch keeps the previous
call's contents, which must not leak into the next result.

This file is collected last on purpose; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _smooth_field(shape, seed, dtype):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    k = np.fft.rfftn(rng.standard_normal((nz, ny, nx)))
    kz = np.fft.fftfreq(nz)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    kx = np.fft.rfftfreq(nx)[None, None, :]
    k *= np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) * 60.0)
    return np.fft.irfftn(k, s=(nz, ny, nx), axes=(0, 1, 2)).astype(dtype)


def _static_call(field_dev, shape, dtype, ths, capacity):
    from mcstar_b200 import lib
    import mcstar_b200._lib as L
    rec = 16 if dtype == np.float32 else 32
    out = torch.zeros(capacity * rec, dtype=torch.uint8, device="cuda")
    n = ctypes.c_int(-1)
    code = L.PFC_F32 if dtype == np.float32 else L.PFC_F64
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib().pfc_findpeaks_static(ctypes.c_void_p(field_dev.data_ptr()), shape[0], shape[1], shape[2], code,
                                    float(ths), ctypes.c_void_p(out.data_ptr()), capacity, ctypes.byref(n), stream)
    return st, n.value, out[: max(n.value, 0) * rec]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_static_peak_finder_matches_context_entry_point_on_two_calls(dtype):
    from mcstar_b200 import get_context
    # two calls in a row on different fields and shapes: the second must not see
    # anything of the first through the shared static scratch
    for call, (shape, seed) in enumerate([((48, 40, 36), 1), ((64, 30, 24), 2)]):
        f = _smooth_field(shape, seed, dtype)
        dev = torch.from_numpy(f.ravel().copy()).cuda()
        ths = float(np.quantile(f, 0.4))
        ctx = get_context(shape, dtype)
        n_ref, rec_ref = ctx.findpeaks(dev, ths)
        st, n, rec = _static_call(dev, shape, dtype, ths, capacity=max(1, f.size // 8))
        assert st == 0, f"call {call}: status {st}"
        assert n == n_ref > 0
        from mcstar_b200 import records_to_host
        got, want = records_to_host(rec, dtype), records_to_host(rec_ref, dtype)
        for name in ("i0", "i1", "i2", "field"):  # peak lists are exact
            np.testing.assert_array_equal(got[name], want[name], err_msg=f"call {call}: {name}")


def test_static_peak_finder_refuses_oversized_grids_and_reports_capacity():
    from mcstar_b200 import lib
    import mcstar_b200._lib as L
    n = ctypes.c_int(-1)
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    # 1024 x 512 x 512 cells exceed the 2^27-cell maximum: refused before any launch
    st = lib().pfc_findpeaks_static(ctypes.c_void_p(dummy.data_ptr()), 1024, 512, 512, L.PFC_F32, 0.0,
                                    ctypes.c_void_p(dummy.data_ptr()), 1, ctypes.byref(n), None)
    assert st == L.PFC_ERR_CAPACITY
    shape = (32, 32, 32)
    f = _smooth_field(shape, 5, np.float32)
    dev = torch.from_numpy(f.ravel().copy()).cuda()
    st, cnt, _ = _static_call(dev, shape, np.float32, float(f.min()) - 1.0, capacity=1)
    assert st == L.PFC_ERR_CAPACITY and cnt > 1
