"""Parity of the pointwise kernels, the noise, the free energy and the peak finder
(CUDA through the C ABI) against the oracle, and against the reference's own CUDA
path (oracle/_ref) where it exists."""
import math
import os

import numpy as np
import pytest
import torch

import pfc_oracle as O
from conftest import ref_lib

pytestmark = pytest.mark.gpu

F32, F64 = np.float32, np.float64


def mk(shape, dtype):
    from mcstar_b200 import get_context
    return get_context(shape, dtype)


def up_c(ctx, X):
    b = ctx.empty_state()
    ct = np.complex64 if ctx.np_dtype == F32 else np.complex128
    b.copy_(torch.from_numpy(np.ascontiguousarray(X, dtype=ct).view(ctx.np_dtype).ravel()))
    return b


def up_r(ctx, x):
    b = ctx.empty_state()
    b[: x.size].copy_(torch.from_numpy(np.ascontiguousarray(x, dtype=ctx.np_dtype).ravel()))
    return b


def down_c(ctx, b):
    nx, ny, nz = ctx.shape
    return torch.view_as_complex(b.view(-1, 2)).view(nz, ny, nx // 2 + 1).cpu().numpy()


def down_r(ctx, b):
    nx, ny, nz = ctx.shape
    return b[: ctx.n_real].cpu().numpy().reshape(nz, ny, nx)


def rand_c(shape, dtype, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((nz, ny, nx // 2 + 1)) + 1j * rng.standard_normal((nz, ny, nx // 2 + 1))
    return z.astype(np.complex64 if dtype == F32 else np.complex128)


REL = {F32: 2e-6, F64: 1e-13}


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", [(16, 12, 10), (15, 9, 7), (64, 48, 1), (27, 27, 27)])
@pytest.mark.parametrize("noise", [False, True])
def test_update_eom(shape, dtype, noise):
    ctx = mk(shape, dtype)
    lens = tuple(n * math.pi / 4 for n in shape)
    kp, kn, kz = rand_c(shape, dtype, 1), rand_c(shape, dtype, 2), rand_c(shape, dtype, 3)
    b = up_c(ctx, kp)
    ctx.update_eom(b, up_c(ctx, kn), up_c(ctx, kz) if noise else None, 0.01, 0.5, 0.3, lens)
    got = down_c(ctx, b)
    want = O.update_eom(kp, kn, kz if noise else None, 0.01, 0.5, 0.3, lens, shape)
    assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < REL[dtype]


@pytest.mark.parametrize("dtype", [F32, F64])
def test_update_eom_with_fen(dtype):
    shape = (16, 12, 10)
    ctx = mk(shape, dtype)
    lens = tuple(n * 0.7 for n in shape)
    kp, kn, kz = rand_c(shape, dtype, 4), rand_c(shape, dtype, 5), rand_c(shape, dtype, 6)
    b, bz = up_c(ctx, kp), up_c(ctx, kz)
    ctx.update_eom_with_fen(b, up_c(ctx, kn), bz, 0.02, 0.25, 0.2, lens)
    new, lk = O.update_eom_with_fen(kp, kn, kz, 0.02, 0.25, 0.2, lens, shape)
    assert np.max(np.abs(down_c(ctx, b) - new)) / np.max(np.abs(new)) < REL[dtype]
    assert np.max(np.abs(down_c(ctx, bz) - lk)) / np.max(np.abs(lk)) < REL[dtype]


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("norm,pot", [(True, False), (False, True)])
def test_psi3_split_and_norm(dtype, norm, pot):
    shape = (20, 10, 6)
    ctx = mk(shape, dtype)
    rng = np.random.default_rng(9)
    x = (rng.standard_normal((6, 10, 20)) * (shape[0] * shape[1] * shape[2] if norm else 1.0)).astype(dtype)
    p = rng.standard_normal((6, 10, 20)).astype(dtype) if pot else None
    b = up_r(ctx, x)
    ctx.psi3_split(b, up_r(ctx, p) if pot else None, 0.13, norm)
    want = O.psi3_split(x.astype(F64), None if p is None else p.astype(F64), 0.13, norm)
    np.testing.assert_allclose(down_r(ctx, b), want, rtol=REL[dtype] * 3, atol=REL[dtype] * 3)
    b = up_r(ctx, x)
    ctx.norm(b)
    np.testing.assert_allclose(down_r(ctx, b), O.norm(x.astype(F64)), rtol=REL[dtype])


@pytest.mark.parametrize("dtype", [F32, F64])
def test_calc_fen_and_free_energy(dtype):
    shape = (24, 20, 18)
    dx = math.pi / 4
    lens = tuple(n * dx for n in shape)
    hh = (dx, dx, dx)
    ctx = mk(shape, dtype)
    rng = np.random.default_rng(3)
    psi = -0.2 + 0.3 * np.cos(np.arange(24) * dx)[None, None, :] + 0.05 * rng.standard_normal((18, 20, 24))
    k = O.r2c(psi)
    want = O.free_energy(k, 0.3, lens, hh, shape)
    got = ctx.free_energy(up_c(ctx, k), 0.3, lens, hh)
    assert abs(got - want) / abs(want) < (1e-5 if dtype == F32 else 1e-12)
    lpsi = O.norm(O.c2r(O.lop(shape, lens, 0.3) * k, shape))
    ps = O.norm(O.c2r(k, shape))
    wsum, wf = O.calc_fen(ps, lpsi, hh)
    bl = up_r(ctx, lpsi)
    s = ctx.calc_fen(up_r(ctx, ps), bl, hh)
    assert abs(s - wsum) / abs(wsum) < (1e-5 if dtype == F32 else 1e-12)
    np.testing.assert_allclose(down_r(ctx, bl), wf, atol=1e-6 if dtype == F32 else 1e-14)


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", [(16, 12, 10), (15, 9, 7), (32, 30, 1)])
def test_noise_kspace_matches_oracle_value_for_value(shape, dtype):
    ctx = mk(shape, dtype)
    b = ctx.empty_state()
    ctx.noise_kspace(b, 1234, 77)
    got = down_c(ctx, b)
    want = O.fill_kspace(shape, 1234, 77, dtype=dtype)
    assert np.max(np.abs(got - want)) < (5e-6 if dtype == F32 else 1e-13)
    r = ctx.empty_state()
    ctx.noise_real(r, 0.5, 99, 3)
    np.testing.assert_allclose(r[: ctx.n_real].cpu().numpy(), O.fill_real(ctx.n_real, 0.5, 99, 3, dtype=dtype),
                               atol=5e-6 if dtype == F32 else 1e-13)


def test_noise_statistics_like_reference_curand():
    """Per-cell mean and variance of C2R(noise)/sqrt(N) over many draws -- the statistical
    test of curand_kspace_unittest/main_corr.cu:35-48 -- for this library's noise and, when
    built, for the reference's cuRAND noise on the same grid."""
    shape = (12, 10, 8)
    nx, ny, nz = shape
    ctx = mk(shape, F64)
    draws = 400
    acc, acc2 = 0.0, 0.0
    b, r = ctx.empty_state(), ctx.empty_state()
    for i in range(draws):
        ctx.noise_kspace(b, 5, i)
        ctx.c2r(b, r)
        v = r[: ctx.n_real].double() / math.sqrt(ctx.n_real)
        acc = acc + v
        acc2 = acc2 + v * v
    mean = (acc / draws).cpu().numpy()
    var = (acc2 / draws).cpu().numpy()
    assert abs(mean.mean()) < 0.02 and abs(var.mean() - 1.0) < 0.02
    ref = ref_lib(F64)
    if ref is not None:
        h = ref["create"](nx, ny, nz, 42)
        buf = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
        s = 0.0
        for i in range(50):
            ref["noise_kspace"](h, buf.ctypes.data)
            s += np.mean(np.abs(buf) ** 2)
        ref["destroy"](h)
        assert abs(s / 50 - 1.0) < 0.05  # both have E|xi|^2 = 1


def smooth_field(shape, seed, dtype):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    k = O.r2c(rng.standard_normal((nz, ny, nx)))
    k2 = O.kgrid(shape, (nx, ny, nz))
    return O.norm(O.c2r(k * np.exp(-k2 * 4.0), shape)).astype(dtype)


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", [(32, 24, 20), (17, 13, 11), (64, 48, 1), (128, 32, 20), (256, 48, 40),
                                   (256, 24, 12)])
def test_findpeaks_bit_exact(shape, dtype):
    ctx = mk(shape, dtype)
    f = smooth_field(shape, 2, dtype)
    ths = float(np.quantile(f, 0.3))
    n, rec = ctx.findpeaks(up_r(ctx, f), ths)
    from mcstar_b200 import records_to_host
    got = records_to_host(rec, dtype)
    if shape[2] == 1:
        idx, val = O.findpeaks2d(f[0], ths)
    else:
        idx, val = O.findpeaks3d(f, ths)
    assert n == len(idx) > 0
    np.testing.assert_array_equal(got["i0"], idx[:, 0])
    np.testing.assert_array_equal(got["i1"], idx[:, 1])
    np.testing.assert_array_equal(got["i2"], idx[:, 2])
    np.testing.assert_array_equal(got["field"], val.astype(np.float32))


@pytest.mark.parametrize("shape", [(32, 24, 20), (128, 32, 36), (256, 16, 20)])
def test_findpeaks_nan_neighbourhoods(shape):
    """A NaN cell is no peak and makes none of its 26 neighbours one (each comparison with
    NaN is false in the reference's stencil), at grid edges (periodic wrap) too."""
    ctx = mk(shape, F32)
    f = smooth_field(shape, 7, F32)
    nx, ny, nz = shape
    for (z, y, x) in [(0, 0, 0), (nz - 1, ny // 2, nx - 1), (nz // 2, ny - 1, nx // 2), (5, 3, 127 % nx), (7, 9 % ny, 255 % nx),
                      (3, 5, 8)]:
        f[z, y, x] = np.nan
    n, rec = ctx.findpeaks(up_r(ctx, f), -10.0)
    from mcstar_b200 import records_to_host
    got = records_to_host(rec, F32)
    idx, _ = O.findpeaks3d(f, -10.0)
    assert n == len(idx) > 0
    np.testing.assert_array_equal(np.stack([got["i0"], got["i1"], got["i2"]], 1).astype(np.int64), idx)


@pytest.mark.parametrize("shape", [(64, 64, 64), (256, 48, 40)])
def test_findpeaks_async_while_stepping(shape):
    """pfc_findpeaks_async: the records go to pinned host memory while the stepper keeps
    stepping on the context's stream; after pfc_findpeaks_wait they equal pfc_findpeaks's.
    Too small a buffer gives PFC_ERR_CAPACITY at the wait; pageable memory is refused."""
    from mcstar_b200 import PfcError, Stepper
    st = Stepper(shape, math.pi / 4, 0.5, 0.3, dtype=F32)
    st.set_real(smooth_field(shape, 5, F32))
    field = st.real_device().contiguous().clone()
    n_sync, rec_sync = st.ctx.findpeaks(field, 0.0)
    assert n_sync > 0
    host = torch.empty(n_sync * 16 + 4096, dtype=torch.uint8).pin_memory()
    st.ctx.findpeaks_async(field, 0.0, host)
    st.step(5)  # the step's kernels on the context's stream, the search on the copy stream
    n, rec = st.ctx.findpeaks_wait()
    assert n == n_sync
    assert torch.equal(rec, rec_sync.cpu())
    small = torch.empty(16, dtype=torch.uint8).pin_memory()
    st.ctx.findpeaks_async(field, 0.0, small)
    with pytest.raises(PfcError) as e:
        st.ctx.findpeaks_wait()
    assert e.value.status == 5
    with pytest.raises(PfcError) as e:
        st.ctx.findpeaks_async(field, 0.0, torch.empty(4096, dtype=torch.uint8))
    assert e.value.status == 1
    with pytest.raises(PfcError) as e:
        st.ctx.findpeaks_wait()  # nothing in flight
    assert e.value.status == 1


def test_findpeaks_plateau_and_capacity():
    from mcstar_b200 import PfcError
    shape = (16, 16, 16)
    ctx = mk(shape, F32)
    f = np.zeros((16, 16, 16), dtype=F32)
    f[4, 4, 4] = f[4, 4, 5] = 1.0  # a two-cell plateau is not a strict maximum
    f[10, 10, 10] = 2.0
    f[12, 2, 7] = 0.5
    n, rec = ctx.findpeaks(up_r(ctx, f), 0.4)
    assert n == 2
    with pytest.raises(PfcError) as e:
        ctx.findpeaks(up_r(ctx, f), 0.4, capacity=1)
    assert e.value.status == 5


def test_findpeaks_vs_reference_cuda(tmp_path):
    ref = ref_lib(F32)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    shape = (32, 32, 32)
    nx, ny, nz = shape
    f = smooth_field(shape, 4, F64)
    k = O.r2c(f).astype(np.complex64)
    h = ref["create"](nx, ny, nz, 1)
    ref["set_kpsi"](h, k.ctypes.data)
    pk, bo = str(tmp_path / "peaks.txt"), str(tmp_path / "bo.txt")
    hx = 0.5
    ref["findpeaks"](h, hx, hx, hx, nx * hx, ny * hx, nz * hx, 0.0, 3.0, pk.encode(), bo.encode())
    ref["destroy"](h)
    ref_rows = sorted(tuple(r) for r in np.loadtxt(pk, ndmin=2).tolist())
    ctx = mk(shape, F32)
    b = up_c(ctx, k)
    real = ctx.empty_state()
    ctx.c2r(b, real)
    real[: ctx.n_real] /= ctx.n_real
    n, rec = ctx.findpeaks(real, 0.0)
    from mcstar_b200 import records_to_host
    got = records_to_host(rec, F32)
    mine = sorted((float("%f" % (np.float32(m["i0"]) * np.float32(hx))), float("%f" % (np.float32(m["i1"]) * np.float32(hx))),
                   float("%f" % (np.float32(m["i2"]) * np.float32(hx))), float("%f" % m["field"])) for m in got)
    assert len(mine) == len(ref_rows)
    np.testing.assert_allclose(np.array(mine)[:, :3], np.array(ref_rows)[:, :3], atol=0)
    np.testing.assert_allclose(np.array(mine)[:, 3], np.array(ref_rows)[:, 3], atol=2e-6)
