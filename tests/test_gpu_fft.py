"""FFT parity on the GPU, through the C ABI: the reference's own FFT tests
(cufft_unittest/my_unit_test.py) with its shapes and tolerances, plus a direct
comparison with the reference's cuFFT wrapper when oracle/_ref is built."""
import math

import numpy as np
import pytest
import torch

import pfc_oracle as O
from conftest import ref_lib

pytestmark = pytest.mark.gpu

# numpy shapes (l1, l2, l3) of TestA/TestB (my_unit_test.py:74-77); the binary receives
# n0 = l3 (x, fastest), n1 = l2, n2 = l1
SHAPES = list(zip([36, 20, 625, 30, 30, 27, 24, 60, 27, 10], [75, 20, 10, 40, 10, 36, 6, 30, 100, 18],
                  [60, 45, 9, 16, 25, 27, 150, 150, 6, 75]))
TOL = {np.float32: 1e-5, np.float64: 1e-14}


def ctx_for(nshape, dtype):
    from mcstar_b200 import get_context
    nz, ny, nx = nshape
    return get_context((nx, ny, nz), dtype)


def dev_real(ctx, x):
    b = ctx.empty_state()
    b[: x.size].copy_(torch.from_numpy(np.ascontiguousarray(x).ravel()))
    return b


def host_cmpl(ctx, b, nshape):
    nz, ny, nx = nshape
    return torch.view_as_complex(b.view(-1, 2)).view(nz, ny, nx // 2 + 1).cpu().numpy()


def r2c_gpu(x):
    ctx = ctx_for(x.shape, x.dtype)
    out = ctx.empty_state()
    ctx.r2c(dev_real(ctx, x), out)
    return host_cmpl(ctx, out, x.shape)


def c2r_gpu(X, nshape, dtype):
    ctx = ctx_for(nshape, dtype)
    b = ctx.empty_state()
    b.copy_(torch.from_numpy(np.ascontiguousarray(X).view(dtype).ravel()))
    out = ctx.empty_state()
    ctx.c2r(b, out)
    return out[: int(np.prod(nshape))].cpu().numpy().reshape(nshape)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nshape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_r2c_vs_numpy_testB(nshape, dtype):
    rng = np.random.default_rng(hash(nshape) % 1000)
    x = rng.standard_normal(nshape).astype(dtype)
    got = r2c_gpu(x)
    want = np.fft.rfftn(x.astype(np.float64))
    s = math.sqrt(x.size)
    err = np.max(np.abs(got / s - want / s))
    assert err <= TOL[dtype], err


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nshape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_roundtrip_testA(nshape, dtype):
    rng = np.random.default_rng(1 + hash(nshape) % 1000)
    x = rng.standard_normal(nshape).astype(dtype)
    X = r2c_gpu(x)
    y = c2r_gpu(X, nshape, dtype)
    err = np.max(np.abs(x - y / x.size))
    assert err <= TOL[dtype], err


@pytest.mark.parametrize("dtype,tol", [(np.float32, 1e-5), (np.float64, 1e-13)])
@pytest.mark.parametrize("n", [1200, 1280, 1600, 1152])
def test_large_2d_testC(n, dtype, tol):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((1, n, n)).astype(dtype)
    got = r2c_gpu(x)
    want = np.fft.rfftn(x.astype(np.float64))
    s = math.sqrt(x.size)
    assert np.max(np.abs(got / s - want / s)) <= tol


@pytest.mark.parametrize("nshape", [(1, 1, 64), (1, 1, 45), (1, 7, 9), (8, 6, 10), (3, 5, 1)])
def test_small_and_odd_shapes(nshape):
    rng = np.random.default_rng(7)
    x = rng.standard_normal(nshape)
    got = r2c_gpu(x)
    np.testing.assert_allclose(got, np.fft.rfftn(x), atol=1e-12)
    y = c2r_gpu(got, nshape, np.float64)
    np.testing.assert_allclose(y / x.size, x, atol=1e-13)


@pytest.mark.parametrize("nshape", [(64, 64, 64), (128, 64, 256), (512, 64, 128), (8, 512, 512), (64, 32, 64),
                                    (256, 128, 512), (3, 256, 64), (96, 192, 96), (192, 96, 192), (16, 192, 192),
                                    (192, 16, 16), (64, 160, 160), (160, 16, 16), (2, 1024, 1024)], ids=lambda s: "x".join(map(str, s)))
def test_register_transform_paths_fp32(nshape):
    """FP32 shapes: register x rows + y columns where nx and ny are in {64, 96, 128, 160,
    192, 256, 512, 1024}, register z columns where nz is, general passes for the other axes."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal(nshape).astype(np.float32)
    want = np.fft.rfftn(x.astype(np.float64))
    got = r2c_gpu(x)
    s = math.sqrt(x.size)
    assert np.max(np.abs(got - want)) / s <= TOL[np.float32]
    y = c2r_gpu(want.astype(np.complex64), nshape, np.float32)
    assert np.max(np.abs(y / x.size - x.astype(np.float64))) <= 1e-5


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_r2c_c2r_vs_reference_cufft(dtype):
    ref = ref_lib(dtype)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    import ctypes
    for nshape in [(36, 75, 60), (16, 32, 64), (1, 128, 96)]:
        nz, ny, nx = nshape
        rng = np.random.default_rng(5)
        x = rng.standard_normal(nshape).astype(dtype)
        h = ref["create"](nx, ny, nz, 1)
        cbuf = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex64 if dtype == np.float32 else np.complex128)
        ref["r2c"](h, x.ctypes.data, cbuf.ctypes.data)
        rbuf = np.zeros(nshape, dtype=dtype)
        ref["c2r"](h, cbuf.ctypes.data, rbuf.ctypes.data)
        ref["destroy"](h)
        got = r2c_gpu(x)
        s = math.sqrt(x.size)
        assert np.max(np.abs(got - cbuf)) / s <= 2 * TOL[dtype]
        y = c2r_gpu(cbuf, nshape, dtype)
        assert np.max(np.abs(y - rbuf)) / x.size <= 2 * TOL[dtype]
