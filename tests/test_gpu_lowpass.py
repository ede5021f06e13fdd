"""The 2D spectral low-pass post-processing (cuda/kernels/gaussian.hpp, lowpass.hpp)
through the C ABI: against the oracle's restatement and against the reference's own
kernels and LOWPASS writer built from its sources (oracle/_ref/libref_lowpass_*.so)."""
import ctypes
import gzip
import math
import os

import numpy as np
import pytest
import torch

import pfc_oracle as O
from conftest import REF_DIR
from test_gpu_kernels import F32, F64, down_c, down_r, mk, up_c, up_r

pytestmark = pytest.mark.gpu

# exp is evaluated by CUDA (ours, the reference's) and numpy (oracle) in the field's
# precision: filter values in [0, 1] agree to two float ulps, or 1e-15 in FP64
GTOL = {F32: 2.5e-7, F64: 1e-15}
SHAPES2D = [(64, 48, 1), (128, 128, 1), (256, 64, 1), (60, 50, 1)]


def ref_lowpass(dtype):
    name = "libref_lowpass_f32.so" if dtype == F32 else "libref_lowpass_f64.so"
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    pre = "refl32_" if dtype == F32 else "refl64_"
    I, D, P, S = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p
    sig = {"gaussian_init": [I, I, I, D, D, D, D, D, D, D, P],
           "write_lowpass_2d": [I, I, P, P, D, D, S],
           "amplitude_lowpass": [I, I, P, P, D, D, S, P]}
    out = {}
    for k, a in sig.items():
        f = getattr(L, pre + k)
        f.argtypes, f.restype = a, None
        out[k] = f
    return out


def geometry(shape):
    h = (math.pi / 4, 0.8, 0.9 if shape[2] > 1 else 1.0)
    lens = tuple(n * hh for n, hh in zip(shape, h))
    return lens, h


def field2d(shape, dtype, seed=3):
    """A stripe / hexagonal pattern with noise, numpy shape (1, ny, nx)."""
    nx, ny, _ = shape
    (lx, ly, _), _ = geometry(shape)
    x = np.arange(nx) * lx / nx
    y = np.arange(ny) * ly / ny
    X, Y = np.meshgrid(x, y)
    q = 2 * math.pi / lx * max(1, nx // 8)
    psi = 0.3 * np.cos(q * X) + 0.2 * np.cos(2 * math.pi / ly * max(1, ny // 8) * Y)
    psi += 0.05 * np.random.default_rng(seed).standard_normal(psi.shape)
    return psi[None].astype(dtype)


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", SHAPES2D + [(32, 16, 8)], ids=lambda s: "x".join(map(str, s)))
def test_gaussian_filter(shape, dtype):
    ctx = mk(shape, dtype)
    lens, h = geometry(shape)
    g = ctx.empty_state()
    ctx.gaussian_init(g, lens, h, 2.0)
    got = down_c(ctx, g)
    want = O.gaussian_init(shape, lens, h, 2.0, dtype)
    assert np.max(np.abs(got - want)) <= GTOL[dtype]
    assert got[0, 0, 0] == 1.0  # e = 1 at k = 0
    ref = ref_lowpass(dtype)
    if ref is not None:
        r = np.zeros_like(want)
        ref["gaussian_init"](*shape, *lens, *h, 2.0, r.ctypes.data)
        assert np.max(np.abs(got - r)) <= GTOL[dtype]


@pytest.mark.parametrize("dtype", [F32, F64])
def test_kmult_and_square_are_exact(dtype):
    shape = (64, 48, 1)
    ctx = mk(shape, dtype)
    lens, h = geometry(shape)
    rng = np.random.default_rng(5)
    nxh = shape[0] // 2 + 1
    X = (rng.standard_normal((1, 48, nxh)) + 1j * rng.standard_normal((1, 48, nxh))).astype(
        np.complex64 if dtype == F32 else np.complex128)
    gk = O.gaussian_init(shape, lens, h, 1.5, dtype)
    g = up_c(ctx, gk)
    for imag in (False, True):
        a = up_c(ctx, X)
        (ctx.kmult_imag if imag else ctx.kmult_real)(a, g)
        assert np.array_equal(down_c(ctx, a), O.kmult(X, gk, imag))
    r = rng.standard_normal((1, 48, 64)).astype(dtype)
    b = up_r(ctx, r)
    ctx.square(b)
    assert np.array_equal(down_r(ctx, b), r * r)


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", [(64, 48, 1), (128, 96, 1), (1024, 1024, 1)], ids=lambda s: "x".join(map(str, s)))
def test_lowpass_dump_matches_reference_bytes(shape, dtype, tmp_path):
    """Same spectrum and filter in, the same LOWPASS file out: the decompressed text equals
    the reference writer's byte for byte (and the oracle's).  A text of one compression
    chunk (1 MB) also gives the same gzip file; longer texts are compressed in parallel
    chunks (gzip.decompress checks their combined CRC-32 and length)."""
    ctx = mk(shape, dtype)
    lens, h = geometry(shape)
    spec = O.r2c(field2d(shape, dtype))
    gk = O.gaussian_init(shape, lens, h, 2.0, dtype)
    ours = tmp_path / "ours.gz"
    s = up_c(ctx, spec)
    ctx.write_lowpass_2d(s, up_c(ctx, gk), lens, str(ours))
    text = gzip.decompress(ours.read_bytes())
    assert text == O.lowpass_text(O.kmult(spec, gk)[0], shape[0], shape[1], lens[0], lens[1], dtype)
    assert np.array_equal(down_c(ctx, s), O.kmult(spec, gk))  # the spectrum is low-passed in place
    ref = ref_lowpass(dtype)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    theirs = tmp_path / "ref.gz"
    ref["write_lowpass_2d"](shape[0], shape[1], np.ascontiguousarray(spec).ctypes.data,
                            np.ascontiguousarray(gk).ctypes.data, lens[0], lens[1], str(theirs).encode())
    assert gzip.decompress(theirs.read_bytes()) == text
    if len(text) <= 1 << 20:
        assert theirs.read_bytes() == ours.read_bytes()
    else:
        assert len(text) > 4 << 20  # several chunks


def parse_dump(raw):
    text = gzip.decompress(raw).decode()
    head, rest = text.split("\n", 2)[:2], text.split("\n", 2)[2]
    n = int(head[1])
    pickle, body = rest[:n], rest[n:]
    rows = {}
    for ln in body.splitlines():
        i0, i1, re, im = ln.split()
        rows[(int(i0), int(i1))] = complex(float(re), float(im))
    return head[0], pickle, rows


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", SHAPES2D, ids=lambda s: "x".join(map(str, s)))
def test_amplitude_lowpass(shape, dtype, tmp_path):
    ctx = mk(shape, dtype)
    lens, h = geometry(shape)
    psi = field2d(shape, dtype)
    spec = O.r2c(psi)
    gk = O.gaussian_init(shape, lens, h, 2.0, dtype)
    s, aux = up_c(ctx, spec), ctx.empty_state()
    ours = tmp_path / "ours.gz"
    ctx.amplitude_lowpass(s, aux, up_c(ctx, gk), lens, str(ours))
    amp = down_r(ctx, aux)
    want_amp, want_low = O.amplitude_lowpass(spec, gk, shape)
    tol = 2e-5 if dtype == F32 else 1e-11
    assert np.linalg.norm(amp - want_amp) / np.linalg.norm(want_amp) < tol
    assert np.linalg.norm(down_c(ctx, s) - want_low) / np.linalg.norm(want_low) < tol
    tag, pickle, rows = parse_dump(ours.read_bytes())
    assert tag == "LOWPASS" and pickle.startswith("(S'n0'\nI%d\n" % shape[0])
    ref = ref_lowpass(dtype)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    theirs = tmp_path / "ref.gz"
    ramp = np.zeros((1, shape[1], shape[0]), dtype=dtype)
    ref["amplitude_lowpass"](shape[0], shape[1], np.ascontiguousarray(spec).ctypes.data,
                             np.ascontiguousarray(gk).ctypes.data, lens[0], lens[1], str(theirs).encode(),
                             ramp.ctypes.data)
    assert np.linalg.norm(amp - ramp) / np.linalg.norm(ramp) < tol
    rtag, rpickle, rrows = parse_dump(theirs.read_bytes())
    assert (rtag, rpickle) == (tag, pickle)
    # the entries: the same modes except, at most, a few whose |a|^2 sits at the 1e-6
    # threshold; the printed values agree to the 6 digits printed (FFT rounding aside)
    common = rows.keys() & rrows.keys()
    assert len(rows.keys() ^ rrows.keys()) <= max(2, len(common) // 1000)
    scale = max(abs(v) for v in rrows.values())
    assert max(abs(rows[k] - rrows[k]) for k in common) <= 2e-5 * scale


def test_amplitude_of_a_cosine_known_answer():
    """psi = A cos(q x): amplitude = (1 - e_q)^2 A^2/2 (1 + e_2q cos 2qx), e the filter."""
    shape, dtype = (128, 32, 1), F64
    ctx = mk(shape, dtype)
    lens, h = geometry(shape)
    nx = shape[0]
    x = np.arange(nx) * lens[0] / nx
    m = 6
    q = 2 * math.pi * m / lens[0]
    A = 0.7
    psi = np.broadcast_to(A * np.cos(q * x), (1, shape[1], nx)).astype(dtype)
    gk = O.gaussian_init(shape, lens, h, 1.0, dtype)
    s, aux = up_c(ctx, O.r2c(psi)), ctx.empty_state()
    ctx.amplitude_lowpass(s, aux, up_c(ctx, gk), lens)
    eq, e2q = gk[0, 0, m].real, gk[0, 0, 2 * m].real
    want = (1 - eq) ** 2 * A * A / 2 * (1 + e2q * np.cos(2 * q * x))
    np.testing.assert_allclose(down_r(ctx, aux)[0], np.broadcast_to(want, (shape[1], nx)), atol=1e-13)


def test_lowpass_rejects_3d_grids(tmp_path):
    from mcstar_b200 import PfcError
    from mcstar_b200._lib import PFC_ERR_INVALID
    ctx = mk((16, 16, 16), F32)
    a, b, g = ctx.empty_state(), ctx.empty_state(), ctx.empty_state()
    for call in (lambda: ctx.amplitude_lowpass(a, b, g, (1, 1, 1)),
                 lambda: ctx.write_lowpass_2d(a, g, (1, 1, 1), str(tmp_path / "x.gz"))):
        with pytest.raises(PfcError) as err:
            call()
        assert err.value.status == PFC_ERR_INVALID


def test_lowpass_unwritable_path_is_reported(tmp_path):
    from mcstar_b200 import PfcError
    from mcstar_b200._lib import PFC_ERR_INVALID
    ctx = mk((32, 32, 1), F32)
    a, g = ctx.empty_state(), ctx.empty_state()
    with pytest.raises(PfcError) as err:
        ctx.write_lowpass_2d(a, g, (1, 1, 1), str(tmp_path / "no" / "such" / "dir" / "x.gz"))
    assert err.value.status == PFC_ERR_INVALID
