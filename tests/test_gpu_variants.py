"""The reference's other per-mode propagators (cuda/kernels/eom-exp.hpp, el.hpp,
el-exp.hpp, and the polynomial and anisotropic-noise updates of eom.hpp) through the
C ABI: against the oracle's restatement and against the reference's own kernels built
from its sources (oracle/_ref/libref_variants_*.so, libref_pfc_*.so)."""
import ctypes
import math
import os

import numpy as np
import pytest

import pfc_oracle as O
from conftest import REF_DIR, ref_lib
from test_gpu_kernels import F32, F64, down_c, mk, rand_c, up_c

pytestmark = pytest.mark.gpu

# FP32 results against an FP64 restatement: a few ulps of the largest mode
TOL = {F32: 4e-6, F64: 1e-12}
# The operators of the exponential forms are exp(-L dt) evaluated by the reference with
# expf, in single precision even for double fields; CUDA's expf and numpy's float32 exp
# may differ by one float ulp, so operator-vs-oracle checks allow 2 float ulps.
EXPF = 2.5e-7
SHAPES = [(16, 12, 10), (32, 32, 32), (64, 48, 1), (15, 9, 7)]


def rel_max(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


def lens_of(shape):
    return tuple(n * math.pi / 4 for n in shape[:2]) + ((shape[2] * math.pi / 4) if shape[2] > 1 else 1.0,)


def ref_variants(dtype):
    name = "libref_variants_f32.so" if dtype == F32 else "libref_variants_f64.so"
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    pre = "refv32_" if dtype == F32 else "refv64_"
    I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    sig = {"init_eom_op": ([I, I, I, D, D, D, D, D, P], None),
           "update_eom_exp": ([I, I, I, P, P, P, P, D, D, D, D, D, D, I, P], None),
           "update_el": ([I, I, I, P, P, D, D, D, D, D], ctypes.c_float),
           "init_el_op": ([I, I, I, D, D, D, D, D, P], None),
           "update_el_exp": ([I, I, I, P, P, P, D, D, D, D, D], ctypes.c_float)}
    out = {}
    for k, (a, r) in sig.items():
        f = getattr(L, pre + k)
        f.argtypes, f.restype = a, r
        out[k] = f
    return out


def ref_extra(dtype):
    """The polynomial and anisotropic-noise updates of the reference's eom.hpp (libref_pfc)."""
    name = "libref_pfc_f32.so" if dtype == F32 else "libref_pfc_f64.so"
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    pre = "ref32_" if dtype == F32 else "ref64_"
    P, D = ctypes.c_void_p, ctypes.c_double
    f = getattr(L, pre + "update_eom_py")
    f.argtypes, f.restype = [P, P, P, P, D, D, D, D, D, D], None
    g = getattr(L, pre + "update_eom_hpfcnoise")
    g.argtypes, g.restype = [P, P, P, P, P, P, D, D, D, D, D, D], None
    return {"update_eom_py": f, "update_eom_hpfcnoise": g}


def cplx(dtype):
    return np.complex64 if dtype == F32 else np.complex128


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_exponential_conserved_update(shape, dtype):
    ctx = mk(shape, dtype)
    lens, dt, eps, namp = lens_of(shape), 0.5, 0.3, 0.01
    kop = ctx.empty_state()
    ctx.init_eom_op(kop, dt, eps, lens)
    kop_w = O.init_eom_op(shape, lens, dt, eps)
    got_kop = down_c(ctx, kop)
    assert rel_max(got_kop.real, kop_w.real) < max(TOL[dtype], EXPF)
    # the second factor (e - 1)/L inherits the float ulp of e, amplified where L dt is
    # small; in single precision it also loses digits to the subtraction
    assert rel_max(got_kop.imag, kop_w.imag) < (2e-4 if dtype == F32 else 1e-5)
    kp, kn, kz = rand_c(shape, dtype, 1), rand_c(shape, dtype, 2), rand_c(shape, dtype, 3)
    for noise, fen in [(False, False), (True, False), (True, True)]:
        b, q, z = up_c(ctx, kp), up_c(ctx, kn), up_c(ctx, kz)
        ctx.update_eom_exp(kop, b, q, z if noise else None, namp, eps, lens, with_fen=fen)
        want = O.update_eom_exp(got_kop.astype(np.complex128), kp, kn, kz if noise else None, namp, eps, lens, shape,
                                with_fen=fen)
        if fen:
            want, lk = want
            assert rel_max(down_c(ctx, z), lk) < TOL[dtype]
        assert rel_max(down_c(ctx, b), want) < TOL[dtype]
    ref = ref_variants(dtype)
    if ref is not None:
        nx, ny, nz = shape
        rk = np.zeros(O.cmpl_shape(shape), dtype=cplx(dtype))
        ref["init_eom_op"](nx, ny, nz, dt, eps, *lens, rk.ctypes.data)
        assert rel_max(got_kop.real, rk.real) < TOL[dtype]
        assert rel_max(got_kop.imag, rk.imag) < (2e-5 if dtype == F32 else 1e-12)
        p = kp.copy()
        fen_out = np.zeros_like(p)
        ref["update_eom_exp"](nx, ny, nz, rk.ctypes.data, p.ctypes.data, kn.ctypes.data, kz.ctypes.data, namp, dt,
                              eps, *lens, 1, fen_out.ctypes.data)
        kop_ref = up_c(ctx, rk)
        b, q, z = up_c(ctx, kp), up_c(ctx, kn), up_c(ctx, kz)
        ctx.update_eom_exp(kop_ref, b, q, z, namp, eps, lens, with_fen=True)
        assert rel_max(down_c(ctx, b), p) < TOL[dtype]
        assert rel_max(down_c(ctx, z), fen_out) < TOL[dtype]


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_relaxation_updates_and_largest_change(shape, dtype):
    ctx = mk(shape, dtype)
    lens, dt, eps = lens_of(shape), 0.5, 0.3
    kp, kn = rand_c(shape, dtype, 4), rand_c(shape, dtype, 5)
    b, q = up_c(ctx, kp), up_c(ctx, kn)
    m = ctx.update_el(b, q, dt, eps, lens)
    want, mw = O.update_el(kp, kn, dt, eps, lens, shape)
    assert rel_max(down_c(ctx, b), want) < TOL[dtype]
    assert abs(m - mw) <= 1e-6 * mw

    kop = ctx.empty_state()
    ctx.init_el_op(kop, dt, eps, lens)
    got_kop = down_c(ctx, kop)
    kop_w = O.init_el_op(shape, lens, dt, eps)
    assert rel_max(got_kop, kop_w) < max(TOL[dtype], EXPF * 4)  # expf, see EXPF
    b, q = up_c(ctx, kp), up_c(ctx, kn)
    m = ctx.update_el_exp(kop, b, q)
    want, mw = O.update_el_exp(got_kop.astype(np.complex128), kp, kn)
    assert rel_max(down_c(ctx, b), want) < TOL[dtype]
    assert abs(m - mw) <= 1e-6 * mw

    ref = ref_variants(dtype)
    if ref is not None:
        nx, ny, nz = shape
        p = kp.copy()
        mr = ref["update_el"](nx, ny, nz, p.ctypes.data, kn.ctypes.data, dt, eps, *lens)
        b, q = up_c(ctx, kp), up_c(ctx, kn)
        m = ctx.update_el(b, q, dt, eps, lens)
        assert rel_max(down_c(ctx, b), p) < TOL[dtype]
        assert abs(m - mr) <= 1e-6 * mr
        rk = np.zeros(O.cmpl_shape(shape), dtype=cplx(dtype))
        ref["init_el_op"](nx, ny, nz, dt, eps, *lens, rk.ctypes.data)
        assert rel_max(got_kop, rk) < TOL[dtype]
        p = kp.copy()
        mr = ref["update_el_exp"](nx, ny, nz, rk.ctypes.data, p.ctypes.data, kn.ctypes.data, dt, eps, *lens)
        kop_ref, b, q = up_c(ctx, rk), up_c(ctx, kp), up_c(ctx, kn)
        m = ctx.update_el_exp(kop_ref, b, q)
        assert rel_max(down_c(ctx, b), p) < TOL[dtype]
        assert abs(m - mr) <= 1e-6 * mr


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_polynomial_kernel_update(shape, dtype):
    ctx = mk(shape, dtype)
    lens, dt, eps, namp = lens_of(shape), 0.1, 0.3, 0.02
    kp, kn, kz = rand_c(shape, dtype, 6), rand_c(shape, dtype, 7), rand_c(shape, dtype, 8)
    b = up_c(ctx, kp)
    ctx.update_eom_py(b, up_c(ctx, kn), up_c(ctx, kz), namp, dt, eps, lens)
    want = O.update_eom_py(kp, kn, kz, namp, dt, eps, lens, shape)
    # P(k^2) (coefficients up to ~180) cancels strongly, so FP32 arithmetic -- the
    # reference's own, checked tightly below -- is ~1e-4 from the FP64 restatement
    assert rel_max(down_c(ctx, b), want) < (5e-4 if dtype == F32 else 1e-11)
    ref, L = ref_lib(dtype), ref_extra(dtype)
    if ref is not None and L is not None:
        nx, ny, nz = shape
        h = ref["create"](nx, ny, nz, 1)
        p = kp.copy()
        L["update_eom_py"](h, p.ctypes.data, kn.ctypes.data, kz.ctypes.data, namp, dt, eps, *lens)
        ref["destroy"](h)
        assert rel_max(down_c(ctx, b), p) < TOL[dtype] * 4


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("shape", [(64, 48, 1), (128, 128, 1), (30, 20, 1)], ids=lambda s: "x".join(map(str, s)))
def test_anisotropic_noise_update_2d(shape, dtype):
    ctx = mk(shape, dtype)
    lens, dt, eps, namp = (shape[0] * 2.0, shape[1] * 2.0, 1.0), 0.5, 0.3, 0.05  # dx = 2: modes below |k| = 0.25
    kp, kn = rand_c(shape, dtype, 9), rand_c(shape, dtype, 10)
    n1, n2, n3 = (rand_c(shape, dtype, s) for s in (11, 12, 13))
    b = up_c(ctx, kp)
    ctx.update_eom_hpfcnoise(b, up_c(ctx, kn), up_c(ctx, n1), up_c(ctx, n2), up_c(ctx, n3), namp, dt, eps, lens)
    want = O.update_eom_hpfcnoise(kp, kn, n1, n2, n3, namp, dt, eps, lens, shape, dtype=dtype)
    assert rel_max(down_c(ctx, b), want) < TOL[dtype]
    ref, L = ref_lib(dtype), ref_extra(dtype)
    if ref is not None and L is not None:
        nx, ny, nz = shape
        h = ref["create"](nx, ny, nz, 1)
        p = kp.copy()
        L["update_eom_hpfcnoise"](h, p.ctypes.data, kn.ctypes.data, n1.ctypes.data, n2.ctypes.data, n3.ctypes.data,
                                  namp, dt, eps, *lens)
        ref["destroy"](h)
        assert rel_max(down_c(ctx, b), p) < TOL[dtype]


def test_anisotropic_noise_rejects_3d():
    from mcstar_b200 import PfcError
    ctx = mk((16, 16, 16), F32)
    bufs = [ctx.empty_state() for _ in range(5)]
    with pytest.raises(PfcError):
        ctx.update_eom_hpfcnoise(*bufs, 0.1, 0.5, 0.3, (1.0, 1.0, 1.0))
