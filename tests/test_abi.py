"""CPU tests of the boundary and of the host logic: the C-ABI library loads and
exports every symbol include/pfc_b200.h declares; host-side helpers behave like the
reference's (no GPU compute here)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def test_library_exports_every_declared_symbol():
    import mcstar_b200 as m
    lib = m.lib()
    header = open(os.path.join(ROOT, "include", "pfc_b200.h")).read()
    declared = set(re.findall(r"\b(pfc_[a-z0-9_]+)\s*\(", header))
    assert declared == set(m._lib.EXPORTED)
    for name in declared:
        assert hasattr(lib, name), name


def test_status_strings_and_null_context():
    import mcstar_b200 as m
    lib = m.lib()
    assert lib.pfc_status_string(0) == b"ok"
    assert lib.pfc_status_string(6).startswith(b"non-finite")
    assert lib.pfc_destroy(None) == m._lib.PFC_ERR_INVALID
    assert lib.pfc_last_error(None) == b"null context"
    assert lib.pfc_state_bytes(None) == 0


def test_create_rejects_bad_shapes_without_gpu_work():
    import mcstar_b200 as m
    lib = m.lib()
    h = ctypes.c_void_p()
    for shape in [(0, 4, 4), (8, 1, 4), (8, 8, -1)]:
        d = m._lib.PfcDesc(*shape, 0)
        assert lib.pfc_create(ctypes.byref(d), ctypes.byref(h)) == m._lib.PFC_ERR_INVALID
    d = m._lib.PfcDesc(8, 8, 8, 7)
    assert lib.pfc_create(ctypes.byref(d), ctypes.byref(h)) == m._lib.PFC_ERR_INVALID


def test_shape_tr_and_cpuarray_npy_roundtrip(tmp_path):
    from mcstar_b200 import CPUArray, shape_tr, AsCmpl
    assert shape_tr((5, 1, 1)) == (5,)
    assert shape_tr((5, 4, 1)) == (4, 5)
    assert shape_tr((5, 4, 3)) == (3, 4, 5)
    a = CPUArray((6, 5, 4), np.float64)
    rng = np.random.default_rng(0)
    data = rng.standard_normal((4, 5, 6))
    fn = tmp_path / "x.npy"
    np.save(fn, data)
    a.load(str(fn))
    out = tmp_path / "y.npy"
    a.save(str(out))
    np.testing.assert_array_equal(np.load(out), data)
    a.save(str(tmp_path / "c.npy"), AsCmpl)
    assert np.load(tmp_path / "c.npy").shape == (4, 5, 4)
    np.save(fn, data[:, :, :5])
    with pytest.raises(RuntimeError):
        a.load(str(fn))
    assert a.m_bytes == 4 * 5 * 4 * 2 * 8


def test_pfc_thermodynamics():
    from mcstar_b200 import mu, omega
    eps, psi0 = 0.3, -0.2
    assert mu(eps, psi0) == pytest.approx((1 - eps) * psi0 + psi0 ** 3)
    assert omega(eps, psi0) == pytest.approx(0.5 * (1 - eps) * psi0 ** 2 + 0.25 * psi0 ** 4 - mu(eps, psi0) * psi0)
    assert omega(eps, psi0, 1.5) == pytest.approx(1.5 - mu(eps, psi0) * psi0)


def test_initial_conditions():
    from mcstar_b200 import bcc_sphere, liquid_random, namp_from_temperature, BCC_Q
    assert np.allclose(np.linalg.norm(BCC_Q, axis=1), 1.0)
    psi = bcc_sphere((32, 32, 32), math.pi / 4, -0.2, 0.2, 6.0)
    assert psi.shape == (32, 32, 32)
    assert psi[0, 0, 0] == -0.2
    centre = psi[16, 16, 16]
    assert centre == pytest.approx(-0.2 + 0.2 * 6)
    a = liquid_random((8, 8, 8), -0.18, 0.05, 1)
    b = liquid_random((8, 8, 8), -0.18, 0.05, 1)
    np.testing.assert_array_equal(a, b)
    assert np.all(np.abs(a + 0.18) <= 0.05)
    assert namp_from_temperature(1e-3, 0.5) == pytest.approx(math.sqrt(2e-3 / 0.5))


def test_bond_table_format_matches_reference_writer():
    import io
    import pfc_oracle as O
    from mcstar_b200 import write_bond_table
    g = np.load(os.path.join(ROOT, "tests", "golden", "bond_fcc_perfect_f32.npz"))
    h = float(g["h"])
    res, _ = O.bond_order(g["idx"], g["field"], (h, h, h), float(g["ths"]), float(g["box"]), float(g["rlim"]))
    rows = np.stack([res[c] for c in O.BOND_COLUMNS], axis=1)
    buf = io.StringIO()
    write_bond_table(buf, rows)
    assert buf.getvalue() == O.format_bond_table(res)
    ref = open(os.path.join(ROOT, "tests", "golden", "bond_fcc_perfect_f32.txt")).read()
    assert buf.getvalue().splitlines()[0] == ref.splitlines()[0]
    assert len(buf.getvalue().splitlines()) == len(ref.splitlines())
