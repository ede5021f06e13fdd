"""The workloads the library is specified on, run end to end as written.

* 2D, 256 x 256, FP64: dx = pi/4, dt = 0.5, eps = 0.25, psi0 = -0.25 + U(-0.01, 0.01)
  (numpy PCG64), no noise, 1000 conserved semi-implicit steps; the free energy every 100
  steps and the 8-neighbour peak list of the final field.  Checked against the
  reference's own FP64 cuFFT path built from its sources (oracle/_ref): field, free
  energy (from the reference's per-cell energy density) and the peak text
  (findpeaks_2d.hpp:29-56).
* 3D, 128^3, FP32: dx = pi/4, dt = 0.5, eps = 0.3, psi0 = -0.2 with a bcc seed of radius
  20 (A = 0.2, the six <110>/sqrt(2) vectors), conserved Philox noise of amplitude
  sqrt(2 dt T) |k|, T = 1e-3, 2000 steps; every 100 steps the peaks and the bond order
  (q4, q6, w6, ...) of the stepper's own field, checked against the oracle on the same
  field (peaks bit-exact, bond order to 1e-9), and the mean density exactly conserved.
"""
import math

import numpy as np
import pytest

import pfc_oracle as O
from conftest import ref_lib

pytestmark = pytest.mark.gpu


def test_config_2d_256_fp64_1000_steps_against_reference(tmp_path):
    ref = ref_lib(np.float64)
    if ref is None:
        pytest.skip("oracle/_ref not built")
    from mcstar_b200 import Stepper, liquid_random, records_to_host
    n, dx, dt, eps = 256, math.pi / 4, 0.5, 0.25
    shape = (n, n, 1)
    lens = (n * dx, n * dx, 1.0)
    hh = (dx, dx, 1.0)
    psi = liquid_random(shape, -0.25, 0.01, 42)
    k0 = np.ascontiguousarray(O.r2c(psi))
    h = ref["create"](n, n, 1, 1)
    ref["set_kpsi"](h, k0.ctypes.data)
    st = Stepper(shape, dx, dt, eps, dtype=np.float64)
    st.set_kspace(k0)
    st.hh = hh
    dens = np.zeros((1, n, n), dtype=np.float64)
    for block in range(10):
        ref["step"](h, 100, 0.0, dt, eps, *lens, 0.0, 0)
        st.step(100)
        # the reference's free energy path (eom.hpp:88-141) leaves the energy density of every
        # cell in lpsi; its returned total is not used: call_kernel_calc_fen accumulates into
        # pinned memory it never clears (cudaMallocHost, eom.hpp:133-137), so a reused
        # allocation carries the previous call's sum.  The density is summed here in FP64.
        ref["free_energy"](h, eps, *lens, *hh, dens.ctypes.data)
        f_ref = float(dens.sum()) * hh[0] * hh[1] * hh[2]
        f_mine = st.free_energy()
        assert abs(f_mine - f_ref) <= 1e-10 * abs(f_ref), (block, f_mine, f_ref)
    want = np.zeros((1, n, n), dtype=np.float64)
    ref["get_psi"](h, want.ctypes.data)
    got = st.real()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-9
    assert abs(st.mean_density() - psi.mean()) < 1e-14
    # the 8-neighbour peak list, in the reference's text form
    pk = str(tmp_path / "peaks.txt")
    ref["findpeaks"](h, dx, dx, 1.0, *lens, -1.0, 1.0, pk.encode(), str(tmp_path / "unused").encode())
    ref["destroy"](h)
    ref_rows = sorted(tuple(r) for r in np.loadtxt(pk, ndmin=2).tolist())
    cnt, rec = st.peaks(-1.0)
    m = records_to_host(rec, np.float64)
    mine = sorted((float("%f" % np.float32(m["i0"][i] * dx)), float("%f" % np.float32(m["i1"][i] * dx)),
                   float("%f" % np.float32(m["i2"][i] * 1.0)), float("%f" % m["field"][i])) for i in range(cnt))
    assert cnt == len(ref_rows) > 0
    np.testing.assert_array_equal(np.array(mine)[:, :3], np.array(ref_rows)[:, :3])
    np.testing.assert_allclose(np.array(mine)[:, 3], np.array(ref_rows)[:, 3], atol=2e-6)


def test_config_3d_128_fp32_noise_2000_steps_peaks_and_bond_order():
    from mcstar_b200 import Stepper, bcc_sphere, namp_from_temperature, records_to_host
    n, dx, dt, eps, T = 128, math.pi / 4, 0.5, 0.3, 1e-3
    shape = (n, n, n)
    st = Stepper(shape, dx, dt, eps, dtype=np.float32, namp=namp_from_temperature(T, dt), seed=2)
    st.set_real(bcc_sphere(shape, dx, -0.2, 0.2, 20.0))
    k0 = st.kpsi[:2].double().cpu().numpy().copy()
    counts = []
    for block in range(20):
        st.step(100)
        field = st.real()
        cnt, rec = st.peaks(0.0)
        m = records_to_host(rec, np.float32)
        idx = np.stack([m["i0"], m["i1"], m["i2"]], axis=1).astype(np.int64)
        widx, wval = O.findpeaks3d(field, 0.0)
        assert np.array_equal(idx, widx), block
        np.testing.assert_array_equal(m["field"], wval.astype(np.float32))
        rows = st.ctx.bond_order(rec, cnt, st.hh, 0.0, st.lens[0], 10.0).cpu().numpy()
        res, _ = O.bond_order(idx, m["field"], st.hh, 0.0, st.lens[0], 10.0)
        assert rows.shape[0] == len(res["x"])
        for i, c in enumerate(O.BOND_COLUMNS):
            np.testing.assert_allclose(rows[:, i], res[c], atol=1e-9, err_msg=f"{c} at step {100 * (block + 1)}")
        counts.append(cnt)
    # the mean density (k = 0 mode) is carried in FP64 and restored: unchanged to the bit
    assert np.array_equal(st.kpsi[:2].double().cpu().numpy(), k0)
    # the seed is a bcc crystal: its atoms stay (it neither melts nor vanishes at T = 1e-3)
    assert min(counts) > 50
    q6 = rows[:, O.BOND_COLUMNS.index("q6")]
    assert 0.3 < float(np.median(q6)) < 0.7
