"""GPU bond order (pfc_bond_order through the C ABI) against the reference's own
output (tests/golden, made by the compiled reference library) and against the oracle
(including w6, which the reference lacks)."""
import glob
import math
import os

import numpy as np
import pytest
import torch

import pfc_oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "bond_*.npz")))


def run_gpu(g):
    from mcstar_b200 import get_context, maximum_dtype
    dt = np.float32 if str(g["dtype"]) == "float32" else np.float64
    M = np.zeros(len(g["idx"]), dtype=maximum_dtype(dt))
    M["i0"], M["i1"], M["i2"] = g["idx"][:, 0], g["idx"][:, 1], g["idx"][:, 2]
    M["field"] = g["field"]
    dev = torch.from_numpy(M.view(np.uint8).ravel().copy()).cuda()
    ctx = get_context((64, 64, 64), dt)
    h = float(g["h"])
    return ctx.bond_order(dev, len(M), (h, h, h), float(g["ths"]), float(g["box"]), float(g["rlim"])).cpu().numpy()


@pytest.mark.parametrize("path", _cases(), ids=lambda p: os.path.basename(p)[5:-4])
def test_bond_order_gpu_vs_reference_and_oracle(path):
    g = np.load(path)
    rows = run_gpu(g)
    ref = O.parse_bond_table(open(path[:-4] + ".txt").read())
    assert rows.shape[0] == len(ref["x"])
    cols = {c: rows[:, i] for i, c in enumerate(O.BOND_COLUMNS)}
    for c in O.BOND_COLUMNS[:13]:
        tol = 1e-4 if c in ("q8", "q8b") else 1.5e-6
        np.testing.assert_allclose(cols[c], ref[c], atol=tol, rtol=0, err_msg=c)
    h = float(g["h"])
    res, _ = O.bond_order(g["idx"], g["field"], (h, h, h), float(g["ths"]), float(g["box"]), float(g["rlim"]))
    for c in O.BOND_COLUMNS:
        np.testing.assert_allclose(cols[c], res[c], atol=1e-10, rtol=0, err_msg=c)


def test_bond_order_from_stepper_peaks():
    """Peaks of a relaxed bcc seed -> bond order on the GPU, all on the device."""
    from mcstar_b200 import Stepper, bcc_sphere, records_to_host
    shape = (64, 64, 64)
    dx = math.pi / 4
    st = Stepper(shape, dx, 0.5, 0.3, dtype=np.float32)
    st.set_real(bcc_sphere(shape, dx, -0.2, 0.2, 20.0))
    st.step(20)
    n, rec = st.peaks(0.0)
    rows = st.ctx.bond_order(rec, n, st.hh, 0.0, st.lens[0], 10.0).cpu().numpy()
    m = records_to_host(rec, np.float32)
    idx = np.stack([m["i0"], m["i1"], m["i2"]], axis=1).astype(np.int64)
    res, _ = O.bond_order(idx, m["field"], st.hh, 0.0, st.lens[0], 10.0)
    assert rows.shape[0] == len(res["x"]) > 10
    for i, c in enumerate(O.BOND_COLUMNS):
        np.testing.assert_allclose(rows[:, i], res[c], atol=1e-9, err_msg=c)


def test_bond_order_beyond_initial_scratch_many_atoms_and_neighbours():
    """A perfect bcc crystal of 8192 sites with rlim past the eighth shell (112 neighbours
    per atom): more atoms and neighbour entries than a context's bond-order
    scratch starts with; the call grows it and matches the oracle.  A second call with
    fewer atoms reuses the grown scratch."""
    from mcstar_b200 import get_context, maximum_dtype
    n_cells, a = 16, 4  # lattice constant 4 grid cells
    g = np.arange(n_cells) * a
    corners = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    idx = np.concatenate([corners, corners + a // 2])
    idx = idx[np.lexsort((idx[:, 0], idx[:, 1], idx[:, 2]))]
    field = 0.1 + 1e-3 * np.random.default_rng(3).uniform(size=len(idx))
    h, box = 0.9, n_cells * a * 0.9
    rlim = 2.25 * a * h  # the bcc shells up to sqrt(5) a: 8 + 6 + 12 + 24 + 8 + 6 + 24 + 24 = 112 neighbours
    ctx = get_context((64, 64, 64), np.float32)
    for take in (len(idx), 3000):
        M = np.zeros(take, dtype=maximum_dtype(np.float32))
        M["i0"], M["i1"], M["i2"] = idx[:take, 0], idx[:take, 1], idx[:take, 2]
        M["field"] = field[:take]
        dev = torch.from_numpy(M.view(np.uint8).ravel().copy()).cuda()
        rows = ctx.bond_order(dev, take, (h, h, h), 0.0, box, rlim).cpu().numpy()
        res, nbrs = O.bond_order(idx[:take], M["field"], (h, h, h), 0.0, box, rlim)
        if take == len(idx):
            assert min(len(v) for v in nbrs) > 64
        assert rows.shape[0] == len(res["x"]) == take
        for i, c in enumerate(O.BOND_COLUMNS):
            np.testing.assert_allclose(rows[:, i], res[c], atol=1e-9, err_msg=c)
