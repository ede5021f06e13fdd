"""The autotuner of the kernel schedules (pfc_tune): it returns options every shape
accepts, the step under the tuned options matches the oracle, and results are cached in a
JSON file keyed by shape, precision and device (a cached entry comes back unchanged,
without timing)."""
import json
import math
import time

import numpy as np
import pytest

import pfc_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(64, 64, 64), (48, 40, 30), (128, 128, 1), (32, 16, 512)])
def test_tuned_schedule_matches_oracle_and_is_cached(shape, tmp_path):
    from mcstar_b200 import Stepper, tune
    cache = tmp_path / "tune.json"
    opts, ms = tune(shape, np.float32, str(cache))
    assert ms > 0.0
    entries = json.loads(cache.read_text())["entries"]
    assert len(entries) == 1
    (key, entry), = entries.items()
    assert key.startswith("x".join(str(v) for v in shape) + ":f32:")
    assert {k: entry[k] for k in opts} == opts
    # a second call reads the cache (the same entry, no timing: fast)
    t0 = time.perf_counter()
    again, ms2 = tune(shape, np.float32, str(cache))
    assert again == opts and ms2 == pytest.approx(ms, rel=1e-5)
    assert time.perf_counter() - t0 < 0.5
    nx, ny, nz = shape
    st = Stepper(shape, math.pi / 4, 0.5, 0.3, dtype=np.float32, namp=0.02, seed=3, options=opts)
    assert st.ctx.options == opts
    k = O.r2c(-0.2 + 0.1 * np.random.default_rng(8).uniform(-1, 1, (nz, ny, nx)))
    st.set_kspace(k.astype(np.complex64))
    st.step(4)
    want = O.step(k, 4, 0.5, 0.3, st.lens, shape, namp=0.02, seed=3, noise_dtype=np.float32)
    assert np.linalg.norm(st.kspace() - want) / np.linalg.norm(want) < 2e-6


def test_cache_holds_entries_of_several_shapes(tmp_path):
    from mcstar_b200 import tune
    cache = tmp_path / "tune.json"
    a, _ = tune((32, 32, 32), np.float32, str(cache))
    b, _ = tune((24, 24, 1), np.float64, str(cache))
    entries = json.loads(cache.read_text())["entries"]
    assert len(entries) == 2
    assert tune((32, 32, 32), np.float32, str(cache))[0] == a
    assert tune((24, 24, 1), np.float64, str(cache))[0] == b
