"""The column-batch autotuner's cache key and cache file (no GPU): batches of the same
shape share an entry, a different shape gets its own, and a stored choice is read back."""
import json

import numpy as np

from lica_boiling1d_b200 import autotune
from lica_boiling1d_b200.column import ColumnBatch, uneven_batch


def test_batch_key_depends_on_the_shape_only():
    n, length, z0, props = uneven_batch(64, seed=0)
    a = ColumnBatch(n, length, props)
    b = ColumnBatch(n.copy(), length.copy(), props)
    c = ColumnBatch(n[:32], length[:32], props[:32])
    assert autotune.batch_key(a) == autotune.batch_key(b)
    assert autotune.batch_key(a) != autotune.batch_key(c)
    assert f"ncol=64,cells={int(np.sum(n))}" in autotune.batch_key(a)


def test_cache_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("LICA_TUNE_CACHE", str(path))
    autotune._store({"GPU|ncol=1": {"threads": 64, "tri_cap": 0, "ms_per_step": {"64/scratch": 1.0}}})
    assert json.loads(path.read_text())["GPU|ncol=1"]["threads"] == 64
    assert autotune._shape(autotune._load()["GPU|ncol=1"]) == (64, 0)
    assert autotune._shape({"threads": 128}) == (128, -1)       # an entry written before the cap axis
    assert autotune._shape({"threads": 96}) is None
    monkeypatch.setenv("LICA_TUNE_CACHE", str(tmp_path / "missing" / "x.json"))
    assert autotune._load() == {}


import pytest  # noqa: E402


@pytest.mark.gpu
def test_tune_picks_a_shape_leaves_the_state_and_caches(tmp_path, monkeypatch):
    import torch
    monkeypatch.setenv("LICA_TUNE_CACHE", str(tmp_path / "tune.json"))
    autotune._memo.clear()
    n, length, z0, props = uneven_batch(48, seed=3, nmin=64, nmax=256)
    batch = ColumnBatch.films(n, length, z0, props).to("cuda")
    before = {k: v.clone() for k, v in batch.arrays.items()}
    th, times = autotune.tune(batch)
    assert th in autotune.SHAPES and set(times) == {autotune._name(x) for x in autotune.SHAPES}
    assert times[autotune._name(th)] == min(times.values())
    for k, v in batch.arrays.items():
        assert torch.equal(v, before[k]), k          # the trial ran on a copy
    th2, times2 = autotune.tune(batch)
    assert th2 == th and times2 is None               # cached
    autotune._memo.clear()
    th3, times3 = autotune.tune(batch)                # from the file
    assert th3 == th and times3 is None
    st = batch.steps(2)                               # threads=0: the tuned shape
    assert int(st.max()) == 0
