"""The autotuner on the GPU: the setting it picks on a sample is applied,
stored for the device and read back by apply(); results under it equal the
oracle's."""

from __future__ import annotations

import numpy as np
import pytest

from gpjson_b200 import datagen, tune
from oracle import oracle

PATHS = ["$.user.lang", "$.id", "$.entities.hashtags[0].text"]


@pytest.mark.gpu
def test_tuner_picks_applies_and_stores(gpjson, tmp_path, monkeypatch):
    monkeypatch.setenv("GPJSON_TUNING_DIR", str(tmp_path))
    for var in tune.ENV.values():
        monkeypatch.delenv(var, raising=False)
    data = datagen.tweets(8 << 20, seed=datagen.SEED_BASE + 70)
    try:
        out = tune.tune(gpjson, data, PATHS, 4, repeats=1, workload="tweets")
        chosen = out["tuning"]
        assert set(chosen) == set(tune.KNOBS) and len(out["measured_ms"]) >= 4
        applied = gpjson.tuning()
        for k in ("query_ctas_per_sm", "index_ctas_per_sm"):
            assert applied[k] == chosen[k]
        assert tune.apply(gpjson) == chosen
        f = gpjson.load_bytes(data)
        try:
            assert np.array_equal(f.query_paths(PATHS), oracle.query(data, PATHS, mt=True))
        finally:
            f.release()
    finally:
        gpjson.set_tuning(long_line_bytes=0, query_ctas_per_sm=0, index_ctas_per_sm=0, chunk_tiles=0)
