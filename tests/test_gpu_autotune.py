"""The project's launch autotuner on a small uneven batch: it times every candidate (direct and pair
kernels over persistent grid sizes, TMA row tiles and stages), applies the fastest, leaves the
simulation state untouched, and the tuned batch evolves bit for bit like the default one (every
candidate runs the same per-cell arithmetic).  The choice is cached per GPU, precision and window
classes, and a second batch of the same classes takes it from the cache."""

import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _specs():
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import WindowSpec

    wins = [wgen.make_window(48, "preloaded", 3), wgen.make_window(64, "passive", 4),
            wgen.make_window(48, "skeleton", 5), wgen.make_window(64, "preloaded", 6)]
    return [WindowSpec(w.n, w.particles, 0.8, (1e-6, 0.0, 0.0), 4) for w in wins]


def test_tune_applies_a_faster_equivalent_launch_and_caches_it(tmp_path, monkeypatch):
    from particuology_hydraulic_penalty_b200 import autotune
    from particuology_hydraulic_penalty_b200.batch import PscBatch

    monkeypatch.setenv(autotune.CACHE_ENV, str(tmp_path / "autotune.json"))
    tuned = PscBatch(_specs(), precision="fp32", graph_steps=20)
    cfg = autotune.tune(tuned, steps=10)
    assert cfg["kernel"] in ("direct", "pair", "tma")
    kinds = {c["kernel"] for c, _ in cfg["candidates"]}
    assert {"direct", "pair", "tma"} <= kinds
    assert len({c.get("grid_ctas") for c, _ in cfg["candidates"] if c["kernel"] == "pair"}) == 4
    times = [t for _, t in cfg["candidates"]]
    assert cfg["ms_per_step"] == min(times) and all(t > 0.0 for t in times)
    assert tuned.steps_done == 0  # tuning restored the state it found

    default = PscBatch(_specs(), precision="fp32", graph_steps=20)
    tuned.run(60)
    default.run(60)
    for k in range(len(tuned.windows)):
        assert np.array_equal(tuned.velocity_field(k), default.velocity_field(k))

    cache = json.loads((tmp_path / "autotune.json").read_text())
    assert len(cache) == 1 and next(iter(cache.values()))["kernel"] == cfg["kernel"]
    again = PscBatch(_specs(), precision="fp32", graph_steps=20)
    cached = autotune.tune(again, steps=10)
    assert cached == cache[next(iter(cache))]
    assert again.launch_config()["kernel"] == cfg["kernel"]
    assert again.launch_config()["grid_ctas"] == cfg.get("grid_ctas", 0)
