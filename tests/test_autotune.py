"""Autotuner: candidate grid, cache round trip and exactness guard (CPU, with an
injected timer), and a real tuning run on the GPU."""
import numpy as np
import pytest


def test_grid_and_cache_roundtrip(tmp_path, monkeypatch):
    from cosmokdtree_b200.autotune import Autotuner, config_key
    cache = tmp_path / "tune.json"
    tuner = Autotuner(str(cache))
    grid = {"leaf": (8, 16), "variant": (3, 2), "warps_per_block": (4,), "blocks_per_sm": (0,),
            "order": (0,)}
    cands = tuner.candidates(grid)
    assert len(cands) == 4
    cost = {(8, 3): 5.0, (8, 2): 7.0, (16, 3): 3.0, (16, 2): 4.0}
    fixed = [np.arange(10)]

    def timer(cfg):
        return cost[(cfg["leaf"], cfg["variant"])], fixed

    key = config_key(3, 32, "float64", True, 1 << 20, "B200")
    assert key == "d3-k32-float64-per-n4^10-B200"
    # apply() needs the library; stub it out so the CPU test exercises the search only
    monkeypatch.setattr(Autotuner, "apply", staticmethod(lambda cfg: int(cfg.get("leaf", 16))))
    best = tuner.tune(np.zeros((1 << 20, 3)), None, 32, boxsize=1.0, grid=grid, timer=timer,
                      key=key)
    assert (best["leaf"], best["variant"]) == (16, 3) and best["ms"] == 3.0
    again = Autotuner(str(cache))
    assert again.lookup(key)["leaf"] == 16 and again.lookup(key)["variant"] == 3
    assert again.lookup("missing") is None


def test_inexact_candidate_is_rejected(tmp_path, monkeypatch):
    from cosmokdtree_b200.autotune import Autotuner
    tuner = Autotuner(str(tmp_path / "t.json"))
    monkeypatch.setattr(Autotuner, "apply", staticmethod(lambda cfg: 16))
    grid = {"leaf": (16,), "variant": (3, 2), "warps_per_block": (4,), "blocks_per_sm": (0,),
            "order": (0,)}

    def timer(cfg):  # a candidate that disagrees with the first
        return 1.0, [np.arange(5) + (cfg["variant"] == 2)]

    with pytest.raises(RuntimeError):
        tuner.tune(np.zeros((100, 3)), None, 4, grid=grid, timer=timer, key="x")


@pytest.mark.gpu
def test_gpu_autotune_small(gpu, tmp_path):
    from cosmokdtree_b200 import autotune, kdtree, synth
    P = synth.clustered_periodic(1 << 16, seed=9, n_clusters=64)
    Q = P[np.random.default_rng(1).integers(0, len(P), 20000)]
    tuner = autotune.Autotuner(str(tmp_path / "tune.json"))
    grid = {"leaf": (8, 16), "variant": (7, 8), "warps_per_block": (2, 4), "blocks_per_sm": (0,),
            "order": (0, 2)}
    best = tuner.tune(P, Q, 16, boxsize=1.0, grid=grid, reps=2)
    assert len(best["results"]) == 16 and all(r["exact"] for r in best["results"])
    leaf = autotune.Autotuner.apply(best)
    t = kdtree.build_kdtree(P, leaf=leaf, boxsize=1.0)
    d, i = kdtree.knn_search(t, Q, 16)
    autotune.Autotuner.apply(autotune.DEFAULT_CONFIG)
    t0 = kdtree.build_kdtree(P, leaf=leaf, boxsize=1.0)
    d0, i0 = kdtree.knn_search(t0, Q, 16)
    np.testing.assert_array_equal(i, i0)
    np.testing.assert_array_equal(d, d0)
