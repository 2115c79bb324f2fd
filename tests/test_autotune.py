"""The tile-shape autotuner's choice and cache (timings injected; the GPU
timing itself runs in the ensemble bench)."""
import importlib


def test_picks_the_fastest_and_caches(pkg, tmp_path):
    at = importlib.import_module("cadmas_b200.autotune")
    c = pkg.cases.random_tank(0)
    calls = []

    def fake(case, ti, tj, **kw):
        calls.append((ti, tj))
        return None if (ti, tj) == (32, 8) else {(16, 16): 3.0, (16, 8): 2.0, (8, 16): 2.5, (8, 8): 4.0}[(ti, tj)]

    cache = at.TileCache(tmp_path / "tiles.json")
    assert at.pick_tiles(c, cache=cache, measure=fake) == (16, 8)
    n = len(calls)
    # a second case of the same grid is answered from the cache, also after a reload
    assert at.pick_tiles(c, cache=cache, measure=fake) == (16, 8)
    assert at.pick_tiles(c, cache=at.TileCache(tmp_path / "tiles.json"), measure=fake) == (16, 8)
    assert len(calls) == n
    assert cache.data[at.grid_key(c)]["s_per_step"]["16x8"] == 2.0
