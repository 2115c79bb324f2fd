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


def test_batch_shape_is_timed_on_the_whole_batch(pkg):
    """The batch tuner times every candidate on all the grids together (one
    call per shape with every case) and keeps the fastest; refused shapes
    are skipped."""
    at = importlib.import_module("cadmas_b200.autotune")
    cases = [pkg.cases.random_tank(s) for s in range(3)]
    seen = []

    def fake(cs, ti, tj, **kw):
        seen.append((len(cs), ti, tj))
        return None if (ti, tj) == (32, 8) else {(16, 16): 1.5, (16, 8): 1.2, (8, 16): 1.4}[(ti, tj)]

    tiles, timings = at.pick_batch_tiles(cases, measure=fake)
    assert tiles == (16, 8)
    assert all(n == 3 for n, _, _ in seen) and len(seen) == len(at.BATCH_CANDIDATES)
    assert set(timings) == {"16x16", "16x8", "8x16"}
