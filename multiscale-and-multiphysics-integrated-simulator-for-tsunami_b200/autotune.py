"""Tile-shape autotuner for the MILU preconditioner blocks.

The solver cuts the interior into blocks of precond_ti x precond_tj columns
(block-Jacobi MILU, as the reference under PARALLEL X/Y with one rank per
block).  The shape sets both the time of a sweep (wavefront length and the
number of thread blocks on the 148 SMs) and the number of BiCGSTAB
iterations (larger blocks precondition better).  `pick_tiles` times a few
steps of the case itself for each candidate shape and keeps the fastest;
every candidate meets the same stopping test.  Choices are cached by grid
size, so members of an ensemble with the same grid are tuned once.
"""
from __future__ import annotations

import json
import pathlib
import time

CANDIDATES = [(16, 16), (16, 8), (8, 16), (32, 8), (8, 8)]


def grid_key(case) -> str:
    return f"{case.ni - 2}x{case.nj - 2}x{case.nk - 2}"


def measure_gpu(case, ti, tj, steps=3, warmup=2, **params):
    """Seconds per step of the case with ti x tj blocks (None if the library
    refuses the shape)."""
    from . import CadmasError, Tank
    try:
        tank = Tank(case, precond_ti=ti, precond_tj=tj, **params)
    except CadmasError:
        return None
    try:
        tank.init_state(case.hydrostatic)
        for _ in range(warmup):
            tank.step(case.dt)
        tank.sync()
        t0 = time.perf_counter()
        for _ in range(steps):
            tank.step(case.dt)
        tank.sync()
        return (time.perf_counter() - t0) / steps
    finally:
        tank.close()


class TileCache:
    """Chosen shapes by grid size, optionally kept in a JSON file."""

    def __init__(self, path=None):
        self.path = pathlib.Path(path) if path else None
        self.data = {}
        if self.path and self.path.exists():
            self.data = json.loads(self.path.read_text())

    def get(self, key):
        v = self.data.get(key)
        return tuple(v["tiles"]) if v else None

    def put(self, key, tiles, timings):
        self.data[key] = {"tiles": list(tiles), "s_per_step": timings}
        if self.path:
            self.path.write_text(json.dumps(self.data, indent=1, sort_keys=True) + "\n")


def pick_tiles(case, candidates=CANDIDATES, cache=None, measure=None, **params):
    """The fastest (ti, tj) of the candidates for this case's grid."""
    key = grid_key(case)
    if cache is not None:
        hit = cache.get(key)
        if hit is not None:
            return hit
    measure = measure or measure_gpu
    timings = {}
    for ti, tj in candidates:
        s = measure(case, ti, tj, **params)
        if s is not None:
            timings[f"{ti}x{tj}"] = s
    if not timings:
        raise RuntimeError(f"no candidate tile shape runs grid {key}")
    best = min(timings, key=timings.get)
    tiles = tuple(int(v) for v in best.split("x"))
    if cache is not None:
        cache.put(key, tiles, timings)
    return tiles


# ---- co-scheduled tuning of a batch -------------------------------------
# A batch (cadmas_batch_step) solves all its grids together with one block
# shape, so the shape is chosen by timing the whole batch stepping together
# for each candidate: the members' kernels then share the SMs as they will
# in the run, which timing each member alone does not show.
BATCH_CANDIDATES = [(16, 16), (16, 8), (8, 16), (32, 8)]


def measure_batch(cases, ti, tj, steps=2, warmup=2, **params):
    """Seconds per step of all the cases stepped together as one batch with
    ti x tj blocks (None if the library refuses the shape)."""
    from . import Batch, CadmasError, Tank
    tanks, batch = [], None
    try:
        try:
            for c in cases:
                tanks.append(Tank(c, precond_ti=ti, precond_tj=tj, **params))
            batch = Batch(tanks)
        except CadmasError:
            return None
        for t, c in zip(tanks, cases):
            t.init_state(c.hydrostatic)
        for _ in range(warmup):
            batch.step()
        for t in tanks:
            t.sync()
        t0 = time.perf_counter()
        for _ in range(steps):
            batch.step()
        for t in tanks:
            t.sync()
        return (time.perf_counter() - t0) / steps
    finally:
        if batch is not None:
            batch.close()
        for t in tanks:
            t.close()


def pick_batch_tiles(cases, candidates=BATCH_CANDIDATES, measure=None, **params):
    """(ti, tj) of the candidates with which the batch of `cases` steps
    fastest, timed co-scheduled; and the seconds per step of each."""
    measure = measure or measure_batch
    timings = {}
    for ti, tj in candidates:
        s = measure(cases, ti, tj, **params)
        if s is not None:
            timings[f"{ti}x{tj}"] = s
    if not timings:
        raise RuntimeError("no candidate tile shape runs the batch")
    best = min(timings, key=timings.get)
    return tuple(int(v) for v in best.split("x")), timings
