"""Pair-tile autotuner for batched runs (tn93g_batch_run).

The pair kernel's tile is 8 x rpw rows by 32 columns (rpw = rows per warp: 1, 2 or 4) and it runs with 2 or 3
resident blocks per SM (128 or 80 registers a thread). Neither changes a result; the best choice depends on the
alignment length (per-pair work grows with the columns, the per-tile column-event staging with the tile height)
and on the GPU. The tuner times the pair stage of a one-alignment batch for every candidate on a calibration
alignment per length band (seeded synthetic data of the benchmark's shape, columns sliced to the band's
midpoint), keeps the fastest tile height per band and the fastest blocks-per-SM overall, and caches the result
per device name.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

BANDS = ((0, 1300), (1300, 2200), (2200, 1 << 30))  # alignment length (columns) bands
BAND_L = (1000, 1750, 2600)                          # calibration length of each band
RPW = (1, 2, 4)
BLOCKS = (2, 3)


def cache_path() -> Path:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return Path(base) / "swifttn93_b200" / "pair_tuning.json"


def band_of(L: int) -> int:
    for b, (lo, hi) in enumerate(BANDS):
        if lo <= L < hi:
            return b
    return len(BANDS) - 1


def rows_per_warp(tuning: dict, L: int) -> int:
    return int(tuning["rows_per_warp"][band_of(L)])


def tune(engine, n: int = 2500, reps: int = 2, seed: int = 77) -> dict:
    """Measures every (blocks per SM, tile height) on one calibration alignment per band; returns the choice and
    the measured pair-stage milliseconds."""
    import numpy as np

    from . import HostAlignment, Options, synth

    names, codes = synth.hiv_bench(seed=seed, n=n, L=max(BAND_L), clusters=max(1, n // 170), tag="tune")
    opts = Options(threshold=0.015, mode="resolve", resolve_fraction=0.05, min_overlap=500)
    ms = {}
    for b, L in enumerate(BAND_L):
        aln = HostAlignment(np.ascontiguousarray(codes[:, :L]), names)
        engine.batch_run([aln], [opts])  # warm-up
        for blocks in BLOCKS:
            for rpw in RPW:
                t = []
                for _ in range(reps):
                    engine.batch_run([aln], [opts], rows_per_warp=[rpw], pair_blocks=blocks)
                    t.append(engine.last_timings()["pair"])
                ms[f"{b}/{blocks}/{rpw}"] = min(t)
    best_blocks = min(BLOCKS, key=lambda bl: sum(min(ms[f"{b}/{bl}/{r}"] for r in RPW) for b in range(len(BANDS))))
    choice = [min(RPW, key=lambda r: ms[f"{b}/{best_blocks}/{r}"]) for b in range(len(BANDS))]
    return {"bands": [list(x) for x in BANDS], "calibration_L": list(BAND_L), "calibration_n": n,
            "pair_blocks": best_blocks, "rows_per_warp": choice, "pair_ms": ms}


def load_or_tune(engine, device_name: str, retune: bool = False) -> dict:
    p = cache_path()
    cache = {}
    if p.exists():
        try:
            cache = json.loads(p.read_text())
        except ValueError:
            cache = {}
    if not retune and device_name in cache:
        return cache[device_name]
    t = tune(engine)
    cache[device_name] = t
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(json.dumps(cache, indent=1))
    except OSError:
        pass
    return t
