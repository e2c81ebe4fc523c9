"""The pair-tile autotuner's host logic (swifttn93_b200.autotune) with a stand-in engine whose pair-stage times are
made up: the choice per length band, the blocks-per-SM choice over all bands, and the per-device cache."""
import json

from swifttn93_b200 import autotune


class FakeEngine:
    """batch_run records the tile choice; last_timings returns a pair time that favours 3 blocks and, per band,
    a different tile height (1 for short, 2 for middle, 4 for long alignments)."""

    best = {1000: 1, 1750: 2, 2600: 4}

    def __init__(self):
        self.calls = 0
        self.last = None

    def batch_run(self, alns, opts, rows_per_warp=None, pair_blocks=0):
        self.calls += 1
        self.last = (alns[0].L, rows_per_warp[0] if rows_per_warp else 4, pair_blocks or 2)

    def last_timings(self):
        L, rpw, blocks = self.last
        t = 1.0 + abs(rpw - self.best[L]) * 0.1 + (0.0 if blocks == 3 else 0.05)
        return {"pair": t}


def test_band_of_edges():
    assert [autotune.band_of(L) for L in (1, 1299, 1300, 2199, 2200, 10 ** 6)] == [0, 0, 1, 1, 2, 2]
    t = {"rows_per_warp": [1, 2, 4]}
    assert [autotune.rows_per_warp(t, L) for L in (900, 1500, 3000)] == [1, 2, 4]


def test_tune_picks_per_band_tiles_and_blocks(monkeypatch):
    from swifttn93_b200 import synth

    real = synth.hiv_bench
    monkeypatch.setattr(synth, "hiv_bench", lambda seed, n, L, clusters, tag: real(seed=seed, n=40, L=L,
                                                                                     clusters=1, tag=tag))
    eng = FakeEngine()
    t = autotune.tune(eng, n=40, reps=1)
    assert t["pair_blocks"] == 3
    assert t["rows_per_warp"] == [1, 2, 4]
    assert len(t["pair_ms"]) == len(autotune.BANDS) * len(autotune.BLOCKS) * len(autotune.RPW)


def test_cache_is_used_per_device(monkeypatch, tmp_path):
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    calls = []
    monkeypatch.setattr(autotune, "tune", lambda engine: calls.append(1) or {"rows_per_warp": [4, 4, 4],
                                                                             "pair_blocks": 3})
    a = autotune.load_or_tune(object(), "GPU A")
    b = autotune.load_or_tune(object(), "GPU A")
    c = autotune.load_or_tune(object(), "GPU B")
    assert a == b == c and len(calls) == 2
    cached = json.loads(autotune.cache_path().read_text())
    assert set(cached) == {"GPU A", "GPU B"}
    autotune.load_or_tune(object(), "GPU A", retune=True)
    assert len(calls) == 3
