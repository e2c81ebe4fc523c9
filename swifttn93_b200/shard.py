"""One alignment split over several GPUs by row bands (one process per GPU, torch.distributed).

Pairs are independent, so the pair triangle is cut into contiguous row bands balanced by pair count, one per
rank; every rank holds the whole packed alignment (MBs) and runs its band (tn93g_run_rows). The only exchange
is an ordered gather to rank 0 of each band's text, per-row sums, counts, maxima and histograms, where the
bands are merged in row order: texts concatenate, and the per-row sums are added in row order from 0, which is
the order tn93 adds them in (swifttn93.cpp:2838-2848), so the merged file and summary equal a one-GPU run byte
for byte. No collective runs on the data path.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import Summary, _Summary


def plan_rows(N: int, n1: int, cross: bool, world: int) -> list:
    """Contiguous row bands [(r0, r1)] for `world` ranks. Under -s every row has the same n2 pairs, so the rows
    are split evenly; otherwise row i has N - i - 1 pairs and the cuts balance the cumulative pair count."""
    rows = n1 if cross else N
    if cross:
        cuts = [rows * k // world for k in range(world + 1)]
    else:
        per_row = np.arange(N - 1, N - 1 - rows, -1, dtype=np.int64)
        cum = np.concatenate([[0], np.cumsum(per_row)])
        total = int(cum[-1])
        cuts = [0] + [int(np.searchsorted(cum, total * k // world, side="left")) for k in range(1, world)] + [rows]
        for k in range(1, world + 1):
            cuts[k] = max(cuts[k], cuts[k - 1])
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


@dataclass
class Partial:
    """One band's results, as tn93g_run_rows returns them."""
    r0: int
    r1: int
    text: bytes
    pairwise: int
    skipped: int
    links: int
    max: list
    hist: np.ndarray      # uint64 [3, 200]
    row_sums: np.ndarray  # float64 [r1 - r0, 6]
    replayed: int = 0
    ambiguous: int = 0
    undecided: int = 0


def partial_from_run(r0, r1, text, summ: Summary, row_sums) -> Partial:
    return Partial(r0, r1, text, summ.pairwise, summ.skipped, summ.links, list(summ.max),
                   np.asarray(summ.hist, dtype=np.uint64), np.asarray(row_sums, dtype=np.float64),
                   summ.pairs_replayed, summ.logs_ambiguous, summ.undecided)


def merge(parts: list) -> tuple:
    """(text, Summary) of the whole run from its bands, in row order."""
    parts = sorted(parts, key=lambda p: p.r0)
    for a, b in zip(parts, parts[1:]):
        if a.r1 != b.r0:
            raise ValueError(f"bands [{a.r0}, {a.r1}) and [{b.r0}, {b.r1}) are not contiguous")
    mean, wc = [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]
    for p in parts:
        for row in p.row_sums.tolist():  # Python floats: one IEEE double addition at a time, in row order
            for q in range(3):
                mean[q] += row[q]
                wc[q] += row[3 + q]
    S = _Summary()
    S.pairwise = sum(p.pairwise for p in parts)
    S.skipped = sum(p.skipped for p in parts)
    S.links = sum(p.links for p in parts)
    hist = np.zeros((3, 200), dtype=np.uint64)
    for p in parts:
        hist += p.hist
    for q in range(3):
        S.max[q] = max([0.0] + [p.max[q] for p in parts])
        S.mean[q] = mean[q]
        S.weighted[q] = wc[q]
        for k in range(200):
            S.hist[q][k] = int(hist[q, k])
    S.pairs_replayed = sum(p.replayed for p in parts)
    S.logs_ambiguous = sum(p.ambiguous for p in parts)
    S.undecided = sum(p.undecided for p in parts)
    text = b"".join(p.text for p in parts)
    S.output_bytes = len(text)
    from . import _plain_summary

    return text, _plain_summary(S)


def run_sharded(compute, N: int, n1: int, cross: bool, group=None):
    """Runs this rank's band with compute(r0, r1) -> Partial and gathers the bands to rank 0, which returns the
    merged (text, Summary); other ranks return None. Every rank takes the same collective step."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    r0, r1 = plan_rows(N, n1, cross, world)[rank]
    part = compute(r0, r1)
    out = [None] * world if rank == 0 else None
    dist.gather_object(part, out, dst=0, group=group)
    if rank != 0:
        return None
    return merge(out)


def engine_compute(engine, dset, opts, n1=None):
    """compute(r0, r1) for run_sharded on this rank's GPU (tn93g_run_rows)."""
    def compute(r0, r1):
        text, summ, rows = engine.run_rows(dset, opts, r0, r1, n1=n1)
        return partial_from_run(r0, r1, text, summ, rows)

    return compute
