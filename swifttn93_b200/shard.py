"""One alignment split over several GPUs by row bands (one process per GPU, torch.distributed).

Pairs are independent, so the pair triangle is cut into contiguous row bands balanced by pair count, one per
rank; every rank holds the whole packed alignment (MBs) and runs its band (tn93g_run_rows). The only exchange
is an ordered gather to rank 0 of each band's text, per-row sums, counts, maxima and histograms, where the
bands are merged in row order: texts concatenate, and the per-row sums are added in row order from 0, which is
the order tn93 adds them in (swifttn93.cpp:2838-2848), so the merged file and summary equal a one-GPU run byte
for byte. No collective runs on the data path.
"""
from __future__ import annotations

import ctypes as C
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
    resolved: int = 0
    # per bin, over the band's pairs with an ambiguous logarithm: largest low and high candidate, spread, count
    amb_bounds: np.ndarray = None


def partial_from_run(r0, r1, text, summ: Summary, row_sums) -> Partial:
    bounds = np.zeros((3, 4))
    if summ.raw is not None and hasattr(summ.raw, "amb_bounds"):
        bounds = np.array([[summ.raw.amb_bounds[u][q] for q in range(4)] for u in range(3)])
    return Partial(r0, r1, text, summ.pairwise, summ.skipped, summ.links, list(summ.max),
                   np.asarray(summ.hist, dtype=np.uint64), np.asarray(row_sums, dtype=np.float64),
                   summ.pairs_replayed, summ.logs_ambiguous, summ.undecided, summ.logs_resolved, bounds)


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
    S.logs_resolved = sum(p.resolved for p in parts)
    # the bands' bounds combine: largest candidates by maximum, spreads and counts by sum
    for u in range(3):
        b = [p.amb_bounds[u] for p in parts if p.amb_bounds is not None]
        if b:
            S.amb_bounds[u][0] = max(x[0] for x in b)
            S.amb_bounds[u][1] = max(x[1] for x in b)
            S.amb_bounds[u][2] = sum(x[2] for x in b)
            S.amb_bounds[u][3] = sum(x[3] for x in b)
    text = b"".join(p.text for p in parts)
    S.output_bytes = len(text)
    from . import _plain_summary

    return text, _plain_summary(S)


def certified(S, N: int, n1: int, cross: bool, fst: bool = False) -> bool:
    """Whether every number the merged JSON summary prints is certain for every rounding of the C library's log
    (tn93g_summary_certified over the combined bounds). Without the library, only a run with no ambiguous
    logarithm is certain."""
    if all(S.raw.amb_bounds[u][3] == 0 for u in range(3)):
        return True
    from . import load_library

    rows = n1 if cross else N
    chain = (N - n1 if cross else N) + rows + 2
    return bool(load_library().tn93g_summary_certified(C.byref(S.raw), chain, int(fst)))


def run_sharded(compute, N: int, n1: int, cross: bool, group=None, exact_compute=None, fst: bool = False):
    """Runs this rank's band with compute(r0, r1) -> Partial and gathers the bands to rank 0, which returns the
    merged (text, Summary); other ranks return None. When the merged JSON numbers are not certain and
    exact_compute is given, every rank runs its band again with exact sums (exact_compute(r0, r1) -> Partial) and
    rank 0 takes the maximum and means from those. Every rank takes the same collective steps."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    r0, r1 = plan_rows(N, n1, cross, world)[rank]
    part = compute(r0, r1)
    out = [None] * world if rank == 0 else None
    dist.gather_object(part, out, dst=0, group=group)
    merged, again = None, [False]
    if rank == 0:
        merged = merge(out)
        again[0] = exact_compute is not None and not certified(merged[1], N, n1, cross, fst)
    dist.broadcast_object_list(again, src=0, group=group)
    if again[0]:
        part2 = exact_compute(r0, r1)
        out2 = [None] * world if rank == 0 else None
        dist.gather_object(part2, out2, dst=0, group=group)
        if rank == 0:
            _, S2 = merge(out2)
            for q in range(3):
                merged[1].max[q] = S2.max[q]
                merged[1].mean[q] = S2.mean[q]
                merged[1].raw.max[q] = S2.max[q]
                merged[1].raw.mean[q] = S2.mean[q]
            merged[1].sums_repass = True
            merged[1].raw.sums_repass = 1
    return merged if rank == 0 else None


def engine_compute(engine, dset, opts, n1=None, exact=False):
    """compute(r0, r1) for run_sharded on this rank's GPU (tn93g_run_rows); exact=True: the exact-sums pass
    (every pair with an ambiguous logarithm finished with the C library's log, no text)."""
    def compute(r0, r1):
        o = opts
        if exact:
            from dataclasses import replace

            o = replace(opts, count_only=True)
            engine.set_exact_sums(True)
        try:
            text, summ, rows = engine.run_rows(dset, o, r0, r1, n1=n1)
        finally:
            if exact:
                engine.set_exact_sums(False)
        return partial_from_run(r0, r1, text, summ, rows)

    return compute
