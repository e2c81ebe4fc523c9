"""Batches of independent alignments (tn93g_batch_run): every alignment's distance file and summary must equal a
run of that alignment alone (tn93g_run, itself parity-tested against the oracle and the reference), whatever the
batch around it and whatever pair-tile height and blocks per SM are chosen. The small alignments are also checked
against the oracle directly."""
import numpy as np
import pytest

from tests.conftest import run_tn93

pytestmark = pytest.mark.gpu

MODE_FLAGS = {"resolve": "resolve", "average": "average", "gapmm": "gapmm", "skip": "skip", "RY": "RY"}


def _mixed_batch():
    """Edge shapes and option mixes: n = 1, 2, 31..65 around tile edges, L around word edges, an all-constant
    alignment, copy numbers, csvn, -0, -c, -g fallback, subsets."""
    from swifttn93_b200 import HostAlignment, Options, synth

    rng = np.random.default_rng(11)
    names0, codes0 = synth.plain_small()
    out = []
    specs = [
        (1, 70, dict(threshold=1.0, mode="resolve")),
        (2, 1, dict(threshold=1.0, mode="average", min_overlap=1)),
        (31, 63, dict(threshold=0.05, mode="gapmm", min_overlap=10)),
        (33, 64, dict(threshold=0.2, mode="resolve", resolve_fraction=0.05, format="csvn", min_overlap=10)),
        (64, 65, dict(threshold=0.1, mode="RY", min_overlap=20, report_self=True)),
        (65, 129, dict(threshold=0.1, mode="skip", min_overlap=50)),
        (97, 700, dict(threshold=0.03, mode="resolve", min_overlap=500, count_only=True)),
        (300, 1300, dict(threshold=0.02, mode="average", min_overlap=500, delimiter=";")),
        (500, 1300, dict(threshold=0.015, mode="resolve", resolve_fraction=0.05, min_overlap=500)),
        (40, 200, dict(threshold=0.05, mode="gapmm", min_overlap=50, report_self=True, format="csvn")),
    ]
    for k, (n, L, kw) in enumerate(specs):
        rows = rng.choice(len(names0), n, replace=False)
        cols = np.sort(rng.choice(codes0.shape[1], L, replace=False))
        codes = codes0[rows][:, cols]
        counts = 1 + (np.arange(n) % 3) if k in (3, 7) else None
        names = [f"b{k}_{names0[r]}" + (f":{counts[i]}" if counts is not None else "") for i, r in enumerate(rows)]
        out.append((HostAlignment(codes, names, counts), Options(**kw)))
    const = np.tile(codes0[0:1, :80], (12, 1))
    const[:, :80] = np.where(const[:, :80] < 4, const[:, :80], 0)
    out.append((HostAlignment(const, [f"c{i}" for i in range(12)]), Options(threshold=1.0, mode="resolve",
                                                                            min_overlap=1)))
    return out


def _alone(eng, aln, opts):
    s = eng.upload(aln._codes, [bytes(aln._names.raw[int(o):int(o) + int(n)]) for o, n in zip(aln._off, aln._len)],
                   aln._cnt)
    body, summ = eng.run(s, opts)
    eng.free(s)
    # the same alignment uploaded as a prepared HostAlignment gives the same run
    s = eng.upload(aln)
    body2, summ2 = eng.run(s, opts)
    eng.free(s)
    assert body2 == body and summ2.json(aln.n) == summ.json(aln.n)
    return body, summ


def test_batch_equals_alone_for_every_tile_shape():
    from swifttn93_b200 import Engine

    items = _mixed_batch()
    eng = Engine()
    alone = [_alone(eng, a, o) for a, o in items]
    alns, opts = [a for a, _ in items], [o for _, o in items]
    for path, rpw, blocks in (("tc", None, 0), ("popc", None, 0), ("tc", [1] * len(items), 2),
                              ("popc", [2] * len(items), 3), ("tc", [4, 1, 2] * 4, 3)):
        eng.set_count_path(path)
        got = eng.batch_run(alns, opts, rows_per_warp=None if rpw is None else rpw[:len(items)], pair_blocks=blocks)
        for k, ((b, s), (wb, ws)) in enumerate(zip(got, alone)):
            assert b == wb, (k, path, rpw, blocks, len(b), len(wb))
            n = alns[k].n
            assert s.json(n) == ws.json(n), (k, path, rpw, blocks)
            assert s.links == ws.links and s.pairwise == ws.pairwise
    eng.close()


def test_batch_small_alignments_against_oracle(oracle_bin, tmp_path):
    from swifttn93_b200 import Engine, synth

    items = _mixed_batch()[:7]
    eng = Engine()
    got = eng.batch_run([a for a, _ in items], [o for _, o in items])
    eng.close()
    for k, ((aln, o), (body, summ)) in enumerate(zip(items, got)):
        names = [bytes(aln._names.raw[int(a):int(a) + int(n)]).decode() for a, n in zip(aln._off, aln._len)]
        p = tmp_path / f"a{k}.fa"
        p.write_bytes(synth.to_fasta(names, aln._codes))
        flags = ["-t", repr(o.threshold), "-l", str(o.min_overlap), "-a", MODE_FLAGS[o.mode], "-f", o.format,
                 "-D", o.delimiter]
        if o.resolve_fraction < 1:
            flags += ["-g", repr(o.resolve_fraction)]
        if o.report_self:
            flags.append("-0")
        if o.count_only:
            flags.append("-c")
        rc, fb, out, _ = run_tn93(oracle_bin, flags, p, tmp_path)
        assert rc == 0, k
        header = b"" if o.count_only else (b"ID1" if o.format == "csv" else b"Seq1") + \
            f"{o.delimiter}{'ID2' if o.format == 'csv' else 'Seq2'}{o.delimiter}Distance\n".encode()
        if o.count_only:
            assert fb == f"Found {summ.links} links among {summ.pairwise - summ.skipped} pairwise comparisons\n".encode()
        else:
            assert header + body == fb, k
        assert summ.json(aln.n) == out, k


def test_batch_workload_slice_equals_alone():
    """The first 10 alignments of the batched benchmark workload (sizes 50-4,000, lengths 900-3,000, per-alignment
    threshold and mode)."""
    from swifttn93_b200 import Engine, HostAlignment, Options, synth

    eng = Engine()
    alns, opts = [], []
    for i in range(10):
        sp, names, codes = synth.batch_alignment(i)
        alns.append(HostAlignment(codes, names))
        opts.append(Options(threshold=sp["threshold"], mode=sp["mode"], resolve_fraction=0.05, min_overlap=500))
    got = eng.batch_run(alns, opts)
    for k, (a, o) in enumerate(zip(alns, opts)):
        wb, ws = _alone(eng, a, o)
        assert got[k][0] == wb, k
        assert got[k][1].json(a.n) == ws.json(a.n), k
    eng.close()
