"""The tensor-core count path (tcgen05 INT8 one-hot products, tn93g_set_count_path(ctx, 1)) must give exactly the
bytes and summaries of the CUDA-core popcount path, which the other parity tests pin to the oracle and the
reference: tile and word edges in every ambiguity mode, the two-file modes, row bands starting off the 32-row
grid, and a real alignment with non-dyadic pairs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _both(eng, s, opts, n1=None, rows=None):
    out = []
    for path in ("popc", "tc"):
        eng.set_count_path(path)
        if rows is None:
            body, summ = eng.run(s, opts, n1=n1)
            out.append((body, summ.json(s.N if n1 is None else n1, 0 if n1 is None else s.N - n1, n1 is not None,
                                        opts.do_fst), summ.links))
        else:
            body, summ, rs = eng.run_rows(s, opts, rows[0], rows[1], n1=n1)
            out.append((body, rs.tobytes(), summ.links, summ.max))
    eng.set_count_path("popc")
    return out


def test_tc_equals_popc_edges():
    from swifttn93_b200 import Engine, Options, synth

    names0, codes0 = synth.plain_small()
    rng = np.random.default_rng(3)
    eng = Engine()
    for n, L in ((1, 70), (2, 1), (31, 63), (32, 64), (33, 65), (65, 129), (100, 300), (97, 1300)):
        rows = rng.choice(len(names0), n, replace=False)
        cols = np.sort(rng.choice(codes0.shape[1], L, replace=False))
        s = eng.upload(codes0[rows][:, cols], [names0[r] for r in rows], 1 + np.arange(n) % 2)
        for kw in (dict(threshold=1.0, mode="resolve", min_overlap=1),
                   dict(threshold=0.1, mode="average", min_overlap=10, format="csvn"),
                   dict(threshold=0.1, mode="gapmm", min_overlap=5, report_self=True),
                   dict(threshold=0.2, mode="skip", min_overlap=1),
                   dict(threshold=0.05, mode="RY", resolve_fraction=0.05, min_overlap=20)):
            a, b = _both(eng, s, Options(**kw))
            assert a == b, (n, L, kw)
        eng.free(s)
    eng.close()


def test_tc_equals_popc_two_files_bands_and_real_data():
    from swifttn93_b200 import Engine, Options, synth
    from tests import cases

    names, codes = synth.plain_small()
    eng = Engine()
    s = eng.upload(codes, names)
    o = Options(threshold=0.03, mode="resolve", resolve_fraction=0.05, min_overlap=500)
    for n1 in (300, 77):
        a, b = _both(eng, s, o, n1=n1)
        assert a == b, n1
    a, b = _both(eng, s, Options(threshold=0.03, mode="average", do_fst=True), n1=300)
    assert a == b
    for r0, r1 in ((0, 500), (5, 37), (33, 250), (499, 500)):
        a, b = _both(eng, s, o, rows=(r0, r1))
        assert a == b, (r0, r1)
    eng.free(s)
    fa = cases.source_bytes("real:hiv_dev")[0].split(b">")[1:601]
    nm = [r.split(b"\n", 1)[0].decode() for r in fa]
    seqs = [r.split(b"\n", 1)[1].replace(b"\n", b"") for r in fa]
    lut = np.full(256, 255, dtype=np.uint8)
    for k, ch in enumerate(synth.ALPHABET):
        lut[ch] = k
        lut[ord(chr(ch).lower())] = k
    c2 = np.stack([lut[np.frombuffer(x, dtype=np.uint8)] for x in seqs])
    s2 = eng.upload(c2, nm)
    for m in ("resolve", "average", "gapmm"):
        a, b = _both(eng, s2, Options(threshold=0.05, mode=m, resolve_fraction=0.05, min_overlap=500))
        assert a == b, m
    eng.free(s2)
    eng.close()


def test_tc_equals_popc_wide_alignment_int32_aggregates():
    """More than 32,767 variable columns: the aggregates no longer fit 16 bits and are stored as int32 (single run
    and batch)."""
    from swifttn93_b200 import Engine, HostAlignment, Options

    rng = np.random.default_rng(21)
    n, L = 40, 33000
    base = rng.integers(0, 4, L).astype(np.uint8)
    codes = np.tile(base, (n, 1))
    mut = rng.random((n, L)) < 0.02
    codes[mut] = rng.integers(0, 4, int(mut.sum())).astype(np.uint8)
    amb = rng.random((n, L)) < 0.003
    codes[amb] = rng.integers(5, 11, int(amb.sum())).astype(np.uint8)
    # every column variable, so none is folded away
    codes[0, :] = (base + 1) % 4
    names = [f"w{i}" for i in range(n)]
    eng = Engine()
    s = eng.upload(codes, names)
    o = Options(threshold=0.05, mode="resolve", resolve_fraction=0.05, min_overlap=500)
    a, b = _both(eng, s, o)
    assert a == b
    eng.free(s)
    aln = HostAlignment(codes, names)
    got = {}
    for path in ("tc", "popc"):
        eng.set_count_path(path)
        got[path] = [(body, summ.json(n)) for body, summ in eng.batch_run([aln], [o])]
    assert got["tc"] == got["popc"]
    eng.close()


@pytest.mark.parametrize("mode", ["resolve", "gapmm", "average"])
def test_split_pair_stage_matches_oracle(engine_cli, oracle_bin, tmp_path, mode):
    """The split pair stage (event kernel, then the formula kernel over the pairs' records; TN93G_PAIR_SPLIT=1)
    prints the oracle's bytes, including an alignment past 2,047 columns, whose records are 32 bytes."""
    from swifttn93_b200 import synth
    from tests.conftest import run_tn93

    for n, L in ((300, 1300), (160, 2500)):
        names, codes = synth.plain_small(seed=3, n=n, L=L)
        inp = tmp_path / f"s{n}.fa"
        inp.write_bytes(synth.to_fasta(names, codes))
        flags = ["-t", "0.5", "-a", mode, "-g", "0.05", "-l", "100"]
        rg, fg, sg, eg = run_tn93(engine_cli, flags, inp, tmp_path, extra_env={"TN93G_PAIR_SPLIT": "1"})
        ro, fo, so, _ = run_tn93(oracle_bin, flags, inp, tmp_path)
        assert ro == 0 and rg == 0, eg[-300:]
        assert fg == fo and sg == so, (mode, n, L)


@pytest.mark.parametrize("mode", ["resolve", "gapmm"])
def test_many_row_chunks_match_oracle(engine_cli, oracle_bin, tmp_path, mode):
    """Bands split into many count/pair chunks (TN93G_TC_CHUNK_PAIRS=40,000; the default chunk holds 16 M pairs,
    more than most bands): chunk edges on the 32-row grid, records reused chunk after chunk."""
    from swifttn93_b200 import synth
    from tests.conftest import run_tn93

    names, codes = synth.plain_small(seed=4, n=900, L=1100)
    inp = tmp_path / "c.fa"
    inp.write_bytes(synth.to_fasta(names, codes))
    flags = ["-t", "0.3", "-a", mode, "-g", "0.05", "-l", "100"]
    rg, fg, sg, eg = run_tn93(engine_cli, flags, inp, tmp_path, extra_env={"TN93G_TC_CHUNK_PAIRS": "40000"})
    ro, fo, so, _ = run_tn93(oracle_bin, flags, inp, tmp_path)
    assert ro == 0 and rg == 0, eg[-300:]
    assert fg == fo and sg == so
