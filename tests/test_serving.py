"""The resident-reference server (tn93g_server_*) and the continuous-batching service on top of it.

Every query's response must equal, byte for byte, what `tn93 -q FLAGS -s QUERY.fa -o OUT REF.fa` produces (exit
status, distance file, JSON summary on stdout; the oracle is the checker), and must be the same whether the query
runs alone or batched with others. The batching policy itself is host logic and is tested on the CPU."""
from collections import deque
from dataclasses import dataclass

import numpy as np
import pytest

from tests.conftest import run_tn93

SERVE_FLAGS = [
    ("hivtrace_s", ["-t", "0.015", "-a", "resolve", "-l", "500"], dict(threshold=0.015, mode="resolve",
                                                                      min_overlap=500)),
    ("fallback_csvn", ["-t", "0.015", "-a", "resolve", "-g", "0.05", "-l", "500", "-f", "csvn"],
     dict(threshold=0.015, mode="resolve", resolve_fraction=0.05, min_overlap=500, format="csvn")),
    ("average_delim", ["-t", "0.03", "-a", "average", "-l", "100", "-D", ";"],
     dict(threshold=0.03, mode="average", min_overlap=100, delimiter=";")),
    ("gapmm", ["-t", "0.02", "-a", "gapmm", "-l", "200"], dict(threshold=0.02, mode="gapmm", min_overlap=200)),
]


@dataclass
class _R:
    n: int


def test_take_batch_policy():
    from swifttn93_b200.serve import take_batch

    q = deque(_R(n) for n in (5, 7, 3, 20, 1, 1))
    assert [r.n for r in take_batch(q, 10, 16)] == [5, 7, 3]
    assert [r.n for r in q] == [20, 1, 1]
    assert take_batch(q, 10, 16) == []          # the head does not fit: it waits, order is kept
    q = deque(_R(1) for _ in range(9))
    assert len(take_batch(q, 4, 100)) == 4 and len(q) == 5
    assert take_batch(deque(), 4, 100) == []


def _workload():
    from swifttn93_b200 import synth

    rng = np.random.default_rng(44)
    rnames, rcodes = synth.serve_reference(seed=9, n=1500, L=1500)
    ref = synth.to_fasta(rnames, rcodes)
    queries = []
    for k, q in enumerate((1, 2, 5, 17, 32, 64, 3, 130)):
        names, codes = synth.serve_query(rng, rcodes, q, f"t{k}")
        if k == 2:
            names = [f"{n}:{1 + i % 4}" for i, n in enumerate(names)]  # copy numbers
        fa = synth.to_fasta(names, codes, wrap=70 if k == 3 else 0)
        if k == 4:
            fa = fa.lower()
        queries.append(fa)
    return ref, queries


@pytest.mark.gpu
@pytest.mark.parametrize("tag,flags,kw", SERVE_FLAGS, ids=[t for t, _, _ in SERVE_FLAGS])
def test_served_queries_match_oracle_alone_and_batched(oracle_bin, tmp_path, tag, flags, kw):
    from swifttn93_b200 import Engine, Fasta, Options, ResidentReference
    from swifttn93_b200.serve import header_line

    ref, queries = _workload()
    refp = tmp_path / "ref.fa"
    refp.write_bytes(ref)
    opts = Options(**kw)
    eng = Engine()
    R = Fasta(ref)
    res = ResidentReference(eng, R, opts, max_batch_sequences=512, max_batch_queries=16)
    Q = [Fasta(q, expect_len=R.L) for q in queries]
    batched = res.batch(Q)
    assert len(batched) == len(Q)
    for k, (qfa, qf) in enumerate(zip(queries, Q)):
        alone = res.batch([qf])[0]
        assert alone[0] == batched[k][0], (tag, k)
        qp = tmp_path / f"q{k}.fa"
        qp.write_bytes(qfa)
        rc, fb, out, _ = run_tn93(oracle_bin, flags + ["-s", str(qp)], refp, tmp_path)
        assert rc == 0
        body, summ = batched[k]
        assert header_line(opts) + body == fb, (tag, k, len(body), len(fb))
        assert summ.json(R.n, qf.n, second_file=True) == out, (tag, k)
        assert summ.pairwise == R.n * qf.n
    res.close()
    eng.close()


@pytest.mark.gpu
def test_service_continuous_batching_same_as_alone(oracle_bin, tmp_path):
    """Requests arriving as a Poisson stream are batched by two workers; each response equals the oracle's run of
    that query file, and a refused query (wrong sequence length) gets tn93's status and message alone."""
    from swifttn93_b200 import Options
    from swifttn93_b200.serve import Service, run_load

    ref, queries = _workload()
    bad = b">x\nACGT\n"
    stream = queries * 3 + [bad]
    refp = tmp_path / "ref.fa"
    refp.write_bytes(ref)
    flags = ["-t", "0.015", "-a", "resolve", "-l", "500"]
    want = []
    for k, qfa in enumerate(queries + [bad]):
        qp = tmp_path / f"q{k}.fa"
        qp.write_bytes(qfa)
        rc, fb, out, err = run_tn93(oracle_bin, flags + ["-s", str(qp)], refp, tmp_path)
        want.append((rc, fb if rc == 0 else None, out if rc == 0 else None, err))
    with Service(ref, Options(threshold=0.015, mode="resolve", min_overlap=500), hbm_budget=4 << 30, workers=2,
                 max_batch_queries=8, max_batch_sequences=300) as svc:
        # a Poisson stream, then a burst (everything queued at once, so that batches fill up)
        runs = [run_load(svc, stream, rate=400.0, seed=3)]
        b0 = svc.stats.batches
        runs.append(run_load(svc, stream, rate=1e7, seed=4))
        burst_batches = svc.stats.batches - b0
        stats = svc.stats
    for r in runs:
        assert r["requests"] == len(stream) and r["ok"] == len(stream) - 1
        for k, resp in enumerate(r["responses"]):
            w = want[len(queries)] if k == len(stream) - 1 else want[k % len(queries)]
            assert resp.rc == w[0], k
            if w[0] == 0:
                assert resp.file == w[1] and resp.stdout == w[2], k
            else:
                assert resp.stderr == w[3], (resp.stderr, w[3])
    assert burst_batches < len(stream) - 1  # the burst's requests were batched together
    assert max(stats.batch_sequences) <= 300


@pytest.mark.gpu
def test_service_refuses_a_query_larger_than_a_batch():
    """A query with more sequences than one batch can hold within the HBM budget is refused with status 2 and a
    message, and the service goes on answering the others."""
    from swifttn93_b200 import Options
    from swifttn93_b200.serve import Service

    ref, queries = _workload()
    big = queries[-1]  # 130 sequences
    with Service(ref, Options(threshold=0.015, mode="resolve", min_overlap=500), hbm_budget=4 << 30, workers=1,
                 max_batch_queries=4, max_batch_sequences=100) as svc:
        r_big = svc.submit(big).result()
        r_small = svc.submit(queries[0]).result()
    assert r_big.rc == 2 and b"larger than a batch" in r_big.stderr and r_big.file == b""
    assert r_small.rc == 0 and r_small.file.startswith(b"ID1,ID2,Distance\n")


@pytest.mark.gpu
def test_server_tensor_core_chunks_equal_popcount():
    """A batch wider than one 1,024-column chunk of the server's tensor-core count path (and a reference whose
    size is not a multiple of 32, so one operand block mixes reference and query rows) gives the same bytes and
    summaries as the popcount path."""
    import numpy as np

    from swifttn93_b200 import Engine, Fasta, Options, ResidentReference, synth

    rng = np.random.default_rng(8)
    rnames, rcodes = synth.serve_reference(seed=12, n=1499, L=1500)
    R = Fasta(synth.to_fasta(rnames, rcodes))
    Q = []
    for k, q in enumerate((400, 1, 350, 33, 300, 64)):
        names, codes = synth.serve_query(rng, rcodes, q, f"c{k}")
        Q.append(Fasta(synth.to_fasta(names, codes), expect_len=R.L))
    opts = Options(threshold=0.015, mode="resolve", resolve_fraction=0.05, min_overlap=500, format="csvn")
    out = {}
    for path in ("tc", "popc"):
        eng = Engine()
        eng.set_count_path(path)
        res = ResidentReference(eng, R, opts, max_batch_sequences=1300, max_batch_queries=8)
        out[path] = [(b, s.json(R.n, q.n, second_file=True)) for (b, s), q in zip(res.batch(Q), Q)]
        res.close()
        eng.close()
    assert out["tc"] == out["popc"]


def test_service_without_a_device_fails_cleanly():
    """With no usable CUDA device the service's constructor raises the engine's error (no CPU fallback) and leaves
    no worker thread behind."""
    import threading

    import torch

    from swifttn93_b200 import Options, Tn93Error, build, synth
    from swifttn93_b200.serve import Service

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    build.build_lib()
    names, codes = synth.plain_small(n=40, L=300)
    before = threading.active_count()
    with pytest.raises(Tn93Error):
        Service(synth.to_fasta(names, codes), Options(threshold=0.015), workers=2)
    assert threading.active_count() == before


class _FakeSummary:
    def __init__(self, n):
        self.pairwise, self.skipped, self.links = n, 0, 0

    def json(self, n1, n2=0, second_file=False, fst=False):
        return f"{n1} {n2}\n".encode()


class _FakeEngine:
    def __init__(self, device=0, hbm_budget=0):
        self.closed = False

    def close(self):
        self.closed = True


class _FakeReference:
    batches = []

    def __init__(self, eng, ref, opts, cap_sequences, cap_queries):
        self.cap = (cap_sequences, cap_queries)

    def batch(self, fastas):
        _FakeReference.batches.append([f.n for f in fastas])
        return [(f"body{f.n}\n".encode(), _FakeSummary(f.n)) for f in fastas]

    def close(self):
        pass


def test_service_scheduling_with_a_stand_in_engine(monkeypatch):
    """The service's host logic on the CPU, with the engine replaced by a stand-in: responses carry each query's
    own body and summary, batches respect the capacity, a refused FASTA gets status 1 and tn93's message, an
    oversized query status 2, and the others are still answered."""
    from swifttn93_b200 import Options, build, synth
    from swifttn93_b200 import serve

    build.build_lib()
    monkeypatch.setattr(serve, "Engine", _FakeEngine)
    monkeypatch.setattr(serve, "ResidentReference", _FakeReference)
    _FakeReference.batches = []
    rng = __import__("numpy").random.default_rng(3)
    rnames, rcodes = synth.serve_reference(seed=5, n=60, L=200)
    ref = synth.to_fasta(rnames, rcodes)
    qs = []
    for k, q in enumerate((3, 1, 7, 2, 9, 4)):
        names, codes = synth.serve_query(rng, rcodes, q, f"s{k}")
        qs.append(synth.to_fasta(names, codes))
    with serve.Service(ref, Options(threshold=0.015), workers=2, max_batch_queries=3,
                       max_batch_sequences=8) as svc:
        futs = [svc.submit(q) for q in qs] + [svc.submit(b">x\nACGT\n")]
        res = [f.result(timeout=60) for f in futs]
    sizes = (3, 1, 7, 2, 9, 4)
    for r, n in zip(res[:6], sizes):
        if n > 8:
            assert r.rc == 2 and b"larger than a batch" in r.stderr
        else:
            assert r.rc == 0 and r.file == b"ID1,ID2,Distance\n" + f"body{n}\n".encode()
            assert r.stdout == f"60 {n}\n".encode() and r.pairs == 60 * n
    assert res[-1].rc == 1 and b"same length" in res[-1].stderr
    done = sorted(n for b in _FakeReference.batches for n in b)
    assert done == [1, 2, 3, 4, 7]
    assert all(len(b) <= 3 and sum(b) <= 8 for b in _FakeReference.batches)


@pytest.mark.gpu
def test_full_size_reference_queries_match_oracle(oracle_bin, tmp_path):
    """The served workload at full size: the 30,000 x 1,500 resident reference, a batch of four queries of 1-200
    sequences at the serving flags; each response equals the oracle's `-s QUERY REF` run byte for byte."""
    from swifttn93_b200 import Engine, Fasta, Options, ResidentReference, synth
    from swifttn93_b200.serve import header_line

    rnames, rcodes = synth.serve_reference()
    ref = synth.to_fasta(rnames, rcodes)
    refp = tmp_path / "ref.fa"
    refp.write_bytes(ref)
    rng = np.random.default_rng(30000)
    queries = []
    for k, q in enumerate((1, 32, 200, 7)):
        names, codes = synth.serve_query(rng, rcodes, q, f"f{k}")
        queries.append(synth.to_fasta(names, codes))
    opts = Options(threshold=0.015, mode="resolve", min_overlap=500)
    eng = Engine()
    R = Fasta(ref)
    res = ResidentReference(eng, R, opts, max_batch_sequences=512, max_batch_queries=8)
    out = res.batch([Fasta(q, expect_len=R.L) for q in queries])
    flags = ["-t", "0.015", "-a", "resolve", "-l", "500"]
    for k, qfa in enumerate(queries):
        qp = tmp_path / f"q{k}.fa"
        qp.write_bytes(qfa)
        rc, fb, so, _ = run_tn93(oracle_bin, flags + ["-s", str(qp)], refp, tmp_path)
        assert rc == 0
        body, summ = out[k]
        assert header_line(opts) + body == fb, (k, len(body), len(fb))
        assert summ.json(R.n, Fasta(qfa).n, second_file=True) == so, k
    res.close()
    eng.close()
