"""The -s mode as a service: a reference alignment resident on the GPU, query FASTAs batched as they arrive.

Each request is one query FASTA; its response is what `tn93 -q FLAGS -s QUERY.fa -o OUT REF.fa` produces with the
service's options: exit status, the distance file (header and lines; rows are the reference's sequences, columns
the query's, swifttn93.cpp:2321-2322, 2392) and the JSON summary on stdout (swifttn93.cpp:2914-2958). A query that
tn93's reader refuses gets status 1 and the reader's message on stderr; nothing else is affected.

Scheduling is continuous batching: `workers` threads each own an engine context (its own CUDA stream and a copy
of the packed reference, a few hundred MB) and loop: take every pending request that fits the context's batch
capacity, run them as one batch (tn93g_server_batch: one cross run of the reference against the batch's
concatenated queries, with statistics and text segmented by query), hand each request its response. A worker
that is busy on the GPU does not hold up the others, so requests that arrive meanwhile are admitted by the next
free worker and their kernels overlap the running batch on the device.

HBM admission: the service's budget is split evenly over the workers and enforced by the engine (each context is
created with its share as its HBM budget). A context's batch capacity (sequences and queries per batch) is sized
so that the resident reference, the per-batch buffers at capacity and a text reserve fit its share; a request
larger than one batch's capacity is refused with status 2 and a message, never run over budget.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import Engine, Fasta, FastaError, Options, ResidentReference

PAIR_BYTES = 16        # distance + replay-queue slot per reference x query-sequence pair
SEGMENT_BYTES = 104    # per (reference sequence, query) statistics
TEXT_RESERVE = 512 << 20


@dataclass
class Response:
    rc: int
    file: bytes = b""
    stdout: bytes = b""
    stderr: bytes = b""
    n: int = 0
    pairs: int = 0
    t_arrive: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrive


@dataclass
class _Request:
    fasta: Fasta | None
    t_arrive: float
    fut: Future
    n: int = 0


@dataclass
class Stats:
    done: int = 0
    refused: int = 0
    pairs: int = 0
    batches: int = 0
    batch_sequences: list = field(default_factory=list)


def header_line(opts: Options) -> bytes:
    """The distance file's header (swifttn93.cpp:2307-2316)."""
    d = opts.delimiter
    return (f"ID1{d}ID2{d}Distance\n" if opts.format == "csv" else f"Seq1{d}Seq2{d}Distance\n").encode()


class Service:
    def __init__(self, ref_fasta: bytes, opts: Options, hbm_budget: int = 8 << 30, workers: int = 2,
                 max_batch_queries: int = 256, max_batch_sequences: int | None = None, no_header: bool = False,
                 counts_sep: str = ":", device: int = 0):
        if opts.format not in ("csv", "csvn") or opts.do_fst or opts.report_self:
            raise ValueError("the service runs tn93 -s with -f csv or csvn (no -m, no -0)")
        self.opts, self.no_header, self.counts_sep = opts, no_header, counts_sep
        self.ref = Fasta(ref_fasta, counts_sep=counts_sep)
        N, L = self.ref.n, self.ref.L
        share = hbm_budget // workers
        W = (L + 63) // 64
        # the reference's codes (3 copies), planes and worst-case events; per query sequence of capacity: its pairs'
        # distance and replay slots, codes (3 copies), planes and events
        resident = N * L * 3 + W * 5 * (N + 64) * 8 + N * L * 4 + len(ref_fasta)
        # tensor-core counts: the one-hot image (4 bytes per sequence and column) and the 16-byte records of one
        # 128-column chunk of query columns
        resident += 4 * L * N + 16 * N * 128
        fixed = max_batch_queries * N * SEGMENT_BYTES
        cap = (share - resident - fixed - TEXT_RESERVE) // (N * PAIR_BYTES + L * 11 + W * 5 * 8)
        if max_batch_sequences is not None:
            cap = min(cap, max_batch_sequences)
        if cap < 1:
            raise ValueError(f"an HBM budget of {hbm_budget} bytes cannot hold the reference and one batch")
        self.cap_sequences, self.cap_queries = int(min(cap, 8192)), max_batch_queries
        self.header = b"" if (no_header or opts.count_only) else header_line(opts)
        self.stats = Stats()
        self._q: deque[_Request] = deque()
        self._cv = threading.Condition()
        self._stop = False
        self._err: BaseException | None = None
        self._ready = threading.Barrier(workers + 1)
        self._threads = [threading.Thread(target=self._worker, args=(device, share), daemon=True)
                         for _ in range(workers)]
        for t in self._threads:
            t.start()
        self._ready.wait()
        if self._err:
            self.close()  # the workers that did start exit once they see the stop flag
            raise self._err

    # ------------------------------------------------------------------ requests
    def submit(self, query_fasta: bytes) -> Future:
        """Queues one query FASTA; the future resolves to its Response."""
        fut: Future = Future()
        t = time.perf_counter()
        try:
            f = Fasta(query_fasta, expect_len=self.ref.L, counts_sep=self.counts_sep)
        except FastaError as e:
            fut.set_result(Response(rc=1, stderr=str(e).encode(), t_arrive=t, t_start=t, t_done=time.perf_counter()))
            with self._cv:
                self.stats.refused += 1
            return fut
        if f.n > self.cap_sequences:
            fut.set_result(Response(rc=2, stderr=(f"query of {f.n} sequences is larger than a batch can hold within "
                                                  f"the HBM budget ({self.cap_sequences})\n").encode(),
                                    n=f.n, t_arrive=t, t_start=t, t_done=time.perf_counter()))
            with self._cv:
                self.stats.refused += 1
            return fut
        with self._cv:
            self._q.append(_Request(f, t, fut, f.n))
            self._cv.notify()
        return fut

    def _admit(self) -> list:
        """Every pending request that fits one batch, in arrival order (blocks until one is pending)."""
        with self._cv:
            while not self._q and not self._stop:
                self._cv.wait()
            return take_batch(self._q, self.cap_queries, self.cap_sequences)

    # ------------------------------------------------------------------ workers
    def _worker(self, device, share):
        eng = None
        try:
            eng = Engine(device, hbm_budget=share)
            res = ResidentReference(eng, self.ref, self.opts, self.cap_sequences, self.cap_queries)
        except BaseException as e:  # noqa: BLE001 - reported by the constructor
            if eng is not None:
                eng.close()
            self._err = e
            self._ready.wait()
            return
        self._ready.wait()
        N = self.ref.n
        try:
            while True:
                batch = self._admit()
                if not batch:
                    break
                t0 = time.perf_counter()
                try:
                    results = res.batch([r.fasta for r in batch])
                except BaseException as e:  # noqa: BLE001 - every request of the batch gets the error
                    for r in batch:
                        r.fut.set_exception(e)
                    continue
                for r, (body, summ) in zip(batch, results):
                    if self.opts.count_only:
                        pairs = summ.pairwise - summ.skipped
                        file = f"Found {summ.links} links among {pairs} pairwise comparisons\n".encode()
                    else:
                        file = self.header + body
                    js = summ.json(N, r.n, second_file=True)
                    r.fut.set_result(Response(rc=0, file=file, stdout=js, n=r.n, pairs=N * r.n, t_arrive=r.t_arrive,
                                              t_start=t0, t_done=time.perf_counter()))
                with self._cv:
                    self.stats.done += len(batch)
                    self.stats.pairs += N * sum(r.n for r in batch)
                    self.stats.batches += 1
                    self.stats.batch_sequences.append(sum(r.n for r in batch))
        finally:
            res.close()
            eng.close()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def take_batch(q: deque, cap_queries: int, cap_sequences: int) -> list:
    """Pops the longest prefix of the queue that fits one batch (at most cap_queries requests and cap_sequences
    sequences); requests keep their arrival order, and a request that does not fit waits for the next batch."""
    out, seqs = [], 0
    while q and len(out) < cap_queries and seqs + q[0].n <= cap_sequences:
        r = q.popleft()
        out.append(r)
        seqs += r.n
    return out


# ---------------------------------------------------------------------------------------------- load generator
def query_stream(ref_codes: np.ndarray, n_requests: int, seed: int = 0, mean_size: float = 32., max_size: int = 512):
    """Query FASTAs of the served workload: sizes geometric with the given mean, truncated to [1, max_size]; every
    sequence derived from a random reference sequence at 0.5-3% divergence with 1% ambiguity codes."""
    from . import synth

    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_requests):
        q = int(min(max_size, rng.geometric(1. / mean_size)))
        names, codes = synth.serve_query(rng, ref_codes, q, f"{seed}_{k}")
        out.append(synth.to_fasta(names, codes))
    return out


def run_load(svc: Service, queries: list, rate: float, seed: int = 0) -> dict:
    """Submits the queries as a Poisson stream of `rate` requests/s and waits for every response. Returns latency
    percentiles (ms), pairs/s over the run (first arrival to last response) and the responses."""
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1. / rate, len(queries))
    futs = []
    t0 = time.perf_counter()
    due = t0
    for q, g in zip(queries, gaps):
        due += g
        d = due - time.perf_counter()
        if d > 0:
            time.sleep(d)
        futs.append(svc.submit(q))
    res = [f.result() for f in futs]
    ok = [r for r in res if r.rc == 0]
    lat = np.array([r.latency for r in ok]) * 1e3
    span = max(r.t_done for r in res) - t0
    pairs = sum(r.pairs for r in ok)
    return dict(requests=len(res), ok=len(ok), rate=rate, span_s=span, pairs=pairs, pairs_per_s=pairs / span,
                p50_ms=float(np.percentile(lat, 50)) if len(lat) else None,
                p99_ms=float(np.percentile(lat, 99)) if len(lat) else None, responses=res)
