"""Row-band sharding of one alignment over several ranks (swifttn93_b200.shard).

CPU tests: the band plan, and a world_size-2 gloo run in which each rank computes its band with the oracle
(TN93_ORACLE_ROWS, the oracle's row-band hook), the bands are gathered to rank 0 and merged, and the merged file
and JSON summary must equal the oracle's whole run byte for byte. The GPU test runs the same merge over
tn93g_run_rows bands of the engine on one GPU, against tn93g_run."""
import os
import socket
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import REPO

CASES = [
    ("average", ["-t", "0.05", "-a", "average", "-l", "500"], None),
    ("resolve_csvn_self", ["-t", "0.02", "-a", "resolve", "-g", "0.05", "-f", "csvn", "-0"], None),
    ("copies", ["-t", "0.04", "-a", "gapmm", "-d", ":"], "copies"),
    ("two_file", ["-t", "0.03", "-a", "resolve", "-l", "500", "-s", "{in2}"], "split"),
    ("fst", ["-t", "0.03", "-s", "{in2}", "-m"], "split"),
]


def test_plan_rows_covers_and_balances():
    from swifttn93_b200.shard import plan_rows

    for N in (1, 2, 3, 10, 97, 1000):
        for world in (1, 2, 3, 4, 8):
            bands = plan_rows(N, N, False, world)
            assert bands[0][0] == 0 and bands[-1][1] == N and len(bands) == world
            assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
            pairs = [sum(N - i - 1 for i in range(r0, r1)) for r0, r1 in bands]
            assert max(pairs) - min(pairs) <= 2 * N
    assert plan_rows(7, 4, True, 2) == [(0, 2), (2, 4)]


def _inputs(kind, td: Path):
    from swifttn93_b200 import synth

    names, codes = synth.plain_small()
    names, codes = names[:240], codes[:240]
    if kind == "copies":
        names = [f"{n}:{1 + i % 3}" for i, n in enumerate(names)]
    p = td / "in.fa"
    if kind == "split":
        p.write_bytes(synth.to_fasta(names[:150], codes[:150]))
        (td / "in2.fa").write_bytes(synth.to_fasta(names[150:], codes[150:]))
        return p, 150, 240
    p.write_bytes(synth.to_fasta(names, codes))
    return p, 240, 240


def _oracle_band(oracle_bin, flags, inp, td: Path, r0, r1, rank):
    from swifttn93_b200.shard import Partial

    out = td / f"band{rank}.csv"
    part = td / f"band{rank}.txt"
    env = {**os.environ, "TN93_ORACLE_ROWS": f"{r0}:{r1}", "TN93_ORACLE_PARTIAL": str(part)}
    r = subprocess.run([str(oracle_bin), "-q", "-n", *flags, "-o", str(out), str(inp)], env=env,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=300)
    assert r.returncode == 0
    rows, hist, kv = [], np.zeros((3, 200), dtype=np.uint64), {}
    for line in part.read_text().splitlines():
        f = line.split()
        if f[0] == "row":
            rows.append([float.fromhex(x) for x in f[2:8]])
        elif f[0].startswith("hist"):
            hist[int(f[0][4])] = np.array([int(x) for x in f[1:]], dtype=np.uint64)
        elif f[0] == "max":
            kv["max"] = [float.fromhex(x) for x in f[1:4]]
        else:
            kv[f[0]] = int(f[1])
    return Partial(r0, r1, out.read_bytes(), kv["pairwise"], kv["skipped"], kv["links"], kv["max"], hist,
                   np.array(rows, dtype=np.float64).reshape(-1, 6))


def _rank_main(rank, world, port, oracle_bin, flags, inp, td, N, n1, cross, result):
    import torch.distributed as dist

    from swifttn93_b200.shard import run_sharded

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        out = run_sharded(lambda r0, r1: _oracle_band(oracle_bin, flags, inp, Path(td), r0, r1, rank), N, n1, cross)
        if rank == 0:
            text, summ = out
            Path(result).write_bytes(text)
            second = "-s" in flags
            n2 = N - n1 if second else 0
            Path(result + ".json").write_bytes(summ.json(n1 if second else N, n2, second, "-m" in flags))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("tag,flags,kind", CASES, ids=[c[0] for c in CASES])
def test_gloo_two_ranks_merge_equals_whole_run(oracle_bin, tmp_path, tag, flags, kind):
    import torch.multiprocessing as mp

    from swifttn93_b200 import build

    build.build_lib()
    inp, n1, N = _inputs(kind, tmp_path)
    flags = [str(tmp_path / "in2.fa") if f == "{in2}" else f for f in flags]
    cross = "-s" in flags and "-m" not in flags
    whole = tmp_path / "whole.csv"
    r = subprocess.run([str(oracle_bin), "-q", *flags, "-o", str(whole), str(inp)], capture_output=True, timeout=300)
    assert r.returncode == 0
    result = str(tmp_path / "merged.csv")
    mp.start_processes(_rank_main, args=(2, _free_port(), str(oracle_bin), flags, str(inp), str(tmp_path), N, n1,
                                         cross, result), nprocs=2, start_method="spawn")
    fmt_csvn = "csvn" in flags
    header = b"Seq1,Seq2,Distance\n" if fmt_csvn else b"ID1,ID2,Distance\n"
    assert header + Path(result).read_bytes() == whole.read_bytes(), tag
    assert Path(result + ".json").read_bytes() == r.stdout, tag


@pytest.mark.gpu
def test_engine_bands_merge_equals_run():
    """tn93g_run_rows over 3 uneven bands on one GPU, merged in row order, equals tn93g_run."""
    from swifttn93_b200 import Engine, Options, synth
    from swifttn93_b200.shard import merge, partial_from_run, plan_rows

    names, codes = synth.plain_small()
    eng = Engine()
    s = eng.upload(codes, names, counts=1 + np.arange(len(names)) % 3)
    for kw, n1 in ((dict(threshold=0.05, mode="average", min_overlap=500), None),
                   (dict(threshold=0.02, mode="resolve", resolve_fraction=0.05, format="csvn", report_self=True), None),
                   (dict(threshold=0.03, mode="resolve", min_overlap=500), 300),
                   (dict(threshold=0.03, mode="gapmm", do_fst=True), 300)):
        o = Options(**kw)
        text, whole = eng.run(s, o, n1=n1)
        cross = n1 is not None and not o.do_fst
        for world in (2, 3):
            parts = []
            for r0, r1 in plan_rows(len(names), n1 or len(names), cross, world):
                t, sm, rows = eng.run_rows(s, o, r0, r1, n1=n1)
                parts.append(partial_from_run(r0, r1, t, sm, rows))
            mt, ms = merge(parts)
            assert mt == text, (kw, world)
            second = n1 is not None
            N = len(names)
            args = ((n1, N - n1, True, o.do_fst) if second else (N, 0, False, False))
            assert ms.json(*args) == whole.json(*args), (kw, world)
    eng.close()
