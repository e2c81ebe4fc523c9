"""Parity of the B200 engine with the reference path, byte for byte (distance file, stdout JSON, exit status).

Oracles: the C restatement oracle/tn93_oracle.c (pinned to the reference's golden hashes by
tests/test_oracle.py), the committed reference outputs tests/golden/ref_outputs.json, and tn93 v1.1.0's own
golden hashes on the 8,766-sequence HIV-1 pol set. Every case runs the product's command line, which reaches
the GPU through the C ABI of include/tn93g.h."""
import json
import random
import tempfile
from pathlib import Path

import numpy as np
import pytest

from tests import cases
from tests.conftest import REPO, run_tn93, sha256

pytestmark = pytest.mark.gpu
GOLDEN = REPO / "tests" / "golden"


def _write(files, td):
    out = {}
    for k, data in files.items():
        p = td / f"{k}.fa"
        p.write_bytes(data)
        out[k] = p
    return out


def _compare(engine_cli, oracle_bin, flags, inp, td):
    ro, fo, so, _ = run_tn93(oracle_bin, flags, inp, td)
    rg, fg, sg, eg = run_tn93(engine_cli, flags, inp, td)
    if ro != 0:
        return rg != 0, (ro, rg, eg[-300:])
    return rg == 0 and fg == fo and sg == so, (ro, rg, eg[-300:])


def test_fuzz_corpus_vs_oracle(engine_cli, oracle_bin):
    rng = random.Random(7)
    bad = []
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for k in range(300):
            files, flags = cases.fuzz_case(rng)
            paths = _write(files, td)
            fl = [str(paths["in2"]) if f == "{in2}" else f for f in flags]
            ok, info = _compare(engine_cli, oracle_bin, fl, paths["in"], td)
            if not ok:
                bad.append((k, flags, info))
    assert not bad, bad[:4]


def _random_alignment(rng, n, L, p_amb, p_gap):
    codes = rng.integers(0, 4, size=(n, L)).astype(np.uint8)
    m = rng.random((n, L))
    codes[m < p_amb] = rng.integers(4, 17, size=int((m < p_amb).sum())).astype(np.uint8)
    codes[(m >= p_amb) & (m < p_amb + p_gap)] = 17
    base = codes[0].copy()
    for i in range(1, n):  # near-duplicates of the first sequence, so thresholds bite
        if rng.random() < 0.5:
            row = base.copy()
            k = rng.integers(0, max(1, L // 20) + 1)
            row[rng.integers(0, L, k)] = rng.integers(0, 18, k)
            codes[i] = row
    return codes


@pytest.mark.parametrize("n,L", [(1, 70), (2, 1), (31, 63), (32, 64), (33, 65), (63, 129), (64, 200), (65, 127),
                                 (97, 300)])
@pytest.mark.parametrize("mode", ["resolve", "average", "gapmm", "skip", "RYN"])
def test_tile_edges_vs_oracle(engine_cli, oracle_bin, n, L, mode):
    """Row/column tile edges (N mod 8, 32) and plane-word edges (L mod 64), every ambiguity mode."""
    from swifttn93_b200 import synth

    rng = np.random.default_rng(n * 1000 + L)
    codes = _random_alignment(rng, n, L, 0.05, 0.05)
    names = [f"s{i}" for i in range(n)]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = td / "a.fa"
        inp.write_bytes(synth.to_fasta(names, codes))
        for flags in (["-t", "1", "-l", "1", "-a", mode, "-g", "0.05"], ["-t", "0.2", "-l", "3", "-a", mode, "-0",
                                                                         "-f", "csvn"]):
            ok, info = _compare(engine_cli, oracle_bin, flags, inp, td)
            assert ok, (flags, info)


SMALL = cases.golden_cases(include_large=False)


@pytest.mark.parametrize("case", SMALL, ids=[c["name"] for c in SMALL])
def test_committed_reference_outputs(engine_cli, case):
    want = json.loads((GOLDEN / "ref_outputs.json").read_text())[case["name"]]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        case = dict(case)
        inp = cases.materialise(case, td)
        rc, fb, so, err = run_tn93(engine_cli, case["flags"], inp, td)
        assert rc == want["rc"], err[-500:]
        assert sha256(fb or b"") == want["file_sha256"]
        assert sha256(so) == want["stdout_sha256"]


LARGE = [c for c in cases.golden_cases() if c["src"] == "synth:hiv_bench"]


@pytest.mark.parametrize("case", LARGE, ids=[c["name"] for c in LARGE])
def test_benchmark_workload_reference_outputs(engine_cli, case):
    """The 6,700 x 1,500 benchmark-shaped workload: all 22.4 M pairs written, -a resolve / average / gapmm."""
    want = json.loads((GOLDEN / "ref_outputs.json").read_text())[case["name"]]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        case = dict(case)
        inp = cases.materialise(case, td)
        rc, fb, so, err = run_tn93(engine_cli, case["flags"], inp, td)
        assert rc == 0, err[-500:]
        assert len(fb) == want["file_bytes"]
        assert sha256(fb) == want["file_sha256"]
        assert sha256(so) == want["stdout_sha256"]


def test_golden_network_hashes(engine_cli):
    """tn93 v1.1.0's published output hashes on the 8,766-sequence HIV-1 pol set at five thresholds
    (application/results/network.jsonl of the reference)."""
    g = json.loads((GOLDEN / "hiv_pol_network_hashes.json").read_text())
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = td / "hiv8766.fa"
        inp.write_bytes(cases.source_bytes("real:hiv_8766")[0])
        for row in g["rows"]:
            flags = [row["t_arg"] if f == "{T}" else f for f in g["flags"] if f != "-q"]
            rc, fb, so, err = run_tn93(engine_cli, flags, inp, td)
            assert rc == 0, err[-500:]
            assert sha256(fb) == row["file_sha256"], row["t_arg"]
            assert sha256(so) == row["stdout_sha256"], row["t_arg"]


def test_api_matches_cli_and_is_deterministic():
    """The Python binding of the C ABI: same bytes as the command line's file body, twice in a row."""
    from swifttn93_b200 import Engine, Options, synth

    names, codes = synth.plain_small()
    eng = Engine()
    s = eng.upload(codes, names)
    opts = Options(threshold=0.015, mode="resolve", resolve_fraction=0.05, min_overlap=500)
    a, sa = eng.run(s, opts)
    b, sb = eng.run(s, opts)
    assert a == b and sa.links == sb.links
    want = json.loads((GOLDEN / "ref_outputs.json").read_text())["plain_small_hivtrace"]
    assert sha256(b"ID1,ID2,Distance\n" + a) == want["file_sha256"]
    ptr, nb, sd = eng.run_to_device(s, opts)
    assert nb == len(a) and ptr
    eng.free(s)
    eng.close()
