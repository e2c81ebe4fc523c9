"""Alignments of 65,535 columns and more.

The reference switches paths there: for L >= 65,535 its engine hands every pair to tn93's own per-pair loop
(Engine::slow, solver/swifttn93.cpp:583-590, 1945-1949 -> refkernel.cpp:212-816) instead of its 16-bit packed
counters. The B200 engine keeps one path (32-bit x16 count lanes, up to L < 2^25), so its output at these lengths
must equal the reference binary's, built from the reference's own sources (oracle/build_ref.sh), byte for byte, in
every ambiguity mode and output format. The oracle (the C restatement) is checked beside it."""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import run_tn93

pytestmark = pytest.mark.gpu


def _long_fasta(seed: int, n: int, L: int) -> bytes:
    """n related sequences of L columns: a random root, 0.5-4% point differences per sequence, 1% two-fold IUPAC
    codes, a few three-fold codes, N runs and gap runs, ragged ends; sequences 0-3 are near-identical so that small
    thresholds report pairs."""
    rng = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ACGT", dtype=np.uint8)
    root = alpha[rng.integers(0, 4, L)]
    rows = []
    for i in range(n):
        s = root.copy()
        div = 0.0005 if i < 4 else rng.uniform(0.005, 0.04)
        m = rng.random(L) < div
        s[m] = alpha[rng.integers(0, 4, int(m.sum()))]
        amb = rng.random(L) < 0.01
        s[amb] = np.frombuffer(b"RYKMSW", dtype=np.uint8)[rng.integers(0, 6, int(amb.sum()))]
        if i % 5 == 2:
            tri = rng.random(L) < 0.0005
            s[tri] = np.frombuffer(b"BDHV", dtype=np.uint8)[rng.integers(0, 4, int(tri.sum()))]
        for _ in range(rng.integers(1, 4)):
            a = int(rng.integers(0, L - 400))
            s[a:a + int(rng.integers(50, 400))] = ord("N")
        for _ in range(rng.integers(0, 3)):
            a = int(rng.integers(0, L - 40))
            s[a:a + int(rng.integers(1, 40))] = ord("-")
        s[:int(rng.integers(0, 300))] = ord("-")
        rows.append(b">long%02d\n" % i + s.tobytes() + b"\n")
    return b"".join(rows)


FLAGS = [
    ["-t", "0.05", "-a", "resolve", "-l", "500"],
    ["-t", "0.05", "-a", "resolve", "-g", "0.0001", "-l", "500", "-f", "csvn"],
    ["-t", "0.1", "-a", "average", "-l", "100"],
    ["-t", "0.1", "-a", "skip", "-l", "100", "-0"],
    ["-t", "1", "-a", "gapmm", "-l", "100", "-f", "csvn"],
    ["-t", "0.05", "-a", "RYN", "-g", "0.01", "-l", "1000"],
    ["-t", "0.2", "-f", "hyphy"],
]


@pytest.mark.parametrize("L", [65534, 65535, 70001])
def test_long_alignment_matches_reference(engine_cli, ref_bin, oracle_bin, L):
    data = _long_fasta(L, 24, L)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = td / "long.fa"
        inp.write_bytes(data)
        bad = []
        for flags in FLAGS:
            rr, fr, sr, er = run_tn93(ref_bin, flags, inp, td)
            rg, fg, sg, eg = run_tn93(engine_cli, flags, inp, td)
            ro, fo, so, _ = run_tn93(oracle_bin, flags, inp, td)
            assert rr == 0, er[-300:]
            if not (rg == 0 and fg == fr and sg == sr):
                bad.append((flags, rg, eg[-200:], len(fg or b""), len(fr or b"")))
            assert ro == 0 and fo == fr and so == sr, ("oracle", flags)
            assert fr and fr.count(b"\n") > 1 or "-f" in flags, flags  # something was reported
    assert not bad, bad
