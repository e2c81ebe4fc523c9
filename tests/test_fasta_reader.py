"""The library's FASTA reader (tn93g_read_fasta, used by the command line and the resident-reference server)
against the oracle's restatement of tn93's reader (swifttn93.cpp:259-406): on the fuzz inputs of the parity
gate, both accept or refuse the same files with the same message, and produce the same names, copy numbers and
codes. Runs on the CPU (the reader is host code)."""
import os
import random
import subprocess

import pytest

from tests import cases
from tests.conftest import REPO

ALPHA = "ACGTURYSWKMBDHVN?-"


def _lib_read(files, sep):
    from swifttn93_b200 import Fasta, FastaError

    recs = []
    L = 0
    for key in ("in", "in2"):
        if key not in files:
            continue
        try:
            f = Fasta(files[key], expect_len=L, counts_sep=sep)
        except FastaError as e:
            return 1, str(e).encode(), None
        L = f.L
        codes = f.codes
        for k, (nm, c) in enumerate(zip(f.names, f.counts)):
            recs.append(nm + b"\t" + str(int(c)).encode() + b"\t" + "".join(ALPHA[x] for x in codes[k]).encode())
    return 0, b"", b"".join(r + b"\n" for r in recs)


def _oracle_read(oracle_bin, files, sep, td):
    paths = {}
    for key, data in files.items():
        p = td / f"{key}.fa"
        p.write_bytes(data)
        paths[key] = p
    dump = td / "dump.txt"
    if dump.exists():
        dump.unlink()
    args = [str(oracle_bin), "-q", "-d", sep]
    if "in2" in paths:
        args += ["-s", str(paths["in2"])]
    args += ["-o", os.devnull, str(paths["in"])]
    r = subprocess.run(args, capture_output=True, env={**os.environ, "TN93_ORACLE_DUMP": str(dump)}, timeout=60)
    return r.returncode, r.stderr, (dump.read_bytes() if r.returncode == 0 else None)


@pytest.mark.parametrize("seed", range(6))
def test_reader_matches_oracle_on_fuzz_inputs(oracle_bin, tmp_path, seed):
    from swifttn93_b200 import build

    build.build_lib()
    rng = random.Random(7100 + seed)
    for k in range(60):
        files, flags = cases.fuzz_case(rng)
        sep = flags[flags.index("-d") + 1] if "-d" in flags else ":"
        want = _oracle_read(oracle_bin, files, sep, tmp_path)
        got = _lib_read(files, sep)
        assert got[0] == want[0], (seed, k, got[1], want[1])
        if want[0]:
            assert got[1] == want[1], (seed, k)
        else:
            assert got[2] == want[2], (seed, k)


def test_reader_messages_and_second_file_length(oracle_bin, tmp_path):
    samples = {
        "empty": {"in": b""},
        "no_sequence": {"in": b">a\n"},
        "empty_name": {"in": b">\nACGT\n"},
        "zero_length": {"in": b">a\n\n>b\nAC\n"},
        "unequal": {"in": b">a\nACGT\n>b\nACG\n"},
        "second_unequal": {"in": b">a\nACGT\n", "in2": b">q\nACGTA\n"},
        "second_ok": {"in": b">a:3\nACGT\n", "in2": b">q:2\nacgu\n"},
        "junk_bytes": {"in": b">a\nAC.X*GT\n>b x:7\nA C G T\n"},
    }
    for tag, files in samples.items():
        want = _oracle_read(oracle_bin, files, ":", tmp_path)
        got = _lib_read(files, ":")
        assert got[0] == want[0], tag
        assert (got[1] if want[0] else got[2]) == (want[1] if want[0] else want[2]), tag


def test_summary_json_formats_like_printf():
    """tn93g_summary_json prints every number as C's %g / %lu, in tn93's field order."""
    import ctypes as C

    import numpy as np

    from swifttn93_b200 import Summary, _Summary

    rng = np.random.default_rng(5)
    S = _Summary()
    S.pairwise, S.skipped, S.links = 123456789, 1234, 4321
    for k in range(3):
        S.max[k] = float(rng.random())
        S.mean[k] = float(rng.random() * 1e5)
        S.weighted[k] = float(rng.integers(1, 10**9))
        for b in range(200):
            S.hist[k][b] = int(rng.integers(0, 10**6))
    summ = Summary(0, 0, 0, [], [], [], None, 0, 0, 0, 0, raw=S)
    got = summ.json(4000, 0, False, False).decode()
    h = ",".join("[%g,%d]" % ((b + 1.0) / 200, S.hist[0][b]) for b in range(200))
    want = ("{\n\t\"Actual comparisons performed\" :%d,\n" % (S.pairwise - S.skipped)
            + "\t\"Comparisons accounting for copy numbers \" :%g,\n" % (S.weighted[0] + S.weighted[1] + S.weighted[2])
            + "\t\"Total comparisons possible\" : %d,\n" % S.pairwise
            + "\t\"Links found\" : %d,\n" % S.links + "\t\"Maximum distance\" : %g,\n" % S.max[0]
            + "\t\"Sequences\" : 4000,\n" + "\t\"Mean distance\" : %g,\n" % (S.mean[0] / S.weighted[0])
            + "\t\"Histogram\" : [" + h + "]\n}\n")
    assert got == want
    got2 = summ.json(30000, 17, True, False).decode()
    assert "\t\"Sequences in first file\" : 30000,\n\t\"Sequences in second file\" : 17,\n" in got2
