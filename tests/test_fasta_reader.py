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


def _check(data, expect_len=0):
    """tn93g_fasta_check: the device ingest's record scan and checks, letters counted on the host."""
    import ctypes as C

    from swifttn93_b200 import load_library

    lib = load_library()
    n, L = C.c_long(), C.c_long()
    msg = C.create_string_buffer(512)
    rc = lib.tn93g_fasta_check(data, len(data), int(expect_len), b":", C.byref(n), C.byref(L), msg, 512)
    return rc, msg.value.decode(errors="replace"), n.value, L.value


def _read(data, expect_len=0):
    from swifttn93_b200 import Fasta, FastaError

    try:
        f = Fasta(data, expect_len=expect_len)
        return 0, "", f.n, f.L
    except FastaError as e:
        return -9, str(e), 0, 0


def test_device_ingest_scan_matches_reader():
    """The device ingest (tn93g_upload_fasta) finds records with byte searches and applies the reader's checks in
    its order from per-record letter counts; with the counts taken on the host (tn93g_fasta_check) it must accept
    and refuse exactly what tn93g_read_fasta does, with the same message and size."""
    from swifttn93_b200 import build

    build.build_lib()
    rng = random.Random(7400)
    accepted = refused = 0
    for k in range(400):
        files, _ = cases.fuzz_case(rng)
        data = files["in"]
        for expect in (0, 7):
            got, want = _check(data, expect), _read(data, expect)
            assert got == want, (k, expect, got, want)
            accepted += got[0] == 0
            refused += got[0] != 0
    extra = [b"", b"ACGT", b">", b">\n", b">a", b">a\nAC\n>\nAC\n", b"#a\nAC\n#b\nAC", b">a\r\nAC\r\n>b\nA>C\n",
             b">a\nACGT\n>b\nAC\n>c\n", b">a b:3\nAC-?N\n>c:x:2\nnnac\n", b"\n\n>a\nA\nC\n#b\nAC"]
    for data in extra:
        for expect in (0, 2, 4):
            assert _check(data, expect) == _read(data, expect), (data, expect)
    assert accepted > 50 and refused > 20, (accepted, refused)
