"""FASTA ingest on the device (tn93g_upload_fasta) against the host reader (tn93g_read_fasta, itself pinned to the
oracle's restatement of tn93's reader in test_fasta_reader.py): on the fuzz inputs of the parity gate and on wrapped,
CRLF and '#'-record files, both refuse the same files with the same message, and accepted files give a set whose
run prints the same distance file and summary as the host reader's codes, names and copy numbers uploaded."""
import random

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu


def _compare(eng, data, opts, expect_len=0):
    from swifttn93_b200 import Fasta, FastaError

    try:
        host = Fasta(data, expect_len=expect_len)
        host_err = None
    except FastaError as e:
        host, host_err = None, str(e)
    try:
        dev = eng.upload_fasta(data, expect_len=expect_len)
        dev_err = None
    except FastaError as e:
        dev, dev_err = None, str(e)
    assert host_err == dev_err, (host_err, dev_err)
    if host_err is not None:
        return False
    assert (dev.N, dev.L) == (host.n, host.L)
    s = eng.upload(host)
    want_body, want = eng.run(s, opts)
    got_body, got = eng.run(dev, opts)
    eng.free(s)
    eng.free(dev)
    assert got_body == want_body
    assert got.json(host.n) == want.json(host.n)
    return True


def test_fuzz_inputs_match_host_reader():
    from swifttn93_b200 import Engine, Options

    eng = Engine()
    opts = Options(threshold=1.0, mode="resolve", min_overlap=1)
    rng = random.Random(7300)
    accepted = refused = 0
    for k in range(200):
        files, _ = cases.fuzz_case(rng)
        if _compare(eng, files["in"], opts):
            accepted += 1
        else:
            refused += 1
    assert accepted > 20 and refused > 5, (accepted, refused)


def _fasta(names, codes, width, eol, opener=b">"):
    alpha = np.frombuffer(b"ACGTURYSWKMBDHVN?-", dtype=np.uint8)
    out = []
    for nm, row in zip(names, codes):
        seq = alpha[row].tobytes()
        lines = [seq[p:p + width] for p in range(0, len(seq), width)] if width else [seq]
        out.append(opener + nm.encode() + eol + eol.join(lines) + eol)
    return b"".join(out)


@pytest.mark.parametrize("width,eol,opener", [(0, b"\n", b">"), (60, b"\r\n", b">"), (61, b"\n", b"#"),
                                              (1, b"\n", b">")],
                         ids=["one-line", "wrapped-crlf", "hash-records", "one-per-line"])
def test_formatted_files_match_host_reader(width, eol, opener):
    from swifttn93_b200 import Engine, Options, synth

    names, codes = synth.plain_small(seed=21, n=180, L=700 if width != 1 else 90)
    names = [f"{nm}:{1 + k % 3}" for k, nm in enumerate(names)]  # copy numbers after the separator
    eng = Engine()
    data = _fasta(names, codes, width, eol, opener)
    assert _compare(eng, data, Options(threshold=0.05, mode="average", min_overlap=50))
    # the required length of a second file: accepted at the right length, refused with the reader's message otherwise
    assert _compare(eng, data, Options(threshold=0.05, mode="average", min_overlap=50), expect_len=codes.shape[1])
    assert not _compare(eng, data, Options(threshold=0.05), expect_len=codes.shape[1] + 1)
