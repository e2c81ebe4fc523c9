"""CPU tests of the oracle (oracle/tn93_oracle.c): pinned against the reference's golden sha256 vectors
(application/results/network.jsonl, copied to tests/golden/hiv_pol_network_hashes.json), against the committed
reference outputs, and against the reference binary itself on the fuzz corpus when it was built here."""
import json
import random
import tempfile
from pathlib import Path

import pytest

from tests import cases
from tests.conftest import REPO, run_tn93, sha256

GOLDEN = REPO / "tests" / "golden"


def _write(files, td):
    paths = {}
    for k, data in files.items():
        p = td / f"{k}.fa"
        p.write_bytes(data)
        paths[k] = p
    return paths


def test_oracle_vs_reference_fuzz(oracle_bin, ref_bin):
    rng = random.Random(20261203)
    bad = []
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for k in range(1000):
            files, flags = cases.fuzz_case(rng)
            paths = _write(files, td)
            fl = [str(paths["in2"]) if f == "{in2}" else f for f in flags]
            rr, fr, sr, _ = run_tn93(ref_bin, fl, paths["in"], td, threads=1)
            ro, fo, so, _ = run_tn93(oracle_bin, fl, paths["in"], td, threads=3)
            ok = (ro != 0) if rr != 0 else (ro == 0 and fo == fr and so == sr)
            if not ok:
                bad.append((k, flags, rr, ro))
    assert not bad, bad[:5]


def test_oracle_golden_network_hash(oracle_bin):
    """tn93 v1.1.0's own output hashes on the 8,766-sequence HIV-1 pol set (one of the five thresholds)."""
    g = json.loads((GOLDEN / "hiv_pol_network_hashes.json").read_text())
    row = g["rows"][0]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = td / "hiv8766.fa"
        inp.write_bytes(cases.source_bytes("real:hiv_8766")[0])
        assert sha256(inp.read_bytes()) == g["input_sha256"]
        flags = [row["t_arg"] if f == "{T}" else f for f in g["flags"] if f != "-q"]
        rc, fb, so, _ = run_tn93(oracle_bin, flags, inp, td)
        assert rc == 0
        assert sha256(fb) == row["file_sha256"] and len(fb) == row["file_bytes"]
        assert sha256(so) == row["stdout_sha256"]


SMALL = [c for c in cases.golden_cases(include_large=False) if c["src"].startswith("synth:plain")]


@pytest.mark.parametrize("case", SMALL, ids=[c["name"] for c in SMALL])
def test_oracle_vs_committed_reference_outputs(oracle_bin, case):
    want = json.loads((GOLDEN / "ref_outputs.json").read_text())[case["name"]]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        case = dict(case)
        inp = cases.materialise(case, td)
        rc, fb, so, _ = run_tn93(oracle_bin, case["flags"], inp, td)
        assert rc == want["rc"]
        assert sha256(fb or b"") == want["file_sha256"]
        assert sha256(so) == want["stdout_sha256"]
