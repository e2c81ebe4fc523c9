"""The command line's host side against the reference binary, on the CPU: option errors and FASTA reader errors
are reported before any GPU work, so for them tn93g must already exit with the reference's status and print the
reference's stdout and stderr bytes (argparse.cpp:117-126, swifttn93.cpp:259-406). Covers a list of bad
invocations and every fuzz input the reference refuses."""
import random
import subprocess
from pathlib import Path

import pytest

from tests import cases

BAD_ARGS = [
    ["-Z"], ["-f", "xml"], ["-g", "2"], ["-D", ";;"], ["-b"], ["-r"], ["-u", "2"], ["-t"], ["-d"],
    ["-s", "{missing}"], ["-o", "/nonexistent_dir/x"], ["-w"], ["-H"], ["-g", "-1"], ["-u", "-0.5"],
]


def _run(binary, args, td: Path):
    r = subprocess.run([str(binary), *args], cwd=td, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=120)
    return r.returncode, r.stdout, r.stderr


@pytest.fixture(scope="module")
def cli():
    from swifttn93_b200 import build

    return build.build_all()[1]


def test_version_matches_reference(ref_bin, cli, tmp_path):
    assert _run(cli, ["-v"], tmp_path) == _run(ref_bin, ["-v"], tmp_path)


@pytest.mark.parametrize("flag", ["-h", "--help"])
def test_help_matches_reference(ref_bin, cli, tmp_path, flag):
    """tn93's usage line and help text (argparse.cpp:41-107) on stderr, exit status 1."""
    want = _run(ref_bin, [flag], tmp_path)
    assert want[0] == 1 and len(want[2]) > 4000
    assert _run(cli, [flag], tmp_path) == want


@pytest.mark.parametrize("args", BAD_ARGS, ids=[" ".join(a) for a in BAD_ARGS])
def test_option_errors_match_reference(ref_bin, cli, tmp_path, args):
    fa = tmp_path / "ok.fa"
    fa.write_bytes(b">a\nACGT\n>b\nACGA\n")
    args = [str(tmp_path / "missing.fa") if a == "{missing}" else a for a in args]
    full = ["-q", *args, str(fa)] if args[-1] not in ("-t", "-d", "-w") else ["-q", str(fa), *args]
    want = _run(ref_bin, full, tmp_path)
    assert want[0] != 0, "the reference accepts this invocation"
    assert _run(cli, full, tmp_path) == want


def test_reader_errors_on_fuzz_inputs_match_reference(ref_bin, cli, tmp_path):
    rng = random.Random(9200)
    checked = 0
    for k in range(400):
        files, flags = cases.fuzz_case(rng)
        p = tmp_path / "in.fa"
        p.write_bytes(files["in"])
        if "in2" in files:
            (tmp_path / "in2.fa").write_bytes(files["in2"])
        args = ["-q", *[str(tmp_path / "in2.fa") if f == "{in2}" else f for f in flags], "-o",
                str(tmp_path / "out.csv"), str(p)]
        want = _run(ref_bin, args, tmp_path)
        if want[0] == 0:
            continue  # accepted input: the rest of the run needs the GPU
        assert _run(cli, args, tmp_path) == want, (k, flags)
        checked += 1
    assert checked >= 5
