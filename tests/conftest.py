import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

ORACLE = REPO / "oracle" / "bin" / "tn93_oracle"
REF_DIR = REPO / "oracle" / "_ref"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")
    config.addinivalue_line("markers", "slow: long-running")


def sha256(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


@pytest.fixture(scope="session")
def oracle_bin():
    """The C restatement of the reference path (built from oracle/tn93_oracle.c)."""
    r = subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return ORACLE


def _cpu_flags():
    try:
        return set(open("/proc/cpuinfo").read().split())
    except OSError:
        return set()


@pytest.fixture(scope="session")
def ref_bin():
    """The reference binary built from its own sources (oracle/build_ref.sh); prefers the libm build and skips
    when it was not built or cannot run on this CPU."""
    for name in ("swifttn93_libm", "swifttn93"):
        p = REF_DIR / name
        if p.exists():
            r = subprocess.run([str(p), "-v"], capture_output=True)
            if r.returncode == 0:
                return p
    pytest.skip("reference binary not built here (oracle/build_ref.sh)")


@pytest.fixture(scope="session")
def engine_cli():
    """The product's command line (needs the built engine and a GPU)."""
    from swifttn93_b200 import build

    lib, cli = build.build_all()
    return cli


def run_tn93(binary, flags, inp, td: Path, threads=None, extra_env=None):
    """Runs a tn93-compatible binary the way the reference's harness does (evaluate.py:75):
    BINARY -q FLAGS -o OUT IN. Returns (rc, file bytes or None, stdout bytes)."""
    out = td / f"out_{Path(binary).name}"
    if out.exists():
        out.unlink()
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    if extra_env:
        env.update(extra_env)
    r = subprocess.run([str(binary), "-q", *map(str, flags), "-o", str(out), str(inp)], cwd=td,
                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env, timeout=1800)
    return r.returncode, (out.read_bytes() if out.exists() else None), r.stdout, r.stderr
