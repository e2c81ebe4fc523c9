"""CPU tests of the product's host-side pieces: the C ABI library loads and exports every declared symbol (no
compute calls without a GPU), the scalar arithmetic shared with the kernels (log certificate, %g, formula)
against the C library, and the workload generator."""
import re
import subprocess
from pathlib import Path

import numpy as np

from tests.conftest import REPO


def test_library_exports_every_declared_symbol():
    from swifttn93_b200 import EXPORTS, build, load_library

    build.build_lib()
    lib = load_library()
    header = (REPO / "include" / "tn93g.h").read_text()
    declared = set(re.findall(r"\b(tn93g_[a-z_]+)\s*\(", header))
    assert declared == set(EXPORTS)
    for name in declared:
        assert getattr(lib, name) is not None


def test_cli_builds():
    from swifttn93_b200 import build

    lib, cli = build.build_all()
    assert cli.exists() and lib.exists()


def test_scalar_math_against_libc(tmp_path):
    exe = tmp_path / "math_check"
    src = REPO / "tests" / "native" / "math_check.cpp"
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{REPO / 'swifttn93_b200' / 'csrc'}",
                        str(src), str(REPO / "swifttn93_b200" / "csrc" / "logtable.cpp"), "-o", str(exe),
                        "-lquadmath", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for seed in (1, 2, 3):
        r = subprocess.run([str(exe), "400000", str(seed)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr


def test_generator_shapes():
    from swifttn93_b200 import synth

    names, codes = synth.plain_small()
    assert codes.shape == (500, 1300) and codes.dtype == np.uint8 and codes.max() <= 17
    assert len(set(names)) == 500
    sp = synth.batch_spec(7)
    assert 50 <= sp["n"] <= 4000 and 900 <= sp["L"] <= 3000
