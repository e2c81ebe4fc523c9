#!/usr/bin/env python3
"""Builds the committed parity fixtures under tests/golden/ from a reference checkout (default
/root/reference). Run once where the reference checkout exists; the parity tests only read the outputs.

Outputs:
  real_hiv_pol_dev.fa.xz, real_hiv_pol_holdout.fa.xz, real_sars2_dev.fa.xz
      Public GenBank alignments shipped with the reference (data/*.fa.xz), copied byte for byte and checked
      against the sha256 values the reference lists in data/README.txt:6-10.
  hiv_pol_network_hashes.json
      The reference's golden vectors for the all-pairs path: sha256 of tn93 v1.1.0's distance file and of its
      stdout JSON on the 8,766-sequence HIV-1 pol set (dev + holdout concatenated) at five thresholds, with
      flags -q -0 -t T -a resolve -l 500 -g 0.05 -f csv (application/results/network.jsonl:1-5,
      application/README.md:4-6).
  ref_outputs.json
      sha256 of the distance file and stdout of the reference binary (oracle/_ref/swifttn93_libm, built by
      oracle/build_ref.sh) on the seeded synthetic workloads and the real sets, for the flag sets that the
      parity tests run. Generated here because the tests run where the reference checkout may not exist.
"""
import hashlib
import json
import lzma
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

DATA_SHA = {  # data/README.txt:6-10
    "real_hiv_pol_dev.fa.xz": "4aaf148a5a307242842ccd1b070573327a705cf2743aa37fc2562d12c8878c91",
    "real_hiv_pol_holdout.fa.xz": "cf2f927b26a51add36f6920792aa382d5eaf3affeeaf3870651ed9a449b799de",
    "real_sars2_dev.fa.xz": "17c103d4b6fbf610475eb8a98ac46a4ef08624301a50d1dc27314715575f44fe",
}


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def copy_data(ref: Path):
    for name, want in DATA_SHA.items():
        src = ref / "data" / name
        got = sha(src.read_bytes())
        if got != want:
            raise SystemExit(f"{src}: sha256 {got} != {want}")
        shutil.copyfile(src, HERE / name)


def network_hashes(ref: Path):
    rows = []
    for line in (ref / "application" / "results" / "network.jsonl").read_text().splitlines():
        r = json.loads(line)
        rows.append(dict(t_arg=r["t_arg"], file_sha256=r["ref_file_sha256"], stdout_sha256=r["ref_stdout_sha256"],
                         file_bytes=r["file_bytes"], links=r["network"]["links"]))
    out = dict(input="real_hiv_pol_dev.fa.xz + real_hiv_pol_holdout.fa.xz (concatenated)",
               input_sha256="70985c02b3ba52585c9ed30db147ca14984a9f5fd03babb3af235432062a0524",
               flags=["-q", "-0", "-t", "{T}", "-a", "resolve", "-l", "500", "-g", "0.05", "-f", "csv"], rows=rows)
    (HERE / "hiv_pol_network_hashes.json").write_text(json.dumps(out, indent=1) + "\n")


def run_ref(binary: Path, flags, inputs, td: Path):
    """Runs the reference the way its own harness does: -q FLAGS -o OUT IN (evaluate.py:75)."""
    out = td / "ref.out"
    out.unlink(missing_ok=True)
    env = {**os.environ, "OMP_NUM_THREADS": str(os.cpu_count())}
    r = subprocess.run([str(binary), "-q", *flags, "-o", str(out), str(inputs)], stdout=subprocess.PIPE,
                       stderr=subprocess.DEVNULL, env=env, timeout=3600)
    fb = out.read_bytes() if out.exists() else b""
    return dict(rc=r.returncode, file_sha256=sha(fb), file_bytes=len(fb), stdout_sha256=sha(r.stdout))


def ref_outputs(binary: Path):
    from tests import cases  # noqa: E402  (the case list shared with the parity tests)

    res = {}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for case in cases.golden_cases():
            inp = cases.materialise(case, td)
            flags = [td / f if isinstance(f, Path) else f for f in case["flags"]]
            flags = [str(f) for f in flags]
            res[case["name"]] = run_ref(binary, flags, inp, td)
            print(case["name"], res[case["name"]], flush=True)
    (HERE / "ref_outputs.json").write_text(json.dumps(res, indent=1, sort_keys=True) + "\n")


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    copy_data(ref)
    network_hashes(ref)
    binary = REPO / "oracle" / "_ref" / "swifttn93_libm"
    if not binary.exists():
        subprocess.run(["bash", str(REPO / "oracle" / "build_ref.sh"), str(ref)], check=True)
    ref_outputs(binary)


if __name__ == "__main__":
    main()
