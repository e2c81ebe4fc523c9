"""Test inputs shared by the parity tests and tests/golden/make_fixtures.py.

fuzz_case(rng): a tiny adversarial FASTA (or two) plus random tn93 flags, covering what the reference's own
black-box gate covers (evaluate.py:61-99): tiny n and L around word boundaries, lowercase and IUPAC codes,
characters the reader drops or rejects, duplicate / odd / empty names, copy numbers, CRLF, wrapped lines,
blank lines, a missing final newline, unequal lengths, empty and truncated files; flags -t -l -a (including
ambiguity lists) -g -w -f -c -n -0 -D -d -s -m.

golden_cases(): the seeded benchmark-shaped workloads and the real sets, with the flag sets whose reference
outputs (sha256 of file and stdout) are committed in tests/golden/ref_outputs.json.
"""
from __future__ import annotations

import lzma
import random
from pathlib import Path

GOLDEN = Path(__file__).resolve().parent / "golden"

CORE = b"ACGT"
EXTRA = b"acgtRYSWKMBDHVNnrykmswbdhvuU-?"
WEIRD = b".X*~ 1"


def _records(rng: random.Random, n, L, p_extra, names, unequal):
    recs = []
    weird = p_extra * 0.1 if rng.random() < 0.1 else 0.0
    for i in range(n):
        if names == "dup" and i and rng.random() < 0.4:
            nm = recs[rng.randrange(len(recs))][0]
        elif names == "copies":
            nm = f"s{i}:{rng.randint(1, 5)}" if rng.random() < 0.8 else f"s{i}"
        elif names == "odd" and rng.random() < 0.3:
            nm = rng.choice(["", " ", "a b", "x,y", "p;q", "t\tu", "w" * 90, "n:0", "m:-2", "k::3"])
        else:
            nm = f"seq{i}"
        Li = L if not unequal or rng.random() < 0.7 else max(0, L + rng.randint(-4, 4))
        out = bytearray()
        for _ in range(Li):
            r = rng.random()
            out.append(rng.choice(WEIRD) if r < weird else rng.choice(EXTRA) if r < p_extra else rng.choice(CORE))
        if rng.random() < 0.15:
            k = rng.randint(0, max(0, Li // 3))
            out[:k] = b"-" * k
        if rng.random() < 0.1:
            k = rng.randint(0, max(0, Li // 3))
            if k:
                out[Li - k:] = b"-" * k
        recs.append((nm, bytes(out)))
    if n >= 2 and rng.random() < 0.5:  # near-duplicates so that thresholds matter
        base = recs[0][1]
        for j in range(1, n):
            if rng.random() < 0.5 and len(recs[j][1]) == len(base):
                s = bytearray(base)
                for _ in range(rng.randint(0, 3)):
                    if s:
                        s[rng.randrange(len(s))] = rng.choice(b"ACGTRNYB-")
                recs[j] = (recs[j][0], bytes(s))
    return recs


def _render(recs, rng: random.Random) -> bytes:
    wrap = rng.choice([0, 0, 0, 7, 60])
    nl = b"\r\n" if rng.random() < 0.05 else b"\n"
    buf = bytearray()
    for nm, s in recs:
        buf += (b"#" if rng.random() < 0.03 else b">") + nm.encode() + nl
        if rng.random() < 0.05:
            buf += nl
        if wrap and s:
            for k in range(0, len(s), wrap):
                buf += s[k:k + wrap] + nl
        else:
            buf += s + nl
    if rng.random() < 0.05:
        buf = buf.rstrip(b"\r\n")
    return bytes(buf)


def fuzz_case(rng: random.Random):
    """(files, flags): files maps "in"/"in2" to bytes; "{in2}" in flags stands for the second file."""
    r = rng.random()
    if r < 0.02:
        return {"in": b""}, []
    if r < 0.04:
        return {"in": rng.choice([b">", b">a\n", b">a\nACGT\n>b\n", b"ACGT\n", b">a\nAC\n>b\nACG\n",
                                  b">\nACGT\n", b">a\n\n"])}, ["-l", "1"]
    n = rng.choice([1, 2, 2, 3, 4, 5, 6, 8, 12, 20, 33])
    L = rng.choice([1, 2, 5, 17, 40, 63, 64, 65, 100, 127, 128, 129, 150, 200, 250, 300, 400])
    p_extra = rng.choice([0.0, 0.0, 0.02, 0.1, 0.4])
    names = rng.choice(["plain", "plain", "dup", "odd", "copies"])
    unequal = rng.random() < 0.03
    files = {"in": _render(_records(rng, n, L, p_extra, names, unequal), rng)}
    flags = ["-t", rng.choice(["0", "0.001", "0.015", "0.05", "0.1", "0.3", "0.75", "1", "2"])]
    flags += ["-l", str(rng.choice([1, 1, 1, 2, max(1, L // 4), max(1, L // 2), L, L + 1, 100]))]
    if rng.random() < 0.6:
        flags += ["-a", rng.choice(["resolve", "average", "skip", "gapmm", "RY", "RYSWKM", "N", "bdhv", "RN?"])]
        if rng.random() < 0.4:
            flags += ["-g", rng.choice(["0", "0.01", "0.05", "0.5", "1"])]
    if rng.random() < 0.15:
        flags += ["-w", rng.choice(["0", "0.001", "0.02"])]
    flags += ["-f", rng.choice(["csv", "csv", "csvn", "hyphy"])]
    for f, p in (("-c", 0.1), ("-n", 0.2), ("-0", 0.2)):
        if rng.random() < p:
            flags.append(f)
    if rng.random() < 0.15:
        flags += ["-D", rng.choice([";", "|", ":"])]
    if names == "copies" or rng.random() < 0.05:
        flags += ["-d", rng.choice([":", ":", "_"])]
    if rng.random() < 0.2:
        n2 = rng.choice([1, 2, 3, 5, 8, 40])
        L2 = L if rng.random() < 0.95 else L + 1
        files["in2"] = _render(_records(rng, n2, L2, p_extra, rng.choice(["plain", "dup", "copies"]), False), rng)
        flags += ["-s", "{in2}"]
        if rng.random() < 0.3:
            flags.append("-m")
    return files, flags


#----------------------------------------------------------------------------------------------- golden cases
HIVTRACE = ["-t", "0.015", "-a", "resolve", "-g", "0.05", "-l", "500"]


def golden_cases(include_large=True):
    """name, input source and flags of every committed reference output."""
    c = [
        dict(name="plain_small_hivtrace", src="synth:plain_small", flags=HIVTRACE + ["-f", "csv"]),
        dict(name="plain_small_average", src="synth:plain_small", flags=["-t", "0.05", "-a", "average", "-l", "500"]),
        dict(name="plain_small_gapmm", src="synth:plain_small", flags=["-t", "0.05", "-a", "gapmm", "-f", "csvn"]),
        dict(name="plain_small_skip_all", src="synth:plain_small", flags=["-t", "1", "-a", "skip", "-l", "200"]),
        dict(name="plain_small_subset", src="synth:plain_small", flags=["-t", "0.03", "-a", "RY", "-g", "0.005"]),
        dict(name="plain_small_self_csvn", src="synth:plain_small", flags=["-t", "0.02", "-0", "-f", "csvn", "-D", ";"]),
        dict(name="plain_small_hyphy", src="synth:plain_small", flags=["-t", "0.03", "-f", "hyphy"]),
        dict(name="plain_small_count", src="synth:plain_small", flags=["-t", "0.02", "-c"]),
        dict(name="plain_small_min_noheader", src="synth:plain_small", flags=["-t", "0.04", "-w", "0.01", "-n"]),
        dict(name="plain_small_two_file", src="synth:plain_small_split", flags=HIVTRACE + ["-s", "{in2}"]),
        dict(name="plain_small_fst", src="synth:plain_small_split", flags=["-t", "0.03", "-s", "{in2}", "-m"]),
        dict(name="real_hiv_dev_hivtrace", src="real:hiv_dev", flags=HIVTRACE),
        dict(name="real_hiv_dev_average", src="real:hiv_dev", flags=["-t", "0.05", "-a", "average", "-l", "500"]),
        dict(name="real_sars2_dev_self", src="real:sars2_dev", flags=["-t", "0.0002", "-l", "20000", "-0"]),
        dict(name="real_sars2_dev_allpairs", src="real:sars2_dev", flags=["-t", "1", "-D", ";"]),
        dict(name="long_n_runs", src="synth:long_n_runs",
             flags=["-t", "0.0001", "-a", "resolve", "-g", "0.05", "-l", "5000", "-f", "csvn"]),
    ]
    if include_large:
        for m in ("resolve", "average", "gapmm"):
            c.append(dict(name=f"hiv_bench_all_{m}", src="synth:hiv_bench",
                          flags=["-t", "1000", "-a", m, "-g", "0.05", "-l", "500", "-f", "csv"]))
        c.append(dict(name="hiv_bench_hivtrace", src="synth:hiv_bench", flags=HIVTRACE + ["-f", "csv"]))
    return c


def _xz(name):
    return lzma.decompress((GOLDEN / name).read_bytes())


_cache = {}


def source_bytes(src: str):
    """(FASTA bytes of the main input, FASTA bytes of the second input or None)."""
    if src in _cache:
        return _cache[src]
    import sys

    sys.path.insert(0, str(GOLDEN.parent.parent))
    from swifttn93_b200 import synth

    if src == "synth:plain_small":
        out = (synth.to_fasta(*synth.plain_small()), None)
    elif src == "synth:plain_small_split":
        names, codes = synth.plain_small()
        out = (synth.to_fasta(names[:300], codes[:300]), synth.to_fasta(names[300:], codes[300:]))
    elif src == "synth:hiv_bench":
        out = (synth.to_fasta(*synth.hiv_bench()), None)
    elif src == "synth:long_n_runs":
        out = (synth.to_fasta(*synth.long_n_runs()), None)
    elif src == "real:hiv_dev":
        out = (_xz("real_hiv_pol_dev.fa.xz"), None)
    elif src == "real:hiv_8766":
        out = (_xz("real_hiv_pol_dev.fa.xz") + _xz("real_hiv_pol_holdout.fa.xz"), None)
    elif src == "real:sars2_dev":
        out = (_xz("real_sars2_dev.fa.xz"), None)
    else:
        raise KeyError(src)
    _cache[src] = out
    return out


def materialise(case, td: Path) -> Path:
    """Writes the case's input(s) under td; replaces "{in2}" in case["flags"] by the second file's path."""
    a, b = source_bytes(case["src"])
    p = td / (case["name"] + ".fa")
    p.write_bytes(a)
    if b is not None:
        p2 = td / (case["name"] + "_2.fa")
        p2.write_bytes(b)
        case["flags"] = [str(p2) if f == "{in2}" else f for f in case["flags"]]
    return p
