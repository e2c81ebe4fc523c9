"""Exactness of every printed byte when the C library's log may round a logarithm the other way.

The engine computes logarithms correctly rounded; tn93 calls the C library's log, which may differ by one ulp
close to a rounding midpoint. A pair whose printed text, histogram bin or link decision depends on that rounding
is "undecided": its logarithms are taken from the host's C library and the pair is finished again on the device.
The JSON maximum and means are certified from per-unit bounds, or come from a second, exact pass.

With the default band (0.03 ulp) undecided pairs are rare, so these tests widen the band and the distance of the
alternative candidate (tn93g_set_log_band, or TN93G_LOG_BAND / TN93G_LOG_SPREAD for the command line). That
exaggerates the uncertainty without changing what tn93 prints: every output must still equal the committed
reference output (or the oracle's) byte for byte, with undecided pairs finished and none left over.

The certificate itself is host arithmetic and is tested on the CPU below."""
import ctypes as C
import json
import re
import tempfile
from pathlib import Path

import numpy as np
import pytest

from tests import cases
from tests.conftest import REPO, run_tn93, sha256

GOLDEN = REPO / "tests" / "golden"
STATS = re.compile(rb"finished with the C library's log (\d+), undecided (\d+), exact-sums pass (\d)")


def _stats(stderr: bytes):
    m = STATS.search(stderr)
    assert m, stderr[-400:]
    return int(m.group(1)), int(m.group(2)), int(m.group(3))


# (committed case, band, spread): spreads of 2^20..2^30 ulps make the candidates differ in the 7th significant
# digit for a few to most printed pairs; 2^34 also makes the mean's bound too wide to certify
WIDENED = [
    ("plain_small_hivtrace", 0.5, 2.0 ** 30),
    ("plain_small_hivtrace", 0.5, 2.0 ** 34),
    ("plain_small_fst", 0.5, 2.0 ** 30),
    ("plain_small_two_file", 0.5, 2.0 ** 28),
    ("plain_small_self_csvn", 0.5, 2.0 ** 30),
    ("real_hiv_dev_hivtrace", 0.5, 2.0 ** 24),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,band,spread", WIDENED, ids=[f"{c}-{int(np.log2(s))}" for c, _, s in WIDENED])
def test_widened_band_still_matches_reference(engine_cli, name, band, spread):
    case = next(c for c in cases.golden_cases(include_large=False) if c["name"] == name)
    want = json.loads((GOLDEN / "ref_outputs.json").read_text())[name]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = cases.materialise(case, td)
        rc, fb, so, se = run_tn93(engine_cli, case["flags"], inp, td,
                                  extra_env={"TN93G_LOG_BAND": str(band), "TN93G_LOG_SPREAD": str(spread),
                                             "TN93G_STATS": "1"})
    assert rc == 0, se[-500:]
    resolved, undecided, repass = _stats(se)
    assert resolved > 0 and undecided == 0, (resolved, undecided)
    assert sha256(fb) == want["file_sha256"] and sha256(so) == want["stdout_sha256"], (name, resolved, repass)
    if spread >= 2.0 ** 34:
        assert repass == 1  # the mean's bound was too wide: the JSON numbers came from the exact pass


@pytest.mark.gpu
def test_default_band_summary_reports_no_undecided(engine_cli):
    """On the real HIV set at the default band every pair is decided: nothing left over, and the certificate of
    the JSON numbers holds without the exact pass."""
    case = next(c for c in cases.golden_cases(include_large=False) if c["name"] == "real_hiv_dev_hivtrace")
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = cases.materialise(case, td)
        rc, fb, so, se = run_tn93(engine_cli, case["flags"], inp, td, extra_env={"TN93G_STATS": "1"})
    assert rc == 0
    _, undecided, repass = _stats(se)
    assert undecided == 0 and repass == 0


@pytest.mark.gpu
@pytest.mark.parametrize("spread", [2.0 ** 30, 2.0 ** 34], ids=["spread30", "spread34"])
def test_widened_band_server_and_batch_match_default(oracle_bin, tmp_path, spread):
    """The resident-reference server and the batched form finish their undecided pairs the same way: with a
    widened band every response equals the oracle's -s run and every batched alignment its default-band run. At
    the wider spread more pairs are undecided than the first lists hold (the server grows its list and runs the
    batch again; the batched form runs those alignments again alone)."""
    from swifttn93_b200 import Engine, Fasta, HostAlignment, Options, ResidentReference, synth

    rng = np.random.default_rng(5)
    rnames, rcodes = synth.serve_reference(seed=9, n=800, L=1200)
    ref = synth.to_fasta(rnames, rcodes)
    (tmp_path / "ref.fa").write_bytes(ref)
    opts = Options(threshold=0.03, mode="resolve", min_overlap=500)
    eng = Engine()
    eng.set_log_band(0.5, spread)
    R = Fasta(ref)
    srv = ResidentReference(eng, R, opts, max_batch_sequences=256, max_batch_queries=8)
    qfa = []
    for k, q in enumerate((3, 40, 17)):
        names, codes = synth.serve_query(rng, rcodes, q, f"w{k}")
        qfa.append(synth.to_fasta(names, codes))
    out = srv.batch([Fasta(q, expect_len=R.L) for q in qfa])
    resolved = out[0][1].logs_resolved
    links = 0
    for k, (body, summ) in enumerate(out):
        qp = tmp_path / f"q{k}.fa"
        qp.write_bytes(qfa[k])
        # tn93 -s QUERY.fa REF.fa: the reference is the positional file (rows), the query the second
        rc, fo, so, _ = run_tn93(oracle_bin, ["-t", "0.03", "-a", "resolve", "-l", "500", "-s", str(qp)],
                                 tmp_path / "ref.fa", tmp_path)
        assert rc == 0
        assert b"ID1,ID2,Distance\n" + body == fo, k
        js = summ.json(R.n, Fasta(qfa[k]).n, second_file=True)
        assert js == so, k
        links += summ.links
    srv.close()
    assert resolved > 0 and links > 0
    # batch: widened band against the default band (itself checked against the oracle in test_batch); small
    # alignments of the batched workload's shape
    ha, ops = [], []
    for i in range(3):
        names, codes = synth.hiv_bench(seed=70 + i, n=150 + 60 * i, L=900 + 200 * i, clusters=2, tag=f"x{i}")
        ha.append(HostAlignment(codes, names))
        ops.append(Options(threshold=0.02, mode="resolve", resolve_fraction=0.05, min_overlap=300))
    widened = eng.batch_run(ha, ops)
    plain = Engine().batch_run(ha, ops)
    assert sum(s.logs_resolved for _, s in widened) > 0
    for (bw, sw), (bp, sp) in zip(widened, plain):
        assert bw == bp
        assert (sw.max, sw.mean, sw.weighted, sw.links, sw.skipped) == (sp.max, sp.mean, sp.weighted, sp.links,
                                                                          sp.skipped)
        assert np.array_equal(sw.hist, sp.hist)


@pytest.mark.gpu
def test_bounded_wait_times_out_and_context_recovers():
    """Failure detection without a fault: one tile of the count kernel never receives its first operand stage
    (tn93g_inject_fault), so its bounded wait runs out; the run returns TN93G_ETIMEOUT, and the next run on the same
    context is correct."""
    from swifttn93_b200 import ETIMEOUT, FAULT_SKIP_FILL, Engine, Options, synth

    names, codes = synth.plain_small(seed=11, n=200, L=700)
    opts = Options(threshold=0.05, mode="resolve", resolve_fraction=0.05, min_overlap=200)
    eng = Engine()
    s = eng.upload(codes, names)
    want, _ = eng.run(s, opts)
    eng.set_wait_limit(0.05)
    eng.inject_fault(FAULT_SKIP_FILL)
    assert eng.run_status(s, opts) == ETIMEOUT
    got, summ = eng.run(s, opts)
    assert got == want and summ.undecided == 0


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_division_scheme_is_exact(seed):
    """The device formula shares one true division per divisor and finishes each quotient with two fused
    multiply-add corrections: its outputs up to the logarithms equal the host's IEEE-division evaluation bit for bit,
    and its quotients over 80 binades equal the device's correctly rounded division."""
    from swifttn93_b200 import Engine

    assert Engine().selftest_division(2_000_000, seed) == (0, 0)


#----------------------------------------------------------------------------------------------- CPU
def _summary(mean, weighted, mx, bounds):
    from swifttn93_b200 import _Summary

    S = _Summary()
    for q in range(3):
        S.mean[q] = mean[q]
        S.weighted[q] = weighted[q]
        S.max[q] = mx[q]
        for k in range(4):
            S.amb_bounds[q][k] = bounds[q][k]
    return S


def _certified(S, chain=1000, fst=0):
    from swifttn93_b200 import load_library

    return load_library().tn93g_summary_certified(C.byref(S), chain, fst)


Z = [0.0, 0.0, 0.0, 0.0]


def test_certificate_without_ambiguous_pairs_holds():
    S = _summary([123.456789, 0, 0], [1000.0, 0, 0], [0.3, 0, 0], [Z, Z, Z])
    assert _certified(S) == 1


def test_certificate_mean_far_from_a_rounding_boundary_holds():
    # mean 0.1234564..., a spread of 1e-12 cannot move its sixth digit
    S = _summary([123.4564, 0, 0], [1000.0, 0, 0], [0.3, 0, 0], [[0.3 - 1e-12, 0.3, 1e-12, 10], Z, Z])
    assert _certified(S) == 1
    # a largest low candidate far below the maximum leaves the maximum itself uncertain
    S = _summary([123.4564, 0, 0], [1000.0, 0, 0], [0.3, 0, 0], [[0.29, 0.3, 1e-12, 10], Z, Z])
    assert _certified(S) == 0


def test_certificate_mean_at_a_rounding_boundary_fails():
    # mean 0.1234565 sits on the sixth digit's rounding boundary: any spread may print either neighbour
    S = _summary([123.4565, 0, 0], [1000.0, 0, 0], [0.3, 0, 0], [[0.3 - 1e-12, 0.3, 1e-9, 10], Z, Z])
    assert _certified(S) == 0


def test_certificate_maximum_straddling_a_digit_fails():
    # the largest pair may be 0.1234565 +- 1e-9 in the C library: "0.123456" or "0.123457"
    S = _summary([10.0, 0, 0], [100.0, 0, 0], [0.1234565, 0, 0], [[0.1234565 - 1e-9, 0.1234565 + 1e-9, 0., 1], Z, Z])
    assert _certified(S) == 0
    # the same candidates below a larger, unambiguous maximum are harmless
    S = _summary([10.0, 0, 0], [100.0, 0, 0], [0.2, 0, 0], [[0.1234565 - 1e-9, 0.1234565 + 1e-9, 0., 1], Z, Z])
    assert _certified(S) == 1


def test_certificate_fst_expressions():
    m = [40.0, 30.0, 90.0]
    w = [400.0, 300.0, 600.0]
    S = _summary(m, w, [0.2, 0.2, 0.3], [[0.19, 0.1, 1e-13, 3], Z, [0.1, 0.1, 1e-13, 2]])
    assert _certified(S, fst=1) == 1
    S = _summary(m, w, [0.2, 0.2, 0.3], [[0.19, 0.1, 1e-3, 3], Z, [0.1, 0.1, 1e-3, 2]])
    assert _certified(S, fst=1) == 0


def test_shard_merge_combines_bounds():
    from swifttn93_b200.shard import Partial, certified, merge

    def part(r0, r1, b):
        return Partial(r0, r1, b"", 1, 0, 0, [0.1, 0, 0], np.zeros((3, 200), dtype=np.uint64),
                       np.array([[0.05, 0, 0, 1.0, 0, 0]] * (r1 - r0)), amb_bounds=np.array(b))
    b1 = [[0.01, 0.02, 2.0 ** -52, 2], Z, Z]
    b2 = [[0.03, 0.04, 2.0 ** -51, 3], Z, Z]
    _, S = merge([part(2, 4, b2), part(0, 2, b1)])
    assert list(S.raw.amb_bounds[0]) == [0.03, 0.04, 3 * 2.0 ** -52, 5]
    assert certified(S, N=4, n1=4, cross=False)
    _, S0 = merge([part(0, 2, [Z, Z, Z]), part(2, 4, [Z, Z, Z])])
    assert certified(S0, N=4, n1=4, cross=False)
