"""The band pipeline's text delivery when links are sparse.

tn93g_run computes the rows in bands; a band's text is written into one of two device/pinned buffer pairs and
handed to the sink while the next bands compute. A band whose rows hold no link writes no text, so two bands that
follow each other in the output can use the same buffer pair: the older text must reach the sink before the
buffers are written again. These cases print a handful of links spread over many bands and compare the bytes with
the oracle (the C restatement)."""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import run_tn93

pytestmark = pytest.mark.gpu


def _sparse_links(seed: int, n: int, L: int, link_rows) -> bytes:
    """Unrelated random sequences (distance about 0.75), except that row i + 1 is row i with 0.5% point changes for
    every i in link_rows: at -t 0.02 each listed row links to the next one."""
    rng = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ACGT", dtype=np.uint8)
    rows = alpha[rng.integers(0, 4, (n, L))]
    for i in link_rows:
        rows[i + 1] = rows[i]
        m = rng.random(L) < 0.005
        rows[i + 1, m] = alpha[rng.integers(0, 4, int(m.sum()))]
    return b"".join(b">s%04d\n" % i + rows[i].tobytes() + b"\n" for i in range(n))


@pytest.mark.parametrize("link_rows,band_pairs", [
    ((0, 60, 120, 180, 240, 300, 360, 420, 480, 540), 2000),
    ((3, 4, 200, 201, 590), 1500),
    ((10, 11, 12, 400), 6000),
], ids=["every60", "clustered", "few"])
def test_sparse_links_with_small_bands(engine_cli, oracle_bin, link_rows, band_pairs):
    flags = ["-t", "0.02", "-a", "resolve", "-l", "100"]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        inp = td / "sparse.fa"
        inp.write_bytes(_sparse_links(7, 600, 800, link_rows))
        rg, fg, sg, eg = run_tn93(engine_cli, flags, inp, td, extra_env={"TN93G_BAND_PAIRS": str(band_pairs)})
        ro, fo, so, _ = run_tn93(oracle_bin, flags, inp, td)
    assert ro == 0 and rg == 0, eg[-300:]
    assert fo.count(b"\n") >= 1 + len(link_rows)  # neighbours of a run of listed rows link too
    assert fg == fo and sg == so


def test_two_links_in_the_batched_workload(oracle_bin, tmp_path):
    """One alignment of the batched benchmark (1,827 x 2,250, -a average, -t 0.0074): two links, in bands of the
    same parity with link-free bands between them. tn93g_run (default bands) must print both."""
    from swifttn93_b200 import Engine, HostAlignment, Options, synth

    sp, names, codes = synth.batch_alignment(25)
    eng = Engine()
    s = eng.upload(HostAlignment(codes, names))
    body, summ = eng.run(s, Options(threshold=sp["threshold"], mode=sp["mode"], resolve_fraction=0.05,
                                    min_overlap=500))
    inp = tmp_path / "a25.fa"
    inp.write_bytes(synth.to_fasta(names, codes))
    ro, fo, so, _ = run_tn93(oracle_bin, ["-t", repr(sp["threshold"]), "-a", sp["mode"], "-g", "0.05", "-l", "500"],
                             inp, tmp_path)
    assert ro == 0
    assert summ.links == 2 and b"ID1,ID2,Distance\n" + body == fo
    assert summ.json(sp["n"]) == so
