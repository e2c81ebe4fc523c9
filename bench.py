#!/usr/bin/env python3
"""Throughput of the all-pairs TN93 path: pairwise distances per second, including the byte-exact text.

Workload (one step): the benchmark-shaped alignment of 6,700 sequences x 1,500 columns (seeded synthetic data,
swifttn93_b200.synth.hiv_bench: coalescent background at 6% divergence, 40 transmission clusters, 1% IUPAC
ambiguity with 4% of sequences at 3-5%, gap runs and ragged ends), run once each with -a resolve, -a average and
-a gapmm at -t 1000 -g 0.05 -l 500 -f csv, so every one of the 3 x 22,441,650 pairs is written.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value  : pairs/s with the alignment resident in HBM and the distance file left in HBM (tn93g_run_to_device),
         device-timed with CUDA events on the engine's stream, L2 flushed between steps (outside the events).
e2e    : pairs/s through the C ABI from host buffers: every step uploads the codes (from pinned host memory) and
         the names, and copies the distance file back to pinned host memory (tn93g_upload + tn93g_run); the host
         alignment (names encoded as bytes with their offsets) is prepared once, before the timed steps.
--impl reference: the reference swifttn93 built from its own sources (oracle/_ref) on the host cores, same
         workload and options, output to a tmpfs file, wall clock.
Multi-GPU (torchrun): every rank runs its own replica of the workload (pairs are independent; no collective on
the data path), value = pairs of all ranks / max over ranks of the device time.
variant_hivtrace_t0.015: the same alignment at -t 0.015 (few pairs written). variant_served_s: the -s serving
loop (serving_variant). variant_batched: 96 independent alignments in one batched call (batched_variant). None
of them is the headline value.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "pairwise distances/sec (incl. byte-exact formatting) on 1 B200 vs host-CPU swifttn93"
MODES = ("resolve", "average", "gapmm")
FLAGS = dict(threshold=1000.0, resolve_fraction=0.05, min_overlap=500, format="csv")
WORKLOAD = "hiv_bench 6700x1500, -t 1000 -g 0.05 -l 500 -f csv, -a resolve/average/gapmm (all pairs written)"


# ncu figures of the pair stage behind the roofline line, 4,000-sequence prefix under -a resolve (one 16 M-pair chunk
# holds all 7,998,000 pairs): DRAM bytes of its count_tc_persist_kernel + pair_kernel launches with the caches kept
# between kernels (profiles/pair_stage_traffic_hiv_bench_n4000.md), the count kernel's tensor-pipe activity
# (profiles/count_tc_kernel_hiv_bench_n4000.md) and the pair kernel's instructions and issue activity
# (profiles/pair_kernel_hiv_bench_n4000.md)
PAIR_STAGE_PROFILE = {"pairs": 7998000, "dram_bytes": 400.36e6, "tensor_pipe_active": 0.417,
                      "pair_kernel_inst_per_pair": 467694944 * 32 / 7998000, "pair_kernel_issue_active": 0.555,
                      "files": ["profiles/pair_stage_traffic_hiv_bench_n4000.md",
                                "profiles/count_tc_kernel_hiv_bench_n4000.md", "profiles/pair_kernel_hiv_bench_n4000.md"]}


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return dict(hbm=d["hbm_gbs"], bf16=d["bf16_tflops"], src="measured")
    return dict(hbm=6650.0, bf16=1590.0, src="fallback")


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index=0):
        self.index, self.samples, self._stop = index, [], threading.Event()

    def __enter__(self):
        def run():
            q = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    r = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                        "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                    if r.returncode == 0 and r.stdout.strip():
                        self.samples.append([x.strip() for x in r.stdout.strip().split(",")])
                except Exception:  # noqa: BLE001
                    pass
                self._stop.wait(0.2)

        self.t = threading.Thread(target=run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 4 + k and s[4 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def workload():
    from swifttn93_b200 import synth

    names, codes = synth.hiv_bench()
    return names, codes


def variable_columns(codes):
    """Columns that are not the same clean base in every sequence (what the engine counts over)."""
    first = codes[0]
    const = (first < 4) & np.all(codes == first[None, :], axis=0)
    return int((~const).sum())


def reference_binary():
    flags = set(open("/proc/cpuinfo").read().split()) if os.path.exists("/proc/cpuinfo") else set()
    need = {"avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512vbmi", "avx512_vbmi2", "avx512ifma",
            "avx512_vpopcntdq", "avx512_bitalg", "avx512_vnni", "gfni", "vaes", "vpclmulqdq"}
    for name, ok in (("swifttn93", need <= flags), ("swifttn93_libm", True)):
        p = REPO / "oracle" / "_ref" / name
        if p.exists() and ok:
            return p
    return None


def run_reference(names, codes, steps, warmup, sample_modes=MODES, tflag="1000"):
    """Wall time of the reference binary on all host cores over the workload; returns (pairs/s, detail)."""
    from swifttn93_b200 import synth

    ref = reference_binary()
    if ref is None:
        return None, "reference binary not built (oracle/build_ref.sh needs the reference sources)"
    tmpdir = Path("/dev/shm") if Path("/dev/shm").is_dir() else Path(tempfile.gettempdir())
    td = Path(tempfile.mkdtemp(dir=tmpdir))
    try:
        inp = td / "hiv_bench.fa"
        inp.write_bytes(synth.to_fasta(names, codes))
        n = codes.shape[0]
        pairs = n * (n - 1) // 2
        env = {**os.environ, "OMP_NUM_THREADS": str(os.cpu_count())}
        times = []
        for it in range(warmup + steps):
            t0 = time.perf_counter()
            for m in sample_modes:
                out = td / "out.csv"
                r = subprocess.run([str(ref), "-q", "-t", tflag, "-a", m, "-g", "0.05", "-l", "500", "-f", "csv",
                                    "-o", str(out), str(inp)], stdout=subprocess.DEVNULL, env=env)
                if r.returncode != 0:
                    return None, f"reference exited {r.returncode}"
                out.unlink()
            if it >= warmup:
                times.append(time.perf_counter() - t0)
        per_step = float(np.mean(times))
        return pairs * len(sample_modes) / per_step, dict(binary=ref.name, cores=os.cpu_count(), step_s=per_step)
    finally:
        shutil.rmtree(td, ignore_errors=True)


def cli_variant(names, codes, steps, warmup):
    """The product's command line (swifttn93_b200/bin/tn93g) on the workload, as the reference arm runs the
    reference binary: -q -t 1000 -a MODE -g 0.05 -l 500 -f csv -o /dev/shm/out.csv, one process per mode, wall
    clock. Also checks that each file and stdout equal the committed reference outputs of this workload."""
    import hashlib

    from swifttn93_b200 import synth

    cli = REPO / "swifttn93_b200" / "bin" / "tn93g"
    if not cli.exists():
        return {"unavailable": "tn93g not built"}
    want = {}
    ref_json = REPO / "tests" / "golden" / "ref_outputs.json"
    if ref_json.exists():
        want = json.loads(ref_json.read_text())
    tmpdir = Path("/dev/shm") if Path("/dev/shm").is_dir() else Path(tempfile.gettempdir())
    td = Path(tempfile.mkdtemp(dir=tmpdir))
    try:
        inp = td / "hiv_bench.fa"
        inp.write_bytes(synth.to_fasta(names, codes))
        n = codes.shape[0]
        times, identical = [], True
        for it in range(warmup + steps):
            t0 = time.perf_counter()
            for m in MODES:
                out = td / "out.csv"
                r = subprocess.run([str(cli), "-q", "-t", "1000", "-a", m, "-g", "0.05", "-l", "500", "-f", "csv",
                                    "-o", str(out), str(inp)], stdout=subprocess.PIPE, stderr=subprocess.PIPE)
                if r.returncode != 0:
                    return {"error": f"tn93g exited {r.returncode}: {r.stderr[-200:]!r}"}
                if it == 0 and f"hiv_bench_all_{m}" in want and n == 6700:
                    w = want[f"hiv_bench_all_{m}"]
                    identical = identical and hashlib.sha256(out.read_bytes()).hexdigest() == w["file_sha256"] and \
                        hashlib.sha256(r.stdout).hexdigest() == w["stdout_sha256"]
                out.unlink()
            if it >= warmup:
                times.append(time.perf_counter() - t0)
        step = float(np.mean(times))
        return {"value": len(MODES) * n * (n - 1) // 2 / step, "unit": "pairs/s", "s_per_step": step,
                "outputs_identical_to_reference": identical if n == 6700 else None,
                "note": "tn93g -q ... -o /dev/shm/out.csv per mode: process start, FASTA parsing, device set-up, "
                        "run and file write inside the wall clock (the reference arm's measurement)"}
    finally:
        shutil.rmtree(td, ignore_errors=True)


SERVE_FLAGS = ["-t", "0.015", "-a", "resolve", "-l", "500"]


def serving_variant(rates=(20.0, 200.0), seconds=4.0, saturate=1200, ref_sample=8, plain_sample=64,
                    worker_counts=(2, 4)):
    """The served form: a resident reference of 30,000 x 1,500 (synth.serve_reference) and query FASTAs of 1-512
    sequences (geometric, mean 32), each derived from a random reference sequence at 0.5-3% divergence with 1%
    ambiguity, run as tn93 -s QUERY REF -t 0.015 -a resolve -l 500 through the continuous-batching service
    (8 GB HBM budget). Poisson streams at each rate for `seconds` (2 workers), then a saturating burst at each
    worker count. Latency is arrival to response (host bytes of the distance file and JSON summary); pairs/s =
    reference x query sequences answered / (first arrival to last response).
    Beside it, on the same queries: the plain path (one tn93g_upload of reference + query and one tn93g_run per
    query, the way a caller without the server runs -s), and the reference binary on a sample of them (one
    process per request, REF.fa from tmpfs, all host cores), whose file and stdout bytes must equal the service's
    responses (responses_identical)."""
    from swifttn93_b200 import Engine, Fasta, Options, synth
    from swifttn93_b200.serve import Service, query_stream, run_load

    rnames, rcodes = synth.serve_reference()
    ref = synth.to_fasta(rnames, rcodes)
    n_req = [int(r * seconds) for r in rates]
    qs = query_stream(rcodes, max(n_req + [saturate]), seed=5)
    opts = Options(threshold=0.015, mode="resolve", min_overlap=500)
    out = {"workload": "resident reference 30000x1500 (serve_reference), queries 1-512 seqs (geometric, mean 32), "
                       "0.5-3% divergence, 1% ambiguity; tn93 -s QUERY REF -t 0.015 -a resolve -l 500",
           "unit": "pairs/s", "hbm_budget_bytes": 8 << 30}
    sample_responses = None
    for w in worker_counts:
        # the budget is split over the workers: at 4 workers a batch holds up to 128 queries
        with Service(ref, opts, hbm_budget=8 << 30, workers=w, max_batch_queries=256 if w <= 2 else 128) as svc:
            run_load(svc, qs[:50], 1e7, seed=1)  # warm-up: buffers reach their working sizes
            if w == worker_counts[0]:
                out["workers"] = w
                out["batch_capacity"] = {"sequences": svc.cap_sequences, "queries": svc.cap_queries}
                for rate, n in zip(rates, n_req):
                    r = run_load(svc, qs[:n], rate, seed=int(rate))
                    out[f"poisson_{int(rate)}rps"] = {k: r[k] for k in ("requests", "ok", "span_s", "pairs",
                                                                       "pairs_per_s", "p50_ms", "p99_ms")}
            b0 = svc.stats.batches
            r = run_load(svc, qs[:saturate], 1e7, seed=9)
            sat = {k: r[k] for k in ("requests", "ok", "span_s", "pairs", "pairs_per_s", "p50_ms", "p99_ms")}
            sat["batches"] = svc.stats.batches - b0
            out[f"saturated_{w}_workers"] = sat
            if w == worker_counts[0]:
                out["saturated"] = sat
                sample_responses = r["responses"][:max(ref_sample, 1)]
    out["value"] = max(out[f"saturated_{w}_workers"]["pairs_per_s"] for w in worker_counts)
    # the plain path on the same queries: reference + query uploaded and run per request (-s orientation)
    eng = Engine()
    R = Fasta(ref)
    pairs, t_plain = 0, 0.0
    for q in qs[:plain_sample]:
        Q = Fasta(q, expect_len=R.L)
        codes = np.concatenate([R.codes, Q.codes])
        names = R.names + Q.names
        counts = np.concatenate([R.counts, Q.counts])
        t0 = time.perf_counter()
        s = eng.upload(codes, names, counts)
        eng.run(s, opts, n1=R.n, sink="discard")
        eng.free(s)
        t_plain += time.perf_counter() - t0
        pairs += R.n * Q.n
    eng.close()
    out["plain_path_value"] = pairs / t_plain
    out["plain_path_note"] = (f"{plain_sample} of the queries, each one tn93g_upload (reference + query codes and "
                              "names from host arrays; array assembly untimed) and one tn93g_run with n1 = 30000, "
                              "text to the engine's pinned buffer")
    binary = reference_binary()
    if binary is not None and ref_sample:
        tmpdir = Path("/dev/shm") if Path("/dev/shm").is_dir() else Path(tempfile.gettempdir())
        td = Path(tempfile.mkdtemp(dir=tmpdir))
        try:
            (td / "ref.fa").write_bytes(ref)
            env = {**os.environ, "OMP_NUM_THREADS": str(os.cpu_count())}
            lat, pairs, same = [], 0, True
            for k, q in enumerate(qs[:ref_sample]):
                (td / "q.fa").write_bytes(q)
                t0 = time.perf_counter()
                r = subprocess.run([str(binary), "-q", *SERVE_FLAGS, "-s", str(td / "q.fa"), "-o", str(td / "o.csv"),
                                    str(td / "ref.fa")], stdout=subprocess.PIPE, env=env)
                lat.append(time.perf_counter() - t0)
                if r.returncode != 0:
                    lat = []
                    break
                resp = sample_responses[k]
                same = same and resp.rc == 0 and resp.file == (td / "o.csv").read_bytes() and resp.stdout == r.stdout
                pairs += rcodes.shape[0] * q.count(b">")
            if lat:
                out["reference"] = {"binary": binary.name, "cores": os.cpu_count(), "requests": len(lat),
                                    "p50_ms": float(np.percentile(lat, 50)) * 1e3,
                                    "pairs_per_s": pairs / float(np.sum(lat)),
                                    "note": "one process per request, sequentially (the reference re-reads REF.fa)"}
                out["responses_identical"] = same
                out["responses_identical_note"] = (f"file and stdout bytes of the first {len(lat)} requests of the "
                                                   "saturated run against the reference binary's")
        finally:
            shutil.rmtree(td, ignore_errors=True)
    return out


def _gen_batch_alignment(i):
    from swifttn93_b200 import synth

    return synth.batch_alignment(i)


def batched_variant(eng, steps, warmup, n_aln=96, ref_sample=6, plain=True):
    """The batched form: 96 independent alignments (synth.batch_spec: sizes log-uniform 50-4,000, lengths
    900-3,000, each with its own -t in 0.005-0.02 and -a mode; -g 0.05 -l 500 -f csv), all run by one
    tn93g_batch_run call per step (inputs in pinned host memory, texts back on the host), against the plain path:
    the same alignments one tn93g_upload + tn93g_run after another. Pair tiles are picked by the autotuner
    (untimed). Every batched output is checked against the plain path's bytes."""
    import concurrent.futures as cf
    import hashlib
    import multiprocessing as mp

    import torch

    from swifttn93_b200 import HostAlignment, Options, autotune

    with cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        gen = list(ex.map(_gen_batch_alignment, range(n_aln)))
    specs = [g[0] for g in gen]
    pinned = []
    alns, opts = [], []
    for sp, names, codes in gen:
        t = torch.empty(codes.shape, dtype=torch.uint8).pin_memory()
        t.numpy()[:] = codes
        pinned.append(t)
        alns.append(HostAlignment(t.numpy(), names))
        opts.append(Options(threshold=sp["threshold"], mode=sp["mode"], resolve_fraction=0.05, min_overlap=500))
    pairs = sum(a.n * (a.n - 1) // 2 for a in alns)
    tuning = autotune.load_or_tune(eng, torch.cuda.get_device_name())
    rpw = [autotune.rows_per_warp(tuning, a.L) for a in alns]
    blocks = tuning["pair_blocks"]
    out = eng.batch_run(alns, opts, rows_per_warp=rpw, pair_blocks=blocks)  # bytes for the parity check
    text_bytes = sum(len(b) for b, _ in out)
    bt, dev, stage = [], [], {}
    for it in range(warmup + steps):
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("batch_step")  # profiling filter (ncu --nvtx-include batch_step/)
        t0 = time.perf_counter()
        eng.batch_run(alns, opts, rows_per_warp=rpw, pair_blocks=blocks, sink="discard")
        t1 = time.perf_counter()
        torch.cuda.nvtx.range_pop()
        if it >= warmup:
            bt.append(t1 - t0)
            tm = eng.last_timings()
            dev.append(tm["total"])
            for k, v in tm.items():
                stage[k] = stage.get(k, 0.0) + v / steps
            launches = eng.last_launches()
    digest_b = hashlib.sha256(b"".join(hashlib.sha256(b).digest() for b, _ in out)).hexdigest()
    # the plain path, alignment after alignment (the same host buffers; texts to the engine's pinned buffer)
    names = [[bytes(a._names.raw[int(x):int(x) + int(n)]) for x, n in zip(a._off, a._len)] for a in alns]
    plain_out = []
    for a, o, nm in (zip(alns, opts, names) if plain else ()):
        s = eng.upload(a)
        plain_out.append(eng.run(s, o)[0])
        eng.free(s)
    digest_p = hashlib.sha256(b"".join(hashlib.sha256(b).digest() for b in plain_out)).hexdigest()
    pt = []
    for it in range(warmup + steps if plain else 0):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for a, o, nm in zip(alns, opts, names):
            s = eng.upload(a)
            eng.run(s, o, sink="discard")
            eng.free(s)
        if it >= warmup:
            pt.append(time.perf_counter() - t0)
    res = {"workload": f"{n_aln} alignments (batch_spec): n log-uniform 50-4000, L 900-3000, per-alignment -t "
                       "0.005-0.02 and -a resolve/average/gapmm, -g 0.05 -l 500 -f csv",
           "pairs_per_step": pairs, "unit": "pairs/s",
           "value": pairs / float(np.mean(bt)), "device_value": pairs / (float(np.mean(dev)) / 1e3),
           "plain_path_value": pairs / float(np.mean(pt)) if pt else None,
           "note": "value = pairs / wall time of one tn93g_batch_run (inputs from pinned host memory, every text "
                   "copied to the engine's pinned host buffer); device_value = pairs / device time of the call; "
                   "plain_path_value = the same alignments one tn93g_upload + tn93g_run after another",
           "outputs_identical_to_plain_path": (digest_b == digest_p) if plain else None,
           "text_bytes_per_step": text_bytes,
           "h2d_bytes_per_step": int(sum(a._codes.nbytes for a in alns)), "gpu_launches": launches,
           "stage_ms": stage, "tuning": {k: tuning[k] for k in ("pair_blocks", "rows_per_warp", "bands")}}
    binary = reference_binary()
    if binary is not None and ref_sample:
        from swifttn93_b200 import synth

        tmpdir = Path("/dev/shm") if Path("/dev/shm").is_dir() else Path(tempfile.gettempdir())
        td = Path(tempfile.mkdtemp(dir=tmpdir))
        try:
            env = {**os.environ, "OMP_NUM_THREADS": str(os.cpu_count())}
            wall, rp = 0.0, 0
            for k in range(0, n_aln, max(1, n_aln // ref_sample))[:ref_sample]:
                sp, names, codes = gen[k]
                (td / "a.fa").write_bytes(synth.to_fasta(names, codes))
                t0 = time.perf_counter()
                r = subprocess.run([str(binary), "-q", "-t", repr(sp["threshold"]), "-a", sp["mode"], "-g", "0.05",
                                    "-l", "500", "-f", "csv", "-o", str(td / "o.csv"), str(td / "a.fa")],
                                   stdout=subprocess.DEVNULL, env=env)
                wall += time.perf_counter() - t0
                if r.returncode != 0:
                    wall = 0.0
                    break
                rp += sp["n"] * (sp["n"] - 1) // 2
            if wall:
                res["reference"] = {"binary": binary.name, "cores": os.cpu_count(), "pairs_per_s": rp / wall,
                                    "sample": f"{ref_sample} of the {n_aln} alignments, one process each"}
        finally:
            shutil.rmtree(td, ignore_errors=True)
    return res


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return ws, int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--n", type=int, default=0, help="use the first N sequences only (profiling runs)")
    ap.add_argument("--no-serving", action="store_true", help="skip the served (-s) variant")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched variant")
    ap.add_argument("--only", choices=["batched", "served"], help="run one variant alone (profiling runs)")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    names, codes = workload()
    if args.n:
        names, codes = names[:args.n], np.ascontiguousarray(codes[:args.n])
    n = codes.shape[0]
    pairs_step = len(MODES) * n * (n - 1) // 2
    config = {"workload": WORKLOAD, "sequences": n, "columns": int(codes.shape[1]), "pairs_per_step": pairs_step,
              "l2": "flushed between steps (256 MiB write), outside the timed events"}

    if args.impl == "reference":
        if rank != 0:
            return
        v, det = run_reference(names, codes, args.steps, max(1, args.warmup))
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": det}))
            return
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": det["step_s"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": det["cores"], "kind": "reference",
                                 "sample": f"full step ({len(MODES)} modes x {n*(n-1)//2} pairs), {det['binary']}, "
                                           "output to tmpfs"},
                "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    from swifttn93_b200 import Engine, HostAlignment, Options

    torch.cuda.set_device(local)
    eng = Engine(device=local)
    if args.only:
        if rank == 0:
            v = (batched_variant(eng, args.steps, args.warmup, ref_sample=0, plain=False) if args.only == "batched"
                 else serving_variant(ref_sample=0))
            print(json.dumps({"variant": args.only, **v}))
        eng.close()
        return
    stream = torch.cuda.ExternalStream(eng.stream, device=local)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{local}")
    opts = [Options(mode=m, **FLAGS) for m in MODES]
    Lc = variable_columns(codes)

    # ---- value: inputs and outputs resident in HBM
    s = eng.upload(codes, names)
    step_ms, stage_ms, launches, out_bytes = [], {}, 0, 0
    stage_by_mode = {m: {} for m in MODES}
    clocks = Clocks(local)
    for it in range(args.warmup + args.steps):
        timed = it >= args.warmup
        if timed and it == args.warmup:
            if ws > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            clocks.__enter__()
        with torch.cuda.stream(stream):
            flush.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        summ = []
        for o in opts:
            ptr, nb, sm = eng.run_to_device(s, o)
            summ.append(sm)
            if timed:
                launches += eng.last_launches()
                out_bytes += nb
                for k, v in sm.timings_ms.items():
                    stage_ms[k] = stage_ms.get(k, 0.0) + v
                    stage_by_mode[o.mode][k] = stage_by_mode[o.mode].get(k, 0.0) + v
        ev1.record(stream)
        ev1.synchronize()
        if timed:
            step_ms.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    clocks.__exit__()
    if ws > 1:
        torch.distributed.barrier()
    total_ms = float(np.sum(step_ms))
    if ws > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = pairs_step * args.steps * ws / (total_ms / 1e3)

    # ---- e2e: host buffers in, host bytes out, through the C ABI
    pinned = torch.empty(codes.shape, dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = codes
    pin_np = pinned.numpy()
    # the host alignment (pinned codes, encoded names): prepared once, uploaded every step
    host_aln = HostAlignment(pin_np, names)
    e2e_ms, h2d, d2h = [], 0, 0
    e2e_parts = {"upload": 0.0, "run": 0.0, "free": 0.0, "d2h_device": 0.0, "write_device": 0.0}
    for it in range(0 if args.no_e2e else args.warmup + args.steps):
        timed = it >= args.warmup
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nbytes = 0
        for o in opts:
            ta = time.perf_counter()
            s2 = eng.upload(host_aln)
            tb = time.perf_counter()
            _, sm = eng.run(s2, o, sink="discard")
            tc = time.perf_counter()
            nbytes += sm.output_bytes
            eng.free(s2)
            td = time.perf_counter()
            if timed:
                e2e_parts["upload"] += (tb - ta) * 1e3 / args.steps
                e2e_parts["run"] += (tc - tb) * 1e3 / args.steps
                e2e_parts["free"] += (td - tc) * 1e3 / args.steps
                e2e_parts["d2h_device"] += sm.timings_ms.get("d2h", 0.0) / args.steps
                e2e_parts["write_device"] += sm.timings_ms.get("write", 0.0) / args.steps
        torch.cuda.synchronize()
        if timed:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            h2d = len(MODES) * (codes.nbytes + sum(len(x) for x in names) + 24 * n)
            d2h = nbytes
    e2e = pairs_step * ws / (float(np.mean(e2e_ms)) / 1e3) if e2e_ms else None

    # ---- roofline of the dominant stage: the pair stage (count_tc_persist_kernel + pair_kernel)
    # Algorithmic work (the clean-site count contraction): 16 x Lc INT8 one-hot MACs per pair, 25 x Lc when the
    # N/gap plane is active (gapmm here), 2 ops per MAC, against dense INT8 = 2 x the bf16 tensor peak. The count
    # kernel is reported alone against the same peak on its 16 x Lc; the pair kernel (CUDA cores: sparse events,
    # formula, certificate) is issue-bound and reported with its instructions per pair from the profile.
    P = peaks()
    pairs_run = n * (n - 1) // 2
    per_mode = stage_by_mode
    work = {m: pairs_run * (25 if m == "gapmm" else 16) * Lc * 2 for m in MODES}
    pair_ms = {m: per_mode[m]["pair"] / args.steps for m in MODES}
    count_ms = {m: per_mode[m].get("count", 0.0) / args.steps for m in MODES}
    achieved = sum(work.values()) / (sum(pair_ms.values()) / 1e3) / 1e12
    peak_tc = 2 * P["bf16"]
    tc_work = sum(pairs_run * 16 * Lc * 2 for _ in MODES)
    tc_ms = sum(count_ms.values())
    # DRAM bytes of one pair-stage launch (count_tc_persist_kernel + pair_kernel) from the ncu capture named below,
    # scaled by pairs; algorithmic bytes: the raw distance written once (8 B per pair) and the operands read once
    # (one-hot image 4 Lc B, bit planes 4 x 8 B per 64 columns, codes and transposed codes 2 Lc B per sequence)
    prof_pairs, prof_bytes = PAIR_STAGE_PROFILE["pairs"], PAIR_STAGE_PROFILE["dram_bytes"]
    traffic = prof_bytes * pairs_run / prof_pairs
    alg_bytes = 8 * pairs_run + n * (4 * Lc + 4 * 8 * ((Lc + 63) // 64) + 2 * Lc)
    roof = {"kernel": "pair stage: count_tc_persist_kernel + pair_kernel", "bound": "tensor", "achieved": achieved,
            "peak": peak_tc, "unit": "TFLOP/s", "frac": achieved / peak_tc, "traffic": traffic,
            "traffic_over_algorithmic": traffic / alg_bytes,
            "peak_note": f"dense INT8 ops = 2 x {P['src']} bf16 ({P['bf16']} TF/s)",
            "work_note": f"16 x Lc INT8 MACs per pair (25 x Lc under gapmm), x2 ops; Lc = {Lc}; per 3-mode step",
            "pair_stage_ms_per_launch": {m: pair_ms[m] for m in MODES},
            "count_tc_kernel": {"name": "count_tc_persist_kernel",
                                "achieved": tc_work / (tc_ms / 1e3) / 1e12 if tc_ms else None, "unit": "TFLOP/s",
                                "frac": (tc_work / (tc_ms / 1e3) / 1e12) / peak_tc if tc_ms else None,
                                "ms_per_launch": {m: count_ms[m] for m in MODES},
                                "tensor_pipe_active": PAIR_STAGE_PROFILE["tensor_pipe_active"]},
            "pair_kernel": {"ms_per_launch": {m: pair_ms[m] - count_ms[m] for m in MODES}, "bound": "issue",
                            "instructions_per_pair": PAIR_STAGE_PROFILE["pair_kernel_inst_per_pair"],
                            "issue_active": PAIR_STAGE_PROFILE["pair_kernel_issue_active"]},
            "profile": PAIR_STAGE_PROFILE["files"]}

    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof, "gpu_launches": launches, "clocks": clocks.summary(),
            "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()},
            "e2e_ms_per_step_parts": e2e_parts,
            "engine": {"Lc": Lc, "ambiguous_log_pairs": int(sum(x.logs_ambiguous for x in summ)),
                       "undecided": int(sum(x.undecided for x in summ)),
                       "replayed": int(sum(x.pairs_replayed for x in summ))}}
    # the drop-in command line, timed the way the reference arm is: one process per mode on the workload's FASTA,
    # the distance file written to tmpfs, wall clock (process start, FASTA parsing, device set-up included)
    if rank == 0 and ws == 1 and not args.no_e2e:
        line["variant_cli"] = cli_variant(names, codes, args.steps, max(1, args.warmup))
    # the compute-bound variant (HIV-TRACE flags: -t 0.015 -a resolve -g 0.05 -l 500): few pairs are written
    if not args.no_e2e:
        o15 = Options(mode="resolve", threshold=0.015, resolve_fraction=0.05, min_overlap=500, format="csv")
        vt, et = [], []
        for it in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            eng.run_to_device(s, o15)
            ev1.record(stream)
            ev1.synchronize()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s3 = eng.upload(host_aln)
            _, sm15 = eng.run(s3, o15, sink="discard")
            eng.free(s3)
            torch.cuda.synchronize()
            if it >= args.warmup:
                vt.append(ev0.elapsed_time(ev1))
                et.append((time.perf_counter() - t0) * 1e3)
        pr = n * (n - 1) // 2
        line["variant_hivtrace_t0.015"] = {"value": pr / (np.mean(vt) / 1e3), "e2e": pr / (np.mean(et) / 1e3),
                                            "unit": "pairs/s", "links": sm15.links,
                                            "flags": "-t 0.015 -a resolve -g 0.05 -l 500 -f csv"}
    if ws > 1 and not args.no_e2e:
        # one alignment split over the ranks by row bands (swifttn93_b200.shard): each rank's band device-timed,
        # max over ranks, then the ordered gather of the bands to rank 0
        from swifttn93_b200.shard import engine_compute, run_sharded

        o15 = Options(mode="resolve", threshold=0.015, resolve_fraction=0.05, min_overlap=500, format="csv")
        comp = engine_compute(eng, s, o15)
        exact = engine_compute(eng, s, o15, exact=True)
        band_ms = []

        def timed_compute(r0, r1):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            part = comp(r0, r1)
            e1.record(stream)
            e1.synchronize()
            band_ms.append(e0.elapsed_time(e1))
            return part

        try:
            run_sharded(comp, n, n, False, exact_compute=exact)  # warm-up
            torch.distributed.barrier()
            t0 = time.perf_counter()
            merged = run_sharded(timed_compute, n, n, False, exact_compute=exact)
            wall = time.perf_counter() - t0
            t = torch.tensor([band_ms[-1]], device=f"cuda:{local}")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            pr = n * (n - 1) // 2
            if rank == 0:
                line["variant_sharded_rows"] = {
                    "value": pr / (float(t.item()) / 1e3), "unit": "pairs/s", "scaling": "strong",
                    "flags": "-t 0.015 -a resolve -g 0.05 -l 500 -f csv", "ranks": ws,
                    "note": "one alignment, row bands balanced by pairs; value = pairs / max over ranks of the "
                            "band's device time; the ordered gather to rank 0 is timed separately",
                    "with_gather_wall_s": wall, "links": merged[1].links}
        except Exception as e:  # noqa: BLE001 - reported in the line, the headline is unaffected
            if rank == 0:
                line["variant_sharded_rows"] = {"error": repr(e)}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, det = run_reference(names, codes, 1, 1)
        if v is not None:
            line["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": det["cores"], "kind": "reference",
                                    "sample": f"one full step ({len(MODES)} x {pairs_run} pairs), {det['binary']}, "
                                              "output to tmpfs"}
        if "variant_hivtrace_t0.015" in line:
            v15, _ = run_reference(names, codes, 1, 1, sample_modes=("resolve",), tflag="0.015")
            if v15 is not None:
                line["variant_hivtrace_t0.015"]["reference"] = v15
    eng.free(s)
    if rank == 0 and ws == 1 and not args.no_batched and not args.n:
        line["variant_batched"] = batched_variant(eng, args.steps, args.warmup)
    eng.close()
    if rank == 0 and ws == 1 and not args.no_serving and not args.n:
        line["variant_served_s"] = serving_variant()
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
