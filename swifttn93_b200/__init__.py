"""swifttn93_b200 -- all-pairs TN93 distances on NVIDIA B200, byte-exact with tn93 v1.1.0 / swifttn93.

The engine is the shared library lib/libtn93g.so (sm_100a kernels behind the C ABI of include/tn93g.h); this
module binds it with ctypes. There is no CPU fallback: importing works anywhere, but creating an Engine needs
the built library and a CUDA device, and raises otherwise.

    from swifttn93_b200 import Engine, Options
    eng = Engine()
    s = eng.upload(codes, names, counts)           # codes: uint8 [N, L] in 0..17 ("ACGTURYSWKMBDHVN?-")
    out, summary = eng.run(s, Options(threshold=0.015, mode="resolve", resolve_fraction=0.05, min_overlap=500))
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libtn93g.so"
CLI_PATH = PKG / "bin" / "tn93g"
ALPHABET = b"ACGTURYSWKMBDHVN?-"

MODES = {"resolve": 0, "average": 1, "skip": 2, "gapmm": 3, "subset": 4}
FORMATS = {"csv": 0, "csvn": 1, "hyphy": 2}

# symbols declared in include/tn93g.h
EXPORTS = ("tn93g_create", "tn93g_destroy", "tn93g_strerror", "tn93g_last_cuda_error", "tn93g_upload",
           "tn93g_free_set", "tn93g_run", "tn93g_run_to_device", "tn93g_stream", "tn93g_last_launches",
           "tn93g_last_timings", "tn93g_pair_distances_noalloc", "tn93g_noalloc_last_error", "tn93g_read_fasta",
           "tn93g_alignment_free", "tn93g_server_create", "tn93g_server_batch", "tn93g_server_destroy",
           "tn93g_summary_json", "tn93g_run_rows", "tn93g_batch_run", "tn93g_set_count_path",
           "tn93g_summary_certified", "tn93g_set_log_band", "tn93g_set_exact_sums", "tn93g_set_wait_limit",
           "tn93g_inject_fault", "tn93g_selftest_division", "tn93g_upload_fasta",
           "tn93g_fasta_check")

# error codes of include/tn93g.h used by the binding
EUNDECIDED = -10
ETIMEOUT = -6
FAULT_SKIP_FILL = 1


class _Opts(C.Structure):
    _fields_ = [("mode", C.c_int), ("threshold", C.c_double), ("min_distance", C.c_double),
                ("resolve_fraction", C.c_double), ("min_overlap", C.c_long), ("format", C.c_int),
                ("delimiter", C.c_char), ("report_self", C.c_int), ("count_only", C.c_int), ("do_fst", C.c_int),
                ("subset", C.c_ubyte * 18)]


class _Summary(C.Structure):
    _fields_ = [("pairwise", C.c_ulong), ("skipped", C.c_long), ("links", C.c_long), ("max", C.c_double * 3),
                ("mean", C.c_double * 3), ("weighted", C.c_double * 3), ("hist", (C.c_ulong * 200) * 3),
                ("pairs_replayed", C.c_long), ("logs_ambiguous", C.c_long), ("undecided", C.c_long),
                ("output_bytes", C.c_size_t), ("logs_resolved", C.c_long), ("sums_repass", C.c_int),
                ("amb_bounds", (C.c_double * 4) * 3)]


class _Alignment(C.Structure):
    _fields_ = [("codes", C.POINTER(C.c_uint8)), ("n", C.c_long), ("L", C.c_long),
                ("copy_counts", C.POINTER(C.c_long)), ("names", C.POINTER(C.c_char)),
                ("name_off", C.POINTER(C.c_size_t)), ("name_len", C.POINTER(C.c_long))]


_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_char), C.c_size_t)
_QSINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_char), C.c_size_t)

_lib = None


def load_library(path: Path | str = LIB_PATH):
    """Loads libtn93g.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path)
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m swifttn93_b200.build`")
    lib = C.CDLL(str(p))
    lib.tn93g_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_size_t]
    lib.tn93g_destroy.argtypes = [C.c_void_p]
    lib.tn93g_strerror.restype = C.c_char_p
    lib.tn93g_strerror.argtypes = [C.c_int]
    lib.tn93g_last_cuda_error.restype = C.c_char_p
    lib.tn93g_last_cuda_error.argtypes = [C.c_void_p]
    lib.tn93g_upload.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p, C.c_long, C.c_long, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    lib.tn93g_free_set.argtypes = [C.c_void_p, C.c_void_p]
    lib.tn93g_run.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.POINTER(_Opts), _SINK, C.c_void_p,
                              C.POINTER(_Summary)]
    lib.tn93g_last_timings.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
    lib.tn93g_run_to_device.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.POINTER(_Opts), C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_size_t), C.POINTER(_Summary)]
    lib.tn93g_stream.restype = C.c_void_p
    lib.tn93g_stream.argtypes = [C.c_void_p]
    lib.tn93g_last_launches.restype = C.c_long
    lib.tn93g_last_launches.argtypes = [C.c_void_p]
    lib.tn93g_read_fasta.argtypes = [C.c_char_p, C.c_size_t, C.c_long, C.c_char, C.POINTER(_Alignment), C.c_char_p,
                                     C.c_size_t]
    lib.tn93g_alignment_free.argtypes = [C.POINTER(_Alignment)]
    lib.tn93g_server_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p, C.c_long, C.c_long,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(_Opts), C.c_long,
                                        C.c_int]
    lib.tn93g_server_batch.argtypes = [C.c_void_p, C.c_int, C.POINTER(_Alignment), _QSINK, C.c_void_p,
                                       C.POINTER(_Summary)]
    lib.tn93g_server_destroy.argtypes = [C.c_void_p]
    lib.tn93g_run_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.POINTER(_Opts), C.c_long, C.c_long, _SINK,
                                   C.c_void_p, C.c_void_p, C.POINTER(_Summary)]
    lib.tn93g_set_count_path.argtypes = [C.c_void_p, C.c_int]
    lib.tn93g_batch_run.argtypes = [C.c_void_p, C.c_int, C.POINTER(_Alignment), C.POINTER(_Opts),
                                    C.POINTER(C.c_int), C.c_int, _QSINK, C.c_void_p, C.POINTER(_Summary)]
    lib.tn93g_summary_json.restype = C.c_size_t
    lib.tn93g_summary_json.argtypes = [C.POINTER(_Summary), C.c_ulong, C.c_ulong, C.c_int, C.c_int, C.c_char_p,
                                       C.c_size_t]
    lib.tn93g_summary_certified.argtypes = [C.POINTER(_Summary), C.c_long, C.c_int]
    lib.tn93g_set_log_band.argtypes = [C.c_void_p, C.c_double, C.c_double]
    lib.tn93g_set_exact_sums.argtypes = [C.c_void_p, C.c_int]
    lib.tn93g_set_wait_limit.argtypes = [C.c_void_p, C.c_double]
    lib.tn93g_inject_fault.argtypes = [C.c_void_p, C.c_int]
    lib.tn93g_selftest_division.argtypes = [C.c_void_p, C.c_long, C.c_ulonglong, C.POINTER(C.c_long)]
    lib.tn93g_upload_fasta.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t, C.c_long, C.c_char,
                                       C.POINTER(C.c_long), C.POINTER(C.c_long), C.c_char_p, C.c_size_t]
    lib.tn93g_fasta_check.argtypes = [C.c_char_p, C.c_size_t, C.c_long, C.c_char, C.POINTER(C.c_long),
                                      C.POINTER(C.c_long), C.c_char_p, C.c_size_t]
    _lib = lib
    return lib


@dataclass
class Options:
    """tn93's options for one run (the -t -w -a -g -l -f -D -0 -c -m flags)."""
    threshold: float = 0.015
    min_distance: float = -1.e-10
    mode: str = "resolve"        # resolve | average | skip | gapmm | an ambiguity list such as "RY"
    resolve_fraction: float = 1.0
    min_overlap: int = 100
    format: str = "csv"
    delimiter: str = ","
    report_self: bool = False
    count_only: bool = False
    do_fst: bool = False

    def to_c(self) -> _Opts:
        o = _Opts()
        if self.mode in MODES:
            o.mode = MODES[self.mode]
        else:
            o.mode = MODES["subset"]
            for ch in self.mode.upper().encode():
                k = ALPHABET.find(bytes([ch]))
                if k > 3:
                    o.subset[k] = 1
        o.threshold = self.threshold
        o.min_distance = self.min_distance
        o.resolve_fraction = self.resolve_fraction
        o.min_overlap = int(self.min_overlap)
        o.format = FORMATS[self.format]
        o.delimiter = self.delimiter.encode()[:1]
        o.report_self = int(self.report_self)
        o.count_only = int(self.count_only)
        o.do_fst = int(self.do_fst)
        return o


@dataclass
class Summary:
    pairwise: int
    skipped: int
    links: int
    max: list
    mean: list
    weighted: list
    hist: np.ndarray
    pairs_replayed: int
    logs_ambiguous: int
    undecided: int
    output_bytes: int
    logs_resolved: int = 0
    sums_repass: bool = False
    timings_ms: dict = field(default_factory=dict)
    raw: object = field(default=None, repr=False)

    def json(self, n1: int, n2: int = 0, second_file: bool = False, fst: bool = False) -> bytes:
        """tn93's JSON summary of this run, byte for byte (tn93g_summary_json)."""
        lib = load_library()
        n = lib.tn93g_summary_json(C.byref(self.raw), n1, n2, int(second_file), int(fst), None, 0)
        buf = C.create_string_buffer(n + 1)
        lib.tn93g_summary_json(C.byref(self.raw), n1, n2, int(second_file), int(fst), buf, n + 1)
        return buf.raw[:n]


class Tn93Error(RuntimeError):
    pass


class FastaError(Tn93Error):
    """The FASTA reader refused the input; str(e) is the message tn93 prints (it then exits with status 1)."""


class HostAlignment:
    """An alignment from arrays (codes uint8 [n, L] in 0..17, names, copy numbers), laid out as tn93g_alignment
    for the batch and server calls (the arrays are kept alive by this object)."""

    def __init__(self, codes: np.ndarray, names, counts=None):
        self._codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self.n, self.L = self._codes.shape
        nb = [x.encode() if isinstance(x, str) else bytes(x) for x in names]
        self._names = C.create_string_buffer(b"".join(nb) + b"\0")
        self._off = np.zeros(self.n, dtype=np.uint64)
        if self.n > 1:
            self._off[1:] = np.cumsum([len(b) for b in nb[:-1]])
        self._len = np.array([len(b) for b in nb], dtype=np.int64)
        self._cnt = (np.ones(self.n, dtype=np.int64) if counts is None
                     else np.ascontiguousarray(counts, dtype=np.int64))
        a = _Alignment()
        a.codes = self._codes.ctypes.data_as(C.POINTER(C.c_uint8))
        a.n, a.L = self.n, self.L
        a.copy_counts = self._cnt.ctypes.data_as(C.POINTER(C.c_long))
        a.names = C.cast(self._names, C.POINTER(C.c_char))
        a.name_off = self._off.ctypes.data_as(C.POINTER(C.c_size_t))
        a.name_len = self._len.ctypes.data_as(C.POINTER(C.c_long))
        self._a = a


class Fasta:
    """A FASTA file parsed by tn93's reader (tn93g_read_fasta): codes, names, copy numbers in host memory."""

    def __init__(self, data: bytes, expect_len: int = 0, counts_sep: str = ":"):
        lib = load_library()
        self._a = _Alignment()
        msg = C.create_string_buffer(512)
        rc = lib.tn93g_read_fasta(data, len(data), int(expect_len), counts_sep.encode()[:1], C.byref(self._a), msg,
                                  512)
        if rc == -9:
            raise FastaError(msg.value.decode(errors="replace"))
        if rc != 0:
            raise Tn93Error(f"tn93g error {rc}: {lib.tn93g_strerror(rc).decode()}")
        self.n, self.L = self._a.n, self._a.L

    @property
    def codes(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._a.codes, shape=(self.n * self.L,)).reshape(self.n, self.L).copy()

    @property
    def counts(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._a.copy_counts, shape=(self.n,)).copy()

    @property
    def names(self) -> list:
        off = np.ctypeslib.as_array(self._a.name_off, shape=(self.n,))
        ln = np.ctypeslib.as_array(self._a.name_len, shape=(self.n,))
        return [C.string_at(C.addressof(self._a.names.contents) + int(o), int(k)) for o, k in zip(off, ln)]

    def __del__(self):
        try:
            if self._a.codes:
                load_library().tn93g_alignment_free(C.byref(self._a))
        except Exception:  # noqa: BLE001
            pass


@dataclass
class DeviceSet:
    """An alignment resident on the device (tn93g_upload)."""
    handle: C.c_void_p
    N: int
    L: int


class Engine:
    """One engine context on a CUDA device (tn93g_create)."""

    STAGES = ("pack", "pair", "replay", "rows", "write", "d2h", "total", "count")

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = load_library()
        self.ctx = C.c_void_p()
        self._servers = weakref.WeakSet()  # servers on this context: destroyed before it
        self._check(self.lib.tn93g_create(C.byref(self.ctx), device, hbm_budget))

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.tn93g_strerror(rc).decode()
            if getattr(self, "ctx", None):
                msg += ": " + (self.lib.tn93g_last_cuda_error(self.ctx) or b"").decode()
            raise Tn93Error(f"tn93g error {rc}: {msg}")

    def upload(self, codes, names=None, counts=None):
        """tn93g_upload: an alignment from arrays (codes uint8 [N, L], names, copy numbers), or a prepared
        HostAlignment / Fasta, whose encoded names and offsets are then used as they are (no per-call encoding)."""
        if isinstance(codes, (HostAlignment, Fasta)):
            a = codes._a
            s = C.c_void_p()
            self._check(self.lib.tn93g_upload(self.ctx, C.byref(s), C.cast(a.codes, C.c_void_p), a.n, a.L,
                                              C.cast(a.copy_counts, C.c_void_p), C.cast(a.names, C.c_void_p),
                                              C.cast(a.name_off, C.c_void_p), C.cast(a.name_len, C.c_void_p)))
            return DeviceSet(s, a.n, a.L)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        N, L = codes.shape
        nb = [n.encode() if isinstance(n, str) else bytes(n) for n in names]
        blob = b"".join(nb) or b"\0"
        off = np.zeros(N, dtype=np.uint64)
        if N > 1:
            off[1:] = np.cumsum([len(b) for b in nb[:-1]])
        ln = np.array([len(b) for b in nb], dtype=np.int64)
        cnt = np.ones(N, dtype=np.int64) if counts is None else np.ascontiguousarray(counts, dtype=np.int64)
        s = C.c_void_p()
        self._check(self.lib.tn93g_upload(self.ctx, C.byref(s), codes.ctypes.data, N, L, cnt.ctypes.data, blob,
                                          off.ctypes.data, ln.ctypes.data))
        return DeviceSet(s, N, L)

    def upload_fasta(self, data: bytes, expect_len: int = 0, counts_sep: str = ":") -> DeviceSet:
        """tn93g_upload_fasta: a FASTA file's bytes read into a set on the device (the byte map and compression run
        on the GPU), with tn93g_read_fasta's rules and messages (FastaError)."""
        s = C.c_void_p()
        n, L = C.c_long(), C.c_long()
        msg = C.create_string_buffer(512)
        rc = self.lib.tn93g_upload_fasta(self.ctx, C.byref(s), data, len(data), int(expect_len),
                                         counts_sep.encode()[:1], C.byref(n), C.byref(L), msg, 512)
        if rc == -9:
            raise FastaError(msg.value.decode(errors="replace"))
        self._check(rc)
        return DeviceSet(s, n.value, L.value)

    def free(self, s: DeviceSet):
        self.lib.tn93g_free_set(self.ctx, s.handle)
        s.handle = C.c_void_p()

    def run(self, s: DeviceSet, opts: Options, n1: int | None = None, sink=None):
        """Runs all pairs of set s. sink(bytes) receives the distance file in order; when sink is None the bytes are
        collected and returned; sink="discard" leaves them in the engine's pinned host buffer (no callback)."""
        chunks = []

        def _sink(_user, ptr, n):
            try:
                mv = C.string_at(ptr, n)
                if sink is None:
                    chunks.append(mv)
                else:
                    sink(mv)
                return 0
            except Exception:  # noqa: BLE001 - an exception must not unwind through C
                return 1

        cb = _SINK() if (isinstance(sink, str) and sink == "discard") else _SINK(_sink)
        o = opts.to_c()
        S = _Summary()
        if n1 is None:
            n1 = s.N
        self._check(self.lib.tn93g_run(self.ctx, s.handle, int(n1), C.byref(o), cb, None, C.byref(S)))
        return b"".join(chunks), self._summary(S)

    def run_rows(self, s: DeviceSet, opts: Options, row_begin: int, row_end: int, n1: int | None = None):
        """tn93g_run_rows: the rows [row_begin, row_end) only. Returns (text bytes of those rows, Summary of their
        pairs, per-row sums as a float64 array [rows, 6]: sums of bins 0-2, then weights of bins 0-2)."""
        chunks = []

        def _sink(_user, ptr, n):
            try:
                chunks.append(C.string_at(ptr, n))
                return 0
            except Exception:  # noqa: BLE001 - an exception must not unwind through C
                return 1

        cb = _SINK(_sink)
        o = opts.to_c()
        S = _Summary()
        rows = np.zeros((max(0, row_end - row_begin), 6), dtype=np.float64)
        self._check(self.lib.tn93g_run_rows(self.ctx, s.handle, int(s.N if n1 is None else n1), C.byref(o),
                                            int(row_begin), int(row_end), cb, None, rows.ctypes.data, C.byref(S)))
        return b"".join(chunks), self._summary(S), rows

    def run_to_device(self, s: DeviceSet, opts: Options, n1: int | None = None):
        """Runs all pairs with the distance file left in HBM; returns (device pointer, nbytes, Summary)."""
        o = opts.to_c()
        S = _Summary()
        ptr, nb = C.c_void_p(), C.c_size_t()
        self._check(self.lib.tn93g_run_to_device(self.ctx, s.handle, int(s.N if n1 is None else n1), C.byref(o),
                                                 C.byref(ptr), C.byref(nb), C.byref(S)))
        return ptr.value, nb.value, self._summary(S)

    def batch_run(self, alignments: list, opts: list, rows_per_warp=None, pair_blocks: int = 0,
                  sink=None) -> list:
        """tn93g_batch_run: many alignments (HostAlignment or Fasta objects), each with its own Options, in one pass.
        Returns [(body bytes, Summary)], each equal to run() on that alignment alone. sink="discard" leaves the
        texts in the engine's pinned host buffer (bodies are returned empty)."""
        K = len(alignments)
        arr = (_Alignment * K)(*[a._a for a in alignments])
        oc = (_Opts * K)(*[o.to_c() for o in opts])
        rpw = None if rows_per_warp is None else (C.c_int * K)(*[int(x) for x in rows_per_warp])
        sums = (_Summary * K)()
        bodies = [[] for _ in range(K)]

        def _sink(_user, k, ptr, n):
            try:
                bodies[k].append(C.string_at(ptr, n))
                return 0
            except Exception:  # noqa: BLE001 - an exception must not unwind through C
                return 1

        cb = _QSINK() if (isinstance(sink, str) and sink == "discard") else _QSINK(_sink)
        self._check(self.lib.tn93g_batch_run(self.ctx, K, arr, oc, rpw, int(pair_blocks), cb, None, sums))
        out = []
        for k in range(K):
            S = _Summary()
            C.memmove(C.byref(S), C.byref(sums[k]), C.sizeof(_Summary))
            out.append((b"".join(bodies[k]), _plain_summary(S)))
        return out

    def set_log_band(self, band_ulps: float, spread_ulps: float = 1.0):
        """Widens the logarithm's ambiguity band (0.03 to 0.5 ulp) and its candidate distance (>= 1 ulp): a test knob
        that drives pairs through the undecided path; results stay exact (tn93g_set_log_band)."""
        self._check(self.lib.tn93g_set_log_band(self.ctx, float(band_ulps), float(spread_ulps)))

    def set_exact_sums(self, on: bool):
        """Every pair with an ambiguous logarithm finished with the C library's log (tn93g_set_exact_sums)."""
        self._check(self.lib.tn93g_set_exact_sums(self.ctx, int(bool(on))))

    def set_wait_limit(self, seconds: float):
        """Limit of each bounded device wait (tn93g_set_wait_limit)."""
        self._check(self.lib.tn93g_set_wait_limit(self.ctx, float(seconds)))

    def selftest_division(self, n: int, seed: int) -> tuple:
        """(formula inputs, quotients) whose device results differ from the host's IEEE division or the device's own
        correctly rounded division (tn93g_selftest_division)."""
        m = (C.c_long * 2)()
        self._check(self.lib.tn93g_selftest_division(self.ctx, int(n), int(seed), m))
        return m[0], m[1]

    def inject_fault(self, fault: int):
        """A TN93G_FAULT_* for the next run only (tn93g_inject_fault)."""
        self._check(self.lib.tn93g_inject_fault(self.ctx, int(fault)))

    def run_status(self, s: DeviceSet, opts: Options, n1: int | None = None) -> int:
        """tn93g_run's return code (0 or a negative TN93G_E*), discarding the output: for failure-path tests."""
        o = opts.to_c()
        S = _Summary()
        return self.lib.tn93g_run(self.ctx, s.handle, int(s.N if n1 is None else n1), C.byref(o), _SINK(), None,
                                  C.byref(S))

    def set_count_path(self, path: str):
        """"popc" (CUDA-core bit-plane counts) or "tc" (tcgen05 INT8 tensor-core counts); results are identical."""
        self._check(self.lib.tn93g_set_count_path(self.ctx, {"popc": 0, "tc": 1}[path]))

    def last_timings(self) -> dict:
        """Device milliseconds of the last call's stages (pack, pair, replay, rows, write, d2h, total, and count:
        the tensor-core count kernel, part of pair)."""
        t = (C.c_double * 8)()
        k = self.lib.tn93g_last_timings(self.ctx, t, 8)
        return {self.STAGES[q]: t[q] for q in range(k)}

    @property
    def stream(self) -> int:
        """The engine's cudaStream_t, as an integer (for torch.cuda.ExternalStream)."""
        return self.lib.tn93g_stream(self.ctx) or 0

    def last_launches(self) -> int:
        return self.lib.tn93g_last_launches(self.ctx)

    def _summary(self, S):
        t = (C.c_double * 8)()
        k = self.lib.tn93g_last_timings(self.ctx, t, 8)
        summ = Summary(pairwise=S.pairwise, skipped=S.skipped, links=S.links, max=list(S.max), mean=list(S.mean),
                       weighted=list(S.weighted), hist=_hist(S),
                       pairs_replayed=S.pairs_replayed, logs_ambiguous=S.logs_ambiguous, undecided=S.undecided,
                       output_bytes=S.output_bytes, logs_resolved=S.logs_resolved, sums_repass=bool(S.sums_repass),
                       timings_ms={self.STAGES[q]: t[q] for q in range(k)}, raw=S)
        return summ

    def close(self):
        for srv in list(getattr(self, "_servers", ())):
            srv.close()
        if self.ctx:
            self.lib.tn93g_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def _hist(S) -> np.ndarray:
    return np.frombuffer(bytes(S.hist), dtype=np.uint64).reshape(3, 200).copy()


def _plain_summary(S) -> Summary:
    return Summary(pairwise=S.pairwise, skipped=S.skipped, links=S.links, max=list(S.max), mean=list(S.mean),
                   weighted=list(S.weighted), hist=_hist(S),
                   pairs_replayed=S.pairs_replayed, logs_ambiguous=S.logs_ambiguous, undecided=S.undecided,
                   output_bytes=S.output_bytes, logs_resolved=S.logs_resolved, sums_repass=bool(S.sums_repass), raw=S)


class ResidentReference:
    """A reference alignment kept packed on the device, run against batches of query alignments
    (tn93g_server_*). Each query's result is the distance file body and summary of
    `tn93 -s QUERY.fa REF.fa` with this server's options (rows = reference, columns = the query)."""

    def __init__(self, engine: Engine, ref: Fasta, opts: Options, max_batch_sequences: int = 4096,
                 max_batch_queries: int = 256):
        self.engine, self.lib, self.ref, self.opts = engine, engine.lib, ref, opts
        self.max_batch_sequences, self.max_batch_queries = max_batch_sequences, max_batch_queries
        self.srv = C.c_void_p()
        a = ref._a
        o = opts.to_c()
        engine._check(self.lib.tn93g_server_create(
            engine.ctx, C.byref(self.srv), C.cast(a.codes, C.c_void_p), a.n, a.L, C.cast(a.copy_counts, C.c_void_p),
            C.cast(a.names, C.c_void_p), C.cast(a.name_off, C.c_void_p), C.cast(a.name_len, C.c_void_p),
            C.byref(o), int(max_batch_sequences), int(max_batch_queries)))
        engine._servers.add(self)

    def batch(self, queries: list) -> list:
        """Runs the queries (Fasta objects of the reference's length) in one batch: [(body bytes, Summary)]."""
        nq = len(queries)
        arr = (_Alignment * nq)(*[q._a for q in queries])
        sums = (_Summary * nq)()
        bodies = [[] for _ in range(nq)]

        def _sink(_user, q, ptr, n):
            try:
                bodies[q].append(C.string_at(ptr, n))
                return 0
            except Exception:  # noqa: BLE001 - an exception must not unwind through C
                return 1

        cb = _QSINK(_sink)
        self.engine._check(self.lib.tn93g_server_batch(self.srv, nq, arr, cb, None, sums))
        out = []
        for q in range(nq):
            S = _Summary()
            C.memmove(C.byref(S), C.byref(sums[q]), C.sizeof(_Summary))
            out.append((b"".join(bodies[q]), _plain_summary(S)))
        return out

    def last_timings(self) -> dict:
        """Device milliseconds of the last batch per stage (pack, pair, replay, rows, write, d2h, total)."""
        t = (C.c_double * 7)()
        k = self.lib.tn93g_last_timings(self.engine.ctx, t, 7)
        return {Engine.STAGES[q]: t[q] for q in range(k)}

    def close(self):
        # a server lives inside its engine's context: it is destroyed first (Engine.close does so as well)
        if self.srv and self.engine.ctx:
            self.lib.tn93g_server_destroy(self.srv)
        self.srv = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
