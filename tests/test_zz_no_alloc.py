"""The allocation-free entry point, tn93g_pair_distances_noalloc, for callers that cannot allocate device
memory (a host application whose own allocator owns the device, or a loop that must not enter the driver's
allocator). The test is the caller: it allocates the input and output buffers itself (with torch) and calls the
entry point through the C ABI; the engine allocates nothing.

Each call's distances, turned into tn93's text exactly as tn93g_run does (clamp at 0, -t/-w link test,
printf %g), must equal tn93g_run's distance file byte for byte, on two calls in a row (the fixed scratch keeps
the previous call's contents, which must not leak into the next result). This file is named so that pytest
collects it last."""
import ctypes as C

import numpy as np
import pytest

from tests.conftest import REPO

pytestmark = pytest.mark.gpu

SKIP_BITS = 0x7FF4000000000BAD


def _lib():
    from swifttn93_b200 import _Opts, load_library

    lib = load_library()
    lib.tn93g_pair_distances_noalloc.restype = C.c_int
    lib.tn93g_pair_distances_noalloc.argtypes = [C.c_void_p, C.c_long, C.c_long, C.POINTER(_Opts), C.c_void_p,
                                                 C.c_void_p]
    lib.tn93g_noalloc_last_error.restype = C.c_char_p
    return lib


def _expected_text(names, dist, opts):
    """tn93's csv lines from raw distances, in row-major pair order (the same rules the row kernel applies)."""
    n = len(names)
    bits = dist.view(np.uint64)
    out = []
    for i in range(n - 1):
        for j in range(i + 1, n):
            if int(bits[i, j]) == SKIP_BITS:
                continue
            d = float(dist[i, j])
            t = 0.0 if d <= 0.0 else d
            if opts.min_distance <= t <= opts.threshold:
                out.append(f"{names[i]},{names[j]},{'%g' % t}\n")
    return "".join(out).encode()


def _workloads():
    from swifttn93_b200 import synth
    from tests import cases

    names, codes = synth.plain_small()
    yield "plain_small_300_resolve", names[:300], codes[:300], dict(threshold=0.03, mode="resolve",
                                                                    resolve_fraction=0.05, min_overlap=500)
    yield "plain_small_300_gapmm", names[:300], codes[:300], dict(threshold=0.05, mode="gapmm", min_overlap=100)
    # real HIV-1 pol sequences carry three-fold codes: non-dyadic pairs take the site-order replay
    fa = cases.source_bytes("real:hiv_dev")[0].split(b">")[1:401]
    nm = [r.split(b"\n", 1)[0].decode() for r in fa]
    seqs = [r.split(b"\n", 1)[1].replace(b"\n", b"") for r in fa]
    lut = np.full(256, 255, dtype=np.uint8)
    for k, ch in enumerate(synth.ALPHABET):
        lut[ch] = k
        lut[ord(chr(ch).lower())] = k
    codes2 = np.stack([lut[np.frombuffer(s, dtype=np.uint8)] for s in seqs])
    assert codes2.max() <= 17
    yield "real_hiv_400_average", nm, codes2, dict(threshold=0.05, mode="average", min_overlap=500)


def test_noalloc_matches_run_two_calls_in_a_row():
    import torch

    from swifttn93_b200 import Engine, Options

    lib = _lib()
    eng = Engine()
    for tag, names, codes, kw in _workloads():
        opts = Options(**kw)
        s = eng.upload(codes, names)
        body, _ = eng.run(s, opts)
        eng.free(s)
        n, L = codes.shape
        d_codes = torch.from_numpy(np.ascontiguousarray(codes)).cuda()
        for call in range(2):
            d_dist = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            o = opts.to_c()
            rc = lib.tn93g_pair_distances_noalloc(d_codes.data_ptr(), n, L, C.byref(o), d_dist.data_ptr(), None)
            assert rc == 0, (tag, rc, lib.tn93g_noalloc_last_error())
            got = _expected_text(names, d_dist.cpu().numpy(), opts)
            assert got == body, (tag, call, len(got), len(body))
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from swifttn93_b200 import Options

    lib = _lib()
    o = Options().to_c()
    d = torch.zeros(16, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    assert lib.tn93g_pair_distances_noalloc(d.data_ptr(), 513, 10, C.byref(o), out.data_ptr(), None) == -8
    assert b"N <= 512" in lib.tn93g_noalloc_last_error()
    assert lib.tn93g_pair_distances_noalloc(d.data_ptr(), 10, 4097, C.byref(o), out.data_ptr(), None) == -8
