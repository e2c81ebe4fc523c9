"""Seeded synthetic alignments shaped like the benchmark workloads of the all-pairs TN93 path.

No public benchmark data is used: every workload is simulated from a fixed seed.

  plain_small      500 x 1,300: coalescent tree, 4% mean pairwise divergence, TN93 rates (kappa_R 6,
                   kappa_Y 9), base frequencies A .39 C .17 G .23 T .21, 0.5% two-fold IUPAC codes, 0.05% N,
                   0.3 gap runs of length 1-30 per sequence, ragged 5'/3' ends of 0-80 columns.
  hiv_bench        6,700 x 1,500: as plain_small, with 40 transmission clusters of 5-60 sequences at 0.2-1.2%
                   intra-cluster divergence over a 6% background; ambiguity 1% (4% of sequences carry 3-5%).
  long_n_runs      2,000 x 29,900: base frequencies .30/.18/.20/.32, 0.1% mean divergence on a star-like
                   tree, N runs of 50-400 at 3 per sequence, leading/trailing N blocks up to 300 columns,
                   0.02% two-fold IUPAC codes.
  batch(i)         alignment i of the batched workload: N log-uniform in [50, 4000], L uniform in [900, 3000],
                   generated as hiv_bench from seed base + i.
  serve_reference  30,000 x 1,500 generated as hiv_bench; queries derive from random reference sequences at
                   0.5-3% divergence with 1% ambiguity.

Sequences are returned as uint8 codes 0..17 in the order "ACGTURYSWKMBDHVN?-" (the tn93 alphabet) together
with their names, and can be rendered as FASTA bytes for the command-line front end.
"""
from __future__ import annotations

import numpy as np

ALPHABET = b"ACGTURYSWKMBDHVN?-"
CODE = {c: i for i, c in enumerate(ALPHABET)}
TWOFOLD = np.array([CODE[c] for c in b"RYKMSW"], dtype=np.uint8)
N_CODE, GAP_CODE = 15, 17


def tn93_rate_matrix(pi, kappa_r=6.0, kappa_y=9.0):
    """TN93 generator over A,C,G,T (purine transitions A<->G at kappa_r, pyrimidine C<->T at kappa_y,
    transversions at 1), scaled to one expected substitution per unit time."""
    pi = np.asarray(pi, dtype=np.float64)
    pi = pi / pi.sum()
    Q = np.zeros((4, 4))
    for a in range(4):
        for b in range(4):
            if a == b:
                continue
            k = kappa_r if {a, b} == {0, 2} else kappa_y if {a, b} == {1, 3} else 1.0
            Q[a, b] = k * pi[b]
    Q[np.diag_indices(4)] = -Q.sum(axis=1)
    Q /= -(pi * np.diag(Q)).sum()
    return Q, pi


class _Evolver:
    """Transition probabilities exp(Qt) through the eigen-decomposition of the symmetrised generator."""

    def __init__(self, Q, pi):
        s = np.sqrt(pi)
        S = (s[:, None] * Q) / s[None, :]
        S = (S + S.T) / 2
        self.w, V = np.linalg.eigh(S)
        self.left = V / s[:, None]
        self.right = V.T * s[None, :]

    def P(self, t):
        P = (self.left * np.exp(self.w * t)) @ self.right
        P = np.clip(P, 0.0, None)
        return P / P.sum(axis=1, keepdims=True)

    def evolve(self, rng, parent, t):
        if t <= 0:
            return parent.copy()
        cum = np.cumsum(self.P(t), axis=1)
        u = rng.random(parent.shape[0])
        return (u[:, None] > cum[parent]).sum(axis=1).astype(np.uint8).clip(0, 3)


def coalescent_tree(rng, n):
    """Kingman coalescent on n leaves. Returns (parent, branch_length) arrays over 2n-1 nodes (root = 2n-2,
    leaves 0..n-1) and the node heights."""
    parent = np.full(2 * n - 1, -1, dtype=np.int64)
    height = np.zeros(2 * n - 1)
    active = list(range(n))
    t, nxt = 0.0, n
    while len(active) > 1:
        k = len(active)
        t += rng.exponential(2.0 / (k * (k - 1)))
        i, j = rng.choice(k, size=2, replace=False)
        a, b = active[i], active[j]
        parent[a] = parent[b] = nxt
        height[nxt] = t
        for idx in sorted((i, j), reverse=True):
            active.pop(idx)
        active.append(nxt)
        nxt += 1
    bl = np.zeros(2 * n - 1)
    for v in range(2 * n - 2):
        bl[v] = height[parent[v]] - height[v]
    return parent, bl, height


def _mean_pairwise_height(rng, parent, height, n, samples=4000):
    """Mean over random leaf pairs of 2 x (height of their most recent common ancestor)."""
    anc = {}

    def path(v):
        if v not in anc:
            p, out = v, []
            while p >= 0:
                out.append(p)
                p = parent[p]
            anc[v] = out
        return anc[v]

    tot = 0.0
    m = min(samples, n * (n - 1) // 2)
    for _ in range(m):
        a, b = rng.choice(n, size=2, replace=False)
        pa = set(path(a))
        for v in path(b):
            if v in pa:
                tot += 2 * height[v]
                break
    return tot / m


def evolve_tree(rng, ev, root, parent, bl, n, scale):
    """Sequences at the n leaves of the tree, evolved from `root` with branch lengths bl * scale."""
    m = parent.shape[0]
    seqs = [None] * m
    seqs[m - 1] = root
    children = [[] for _ in range(m)]
    for v in range(m - 1):
        children[parent[v]].append(v)
    stack = [m - 1]
    while stack:
        v = stack.pop()
        for c in children[v]:
            seqs[c] = ev.evolve(rng, seqs[v], bl[c] * scale)
            stack.append(c)
    return [seqs[i] for i in range(n)]


def tree_sample(rng, ev, root, n, divergence):
    """n sequences on a coalescent tree whose mean pairwise divergence is `divergence` substitutions/site."""
    if n == 1:
        return [root.copy()]
    parent, bl, height = coalescent_tree(rng, n)
    mph = _mean_pairwise_height(rng, parent, height, n)
    return evolve_tree(rng, ev, root, parent, bl, n, divergence / mph)


def _decorate(rng, seqs, L, iupac_rate, n_rate, gap_runs=0.3, gap_max=30, ragged=80, high_ambig=None):
    """IUPAC two-fold codes, N, internal gap runs and ragged ends, in that order."""
    out = []
    for s in seqs:
        s = s.copy()
        rate = iupac_rate
        if high_ambig is not None and rng.random() < high_ambig[0]:
            rate = rng.uniform(high_ambig[1], high_ambig[2])
        hit = np.nonzero(rng.random(L) < rate)[0]
        s[hit] = TWOFOLD[rng.integers(0, 6, hit.size)]
        if n_rate > 0:
            s[rng.random(L) < n_rate] = N_CODE
        for _ in range(rng.poisson(gap_runs)):
            ln = int(rng.integers(1, gap_max + 1))
            st = int(rng.integers(0, max(1, L - ln)))
            s[st:st + ln] = GAP_CODE
        if ragged:
            a, b = int(rng.integers(0, ragged + 1)), int(rng.integers(0, ragged + 1))
            s[:a] = GAP_CODE
            if b:
                s[L - b:] = GAP_CODE
        out.append(s)
    return out


def _root(rng, L, pi):
    return rng.choice(4, size=L, p=np.asarray(pi) / np.sum(pi)).astype(np.uint8)


def _names(tag, seed, n):
    return [f"{tag}_{seed}_{i:06d}" for i in range(n)]


def plain_small(seed=1, n=500, L=1300):
    rng = np.random.default_rng(seed)
    pi = (0.39, 0.17, 0.23, 0.21)
    Q, pi = tn93_rate_matrix(pi)
    ev = _Evolver(Q, pi)
    seqs = tree_sample(rng, ev, _root(rng, L, pi), n, 0.04)
    seqs = _decorate(rng, seqs, L, 0.005, 0.0005)
    return _names("cfg0", seed, n), np.stack(seqs)


def hiv_bench(seed=2, n=6700, L=1500, clusters=40, tag="cfg1"):
    """Background coalescent at 6% plus `clusters` transmission clusters of 5-60 sequences at 0.2-1.2%."""
    rng = np.random.default_rng(seed)
    pi = (0.39, 0.17, 0.23, 0.21)
    Q, pi = tn93_rate_matrix(pi)
    ev = _Evolver(Q, pi)
    clusters = min(clusters, max(0, n // 10))
    sizes = [int(rng.integers(5, 61)) for _ in range(clusters)]
    while sum(sizes) > n // 2 and sizes:
        sizes.pop()
    n_bg = n - sum(sizes)
    founders_and_bg = tree_sample(rng, ev, _root(rng, L, pi), n_bg + len(sizes), 0.06)
    seqs = founders_and_bg[:n_bg]
    for k, sz in enumerate(sizes):
        seqs += tree_sample(rng, ev, founders_and_bg[n_bg + k], sz, rng.uniform(0.002, 0.012))
    order = rng.permutation(n)
    seqs = [seqs[i] for i in order]
    seqs = _decorate(rng, seqs, L, 0.01, 0.0005, high_ambig=(0.04, 0.03, 0.05))
    return _names(tag, seed, n), np.stack(seqs)


def long_n_runs(seed=3, n=2000, L=29900):
    rng = np.random.default_rng(seed)
    pi = (0.30, 0.18, 0.20, 0.32)
    Q, pi = tn93_rate_matrix(pi)
    ev = _Evolver(Q, pi)
    root = _root(rng, L, pi)
    # star-like tree: every sequence on its own branch from the root, 0.1% mean pairwise divergence
    seqs = [ev.evolve(rng, root, rng.exponential(0.0005)) for _ in range(n)]
    seqs = _decorate(rng, seqs, L, 0.0002, 0.0, gap_runs=0.0, ragged=0)
    out = []
    for s in seqs:
        for _ in range(rng.poisson(3)):
            ln = int(rng.integers(50, 401))
            st = int(rng.integers(0, L - ln))
            s[st:st + ln] = N_CODE
        a, b = int(rng.integers(0, 301)), int(rng.integers(0, 301))
        s[:a] = N_CODE
        if b:
            s[L - b:] = N_CODE
        out.append(s)
    return _names("cfg2", seed, n), np.stack(out)


BATCH_MODES = ("resolve", "average", "gapmm", "skip")


def batch_spec(i, base_seed=1000):
    """Shape and options of alignment i of the batched workload (96 alignments)."""
    rng = np.random.default_rng(base_seed + i)
    n = int(round(np.exp(rng.uniform(np.log(50), np.log(4000)))))
    L = int(rng.integers(900, 3001))
    t = float(rng.uniform(0.005, 0.02))
    mode = BATCH_MODES[int(rng.integers(0, 3))]
    return dict(n=n, L=L, threshold=t, mode=mode, seed=base_seed + i)


def batch_alignment(i, base_seed=1000):
    sp = batch_spec(i, base_seed)
    names, codes = hiv_bench(seed=sp["seed"], n=sp["n"], L=sp["L"], clusters=max(1, sp["n"] // 170),
                             tag=f"cfg3a{i:02d}")
    return sp, names, codes


def serve_reference(seed=4, n=30000, L=1500):
    return hiv_bench(seed=seed, n=n, L=L, clusters=180, tag="cfg4r")


def serve_query(rng, ref_codes, q, seed_tag):
    """A query of q sequences, each derived from a random reference sequence at 0.5-3% divergence with 1%
    two-fold ambiguity codes."""
    L = ref_codes.shape[1]
    pi = (0.39, 0.17, 0.23, 0.21)
    Q, pi = tn93_rate_matrix(pi)
    ev = _Evolver(Q, pi)
    out = []
    for _ in range(q):
        src = ref_codes[int(rng.integers(0, ref_codes.shape[0]))].copy()
        clean = src < 4
        evolved = ev.evolve(rng, np.where(clean, src, 0).astype(np.uint8), rng.uniform(0.005, 0.03))
        s = np.where(clean, evolved, src).astype(np.uint8)
        hit = np.nonzero((rng.random(L) < 0.01) & (s < 4))[0]
        s[hit] = TWOFOLD[rng.integers(0, 6, hit.size)]
        out.append(s)
    return [f"q{seed_tag}_{i:04d}" for i in range(q)], np.stack(out)


def to_fasta(names, codes, wrap=0) -> bytes:
    """FASTA bytes of the alignment (uppercase letters, '-' for gaps)."""
    lut = np.frombuffer(ALPHABET, dtype=np.uint8)
    parts = []
    for nm, row in zip(names, codes):
        s = lut[row].tobytes()
        parts.append(b">" + nm.encode() + b"\n")
        if wrap:
            parts.extend(s[k:k + wrap] + b"\n" for k in range(0, len(s), wrap))
        else:
            parts.append(s + b"\n")
    return b"".join(parts)


WORKLOADS = {
    "plain_small": plain_small,
    "hiv_bench": hiv_bench,
    "long_n_runs": long_n_runs,
}
