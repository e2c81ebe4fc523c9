// engine.cu -- sm_100a kernels of the all-pairs TN93 engine and the C ABI of include/tn93g.h.
//
// One run (tn93g_run) is a pipeline over bands of rows:
//   pack      colscan_kernel, pack_kernel, events_kernel, transpose_kernel: constant-column fold, bit planes,
//             compressed codes and sparse event lists (replaces Engine::prepare, swifttn93.cpp:570-1044)
//   pair      pair_kernel: per pair the clean-site counts by AND/XOR + POPC over 64-column plane words, the
//             N-plane cross counts, the sparse ambiguity events through the x16 tables, tn93's -l / -g
//             decisions, the TN93 formula in FP64 and the log certificate; writes the raw distance
//             (replaces kernel8/kernel16/kernelW/sparse_*/phaseA/tail8, swifttn93.cpp:1241-2170)
//   replay    replay_kernel: pairs with a contribution that is not a multiple of 1/16 are recomputed by a
//             site-order walk with tn93's float sums (replaces replay/ordered, swifttn93.cpp:1050-1232)
//   rows      stats_kernel (per row segment: histogram, links, skipped pairs, maxima, text length) and
//             sum_kernel (per row, the FP64 sums in tn93's column order) (phase C, swifttn93.cpp:2479-2604)
//   write     write_kernel: the distance-file text of the band at scanned segment offsets (the ordered writer,
//             swifttn93.cpp:2811-2858, and fastfmt)
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <math.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "tc_count.cuh"
#include "tn93g.h"

namespace tn93 {
void build_log_table(LogTable *T);
}

using namespace tn93;

namespace {

constexpr int kWarps = 8;  // warps per block of the pair / row kernels

__device__ __forceinline__ int popc(uint64_t x) { return __popcll(x); }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

__device__ __forceinline__ bool sparse_code(int c, bool wplane) { return c >= 4 && c < 17 && !(wplane && c == 15); }

//------------------------------------------------------------------------------------------------ pack
// Each packing kernel's body takes its block coordinates as arguments, so that a batch of alignments can run one
// launch for all of them (the *_batch_kernel forms below map each block to its alignment and local block).

// per column: the set of codes seen (bit c), per launch the number of N codes; block (bx, by) covers 256 columns
// of 64 sequences
__device__ __forceinline__ void colscan_body(const uint8_t *__restrict__ codes, long N, long L, uint32_t *seen,
                                             unsigned long long *nN, long bx, long by)
{
  const long p = bx * 256l + threadIdx.x;
  const long i0 = by * 64l, i1 = min(N, i0 + 64);
  uint32_t m = 0;
  unsigned cn = 0;
  if (p < L)
    for (long i = i0; i < i1; i++) {
      const unsigned c = codes[i * L + p];
      m |= 1u << c;
      cn += c == 15;
    }
  if (p < L && m) atomicOr(&seen[p], m);
  for (int o = 16; o; o >>= 1) cn += __shfl_xor_sync(0xffffffffu, cn, o);
  if ((threadIdx.x & 31) == 0 && cn) atomicAdd(nN, (unsigned long long)cn);
}

__global__ void colscan_kernel(const uint8_t *__restrict__ codes, long N, long L, uint32_t *seen,
                               unsigned long long *nN)
{
  colscan_body(codes, N, L, seen, nN, blockIdx.x, blockIdx.y);
}

// one warp per (sequence, 64-column word): bit planes, compressed codes, sparse event counts; block bx covers 8
// sequences, and the words w0, w0 + wstep, ...
__device__ __forceinline__ void pack_body(const PackArgs &a, long bx, long w0, long wstep)
{
  const int lane = threadIdx.x & 31;
  const long i = bx * (long)kWarps + (threadIdx.x >> 5);
  if (i >= a.N) return;
  for (long w = w0; w < a.W; w += wstep) {
  const long k0 = w * 64 + lane, k1 = k0 + 32;
  const int c0 = k0 < a.Lc ? a.codes[i * a.L + a.varcol[k0]] : 17;
  const int c1 = k1 < a.Lc ? a.codes[i * a.L + a.varcol[k1]] : 17;
  if (k0 < a.Lc) a.cc[i * a.Lc + k0] = (uint8_t)c0;
  if (k1 < a.Lc) a.cc[i * a.Lc + k1] = (uint8_t)c1;
  auto both = [&](bool p0, bool p1) -> uint64_t {
    return (uint64_t)__ballot_sync(0xffffffffu, p0) | ((uint64_t)__ballot_sync(0xffffffffu, p1) << 32);
  };
  const uint64_t clean = both(c0 < 4, c1 < 4);
  const uint64_t hi = both(c0 < 4 && (c0 & 1), c1 < 4 && (c1 & 1));
  const uint64_t lo = both(c0 < 4 && (c0 & 2), c1 < 4 && (c1 & 2));
  const bool g0 = k0 < a.Lc && c0 == 17, g1 = k1 < a.Lc && c1 == 17;
  const uint64_t wn = a.wplane ? both(c0 == 15 || (a.gapmm && g0), c1 == 15 || (a.gapmm && g1)) : 0;
  const uint64_t gp = a.gapmm ? both(g0, g1) : 0;
  const uint64_t sp = both(sparse_code(c0, a.wplane), sparse_code(c1, a.wplane));
  if (lane == 0) {
    uint64_t *P = a.planes + (size_t)w * a.NP * a.Npad + i;
    P[0] = hi;
    P[a.Npad] = lo;
    P[2 * a.Npad] = clean;
    P[3 * a.Npad] = wn;
    if (a.NP > 4) P[4 * a.Npad] = gp;
    if (sp) atomicAdd(&a.evcount[i], (unsigned)popc(sp));
  }
  }
}

__global__ void pack_kernel(PackArgs a) { pack_body(a, blockIdx.x, blockIdx.y, gridDim.y); }

// one thread per sequence: how many of its N-plane words (plane 3 of each word) are nonzero
__global__ void wcount_kernel(const uint64_t *planes, long N, long W, int NP, long Npad, uint32_t *wcount)
{
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  uint32_t n = 0;
  for (long w = 0; w < W; w++) n += planes[((size_t)w * NP + 3) * Npad + i] != 0;
  wcount[i] = n;
}

// one thread per sequence: the indices of its nonzero N-plane words, in order, from wl_off[i]
__global__ void wlist_kernel(const uint64_t *planes, long N, long W, int NP, long Npad, const uint32_t *wl_off,
                             uint32_t *wl)
{
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  uint32_t o = wl_off[i];
  for (long w = 0; w < W; w++)
    if (planes[((size_t)w * NP + 3) * Npad + i] != 0) wl[o++] = (uint32_t)w;
}

// one warp per sequence: its sparse events in site order (block bx: 8 sequences)
__device__ __forceinline__ void events_body(const PackArgs &a, long bx)
{
  const int lane = threadIdx.x & 31;
  const long i = bx * (long)kWarps + (threadIdx.x >> 5);
  if (i >= a.N) return;
  uint32_t off = a.ev_off[i];
  const uint8_t *row = a.cc + i * a.Lc;
  for (long w = 0; w < a.W; w++) {
    const long k0 = w * 64 + lane, k1 = k0 + 32;
    const int c0 = k0 < a.Lc ? row[k0] : 17, c1 = k1 < a.Lc ? row[k1] : 17;
    const bool s0 = sparse_code(c0, a.wplane), s1 = sparse_code(c1, a.wplane);
    const unsigned b0 = __ballot_sync(0xffffffffu, s0), b1 = __ballot_sync(0xffffffffu, s1);
    if (s0) a.ev[off + __popc(b0 & lanemask_lt())] = ((uint32_t)k0 << 5) | (uint32_t)c0;
    if (s1) a.ev[off + __popc(b0) + __popc(b1 & lanemask_lt())] = ((uint32_t)k1 << 5) | (uint32_t)c1;
    off += __popc(b0) + __popc(b1);
  }
}

__global__ void events_kernel(PackArgs a) { events_body(a, blockIdx.x); }

// ccT[k][i] = cc[i][k] (padding sequences read as gaps); block (bx, by) of 32 x 8 threads: 32 columns x 32 sequences
__device__ __forceinline__ void transpose_body(const uint8_t *__restrict__ cc, uint8_t *ccT, long N, long Lc, long Npad,
                                               long bx, long by)
{
  __shared__ uint8_t tile[32][33];
  const long k0 = bx * 32l, i0 = by * 32l;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += 8) {
    const long i = i0 + r, k = k0 + tx;
    tile[r][tx] = (i < N && k < Lc) ? cc[i * Lc + k] : (uint8_t)17;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long k = k0 + r, i = i0 + tx;
    if (k < Lc && i < Npad) ccT[k * Npad + i] = tile[tx][r];
  }
}

__global__ void transpose_kernel(const uint8_t *__restrict__ cc, uint8_t *ccT, long N, long Lc, long Npad)
{
  transpose_body(cc, ccT, N, Lc, Npad, blockIdx.x, blockIdx.y);
}

//------------------------------------------------------------------------------------------------ pair
// powers of ten for the certificate's fast test
__device__ __constant__ double kP10[12] = {1e-5, 1e-4, 1e-3, 1e-2, 1e-1, 1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6};
__device__ __constant__ double kScale[11] = {1e10, 1e9, 1e8, 1e7, 1e6, 1e5, 1e4, 1e3, 1e2, 1e1, 1e0};

// Do lo <= hi print the same six significant digits? Fast test: scale both into [1e5, 1e6) and require the same
// integer part with both fractions clear of 1/2 by 1e-4 (the scaled doubles are within 1e-9 of the exact scaled
// values). Returns -1 when the test cannot decide (then the caller compares the printed strings).
__device__ __forceinline__ int same_g_fast(double lo, double hi)
{
  if (!(lo >= 1e-5 && hi < 1e5)) return -1;
  int X = 0;
#pragma unroll
  for (int k = 1; k < 10; k++) X += lo >= kP10[k];
  const double s = kScale[X];
  const double ta = __dmul_rn(lo, s), tb = __dmul_rn(hi, s);
  if (!(ta >= 1e5 && tb < 1e6)) return -1;
  const double fa = floor(ta), fb = floor(tb);
  if (fa != fb) return -1;
  const double ra = ta - fa, rb = tb - fb;
  if (rb < 0.4999 || ra > 0.5001) return 1;
  return -1;
}

// Do lo and hi print the same text? The certificate's exact test when the fast one cannot decide; out of line, so
// that the big-number scratch of the decimal conversion lives in its own stack frame, not in its callers'.
__device__ __noinline__ bool same_g_text(double lo, double hi)
{
  char x[24], y[24];
  const int nx = fmt_g(lo, x), ny = fmt_g(hi, y);
  if (nx != ny) return false;
  for (int k = 0; k < nx; k++)
    if (x[k] != y[k]) return false;
  return true;
}

// decision-stability certificate: do the histogram bin, the link decision and the printed text agree for
// every distance the C library's log may lead to?
__device__ bool certified(const Dist &D, const RunConsts &rc)
{
  if (hist_bin(D.lo) != hist_bin(D.hi)) return false;
  const double tlo = D.lo <= 0. ? 0. : D.lo, thi = D.hi <= 0. ? 0. : D.hi;
  const bool llo = tlo >= rc.min_distance && tlo <= rc.threshold;
  const bool lhi = thi >= rc.min_distance && thi <= rc.threshold;
  if (llo != lhi) return false;
  if (!llo && tlo < rc.min_distance && thi > rc.threshold) return false;
  if (llo && rc.emit && tlo != thi) {
    const int f = same_g_fast(tlo, thi);
    if (f >= 0) return f == 1;
    return same_g_text(tlo, thi);
  }
  return true;
}

// Per-lane running totals of the ambiguous pairs' effect on one summary unit (ExactSink::amb): flushed with
// atomics when the unit changes, and warp by warp at the end of a tile.
struct AmbLane {
  int unit;  // -1: empty
  int n;     // ambiguous pairs
  double lo, hi, spread;
};

__device__ __forceinline__ void amb_flush(unsigned long long *acc, int unit, int n, double lo, double hi,
                                          double spread)
{
  unsigned long long *w = acc + 4 * unit;
  atomicMax(&w[0], (unsigned long long)__double_as_longlong(lo));
  atomicMax(&w[1], (unsigned long long)__double_as_longlong(hi));
  atomicAdd(reinterpret_cast<double *>(&w[2]), spread);
  atomicAdd(&w[3], (unsigned long long)n);
}

__device__ __forceinline__ void amb_add(unsigned long long *acc, AmbLane &L, int unit, double lo, double hi, double w)
{
  if (L.unit != unit) {
    if (L.unit >= 0) amb_flush(acc, L.unit, L.n, L.lo, L.hi, L.spread);
    L.unit = unit;
    L.n = 0;
    L.lo = L.hi = L.spread = 0.;
  }
  L.n++;
  L.lo = fmax(L.lo, lo);
  L.hi = fmax(L.hi, hi);
  L.spread += (hi - lo) * w;
}

// all 32 lanes: each unit held by some lane is reduced over the warp and added once
__device__ __forceinline__ void amb_warp_flush(unsigned long long *acc, AmbLane &L)
{
  for (;;) {
    const unsigned act = __ballot_sync(0xffffffffu, L.unit >= 0);
    if (!act) break;
    const int u = __shfl_sync(0xffffffffu, L.unit, __ffs(act) - 1);
    const bool me = L.unit == u;
    double lo = me ? L.lo : 0., hi = me ? L.hi : 0., sp = me ? L.spread : 0.;
    int n = me ? L.n : 0;
    for (int o = 16; o; o >>= 1) {
      lo = fmax(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      sp += __shfl_xor_sync(0xffffffffu, sp, o);
      n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) amb_flush(acc, u, n, lo, hi, sp);
    if (me) L.unit = -1;
  }
}

// histogram bin of pair (i, j) under -m (0 within the first file, 1 within the second, 2 between them)
__device__ __forceinline__ int fst_bin(const RunConsts &rc, long i, long j)
{
  return rc.fst ? (i < rc.n1 ? (j >= rc.n1 ? 2 : 0) : 1) : 0;
}

// The formula and its certificate for exact inputs; returns the raw distance (from the correctly rounded
// logarithms). A pair whose printed bytes or decisions depend on the C library's rounding (or, in resolve-all
// mode, any pair with an ambiguous logarithm) is appended to the undecided list, to be finished with the C
// library's own logarithms; every pair with an ambiguous logarithm widens its summary unit's bounds.
__device__ __forceinline__ double finish_exact(const LogTable &T, const RunConsts &rc, const ExactSink &ex,
                                               const double nf[4], double diag, double ag, double ct, long i, long j,
                                               long colbase, int &namb, int &nund, AmbLane &al)
{
  const Dist D = tn93_distance(T, nf, diag, ag, ct, rc.log_band, rc.log_spread);
  if (D.amb) {
    namb++;
    if (rc.resolve_all || !certified(D, rc)) {
      nund++;
      if (ex.und_list) {
        const unsigned idx = atomicAdd(ex.und_n, 1u);
        if (idx < ex.und_cap) {
          ex.und_list[2 * (size_t)idx] = (unsigned long long)ex.und_k;
          ex.und_list[2 * (size_t)idx + 1] = ((unsigned long long)i << 32) | (unsigned long long)j;
        }
      }
    }
    if (ex.amb) {
      const int unit = ex.colunit ? ex.colunit[j - colbase] : fst_bin(rc, i, j);
      const double w = (double)(ex.counts[i] * ex.counts[j]);
      amb_add(ex.amb, al, unit, D.lo <= 0. ? 0. : D.lo, D.hi <= 0. ? 0. : D.hi, w);
    }
  }
  return D.d;
}

// warp-level total of the per-lane counts, one atomic per warp (all 32 lanes must call it)
__device__ __forceinline__ void count_flags(unsigned long long *counters, int namb, int nund)
{
  for (int o = 16; o; o >>= 1) {
    namb += __shfl_xor_sync(0xffffffffu, namb, o);
    nund += __shfl_xor_sync(0xffffffffu, nund, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (namb) atomicAdd(&counters[0], (unsigned long long)namb);
    if (nund) atomicAdd(&counters[1], (unsigned long long)nund);
  }
}

__device__ __forceinline__ void add_entry(int acc[9], const int32_t *t)
{
#pragma unroll
  for (int q = 0; q < 8; q++) acc[q] += t[q];
  acc[8] |= t[8];
}

// Block tile of the pair kernel: 32 rows x 32 columns, 8 warps. Column-side sparse events are summed with the
// lanes over the tile's rows (warp-uniform event lists, coalesced position-major partner codes) into shared
// memory; then each warp takes 4 of the tile's rows, one at a time, with the lanes over the columns: clean-site
// counts, row-side events (warp-uniform list) and the epilogue.
constexpr int kTile = 32;
constexpr int kRowsPerWarp = kTile / kWarps;
constexpr int kColAccStride = kTile * 9 + 1;  // ints per tile row (+1: conflict-free in both phases)
constexpr int kAggInts = (kSparseCodes * kCodes + 5) * kLanes;
// shared-memory tables of a pair block: the x16 table (unpacked runs), or the packed table and the N-plane entries
constexpr size_t kPackedSmem = sizeof(PackedTables) + 5 * sizeof(AggEntry);
constexpr size_t kTabSmem = ((size_t)kAggInts * 4 > kPackedSmem ? (size_t)kAggInts * 4 : kPackedSmem + 15) / 16 * 16;
constexpr size_t kPairSmem = kTabSmem + (size_t)kTile * kColAccStride * 4;

// copies the run's tables into the block's shared memory (all threads; the caller synchronises)
__device__ __forceinline__ void load_pair_tables(const PairTables *g, unsigned char *smem, bool packed)
{
  if (packed) {
    const int n0 = (int)(sizeof(PackedTables) / 16), n1 = (int)(5 * sizeof(AggEntry) / 16);
    const uint4 *src = reinterpret_cast<const uint4 *>(&g->packed);
    const uint4 *src2 = reinterpret_cast<const uint4 *>(&g->agg[kEvEntries]);
    uint4 *dst = reinterpret_cast<uint4 *>(smem);
    for (int t = threadIdx.x; t < n0 + n1; t += blockDim.x) dst[t] = t < n0 ? src[t] : src2[t - n0];
  } else {
    const uint4 *src = reinterpret_cast<const uint4 *>(g->agg);
    uint4 *dst = reinterpret_cast<uint4 *>(smem);
    for (int t = threadIdx.x; t < kAggInts / 4; t += blockDim.x) dst[t] = src[t];
  }
}

// the N-plane entries (ew[4], eww) in the block's tables
__device__ __forceinline__ const AggEntry *ew_entries(const unsigned char *smem, bool packed)
{
  return packed ? reinterpret_cast<const AggEntry *>(smem + sizeof(PackedTables))
                : reinterpret_cast<const AggEntry *>(smem) + kEvEntries;
}

struct Counts {
  int T, MM, TS, CT, Y1, Y2, L1, L2, T1, T2;
  int nWc, nWh, nWl, nWt, nWW, nGG;
};

// The final aggregates of a pair for formula_kernel, written over its tensor-core record at: ag[0..6] and a state
// lane (0: the formula kernel finishes the pair; 1: finished here, skipped or queued for the site-order replay)
__device__ __forceinline__ void store_final(const PairArgs &a, size_t at, const int ag[7], bool formula)
{
  const uint32_t st = formula ? 0u : 1u;
  if (a.tc16) {
    reinterpret_cast<uint4 *>(a.tcagg)[at] =
        make_uint4((uint32_t)ag[0] | (uint32_t)ag[1] << 16, (uint32_t)ag[2] | (uint32_t)ag[3] << 16,
                   (uint32_t)ag[4] | (uint32_t)ag[5] << 16, (uint32_t)ag[6] | st << 16);
  } else {
    uint4 *d = reinterpret_cast<uint4 *>(a.tcagg) + 2 * at;
    d[0] = make_uint4((uint32_t)ag[0], (uint32_t)ag[1], (uint32_t)ag[2], (uint32_t)ag[3]);
    d[1] = make_uint4((uint32_t)ag[4], (uint32_t)ag[5], (uint32_t)ag[6], st);
  }
}

// the per-pair epilogue: exact x16 aggregates, tn93's -l / -g / order decisions, formula, certificate (SPLIT: the
// aggregates go back into the pair's tensor-core record at, and formula_kernel runs the formula)
template <bool WPLANE, bool SPLIT>
// cl: the clean-site aggregates of the pair (jointly clean sites, matches, A<->G and C<->T transitions, A, C and G
// base counts over both sequences), from the popcount loop or the tensor-core count kernel; c: N-plane counts
__device__ __forceinline__ void pair_epilogue(const PairArgs &a, const AggEntry *EW, const Counts &c, const int cl[7],
                                              const int acc[9], long i, long j, size_t at, int &namb, int &nund,
                                              AmbLane &al)
{
  const RunConsts &rc = a.rc;
  const int base[7] = {16 * (cl[0] + (int)rc.constT), 16 * (cl[1] + (int)rc.constT), 16 * cl[2], 16 * cl[3],
                       16 * (cl[4] + (int)rc.constNf[0]), 16 * (cl[5] + (int)rc.constNf[1]),
                       16 * (cl[6] + (int)rc.constNf[2])};
  int wb[4] = {0, 0, 0, 0}, nww = 0;
  if (WPLANE) {
    wb[3] = c.nWt;
    wb[1] = c.nWh - c.nWt;
    wb[2] = c.nWl - c.nWt;
    wb[0] = c.nWc - wb[1] - wb[2] - wb[3];
    nww = c.nWW - c.nGG;
  }
  int ag[7];
#pragma unroll
  for (int q = 0; q < 7; q++) {
    int v = base[q] + acc[q];
    if (WPLANE) v += wb[0] * EW[0].v[q] + wb[1] * EW[1].v[q] + wb[2] * EW[2].v[q] + wb[3] * EW[3].v[q] + nww * EW[4].v[q];
    ag[q] = v;
  }
  int amb = acc[7];
  if (WPLANE) amb += wb[0] * EW[0].v[7] + wb[1] * EW[1].v[7] + wb[2] * EW[2].v[7] + wb[3] * EW[3].v[7] + nww * EW[4].v[7];
  double *slot = a.dist + (size_t)(i - a.r0) * a.ncols + (j - a.colbase);
  unsigned long long qentry = 0;
  bool to_replay = false, formula = false;
  if (acc[8] & 1) {
    to_replay = true;  // order-dependent float sums in the main mode
  } else {
    const double tng = (double)ag[0] / 16.0;
    if (tng <= (double)rc.min_overlap) {
      *slot = __longlong_as_double((long long)kSkipBits);
    } else if (rc.fallback_avg && tng * rc.resolve_fraction <= (double)amb) {
      // tn93 recomputes the pair with -a average (refkernel.cpp:742-750): the site-order path does that exactly
      to_replay = true;
      qentry = 1ull << 63;
    } else if (SPLIT) {
      formula = true;
    } else {
      const double nf[4] = {(double)ag[4] / 16.0, (double)ag[5] / 16.0, (double)ag[6] / 16.0,
                            (double)(2 * ag[0] - ag[4] - ag[5] - ag[6]) / 16.0};
      *slot = finish_exact(*a.logt, rc, a.ex, nf, (double)ag[1] / 16.0, (double)ag[2] / 16.0, (double)ag[3] / 16.0, i,
                           j, a.colbase, namb, nund, al);
    }
  }
  if (SPLIT) store_final(a, at, ag, formula);
  if (to_replay) {
    const unsigned idx = atomicAdd(a.replay_n, 1u);
    if (idx < a.replay_cap) a.replay_q[idx] = qentry | ((unsigned long long)i << 31) | (unsigned long long)j;
  }
}

// packed event sums (PackedTables) of one lane: four words of 16-bit lanes and the non-dyadic flag
struct PackedAcc {
  uint32_t w0, w1, w2, w3, f;
};

__device__ __forceinline__ void add_packed(PackedAcc &p, const uint32_t (*tab)[4], const uint32_t *flags, int k)
{
  const uint4 t = *reinterpret_cast<const uint4 *>(tab[k]);
  p.w0 += t.x;
  p.w1 += t.y;
  p.w2 += t.z;
  p.w3 += t.w;
  p.f |= flags[k];
}

// Drops from L2 the tensor-core records of one tile row once every lane of the warp has read its own (all 32 lanes
// call it): the 128-byte lines wholly inside the tile row's records [rec0, rec0 + nrec) (nrec <= 32: the tile's
// columns that lie in this row of the record array) are invalidated without being written back
// (discard.global.L2), so records that the count kernel left in L2 never travel to DRAM. A line that straddles
// either edge also holds records of another tile or row and is kept. Each record is read once, by this warp.
__device__ __forceinline__ void discard_records(const void *base, size_t rec0, long nrec, int rec_bytes, int lane)
{
  __syncwarp();
  const uintptr_t lo = (uintptr_t)base + rec0 * (uintptr_t)rec_bytes, hi = lo + (uintptr_t)nrec * rec_bytes;
  const uintptr_t line = ((lo + 127) & ~(uintptr_t)127) + (uintptr_t)lane * 128;
  if (line + 128 <= hi) asm volatile("discard.global.L2 [%0], 128;" ::"l"(line) : "memory");
}

// Adds the packed table entries of the events [e0, e1) of one sequence against the partner at column p of the
// position-major code matrix. Four events per step: their words and partner codes are loaded before any sum, so
// that four partner-code loads (mostly from L2) are in flight at once.
__device__ __forceinline__ void add_events(PackedAcc &p, const uint32_t (*tab)[4], const uint32_t *flags,
                                           const uint32_t *ev, const uint8_t *ccT, long Np, long partner,
                                           uint32_t e0, uint32_t e1)
{
  uint32_t e = e0;
  for (; e + 4 <= e1; e += 4) {
    uint32_t v[4];
    int pc[4];
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = __ldg(ev + e + q);
#pragma unroll
    for (int q = 0; q < 4; q++) pc[q] = __ldg(ccT + (size_t)(v[q] >> 5) * Np + partner);
#pragma unroll
    for (int q = 0; q < 4; q++) add_packed(p, tab, flags, ((v[q] & 31) - 4) * kCodes + pc[q]);
  }
  for (; e < e1; e++) {
    const uint32_t v = __ldg(ev + e);
    add_packed(p, tab, flags, ((v & 31) - 4) * kCodes + __ldg(ccT + (size_t)(v >> 5) * Np + partner));
  }
}

// One tile of pairs: rows [i0, i0 + 8 * rpw) (rpw = rows per warp, 1..4) x columns [j0, j0 + 32). The block's
// tables must be in smem (load_pair_tables). All threads of the block call it with the same arguments.
template <bool WPLANE, bool GAPMM, bool SPLIT>
__device__ __forceinline__ void pair_tile(const PairArgs &a, const unsigned char *smem, int *colacc, long i0, long j0,
                                          int rpw)
{
  const RunConsts &rc = a.rc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int trows = kWarps * rpw;
  const bool packed = rc.packed;
  const AggEntry *sagg = reinterpret_cast<const AggEntry *>(smem);
  const PackedTables &PT = *reinterpret_cast<const PackedTables *>(smem);
  const AggEntry *EW = ew_entries(smem, packed);
  // block-uniform exits: no valid pair in the tile
  if (i0 >= a.r1 || j0 >= rc.N) return;
  if (!rc.cross && j0 + kTile - 1 <= i0) return;
  const long Np = rc.Npad;
  // N-plane cross terms from the sequences' nonzero N words (row side and column side), when the clean-site counts
  // come from the tensor cores and the events are packed (the column accumulator has room); else every word
  const bool sparse_w = WPLANE && packed && a.tcagg != nullptr && a.wl_off != nullptr;
  // ---- column-side sparse events: lane = tile row, warp-uniform column; skipped where the row is sparse too
  // (packed: the column-side table holds zeros there)
  if (lane < trows) {
    const long ib = min(i0 + lane, rc.N - 1);
    for (int cl = warp; cl < kTile; cl += kWarps) {
      const long j = j0 + cl;
      int *dst = colacc + lane * kColAccStride + cl * 9;
      if (packed) {
        PackedAcc p = {0u, 0u, 0u, 0u, 0u};
        if (j < rc.N) add_events(p, PT.col, PT.colf, a.ev, a.ccT, Np, ib, a.ev_off[j], a.ev_off[j + 1]);
        dst[0] = (int)p.w0;
        dst[1] = (int)p.w1;
        dst[2] = (int)p.w2;
        dst[3] = (int)p.w3;
        dst[4] = (int)p.f;
        if (sparse_w) {
          // the column's N sites against the row's clean bases (its share of the N-plane cross terms)
          int xc = 0, xh = 0, xl = 0, xt = 0;
          if (j < rc.N)
            for (uint32_t q = a.wl_off[j]; q < a.wl_off[j + 1]; q++) {
              const uint64_t *P = a.planes + (size_t)__ldg(a.wl + q) * rc.NP * Np;
              const uint64_t nj = __ldg(P + 3 * Np + j);
              const uint64_t hi = __ldg(P + ib), lo = __ldg(P + Np + ib), ci = __ldg(P + 2 * Np + ib);
              xc += popc(nj & ci);
              xh += popc(nj & hi);
              xl += popc(nj & lo);
              xt += popc(nj & hi & lo);
            }
          dst[5] = xc;
          dst[6] = xh;
          dst[7] = xl;
          dst[8] = xt;
        }
      } else {
        int acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (j < rc.N) {
          const uint32_t f0 = a.ev_off[j], f1 = a.ev_off[j + 1];
          for (uint32_t e = f0; e < f1; e++) {
            const uint32_t v = __ldg(a.ev + e);
            const int pc = a.ccT[(size_t)(v >> 5) * Np + ib];
            if (sparse_code(pc, WPLANE)) continue;
            add_entry(acc, sagg[((v & 31) - 4) * kCodes + pc].v);
          }
        }
#pragma unroll
        for (int q = 0; q < 9; q++) dst[q] = acc[q];
      }
    }
  }
  __syncthreads();
  // ---- per row of this warp (4 rows, one at a time): clean-site counts against lane = column, the row-side
  // sparse events (warp-uniform list), then the epilogue
  const long j = j0 + lane;
  const long jj = j < rc.N ? j : rc.N - 1;
  int namb = 0, nund = 0;
  AmbLane al;
  al.unit = -1;
#pragma unroll 1
  for (int r = 0; r < rpw; r++) {
    const long i = i0 + warp + kWarps * r;
    if (i >= a.r1) break;
    const long lb = rc.cross ? rc.n1 : i + 1;
    const bool valid = j >= lb && j < rc.N;
    if (!__any_sync(0xffffffffu, valid)) continue;
    Counts c = Counts{0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool tc = a.tcagg != nullptr;  // clean-site counts from the tensor-core kernel
    const int *src = colacc + (int)(i - i0) * kColAccStride + lane * 9;
    if (sparse_w) {
      // the row's N sites against the column's clean bases and N sites (warp-uniform word list), then the column's
      // share from the column phase: each union term of the dense loop below splits into these disjoint parts
      for (uint32_t q = a.wl_off[i]; q < a.wl_off[i + 1]; q++) {
        const uint64_t *Pw = a.planes + (size_t)__ldg(a.wl + q) * rc.NP * Np;
        const uint64_t ni = __ldg(Pw + 3 * Np + i);
        const uint64_t hj = __ldg(Pw + jj), lj = __ldg(Pw + Np + jj), cj = __ldg(Pw + 2 * Np + jj);
        const uint64_t nj = __ldg(Pw + 3 * Np + jj);
        c.nWc += popc(ni & cj);
        c.nWh += popc(ni & hj);
        c.nWl += popc(ni & lj);
        c.nWt += popc(ni & hj & lj);
        c.nWW += popc(ni & nj);
        if (GAPMM) c.nGG += popc(__ldg(Pw + 4 * Np + i) & __ldg(Pw + 4 * Np + jj));
      }
      c.nWc += src[5];
      c.nWh += src[6];
      c.nWl += src[7];
      c.nWt += src[8];
    }
    const uint64_t *P = a.planes;
    for (long w = 0; w < ((tc && (!WPLANE || sparse_w)) ? 0 : rc.W); w++, P += (size_t)rc.NP * Np) {
      const uint64_t hj = __ldg(P + jj), lj = __ldg(P + Np + jj), cj = __ldg(P + 2 * Np + jj);
      const uint64_t hi = __ldg(P + i), lo = __ldg(P + Np + i), ci = __ldg(P + 2 * Np + i);
      if (!tc) {
        const uint64_t b = ci & cj, x = hi ^ hj, y = lo ^ lj;
        const uint64_t ts = b & ~x & y;
        c.T += popc(b);
        c.MM += popc(b & (x | y));
        c.TS += popc(ts);
        c.CT += popc(ts & hi);
        c.Y1 += popc(b & hi);
        c.Y2 += popc(b & hj);
        c.L1 += popc(b & lo);
        c.L2 += popc(b & lj);
        c.T1 += popc(b & hi & lo);
        c.T2 += popc(b & hj & lj);
      }
      if (WPLANE) {
        // The N plane and the clean plane of one sequence are disjoint, so each pair of cross terms (this row's N
        // sites against the column's clean bases, and the other way round) covers disjoint sites: one popcount
        // of their union counts both.
        const uint64_t ni = __ldg(P + 3 * Np + i), nj = __ldg(P + 3 * Np + jj);
        c.nWc += popc((ni & cj) | (nj & ci));
        c.nWh += popc((ni & hj) | (nj & hi));
        c.nWl += popc((ni & lj) | (nj & lo));
        c.nWt += popc((ni & hj & lj) | (nj & hi & lo));
        c.nWW += popc(ni & nj);
        if (GAPMM) c.nGG += popc(__ldg(P + 4 * Np + i) & __ldg(P + 4 * Np + jj));
      }
    }
    int acc[9];
    const uint32_t e0 = a.ev_off[i], e1 = a.ev_off[i + 1];
    if (packed) {
      PackedAcc p = {(uint32_t)src[0], (uint32_t)src[1], (uint32_t)src[2], (uint32_t)src[3], (uint32_t)src[4]};
      add_events(p, PT.row, PT.rowf, a.ev, a.ccT, Np, jj, e0, e1);
      acc[0] = (int)(p.w0 & 0xFFFFu);
      acc[1] = (int)(p.w0 >> 16);
      acc[2] = (int)(p.w1 & 0xFFFFu);
      acc[3] = (int)(p.w1 >> 16);
      acc[4] = (int)(p.w2 & 0xFFFFu);
      acc[5] = (int)(p.w2 >> 16);
      acc[6] = (int)(p.w3 & 0xFFFFu);
      acc[7] = (int)(p.w3 >> 16);
      acc[8] = (int)p.f;
    } else {
#pragma unroll
      for (int q = 0; q < 9; q++) acc[q] = src[q];
      for (uint32_t e = e0; e < e1; e++) {
        const uint32_t v = __ldg(a.ev + e);
        const int pc = a.ccT[(size_t)(v >> 5) * Np + jj];
        add_entry(acc, sagg[((v & 31) - 4) * kCodes + pc].v);
      }
    }
    int cl[7];
    size_t at = 0;
    if (tc) {
      // the pair's record from the tensor-core kernel (8 lanes, 7 used); plain loads when SPLIT writes it back
      const long tn = a.tcncols ? a.tcncols : a.ncols, tb = a.tcncols ? a.tccolbase : a.colbase;
      at = (size_t)(i - a.r0) * tn + (jj - tb);
      if (a.tc16) {
        const uint4 *gp = reinterpret_cast<const uint4 *>(a.tcagg) + at;
        const uint4 g = valid ? (SPLIT ? *gp : __ldg(gp)) : make_uint4(0, 0, 0, 0);
        cl[0] = (int)(g.x & 0xFFFFu);
        cl[1] = (int)(g.x >> 16);
        cl[2] = (int)(g.y & 0xFFFFu);
        cl[3] = (int)(g.y >> 16);
        cl[4] = (int)(g.z & 0xFFFFu);
        cl[5] = (int)(g.z >> 16);
        cl[6] = (int)(g.w & 0xFFFFu);
      } else {
        const uint4 *g = reinterpret_cast<const uint4 *>(a.tcagg) + 2 * at;
        const uint4 g0 = valid ? (SPLIT ? g[0] : __ldg(g)) : make_uint4(0, 0, 0, 0);
        const uint4 g1 = valid ? (SPLIT ? g[1] : __ldg(g + 1)) : make_uint4(0, 0, 0, 0);
        cl[0] = (int)g0.x;
        cl[1] = (int)g0.y;
        cl[2] = (int)g0.z;
        cl[3] = (int)g0.w;
        cl[4] = (int)g1.x;
        cl[5] = (int)g1.y;
        cl[6] = (int)g1.z;
      }
      // the records are read once; the split form's formula kernel reads them again
      if (!SPLIT)
        discard_records(a.tcagg, (size_t)(i - a.r0) * tn + (size_t)(j0 - tb), min((long)kTile, tb + tn - j0),
                        a.tc16 ? 16 : 32, lane);
    } else {
      const int nfT = c.T1 + c.T2, nfC = c.Y1 + c.Y2 - nfT, nfG = c.L1 + c.L2 - nfT;
      cl[0] = c.T;
      cl[1] = c.T - c.MM;
      cl[2] = c.TS - c.CT;
      cl[3] = c.CT;
      cl[4] = 2 * c.T - nfC - nfG - nfT;
      cl[5] = nfC;
      cl[6] = nfG;
    }
    if (valid) pair_epilogue<WPLANE, SPLIT>(a, EW, c, cl, acc, i, j, at, namb, nund, al);
  }
  if (!SPLIT) {
    count_flags(a.counters, namb, nund);
    if (a.ex.amb) amb_warp_flush(a.ex.amb, al);
  }
}

template <bool WPLANE, bool GAPMM, int MINB, bool SPLIT>
__global__ void __launch_bounds__(256, MINB) pair_kernel(PairArgs a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int *colacc = reinterpret_cast<int *>(smem_raw + kTabSmem);
  const long i0 = a.r0 + blockIdx.y * (long)kTile;
  const long j0 = a.cstart + blockIdx.x * (long)kTile;
  if (i0 >= a.r1 || j0 >= a.rc.N || (!a.rc.cross && j0 + kTile - 1 <= i0)) return;
  load_pair_tables(a.tab, smem_raw, a.rc.packed);
  __syncthreads();
  pair_tile<WPLANE, GAPMM, SPLIT>(a, smem_raw, colacc, i0, j0, kRowsPerWarp);
}

// The formula for the pairs of one split pair-kernel launch (rows [r0, r1), columns [cstart, cstart + ncol)): one
// thread per pair slot, lanes along a row's columns, reading the final aggregates the pair kernel left in the
// pair's tensor-core record (state 0) and writing the distance. No shared memory; the registers of the formula
// alone decide the occupancy (MINB resident blocks per SM).
template <bool REC16, int MINB>
__global__ void __launch_bounds__(256, MINB) formula_kernel(PairArgs a, long ncol)
{
  const RunConsts &rc = a.rc;
  const long tn = a.tcncols ? a.tcncols : a.ncols, tb = a.tcncols ? a.tccolbase : a.colbase;
  const long j = a.cstart + blockIdx.x * 256l + threadIdx.x;
  int namb = 0, nund = 0;
  AmbLane al;
  al.unit = -1;
  for (long i = a.r0 + blockIdx.y; i < a.r1; i += gridDim.y) {
    const long lb = rc.cross ? rc.n1 : i + 1;
    if (j < lb || j >= rc.N || j >= a.cstart + ncol) continue;
    const size_t at = (size_t)(i - a.r0) * tn + (j - tb);
    int ag[7];
    uint32_t st;
    if (REC16) {
      const uint4 g = reinterpret_cast<const uint4 *>(a.tcagg)[at];
      ag[0] = (int)(g.x & 0xFFFFu);
      ag[1] = (int)(g.x >> 16);
      ag[2] = (int)(g.y & 0xFFFFu);
      ag[3] = (int)(g.y >> 16);
      ag[4] = (int)(g.z & 0xFFFFu);
      ag[5] = (int)(g.z >> 16);
      ag[6] = (int)(g.w & 0xFFFFu);
      st = g.w >> 16;
    } else {
      const uint4 *g = reinterpret_cast<const uint4 *>(a.tcagg) + 2 * at;
      const uint4 g0 = g[0], g1 = g[1];
      ag[0] = (int)g0.x;
      ag[1] = (int)g0.y;
      ag[2] = (int)g0.z;
      ag[3] = (int)g0.w;
      ag[4] = (int)g1.x;
      ag[5] = (int)g1.y;
      ag[6] = (int)g1.z;
      st = g1.w;
    }
    if (st) continue;
    const double nf[4] = {(double)ag[4] / 16.0, (double)ag[5] / 16.0, (double)ag[6] / 16.0,
                          (double)(2 * ag[0] - ag[4] - ag[5] - ag[6]) / 16.0};
    a.dist[(size_t)(i - a.r0) * a.ncols + (j - a.colbase)] =
        finish_exact(*a.logt, rc, a.ex, nf, (double)ag[1] / 16.0, (double)ag[2] / 16.0, (double)ag[3] / 16.0, i, j,
                     a.colbase, namb, nund, al);
  }
  count_flags(a.counters, namb, nund);
  if (a.ex.amb) amb_warp_flush(a.ex.amb, al);
}

static_assert(sizeof(PairArgs) % 4 == 0, "PairArgs is copied as 32-bit words");

// A tile of a batch: alignment k, first row i0, first column j0, rows per warp.
struct BatchTile {
  int k, rpw;
  int i0, j0;
};

// Batched pair kernel over many alignments: a persistent grid takes tiles from a queue (one atomic per tile),
// loads the tile's alignment descriptor and agg table into shared memory when the alignment changes, and runs
// pair_tile. Tiles are ordered longest alignments first, so the tail is short.
template <bool WPLANE, bool GAPMM, int MINB>
__global__ void __launch_bounds__(256, MINB)
    pair_batch_kernel(const PairArgs *descs, const BatchTile *tiles, int ntiles, unsigned *next)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int *colacc = reinterpret_cast<int *>(smem_raw + kTabSmem);
  __shared__ __align__(16) unsigned char sd_raw[sizeof(PairArgs)];
  const PairArgs &sd = *reinterpret_cast<const PairArgs *>(sd_raw);
  __shared__ int s_t;
  int cur = -1;
  for (;;) {
    if (threadIdx.x == 0) s_t = (int)atomicAdd(next, 1u);
    __syncthreads();
    const int t = s_t;
    if (t >= ntiles) break;
    const BatchTile T = tiles[t];
    if (T.k != cur) {
      for (int q = threadIdx.x; q < (int)(sizeof(PairArgs) / 4); q += blockDim.x)
        reinterpret_cast<int32_t *>(sd_raw)[q] = reinterpret_cast<const int32_t *>(&descs[T.k])[q];
      __syncthreads();
      load_pair_tables(sd.tab, smem_raw, sd.rc.packed);
      cur = T.k;
    }
    __syncthreads();
    pair_tile<WPLANE, GAPMM, false>(sd, smem_raw, colacc, T.i0, T.j0, T.rpw);
    __syncthreads();
  }
}

//------------------------------------------------------------------------------------------------ replay
// position of the n-th set bit (0-based) of x; x has more than n set bits
__device__ __forceinline__ int nth_bit32(unsigned x, int n)
{
  int pos = 0;
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    const int c = __popc(x & ((1u << s) - 1u));
    if (n >= c) {
      n -= c;
      x >>= s;
      pos += s;
    }
  }
  return pos;
}

// tn93's own per-pair computation (refkernel.cpp:622-750) for one pair, by one warp:
//   * clean/clean cells: the 4x4 table from the bit planes (lanes over 64-column words);
//   * every other site in site order: per word, the lanes fetch the codes of the word's non-clean sites (in
//     order) and lane q adds the site's contribution to float cell q, so each cell is summed in site order as
//     tn93 does; lanes 16..19 add the integer diagonal resolutions, lane 20 the ambiguity count;
//   * lane 0: tn93's c1-major merge of float and integer cells and the -l / -g tests, leaving the formula's exact
//     inputs. t = 1 starts in AVERAGE mode (a pair the -g test already sent there).
// All lanes call it; the result is valid in lane 0.
struct WalkOut {
  bool skip;  // below the overlap (-l)
  double nf[4], diag, ag, ct;
};

__device__ WalkOut walk_pair(const ReplayArgs &a, long i, long j, int t, unsigned char *sc1, unsigned char *sc2)
{
  const int lane = threadIdx.x & 31;
  const RunConsts &rc = a.rc;
  const long Np = rc.Npad;
  const uint64_t last_valid = (rc.Lc & 63) ? ((1ull << (rc.Lc & 63)) - 1ull) : ~0ull;
  const uint8_t *s1 = a.cc + (size_t)i * rc.Lc, *s2 = a.cc + (size_t)j * rc.Lc;
  // clean/clean 4x4 counts (the same in every mode)
  int cnt[16];
#pragma unroll
  for (int q = 0; q < 16; q++) cnt[q] = 0;
  for (long w = lane; w < rc.W; w += 32) {
    const uint64_t *P = a.planes + (size_t)w * rc.NP * Np;
    const uint64_t hi = P[i], lo = P[Np + i], ci = P[2 * Np + i];
    const uint64_t hj = P[j], lj = P[Np + j], cj = P[2 * Np + j];
    const uint64_t xi[4] = {ci & ~hi & ~lo, ci & hi & ~lo, ci & ~hi & lo, ci & hi & lo};
    const uint64_t xj[4] = {cj & ~hj & ~lj, cj & hj & ~lj, cj & ~hj & lj, cj & hj & lj};
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
      for (int y = 0; y < 4; y++) cnt[x * 4 + y] += popc(xi[x] & xj[y]);
  }
#pragma unroll
  for (int q = 0; q < 16; q++)
    for (int o = 16; o; o >>= 1) cnt[q] += __shfl_xor_sync(0xffffffffu, cnt[q], o);
  WalkOut R;
  R.skip = false;
  R.diag = R.ag = R.ct = 0.;
  R.nf[0] = R.nf[1] = R.nf[2] = R.nf[3] = 0.;
  for (;;) {
    const SiteEntry *S = a.site + t * kCodes * kCodes;
    double acc = 0.;  // lane q < 16: float cell q
    long iacc = 0;    // lanes 16..19: diagonal resolutions, lane 20: ambiguity count
    for (long w = 0; w < rc.W; w++) {
      const uint64_t *P = a.planes + (size_t)w * rc.NP * Np;
      uint64_t E = ~(P[2 * Np + i] & P[2 * Np + j]);
      if (w == rc.W - 1) E &= last_valid;
      if (!E) continue;
      const int ne = __popcll(E), nlo = __popc((unsigned)E);
      for (int rk = lane; rk < ne; rk += 32) {
        const int bit = rk < nlo ? nth_bit32((unsigned)E, rk) : 32 + nth_bit32((unsigned)(E >> 32), rk - nlo);
        const long k = w * 64 + bit;
        sc1[rk] = s1[k];
        sc2[rk] = s2[k];
      }
      __syncwarp();
      if (lane < 16) {
        for (int l = 0; l < ne; l++) {
          const double v = S[sc1[l] * kCodes + sc2[l]].fc[lane];
          if (v != 0.) acc = __dadd_rn(acc, v);
        }
      } else if (lane < 20) {
        for (int l = 0; l < ne; l++) iacc += S[sc1[l] * kCodes + sc2[l]].icd[lane - 16];
      } else if (lane == 20) {
        for (int l = 0; l < ne; l++) iacc += S[sc1[l] * kCodes + sc2[l]].amb;
      }
      __syncwarp();
    }
    // lane 0: gather the cells, then tn93's merge and decisions
    double fc[16];
    long icd[4];
#pragma unroll
    for (int q = 0; q < 16; q++) fc[q] = __shfl_sync(0xffffffffu, acc, q);
#pragma unroll
    for (int q = 0; q < 4; q++) icd[q] = __shfl_sync(0xffffffffu, iacc, 16 + q);
    const long amb = __shfl_sync(0xffffffffu, iacc, 20);
    int next = 0;  // 0 done, 1 recompute with -a average
    if (lane == 0) {
      long ic[16];
      for (int q = 0; q < 16; q++) ic[q] = cnt[q];
      for (int x = 0; x < 4; x++) ic[x * 5] += icd[x] + rc.constCnt[x];
      double tot = 0., nf[4] = {0., 0., 0., 0.};
      for (int c1 = 0; c1 < 4; c1++)
        for (int c2 = 0; c2 < 4; c2++) {
          const double pc = fc[c1 * 4 + c2] = __dadd_rn(fc[c1 * 4 + c2], (double)ic[c1 * 4 + c2]);
          tot = __dadd_rn(tot, pc);
          nf[c1] = __dadd_rn(nf[c1], pc);
          nf[c2] = __dadd_rn(nf[c2], pc);
        }
      if (tot <= (double)rc.min_overlap) {
        R.skip = true;
      } else if (t == 0 && rc.fallback_avg && __dmul_rn(tot, rc.resolve_fraction) <= (double)(unsigned long)amb) {
        next = 1;
      } else {
        R.diag = __dadd_rn(__dadd_rn(__dadd_rn(fc[0], fc[5]), fc[10]), fc[15]);
        R.ag = __dadd_rn(fc[2], fc[8]);
        R.ct = __dadd_rn(fc[7], fc[13]);
        for (int q = 0; q < 4; q++) R.nf[q] = nf[q];
      }
    }
    next = __shfl_sync(0xffffffffu, next, 0);
    if (!next) break;
    t = 1;
  }
  return R;
}

// The order-dependent pairs (a contribution that is not a multiple of 1/16), one warp per pair from the queue.
__device__ __forceinline__ void replay_run(const ReplayArgs &a)
{
  __shared__ unsigned char sc1[kWarps][64], sc2[kWarps][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long n = min((unsigned long long)*a.qn, a.qcap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(&a.counters[2], n);
  AmbLane al;
  al.unit = -1;
  for (unsigned long long idx = (unsigned long long)blockIdx.x * kWarps + warp; idx < n;
       idx += (unsigned long long)gridDim.x * kWarps) {
    const unsigned long long e = a.q[idx];
    const int t = (int)(e >> 63);
    const long i = (long)((e >> 31) & 0xFFFFFFFFull), j = (long)(e & 0x7FFFFFFFull);
    const WalkOut W = walk_pair(a, i, j, t, sc1[warp], sc2[warp]);
    if (lane == 0) {
      int qa = 0, qu = 0;
      const double res = W.skip ? __longlong_as_double((long long)kSkipBits)
                                : finish_exact(*a.logt, a.rc, a.ex, W.nf, W.diag, W.ag, W.ct, i, j, a.colbase, qa,
                                               qu, al);
      a.dist[(size_t)(i - a.r0) * a.ncols + (j - a.colbase)] = res;
      if (qa) atomicAdd(&a.counters[0], 1ull);
      if (qu) atomicAdd(&a.counters[1], 1ull);
    }
  }
  if (a.ex.amb && lane == 0 && al.unit >= 0) amb_flush(a.ex.amb, al.unit, al.n, al.lo, al.hi, al.spread);
}

// Undecided pairs, step 1 (one warp per listed pair): the site-order walk gives the formula's exact inputs in any
// mode (for a pair the pair kernel finished, its x16 aggregates and the walk's float sums are the same numbers),
// then the arguments of its logarithms. descs[k] describes run k of the list's entries.
__global__ void __launch_bounds__(256) und_args_kernel(const ReplayArgs *descs, const unsigned long long *list,
                                                       unsigned n, UndEntry *out)
{
  __shared__ unsigned char sc1[kWarps][64], sc2[kWarps][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned idx = blockIdx.x * kWarps + warp; idx < n; idx += gridDim.x * kWarps) {
    const int k = (int)list[2 * (size_t)idx];
    const unsigned long long ij = list[2 * (size_t)idx + 1];
    const long i = (long)(ij >> 32), j = (long)(ij & 0xFFFFFFFFull);
    const ReplayArgs &a = descs[k];
    const WalkOut W = walk_pair(a, i, j, 0, sc1[warp], sc2[warp]);
    if (lane == 0) {
      UndEntry &E = out[idx];
      E.k = k;
      E.slot = (long)((i - a.r0) * a.ncols + (j - a.colbase));
      E.state = W.skip ? 1 : 0;
      E.nlog = 0;
      for (int q = 0; q < 4; q++) E.in[q] = W.nf[q];
      E.in[4] = W.diag;
      E.in[5] = W.ag;
      E.in[6] = W.ct;
      E.arg[0] = E.arg[1] = E.arg[2] = 1.0;
      if (!W.skip) {
        const Prep P = tn93_prep(W.nf, W.diag, W.ag, W.ct);
        E.nlog = P.nlog;
        for (int q = 0; q < 3; q++) E.arg[q] = P.arg[q];
      }
    }
  }
}

// Undecided pairs, step 2 (one thread per pair): the formula from the C library's logarithms (UndEntry::lg)
__global__ void und_finish_kernel(const ReplayArgs *descs, const UndEntry *e, unsigned n)
{
  const unsigned idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const UndEntry &E = e[idx];
  if (E.state) return;
  const double nf[4] = {E.in[0], E.in[1], E.in[2], E.in[3]};
  const Prep P = tn93_prep(nf, E.in[4], E.in[5], E.in[6]);
  descs[E.k].dist[E.slot] = tn93_combine(P, E.lg[0], E.lg[1], E.lg[2]);
}

__global__ void __launch_bounds__(256) replay_kernel(ReplayArgs a) { replay_run(a); }

// the replay queues of a batch's alignments, one after the other (each is usually empty or short)
__global__ void __launch_bounds__(256) replay_batch_kernel(const ReplayArgs *descs, int K)
{
  for (int k = 0; k < K; k++)
    if (*descs[k].qn) replay_run(descs[k]);
}

// exclusive scan of a band's segment byte counts (one block), and the band total
__global__ void __launch_bounds__(1024) scan_kernel(const unsigned long long *in, unsigned long long *out, long n,
                                                   unsigned long long *total)
{
  __shared__ unsigned long long part[1024];
  const long per = (n + 1023) / 1024;
  const long b = threadIdx.x * per, e = min(n, b + per);
  unsigned long long s = 0;
  for (long k = b; k < e; k++) s += in[k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const unsigned long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (long k = b; k < e; k++) {
    out[k] = run;
    run += in[k];
  }
  if (threadIdx.x == 1023) *total = part[1023];
}

// Large exclusive scans in three coalesced passes: tile sums, a scan of the tile sums (scan_kernel), then each
// tile's scan from its offset. A tile is 256 threads x 16 consecutive elements.
constexpr int kScanTile = 4096;

__global__ void __launch_bounds__(256) tile_sum_kernel(const unsigned long long *in, long n,
                                                       unsigned long long *tile_sum)
{
  __shared__ unsigned long long ws[8];
  const long b = blockIdx.x * (long)kScanTile;
  unsigned long long s = 0;
  for (int k = threadIdx.x; k < kScanTile; k += 256) {
    const long e = b + k;
    if (e < n) s += in[e];
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < 8; w++) t += ws[w];
    tile_sum[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(256) tile_scan_kernel(const unsigned long long *in, unsigned long long *out, long n,
                                                        const unsigned long long *tile_off)
{
  __shared__ unsigned long long ws[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long b = blockIdx.x * (long)kScanTile + threadIdx.x * 16l;
  unsigned long long v[16], s = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    v[k] = b + k < n ? in[b + k] : 0;
    s += v[k];
  }
  // exclusive scan of the per-thread sums over the block
  unsigned long long inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  unsigned long long base = tile_off[blockIdx.x];
  for (int w = 0; w < warp; w++) base += ws[w];
  unsigned long long run = base + inc - s;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    if (b + k < n) out[b + k] = run;
    run += v[k];
  }
}

// exclusive scan of n counters into out, the sum into *total; tmp holds 2 * ceil(n / kScanTile) + 1 counters
cudaError_t launch_scan(const unsigned long long *in, unsigned long long *out, long n, unsigned long long *total,
                        unsigned long long *tmp, cudaStream_t st)
{
  if (n <= 65536) {
    scan_kernel<<<1, 1024, 0, st>>>(in, out, n, total);
    return cudaGetLastError();
  }
  const long nt = (n + kScanTile - 1) / kScanTile;
  tile_sum_kernel<<<(unsigned)nt, 256, 0, st>>>(in, n, tmp);
  scan_kernel<<<1, 1024, 0, st>>>(tmp, tmp + nt, nt, total);
  tile_scan_kernel<<<(unsigned)nt, 256, 0, st>>>(in, out, n, tmp + nt);
  return cudaGetLastError();
}

//------------------------------------------------------------------------------------------------ rows
__device__ __forceinline__ int digits_of(long v)
{
  int n = 1;
  while (v >= 10) {
    v /= 10;
    n++;
  }
  return n;
}

struct PairView {
  bool valid, computed, linked, counted;  // counted: contributes to the sums (not a -l skip)
  int bin, hb;
  long w;
  double thisD;
};

__device__ __forceinline__ PairView view_pair(const RowArgs &a, long i, long j, long cnt_i)
{
  const RunConsts &rc = a.rc;
  PairView v;
  v.valid = j < rc.N;
  v.computed = v.linked = v.counted = false;
  v.bin = 0;
  v.hb = 0;
  v.w = 0;
  v.thisD = -1.0;
  if (!v.valid) return v;
  const double raw = a.dist[(size_t)(i - a.r0) * a.ncols + (j - a.colbase)];
  v.w = cnt_i * a.counts[j];
  if (rc.fst) v.bin = i < rc.n1 ? (j >= rc.n1 ? 2 : 0) : 1;
  if ((uint64_t)__double_as_longlong(raw) != kSkipBits) {
    v.computed = true;
    v.hb = hist_bin(raw);
    v.thisD = raw <= 0. ? 0. : raw;
  }
  v.linked = v.thisD >= rc.min_distance && v.thisD <= rc.threshold;
  v.counted = !(v.thisD <= -0.5);
  return v;
}

// A printed distance handed from the stats kernel to the writer, one 32-bit word per pair slot: 0 = not printed;
// kind 1 (bits 30-31) = the six digits q (bits 0-19) and the decimal exponent X + 16 (bits 20-25) of a value in
// [1e-5, 1e5); kind 2 = zero ("0"); kind 3 = any other value (the writer formats the double itself). len receives
// the length of the text. d is a reported distance: not negative, not NaN.
__device__ __forceinline__ uint32_t print_code(double d, int &len)
{
  if (d == 0.0) {
    len = 1;
    return 2u << 30;
  }
  if (d >= 1e-5 && d < 1e5) {
    const Dec D = decimal6(d);
    len = dec_len(D);
    return (1u << 30) | ((uint32_t)(D.X + 16) << 20) | D.q;
  }
  len = fmt_g_len(d);
  return 3u << 30;
}

// the text of a printed-distance code (d: the distance, read only for kind 3); returns the length
__device__ __forceinline__ int fmt_code(uint32_t code, double d, char *out)
{
  const uint32_t kind = code >> 30;
  if (kind == 1) {
    Dec D;
    D.q = code & 0xFFFFFu;
    D.X = (int)((code >> 20) & 63u) - 16;
    return fmt_dec(D, out);
  }
  if (kind == 2) {
    out[0] = '0';
    return 1;
  }
  return fmt_g(d, out);
}

// what the text writers need of a pair: whether it is reported, and its printed distance (tn93's "<= 0 -> 0")
__device__ __forceinline__ bool linked_pair(const RowArgs &a, long i, long j, double &thisD)
{
  const RunConsts &rc = a.rc;
  if (j >= rc.N) return false;
  const double raw = a.dist[(size_t)(i - a.r0) * a.ncols + (j - a.colbase)];
  if ((uint64_t)__double_as_longlong(raw) == kSkipBits) return false;
  thisD = raw <= 0. ? 0. : raw;
  return thisD >= rc.min_distance && thisD <= rc.threshold;
}

__device__ __forceinline__ int self_len(const RowArgs &a, long i)
{
  if (!a.rc.report_self || a.rc.cross) return 0;
  if (a.rc.format == 0) return 2 * a.name_len[i] + 4;
  if (a.rc.format == 1) return 2 * digits_of(i) + 4;
  return 0;
}

// Columns per segment of the stats and write kernels: a warp handles one (row, segment), so a band of a few
// long rows still fills the GPU.
constexpr int kSeg = 1024;

// one warp per (row, segment): histogram, links, skips, maxima and the byte count of the segment's text
__device__ __forceinline__ void stats_rows(const RowArgs &a, long bx, int sg)
{
  __shared__ unsigned long long sh[3 * kHistBins];
  for (int t = threadIdx.x; t < 3 * kHistBins; t += blockDim.x) sh[t] = 0;
  __syncthreads();
  const RunConsts &rc = a.rc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long i = a.r0 + bx * kWarps + warp;
  if (i < a.r1) {
    const long r = i - a.r0;
    const long slot = r * a.maxseg + sg;
    const long lb = rc.cross ? rc.n1 : i + 1;
    const long c0 = lb + (long)sg * kSeg, c1 = min(rc.N, c0 + kSeg);
    const long cnt_i = a.counts[i];
    const int nli = a.name_len[i];
    const int dli = rc.format == 1 ? digits_of(i) : 0;
    double m0 = 0., m1 = 0., m2 = 0.;
    long long links = 0, skipped = 0;
    unsigned long long bytes = 0;
    if (sg == 0 && !rc.cross) {
      if (cnt_i > 1 && lane == 0) {
        const unsigned long long svs = (unsigned long long)(cnt_i * (cnt_i - 1l)) >> 1;
        atomicAdd(&sh[i < rc.n1 ? 0 : kHistBins], svs);
      }
      if (lane == 0 && rc.emit) bytes += self_len(a, i);
    }
    for (long j0 = c0; j0 < c1; j0 += 32) {
      const long j = j0 + lane;
      PairView v = view_pair(a, i, j, cnt_i);
      if (j >= c1) v.valid = v.computed = v.linked = false;
      // histogram: lanes with the same bin add once (their weights summed when all are 1)
      const int key = v.computed ? v.bin * kHistBins + v.hb : -1;
      const unsigned peers = __match_any_sync(0xffffffffu, key);
      if (__all_sync(0xffffffffu, !v.computed || v.w == 1)) {
        if (v.computed && lane == __ffs(peers) - 1) atomicAdd(&sh[key], (unsigned long long)__popc(peers));
      } else if (v.computed) {
        atomicAdd(&sh[key], (unsigned long long)v.w);
      }
      uint32_t code = 0;
      if (v.valid && v.linked) {
        links += v.w;
        if (rc.emit) {
          if (rc.format != 2) {
            int gl;
            if (a.dcode)
              code = print_code(v.thisD, gl);
            else
              gl = fmt_g_len(v.thisD);
            bytes += rc.format == 0 ? nli + a.name_len[j] + gl + 3 : dli + digits_of(j) + gl + 3;
          } else {
            a.hy[(size_t)i * rc.N + j] = v.thisD;
            a.hy[(size_t)j * rc.N + i] = v.thisD;
          }
        }
      }
      if (a.dcode && v.valid) a.dcode[(size_t)(i - a.r0) * a.ncols + (j - a.colbase)] = code;
      if (v.valid && !v.counted) skipped++;
      if (v.valid && v.counted) {
        if (v.bin == 0) m0 = v.thisD > m0 ? v.thisD : m0;
        else if (v.bin == 1) m1 = v.thisD > m1 ? v.thisD : m1;
        else m2 = v.thisD > m2 ? v.thisD : m2;
      }
    }
    for (int o = 16; o; o >>= 1) {
      links += __shfl_xor_sync(0xffffffffu, links, o);
      skipped += __shfl_xor_sync(0xffffffffu, skipped, o);
      bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
      m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
      m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
      m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    if (lane == 0) {
      a.seg_bytes[slot] = bytes;
      a.seg_links[slot] = links;
      a.seg_skip[slot] = skipped;
      a.seg_max[slot * 3] = m0;
      a.seg_max[slot * 3 + 1] = m1;
      a.seg_max[slot * 3 + 2] = m2;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 3 * kHistBins; t += blockDim.x)
    if (sh[t]) atomicAdd(&a.hist[t], sh[t]);
}

// Resident blocks per SM for the stats kernel 6 (40 registers) and the write kernel 4 (64): more warps hide their load
// latency better than fewer spills would (same box, per 22.4 M pairs: stats + sums 0.80 ms with 3 blocks, 0.76 with
// 4, 0.72 with 6; write 0.78 ms with 3, 0.68 with 4, 0.91 with 6; 2 blocks without spills were slower still)
__global__ void __launch_bounds__(256, 6) stats_kernel(RowArgs a) { stats_rows(a, blockIdx.x, blockIdx.y); }


// one warp per row: tn93's row sums in column order (swifttn93.cpp:2594-2602); lane 0 adds each chunk's terms in
// order. The self-pair weights come first, as tn93 adds them when the row starts (swifttn93.cpp:2405-2415).
__device__ __forceinline__ void sum_rows(const RowArgs &a, long bx)
{
  __shared__ double sterm[kWarps][32], sw[kWarps][32];
  __shared__ unsigned char sbin[kWarps][32];
  const RunConsts &rc = a.rc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long i = a.r0 + bx * kWarps + warp;
  if (i >= a.r1) return;
  const long cnt_i = a.counts[i];
  double s0 = 0., s1 = 0., s2 = 0., w0 = 0., w1 = 0., w2 = 0.;
  const long lb = rc.cross ? rc.n1 : i + 1, cend = rc.N, out_row = i - a.r0;
  if (!rc.cross && cnt_i > 1) {
    const unsigned long long svs = (unsigned long long)(cnt_i * (cnt_i - 1l)) >> 1;
    if (i < rc.n1)
      w0 += (double)svs;
    else
      w1 += (double)svs;
  }
  const double *drow = a.dist + (size_t)(i - a.r0) * a.ncols - a.colbase;
  if (!rc.fst) {
    // Single bin: every lane adds the chunk's 32 terms in column order (the same chain in every lane, so no lane
    // waits for another); skipped pairs and columns past the end add +0.0, which leaves a non-negative sum
    // unchanged. The weights are integers: their double sum is exact, in any order, while the total stays below
    // 2^53, so they are added as integers (and re-added one by one in the rare case the total is larger).
    // The next chunk's distance and count are loaded before this chunk's chain runs, so the loads overlap it.
    unsigned long long wsum = 0;
    double raw = 0.;
    long cj = 0;
    if (lb + lane < cend) {
      raw = drow[lb + lane];
      cj = a.counts[lb + lane];
    }
    for (long j0 = lb; j0 < cend; j0 += 32) {
      const long j = j0 + lane, jn = j + 32;
      double raw_n = 0.;
      long cj_n = 0;
      if (jn < cend) {
        raw_n = drow[jn];
        cj_n = a.counts[jn];
      }
      double term = 0.;
      if (j < cend && (uint64_t)__double_as_longlong(raw) != kSkipBits) {
        const double t = raw <= 0. ? 0. : raw;
        const long w = cnt_i * cj;
        term = __dmul_rn(t, (double)w);
        wsum += (unsigned long long)w;
      }
#pragma unroll
      for (int l = 0; l < 32; l++) s0 = __dadd_rn(s0, __shfl_sync(0xffffffffu, term, l));
      raw = raw_n;
      cj = cj_n;
    }
    for (int o = 16; o; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    const unsigned long long svs = (!rc.cross && cnt_i > 1) ? (unsigned long long)(cnt_i * (cnt_i - 1l)) >> 1 : 0;
    if (wsum + svs < (1ull << 53)) {
      w0 = (double)(wsum + svs);
    } else {
      w0 = (double)svs;
      for (long j0 = lb; j0 < cend; j0 += 32) {
        const long j = j0 + lane;
        double wl = 0.;
        if (j < cend && (uint64_t)__double_as_longlong(drow[j]) != kSkipBits) wl = (double)(cnt_i * a.counts[j]);
#pragma unroll
        for (int l = 0; l < 32; l++) w0 = __dadd_rn(w0, __shfl_sync(0xffffffffu, wl, l));
      }
    }
    if (lane == 0) {
      const long r = out_row;
      a.row_sum[r * 3] = s0;
      a.row_sum[r * 3 + 1] = 0.;
      a.row_sum[r * 3 + 2] = 0.;
      a.row_w[r * 3] = w0;
      a.row_w[r * 3 + 1] = 0.;
      a.row_w[r * 3 + 2] = 0.;
    }
    return;
  }
  for (long j0 = lb; j0 < cend; j0 += 32) {
    const long j = j0 + lane;
    bool inc = false;
    double term = 0., wl = 0.;
    int bin = 0;
    if (j < cend) {
      const double raw = drow[j];
      if ((uint64_t)__double_as_longlong(raw) != kSkipBits) {
        const double t = raw <= 0. ? 0. : raw;
        const long w = cnt_i * a.counts[j];
        if (rc.fst) bin = i < rc.n1 ? (j >= rc.n1 ? 2 : 0) : 1;
        inc = true;
        term = __dmul_rn(t, (double)w);
        wl = (double)w;
      }
    }
    sterm[warp][lane] = term;
    sw[warp][lane] = wl;
    sbin[warp][lane] = inc ? (unsigned char)bin : (unsigned char)255;
    __syncwarp();
    if (lane == 0) {
      const int n = (int)min(32l, cend - j0);
      if (!rc.fst) {
        for (int l = 0; l < n; l++)
          if (sbin[warp][l] == 0) {
            s0 = __dadd_rn(s0, sterm[warp][l]);
            w0 = __dadd_rn(w0, sw[warp][l]);
          }
      } else {
        for (int l = 0; l < n; l++) {
          const int bl = sbin[warp][l];
          if (bl == 0) {
            s0 = __dadd_rn(s0, sterm[warp][l]);
            w0 = __dadd_rn(w0, sw[warp][l]);
          } else if (bl == 1) {
            s1 = __dadd_rn(s1, sterm[warp][l]);
            w1 = __dadd_rn(w1, sw[warp][l]);
          } else if (bl == 2) {
            s2 = __dadd_rn(s2, sterm[warp][l]);
            w2 = __dadd_rn(w2, sw[warp][l]);
          }
        }
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    const long r = out_row;
    a.row_sum[r * 3] = s0;
    a.row_sum[r * 3 + 1] = s1;
    a.row_sum[r * 3 + 2] = s2;
    a.row_w[r * 3] = w0;
    a.row_w[r * 3 + 1] = w1;
    a.row_w[r * 3 + 2] = w2;
  }
}

__global__ void __launch_bounds__(256) sum_kernel(RowArgs a) { sum_rows(a, blockIdx.x); }

__device__ __forceinline__ char *put_bytes(char *o, const char *s, int n)
{
  for (int k = 0; k < n; k++) o[k] = s[k];
  return o + n;
}

// the text of one reported pair at o (generic pointer: shared staging or global); csvn prints column j as j - jshift
__device__ __forceinline__ void put_line(char *o, const RowArgs &a, long i, long j, long jshift, const char *ni,
                                         int nli, const char *g, int gl)
{
  const RunConsts &rc = a.rc;
  if (rc.format == 0) {
    o = put_bytes(o, ni, nli);
    *o++ = rc.delim;
    o = put_bytes(o, a.names + a.name_off[j], a.name_len[j]);
    *o++ = rc.delim;
  } else {
    char t[24];
    int n = fmt_long(i, t);
    o = put_bytes(o, t, n);
    *o++ = rc.delim;
    n = fmt_long(j - jshift, t);
    o = put_bytes(o, t, n);
    *o++ = rc.delim;
  }
  o = put_bytes(o, g, gl);
  *o = '\n';
}

// Output staging: each warp assembles its lines in shared memory at the same offset modulo 16 as their
// destination, then stores whole 16-byte blocks (edges byte by byte), so global writes are coalesced. Nothing is
// written at or past the end of the counted range.
constexpr int kStage = 4096;

struct Stager {
  char *buf;       // this warp's staging buffer (16-byte aligned)
  uintptr_t gpos;  // global address of the first staged byte
  uintptr_t gend;  // end of the counted range
  int head, fill;  // buf[head .. head + fill) holds global [gpos, gpos + fill)
  bool over;       // the text ran past its counted length (reported as an internal error)
  __device__ void flush(int lane)
  {
    const uintptr_t g0 = gpos - (uintptr_t)head;
    if (gpos + fill > gend) over = true;
    const int end = (int)min((uintptr_t)(head + fill), gend > g0 ? gend - g0 : 0), nblk = (end + 15) >> 4;
    for (int b = lane; b < nblk; b += 32) {
      const int lo = b << 4, hi = lo + 16;
      if (lo >= head && hi <= end)
        *reinterpret_cast<uint4 *>(g0 + lo) = *reinterpret_cast<const uint4 *>(buf + lo);
      else
        for (int k = max(lo, head); k < min(hi, end); k++) *reinterpret_cast<char *>(g0 + k) = buf[k];
    }
    __syncwarp();
    gpos += fill;
    head = (int)(gpos & 15);
    fill = 0;
  }
};

// one warp per (row, segment): the segment's text at its scanned offset (the row's self line in segment 0)
__device__ __forceinline__ void write_rows(const RowArgs &a, long bx, int sg)
{
  __shared__ __align__(16) char stage[kWarps][kStage];
  const RunConsts &rc = a.rc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long i = a.r0 + bx * kWarps + warp;
  if (i >= a.r1) return;
  const long slot = (i - a.r0) * a.maxseg + sg;
  const long lb = rc.cross ? rc.n1 : i + 1;
  const long c0 = lb + (long)sg * kSeg, c1 = min(rc.N, c0 + kSeg);
  if (a.seg_bytes[slot] == 0) return;
  const int nli = a.name_len[i];
  const char *ni = a.names + a.name_off[i];
  Stager S;
  S.buf = stage[warp];
  S.gpos = (uintptr_t)(a.out + a.seg_off[slot]);
  S.gend = S.gpos + a.seg_bytes[slot];
  S.head = (int)(S.gpos & 15);
  S.fill = 0;
  S.over = false;
  const int sl = sg == 0 ? self_len(a, i) : 0;
  if (sl) {
    const bool direct = S.head + sl > kStage;
    if (direct && S.gpos + sl > S.gend) {
      if (lane == 0) atomicAdd(a.err, 1ull);
      return;
    }
    if (lane == 0) {
      char *o = direct ? (char *)S.gpos : S.buf + S.head;
      if (rc.format == 0) {
        o = put_bytes(o, ni, nli);
        *o++ = rc.delim;
        o = put_bytes(o, ni, nli);
        *o++ = rc.delim;
      } else {
        char t[24];
        const int n = fmt_long(i, t);
        o = put_bytes(o, t, n);
        *o++ = rc.delim;
        o = put_bytes(o, t, n);
        *o++ = rc.delim;
      }
      *o++ = '0';
      *o = '\n';
    }
    __syncwarp();
    if (direct) {
      S.gpos += sl;
      S.head = (int)(S.gpos & 15);
    } else
      S.fill = sl;
  }
  const int dli = rc.format == 1 ? digits_of(i) : 0;
  for (long j0 = c0; j0 < c1; j0 += 32) {
    const long j = j0 + lane;
    double thisD = 0.;
    bool put;
    uint32_t code = 0;
    if (a.dcode) {
      // the stats kernel's code of this pair: printed or not, and its digits
      code = j < c1 ? a.dcode[(size_t)(i - a.r0) * a.ncols + (j - a.colbase)] : 0u;
      put = code != 0;
      if (put && (code >> 30) == 3u) linked_pair(a, i, j, thisD);
    } else {
      put = j < c1 && linked_pair(a, i, j, thisD);
    }
    char g[24];
    int gl = 0, len = 0;
    if (put) {
      gl = a.dcode ? fmt_code(code, thisD, g) : fmt_g(thisD, g);
      len = rc.format == 0 ? nli + a.name_len[j] + gl + 3 : dli + digits_of(j) + gl + 3;
    }
    int pre = len;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, pre, o);
      if (lane >= o) pre += t;
    }
    const int total = __shfl_sync(0xffffffffu, pre, 31);
    if (total == 0) continue;
    if (S.head + S.fill + total > kStage) S.flush(lane);
    if (S.head + total > kStage) {
      // a chunk larger than the staging buffer (very long names): write it in place
      if (S.gpos + total > S.gend) {
        S.over = true;
        break;
      }
      if (put) put_line((char *)(S.gpos + pre - len), a, i, j, 0, ni, nli, g, gl);
      __syncwarp();
      S.gpos += total;
      S.head = (int)(S.gpos & 15);
    } else {
      if (put) put_line(S.buf + S.head + S.fill + (pre - len), a, i, j, 0, ni, nli, g, gl);
      __syncwarp();
      S.fill += total;
    }
  }
  S.flush(lane);
  if (S.over && lane == 0) atomicAdd(a.err, 1ull);
}

__global__ void __launch_bounds__(256, 4) write_kernel(RowArgs a) { write_rows(a, blockIdx.x, blockIdx.y); }

// Batched row stage: block b of the batch is row block blocks[b].y of alignment blocks[b].x; blockIdx.y is the
// segment (blocks past an alignment's segment count exit).
__global__ void __launch_bounds__(256) stats_batch_kernel(const RowArgs *descs, const int2 *blocks)
{
  const int2 B = blocks[blockIdx.x];
  const RowArgs &a = descs[B.x];
  if ((long)blockIdx.y >= a.maxseg) return;
  stats_rows(a, B.y, blockIdx.y);
}

__global__ void __launch_bounds__(256) sum_batch_kernel(const RowArgs *descs, const int2 *blocks)
{
  const int2 B = blocks[blockIdx.x];
  sum_rows(descs[B.x], B.y);
}

__global__ void __launch_bounds__(256) write_batch_kernel(const RowArgs *descs, const int2 *blocks)
{
  const int2 B = blocks[blockIdx.x];
  const RowArgs &a = descs[B.x];
  if ((long)blockIdx.y >= a.maxseg) return;
  write_rows(a, B.y, blockIdx.y);
}

// Per alignment of a batch (single-file runs, bin 0 only): links, skips and maximum over its (row, segment)
// slots, and tn93's mean numerator and weight: the rows' sums added in row order from 0 (swifttn93.cpp:2838-2848).
// One block per alignment; thread 0 adds a shared-memory stage of the row sums in order.
__global__ void __launch_bounds__(256) aln_reduce_kernel(const RowArgs *descs, double *out /* [K][3] */,
                                                         long long *cnt /* [K][2] */)
{
  __shared__ double ss[2048], sw[2048];
  __shared__ long long rl[8], rs[8];
  __shared__ double rm[8];
  const RowArgs &a = descs[blockIdx.x];
  const long nr = a.r1 - a.r0, ms = a.maxseg;
  long long links = 0, skipped = 0;
  double m = 0., s0 = 0., w0 = 0.;
  for (long g = threadIdx.x; g < nr * ms; g += 256) {
    links += a.seg_links[g];
    skipped += a.seg_skip[g];
    m = fmax(m, a.seg_max[g * 3]);
  }
  for (long r0 = 0; r0 < nr; r0 += 2048) {
    const int n = (int)min(2048l, nr - r0);
    for (int k = threadIdx.x; k < n; k += 256) {
      ss[k] = a.row_sum[(r0 + k) * 3];
      sw[k] = a.row_w[(r0 + k) * 3];
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int k = 0; k < n; k++) {
        s0 = __dadd_rn(s0, ss[k]);
        w0 = __dadd_rn(w0, sw[k]);
      }
    __syncthreads();
  }
  for (int o = 16; o; o >>= 1) {
    links += __shfl_xor_sync(0xffffffffu, links, o);
    skipped += __shfl_xor_sync(0xffffffffu, skipped, o);
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    rl[threadIdx.x >> 5] = links;
    rs[threadIdx.x >> 5] = skipped;
    rm[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; w++) {
      links += rl[w];
      skipped += rs[w];
      m = fmax(m, rm[w]);
    }
    out[blockIdx.x * 3] = m;
    out[blockIdx.x * 3 + 1] = s0;
    out[blockIdx.x * 3 + 2] = w0;
    cnt[blockIdx.x * 2] = links;
    cnt[blockIdx.x * 2 + 1] = skipped;
  }
}

// -f hyphy: per matrix row the byte count, then the text: "\n{" d(r,0) "," ... "}" with 0 on the diagonal, the
// reported distance where the pair was reported and 100 elsewhere (swifttn93.cpp:2869-2897)
__device__ __forceinline__ int hy_entry(const double *hy, long N, long r, long c, char *buf)
{
  if (c == r) {
    buf[0] = '0';
    return 1;
  }
  const double d = hy[(size_t)r * N + c];
  if (d != d) {
    buf[0] = '1';
    buf[1] = '0';
    buf[2] = '0';
    return 3;
  }
  return fmt_g(d, buf);
}

__global__ void hy_len_kernel(const double *hy, long N, unsigned long long *row_bytes)
{
  const int lane = threadIdx.x & 31;
  const long r = blockIdx.x * (long)kWarps + (threadIdx.x >> 5);
  if (r >= N) return;
  unsigned long long b = 0;
  for (long c = lane; c < N; c += 32) {
    char t[24];
    b += hy_entry(hy, N, r, c, t) + (c ? 1 : 0);
  }
  for (int o = 16; o; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
  if (lane == 0) row_bytes[r] = b + 3;  // "\n{" and "}"
}

__global__ void hy_write_kernel(const double *hy, long N, const unsigned long long *row_off, char *out)
{
  const int lane = threadIdx.x & 31;
  const long r = blockIdx.x * (long)kWarps + (threadIdx.x >> 5);
  if (r >= N) return;
  char *o = out + row_off[r];
  if (lane == 0) {
    o[0] = '\n';
    o[1] = '{';
  }
  o += 2;
  for (long c0 = 0; c0 < N; c0 += 32) {
    const long c = c0 + lane;
    char t[24];
    int len = 0;
    if (c < N) len = hy_entry(hy, N, r, c, t) + (c ? 1 : 0);
    int pre = len;
    for (int s = 1; s < 32; s <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, pre, s);
      if (lane >= s) pre += v;
    }
    const int total = __shfl_sync(0xffffffffu, pre, 31);
    if (c < N) {
      char *p = o + (pre - len);
      if (c) *p++ = ',';
      put_bytes(p, t, len - (c ? 1 : 0));
    }
    o += total;
  }
  if (lane == 0) *o = '}';
}

__global__ void fill_nan_kernel(double *p, size_t n)
{
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    p[k] = __longlong_as_double(0x7FF8000000000000ll);
}

// Kernel attributes (the opt-in to more than 48 KB of dynamic shared memory) belong to each device's context, so
// they are set once per device. PerDevice::once runs set() for the current device unless it already succeeded
// there; callers on other threads wait for it (the lock is held while set() runs), and a failed set() is retried
// by the next call, so no launch can see the flag before the attribute is in place.
struct PerDevice {
  std::mutex mu;
  std::atomic<unsigned long long> done{0};
  template <class F>
  cudaError_t once(F set)
  {
    int d = 0;
    cudaError_t e = cudaGetDevice(&d);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (d & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    std::lock_guard<std::mutex> g(mu);
    if (done.load(std::memory_order_relaxed) & bit) return cudaSuccess;
    e = set();
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
    return e;
  }
};

// pair kernel launch (dynamic shared memory above the 48 KB default needs the opt-in attribute once per device).
// Register budgets: 2 blocks per SM (128 registers, no spills) and 3 (80 registers, some spills) for the fused
// kernel; 4 (64 registers) for the split kernel, which holds no formula state.
template <int MINB, bool SPLIT>
cudaError_t launch_pair_t(const PairArgs &A, dim3 g, cudaStream_t st)
{
  static PerDevice attr;
  cudaError_t e = attr.once([] {
    cudaError_t r;
    if ((r = cudaFuncSetAttribute(pair_kernel<false, false, MINB, SPLIT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmem)) != cudaSuccess)
      return r;
    if ((r = cudaFuncSetAttribute(pair_kernel<true, false, MINB, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kPairSmem)) != cudaSuccess)
      return r;
    return cudaFuncSetAttribute(pair_kernel<true, true, MINB, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kPairSmem);
  });
  if (e != cudaSuccess) return e;
  if (A.rc.wplane) {
    if (A.rc.gapmm)
      pair_kernel<true, true, MINB, SPLIT><<<g, 256, kPairSmem, st>>>(A);
    else
      pair_kernel<true, false, MINB, SPLIT><<<g, 256, kPairSmem, st>>>(A);
  } else
    pair_kernel<false, false, MINB, SPLIT><<<g, 256, kPairSmem, st>>>(A);
  return cudaGetLastError();
}

// Whether the tensor-core path splits the pair stage into the event kernel and formula_kernel. One fused kernel
// overlaps the formula with the event sums and is the faster form on the 6,700 x 1,500 HIV benchmark set in every
// mode once the event loads are batched (fused 3.31 / 5.44 ms vs split 3.62 / 6.13 ms per resolve / gapmm pair
// stage), so it is the default; TN93G_PAIR_SPLIT=1 selects the split form, which gives the same bytes.
int pair_split(const RunConsts &)
{
  static const int v = [] {
    const char *e = getenv("TN93G_PAIR_SPLIT");
    return e && atoi(e) ? 1 : 0;
  }();
  return v;
}

// Resident blocks per SM with the tensor-core counts: 4 (64 registers a thread) when the N plane is off, 3 (80) when
// it is on (6,700 x 1,500 benchmark set, same box: resolve 3.18 ms with 4 vs 3.25 ms with 3 per pair stage, gapmm
// 3.82 ms with 3 vs 3.89 ms with 4; 2 blocks, 128 registers without spills, 3.60 ms under resolve); 2 with the
// popcount loop, which needs the registers. TN93G_PAIR_BLOCKS=2|3|4 overrides.
cudaError_t launch_pair(const PairArgs &A, long ncolblocks, long nrows, cudaStream_t st)
{
  static const int forced = [] {
    const char *e = getenv("TN93G_PAIR_BLOCKS");
    return e ? (atoi(e) == 4 ? 4 : atoi(e) == 3 ? 3 : 2) : 0;
  }();
  dim3 g((unsigned)ncolblocks, (unsigned)((nrows + kTile - 1) / kTile));
  if (A.split && A.tcagg) {
    cudaError_t e = launch_pair_t<4, true>(A, g, st);
    if (e != cudaSuccess) return e;
    const long ncol = ncolblocks * kTile;
    // a few row groups per launch: each thread takes many rows, so that its ambiguity bounds and counters reach the
    // global atomics once per launch, not once per row
    const dim3 gf((unsigned)((ncol + 255) / 256), (unsigned)std::min<long>(nrows, 16));
    static const int fb = [] {
      const char *v = getenv("TN93G_FORMULA_BLOCKS");  // tuning knob: 2 (128 registers) or 3 (80)
      return v && atoi(v) == 2 ? 2 : 3;
    }();
    if (fb == 2) {
      if (A.tc16)
        formula_kernel<true, 2><<<gf, 256, 0, st>>>(A, ncol);
      else
        formula_kernel<false, 2><<<gf, 256, 0, st>>>(A, ncol);
    } else {
      if (A.tc16)
        formula_kernel<true, 3><<<gf, 256, 0, st>>>(A, ncol);
      else
        formula_kernel<false, 3><<<gf, 256, 0, st>>>(A, ncol);
    }
    return cudaGetLastError();
  }
  const int minb = forced ? forced : (A.tcagg ? (A.rc.wplane ? 3 : 4) : 2);
  if (minb == 4) return launch_pair_t<4, false>(A, g, st);
  return minb == 3 ? launch_pair_t<3, false>(A, g, st) : launch_pair_t<2, false>(A, g, st);
}

// the tensor-core count kernels' opt-in to their dynamic shared memory, once per device
cudaError_t tc_attr_once()
{
  static PerDevice attr;
  return attr.once([] {
    cudaError_t e = cudaFuncSetAttribute(count_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(count_tc_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(count_tc_persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPSmem);
  });
}

// TN93G_TC_KERNEL=tile selects the one-tile-per-CTA count kernel instead of the persistent one (same records)
bool tc_tile_kernel()
{
  static const bool tile = [] {
    const char *e = getenv("TN93G_TC_KERNEL");
    return e && strcmp(e, "tile") == 0;
  }();
  return tile;
}

// Tensor-core counts over the count_tc_kernel grid (gx column tiles x gy row tiles) of T: the persistent kernel on
// min(tiles, SMs) CTAs, or one CTA per tile.
cudaError_t launch_count_grid(const TcArgs &T, long gx, long gy, int sms, cudaStream_t st)
{
  cudaError_t e = tc_attr_once();
  if (e != cudaSuccess) return e;
  if (tc_tile_kernel()) {
    count_tc_kernel<<<dim3((unsigned)gx, (unsigned)gy), 128, kTcSmem, st>>>(T);
  } else {
    const long nt = gx * gy;
    count_tc_persist_kernel<<<(unsigned)std::min<long>(nt, sms), kPThreads, kPSmem, st>>>(T, nullptr, nullptr, 0);
  }
  return cudaGetLastError();
}

// the same over a list of (descriptor, first row, first column) tiles; G carries the wait limit, the error word
// and the test hook for the persistent kernel
cudaError_t launch_count_list(const TcArgs &G, const TcArgs *descs, const int4 *tiles, int ntiles, int sms,
                              cudaStream_t st)
{
  cudaError_t e = tc_attr_once();
  if (e != cudaSuccess) return e;
  if (tc_tile_kernel())
    count_tc_batch_kernel<<<(unsigned)ntiles, 128, kTcSmem, st>>>(descs, tiles);
  else
    count_tc_persist_kernel<<<(unsigned)std::min(ntiles, sms), kPThreads, kPSmem, st>>>(G, descs, tiles, ntiles);
  return cudaGetLastError();
}

}  // namespace

//================================================================================================== host side

struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
};

constexpr int kBatchBufs = 56;
constexpr int kMaxTcChunks = 48;         // row chunks of a band on the tensor-core count path
// Pairs per chunk of the tensor-core path (count kernel, then pair kernel): 16 M pairs, 256 MB of 16-byte records.
// Larger chunks amortise the persistent count kernel's pipeline fill and drain and the pair kernel's last wave
// (6,700 x 1,500 benchmark set, resolve pair stage per 22.4 M pairs: 3.17 ms with 2 M-pair chunks, 2.94 with 4 M,
// 2.77 with 8 M, 2.71 with 16 M, 2.67 with one chunk); the records then travel through HBM, which the pair stage
// leaves almost idle. TN93G_TC_CHUNK_PAIRS overrides.
constexpr long kTcChunkPairs = 16l << 20;

struct tn93g_set {
  long N = 0, L = 0;
  size_t cap[5] = {0, 0, 0, 0, 0};  // bytes of d_codes, d_counts, d_names, d_name_off, d_name_len
  uint8_t *d_codes = nullptr;
  long *d_counts = nullptr;
  char *d_names = nullptr;
  uint64_t *d_name_off = nullptr;
  int32_t *d_name_len = nullptr;
  std::vector<long> counts, name_len;
};

struct tn93g_ctx {
  int device = 0;
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  LogTable *d_logt = nullptr;
  Tables *h_tab = nullptr;
  PairTables *h_ptab = nullptr;  // host staging of the pair stage's tables
  DevBuf seen, nN, varcol, planes, cc, ccT, evcount, evoff, ev, agg, site, dist, dcode, wcount, wloff, wl, rq, rqn, counters,
      rbytes, rsum, rw, fraw, fspan, flen, fcode,
      rmax, rlinks, rskip, hist, roff, out, hy;
  void *pinned = nullptr;
  size_t pinned_n = 0;
  cudaEvent_t evs[16];
  cudaStream_t copy_stream = nullptr;   // device->host copies of finished bands
  cudaStream_t write_stream = nullptr;  // text writers of finished bands (beside the next bands' kernels)
  cudaEvent_t evw0[2], evw1[2], evc0[2], evc1[2];
  cudaEvent_t evk[2][5];  // per band parity: start, after pair, after replay, after stats+sums+scan, stats on host
  cudaEvent_t evcnt[2][2 * kMaxTcChunks];  // per band parity: around each chunk's tensor-core count kernel
  DevBuf out2[2], total;
  void *pin2[2] = {nullptr, nullptr};
  size_t pin2_n[2] = {0, 0};
  void *pstats = nullptr;
  size_t pstats_n = 0;
  // device buffers of freed sets, kept for the next upload (repeated upload/free skips the allocator)
  std::vector<std::pair<void *, size_t>> set_pool;
  double timings[8] = {0};
  long launches = 0;
  size_t dev_out_n = 0;
  DevBuf bb[kBatchBufs];  // buffers of tn93g_batch_run (indexed by BatchBuf)
  int count_path = 1;  // clean-site counts: 0 popcounts on the CUDA cores, 1 tensor cores (tcgen05)
  int sms = 148;       // streaming multiprocessors of the device (persistent and grid-stride launches)
  DevBuf ohimg, tcagg, tcerr;
  uint64_t wait_ns = kTcWaitNs;  // limit of each bounded device wait
  bool exact_sums = false;       // tn93g_set_exact_sums
  int fault = TN93G_FAULT_NONE;  // test hook for the next run (tn93g_inject_fault)
  // exactness: undecided lists and counts per band parity, the summary units' bounds, the resolver's entries and
  // run descriptors, and the logarithm's band and candidate spread (tn93g_set_log_band)
  DevBuf und[2], undn, amb, undwork, rdesc;
  double log_band = kLogBand, log_spread = kLogSpread;
};

namespace {

#define CU(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                  \
      return e_ == cudaErrorMemoryAllocation ? TN93G_ENOMEM : TN93G_ECUDA;            \
    }                                                                                 \
  } while (0)

int ensure(tn93g_ctx *ctx, DevBuf &b, size_t bytes)
{
  if (bytes <= b.n && b.p) return TN93G_OK;
  if (b.p) {
    cudaFree(b.p);
    ctx->used -= b.n;
    b.p = nullptr;
    b.n = 0;
  }
  bytes = std::max<size_t>(bytes, 256);
  if (ctx->budget && ctx->used + bytes > ctx->budget) {
    ctx->err = "over the context's HBM budget";
    return TN93G_ENOMEM;
  }
  CU(cudaMalloc(&b.p, bytes));
  b.n = bytes;
  ctx->used += bytes;
  return TN93G_OK;
}

int ensure_pinned(tn93g_ctx *ctx, size_t bytes)
{
  if (bytes <= ctx->pinned_n) return TN93G_OK;
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  ctx->pinned = nullptr;
  ctx->pinned_n = 0;
  bytes = std::max<size_t>(bytes + bytes / 4, 1 << 20);
  CU(cudaHostAlloc(&ctx->pinned, bytes, cudaHostAllocDefault));
  ctx->pinned_n = bytes;
  return TN93G_OK;
}

int ensure_pinned_at(tn93g_ctx *ctx, void *&p, size_t &n, size_t bytes, unsigned flags = cudaHostAllocDefault)
{
  if (bytes <= n && p) return TN93G_OK;
  if (p) cudaFreeHost(p);
  p = nullptr;
  n = 0;
  bytes = std::max<size_t>(bytes + bytes / 4, 1 << 20);
  CU(cudaHostAlloc(&p, bytes, flags));
  n = bytes;
  return TN93G_OK;
}

// grows b to `bytes`, keeping its first `keep` bytes (stream-ordered copy)
int ensure_keep(tn93g_ctx *ctx, DevBuf &b, size_t bytes, size_t keep)
{
  if (bytes <= b.n && b.p) return TN93G_OK;
  bytes = std::max<size_t>(bytes + bytes / 2, 1 << 20);
  if (ctx->budget && ctx->used + bytes > ctx->budget) {
    ctx->err = "over the context's HBM budget";
    return TN93G_ENOMEM;
  }
  void *p = nullptr;
  CU(cudaMalloc(&p, bytes));
  if (keep && b.p) CU(cudaMemcpyAsync(p, b.p, keep, cudaMemcpyDeviceToDevice, ctx->stream));
  if (b.p) {
    CU(cudaStreamSynchronize(ctx->stream));
    cudaFree(b.p);
    ctx->used -= b.n;
  }
  b.p = p;
  b.n = bytes;
  ctx->used += bytes;
  return TN93G_OK;
}

#define TRY(x)                   \
  do {                           \
    int r_ = (x);                \
    if (r_ != TN93G_OK) return r_; \
  } while (0)

// The host's C library log of every listed argument: the decision oracle for pairs whose printed bytes or
// decisions depend on how that log rounds (the reference calls the same function, swifttn93.cpp:1954-2001).
// Large lists (resolve-all passes) are split over the host's threads.
void host_logs(std::vector<UndEntry> &E)
{
  auto work = [&E](size_t b, size_t e) {
    for (size_t k = b; k < e; k++)
      for (int q = 0; q < 3; q++) E[k].lg[q] = q < E[k].nlog ? log(E[k].arg[q]) : 0.;
  };
  const size_t n = E.size();
  const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), (unsigned)(n / 65536 + 1)));
  if (nt == 1) {
    work(0, n);
    return;
  }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; t++) th.emplace_back(work, n * t / nt, n * (t + 1) / nt);
  for (auto &t : th) t.join();
}

// Finishes the n listed pairs (entries (k, i << 32 | j), run k described by d_descs[k] in device memory) with the
// C library's logarithms: the site-order walk gives each pair's formula arguments on the device, the host takes
// their logs, and the device evaluates the formula with them into the pair's raw-distance slot.
int resolve_listed(tn93g_ctx *ctx, const ReplayArgs *d_descs, const unsigned long long *d_list, unsigned n,
                   cudaStream_t st)
{
  if (!n) return TN93G_OK;
  TRY(ensure(ctx, ctx->undwork, (size_t)n * sizeof(UndEntry)));
  UndEntry *dw = (UndEntry *)ctx->undwork.p;
  und_args_kernel<<<(unsigned)std::min<unsigned long>((n + kWarps - 1) / kWarps, 8ul * ctx->sms), 256, 0, st>>>(
      d_descs, d_list, n, dw);
  CU(cudaGetLastError());
  std::vector<UndEntry> h(n);
  CU(cudaMemcpyAsync(h.data(), dw, (size_t)n * sizeof(UndEntry), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  host_logs(h);
  CU(cudaMemcpyAsync(dw, h.data(), (size_t)n * sizeof(UndEntry), cudaMemcpyHostToDevice, st));
  und_finish_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_descs, dw, n);
  CU(cudaGetLastError());
  ctx->launches += 2;
  return TN93G_OK;
}

// a tn93g_sink that appends to the std::string at user
int append_sink(void *user, const char *bytes, size_t n)
{
  static_cast<std::string *>(user)->append(bytes, n);
  return 0;
}

// the pair stage's tables for a run: the x16 event table (with the N-plane entries) and its packed form
void fill_pair_tables(const Tables &T, bool wplane, PairTables *out)
{
  memcpy(out->agg, T.ev, sizeof out->agg);
  pack_tables(T, wplane, &out->packed);
}

// the summary units' bounds (ExactSink::amb words) as doubles: {largest low, largest high, spread, count}
void amb_bounds(const unsigned long long *w, double out[4])
{
  memcpy(&out[0], &w[0], 8);
  memcpy(&out[1], &w[1], 8);
  memcpy(&out[2], &w[2], 8);
  out[3] = (double)w[3];
}

}  // namespace

namespace tn93 {
bool summary_certified(const tn93g_summary *s, const double bounds[3][4], long chain, int fst);
}

extern "C" {

const char *tn93g_strerror(int code)
{
  switch (code) {
    case TN93G_OK: return "ok";
    case TN93G_EINVAL: return "invalid argument";
    case TN93G_ECUDA: return "CUDA runtime error";
    case TN93G_ENOMEM: return "out of device or pinned memory";
    case TN93G_ESINK: return "output callback aborted the run";
    case TN93G_ENODEV: return "no usable CUDA device";
    case TN93G_ETIMEOUT: return "device wait timed out";
    case TN93G_ETOOBIG: return "alignment too long (L >= 2^25)";
    case TN93G_ESCRATCH: return "alignment exceeds the allocation-free entry point's limits (N <= 512, L <= 4096)";
    case TN93G_EFASTA: return "the FASTA reader refused the input";
    case TN93G_EUNDECIDED: return "a distance could not be decided exactly";
    default: return "unknown error";
  }
}

const char *tn93g_last_cuda_error(tn93g_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

int tn93g_set_count_path(tn93g_ctx *ctx, int path)
{
  if (!ctx || path < 0 || path > 1) return TN93G_EINVAL;
  ctx->count_path = path;
  return TN93G_OK;
}

int tn93g_set_log_band(tn93g_ctx *ctx, double band_ulps, double spread_ulps)
{
  if (!ctx || !(band_ulps >= kLogBand && band_ulps <= 0.5) || !(spread_ulps >= 1.0 && spread_ulps <= 0x1p40))
    return TN93G_EINVAL;
  ctx->log_band = band_ulps;
  ctx->log_spread = floor(spread_ulps);
  return TN93G_OK;
}

int tn93g_set_exact_sums(tn93g_ctx *ctx, int on)
{
  if (!ctx) return TN93G_EINVAL;
  ctx->exact_sums = on != 0;
  return TN93G_OK;
}

int tn93g_set_wait_limit(tn93g_ctx *ctx, double seconds)
{
  if (!ctx || !(seconds > 0. && seconds <= 60.)) return TN93G_EINVAL;
  ctx->wait_ns = (uint64_t)(seconds * 1e9);
  return TN93G_OK;
}

int tn93g_inject_fault(tn93g_ctx *ctx, int fault)
{
  if (!ctx || fault < TN93G_FAULT_NONE || fault > TN93G_FAULT_SKIP_FILL) return TN93G_EINVAL;
  ctx->fault = fault;
  return TN93G_OK;
}

// Copies up to nine ranges of 8-byte words into pinned host memory that the device maps (a band's statistics), so
// that they reach the host without a copy-engine transfer, which would queue behind the band texts in flight.
struct Gather {
  const unsigned long long *src[9];
  unsigned long long *dst[9];
  long n[9];
  int k;
};

__global__ void __launch_bounds__(256) gather_kernel(Gather g)
{
  const long stride = (long)gridDim.x * blockDim.x;
  for (int r = 0; r < g.k; r++)
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < g.n[r]; t += stride) g.dst[r][t] = g.src[r][t];
}

//------------------------------------------------------------------------------------------------ self-test
// one thread per input: the formula up to its logarithms (in: nf[4], diag, ag, ct; out: nlog, k2p, K1..K3, arg[3]),
// and the quotient xb[0] / xb[1] by div_by against the device's division (bad: differing bits)
__global__ void selftest_division_kernel(const double *in, double *out, const double *xb, long n,
                                         unsigned long long *bad)
{
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double *p = in + 7 * t;
  const double nf[4] = {p[0], p[1], p[2], p[3]};
  const Prep P = tn93_prep(nf, p[4], p[5], p[6]);
  double *o = out + 8 * t;
  o[0] = P.nlog;
  o[1] = P.k2p;
  o[2] = P.K1;
  o[3] = P.K2;
  o[4] = P.K3;
  o[5] = P.arg[0];
  o[6] = P.arg[1];
  o[7] = P.arg[2];
  const double x = xb[2 * t], b = xb[2 * t + 1];
  const double q = div_by(x, b, __ddiv_rn(1.0, b)), r = __ddiv_rn(x, b);
  if (__double_as_longlong(q) != __double_as_longlong(r)) atomicAdd(bad, 1ull);
}

int tn93g_selftest_division(tn93g_ctx *ctx, long n, unsigned long long seed, long mismatches[2])
{
  if (!ctx || n <= 0 || !mismatches) return TN93G_EINVAL;
  cudaSetDevice(ctx->device);
  uint64_t st = seed * 2654435761ull + 0x9E3779B97F4A7C15ull;
  auto rnd = [&]() {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return st;
  };
  std::vector<double> in(7 * (size_t)n), out(8 * (size_t)n), xb(2 * (size_t)n);
  for (long t = 0; t < n; t++) {
    // counts as the pair kernel forms them: T clean-equivalent sites (sixteenths), base totals over both sequences
    // summing to 2T, matches, and A<->G / C<->T transitions among the mismatches; some inputs have a base absent
    // (K2P) or more mismatches than the formula takes (no logarithms)
    const long L = 50 + (long)(rnd() % 30000);
    const long T16 = 16 * (L / 2) + (long)(rnd() % (16 * (L / 2)));
    long rest = 2 * T16, nf16[4];
    for (int k = 0; k < 3; k++) {
      nf16[k] = (rnd() % 8 == 0) ? 0 : (long)(rnd() % (uint64_t)(rest / 2 + 1));
      rest -= nf16[k];
    }
    nf16[3] = rest;
    const long mis16 = (long)(rnd() % (uint64_t)(T16 / (rnd() % 4 == 0 ? 1 : 8) + 1));
    const long ag16 = (long)(rnd() % (uint64_t)(mis16 + 1)), ct16 = (long)(rnd() % (uint64_t)(mis16 - ag16 + 1));
    double *p = &in[7 * (size_t)t];
    for (int k = 0; k < 4; k++) p[k] = (double)nf16[k] / 16.0;
    p[4] = (double)(T16 - mis16) / 16.0;
    p[5] = (double)ag16 / 16.0;
    p[6] = (double)ct16 / 16.0;
    // quotients over 80 binades of divisor, either sign of dividend
    const double m = 1.0 + (double)(rnd() >> 12) * 0x1p-52, mb = 1.0 + (double)(rnd() >> 12) * 0x1p-52;
    const int ex = (int)(rnd() % 81) - 40, eb = (int)(rnd() % 81) - 40;
    xb[2 * (size_t)t] = ldexp(rnd() & 1 ? -m : m, ex);
    xb[2 * (size_t)t + 1] = ldexp(mb, eb);
  }
  DevBuf din, dout, dxb, dbad;
  const cudaStream_t st2 = ctx->stream;
  int rc = TN93G_OK;
  do {
    if ((rc = ensure(ctx, din, in.size() * 8)) != TN93G_OK || (rc = ensure(ctx, dout, out.size() * 8)) != TN93G_OK ||
        (rc = ensure(ctx, dxb, xb.size() * 8)) != TN93G_OK || (rc = ensure(ctx, dbad, 8)) != TN93G_OK)
      break;
    unsigned long long bad = 0;
    if (cudaMemcpyAsync(din.p, in.data(), in.size() * 8, cudaMemcpyHostToDevice, st2) != cudaSuccess ||
        cudaMemcpyAsync(dxb.p, xb.data(), xb.size() * 8, cudaMemcpyHostToDevice, st2) != cudaSuccess ||
        cudaMemsetAsync(dbad.p, 0, 8, st2) != cudaSuccess) {
      rc = TN93G_ECUDA;
      break;
    }
    selftest_division_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st2>>>(
        (const double *)din.p, (double *)dout.p, (const double *)dxb.p, n, (unsigned long long *)dbad.p);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(out.data(), dout.p, out.size() * 8, cudaMemcpyDeviceToHost, st2) != cudaSuccess ||
        cudaMemcpyAsync(&bad, dbad.p, 8, cudaMemcpyDeviceToHost, st2) != cudaSuccess ||
        cudaStreamSynchronize(st2) != cudaSuccess) {
      rc = TN93G_ECUDA;
      break;
    }
    long diff = 0;
    for (long t = 0; t < n; t++) {
      const double *p = &in[7 * (size_t)t];
      const double nf[4] = {p[0], p[1], p[2], p[3]};
      const Prep P = tn93_prep(nf, p[4], p[5], p[6]);
      const double want[8] = {(double)P.nlog, (double)P.k2p, P.K1, P.K2, P.K3, P.arg[0], P.arg[1], P.arg[2]};
      if (memcmp(want, &out[8 * (size_t)t], sizeof want) != 0) diff++;
    }
    mismatches[0] = diff;
    mismatches[1] = (long)bad;
  } while (0);
  for (DevBuf *b : {&din, &dout, &dxb, &dbad})
    if (b->p) {
      cudaFree(b->p);
      ctx->used -= b->n;
    }
  return rc;
}

int tn93g_create(tn93g_ctx **out, int device, size_t hbm_budget)
{
  if (!out) return TN93G_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return TN93G_ENODEV;
  tn93g_ctx *ctx = new tn93g_ctx();
  ctx->device = device;
  ctx->budget = hbm_budget;
  int rc = TN93G_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess) {
      rc = TN93G_ENODEV;
      break;
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      rc = TN93G_ECUDA;
      break;
    }
    for (auto &e : ctx->evs)
      if (cudaEventCreate(&e) != cudaSuccess) rc = TN93G_ECUDA;
    for (int q = 0; q < 2; q++) {
      if (cudaEventCreate(&ctx->evw0[q]) != cudaSuccess || cudaEventCreate(&ctx->evw1[q]) != cudaSuccess ||
          cudaEventCreate(&ctx->evc0[q]) != cudaSuccess || cudaEventCreate(&ctx->evc1[q]) != cudaSuccess)
        rc = TN93G_ECUDA;
      for (auto &e : ctx->evk[q])
        if (cudaEventCreate(&e) != cudaSuccess) rc = TN93G_ECUDA;
      for (auto &e : ctx->evcnt[q])
        if (cudaEventCreate(&e) != cudaSuccess) rc = TN93G_ECUDA;
    }
    if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) rc = TN93G_ECUDA;
    if (cudaStreamCreateWithFlags(&ctx->write_stream, cudaStreamNonBlocking) != cudaSuccess) rc = TN93G_ECUDA;
    if (const char *e = getenv("TN93G_COUNT")) ctx->count_path = strcmp(e, "popc") == 0 ? 0 : 1;
    {
      const char *b = getenv("TN93G_LOG_BAND"), *p = getenv("TN93G_LOG_SPREAD");
      if (b || p) tn93g_set_log_band(ctx, b ? atof(b) : kLogBand, p ? atof(p) : kLogSpread);
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
      ctx->sms = sms;
    LogTable h;
    build_log_table(&h);
    if (cudaMalloc(&ctx->d_logt, sizeof(LogTable)) != cudaSuccess ||
        cudaMemcpy(ctx->d_logt, &h, sizeof h, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = TN93G_ECUDA;
    ctx->h_tab = new Tables();
    ctx->h_ptab = new PairTables();
  } while (0);
  if (rc != TN93G_OK) {
    tn93g_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return TN93G_OK;
}

void tn93g_destroy(tn93g_ctx *ctx)
{
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  DevBuf *bufs[] = {&ctx->seen, &ctx->nN, &ctx->varcol, &ctx->planes, &ctx->cc, &ctx->ccT, &ctx->evcount,
                    &ctx->evoff, &ctx->ev, &ctx->agg, &ctx->site, &ctx->dist, &ctx->dcode, &ctx->wcount, &ctx->wloff, &ctx->wl, &ctx->fraw, &ctx->fspan, &ctx->flen, &ctx->fcode, &ctx->rq, &ctx->rqn, &ctx->counters,
                    &ctx->rbytes, &ctx->rsum, &ctx->rw, &ctx->rmax, &ctx->rlinks, &ctx->rskip, &ctx->hist,
                    &ctx->roff, &ctx->out, &ctx->hy};
  for (DevBuf *b : bufs)
    if (b->p) cudaFree(b->p);
  for (DevBuf &b : ctx->bb)
    if (b.p) cudaFree(b.p);
  for (DevBuf *b : {&ctx->ohimg, &ctx->tcagg, &ctx->tcerr, &ctx->und[0], &ctx->und[1], &ctx->undn, &ctx->amb,
                    &ctx->undwork, &ctx->rdesc})
    if (b->p) cudaFree(b->p);
  if (ctx->d_logt) cudaFree(ctx->d_logt);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  for (int q = 0; q < 2; q++) {
    if (ctx->out2[q].p) cudaFree(ctx->out2[q].p);
    if (ctx->pin2[q]) cudaFreeHost(ctx->pin2[q]);
    for (cudaEvent_t e : {ctx->evw0[q], ctx->evw1[q], ctx->evc0[q], ctx->evc1[q]})
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->evk[q])
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->evcnt[q])
      if (e) cudaEventDestroy(e);
  }
  if (ctx->total.p) cudaFree(ctx->total.p);
  for (auto &b : ctx->set_pool) cudaFree(b.first);
  if (ctx->pstats) cudaFreeHost(ctx->pstats);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->write_stream) cudaStreamDestroy(ctx->write_stream);
  for (auto &e : ctx->evs)
    if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx->h_tab;
  delete ctx->h_ptab;
  delete ctx;
}

// A new set from codes (host memory, or device memory when codes_kind says so), copy numbers and names (host).
static int upload_set(tn93g_ctx *ctx, tn93g_set **out, const uint8_t *codes, cudaMemcpyKind codes_kind, long N, long L,
                      const long *copy_counts, const char *names, const size_t *name_off, const long *name_len);

int tn93g_upload(tn93g_ctx *ctx, tn93g_set **out, const uint8_t *codes, long N, long L, const long *copy_counts,
                 const char *names, const size_t *name_off, const long *name_len)
{
  return upload_set(ctx, out, codes, cudaMemcpyHostToDevice, N, L, copy_counts, names, name_off, name_len);
}

static int upload_set(tn93g_ctx *ctx, tn93g_set **out, const uint8_t *codes, cudaMemcpyKind codes_kind, long N, long L,
                      const long *copy_counts, const char *names, const size_t *name_off, const long *name_len)
{
  if (!ctx || !out || !codes || N <= 0 || L <= 0 || !copy_counts || !names || !name_off || !name_len)
    return TN93G_EINVAL;
  if (L >= (1l << 25)) return TN93G_ETOOBIG;
  cudaSetDevice(ctx->device);
  tn93g_set *s = new tn93g_set();
  s->N = N;
  s->L = L;
  s->counts.assign(copy_counts, copy_counts + N);
  s->name_len.assign(name_len, name_len + N);
  size_t nbytes = 0;
  for (long i = 0; i < N; i++) nbytes = std::max(nbytes, name_off[i] + (size_t)name_len[i]);
  std::vector<uint64_t> off(name_off, name_off + N);
  std::vector<int32_t> nl(N);
  for (long i = 0; i < N; i++) nl[i] = (int32_t)name_len[i];
  auto fail = [&](cudaError_t e) {
    ctx->err = cudaGetErrorString(e);
    tn93g_free_set(ctx, s);
    return e == cudaErrorMemoryAllocation ? TN93G_ENOMEM : TN93G_ECUDA;
  };
  cudaError_t e;
  // smallest pooled buffer that fits, else a new allocation
  auto take = [&](void **p, size_t bytes, int k) -> cudaError_t {
    bytes = std::max<size_t>(bytes, 256);
    long best = -1;
    for (size_t q = 0; q < ctx->set_pool.size(); q++)
      if (ctx->set_pool[q].second >= bytes && (best < 0 || ctx->set_pool[q].second < ctx->set_pool[best].second))
        best = (long)q;
    if (best >= 0) {
      *p = ctx->set_pool[best].first;
      s->cap[k] = ctx->set_pool[best].second;
      ctx->set_pool.erase(ctx->set_pool.begin() + best);
      return cudaSuccess;
    }
    s->cap[k] = bytes;
    return cudaMalloc(p, bytes);
  };
  if ((e = take((void **)&s->d_codes, (size_t)N * L, 0)) != cudaSuccess) return fail(e);
  if ((e = take((void **)&s->d_counts, N * sizeof(long), 1)) != cudaSuccess) return fail(e);
  if ((e = take((void **)&s->d_names, nbytes + 1, 2)) != cudaSuccess) return fail(e);
  if ((e = take((void **)&s->d_name_off, N * sizeof(uint64_t), 3)) != cudaSuccess) return fail(e);
  if ((e = take((void **)&s->d_name_len, N * sizeof(int32_t), 4)) != cudaSuccess) return fail(e);
  if ((e = cudaMemcpyAsync(s->d_codes, codes, (size_t)N * L, codes_kind, ctx->stream)) != cudaSuccess) return fail(e);
  if ((e = cudaMemcpyAsync(s->d_counts, copy_counts, N * sizeof(long), cudaMemcpyHostToDevice, ctx->stream)) !=
      cudaSuccess)
    return fail(e);
  if (nbytes && (e = cudaMemcpyAsync(s->d_names, names, nbytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
    return fail(e);
  if ((e = cudaMemcpyAsync(s->d_name_off, off.data(), N * sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream)) !=
      cudaSuccess)
    return fail(e);
  if ((e = cudaMemcpyAsync(s->d_name_len, nl.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream)) !=
      cudaSuccess)
    return fail(e);
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(e);
  *out = s;
  return TN93G_OK;
}

//------------------------------------------------------------------------------------------------ FASTA on device
// The byte map of tn93's reader: the index of a byte in "ACGTURYSWKMBDHVN?-" (either case), -1 for any other byte
struct ByteMap {
  signed char v[256];
};

static ByteMap make_byte_map()
{
  ByteMap m;
  static const char kValid[] = "ACGTURYSWKMBDHVN?-";
  for (int c = 0; c < 256; c++) {
    m.v[c] = -1;
    const int u = (c >= 'a' && c <= 'z') ? c - 32 : c;
    if (!u) continue;
    const char *f = strchr(kValid, u);
    if (f) m.v[c] = (signed char)(f - kValid);
  }
  return m;
}

// one warp per record: how many of the bytes in its sequence range [span.x, span.y) of raw are letters of the map
__global__ void __launch_bounds__(256) fasta_count_kernel(const unsigned char *raw, const ulonglong2 *spans, long m,
                                                          ByteMap map, long *len)
{
  __shared__ signed char sm[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) sm[t] = map.v[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long k = blockIdx.x * (long)kWarps + (threadIdx.x >> 5);
  if (k >= m) return;
  const unsigned long long b = spans[k].x, e = spans[k].y;
  long n = 0;
  for (unsigned long long p = b + lane; p < e; p += 32) n += sm[raw[p]] >= 0;
  for (int o = 16; o; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if (lane == 0) len[k] = n;
}

// one warp per record: its sequence letters mapped to codes and compressed, in file order, to codes[k * L ...] (every
// record has L letters, checked on the host before the launch)
__global__ void __launch_bounds__(256) fasta_compress_kernel(const unsigned char *raw, const ulonglong2 *spans, long m,
                                                             ByteMap map, long L, uint8_t *codes)
{
  __shared__ signed char sm[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) sm[t] = map.v[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long k = blockIdx.x * (long)kWarps + (threadIdx.x >> 5);
  if (k >= m) return;
  const unsigned long long b = spans[k].x, e = spans[k].y;
  uint8_t *row = codes + (size_t)k * L;
  long base = 0;
  for (unsigned long long p0 = b; p0 < e; p0 += 32) {
    const unsigned long long p = p0 + lane;
    const int v = p < e ? sm[raw[p]] : -1;
    const unsigned mask = __ballot_sync(0xffffffffu, v >= 0);
    if (v >= 0) row[base + __popc(mask & ((1u << lane) - 1u))] = (uint8_t)v;
    base += __popc(mask);
  }
}

// The records of a FASTA file as tn93's reader finds them (swifttn93.cpp:259-406): '>' or '#' opens a record whose
// name runs to the end of the line, and its sequence is every byte up to the next '>' or '#'. memchr (vectorised in
// the C library) finds those bytes, so the host does not touch the sequence letters.
struct FastaRecords {
  std::vector<char> names;
  std::vector<size_t> name_off;
  std::vector<long> name_len, counts;
  std::vector<ulonglong2> spans;
  int eof_state = 2;     // the reader's state at the end of the file (2: inside a sequence, the normal end)
  std::string name_err;  // the record after the last span has an empty name (reported after the spans' lengths)
};

static void fasta_records(const char *bytes, size_t n, char counts_sep, FastaRecords &R)
{
  // the next '>' and '#' at or after the last search start (n: none); still the next ones for any later start that
  // does not pass them
  size_t ngt = 0, nhs = 0;
  bool have = false;
  auto next_open = [&](size_t i) -> size_t {
    if (!have || ngt < i) {
      const void *g = i < n ? memchr(bytes + i, '>', n - i) : nullptr;
      ngt = g ? (size_t)((const char *)g - bytes) : n;
    }
    if (!have || nhs < i) {
      const void *h = i < n ? memchr(bytes + i, '#', n - i) : nullptr;
      nhs = h ? (size_t)((const char *)h - bytes) : n;
    }
    have = true;
    return std::min(ngt, nhs);
  };
  size_t o = next_open(0);
  if (o == n) {
    R.eof_state = 0;
    return;
  }
  size_t i = o + 1;
  for (;;) {
    size_t q = i;
    while (q < n && bytes[q] != '\n' && bytes[q] != '\r') q++;
    if (q == n) {
      R.eof_state = 1;
      return;
    }
    const long len = (long)(q - i);
    if (len <= 0) {
      R.name_err = "Sequence names must be non-empty.\n";
      return;
    }
    const size_t begin = R.names.size();
    R.names.insert(R.names.end(), bytes + i, bytes + q);
    R.names.push_back('\0');
    unsigned long count = 1;
    if (len >= 3) {
      const char *nm = R.names.data() + begin;
      long k = len - 2;
      while (k >= 1 && nm[k] != counts_sep) k--;
      if (k >= 1) count = (unsigned long)(long)(int)strtol(nm + k + 1, nullptr, 10);
      if (count < 1) count = 1;
    }
    R.counts.push_back((long)count);
    R.name_off.push_back(begin);
    R.name_len.push_back(len);
    i = q + 1;
    o = next_open(i);
    R.spans.push_back(make_ulonglong2(i, o));
    if (o == n) {
      R.eof_state = 2;
      return;
    }
    i = o + 1;
  }
}

// The reader's checks in its order, given each record's letter count: each length when its sequence closes, then
// what stopped the scan. Returns the message (empty when the file is accepted) and the length in *first_len.
static std::string fasta_check(const FastaRecords &R, const std::vector<long> &lens, long expect_len, long *first_len)
{
  std::string err;
  const long m = (long)R.spans.size();
  const bool have_len = expect_len > 0;
  long L = have_len ? expect_len : 0;
  for (long k = 0; k < m && err.empty(); k++) {
    if (k == 0 && !have_len) {
      L = lens[0];
      if (L <= 0) err = "First sequence length must be positive.\n";
    } else if (lens[k] != L) {
      err = "All sequences must have the same length (" + std::to_string(L) + "), but sequence '" +
            std::string(R.names.data() + R.name_off[k]) + "' had length " + std::to_string(lens[k]);
    }
  }
  if (err.empty() && !R.name_err.empty()) err = R.name_err;
  if (err.empty() && R.eof_state != 2) err = "Unexpected end of file: state " + std::to_string(R.eof_state) + "\n";
  *first_len = L;
  return err;
}

static void copy_msg(const std::string &err, char *msg, size_t msg_cap)
{
  if (!msg || !msg_cap) return;
  const size_t k = err.size() < msg_cap ? err.size() : msg_cap - 1;
  memcpy(msg, err.data(), k);
  msg[k] = 0;
}

// The device ingest's host half with the letters counted on the host: its record scan and checks, for tests on
// machines without a GPU. Returns TN93G_OK (with the size in n_out, L_out) or TN93G_EFASTA (message in msg).
int tn93g_fasta_check(const char *bytes, size_t nbytes, long expect_len, char counts_sep, long *n_out, long *L_out,
                      char *msg, size_t msg_cap)
{
  if (!bytes && nbytes) return TN93G_EINVAL;
  FastaRecords R;
  fasta_records(bytes, nbytes, counts_sep, R);
  const ByteMap map = make_byte_map();
  std::vector<long> lens(R.spans.size());
  for (size_t k = 0; k < R.spans.size(); k++) {
    long c = 0;
    for (unsigned long long p = R.spans[k].x; p < R.spans[k].y; p++) c += map.v[(unsigned char)bytes[p]] >= 0;
    lens[k] = c;
  }
  long L = 0;
  const std::string err = fasta_check(R, lens, expect_len, &L);
  copy_msg(err, msg, msg_cap);
  if (!err.empty()) return TN93G_EFASTA;
  if (n_out) *n_out = (long)R.spans.size();
  if (L_out) *L_out = L;
  return TN93G_OK;
}

int tn93g_upload_fasta(tn93g_ctx *ctx, tn93g_set **out, const char *bytes, size_t nbytes, long expect_len,
                       char counts_sep, long *n_out, long *L_out, char *msg, size_t msg_cap)
{
  if (!ctx || !out || (!bytes && nbytes)) return TN93G_EINVAL;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  const cudaStream_t st = ctx->stream;
  FastaRecords R;
  fasta_records(bytes, nbytes, counts_sep, R);
  const long m = (long)R.spans.size();
  std::vector<long> lens(m);
  const ByteMap map = make_byte_map();
  if (m) {
    TRY(ensure(ctx, ctx->fraw, nbytes));
    TRY(ensure(ctx, ctx->fspan, m * sizeof(ulonglong2)));
    TRY(ensure(ctx, ctx->flen, m * sizeof(long)));
    CU(cudaMemcpyAsync(ctx->fraw.p, bytes, nbytes, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(ctx->fspan.p, R.spans.data(), m * sizeof(ulonglong2), cudaMemcpyHostToDevice, st));
    fasta_count_kernel<<<(unsigned)((m + kWarps - 1) / kWarps), 256, 0, st>>>(
        (const unsigned char *)ctx->fraw.p, (const ulonglong2 *)ctx->fspan.p, m, map, (long *)ctx->flen.p);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(lens.data(), ctx->flen.p, m * sizeof(long), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
  }
  long first_len = 0;
  const std::string err = fasta_check(R, lens, expect_len, &first_len);
  copy_msg(err, msg, msg_cap);
  if (!err.empty()) return TN93G_EFASTA;
  if (first_len >= (1l << 25)) return TN93G_ETOOBIG;
  TRY(ensure(ctx, ctx->fcode, (size_t)m * first_len));
  fasta_compress_kernel<<<(unsigned)((m + kWarps - 1) / kWarps), 256, 0, st>>>(
      (const unsigned char *)ctx->fraw.p, (const ulonglong2 *)ctx->fspan.p, m, map, first_len, (uint8_t *)ctx->fcode.p);
  CU(cudaGetLastError());
  const int rc = upload_set(ctx, out, (const uint8_t *)ctx->fcode.p, cudaMemcpyDeviceToDevice, m, first_len,
                            R.counts.data(), R.names.data(), R.name_off.data(), R.name_len.data());
  if (rc != TN93G_OK) return rc;
  if (n_out) *n_out = m;
  if (L_out) *L_out = first_len;
  return TN93G_OK;
}

void tn93g_free_set(tn93g_ctx *ctx, tn93g_set *s)
{
  if (!s) return;
  void *bufs[5] = {s->d_codes, s->d_counts, s->d_names, s->d_name_off, s->d_name_len};
  if (ctx) {
    // the buffers go back to the context's pool (the context's stream has no work left on them: every run and
    // upload synchronises it before returning)
    for (int k = 0; k < 5; k++)
      if (bufs[k]) ctx->set_pool.push_back({bufs[k], s->cap[k]});
  } else {
    for (int k = 0; k < 5; k++)
      if (bufs[k]) cudaFree(bufs[k]);
  }
  delete s;
}

int tn93g_last_timings(tn93g_ctx *ctx, double *ms, int n)
{
  if (!ctx || !ms) return 0;
  const int k = std::min(n, 8);
  for (int q = 0; q < k; q++) ms[q] = ctx->timings[q];
  return k;
}

void *tn93g_stream(tn93g_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

long tn93g_last_launches(tn93g_ctx *ctx) { return ctx ? ctx->launches : 0; }

// flags of run_impl: a second, exact pass for the JSON numbers (every ambiguous logarithm taken from the C library)
constexpr int kRunResolveAll = 1;
static int run_impl(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, tn93g_sink sink, void *user,
                    tn93g_summary *sum, bool to_device, long row_begin = 0, long row_end = -1,
                    double *row_sums = nullptr, int flags = 0);

int tn93g_run(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, tn93g_sink sink, void *user,
              tn93g_summary *sum)
{
  return run_impl(ctx, set, n1, opts, sink, user, sum, false);
}

int tn93g_run_rows(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, long row_begin,
                   long row_end, tn93g_sink sink, void *user, double *row_sums, tn93g_summary *sum)
{
  if (!opts || opts->format == TN93G_HYPHY || row_begin < 0 || row_end < row_begin) return TN93G_EINVAL;
  return run_impl(ctx, set, n1, opts, sink, user, sum, false, row_begin, row_end, row_sums);
}

int tn93g_run_to_device(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, void **dev_out,
                        size_t *nbytes, tn93g_summary *sum)
{
  if (!dev_out || !nbytes) return TN93G_EINVAL;
  const int rc = run_impl(ctx, set, n1, opts, nullptr, nullptr, sum, true);
  *dev_out = rc == TN93G_OK ? ctx->out.p : nullptr;
  *nbytes = rc == TN93G_OK ? ctx->dev_out_n : 0;
  return rc;
}

static int run_impl(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, tn93g_sink sink, void *user,
                    tn93g_summary *sum, bool to_device, long row_begin, long row_end, double *row_sums, int flags)
{
  if (!ctx || !set || !opts || !sum || n1 <= 0 || n1 > set->N) return TN93G_EINVAL;
  if (opts->mode < 0 || opts->mode > 4 || opts->format < 0 || opts->format > 2) return TN93G_EINVAL;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const long N = set->N, L = set->L;
  memset(sum, 0, sizeof *sum);
  for (double &t : ctx->timings) t = 0;
  ctx->launches = 0;
  ctx->dev_out_n = 0;
  size_t dev_off = 0;  // to_device: bytes of the distance file already in ctx->out
  RunConsts rc;
  memset(&rc, 0, sizeof rc);
  rc.N = N;
  rc.n1 = n1;
  rc.mode = opts->mode;
  rc.gapmm = opts->mode == TN93G_GAPMM;
  rc.fst = n1 < N && opts->do_fst;
  rc.cross = n1 < N && !opts->do_fst;
  rc.fallback_avg = (opts->mode == TN93G_RESOLVE || opts->mode == TN93G_SUBSET) && opts->resolve_fraction < 1.;
  rc.emit = !opts->count_only;
  rc.format = opts->format;
  rc.delim = opts->delimiter;
  rc.report_self = opts->report_self && !rc.cross && n1 == N && rc.emit;
  rc.threshold = opts->threshold;
  rc.min_distance = opts->min_distance;
  rc.resolve_fraction = opts->resolve_fraction;
  rc.min_overlap = opts->min_overlap;
  rc.log_band = ctx->log_band;
  rc.log_spread = ctx->log_spread;
  rc.resolve_all = (flags & kRunResolveAll) != 0 || ctx->exact_sums;
  bool fault_pending = ctx->fault == TN93G_FAULT_SKIP_FILL;  // injected into the first count launch only
  ctx->fault = TN93G_FAULT_NONE;
  const bool hyphy = rc.emit && opts->format == TN93G_HYPHY;
  cudaEvent_t *E = ctx->evs;
  CU(cudaEventRecord(E[0], st));

  //------------------------------------------------------------------ pack
  TRY(ensure(ctx, ctx->seen, L * sizeof(uint32_t)));
  TRY(ensure(ctx, ctx->nN, sizeof(unsigned long long)));
  CU(cudaMemsetAsync(ctx->seen.p, 0, L * sizeof(uint32_t), st));
  CU(cudaMemsetAsync(ctx->nN.p, 0, sizeof(unsigned long long), st));
  {
    dim3 g((unsigned)((L + 255) / 256), (unsigned)((N + 63) / 64));
    colscan_kernel<<<g, 256, 0, st>>>(set->d_codes, N, L, (uint32_t *)ctx->seen.p, (unsigned long long *)ctx->nN.p);
    CU(cudaGetLastError());
    ctx->launches++;
  }
  std::vector<uint32_t> seen(L);
  unsigned long long nN = 0;
  CU(cudaMemcpyAsync(seen.data(), ctx->seen.p, L * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(&nN, ctx->nN.p, sizeof nN, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  // a column is constant when every sequence has the same clean base there: each pair gets (b, b)
  std::vector<int32_t> varcol;
  varcol.reserve(L);
  for (long p = 0; p < L; p++) {
    const uint32_t m = seen[p];
    if (m && !(m & (m - 1)) && m < 16) {
      const int b = __builtin_ctz(m);
      rc.constT++;
      rc.constNf[b] += 2;
      rc.constCnt[b]++;
    } else
      varcol.push_back((int32_t)p);
  }
  const long Lc = (long)varcol.size();
  const long W = (Lc + 63) / 64;
  const long Npad = (N + 31) / 32 * 32;
  rc.Lc = Lc;
  rc.W = W;
  rc.Npad = Npad;
  // N gets its own bit plane when frequent (more than 16 per sequence); gapmm always (gaps join it)
  rc.wplane = rc.gapmm || nN > 16ull * (unsigned long long)N;
  rc.NP = rc.gapmm ? 5 : 4;
  TRY(ensure(ctx, ctx->varcol, std::max<long>(Lc, 1) * sizeof(int32_t)));
  TRY(ensure(ctx, ctx->planes, (size_t)std::max<long>(W, 1) * rc.NP * Npad * sizeof(uint64_t)));
  TRY(ensure(ctx, ctx->cc, (size_t)N * std::max<long>(Lc, 1)));
  TRY(ensure(ctx, ctx->ccT, (size_t)std::max<long>(Lc, 1) * Npad));
  TRY(ensure(ctx, ctx->evcount, N * sizeof(uint32_t)));
  TRY(ensure(ctx, ctx->evoff, (N + 1) * sizeof(uint32_t)));
  if (Lc) CU(cudaMemcpyAsync(ctx->varcol.p, varcol.data(), Lc * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  CU(cudaMemsetAsync(ctx->planes.p, 0, (size_t)std::max<long>(W, 1) * rc.NP * Npad * sizeof(uint64_t), st));
  CU(cudaMemsetAsync(ctx->evcount.p, 0, N * sizeof(uint32_t), st));
  PackArgs pa;
  pa.codes = set->d_codes;
  pa.N = N;
  pa.L = L;
  pa.Lc = Lc;
  pa.W = W;
  pa.Npad = Npad;
  pa.varcol = (const int32_t *)ctx->varcol.p;
  pa.NP = rc.NP;
  pa.wplane = rc.wplane;
  pa.gapmm = rc.gapmm;
  pa.planes = (uint64_t *)ctx->planes.p;
  pa.cc = (uint8_t *)ctx->cc.p;
  pa.evcount = (uint32_t *)ctx->evcount.p;
  pa.ev_off = (const uint32_t *)ctx->evoff.p;
  if (W) {
    pack_kernel<<<dim3((unsigned)((N + kWarps - 1) / kWarps), (unsigned)std::min<long>(W, 65535)), 256, 0, st>>>(pa);
    CU(cudaGetLastError());
    ctx->launches++;
    transpose_kernel<<<dim3((unsigned)((Lc + 31) / 32), (unsigned)(Npad / 32)), dim3(32, 8), 0, st>>>(
        (const uint8_t *)ctx->cc.p, (uint8_t *)ctx->ccT.p, N, Lc, Npad);
    CU(cudaGetLastError());
    ctx->launches++;
  }
  // per sequence, its nonzero N-plane words (the pair kernel's sparse N-plane pass); counted here, listed below
  bool sparse_w = rc.wplane && W > 0;
  std::vector<uint32_t> wcnt;
  if (sparse_w) {
    TRY(ensure(ctx, ctx->wcount, N * sizeof(uint32_t)));
    wcount_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>((const uint64_t *)ctx->planes.p, N, W, rc.NP, Npad,
                                                                (uint32_t *)ctx->wcount.p);
    CU(cudaGetLastError());
    ctx->launches++;
    wcnt.resize(N);
    CU(cudaMemcpyAsync(wcnt.data(), ctx->wcount.p, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  }
  std::vector<uint32_t> evc(N), evoff(N + 1);
  CU(cudaMemcpyAsync(evc.data(), ctx->evcount.p, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (sparse_w) {
    std::vector<uint32_t> woff(N + 1);
    unsigned long long t = 0;
    for (long i = 0; i < N; i++) {
      woff[i] = (uint32_t)t;
      t += wcnt[i];
    }
    sparse_w = t < 0xFFFFFFFFull;  // 32-bit offsets; beyond them every word is visited
    if (sparse_w) {
      woff[N] = (uint32_t)t;
      TRY(ensure(ctx, ctx->wloff, (N + 1) * sizeof(uint32_t)));
      TRY(ensure(ctx, ctx->wl, std::max<size_t>(t, 1) * sizeof(uint32_t)));
      CU(cudaMemcpyAsync(ctx->wloff.p, woff.data(), (N + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
      wlist_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>((const uint64_t *)ctx->planes.p, N, W, rc.NP, Npad,
                                                                 (const uint32_t *)ctx->wloff.p, (uint32_t *)ctx->wl.p);
      CU(cudaGetLastError());
      ctx->launches++;
      // the host copy must outlive the asynchronous upload
      CU(cudaStreamSynchronize(st));
    }
  }
  evoff[0] = 0;
  uint32_t max_ev = 0;
  for (long i = 0; i < N; i++) {
    evoff[i + 1] = evoff[i] + evc[i];
    max_ev = std::max(max_ev, evc[i]);
  }
  rc.packed = max_ev <= (uint32_t)kPackedMaxEvents;
  TRY(ensure(ctx, ctx->ev, std::max<size_t>(evoff[N], 1) * sizeof(uint32_t)));
  CU(cudaMemcpyAsync(ctx->evoff.p, evoff.data(), (N + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  pa.ev = (uint32_t *)ctx->ev.p;
  if (W && evoff[N]) {
    events_kernel<<<(unsigned)((N + kWarps - 1) / kWarps), 256, 0, st>>>(pa);
    CU(cudaGetLastError());
    ctx->launches++;
  }
  // tables of this mode
  build_tables(ctx->h_tab, opts->mode, opts->subset);
  fill_pair_tables(*ctx->h_tab, rc.wplane, ctx->h_ptab);
  TRY(ensure(ctx, ctx->agg, sizeof(PairTables)));
  TRY(ensure(ctx, ctx->site, sizeof(ctx->h_tab->site)));
  CU(cudaMemcpyAsync(ctx->agg.p, ctx->h_ptab, sizeof(PairTables), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ctx->site.p, ctx->h_tab->site, sizeof(ctx->h_tab->site), cudaMemcpyHostToDevice, st));
  // tensor-core count path: the one-hot operand image of every sequence (an extra 32-sequence block at the end,
  // which the last 64-column tile reads)
  const bool use_tc = ctx->count_path == 1 && Lc > 0;
  const long tc_NB = (N + 31) / 32 + 1, tc_KS = (Lc + kTcStageK - 1) / kTcStageK;
  if (use_tc) {
    TRY(ensure(ctx, ctx->ohimg, (size_t)tc_KS * tc_NB * kTcBlockBytes));
    TRY(ensure(ctx, ctx->tcerr, sizeof(unsigned long long)));
    CU(cudaMemsetAsync(ctx->tcerr.p, 0, sizeof(unsigned long long), st));
    const long nthr = tc_NB * 32 * tc_KS * (kTcStageK / 16);
    onehot_kernel<<<(unsigned)((nthr + 255) / 256), 256, 0, st>>>((const uint8_t *)ctx->cc.p, N, Lc, tc_NB, tc_KS,
                                                                  (uint8_t *)ctx->ohimg.p, 0, tc_NB * 32);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(tc_attr_once());
  }
  CU(cudaEventRecord(E[1], st));

  //------------------------------------------------------------------ bands
  // rows of the pair triangle (or of the first file under -s): all of them, or the caller's range
  const long all_rows = rc.cross ? n1 : N;
  if (row_end < 0) row_end = all_rows;
  if (row_begin > all_rows || row_end > all_rows) return TN93G_EINVAL;
  const long upper = row_end;
  const long colbase = rc.cross ? n1 : 0;
  const long ncols = N - colbase;
  if (rc.cross)
    sum->pairwise = (unsigned long)(N - n1) * (unsigned long)(row_end - row_begin);
  else  // pairs (i, j > i) of rows [row_begin, row_end)
    sum->pairwise = (unsigned long)((row_end - row_begin) * (2 * N - row_begin - row_end - 1) / 2);
  // Band schedule. When the text goes to the host, a band holds about 3 M pairs (at most 16 M pair slots), so
  // that the copy of one band overlaps the kernels of the next; otherwise up to 64 M slots (512 MB of distances).
  const bool stream_text = !(to_device || hyphy || !rc.emit);
  static const long band_pairs = [] {
    const char *e = getenv("TN93G_BAND_PAIRS");  // tuning knob: pairs per band when streaming text
    return e && atol(e) > 0 ? atol(e) : (3l << 20);
  }();
  const long target_pairs = (stream_text || rc.resolve_all) ? band_pairs : (1l << 62);
  const long cap_slots = (stream_text || rc.resolve_all) ? (16l << 20) : (64l << 20);
  // When the text streams to the host, the bands ramp up from 1/16 of the target, 1.4 times larger each (a band's
  // kernels take about 0.7 of its copy's time, so each band's kernels end before the previous band's copy does and
  // the copies run back to back), and taper at the end (half of what is left, down to 1/8), so that the first copy
  // starts early and the last one, which nothing overlaps, is short.
  std::vector<std::pair<long, long>> bands;
  long maxrows = 1;
  long left = 0;
  for (long r = row_begin; r < upper; r++) left += rc.cross ? ncols : (N - r - 1);
  for (long r0 = row_begin; r0 < upper;) {
    long tgt = target_pairs;
    if (stream_text) {
      const double ramp = std::pow(1.4, (double)bands.size()) / 16.0;
      if (ramp < 1.0) tgt = std::max<long>(1, (long)((double)target_pairs * ramp));
      if (left < 2 * target_pairs) tgt = std::min(tgt, std::max(target_pairs / 8, left / 2));
    }
    long r = r0, pairs = 0;
    while (r < upper && (r == r0 || ((r - r0 + 1) * ncols <= cap_slots && pairs < tgt && r - r0 < 65535l * kTile))) {
      pairs += rc.cross ? ncols : (N - r - 1);
      r++;
    }
    bands.push_back({r0, r});
    maxrows = std::max(maxrows, r - r0);
    left -= pairs;
    r0 = r;
  }
  const long band = maxrows;
  const long maxseg = std::max<long>(1, (ncols + kSeg - 1) / kSeg);
  const long nseg = band * maxseg;  // per band parity
  if (hyphy) {
    TRY(ensure(ctx, ctx->hy, (size_t)N * N * sizeof(double)));
    fill_nan_kernel<<<1024, 256, 0, st>>>((double *)ctx->hy.p, (size_t)N * N);
    CU(cudaGetLastError());
    ctx->launches++;
  }
  // per band parity (double-buffered): distances, segment statistics, row sums; the replay queue is per band
  const size_t dslots = (size_t)band * ncols;
  TRY(ensure(ctx, ctx->dist, 2 * dslots * sizeof(double)));
  if (rc.emit && !hyphy) TRY(ensure(ctx, ctx->dcode, 2 * dslots * sizeof(uint32_t)));
  const int tc16 = 32 * L < 65536;  // the final x16 aggregates fit 16-bit lanes
  // the tensor-core path's row chunks per band (boundaries on the count kernel's 32-row tiles)
  std::vector<std::vector<std::pair<long, long>>> band_chunks(bands.size());
  size_t chunk_slots = 1;
  int nchunks[2] = {0, 0};
  if (use_tc) {
    for (size_t b = 0; b < bands.size(); b++) {
      const long r0 = bands[b].first, r1 = bands[b].second;
      long bp = 0;
      for (long r = r0; r < r1; r++) bp += rc.cross ? ncols : (N - r - 1);
      static const long chunk_pairs = [] {
        const char *e = getenv("TN93G_TC_CHUNK_PAIRS");  // tuning knob: pairs per count/pair chunk
        return e && atol(e) > 0 ? atol(e) : kTcChunkPairs;
      }();
      const long target = std::max(chunk_pairs, (bp + kMaxTcChunks - 2) / (kMaxTcChunks - 1));
      for (long c0 = r0; c0 < r1;) {
        long c1 = c0, pairs = 0;
        while (c1 < r1 && (c1 == c0 || pairs < target)) {
          pairs += rc.cross ? ncols : (N - c1 - 1);
          c1++;
        }
        c1 = std::min(r1, (c1 + kTcRows - 1) / kTcRows * kTcRows);
        if ((int)band_chunks[b].size() == kMaxTcChunks - 1) c1 = r1;  // never more chunks than events
        band_chunks[b].push_back({c0, c1});
        chunk_slots = std::max(chunk_slots, (size_t)(c1 - c0) * ncols);
        c0 = c1;
      }
    }
    TRY(ensure(ctx, ctx->tcagg, chunk_slots * (tc16 ? 16 : 32)));
  }
  TRY(ensure(ctx, ctx->rq, dslots * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->rqn, sizeof(unsigned)));
  TRY(ensure(ctx, ctx->counters, 4 * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->rbytes, 2 * nseg * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->roff, 2 * nseg * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->rsum, 2 * band * 3 * sizeof(double)));
  TRY(ensure(ctx, ctx->rw, 2 * band * 3 * sizeof(double)));
  TRY(ensure(ctx, ctx->rmax, 2 * nseg * 3 * sizeof(double)));
  TRY(ensure(ctx, ctx->rlinks, 2 * nseg * sizeof(long long)));
  TRY(ensure(ctx, ctx->rskip, 2 * nseg * sizeof(long long)));
  // per band parity: its histogram (added on the host, so a band's row stage can run again), its undecided list
  TRY(ensure(ctx, ctx->hist, 2 * 3 * kHistBins * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->total, 2 * sizeof(unsigned long long)));
  const unsigned und_cap = (unsigned)std::min<size_t>(rc.resolve_all ? dslots : std::max<size_t>(4096, dslots / 64),
                                                      0xFFFFFFF0u);
  for (int q = 0; q < 2; q++) TRY(ensure(ctx, ctx->und[q], (size_t)und_cap * 2 * sizeof(unsigned long long)));
  unsigned und_cap_par[2] = {und_cap, und_cap};  // grown per parity when a band lists more
  TRY(ensure(ctx, ctx->undn, 2 * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->amb, 3 * 4 * sizeof(unsigned long long)));
  TRY(ensure(ctx, ctx->rdesc, 2 * sizeof(ReplayArgs)));
  CU(cudaMemsetAsync(ctx->amb.p, 0, 3 * 4 * sizeof(unsigned long long), st));
  // pinned staging of a band's statistics: row sums and weights (3 each), segment maxima (3 each), segment links
  // and skips, total bytes, the band's histogram, its undecided count and the count kernel's error word
  const size_t stat_stride = (size_t)band * 6 * sizeof(double) +
                             (size_t)nseg * (3 * sizeof(double) + 2 * sizeof(long long)) +
                             (3 + 3 * kHistBins) * sizeof(unsigned long long);
  TRY(ensure_pinned_at(ctx, ctx->pstats, ctx->pstats_n, 2 * stat_stride, cudaHostAllocMapped));
  char *d_pstats = nullptr;  // the device's address of the staging
  CU(cudaHostGetDevicePointer((void **)&d_pstats, ctx->pstats, 0));
  CU(cudaMemsetAsync(ctx->counters.p, 0, 4 * sizeof(unsigned long long), st));
  double max_[3] = {0, 0, 0}, mean[3] = {0, 0, 0}, wc[3] = {0, 0, 0};
  unsigned long long hist_total[3 * kHistBins];
  memset(hist_total, 0, sizeof hist_total);
  long links = 0, skipped = 0, resolved = 0;
  float ms = 0;
  struct HostStats {
    double *sum, *w, *max;
    long long *links, *skip;
    unsigned long long *total, *hist, *und, *tcerr;
  };
  auto host_stats = [&](int par) {
    char *base = (char *)ctx->pstats + par * stat_stride;
    HostStats h;
    h.sum = (double *)base;
    h.w = h.sum + band * 3;
    h.max = h.w + band * 3;
    h.links = (long long *)(h.max + nseg * 3);
    h.skip = h.links + nseg;
    h.total = (unsigned long long *)(h.skip + nseg);
    h.hist = h.total + 1;
    h.und = h.hist + 3 * kHistBins;
    h.tcerr = h.und + 1;
    return h;
  };
  ReplayArgs rdesc_h[2];
  auto row_args = [&](int bi) {
    const int par = bi & 1;
    RowArgs RA;
    RA.rc = rc;
    RA.dist = (const double *)ctx->dist.p + par * dslots;
    RA.r0 = bands[bi].first;
    RA.r1 = bands[bi].second;
    RA.ncols = ncols;
    RA.colbase = colbase;
    RA.counts = set->d_counts;
    RA.name_len = set->d_name_len;
    RA.name_off = set->d_name_off;
    RA.names = set->d_names;
    RA.maxseg = maxseg;
    RA.seg_bytes = (unsigned long long *)ctx->rbytes.p + par * nseg;
    RA.seg_links = (long long *)ctx->rlinks.p + par * nseg;
    RA.seg_skip = (long long *)ctx->rskip.p + par * nseg;
    RA.seg_max = (double *)ctx->rmax.p + par * nseg * 3;
    RA.row_sum = (double *)ctx->rsum.p + par * band * 3;
    RA.row_w = (double *)ctx->rw.p + par * band * 3;
    RA.hist = (unsigned long long *)ctx->hist.p + par * 3 * kHistBins;
    RA.seg_off = (const unsigned long long *)ctx->roff.p + par * nseg;
    RA.seg_cols = nullptr;
    RA.nrows = RA.r1 - RA.r0;
    RA.out = nullptr;
    RA.hy = (double *)ctx->hy.p;
    RA.err = (unsigned long long *)ctx->counters.p + 3;
    RA.dcode = (rc.emit && !hyphy) ? (uint32_t *)ctx->dcode.p + par * dslots : nullptr;
    return RA;
  };
  // stats -> sums -> scan of band bi, then its statistics to the host (on the compute stream)
  auto enqueue_rows = [&](int bi) -> int {
    const int par = bi & 1;
    const long nr = bands[bi].second - bands[bi].first;
    cudaEvent_t *K = ctx->evk[par];
    RowArgs RA = row_args(bi);
    CU(cudaMemsetAsync(RA.hist, 0, 3 * kHistBins * sizeof(unsigned long long), st));
    stats_kernel<<<dim3((unsigned)((nr + kWarps - 1) / kWarps), (unsigned)maxseg), 256, 0, st>>>(RA);
    CU(cudaGetLastError());
    ctx->launches++;
    sum_kernel<<<(unsigned)((nr + kWarps - 1) / kWarps), 256, 0, st>>>(RA);
    CU(cudaGetLastError());
    ctx->launches++;
    unsigned long long *dtot = (unsigned long long *)ctx->total.p + par;
    scan_kernel<<<1, 1024, 0, st>>>(RA.seg_bytes, (unsigned long long *)RA.seg_off, nr * maxseg, dtot);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(K[3], st));
    // the band's statistics into the mapped staging (device addresses at the same offsets as host_stats')
    const HostStats h = host_stats(par);
    auto dev = [&](const void *hp) {
      return (unsigned long long *)(d_pstats + ((const char *)hp - (const char *)ctx->pstats));
    };
    Gather g;
    g.k = 0;
    auto add = [&](const void *src, const void *hdst, long nwords) {
      g.src[g.k] = (const unsigned long long *)src;
      g.dst[g.k] = dev(hdst);
      g.n[g.k++] = nwords;
    };
    add(RA.row_sum, h.sum, nr * 3);
    add(RA.row_w, h.w, nr * 3);
    add(RA.seg_max, h.max, nr * maxseg * 3);
    add(RA.seg_links, h.links, nr * maxseg);
    add(RA.seg_skip, h.skip, nr * maxseg);
    add(dtot, h.total, 1);
    add(RA.hist, h.hist, 3 * kHistBins);
    add((unsigned long long *)ctx->undn.p + par, h.und, 1);
    if (use_tc)
      add(ctx->tcerr.p, h.tcerr, 1);
    else
      *h.tcerr = 0;
    gather_kernel<<<32, 256, 0, st>>>(g);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(K[4], st));
    return TN93G_OK;
  };
  // pair -> replay of band bi, then its row stage
  auto enqueue_compute = [&](int bi) -> int {
    const int par = bi & 1;
    const long r0 = bands[bi].first, r1 = bands[bi].second, nr = r1 - r0;
    cudaEvent_t *K = ctx->evk[par];
    // this parity's distances, codes and row arrays are read by band bi - 2's text writer on the write stream
    if (bi >= 2 && stream_text) CU(cudaStreamWaitEvent(st, ctx->evw1[par], 0));
    CU(cudaEventRecord(K[0], st));
    CU(cudaMemsetAsync(ctx->rqn.p, 0, sizeof(unsigned), st));
    CU(cudaMemsetAsync((unsigned long long *)ctx->undn.p + par, 0, sizeof(unsigned long long), st));
    ExactSink ex;
    ex.und_list = (unsigned long long *)ctx->und[par].p;
    ex.und_n = (unsigned *)((unsigned long long *)ctx->undn.p + par);
    ex.und_cap = und_cap_par[par];
    ex.und_k = 0;
    ex.amb = (unsigned long long *)ctx->amb.p;
    ex.counts = set->d_counts;
    ex.colunit = nullptr;
    PairArgs A;
    A.rc = rc;
    A.planes = (const uint64_t *)ctx->planes.p;
    A.cc = (const uint8_t *)ctx->cc.p;
    A.ccT = (const uint8_t *)ctx->ccT.p;
    A.ev_off = (const uint32_t *)ctx->evoff.p;
    A.ev = (const uint32_t *)ctx->ev.p;
    A.tab = (const PairTables *)ctx->agg.p;
    A.r0 = r0;
    A.r1 = r1;
    A.ncols = ncols;
    A.colbase = colbase;
    A.dist = (double *)ctx->dist.p + par * dslots;
    A.replay_q = (unsigned long long *)ctx->rq.p;
    A.replay_n = (unsigned *)ctx->rqn.p;
    A.replay_cap = (unsigned long long)dslots;
    A.counters = (unsigned long long *)ctx->counters.p;
    A.logt = ctx->d_logt;
    A.ex = ex;
    A.wl_off = sparse_w ? (const uint32_t *)ctx->wloff.p : nullptr;
    A.wl = sparse_w ? (const uint32_t *)ctx->wl.p : nullptr;
    // columns: the smallest lower bound of the band's rows onwards
    const long cstart = rc.cross ? n1 : r0 + 1;
    const long cblk0 = (cstart - colbase) / 32;
    const long cblks = (ncols + 31) / 32 - cblk0;
    if (use_tc && cblks > 0) {
      // Clean-site aggregates on the tensor cores, then the pair kernel, chunk by chunk of rows (about kTcChunkPairs
      // pairs each); the pair kernel reads each record once and drops its cache line.
      const std::vector<std::pair<long, long>> &chunks = band_chunks[bi];
      for (size_t q = 0; q < chunks.size(); q++) {
        const long c0 = chunks[q].first, c1 = chunks[q].second;
        const long ccs = rc.cross ? n1 : c0 + 1;
        TcArgs T;
        T.onehot = (const uint8_t *)ctx->ohimg.p;
        T.NB = tc_NB;
        T.KS = tc_KS;
        T.N = N;
        T.n1 = n1;
        T.cross = rc.cross;
        T.r0 = c0;
        T.r1 = c1;
        T.ncols = ncols;
        T.colbase = colbase;
        T.cstart = ccs / kTcCols * kTcCols;
        T.cend = N;
        T.agg = ctx->tcagg.p;
        T.agg16 = tc16;
        T.err = (unsigned long long *)ctx->tcerr.p;
        T.wait_ns = ctx->wait_ns;
        T.skip_fill_block = fault_pending ? 0 : -1;
        fault_pending = false;
        const long rt0 = c0 / kTcRows * kTcRows;
        const dim3 g((unsigned)((N - T.cstart + kTcCols - 1) / kTcCols), (unsigned)((c1 - rt0 + kTcRows - 1) / kTcRows));
        CU(cudaEventRecord(ctx->evcnt[par][2 * q], st));
        CU(launch_count_grid(T, g.x, g.y, ctx->sms, st));
        CU(cudaEventRecord(ctx->evcnt[par][2 * q + 1], st));
        ctx->launches++;
        PairArgs AC = A;
        AC.r0 = c0;
        AC.r1 = c1;
        AC.dist = A.dist + (size_t)(c0 - r0) * ncols;
        AC.tcagg = ctx->tcagg.p;
        AC.tc16 = tc16;
        AC.split = pair_split(AC.rc);
        const long cb0 = (ccs - colbase) / 32, cbs = (ncols + 31) / 32 - cb0;
        if (cbs > 0) {
          AC.cstart = colbase + cb0 * 32;
          CU(launch_pair(AC, cbs, c1 - c0, st));
          ctx->launches += AC.split ? 2 : 1;
        }
      }
      nchunks[par] = (int)chunks.size();
    } else if (cblks > 0) {
      A.cstart = colbase + cblk0 * 32;
      CU(launch_pair(A, cblks, nr, st));
      ctx->launches++;
      nchunks[par] = 0;
    } else {
      nchunks[par] = 0;
    }
    CU(cudaEventRecord(K[1], st));
    ReplayArgs R;
    R.rc = rc;
    R.cc = (const uint8_t *)ctx->cc.p;
    R.planes = (const uint64_t *)ctx->planes.p;
    R.site = (const SiteEntry *)ctx->site.p;
    R.q = (const unsigned long long *)ctx->rq.p;
    R.qn = (const unsigned *)ctx->rqn.p;
    R.qcap = (unsigned long long)dslots;
    R.r0 = r0;
    R.ncols = ncols;
    R.colbase = colbase;
    R.dist = A.dist;
    R.counters = (unsigned long long *)ctx->counters.p;
    R.logt = ctx->d_logt;
    R.ex = ex;
    rdesc_h[par] = R;
    replay_kernel<<<2 * ctx->sms, 256, 0, st>>>(R);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(K[2], st));
    return enqueue_rows(bi);
  };
  // bands whose text is on its way to the host: parities, oldest first
  int pend_par[2] = {0, 0}, pend_n = 0;
  size_t pend_bytes[2] = {0, 0};
  bool par_used[2] = {false, false};
  // TN93G_TRACE=1: one stderr line per delivered band (device milliseconds from the run's first event: write
  // start and end, copy start and end; host milliseconds when the copy was seen complete), for pipeline tuning
  static const bool trace = getenv("TN93G_TRACE") != nullptr;
  const auto host0 = std::chrono::steady_clock::now();
  int delivered = 0;
  auto deliver_oldest = [&]() -> int {
    const int q = pend_par[0];
    CU(cudaEventSynchronize(ctx->evc1[q]));
    CU(cudaEventElapsedTime(&ms, ctx->evw0[q], ctx->evw1[q]));
    ctx->timings[4] += ms;
    CU(cudaEventElapsedTime(&ms, ctx->evc0[q], ctx->evc1[q]));
    ctx->timings[5] += ms;
    if (trace) {
      float w0, w1, c0, c1;
      CU(cudaEventElapsedTime(&w0, E[0], ctx->evw0[q]));
      CU(cudaEventElapsedTime(&w1, E[0], ctx->evw1[q]));
      CU(cudaEventElapsedTime(&c0, E[0], ctx->evc0[q]));
      CU(cudaEventElapsedTime(&c1, E[0], ctx->evc1[q]));
      const double h = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host0).count();
      fprintf(stderr, "tn93g trace: band %d bytes %zu write %.3f-%.3f copy %.3f-%.3f host %.3f\n", delivered++,
              pend_bytes[q], w0, w1, c0, c1, h);
    }
    pend_par[0] = pend_par[1];
    pend_n--;
    if (sink && sink(user, (const char *)ctx->pin2[q], pend_bytes[q])) return TN93G_ESINK;
    return TN93G_OK;
  };
  // statistics of band bi in row order, then its text: written on the compute stream (behind the next band's
  // kernels) and copied to the host on the copy stream
  auto finish = [&](int bi) -> int {
    const int par = bi & 1;
    const long nr = bands[bi].second - bands[bi].first;
    cudaEvent_t *K = ctx->evk[par];
    CU(cudaEventSynchronize(K[4]));
    CU(cudaEventElapsedTime(&ms, K[0], K[1]));
    ctx->timings[1] += ms;
    for (int q = 0; q < nchunks[par]; q++) {
      CU(cudaEventElapsedTime(&ms, ctx->evcnt[par][2 * q], ctx->evcnt[par][2 * q + 1]));
      ctx->timings[7] += ms;
    }
    CU(cudaEventElapsedTime(&ms, K[1], K[2]));
    ctx->timings[2] += ms;
    CU(cudaEventElapsedTime(&ms, K[2], K[3]));
    ctx->timings[3] += ms;
    const HostStats h = host_stats(par);
    if (*h.tcerr) {
      // the next band's kernels may still be queued: let them drain so the context is idle for the next run
      cudaStreamSynchronize(st);
      ctx->err = "the tensor-core count kernel timed out waiting for its pipeline";
      return TN93G_ETIMEOUT;
    }
    if (*h.und) {
      // pairs whose bytes or decisions depend on the C library's rounding of a logarithm: finish them with its
      // logarithms, then run the band's row stage again
      if (*h.und > und_cap_par[par]) {
        // more than the list holds: grow this parity's list and run the band's pair stage again (the same pairs
        // are listed; the summary bounds only widen, which keeps them valid)
        const unsigned long long lim = std::min<unsigned long long>(dslots, 0xFFFFFFF0ull);
        const unsigned need = (unsigned)std::min<unsigned long long>(
            std::max<unsigned long long>(*h.und + *h.und / 4 + 1024, 2ull * und_cap_par[par]), lim);
        CU(cudaStreamSynchronize(st));
        TRY(ensure(ctx, ctx->und[par], (size_t)need * 2 * sizeof(unsigned long long)));
        und_cap_par[par] = need;
        TRY(enqueue_compute(bi));
        CU(cudaEventSynchronize(K[4]));
        if (*h.und > und_cap_par[par]) {
          ctx->err = "more undecided pairs in a band than its list holds";
          return TN93G_EUNDECIDED;
        }
      }
      ReplayArgs *dd = (ReplayArgs *)ctx->rdesc.p + par;
      CU(cudaMemcpyAsync(dd, &rdesc_h[par], sizeof(ReplayArgs), cudaMemcpyHostToDevice, st));
      TRY(resolve_listed(ctx, dd, (const unsigned long long *)ctx->und[par].p, (unsigned)*h.und, st));
      resolved += (long)*h.und;
      TRY(enqueue_rows(bi));
      CU(cudaEventSynchronize(K[4]));
    }
    for (int q = 0; q < 3 * kHistBins; q++) hist_total[q] += h.hist[q];
    // rows in order (swifttn93.cpp:2838-2848)
    for (long r = 0; r < nr; r++) {
      for (long g = r * maxseg; g < (r + 1) * maxseg; g++) {
        links += h.links[g];
        skipped += h.skip[g];
        for (int q = 0; q < 3; q++)
          if (h.max[g * 3 + q] > max_[q]) max_[q] = h.max[g * 3 + q];
      }
      for (int q = 0; q < 3; q++) {
        mean[q] += h.sum[r * 3 + q];
        wc[q] += h.w[r * 3 + q];
      }
      if (row_sums) {
        double *o = row_sums + (size_t)(bands[bi].first - row_begin + r) * 6;
        for (int q = 0; q < 3; q++) {
          o[q] = h.sum[r * 3 + q];
          o[3 + q] = h.w[r * 3 + q];
        }
      }
    }
    const unsigned long long tot = *h.total;
    if (!(rc.emit && !hyphy && tot)) return TN93G_OK;
    sum->output_bytes += tot;
    RowArgs RA = row_args(bi);
    const dim3 wgrid((unsigned)((nr + kWarps - 1) / kWarps), (unsigned)maxseg);
    if (to_device) {
      TRY(ensure_keep(ctx, ctx->out, dev_off + tot, dev_off));
      RA.out = (char *)ctx->out.p + dev_off;
      CU(cudaEventRecord(ctx->evw0[0], st));
      write_kernel<<<wgrid, 256, 0, st>>>(RA);
      CU(cudaGetLastError());
      ctx->launches++;
      CU(cudaEventRecord(ctx->evw1[0], st));
      CU(cudaEventSynchronize(ctx->evw1[0]));
      CU(cudaEventElapsedTime(&ms, ctx->evw0[0], ctx->evw1[0]));
      ctx->timings[4] += ms;
      dev_off += tot;
      return TN93G_OK;
    }
    // The band's text is written on the write stream, beside the next band's kernels, once its statistics are final
    // (K[4]), then copied on the copy stream. The older band of this parity (or, when the bands between them wrote
    // no text, an even older one) goes to the sink first: its copy has then left the device buffer, the sink has
    // taken the pinned buffer, and its write and copy events are free to record this band's. Meanwhile the copy
    // engine works on the band in between.
    for (;;) {
      bool held = false;
      for (int q = 0; q < pend_n; q++) held |= pend_par[q] == par;
      if (!held) break;
      TRY(deliver_oldest());
    }
    const cudaStream_t ws = ctx->write_stream;
    TRY(ensure(ctx, ctx->out2[par], tot));
    TRY(ensure_pinned_at(ctx, ctx->pin2[par], ctx->pin2_n[par], tot));
    RA.out = (char *)ctx->out2[par].p;
    CU(cudaStreamWaitEvent(ws, K[4], 0));
    if (par_used[par]) CU(cudaStreamWaitEvent(ws, ctx->evc1[par], 0));
    CU(cudaEventRecord(ctx->evw0[par], ws));
    write_kernel<<<wgrid, 256, 0, ws>>>(RA);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(ctx->evw1[par], ws));
    CU(cudaStreamWaitEvent(ctx->copy_stream, ctx->evw1[par], 0));
    CU(cudaEventRecord(ctx->evc0[par], ctx->copy_stream));
    CU(cudaMemcpyAsync(ctx->pin2[par], ctx->out2[par].p, tot, cudaMemcpyDeviceToHost, ctx->copy_stream));
    CU(cudaEventRecord(ctx->evc1[par], ctx->copy_stream));
    par_used[par] = true;
    pend_bytes[par] = tot;
    pend_par[pend_n++] = par;
    return TN93G_OK;
  };
  // Band bi + 1's kernels are queued before band bi is finished, so the device computes while the host takes band
  // bi's statistics; texts reach the sink when their pinned buffer is needed again, or at the end (at most one band
  // per parity waits).
  const int nb = (int)bands.size();
  for (int bi = 0; bi <= nb; bi++) {
    if (bi < nb) TRY(enqueue_compute(bi));
    if (bi >= 1) TRY(finish(bi - 1));
  }
  while (pend_n) TRY(deliver_oldest());
  if (hyphy) {
    TRY(ensure(ctx, ctx->rbytes, N * sizeof(unsigned long long)));
    TRY(ensure(ctx, ctx->roff, N * sizeof(unsigned long long)));
    const unsigned blocks = (unsigned)((N + kWarps - 1) / kWarps);
    CU(cudaEventRecord(E[6], st));
    hy_len_kernel<<<blocks, 256, 0, st>>>((const double *)ctx->hy.p, N, (unsigned long long *)ctx->rbytes.p);
    CU(cudaGetLastError());
    ctx->launches++;
    std::vector<unsigned long long> hb(N), ho(N);
    CU(cudaMemcpyAsync(hb.data(), ctx->rbytes.p, N * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    unsigned long long tot = 1;  // leading "{"
    for (long r = 0; r < N; r++) {
      ho[r] = tot;
      tot += hb[r];
    }
    tot += 2;  // "\n}"
    TRY(ensure(ctx, ctx->out, tot));
    if (!to_device) TRY(ensure_pinned(ctx, tot));
    CU(cudaMemcpyAsync(ctx->roff.p, ho.data(), N * sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(ctx->out.p, "{", 1, cudaMemcpyHostToDevice, st));
    hy_write_kernel<<<blocks, 256, 0, st>>>((const double *)ctx->hy.p, N, (const unsigned long long *)ctx->roff.p,
                                            (char *)ctx->out.p);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaMemcpyAsync((char *)ctx->out.p + tot - 2, "\n}", 2, cudaMemcpyHostToDevice, st));
    CU(cudaEventRecord(E[7], st));
    if (!to_device) CU(cudaMemcpyAsync(ctx->pinned, ctx->out.p, tot, cudaMemcpyDeviceToHost, st));
    CU(cudaEventRecord(E[8], st));
    CU(cudaStreamSynchronize(st));
    CU(cudaEventElapsedTime(&ms, E[6], E[7]));
    ctx->timings[4] += ms;
    CU(cudaEventElapsedTime(&ms, E[7], E[8]));
    ctx->timings[5] += ms;
    sum->output_bytes += tot;
    dev_off = tot;
    if (!to_device && sink && sink(user, (const char *)ctx->pinned, tot)) return TN93G_ESINK;
  }
  unsigned long long counters[4], ambw[12];
  CU(cudaMemcpyAsync(counters, ctx->counters.p, sizeof counters, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(ambw, ctx->amb.p, sizeof ambw, cudaMemcpyDeviceToHost, st));
  CU(cudaEventRecord(E[9], st));
  CU(cudaStreamSynchronize(st));
  if (trace) {
    float d9;
    CU(cudaEventElapsedTime(&d9, E[0], E[9]));
    fprintf(stderr, "tn93g trace: end device %.3f host %.3f bands %d\n", d9,
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host0).count(), nb);
  }
  CU(cudaEventElapsedTime(&ms, E[0], E[1]));
  ctx->timings[0] = ms;
  CU(cudaEventElapsedTime(&ms, E[0], E[9]));
  ctx->timings[6] = ms;
  for (int q = 0; q < 3; q++) {
    sum->max[q] = max_[q];
    sum->mean[q] = mean[q];
    sum->weighted[q] = wc[q];
    for (int k = 0; k < kHistBins; k++) sum->hist[q][k] = hist_total[q * kHistBins + k];
  }
  sum->links = links;
  sum->skipped = skipped;
  sum->logs_ambiguous = (long)counters[0];
  sum->logs_resolved = resolved;
  sum->undecided = 0;  // every listed pair was finished with the C library's logarithms
  sum->pairs_replayed = (long)counters[2];
  ctx->dev_out_n = dev_off;
  if (use_tc) {
    unsigned long long tcerr = 0;
    CU(cudaMemcpy(&tcerr, ctx->tcerr.p, sizeof tcerr, cudaMemcpyDeviceToHost));
    if (tcerr) {
      ctx->err = "the tensor-core count kernel timed out waiting for its pipeline";
      return TN93G_ETIMEOUT;
    }
  }
  if (counters[3]) {
    ctx->err = "internal error: a row's text did not match its counted length";
    return TN93G_ECUDA;
  }
  // The JSON numbers (maximum, means): certain for every rounding of the C library's log, or taken from a second
  // pass that finishes every pair with an ambiguous logarithm with the C library's own (rows in the same order).
  // (A proper range of rows is a part of a larger run: its caller certifies the merged summary.)
  for (int u = 0; u < 3; u++) amb_bounds(ambw + 4 * u, sum->amb_bounds[u]);
  if (rc.resolve_all) memset(sum->amb_bounds, 0, sizeof sum->amb_bounds);  // every ambiguous pair was finished exactly
  const long chain = (rc.cross ? N - n1 : N) + (row_end - row_begin) + 2;
  const bool whole = row_begin == 0 && row_end == all_rows;
  if (!rc.resolve_all && whole && !summary_certified(sum, sum->amb_bounds, chain, rc.fst)) {
    tn93g_opts o2 = *opts;
    o2.count_only = 1;
    tn93g_summary s2;
    std::vector<double> rs2(row_sums ? (size_t)(row_end - row_begin) * 6 : 0);
    const double t6 = ctx->timings[6];
    TRY(run_impl(ctx, set, n1, &o2, nullptr, nullptr, &s2, false, row_begin, row_end,
                 row_sums ? rs2.data() : nullptr, kRunResolveAll));
    for (int q = 0; q < 3; q++) {
      sum->max[q] = s2.max[q];
      sum->mean[q] = s2.mean[q];
    }
    if (row_sums) memcpy(row_sums, rs2.data(), rs2.size() * sizeof(double));
    sum->logs_resolved += s2.logs_resolved;
    sum->sums_repass = 1;
    memset(sum->amb_bounds, 0, sizeof sum->amb_bounds);
    ctx->timings[6] += t6;
    ctx->dev_out_n = dev_off;
  }
  return TN93G_OK;
}

}  // extern "C"

//================================================================================================== allocation-free entry point
// tn93g_pair_distances_noalloc: the pack -> pair -> site-order replay pipeline of tn93g_run for one alignment,
// with every intermediate buffer carved out of one fixed file-scope device array instead of cudaMalloc, for
// callers that must not allocate device memory. Inputs and outputs are the caller's device buffers.
namespace {

constexpr long kNaMaxN = 512;   // sequences
constexpr long kNaMaxL = 4096;  // columns
constexpr long kNaW = (kNaMaxL + 63) / 64;
constexpr size_t na_al(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kNaLog = 0;
constexpr size_t kNaAgg = kNaLog + na_al(sizeof(LogTable));
constexpr size_t kNaSite = kNaAgg + na_al(sizeof(PairTables));
constexpr size_t kNaSeen = kNaSite + na_al(2 * kCodes * kCodes * sizeof(SiteEntry));
constexpr size_t kNaNN = kNaSeen + na_al(kNaMaxL * sizeof(uint32_t));
constexpr size_t kNaVarcol = kNaNN + na_al(sizeof(unsigned long long));
constexpr size_t kNaPlanes = kNaVarcol + na_al(kNaMaxL * sizeof(int32_t));
constexpr size_t kNaCC = kNaPlanes + na_al((size_t)kNaW * 5 * kNaMaxN * sizeof(uint64_t));
constexpr size_t kNaCCT = kNaCC + na_al((size_t)kNaMaxN * kNaMaxL);
constexpr size_t kNaEvcount = kNaCCT + na_al((size_t)kNaMaxL * kNaMaxN);
constexpr size_t kNaEvoff = kNaEvcount + na_al(kNaMaxN * sizeof(uint32_t));
constexpr size_t kNaEv = kNaEvoff + na_al((kNaMaxN + 1) * sizeof(uint32_t));
constexpr size_t kNaRq = kNaEv + na_al((size_t)kNaMaxN * kNaMaxL * sizeof(uint32_t));
constexpr size_t kNaRqn = kNaRq + na_al((size_t)kNaMaxN * kNaMaxN * sizeof(unsigned long long));
constexpr size_t kNaCounters = kNaRqn + na_al(sizeof(unsigned));
constexpr size_t kNaBytes = kNaCounters + na_al(4 * sizeof(unsigned long long));  // about 15.6 MB

// The scratch. Every GPU that loads this library holds it until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Per device: the scratch's device address (cudaGetSymbolAddress, taken with that device current) and whether
// the log table has been written into it. Host code must never pass the symbol itself to a kernel.
constexpr int kNaMaxDevices = 64;
std::mutex g_na_mu;
unsigned char *g_na_base[kNaMaxDevices];

// message of the last failure of a call made by this thread
thread_local char g_na_err[256];

void na_error(const char *what, cudaError_t e)
{
  snprintf(g_na_err, sizeof g_na_err, "%s: %s", what, cudaGetErrorString(e));
}

// caller holds g_na_mu
int noalloc_setup(int dev, unsigned char **base)
{
  if (dev < 0 || dev >= kNaMaxDevices) return TN93G_ENODEV;
  if (g_na_base[dev]) {
    *base = g_na_base[dev];
    return TN93G_OK;
  }
  unsigned char *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    na_error("cudaGetSymbolAddress", e);
    return TN93G_ECUDA;
  }
  LogTable h;
  build_log_table(&h);
  e = cudaMemcpy(p + kNaLog, &h, sizeof h, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    na_error("cudaMemcpy", e);
    return TN93G_ECUDA;
  }
  g_na_base[dev] = p;
  *base = p;
  return TN93G_OK;
}

Tables g_na_tables;     // host staging of the contribution tables (static storage; used with g_na_mu held)
PairTables g_na_ptab;  // and of the pair stage's form of them

// caller holds g_na_mu
int noalloc_run(const uint8_t *d_codes, long N, long L, const tn93g_opts *opts, double *d_dist, cudaStream_t st)
{
#define NA(call)                  \
  do {                            \
    cudaError_t e_ = (call);      \
    if (e_ != cudaSuccess) {      \
      na_error(#call, e_);        \
      return TN93G_ECUDA;         \
    }                             \
  } while (0)
  int dev = 0;
  NA(cudaGetDevice(&dev));
  unsigned char *S = nullptr;
  const int src = noalloc_setup(dev, &S);
  if (src != TN93G_OK) return src;
  RunConsts rc;
  memset(&rc, 0, sizeof rc);
  rc.N = N;
  rc.n1 = N;
  rc.mode = opts->mode;
  rc.gapmm = opts->mode == TN93G_GAPMM;
  rc.fallback_avg = (opts->mode == TN93G_RESOLVE || opts->mode == TN93G_SUBSET) && opts->resolve_fraction < 1.;
  rc.emit = !opts->count_only;
  rc.format = opts->format;
  rc.delim = opts->delimiter;
  rc.threshold = opts->threshold;
  rc.min_distance = opts->min_distance;
  rc.resolve_fraction = opts->resolve_fraction;
  rc.min_overlap = opts->min_overlap;
  rc.log_band = kLogBand;
  rc.log_spread = kLogSpread;
  rc.resolve_all = false;
  uint32_t *seen = (uint32_t *)(S + kNaSeen);
  unsigned long long *nN = (unsigned long long *)(S + kNaNN);
  NA(cudaMemsetAsync(seen, 0, L * sizeof(uint32_t), st));
  NA(cudaMemsetAsync(nN, 0, sizeof(unsigned long long), st));
  colscan_kernel<<<dim3((unsigned)((L + 255) / 256), (unsigned)((N + 63) / 64)), 256, 0, st>>>(d_codes, N, L, seen, nN);
  NA(cudaGetLastError());
  uint32_t h_seen[kNaMaxL];
  int32_t h_varcol[kNaMaxL];
  unsigned long long h_nN = 0;
  NA(cudaMemcpyAsync(h_seen, seen, L * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA(cudaMemcpyAsync(&h_nN, nN, sizeof h_nN, cudaMemcpyDeviceToHost, st));
  NA(cudaStreamSynchronize(st));
  long Lc = 0;
  for (long p = 0; p < L; p++) {
    const uint32_t m = h_seen[p];
    if (m && !(m & (m - 1)) && m < 16) {
      const int b = __builtin_ctz(m);
      rc.constT++;
      rc.constNf[b] += 2;
      rc.constCnt[b]++;
    } else
      h_varcol[Lc++] = (int32_t)p;
  }
  const long W = (Lc + 63) / 64, Npad = (N + 31) / 32 * 32;
  rc.Lc = Lc;
  rc.W = W;
  rc.Npad = Npad;
  rc.wplane = rc.gapmm || h_nN > 16ull * (unsigned long long)N;
  rc.NP = rc.gapmm ? 5 : 4;
  PackArgs pa;
  pa.codes = d_codes;
  pa.N = N;
  pa.L = L;
  pa.Lc = Lc;
  pa.W = W;
  pa.Npad = Npad;
  pa.varcol = (const int32_t *)(S + kNaVarcol);
  pa.NP = rc.NP;
  pa.wplane = rc.wplane;
  pa.gapmm = rc.gapmm;
  pa.planes = (uint64_t *)(S + kNaPlanes);
  pa.cc = S + kNaCC;
  pa.evcount = (uint32_t *)(S + kNaEvcount);
  pa.ev_off = (const uint32_t *)(S + kNaEvoff);
  pa.ev = (uint32_t *)(S + kNaEv);
  if (Lc) NA(cudaMemcpyAsync(S + kNaVarcol, h_varcol, Lc * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  NA(cudaMemsetAsync(pa.planes, 0, (size_t)std::max<long>(W, 1) * rc.NP * Npad * sizeof(uint64_t), st));
  NA(cudaMemsetAsync(pa.evcount, 0, N * sizeof(uint32_t), st));
  if (W) {
    pack_kernel<<<dim3((unsigned)((N + kWarps - 1) / kWarps), (unsigned)W), 256, 0, st>>>(pa);
    NA(cudaGetLastError());
    transpose_kernel<<<dim3((unsigned)((Lc + 31) / 32), (unsigned)(Npad / 32)), dim3(32, 8), 0, st>>>(
        pa.cc, S + kNaCCT, N, Lc, Npad);
    NA(cudaGetLastError());
  }
  uint32_t h_evc[kNaMaxN], h_evoff[kNaMaxN + 1];
  NA(cudaMemcpyAsync(h_evc, pa.evcount, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA(cudaStreamSynchronize(st));
  h_evoff[0] = 0;
  uint32_t max_ev = 0;
  for (long i = 0; i < N; i++) {
    h_evoff[i + 1] = h_evoff[i] + h_evc[i];
    max_ev = std::max(max_ev, h_evc[i]);
  }
  rc.packed = max_ev <= (uint32_t)kPackedMaxEvents;
  NA(cudaMemcpyAsync(S + kNaEvoff, h_evoff, (N + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  if (W && h_evoff[N]) {
    events_kernel<<<(unsigned)((N + kWarps - 1) / kWarps), 256, 0, st>>>(pa);
    NA(cudaGetLastError());
  }
  build_tables(&g_na_tables, opts->mode, opts->subset);
  fill_pair_tables(g_na_tables, rc.wplane, &g_na_ptab);
  NA(cudaMemcpyAsync(S + kNaAgg, &g_na_ptab, sizeof(PairTables), cudaMemcpyHostToDevice, st));
  NA(cudaMemcpyAsync(S + kNaSite, g_na_tables.site, sizeof(g_na_tables.site), cudaMemcpyHostToDevice, st));
  unsigned *rqn = (unsigned *)(S + kNaRqn);
  unsigned long long *counters = (unsigned long long *)(S + kNaCounters);
  NA(cudaMemsetAsync(rqn, 0, sizeof(unsigned), st));
  NA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st));
  PairArgs A;
  A.rc = rc;
  A.planes = pa.planes;
  A.cc = pa.cc;
  A.ccT = S + kNaCCT;
  A.ev_off = pa.ev_off;
  A.ev = pa.ev;
  A.tab = (const PairTables *)(S + kNaAgg);
  A.r0 = 0;
  A.r1 = N;
  A.ncols = N;
  A.colbase = 0;
  A.cstart = 0;
  A.dist = d_dist;
  A.replay_q = (unsigned long long *)(S + kNaRq);
  A.replay_n = rqn;
  A.replay_cap = (unsigned long long)kNaMaxN * kNaMaxN;
  A.counters = counters;
  A.logt = (const LogTable *)(S + kNaLog);
  memset(&A.ex, 0, sizeof A.ex);  // raw distances only: no undecided list, no summary bounds
  NA(launch_pair(A, (N + 31) / 32, N, st));
  unsigned nq = 0;
  NA(cudaMemcpyAsync(&nq, rqn, sizeof nq, cudaMemcpyDeviceToHost, st));
  NA(cudaStreamSynchronize(st));
  if (nq) {
    ReplayArgs R;
    R.rc = rc;
    R.cc = pa.cc;
    R.planes = pa.planes;
    R.site = (const SiteEntry *)(S + kNaSite);
    R.q = A.replay_q;
    R.qn = rqn;
    R.qcap = A.replay_cap;
    R.r0 = 0;
    R.ncols = N;
    R.colbase = 0;
    R.dist = d_dist;
    R.counters = counters;
    R.logt = A.logt;
    R.ex = A.ex;
    replay_kernel<<<(unsigned)std::min<unsigned>(296, (nq + kWarps - 1) / kWarps), 256, 0, st>>>(R);
    NA(cudaGetLastError());
  }
  NA(cudaStreamSynchronize(st));
  return TN93G_OK;
#undef NA
}

}  // namespace

extern "C" {

int tn93g_pair_distances_noalloc(const uint8_t *d_codes, long N, long L, const tn93g_opts *opts, double *d_dist,
                                 void *stream)
{
  if (!d_codes || !opts || !d_dist || N <= 0 || L <= 0) {
    snprintf(g_na_err, sizeof g_na_err, "invalid argument: a null pointer or a size <= 0 (N = %ld, L = %ld)", N, L);
    return TN93G_EINVAL;
  }
  if (opts->mode < 0 || opts->mode > 4) {
    snprintf(g_na_err, sizeof g_na_err, "invalid argument: ambiguity mode %d", opts->mode);
    return TN93G_EINVAL;
  }
  g_na_err[0] = 0;
  std::lock_guard<std::mutex> g(g_na_mu);
  if (N > kNaMaxN || L > kNaMaxL) {
    snprintf(g_na_err, sizeof g_na_err,
             "alignment of %ld x %ld exceeds the fixed scratch of the allocation-free entry point (N <= %ld, L <= %ld)",
             N, L, kNaMaxN, kNaMaxL);
    return TN93G_ESCRATCH;
  }
  return noalloc_run(d_codes, N, L, opts, d_dist, (cudaStream_t)stream);
}

const char *tn93g_noalloc_last_error(void) { return g_na_err; }

}  // extern "C"

//================================================================================================== resident-reference server
// The -s mode as a service: a reference alignment stays packed on the device (bit planes, codes, sparse events,
// with room after it for query sequences) and batches of query alignments are run against it. One batch is one
// cross run (rows = reference, columns = the batch's queries, as tn93 -s QUERY REF orders them,
// swifttn93.cpp:2321-2322, 2392) whose stats, sums and text are segmented by query, so every query gets the
// distance file and summary of its own tn93 run. Columns are not folded (a fold must hold for every query that
// will ever come), which changes no result.
namespace {

// Server rows: one thread per (reference row, query). The 256 threads of a block are 256 consecutive rows of one
// query, so a warp walks the query's columns together (warp-uniform loop) while each thread adds its row's terms
// in column order, the order tn93 adds a row's pairs in (swifttn93.cpp:2594-2602). Statistics and row sums are
// fused; the histogram is aggregated per warp (lanes with the same bin add once) and per block in shared memory.
__global__ void __launch_bounds__(256) qstats_kernel(RowArgs a)
{
  __shared__ unsigned long long sh[kHistBins];
  for (int t = threadIdx.x; t < kHistBins; t += blockDim.x) sh[t] = 0;
  __syncthreads();
  const RunConsts &rc = a.rc;
  const int q = blockIdx.y;
  const long i = a.r0 + blockIdx.x * 256l + threadIdx.x;
  const bool row = i < a.r1;
  const long c0 = a.seg_cols[q], c1 = a.seg_cols[q + 1], jshift = c0 - rc.n1;
  const long ii = row ? i : a.r0;
  const long cnt_i = a.counts[ii];
  const int nli = a.name_len[ii];
  const int dli = rc.format == 1 ? digits_of(ii) : 0;
  double mx = 0., s0 = 0., w0 = 0.;
  long long links = 0, skipped = 0;
  unsigned long long bytes = 0;
  for (long j = c0; j < c1; j++) {
    PairView v = view_pair(a, ii, j, cnt_i);
    if (!row) v.valid = v.computed = v.linked = false;
    const int key = v.computed ? v.hb : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (__all_sync(0xffffffffu, !v.computed || v.w == 1)) {
      if (v.computed && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&sh[key], (unsigned long long)__popc(peers));
    } else if (v.computed) {
      atomicAdd(&sh[key], (unsigned long long)v.w);
    }
    if (!v.valid) continue;
    if (v.linked) {
      links += v.w;
      if (rc.emit) {
        const int gl = fmt_g_len(v.thisD);
        bytes += rc.format == 0 ? nli + a.name_len[j] + gl + 3 : dli + digits_of(j - jshift) + gl + 3;
      }
    }
    if (!v.counted) {
      skipped++;
    } else {
      mx = v.thisD > mx ? v.thisD : mx;
      s0 = __dadd_rn(s0, __dmul_rn(v.thisD, (double)v.w));
      w0 = __dadd_rn(w0, (double)v.w);
    }
  }
  if (row) {
    const size_t slot = (size_t)q * a.nrows + (i - a.r0);
    a.seg_bytes[slot] = bytes;
    a.seg_links[slot] = links;
    a.seg_skip[slot] = skipped;
    a.seg_max[slot * 3] = mx;
    a.seg_max[slot * 3 + 1] = 0.;
    a.seg_max[slot * 3 + 2] = 0.;
    a.row_sum[slot * 3] = s0;
    a.row_sum[slot * 3 + 1] = 0.;
    a.row_sum[slot * 3 + 2] = 0.;
    a.row_w[slot * 3] = w0;
    a.row_w[slot * 3 + 1] = 0.;
    a.row_w[slot * 3 + 2] = 0.;
  }
  __syncthreads();
  unsigned long long *hist = a.hist + (size_t)q * 3 * kHistBins;
  for (int t = threadIdx.x; t < kHistBins; t += blockDim.x)
    if (sh[t]) atomicAdd(&hist[t], sh[t]);
}

// Server text: one thread per (reference row, query) writes that row's lines for the query's columns at its
// scanned offset (the text is sparse at serving thresholds, so direct byte stores suffice).
__global__ void __launch_bounds__(256) qwrite_kernel(RowArgs a)
{
  const RunConsts &rc = a.rc;
  const int q = blockIdx.y;
  const long i = a.r0 + blockIdx.x * 256l + threadIdx.x;
  if (i >= a.r1) return;
  const size_t slot = (size_t)q * a.nrows + (i - a.r0);
  const unsigned long long nb = a.seg_bytes[slot];
  if (nb == 0) return;
  const long c0 = a.seg_cols[q], c1 = a.seg_cols[q + 1], jshift = c0 - rc.n1;
  const int nli = a.name_len[i];
  const char *ni = a.names + a.name_off[i];
  const int dli = rc.format == 1 ? digits_of(i) : 0;
  char *o = a.out + a.seg_off[slot], *const end = o + nb;
  for (long j = c0; j < c1; j++) {
    double thisD = 0.;
    if (!linked_pair(a, i, j, thisD)) continue;
    char g[24];
    const int gl = fmt_g(thisD, g);
    const int len = rc.format == 0 ? nli + a.name_len[j] + gl + 3 : dli + digits_of(j - jshift) + gl + 3;
    if (o + len > end) {
      atomicAdd(a.err, 1ull);
      return;
    }
    put_line(o, a, i, j, jshift, ni, nli, g, gl);
    o += len;
  }
  if (o != end) atomicAdd(a.err, 1ull);
}

// Per query: links, skips and maxima over the reference rows, and tn93's mean numerator and weight: the rows' sums
// added in row order, as tn93's writer adds them (swifttn93.cpp:2838-2848). One block per query: the block stages
// chunks of row sums in shared memory with coalesced loads (and reduces the order-free counts and maxima), then
// thread 0 adds the chunk in row order. Only bin 0 is used in a server batch (no -m).
constexpr int kReduceChunk = 2048;

__global__ void __launch_bounds__(256) query_reduce_kernel(RowArgs a, int nq, double *qout /* [nq][9] */,
                                                           long long *qlinks /* [nq][2] */)
{
  __shared__ double ss[kReduceChunk], sw[kReduceChunk];
  __shared__ long long rl[8], rs[8];
  __shared__ double rm[8];
  const int q = blockIdx.x;
  const long nr = a.nrows;
  const size_t base = (size_t)q * nr;
  long long links = 0, skipped = 0;
  double m = 0., s0 = 0., w0 = 0.;
  for (long r0 = 0; r0 < nr; r0 += kReduceChunk) {
    const int n = (int)min((long)kReduceChunk, nr - r0);
    for (int k = threadIdx.x; k < n; k += 256) {
      const size_t slot = base + r0 + k;
      links += a.seg_links[slot];
      skipped += a.seg_skip[slot];
      m = fmax(m, a.seg_max[slot * 3]);
      ss[k] = a.row_sum[slot * 3];
      sw[k] = a.row_w[slot * 3];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll 8
      for (int k = 0; k < n; k++) {
        s0 = __dadd_rn(s0, ss[k]);
        w0 = __dadd_rn(w0, sw[k]);
      }
    }
    __syncthreads();
  }
  for (int o = 16; o; o >>= 1) {
    links += __shfl_xor_sync(0xffffffffu, links, o);
    skipped += __shfl_xor_sync(0xffffffffu, skipped, o);
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    rl[threadIdx.x >> 5] = links;
    rs[threadIdx.x >> 5] = skipped;
    rm[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; w++) {
      links += rl[w];
      skipped += rs[w];
      m = fmax(m, rm[w]);
    }
    double *o = qout + (size_t)q * 9;
    o[0] = m;
    o[1] = o[2] = 0.;
    o[3] = s0;
    o[4] = o[5] = 0.;
    o[6] = w0;
    o[7] = o[8] = 0.;
    qlinks[q * 2] = links;
    qlinks[q * 2 + 1] = skipped;
  }
}

}  // namespace

struct tn93g_server {
  tn93g_ctx *ctx = nullptr;
  RunConsts base;
  long Nref = 0, L = 0, W = 0, Npad = 0, cap_q = 0;
  int cap_nq = 0;
  size_t ev_ref = 0, ev_cap = 0, names_ref = 0;
  DevBuf planes, cc, ccT, evcount, evoff, ev, agg, site, varcol, qcodes, counts, names, name_off, name_len, dist, rq,
      rqn, counters, segcols, sbytes, soff, slinks, sskip, smax, rsum, rw, hist, total, out, qout, qlinks, scantmp;
  void *pin = nullptr;
  size_t pin_n = 0;
  // tensor-core counts: the one-hot image of the reference and the batch's queries, and the aggregates of one
  // chunk of query columns at a time
  bool tc = false;
  int tc16 = 0;
  long tc_NB = 0, tc_KS = 0;
  DevBuf ohimg, tcagg, tcerr;
  // exactness: the undecided list (capacity und_cap entries; grown for an exact-sums pass), its count, the
  // per-query bounds, the query of each column, the replay descriptor the resolver reads
  DevBuf und, undn, amb, colunit, rdesc;
  unsigned und_cap = 0;
  uint32_t ref_max_ev = 0;  // most sparse events of a reference sequence (the packed sums need <= kPackedMaxEvents)
};

namespace {
constexpr long kServerTcChunk = 128;  // query columns per tensor-core count launch (a multiple of 64): the
                                      // records of a 30,000-sequence reference x 128 columns (61 MB) stay in L2

// opt-in to the count kernel's dynamic shared memory on the current device
int tc_attr(tn93g_ctx *ctx)
{
  CU(tc_attr_once());
  return TN93G_OK;
}
}  // namespace

extern "C" {

void tn93g_server_destroy(tn93g_server *srv)
{
  if (!srv) return;
  tn93g_ctx *ctx = srv->ctx;
  if (ctx) cudaSetDevice(ctx->device);
  DevBuf *bufs[] = {&srv->planes, &srv->cc, &srv->ccT, &srv->evcount, &srv->evoff, &srv->ev, &srv->agg, &srv->site,
                    &srv->varcol, &srv->qcodes, &srv->counts, &srv->names, &srv->name_off, &srv->name_len,
                    &srv->dist, &srv->rq, &srv->rqn, &srv->counters, &srv->segcols, &srv->sbytes, &srv->soff,
                    &srv->slinks, &srv->sskip, &srv->smax, &srv->rsum, &srv->rw, &srv->hist, &srv->total,
                    &srv->out, &srv->qout, &srv->qlinks, &srv->scantmp, &srv->ohimg, &srv->tcagg, &srv->tcerr,
                    &srv->und, &srv->undn, &srv->amb, &srv->colunit, &srv->rdesc};
  for (DevBuf *b : bufs)
    if (b->p) {
      cudaFree(b->p);
      if (ctx) ctx->used -= b->n;
    }
  if (srv->pin) cudaFreeHost(srv->pin);
  delete srv;
}

int tn93g_server_create(tn93g_ctx *ctx, tn93g_server **out, const uint8_t *codes, long N, long L,
                        const long *copy_counts, const char *names, const size_t *name_off, const long *name_len,
                        const tn93g_opts *opts, long max_batch_sequences, int max_batch_queries)
{
  if (!ctx || !out || !codes || N <= 0 || L <= 0 || !copy_counts || !names || !name_off || !name_len || !opts ||
      max_batch_sequences <= 0 || max_batch_queries <= 0 || max_batch_queries > 65535)
    return TN93G_EINVAL;
  if (opts->mode < 0 || opts->mode > 4 || opts->format < 0 || opts->format > 1) return TN93G_EINVAL;
  if (L >= (1l << 25) || N > 65535l * 32 || (unsigned long)(N + max_batch_sequences) * (unsigned long)L >= (1ul << 32))
    return TN93G_ETOOBIG;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  tn93g_server *srv = new tn93g_server();
  srv->ctx = ctx;
  int rc_ = TN93G_OK;
#define SV(x)                   \
  do {                          \
    rc_ = (x);                  \
    if (rc_ != TN93G_OK) {      \
      tn93g_server_destroy(srv); \
      return rc_;               \
    }                           \
  } while (0)
#define SVC(call)                                                     \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) {                                          \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);  \
      tn93g_server_destroy(srv);                                      \
      return TN93G_ECUDA;                                             \
    }                                                                 \
  } while (0)
  RunConsts &rc = srv->base;
  memset(&rc, 0, sizeof rc);
  rc.mode = opts->mode;
  rc.gapmm = opts->mode == TN93G_GAPMM;
  rc.cross = true;
  rc.fallback_avg = (opts->mode == TN93G_RESOLVE || opts->mode == TN93G_SUBSET) && opts->resolve_fraction < 1.;
  rc.emit = !opts->count_only;
  rc.format = opts->format;
  rc.delim = opts->delimiter;
  rc.threshold = opts->threshold;
  rc.min_distance = opts->min_distance;
  rc.resolve_fraction = opts->resolve_fraction;
  rc.min_overlap = opts->min_overlap;
  rc.log_band = ctx->log_band;
  rc.log_spread = ctx->log_spread;
  rc.resolve_all = ctx->exact_sums;
  srv->Nref = N;
  srv->L = L;
  srv->W = (L + 63) / 64;
  srv->cap_q = max_batch_sequences;
  srv->cap_nq = max_batch_queries;
  srv->Npad = (N + max_batch_sequences + 63) / 32 * 32;
  const long cap_n = N + max_batch_sequences, Np = srv->Npad, W = srv->W;
  rc.Lc = L;
  rc.W = W;
  rc.Npad = Np;
  rc.NP = rc.gapmm ? 5 : 4;
  // the reference's codes, its N count (the N plane is used when N is frequent, as in tn93g_run)
  SV(ensure(ctx, srv->qcodes, std::max<size_t>((size_t)N, (size_t)max_batch_sequences) * L));
  SVC(cudaMemcpyAsync(srv->qcodes.p, codes, (size_t)N * L, cudaMemcpyHostToDevice, st));
  SV(ensure(ctx, ctx->seen, L * sizeof(uint32_t)));
  SV(ensure(ctx, ctx->nN, sizeof(unsigned long long)));
  SVC(cudaMemsetAsync(ctx->seen.p, 0, L * sizeof(uint32_t), st));
  SVC(cudaMemsetAsync(ctx->nN.p, 0, sizeof(unsigned long long), st));
  colscan_kernel<<<dim3((unsigned)((L + 255) / 256), (unsigned)((N + 63) / 64)), 256, 0, st>>>(
      (const uint8_t *)srv->qcodes.p, N, L, (uint32_t *)ctx->seen.p, (unsigned long long *)ctx->nN.p);
  SVC(cudaGetLastError());
  unsigned long long nN = 0;
  SVC(cudaMemcpyAsync(&nN, ctx->nN.p, sizeof nN, cudaMemcpyDeviceToHost, st));
  SVC(cudaStreamSynchronize(st));
  rc.wplane = rc.gapmm || nN > 16ull * (unsigned long long)N;
  // resident arrays with room for max_batch_sequences query sequences after the reference
  SV(ensure(ctx, srv->planes, (size_t)W * rc.NP * Np * sizeof(uint64_t)));
  SV(ensure(ctx, srv->cc, (size_t)cap_n * L));
  SV(ensure(ctx, srv->ccT, (size_t)L * Np));
  SV(ensure(ctx, srv->evcount, cap_n * sizeof(uint32_t)));
  SV(ensure(ctx, srv->evoff, (cap_n + 1) * sizeof(uint32_t)));
  SV(ensure(ctx, srv->varcol, L * sizeof(int32_t)));
  SVC(cudaMemsetAsync(srv->planes.p, 0, (size_t)W * rc.NP * Np * sizeof(uint64_t), st));
  SVC(cudaMemsetAsync(srv->evcount.p, 0, cap_n * sizeof(uint32_t), st));
  {
    std::vector<int32_t> id(L);
    for (long p = 0; p < L; p++) id[p] = (int32_t)p;
    SVC(cudaMemcpy(srv->varcol.p, id.data(), L * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  PackArgs pa;
  pa.codes = (const uint8_t *)srv->qcodes.p;
  pa.N = N;
  pa.L = L;
  pa.Lc = L;
  pa.W = W;
  pa.Npad = Np;
  pa.varcol = (const int32_t *)srv->varcol.p;
  pa.NP = rc.NP;
  pa.wplane = rc.wplane;
  pa.gapmm = rc.gapmm;
  pa.planes = (uint64_t *)srv->planes.p;
  pa.cc = (uint8_t *)srv->cc.p;
  pa.evcount = (uint32_t *)srv->evcount.p;
  pack_kernel<<<dim3((unsigned)((N + kWarps - 1) / kWarps), (unsigned)std::min<long>(W, 65535)), 256, 0, st>>>(pa);
  SVC(cudaGetLastError());
  transpose_kernel<<<dim3((unsigned)((L + 31) / 32), (unsigned)((N + 31) / 32)), dim3(32, 8), 0, st>>>(
      (const uint8_t *)srv->cc.p, (uint8_t *)srv->ccT.p, N, L, Np);
  SVC(cudaGetLastError());
  std::vector<uint32_t> evc(N), evo(N + 1);
  SVC(cudaMemcpyAsync(evc.data(), srv->evcount.p, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  SVC(cudaStreamSynchronize(st));
  evo[0] = 0;
  for (long i = 0; i < N; i++) {
    evo[i + 1] = evo[i] + evc[i];
    srv->ref_max_ev = std::max(srv->ref_max_ev, evc[i]);
  }
  srv->ev_ref = evo[N];
  srv->ev_cap = srv->ev_ref + (size_t)max_batch_sequences * L;
  SV(ensure(ctx, srv->ev, std::max<size_t>(srv->ev_cap, 1) * sizeof(uint32_t)));
  SVC(cudaMemcpyAsync(srv->evoff.p, evo.data(), (N + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  pa.ev_off = (const uint32_t *)srv->evoff.p;
  pa.ev = (uint32_t *)srv->ev.p;
  if (srv->ev_ref) {
    events_kernel<<<(unsigned)((N + kWarps - 1) / kWarps), 256, 0, st>>>(pa);
    SVC(cudaGetLastError());
  }
  // tables of the server's mode
  build_tables(ctx->h_tab, opts->mode, opts->subset);
  fill_pair_tables(*ctx->h_tab, rc.wplane, ctx->h_ptab);
  SV(ensure(ctx, srv->agg, sizeof(PairTables)));
  SV(ensure(ctx, srv->site, sizeof(ctx->h_tab->site)));
  SVC(cudaMemcpyAsync(srv->agg.p, ctx->h_ptab, sizeof(PairTables), cudaMemcpyHostToDevice, st));
  SVC(cudaMemcpyAsync(srv->site.p, ctx->h_tab->site, sizeof(ctx->h_tab->site), cudaMemcpyHostToDevice, st));
  // names, name offsets and lengths, copy numbers of every sequence (the reference's now, the queries' per batch)
  size_t nbytes = 0;
  for (long i = 0; i < N; i++) nbytes = std::max(nbytes, name_off[i] + (size_t)name_len[i]);
  srv->names_ref = nbytes;
  SV(ensure(ctx, srv->names, nbytes + 1 + (size_t)max_batch_sequences * 64));
  SV(ensure(ctx, srv->name_off, cap_n * sizeof(uint64_t)));
  SV(ensure(ctx, srv->name_len, cap_n * sizeof(int32_t)));
  SV(ensure(ctx, srv->counts, cap_n * sizeof(long)));
  std::vector<uint64_t> off(name_off, name_off + N);
  std::vector<int32_t> nl(N);
  for (long i = 0; i < N; i++) nl[i] = (int32_t)name_len[i];
  if (nbytes) SVC(cudaMemcpyAsync(srv->names.p, names, nbytes, cudaMemcpyHostToDevice, st));
  SVC(cudaMemcpyAsync(srv->name_off.p, off.data(), N * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  SVC(cudaMemcpyAsync(srv->name_len.p, nl.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  SVC(cudaMemcpyAsync(srv->counts.p, copy_counts, N * sizeof(long), cudaMemcpyHostToDevice, st));
  // per-batch buffers at capacity (a batch never reallocates them): distances and the replay queue of every
  // pair, per (query, row) statistics, per-query histograms and results
  {
    const size_t dslots = (size_t)N * max_batch_sequences, nslot = (size_t)max_batch_queries * N;
    const int nq = max_batch_queries;
    SV(ensure(ctx, srv->dist, dslots * sizeof(double)));
    SV(ensure(ctx, srv->rq, dslots * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->rqn, sizeof(unsigned)));
    SV(ensure(ctx, srv->counters, 4 * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->sbytes, nslot * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->soff, nslot * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->slinks, nslot * sizeof(long long)));
    SV(ensure(ctx, srv->sskip, nslot * sizeof(long long)));
    SV(ensure(ctx, srv->smax, nslot * 3 * sizeof(double)));
    SV(ensure(ctx, srv->rsum, nslot * 3 * sizeof(double)));
    SV(ensure(ctx, srv->rw, nslot * 3 * sizeof(double)));
    SV(ensure(ctx, srv->hist, (size_t)nq * 3 * kHistBins * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->total, sizeof(unsigned long long)));
    SV(ensure(ctx, srv->segcols, (nq + 1) * sizeof(long)));
    SV(ensure(ctx, srv->qout, (size_t)nq * 9 * sizeof(double)));
    SV(ensure(ctx, srv->qlinks, (size_t)nq * 2 * sizeof(long long)));
    SV(ensure(ctx, srv->scantmp, (2 * (nslot / kScanTile + 1) + 1) * sizeof(unsigned long long)));
    srv->und_cap = (unsigned)std::min<size_t>(std::max<size_t>(4096, dslots / 64), 0xFFFFFFF0u);
    SV(ensure(ctx, srv->und, (size_t)srv->und_cap * 2 * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->undn, sizeof(unsigned long long)));
    SV(ensure(ctx, srv->amb, (size_t)nq * 4 * sizeof(unsigned long long)));
    SV(ensure(ctx, srv->colunit, (size_t)max_batch_sequences * sizeof(int)));
    SV(ensure(ctx, srv->rdesc, sizeof(ReplayArgs)));
    // a first text buffer (device and pinned host), so that early batches do not stall on growth
    const size_t text0 = 32u << 20;
    SV(ensure(ctx, srv->out, text0));
    SVC(cudaHostAlloc(&srv->pin, text0, cudaHostAllocDefault));
    srv->pin_n = text0;
  }
  // tensor-core counts (the context's count path): the reference's blocks of the one-hot image now, the blocks
  // holding queries per batch; when the budget cannot hold the image and one chunk of aggregates, the server
  // counts with POPC instead (same results)
  if (ctx->count_path == 1) {
    srv->tc_NB = (N + max_batch_sequences + 31) / 32 + 1;
    srv->tc_KS = (L + kTcStageK - 1) / kTcStageK;
    srv->tc16 = 32 * L < 65536;
    const size_t img = (size_t)srv->tc_KS * srv->tc_NB * kTcBlockBytes;
    const size_t agg = (size_t)N * kServerTcChunk * (srv->tc16 ? 16 : 32);
    if (ensure(ctx, srv->ohimg, img) == TN93G_OK && ensure(ctx, srv->tcagg, agg) == TN93G_OK &&
        ensure(ctx, srv->tcerr, sizeof(unsigned long long)) == TN93G_OK) {
      srv->tc = true;
      SV(tc_attr(ctx));
      const long nfull = N / 32 * 32;  // whole reference blocks (the block shared with queries is built per batch)
      if (nfull) {
        const long nthr = nfull * srv->tc_KS * (kTcStageK / 16);
        onehot_kernel<<<(unsigned)((nthr + 255) / 256), 256, 0, st>>>((const uint8_t *)srv->cc.p, N, L, srv->tc_NB,
                                                                      srv->tc_KS, (uint8_t *)srv->ohimg.p, 0, nfull);
        SVC(cudaGetLastError());
      }
    } else {
      for (DevBuf *b : {&srv->ohimg, &srv->tcagg, &srv->tcerr})
        if (b->p) {
          cudaFree(b->p);
          ctx->used -= b->n;
          b->p = nullptr;
          b->n = 0;
        }
      ctx->err.clear();
    }
  }
  SVC(cudaStreamSynchronize(st));
#undef SV
#undef SVC
  *out = srv;
  return TN93G_OK;
}

int tn93g_server_batch(tn93g_server *srv, int nq, const tn93g_alignment *queries, tn93g_query_sink sink, void *user,
                       tn93g_summary *sums)
{
  if (!srv || nq <= 0 || !queries || !sums) return TN93G_EINVAL;
  tn93g_ctx *ctx = srv->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  ctx->launches = 0;
  for (double &t : ctx->timings) t = 0;
  cudaEvent_t *E = ctx->evs;  // stage boundaries: start, packed, pair, replay, rows, written, copied
  const long Nref = srv->Nref, L = srv->L, Np = srv->Npad, W = srv->W;
  if (nq > srv->cap_nq) {
    ctx->err = "more queries than the server's batch capacity";
    return TN93G_EINVAL;
  }
  std::vector<long> qstart(nq + 1);
  qstart[0] = 0;
  for (int q = 0; q < nq; q++) {
    if (queries[q].n <= 0 || queries[q].L != srv->L || !queries[q].codes || !queries[q].copy_counts ||
        !queries[q].names || !queries[q].name_off || !queries[q].name_len)
      return TN93G_EINVAL;
    qstart[q + 1] = qstart[q] + queries[q].n;
  }
  const long Q = qstart[nq];
  if (Q > srv->cap_q) {
    ctx->err = "batch larger than the server's query capacity";
    return TN93G_EINVAL;
  }
  // query codes, names, offsets, lengths and copy numbers into the slots after the reference
  std::vector<uint64_t> off(Q);
  std::vector<int32_t> nl(Q);
  std::vector<long> cnt(Q);
  size_t nb = srv->names_ref;
  std::vector<size_t> qname_base(nq);
  for (int q = 0; q < nq; q++) {
    size_t qn = 0;
    for (long k = 0; k < queries[q].n; k++) qn = std::max(qn, queries[q].name_off[k] + (size_t)queries[q].name_len[k]);
    qname_base[q] = nb;
    for (long k = 0; k < queries[q].n; k++) {
      off[qstart[q] + k] = nb + queries[q].name_off[k];
      nl[qstart[q] + k] = (int32_t)queries[q].name_len[k];
      cnt[qstart[q] + k] = queries[q].copy_counts[k];
    }
    nb += qn;
  }
  TRY(ensure_keep(ctx, srv->names, nb + 1, srv->names_ref));
  CU(cudaEventRecord(E[0], st));
  for (int q = 0; q < nq; q++) {
    CU(cudaMemcpyAsync((uint8_t *)srv->qcodes.p + (size_t)qstart[q] * L, queries[q].codes, (size_t)queries[q].n * L,
                       cudaMemcpyHostToDevice, st));
    size_t qn = 0;
    for (long k = 0; k < queries[q].n; k++) qn = std::max(qn, queries[q].name_off[k] + (size_t)queries[q].name_len[k]);
    if (qn) CU(cudaMemcpyAsync((char *)srv->names.p + qname_base[q], queries[q].names, qn, cudaMemcpyHostToDevice, st));
  }
  CU(cudaMemcpyAsync((uint64_t *)srv->name_off.p + Nref, off.data(), Q * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync((int32_t *)srv->name_len.p + Nref, nl.data(), Q * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync((long *)srv->counts.p + Nref, cnt.data(), Q * sizeof(long), cudaMemcpyHostToDevice, st));
  // pack the queries into their slots
  RunConsts rc = srv->base;
  rc.N = Nref + Q;
  rc.n1 = Nref;
  PackArgs pa;
  pa.codes = (const uint8_t *)srv->qcodes.p;
  pa.N = Q;
  pa.L = L;
  pa.Lc = L;
  pa.W = W;
  pa.Npad = Np;
  pa.varcol = (const int32_t *)srv->varcol.p;
  pa.NP = rc.NP;
  pa.wplane = rc.wplane;
  pa.gapmm = rc.gapmm;
  pa.planes = (uint64_t *)srv->planes.p + Nref;
  pa.cc = (uint8_t *)srv->cc.p + (size_t)Nref * L;
  pa.evcount = (uint32_t *)srv->evcount.p + Nref;
  CU(cudaMemsetAsync(pa.evcount, 0, Q * sizeof(uint32_t), st));
  pack_kernel<<<dim3((unsigned)((Q + kWarps - 1) / kWarps), (unsigned)std::min<long>(W, 65535)), 256, 0, st>>>(pa);
  CU(cudaGetLastError());
  ctx->launches++;
  transpose_kernel<<<dim3((unsigned)((L + 31) / 32), (unsigned)((Q + 31) / 32)), dim3(32, 8), 0, st>>>(
      pa.cc, (uint8_t *)srv->ccT.p + Nref, Q, L, Np);
  CU(cudaGetLastError());
  ctx->launches++;
  std::vector<uint32_t> evc(Q), evo(Q + 1);
  CU(cudaMemcpyAsync(evc.data(), pa.evcount, Q * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  evo[0] = (uint32_t)srv->ev_ref;
  uint32_t max_ev = srv->ref_max_ev;
  for (long k = 0; k < Q; k++) {
    evo[k + 1] = evo[k] + evc[k];
    max_ev = std::max(max_ev, evc[k]);
  }
  rc.packed = max_ev <= (uint32_t)kPackedMaxEvents;
  CU(cudaMemcpyAsync((uint32_t *)srv->evoff.p + Nref, evo.data(), (Q + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                     st));
  pa.ev_off = (const uint32_t *)srv->evoff.p + Nref;
  pa.ev = (uint32_t *)srv->ev.p;
  if (evo[Q] > evo[0]) {
    events_kernel<<<(unsigned)((Q + kWarps - 1) / kWarps), 256, 0, st>>>(pa);
    CU(cudaGetLastError());
    ctx->launches++;
  }
  CU(cudaEventRecord(E[1], st));
  // the cross run: rows = reference, columns = the batch's queries
  const size_t dslots = (size_t)Nref * Q;
  const size_t nslot = (size_t)nq * Nref;
  CU(cudaMemsetAsync(srv->counters.p, 0, 4 * sizeof(unsigned long long), st));
  CU(cudaMemsetAsync(srv->amb.p, 0, (size_t)nq * 4 * sizeof(unsigned long long), st));
  std::vector<long> segc(nq + 1);
  for (int q = 0; q <= nq; q++) segc[q] = Nref + qstart[q];
  CU(cudaMemcpyAsync(srv->segcols.p, segc.data(), (nq + 1) * sizeof(long), cudaMemcpyHostToDevice, st));
  {
    std::vector<int> cu(Q);
    for (int q = 0; q < nq; q++)
      for (long k = qstart[q]; k < qstart[q + 1]; k++) cu[k] = q;
    CU(cudaMemcpyAsync(srv->colunit.p, cu.data(), Q * sizeof(int), cudaMemcpyHostToDevice, st));
  }
  if (srv->tc) {
    // the image blocks from the one shared by the reference's last rows and the first queries, through one zero
    // block past the last query
    const long b0 = Nref / 32, b1 = (Nref + Q + 31) / 32 + 1;
    const long nthr = (b1 - b0) * 32 * srv->tc_KS * (kTcStageK / 16);
    CU(cudaMemsetAsync(srv->tcerr.p, 0, sizeof(unsigned long long), st));
    onehot_kernel<<<(unsigned)((nthr + 255) / 256), 256, 0, st>>>((const uint8_t *)srv->cc.p, Nref + Q, L, srv->tc_NB,
                                                                  srv->tc_KS, (uint8_t *)srv->ohimg.p, b0 * 32,
                                                                  (b1 - b0) * 32);
    CU(cudaGetLastError());
    ctx->launches++;
  }
  ReplayArgs R;
  // pair stage (and the site-order replay) of the whole batch; resolve_all: an exact-sums pass
  auto enqueue_pairs = [&](bool resolve_all) -> int {
    RunConsts rcp = rc;
    rcp.resolve_all = rc.resolve_all || resolve_all;
    CU(cudaMemsetAsync(srv->rqn.p, 0, sizeof(unsigned), st));
    CU(cudaMemsetAsync(srv->undn.p, 0, sizeof(unsigned long long), st));
    ExactSink ex;
    ex.und_list = (unsigned long long *)srv->und.p;
    ex.und_n = (unsigned *)srv->undn.p;
    ex.und_cap = srv->und_cap;
    ex.und_k = 0;
    ex.amb = resolve_all ? nullptr : (unsigned long long *)srv->amb.p;
    ex.counts = (const long *)srv->counts.p;
    ex.colunit = (const int *)srv->colunit.p;
    PairArgs A;
    A.rc = rcp;
    A.planes = (const uint64_t *)srv->planes.p;
    A.cc = (const uint8_t *)srv->cc.p;
    A.ccT = (const uint8_t *)srv->ccT.p;
    A.ev_off = (const uint32_t *)srv->evoff.p;
    A.ev = (const uint32_t *)srv->ev.p;
    A.tab = (const PairTables *)srv->agg.p;
    A.r0 = 0;
    A.r1 = Nref;
    A.ncols = Q;
    A.colbase = Nref;
    A.cstart = Nref;
    A.dist = (double *)srv->dist.p;
    A.replay_q = (unsigned long long *)srv->rq.p;
    A.replay_n = (unsigned *)srv->rqn.p;
    A.replay_cap = dslots;
    A.counters = (unsigned long long *)srv->counters.p;
    A.logt = ctx->d_logt;
    A.ex = ex;
    if (srv->tc) {
      // per chunk of query columns: counts on the tensor cores, then the pair kernel
      for (long c0 = Nref; c0 < Nref + Q; c0 += kServerTcChunk) {
        const long c1 = std::min(Nref + Q, c0 + kServerTcChunk);
        TcArgs T;
        T.onehot = (const uint8_t *)srv->ohimg.p;
        T.NB = srv->tc_NB;
        T.KS = srv->tc_KS;
        T.N = Nref + Q;
        T.n1 = Nref;
        T.cross = true;
        T.r0 = 0;
        T.r1 = Nref;
        T.ncols = kServerTcChunk;
        T.colbase = c0;
        T.cstart = c0 / kTcCols * kTcCols;
        T.cend = c1;
        T.agg = srv->tcagg.p;
        T.agg16 = srv->tc16;
        T.err = (unsigned long long *)srv->tcerr.p;
        T.wait_ns = ctx->wait_ns;
        T.skip_fill_block = -1;
        const dim3 g((unsigned)((c1 - T.cstart + kTcCols - 1) / kTcCols), (unsigned)((Nref + kTcRows - 1) / kTcRows));
        CU(launch_count_grid(T, g.x, g.y, ctx->sms, st));
        PairArgs AC = A;
        AC.tcagg = srv->tcagg.p;
        AC.tc16 = srv->tc16;
        AC.split = pair_split(AC.rc);
        AC.tcncols = kServerTcChunk;
        AC.tccolbase = c0;
        AC.cstart = c0;
        CU(launch_pair(AC, (c1 - c0 + 31) / 32, Nref, st));
        ctx->launches += AC.split ? 3 : 2;
      }
    } else {
      CU(launch_pair(A, (Q + 31) / 32, Nref, st));
      ctx->launches++;
    }
    CU(cudaEventRecord(E[2], st));
    R.rc = rcp;
    R.cc = A.cc;
    R.planes = A.planes;
    R.site = (const SiteEntry *)srv->site.p;
    R.q = A.replay_q;
    R.qn = A.replay_n;
    R.qcap = dslots;
    R.r0 = 0;
    R.ncols = Q;
    R.colbase = Nref;
    R.dist = A.dist;
    R.counters = A.counters;
    R.logt = ctx->d_logt;
    R.ex = ex;
    replay_kernel<<<2 * ctx->sms, 256, 0, st>>>(R);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(E[3], st));
    return TN93G_OK;
  };
  RowArgs RA;
  RA.rc = rc;
  RA.dist = (const double *)srv->dist.p;
  RA.r0 = 0;
  RA.r1 = Nref;
  RA.ncols = Q;
  RA.colbase = Nref;
  RA.counts = (const long *)srv->counts.p;
  RA.name_len = (const int32_t *)srv->name_len.p;
  RA.name_off = (const uint64_t *)srv->name_off.p;
  RA.names = (const char *)srv->names.p;
  RA.maxseg = nq;
  RA.seg_cols = (const long *)srv->segcols.p;
  RA.nrows = Nref;
  RA.seg_bytes = (unsigned long long *)srv->sbytes.p;
  RA.seg_links = (long long *)srv->slinks.p;
  RA.seg_skip = (long long *)srv->sskip.p;
  RA.seg_max = (double *)srv->smax.p;
  RA.row_sum = (double *)srv->rsum.p;
  RA.row_w = (double *)srv->rw.p;
  RA.hist = (unsigned long long *)srv->hist.p;
  RA.seg_off = (const unsigned long long *)srv->soff.p;
  RA.hy = nullptr;
  RA.err = (unsigned long long *)srv->counters.p + 3;
  RA.out = nullptr;
  const dim3 g2((unsigned)((Nref + 255) / 256), (unsigned)nq);
  unsigned long long total = 0, und = 0;
  std::vector<double> qo((size_t)nq * 9);
  std::vector<long long> ql((size_t)nq * 2);
  std::vector<unsigned long long> qoff(nq + 1), hist((size_t)nq * 3 * kHistBins), ambw((size_t)nq * 4);
  unsigned long long counters[4];
  // row stage (per-query statistics and row sums, scan, per-query reduction) and its results on the host
  auto rows_and_read = [&]() -> int {
    CU(cudaMemsetAsync(srv->hist.p, 0, (size_t)nq * 3 * kHistBins * sizeof(unsigned long long), st));
    qstats_kernel<<<g2, 256, 0, st>>>(RA);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(launch_scan(RA.seg_bytes, (unsigned long long *)RA.seg_off, (long)nslot, (unsigned long long *)srv->total.p,
                   (unsigned long long *)srv->scantmp.p, st));
    ctx->launches++;
    query_reduce_kernel<<<(unsigned)nq, 256, 0, st>>>(RA, nq, (double *)srv->qout.p, (long long *)srv->qlinks.p);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(E[4], st));
    CU(cudaMemcpyAsync(&total, srv->total.p, sizeof total, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(qo.data(), srv->qout.p, qo.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(ql.data(), srv->qlinks.p, ql.size() * sizeof(long long), cudaMemcpyDeviceToHost, st));
    for (int q = 0; q < nq; q++)
      CU(cudaMemcpyAsync(&qoff[q], (unsigned long long *)srv->soff.p + (size_t)q * Nref, sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(hist.data(), srv->hist.p, hist.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       st));
    CU(cudaMemcpyAsync(counters, srv->counters.p, sizeof counters, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(&und, srv->undn.p, sizeof und, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return TN93G_OK;
  };
  // finishes the listed undecided pairs with the C library's logarithms and runs the row stage again
  long resolved = 0;
  auto resolve_and_reread = [&]() -> int {
    if (und > srv->und_cap) {
      ctx->err = "more undecided pairs in a batch than its list holds";
      return TN93G_EUNDECIDED;
    }
    CU(cudaMemcpyAsync(srv->rdesc.p, &R, sizeof R, cudaMemcpyHostToDevice, st));
    TRY(resolve_listed(ctx, (const ReplayArgs *)srv->rdesc.p, (const unsigned long long *)srv->und.p, (unsigned)und,
                       st));
    resolved += (long)und;
    return rows_and_read();
  };
  TRY(enqueue_pairs(false));
  TRY(rows_and_read());
  if (srv->tc) {
    unsigned long long tcerr = 0;
    CU(cudaMemcpy(&tcerr, srv->tcerr.p, sizeof tcerr, cudaMemcpyDeviceToHost));
    if (tcerr) {
      ctx->err = "the tensor-core count kernel timed out waiting for its pipeline";
      return TN93G_ETIMEOUT;
    }
  }
  const long ambiguous0 = (long)counters[0];
  // more undecided pairs than the list holds: grow it and run the batch's pair stage again (the same pairs are
  // listed; the per-query bounds only widen)
  auto grow_and_rerun = [&](bool resolve_all) -> int {
    const unsigned cap = (unsigned)std::min<unsigned long long>(
        std::max<unsigned long long>(und + und / 4 + 1024, 2ull * srv->und_cap), std::min<size_t>(dslots, 0xFFFFFFF0u));
    TRY(ensure(ctx, srv->und, (size_t)cap * 2 * sizeof(unsigned long long)));
    srv->und_cap = cap;
    TRY(enqueue_pairs(resolve_all));
    return rows_and_read();
  };
  if (und > srv->und_cap) TRY(grow_and_rerun(false));
  if (und) TRY(resolve_and_reread());
  // per query: the JSON numbers certain for every rounding of the C library's log, or an exact-sums pass
  CU(cudaMemcpy(ambw.data(), srv->amb.p, ambw.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  std::vector<tn93g_summary> S(nq);
  auto fill_summaries = [&]() {
    for (int q = 0; q < nq; q++) {
      tn93g_summary &X = S[q];
      memset(&X, 0, sizeof X);
      X.pairwise = (unsigned long)Nref * (unsigned long)queries[q].n;
      X.links = (long)ql[q * 2];
      X.skipped = (long)ql[q * 2 + 1];
      for (int k = 0; k < 3; k++) {
        X.max[k] = qo[q * 9 + k];
        X.mean[k] = qo[q * 9 + 3 + k];
        X.weighted[k] = qo[q * 9 + 6 + k];
        for (int b = 0; b < kHistBins; b++) X.hist[k][b] = hist[((size_t)q * 3 + k) * kHistBins + b];
      }
    }
  };
  fill_summaries();
  bool repass = false;
  for (int q = 0; q < nq && !rc.resolve_all; q++) {
    amb_bounds(&ambw[(size_t)q * 4], S[q].amb_bounds[0]);
    if (!summary_certified(&S[q], S[q].amb_bounds, Nref + queries[q].n + 2, 0)) repass = true;
  }
  if (repass) {
    // every pair with an ambiguous logarithm finished with the C library's log (the list must hold all of them)
    const unsigned cap = (unsigned)std::min<size_t>(dslots, 0xFFFFFFF0u);
    if (cap > srv->und_cap) {
      TRY(ensure(ctx, srv->und, (size_t)cap * 2 * sizeof(unsigned long long)));
      srv->und_cap = cap;
    }
    TRY(enqueue_pairs(true));
    TRY(rows_and_read());
    if (und > srv->und_cap) TRY(grow_and_rerun(true));
    if (und) TRY(resolve_and_reread());
    fill_summaries();
  }
  qoff[nq] = total;
  if (rc.emit && total) {
    if (srv->out.n < total) TRY(ensure(ctx, srv->out, total + total / 2));
    if (srv->pin_n < total) {
      if (srv->pin) cudaFreeHost(srv->pin);
      srv->pin = nullptr;
      srv->pin_n = 0;
      CU(cudaHostAlloc(&srv->pin, total + total / 4, cudaHostAllocDefault));
      srv->pin_n = total + total / 4;
    }
    RA.out = (char *)srv->out.p;
    qwrite_kernel<<<g2, 256, 0, st>>>(RA);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(E[5], st));
    CU(cudaMemcpyAsync(srv->pin, srv->out.p, total, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(&counters[3], (unsigned long long *)srv->counters.p + 3, sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, st));
    CU(cudaEventRecord(E[6], st));
    CU(cudaStreamSynchronize(st));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, E[4], E[5]));
    ctx->timings[4] = ms;
    CU(cudaEventElapsedTime(&ms, E[5], E[6]));
    ctx->timings[5] = ms;
    CU(cudaEventElapsedTime(&ms, E[0], E[6]));
    ctx->timings[6] = ms;
  } else {
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, E[0], E[4]));
    ctx->timings[6] = ms;
  }
  {
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, E[0], E[1]));
    ctx->timings[0] = ms;
    CU(cudaEventElapsedTime(&ms, E[1], E[2]));
    ctx->timings[1] = ms;
    CU(cudaEventElapsedTime(&ms, E[2], E[3]));
    ctx->timings[2] = ms;
    CU(cudaEventElapsedTime(&ms, E[3], E[4]));
    ctx->timings[3] = ms;
  }
  if (counters[3]) {
    ctx->err = "internal error: a query's text did not match its counted length";
    return TN93G_ECUDA;
  }
  for (int q = 0; q < nq; q++) {
    tn93g_summary &X = sums[q];
    X = S[q];
    if (repass) memset(X.amb_bounds, 0, sizeof X.amb_bounds);
    X.output_bytes = qoff[q + 1] - qoff[q];
    if (q == 0) {
      X.pairs_replayed = (long)counters[2];
      X.logs_ambiguous = ambiguous0;
      X.logs_resolved = resolved;
      X.undecided = 0;  // every listed pair was finished with the C library's logarithms
      X.sums_repass = repass ? 1 : 0;
    }
    if (rc.emit && sink && sink(user, q, (const char *)srv->pin + qoff[q], (size_t)(qoff[q + 1] - qoff[q])))
      return TN93G_ESINK;
  }
  return TN93G_OK;
}

}  // extern "C"

//================================================================================================== batched runs
// Many independent alignments in one pass (each with its own options): every stage runs over all of them at once.
// Packing is per alignment on one stream; the pair stage is one persistent launch per kernel class over a queue of
// all alignments' tiles (longest alignments first); the replay, statistics, sums, scan, reduction and text are
// batched kernels over all alignments' rows. Each alignment's output equals its own tn93g_run byte for byte.
namespace {

enum BatchBuf {
  BB_CODES, BB_SEEN, BB_NN, BB_VARCOL, BB_PLANES, BB_CC, BB_CCT, BB_EVCOUNT, BB_EVOFF, BB_EV, BB_AGG, BB_SITE,
  BB_NAMES, BB_NAMEOFF, BB_NAMELEN, BB_COUNTS, BB_DIST, BB_RQ, BB_RQN, BB_COUNTERS, BB_PDESC, BB_RDESC, BB_ROWDESC,
  BB_TILES, BB_NEXT, BB_BLOCKS, BB_SBYTES, BB_SOFF, BB_SLINKS, BB_SSKIP, BB_SMAX, BB_RSUM, BB_RW, BB_HIST, BB_TOTAL,
  BB_SCANTMP, BB_RED, BB_REDC, BB_FIRST, BB_FIRSTIDX, BB_OUT, BB_OH, BB_TCAGG, BB_TCDESC, BB_TCTILES, BB_TCERR,
  BB_UND, BB_UNDN, BB_AMB, BB_SCANDESC, BB_PACKDESC, BB_TRDESC, BB_OHDESC, BB_BOFF, BB_COUNT
};
static_assert(BB_COUNT <= kBatchBufs, "batch buffer table");

// Packing of a batch, one launch per step over all alignments: block b belongs to the alignment k with
// off[k] <= b < off[k + 1] (off[] is the prefix sum of the alignments' block counts) and is its block b - off[k].
__device__ __forceinline__ int batch_owner(const int *off, int K, int b)
{
  int lo = 0, hi = K - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

struct ScanDesc {
  const uint8_t *codes;
  long N, L;
  uint32_t *seen;
  unsigned long long *nN;
};
struct TransDesc {
  const uint8_t *cc;
  uint8_t *ccT;
  long N, Lc, Npad;
};
struct OneHotDesc {
  const uint8_t *cc;
  long N, Lc, NB, KS;
  uint8_t *img;
};

__global__ void __launch_bounds__(256) colscan_batch_kernel(const ScanDesc *d, const int *off, int K)
{
  const int k = batch_owner(off, K, blockIdx.x);
  const long lb = (long)blockIdx.x - off[k];
  const ScanDesc &a = d[k];
  const long gx = (a.L + 255) / 256;
  colscan_body(a.codes, a.N, a.L, a.seen, a.nN, lb % gx, lb / gx);
}

// one block per (8 sequences, one 64-column word)
__global__ void __launch_bounds__(256) pack_batch_kernel(const PackArgs *d, const int *off, int K)
{
  const int k = batch_owner(off, K, blockIdx.x);
  const long lb = (long)blockIdx.x - off[k];
  const PackArgs &a = d[k];
  const long gx = (a.N + kWarps - 1) / kWarps;
  pack_body(a, lb % gx, lb / gx, a.W);
}

__global__ void __launch_bounds__(256) events_batch_kernel(const PackArgs *d, const int *off, int K)
{
  const int k = batch_owner(off, K, blockIdx.x);
  events_body(d[k], (long)blockIdx.x - off[k]);
}

__global__ void __launch_bounds__(256) transpose_batch_kernel(const TransDesc *d, const int *off, int K)
{
  const int k = batch_owner(off, K, blockIdx.x);
  const long lb = (long)blockIdx.x - off[k];
  const TransDesc &a = d[k];
  const long gx = (a.Lc + 31) / 32;
  transpose_body(a.cc, a.ccT, a.N, a.Lc, a.Npad, lb % gx, lb / gx);
}

__global__ void __launch_bounds__(256) onehot_batch_kernel(const OneHotDesc *d, const int *off, int K)
{
  const int k = batch_owner(off, K, blockIdx.x);
  const OneHotDesc &a = d[k];
  onehot_body(a.cc, a.N, a.Lc, a.NB, a.KS, a.img, 0, a.NB * 32, (long)blockIdx.x - off[k]);
}

// the prefix sum of per-alignment block counts, uploaded to slot q of the offsets buffer; returns the total
int upload_offsets(tn93g_ctx *ctx, DevBuf &buf, int q, int K, const std::vector<long> &blocks, cudaStream_t st,
                   int *total)
{
  std::vector<int> off(K + 1);
  long t = 0;
  for (int k = 0; k < K; k++) {
    off[k] = (int)t;
    t += blocks[k];
  }
  off[K] = (int)t;
  if (t >= (1l << 31)) return TN93G_ETOOBIG;
  CU(cudaMemcpyAsync((int *)buf.p + (size_t)q * (K + 1), off.data(), (K + 1) * sizeof(int), cudaMemcpyHostToDevice,
                     st));
  *total = (int)t;
  return TN93G_OK;
}

__global__ void gather_u64_kernel(const unsigned long long *src, const long *idx, unsigned long long *dst, int n)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[k] = src[idx[k]];
}

template <int MINB>
cudaError_t launch_pair_batch_t(int sms, bool wplane, bool gapmm, const PairArgs *descs, const BatchTile *tiles,
                                int ntiles, unsigned *next, cudaStream_t st)
{
  static PerDevice attr;
  const cudaError_t e = attr.once([] {
    cudaError_t r;
    if ((r = cudaFuncSetAttribute(pair_batch_kernel<true, true, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kPairSmem)) != cudaSuccess)
      return r;
    if ((r = cudaFuncSetAttribute(pair_batch_kernel<true, false, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kPairSmem)) != cudaSuccess)
      return r;
    return cudaFuncSetAttribute(pair_batch_kernel<false, false, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kPairSmem);
  });
  if (e != cudaSuccess) return e;
  const dim3 g((unsigned)(sms * MINB));
  if (gapmm)
    pair_batch_kernel<true, true, MINB><<<g, 256, kPairSmem, st>>>(descs, tiles, ntiles, next);
  else if (wplane)
    pair_batch_kernel<true, false, MINB><<<g, 256, kPairSmem, st>>>(descs, tiles, ntiles, next);
  else
    pair_batch_kernel<false, false, MINB><<<g, 256, kPairSmem, st>>>(descs, tiles, ntiles, next);
  return cudaGetLastError();
}

}  // namespace

extern "C" int tn93g_batch_run(tn93g_ctx *ctx, int K, const tn93g_alignment *alns, const tn93g_opts *opts,
                               const int *rows_per_warp, int pair_blocks, tn93g_query_sink sink, void *user,
                               tn93g_summary *sums)
{
  if (!ctx || K <= 0 || !alns || !opts || !sums) return TN93G_EINVAL;
  for (int k = 0; k < K; k++) {
    const tn93g_alignment &A = alns[k];
    const tn93g_opts &o = opts[k];
    if (A.n <= 0 || A.L <= 0 || !A.codes || !A.copy_counts || !A.names || !A.name_off || !A.name_len)
      return TN93G_EINVAL;
    if (o.mode < 0 || o.mode > 4 || (o.format != TN93G_CSV && o.format != TN93G_CSVN) || o.do_fst) return TN93G_EINVAL;
    if (A.L >= (1l << 25) || A.n >= (1l << 31)) return TN93G_ETOOBIG;
    if (rows_per_warp && rows_per_warp[k] != 1 && rows_per_warp[k] != 2 && rows_per_warp[k] != 4) return TN93G_EINVAL;
  }
  if (pair_blocks == 0) pair_blocks = 2;
  if (pair_blocks != 2 && pair_blocks != 3) return TN93G_EINVAL;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  for (double &t : ctx->timings) t = 0;
  ctx->launches = 0;
  DevBuf *bb = ctx->bb;
  cudaEvent_t *E = ctx->evs;
  float ms = 0.f;
  CU(cudaEventRecord(E[0], st));
  //------------------------------------------------------------------ inputs
  std::vector<size_t> code_off(K + 1), seen_off(K + 1), name_base(K + 1), row_base(K + 1);
  code_off[0] = seen_off[0] = name_base[0] = row_base[0] = 0;
  for (int k = 0; k < K; k++) {
    size_t nb = 0;
    for (long i = 0; i < alns[k].n; i++) nb = std::max(nb, alns[k].name_off[i] + (size_t)alns[k].name_len[i]);
    code_off[k + 1] = code_off[k] + (size_t)alns[k].n * alns[k].L;
    seen_off[k + 1] = seen_off[k] + alns[k].L;
    name_base[k + 1] = name_base[k] + nb;
    row_base[k + 1] = row_base[k] + alns[k].n;
  }
  const size_t NR = row_base[K];
  TRY(ensure(ctx, bb[BB_CODES], code_off[K]));
  TRY(ensure(ctx, bb[BB_NAMES], name_base[K] + 1));
  TRY(ensure(ctx, bb[BB_NAMEOFF], NR * sizeof(uint64_t)));
  TRY(ensure(ctx, bb[BB_NAMELEN], NR * sizeof(int32_t)));
  TRY(ensure(ctx, bb[BB_COUNTS], NR * sizeof(long)));
  std::vector<uint64_t> noff(NR);
  std::vector<int32_t> nlen(NR);
  std::vector<long> cnts(NR);
  for (int k = 0; k < K; k++) {
    CU(cudaMemcpyAsync((uint8_t *)bb[BB_CODES].p + code_off[k], alns[k].codes, code_off[k + 1] - code_off[k],
                       cudaMemcpyHostToDevice, st));
    if (name_base[k + 1] > name_base[k])
      CU(cudaMemcpyAsync((char *)bb[BB_NAMES].p + name_base[k], alns[k].names, name_base[k + 1] - name_base[k],
                         cudaMemcpyHostToDevice, st));
    for (long i = 0; i < alns[k].n; i++) {
      noff[row_base[k] + i] = name_base[k] + alns[k].name_off[i];
      nlen[row_base[k] + i] = (int32_t)alns[k].name_len[i];
      cnts[row_base[k] + i] = alns[k].copy_counts[i];
    }
  }
  CU(cudaMemcpyAsync(bb[BB_NAMEOFF].p, noff.data(), NR * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(bb[BB_NAMELEN].p, nlen.data(), NR * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(bb[BB_COUNTS].p, cnts.data(), NR * sizeof(long), cudaMemcpyHostToDevice, st));
  //------------------------------------------------------------------ column scan and folding
  TRY(ensure(ctx, bb[BB_SEEN], seen_off[K] * sizeof(uint32_t)));
  TRY(ensure(ctx, bb[BB_NN], K * sizeof(unsigned long long)));
  CU(cudaMemsetAsync(bb[BB_SEEN].p, 0, seen_off[K] * sizeof(uint32_t), st));
  CU(cudaMemsetAsync(bb[BB_NN].p, 0, K * sizeof(unsigned long long), st));
  TRY(ensure(ctx, bb[BB_BOFF], 5 * (size_t)(K + 1) * sizeof(int)));
  TRY(ensure(ctx, bb[BB_SCANDESC], K * sizeof(ScanDesc)));
  TRY(ensure(ctx, bb[BB_PACKDESC], K * sizeof(PackArgs)));
  TRY(ensure(ctx, bb[BB_TRDESC], K * sizeof(TransDesc)));
  TRY(ensure(ctx, bb[BB_OHDESC], K * sizeof(OneHotDesc)));
  const int *boff = (const int *)bb[BB_BOFF].p;
  {
    std::vector<ScanDesc> sd(K);
    std::vector<long> nb(K);
    for (int k = 0; k < K; k++) {
      const long N = alns[k].n, L = alns[k].L;
      sd[k] = ScanDesc{(const uint8_t *)bb[BB_CODES].p + code_off[k], N, L, (uint32_t *)bb[BB_SEEN].p + seen_off[k],
                       (unsigned long long *)bb[BB_NN].p + k};
      nb[k] = ((L + 255) / 256) * ((N + 63) / 64);
    }
    CU(cudaMemcpyAsync(bb[BB_SCANDESC].p, sd.data(), K * sizeof(ScanDesc), cudaMemcpyHostToDevice, st));
    int total = 0;
    TRY(upload_offsets(ctx, bb[BB_BOFF], 0, K, nb, st, &total));
    if (total) {
      colscan_batch_kernel<<<(unsigned)total, 256, 0, st>>>((const ScanDesc *)bb[BB_SCANDESC].p, boff, K);
      CU(cudaGetLastError());
      ctx->launches++;
    }
  }
  std::vector<uint32_t> seen(seen_off[K]);
  std::vector<unsigned long long> nN(K);
  CU(cudaMemcpyAsync(seen.data(), bb[BB_SEEN].p, seen_off[K] * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(nN.data(), bb[BB_NN].p, K * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  std::vector<RunConsts> RC(K);
  std::vector<int32_t> varcol;
  std::vector<size_t> vc_off(K + 1), pl_off(K + 1), cc_off(K + 1), cct_off(K + 1), evo_off(K + 1);
  vc_off[0] = pl_off[0] = cc_off[0] = cct_off[0] = evo_off[0] = 0;
  for (int k = 0; k < K; k++) {
    const long N = alns[k].n, L = alns[k].L;
    const tn93g_opts *o = &opts[k];
    RunConsts &rc = RC[k];
    memset(&rc, 0, sizeof rc);
    rc.N = N;
    rc.n1 = N;
    rc.mode = o->mode;
    rc.gapmm = o->mode == TN93G_GAPMM;
    rc.fallback_avg = (o->mode == TN93G_RESOLVE || o->mode == TN93G_SUBSET) && o->resolve_fraction < 1.;
    rc.emit = !o->count_only;
    rc.format = o->format;
    rc.delim = o->delimiter;
    rc.report_self = o->report_self && rc.emit;
    rc.threshold = o->threshold;
    rc.min_distance = o->min_distance;
    rc.resolve_fraction = o->resolve_fraction;
    rc.min_overlap = o->min_overlap;
    rc.log_band = ctx->log_band;
    rc.log_spread = ctx->log_spread;
    rc.resolve_all = ctx->exact_sums;
    for (long p = 0; p < L; p++) {
      const uint32_t m = seen[seen_off[k] + p];
      if (m && !(m & (m - 1)) && m < 16) {
        const int b = __builtin_ctz(m);
        rc.constT++;
        rc.constNf[b] += 2;
        rc.constCnt[b]++;
      } else
        varcol.push_back((int32_t)p);
    }
    vc_off[k + 1] = varcol.size();
    rc.Lc = (long)(vc_off[k + 1] - vc_off[k]);
    rc.W = (rc.Lc + 63) / 64;
    rc.Npad = (N + 31) / 32 * 32;
    rc.wplane = rc.gapmm || nN[k] > 16ull * (unsigned long long)N;
    rc.NP = rc.gapmm ? 5 : 4;
    pl_off[k + 1] = pl_off[k] + (size_t)std::max<long>(rc.W, 1) * rc.NP * rc.Npad;
    cc_off[k + 1] = cc_off[k] + (size_t)N * std::max<long>(rc.Lc, 1);
    cct_off[k + 1] = cct_off[k] + (size_t)std::max<long>(rc.Lc, 1) * rc.Npad;
    evo_off[k + 1] = evo_off[k] + N + 1;
  }
  TRY(ensure(ctx, bb[BB_VARCOL], std::max<size_t>(varcol.size(), 1) * sizeof(int32_t)));
  TRY(ensure(ctx, bb[BB_PLANES], pl_off[K] * sizeof(uint64_t)));
  TRY(ensure(ctx, bb[BB_CC], cc_off[K]));
  TRY(ensure(ctx, bb[BB_CCT], cct_off[K]));
  TRY(ensure(ctx, bb[BB_EVCOUNT], NR * sizeof(uint32_t)));
  TRY(ensure(ctx, bb[BB_EVOFF], evo_off[K] * sizeof(uint32_t)));
  if (!varcol.empty())
    CU(cudaMemcpyAsync(bb[BB_VARCOL].p, varcol.data(), varcol.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  CU(cudaMemsetAsync(bb[BB_PLANES].p, 0, pl_off[K] * sizeof(uint64_t), st));
  CU(cudaMemsetAsync(bb[BB_EVCOUNT].p, 0, NR * sizeof(uint32_t), st));
  std::vector<PackArgs> PA(K);
  for (int k = 0; k < K; k++) {
    const RunConsts &rc = RC[k];
    PackArgs &pa = PA[k];
    pa.codes = (const uint8_t *)bb[BB_CODES].p + code_off[k];
    pa.N = rc.N;
    pa.L = alns[k].L;
    pa.Lc = rc.Lc;
    pa.W = rc.W;
    pa.Npad = rc.Npad;
    pa.varcol = (const int32_t *)bb[BB_VARCOL].p + vc_off[k];
    pa.NP = rc.NP;
    pa.wplane = rc.wplane;
    pa.gapmm = rc.gapmm;
    pa.planes = (uint64_t *)bb[BB_PLANES].p + pl_off[k];
    pa.cc = (uint8_t *)bb[BB_CC].p + cc_off[k];
    pa.evcount = (uint32_t *)bb[BB_EVCOUNT].p + row_base[k];
    pa.ev_off = (const uint32_t *)bb[BB_EVOFF].p + evo_off[k];
    pa.ev = nullptr;
  }
  {
    // bit planes and codes (one block per 8 sequences and word), and the transposed codes, of every alignment
    std::vector<long> nbp(K), nbt(K);
    std::vector<TransDesc> td(K);
    for (int k = 0; k < K; k++) {
      const RunConsts &rc = RC[k];
      nbp[k] = rc.W ? ((rc.N + kWarps - 1) / kWarps) * rc.W : 0;
      nbt[k] = rc.W ? ((rc.Lc + 31) / 32) * (rc.Npad / 32) : 0;
      td[k] = TransDesc{PA[k].cc, (uint8_t *)bb[BB_CCT].p + cct_off[k], rc.N, rc.Lc, rc.Npad};
    }
    CU(cudaMemcpyAsync(bb[BB_PACKDESC].p, PA.data(), K * sizeof(PackArgs), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(bb[BB_TRDESC].p, td.data(), K * sizeof(TransDesc), cudaMemcpyHostToDevice, st));
    int tp = 0, tt = 0;
    TRY(upload_offsets(ctx, bb[BB_BOFF], 1, K, nbp, st, &tp));
    TRY(upload_offsets(ctx, bb[BB_BOFF], 2, K, nbt, st, &tt));
    if (tp) {
      pack_batch_kernel<<<(unsigned)tp, 256, 0, st>>>((const PackArgs *)bb[BB_PACKDESC].p, boff + (K + 1), K);
      CU(cudaGetLastError());
      ctx->launches++;
    }
    if (tt) {
      transpose_batch_kernel<<<(unsigned)tt, dim3(32, 8), 0, st>>>((const TransDesc *)bb[BB_TRDESC].p,
                                                                  boff + 2 * (K + 1), K);
      CU(cudaGetLastError());
      ctx->launches++;
    }
  }
  std::vector<uint32_t> evc(NR), evo(evo_off[K]);
  CU(cudaMemcpyAsync(evc.data(), bb[BB_EVCOUNT].p, NR * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  size_t nev = 0;
  for (int k = 0; k < K; k++) {
    uint32_t max_ev = 0;
    for (long i = 0; i < alns[k].n; i++) {
      evo[evo_off[k] + i] = (uint32_t)nev;
      nev += evc[row_base[k] + i];
      max_ev = std::max(max_ev, evc[row_base[k] + i]);
    }
    evo[evo_off[k] + alns[k].n] = (uint32_t)nev;
    RC[k].packed = max_ev <= (uint32_t)kPackedMaxEvents;
  }
  if (nev >= (1ull << 32)) return TN93G_ETOOBIG;
  TRY(ensure(ctx, bb[BB_EV], std::max<size_t>(nev, 1) * sizeof(uint32_t)));
  CU(cudaMemcpyAsync(bb[BB_EVOFF].p, evo.data(), evo_off[K] * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  {
    // every alignment's sparse events (one block per 8 sequences)
    std::vector<long> nbe(K);
    for (int k = 0; k < K; k++) {
      PA[k].ev = (uint32_t *)bb[BB_EV].p;
      nbe[k] = (RC[k].W && evo[evo_off[k] + alns[k].n] > evo[evo_off[k]]) ? (RC[k].N + kWarps - 1) / kWarps : 0;
    }
    CU(cudaMemcpyAsync(bb[BB_PACKDESC].p, PA.data(), K * sizeof(PackArgs), cudaMemcpyHostToDevice, st));
    int te = 0;
    TRY(upload_offsets(ctx, bb[BB_BOFF], 3, K, nbe, st, &te));
    if (te) {
      events_batch_kernel<<<(unsigned)te, 256, 0, st>>>((const PackArgs *)bb[BB_PACKDESC].p, boff + 3 * (K + 1), K);
      CU(cudaGetLastError());
      ctx->launches++;
    }
  }
  // tables: one copy per distinct (mode, ambiguity subset, N plane); the site tables per (mode, subset)
  std::vector<int> tab_of(K), site_of(K);
  std::vector<std::pair<int, std::string>> keys, site_keys;
  std::vector<PairTables> h_agg;
  std::vector<SiteEntry> h_site;
  for (int k = 0; k < K; k++) {
    const std::string sub((const char *)opts[k].subset, sizeof opts[k].subset);
    const std::string sk = opts[k].mode == TN93G_SUBSET ? sub : std::string();
    const std::pair<int, std::string> key(opts[k].mode * 2 + (RC[k].wplane ? 1 : 0), sk), skey(opts[k].mode, sk);
    int t = -1, u = -1;
    for (size_t q = 0; q < keys.size(); q++)
      if (keys[q] == key) t = (int)q;
    for (size_t q = 0; q < site_keys.size(); q++)
      if (site_keys[q] == skey) u = (int)q;
    if (t < 0 || u < 0) build_tables(ctx->h_tab, opts[k].mode, opts[k].subset);
    if (t < 0) {
      h_agg.emplace_back();
      fill_pair_tables(*ctx->h_tab, RC[k].wplane, &h_agg.back());
      t = (int)keys.size();
      keys.push_back(key);
    }
    if (u < 0) {
      const SiteEntry *se = &ctx->h_tab->site[0][0];
      h_site.insert(h_site.end(), se, se + sizeof(ctx->h_tab->site) / sizeof(SiteEntry));
      u = (int)site_keys.size();
      site_keys.push_back(skey);
    }
    tab_of[k] = t;
    site_of[k] = u;
  }
  const size_t site_n = sizeof(ctx->h_tab->site) / sizeof(SiteEntry);
  TRY(ensure(ctx, bb[BB_AGG], h_agg.size() * sizeof(PairTables)));
  TRY(ensure(ctx, bb[BB_SITE], h_site.size() * sizeof(SiteEntry)));
  CU(cudaMemcpyAsync(bb[BB_AGG].p, h_agg.data(), h_agg.size() * sizeof(PairTables), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(bb[BB_SITE].p, h_site.data(), h_site.size() * sizeof(SiteEntry), cudaMemcpyHostToDevice, st));
  CU(cudaEventRecord(E[1], st));
  //------------------------------------------------------------------ pair stage
  std::vector<size_t> d_off(K + 1), q_off(K + 1), seg_base(K + 1);
  d_off[0] = q_off[0] = seg_base[0] = 0;
  std::vector<long> maxseg(K);
  for (int k = 0; k < K; k++) {
    const size_t N = alns[k].n;
    d_off[k + 1] = d_off[k] + N * N;
    q_off[k + 1] = q_off[k] + std::max<size_t>(N * (N - 1) / 2, 1);
    maxseg[k] = std::max<long>(1, ((long)N + kSeg - 1) / kSeg);
    seg_base[k + 1] = seg_base[k] + N * maxseg[k];
  }
  TRY(ensure(ctx, bb[BB_DIST], d_off[K] * sizeof(double)));
  TRY(ensure(ctx, bb[BB_RQ], q_off[K] * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_RQN], K * sizeof(unsigned)));
  TRY(ensure(ctx, bb[BB_COUNTERS], (size_t)K * 4 * sizeof(unsigned long long)));
  CU(cudaMemsetAsync(bb[BB_RQN].p, 0, K * sizeof(unsigned), st));
  CU(cudaMemsetAsync(bb[BB_COUNTERS].p, 0, (size_t)K * 4 * sizeof(unsigned long long), st));
  // one undecided list for every alignment (entries carry the alignment), per-alignment summary bounds
  const unsigned und_cap = (unsigned)std::min<size_t>(std::max<size_t>(4096, q_off[K] / 64), 0xFFFFFFF0u);
  TRY(ensure(ctx, bb[BB_UND], (size_t)und_cap * 2 * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_UNDN], sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_AMB], (size_t)K * 4 * sizeof(unsigned long long)));
  CU(cudaMemsetAsync(bb[BB_UNDN].p, 0, sizeof(unsigned long long), st));
  CU(cudaMemsetAsync(bb[BB_AMB].p, 0, (size_t)K * 4 * sizeof(unsigned long long), st));
  std::vector<PairArgs> PD(K);
  std::vector<ReplayArgs> RD(K);
  for (int k = 0; k < K; k++) {
    PairArgs &A = PD[k];
    memset(&A, 0, sizeof A);
    A.rc = RC[k];
    A.planes = (const uint64_t *)bb[BB_PLANES].p + pl_off[k];
    A.cc = (const uint8_t *)bb[BB_CC].p + cc_off[k];
    A.ccT = (const uint8_t *)bb[BB_CCT].p + cct_off[k];
    A.ev_off = (const uint32_t *)bb[BB_EVOFF].p + evo_off[k];
    A.ev = (const uint32_t *)bb[BB_EV].p;
    A.tab = (const PairTables *)bb[BB_AGG].p + tab_of[k];
    A.r0 = 0;
    A.r1 = alns[k].n;
    A.ncols = alns[k].n;
    A.colbase = 0;
    A.cstart = 0;
    A.dist = (double *)bb[BB_DIST].p + d_off[k];
    A.replay_q = (unsigned long long *)bb[BB_RQ].p + q_off[k];
    A.replay_n = (unsigned *)bb[BB_RQN].p + k;
    A.replay_cap = q_off[k + 1] - q_off[k];
    A.counters = (unsigned long long *)bb[BB_COUNTERS].p + 4 * k;
    A.logt = ctx->d_logt;
    A.ex.und_list = (unsigned long long *)bb[BB_UND].p;
    A.ex.und_n = (unsigned *)bb[BB_UNDN].p;
    A.ex.und_cap = und_cap;
    A.ex.und_k = k;
    A.ex.amb = (unsigned long long *)bb[BB_AMB].p + 4 * k;
    A.ex.counts = (const long *)bb[BB_COUNTS].p + row_base[k];
    A.ex.colunit = nullptr;
    ReplayArgs &R = RD[k];
    memset(&R, 0, sizeof R);
    R.rc = RC[k];
    R.cc = A.cc;
    R.planes = A.planes;
    R.site = (const SiteEntry *)bb[BB_SITE].p + (size_t)site_of[k] * site_n;
    R.q = A.replay_q;
    R.qn = A.replay_n;
    R.qcap = A.replay_cap;
    R.r0 = 0;
    R.ncols = A.ncols;
    R.colbase = 0;
    R.dist = A.dist;
    R.counters = A.counters;
    R.logt = ctx->d_logt;
    R.ex = A.ex;
  }
  std::vector<int> order(K);
  for (int k = 0; k < K; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return RC[a].Lc > RC[b].Lc; });
  // tensor-core count path: per alignment a one-hot operand image and its clean-site aggregates ([7][n][n]),
  // computed by one launch over every alignment's 32 x 64 tiles
  const bool use_tc = ctx->count_path == 1;
  if (use_tc) {
    std::vector<size_t> oh_off(K + 1, 0), ag_off(K + 1, 0);
    std::vector<TcArgs> TD(K);
    std::vector<int4> tct;
    for (int k = 0; k < K; k++) {
      const long N = alns[k].n;
      const bool on = RC[k].W > 0 && N > 1;
      const long NB = (N + 31) / 32 + 1, KS = (RC[k].Lc + kTcStageK - 1) / kTcStageK;
      oh_off[k + 1] = oh_off[k] + (on ? (size_t)KS * NB * kTcBlockBytes : 0);
      // byte offsets, each alignment's block 16-byte aligned
      const size_t rec = 2 * RC[k].Lc < 65536 ? 16 : 32;  // bytes of a pair's record
      ag_off[k + 1] = ag_off[k] + (on ? (size_t)N * N * rec : 0);
      TcArgs &T = TD[k];
      memset(&T, 0, sizeof T);
      T.NB = NB;
      T.KS = KS;
      T.N = N;
      T.n1 = N;
      T.cross = false;
      T.r0 = 0;
      T.r1 = N;
      T.ncols = N;
      T.colbase = 0;
      T.cstart = 0;
      T.cend = N;
    }
    TRY(ensure(ctx, bb[BB_OH], std::max<size_t>(oh_off[K], 16)));
    TRY(ensure(ctx, bb[BB_TCAGG], std::max<size_t>(ag_off[K], 16)));
    TRY(ensure(ctx, bb[BB_TCERR], sizeof(unsigned long long)));
    CU(cudaMemsetAsync(bb[BB_TCERR].p, 0, sizeof(unsigned long long), st));
    std::vector<OneHotDesc> ohd(K);
    std::vector<long> nbo(K, 0);
    for (int k : order) {
      if (oh_off[k + 1] == oh_off[k]) continue;
      TcArgs &T = TD[k];
      T.onehot = (const uint8_t *)bb[BB_OH].p + oh_off[k];
      T.agg = (char *)bb[BB_TCAGG].p + ag_off[k];
      T.agg16 = 2 * RC[k].Lc < 65536;
      T.err = (unsigned long long *)bb[BB_TCERR].p;
      T.wait_ns = ctx->wait_ns;
      T.skip_fill_block = -1;
      ohd[k] = OneHotDesc{PA[k].cc, T.N, RC[k].Lc, T.NB, T.KS, (uint8_t *)bb[BB_OH].p + oh_off[k]};
      nbo[k] = (T.NB * 32 * T.KS * (kTcStageK / 16) + 255) / 256;
      for (long i0 = 0; i0 < T.N - 1; i0 += kTcRows)
        for (long j0 = (i0 + 1) / kTcCols * kTcCols; j0 < T.N; j0 += kTcCols) tct.push_back(make_int4(k, (int)i0, (int)j0, 0));
      PD[k].tcagg = T.agg;
      PD[k].tc16 = T.agg16;
    }
    {
      // every alignment's one-hot operand image in one launch
      int to = 0;
      TRY(upload_offsets(ctx, bb[BB_BOFF], 4, K, nbo, st, &to));
      CU(cudaMemcpyAsync(bb[BB_OHDESC].p, ohd.data(), K * sizeof(OneHotDesc), cudaMemcpyHostToDevice, st));
      if (to) {
        onehot_batch_kernel<<<(unsigned)to, 256, 0, st>>>((const OneHotDesc *)bb[BB_OHDESC].p, boff + 4 * (K + 1), K);
        CU(cudaGetLastError());
        ctx->launches++;
      }
    }
    if (!tct.empty()) {
      TRY(ensure(ctx, bb[BB_TCDESC], K * sizeof(TcArgs)));
      TRY(ensure(ctx, bb[BB_TCTILES], tct.size() * sizeof(int4)));
      CU(cudaMemcpyAsync(bb[BB_TCDESC].p, TD.data(), K * sizeof(TcArgs), cudaMemcpyHostToDevice, st));
      CU(cudaMemcpyAsync(bb[BB_TCTILES].p, tct.data(), tct.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
      TcArgs G;
      memset(&G, 0, sizeof G);
      G.err = (unsigned long long *)bb[BB_TCERR].p;
      G.wait_ns = ctx->wait_ns;
      G.skip_fill_block = -1;
      CU(launch_count_list(G, (const TcArgs *)bb[BB_TCDESC].p, (const int4 *)bb[BB_TCTILES].p, (int)tct.size(),
                           ctx->sms, st));
      ctx->launches++;
    }
  }
  // the tile queue: per kernel class, longest alignments first
  std::vector<BatchTile> tiles;
  int cls_n[3] = {0, 0, 0};
  for (int cls = 0; cls < 3; cls++)
    for (int k : order) {
      const int kc = RC[k].gapmm ? 2 : RC[k].wplane ? 1 : 0;
      if (kc != cls || !RC[k].W) continue;
      const int rpw = rows_per_warp ? rows_per_warp[k] : kRowsPerWarp, trows = kWarps * rpw;
      const long N = alns[k].n;
      for (long i0 = 0; i0 < N - 1; i0 += trows)
        for (long j0 = (i0 + 1) / kTile * kTile; j0 < N; j0 += kTile) {
          tiles.push_back(BatchTile{k, rpw, (int)i0, (int)j0});
          cls_n[cls]++;
        }
    }
  // alignments whose columns are all constant (Lc = 0) have no tiles: the epilogue runs on the constants alone
  // in tn93g_run; here they take the single-alignment kernel
  TRY(ensure(ctx, bb[BB_PDESC], K * sizeof(PairArgs)));
  TRY(ensure(ctx, bb[BB_RDESC], K * sizeof(ReplayArgs)));
  TRY(ensure(ctx, bb[BB_TILES], std::max<size_t>(tiles.size(), 1) * sizeof(BatchTile)));
  TRY(ensure(ctx, bb[BB_NEXT], 3 * sizeof(unsigned)));
  CU(cudaMemcpyAsync(bb[BB_PDESC].p, PD.data(), K * sizeof(PairArgs), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(bb[BB_RDESC].p, RD.data(), K * sizeof(ReplayArgs), cudaMemcpyHostToDevice, st));
  if (!tiles.empty())
    CU(cudaMemcpyAsync(bb[BB_TILES].p, tiles.data(), tiles.size() * sizeof(BatchTile), cudaMemcpyHostToDevice, st));
  CU(cudaMemsetAsync(bb[BB_NEXT].p, 0, 3 * sizeof(unsigned), st));
  int tbase = 0;
  for (int cls = 0; cls < 3; cls++) {
    if (!cls_n[cls]) continue;
    const BatchTile *tp = (const BatchTile *)bb[BB_TILES].p + tbase;
    unsigned *nx = (unsigned *)bb[BB_NEXT].p + cls;
    const PairArgs *dp = (const PairArgs *)bb[BB_PDESC].p;
    CU(pair_blocks == 3 ? launch_pair_batch_t<3>(ctx->sms, cls >= 1, cls == 2, dp, tp, cls_n[cls], nx, st)
                        : launch_pair_batch_t<2>(ctx->sms, cls >= 1, cls == 2, dp, tp, cls_n[cls], nx, st));
    ctx->launches++;
    tbase += cls_n[cls];
  }
  for (int k = 0; k < K; k++)
    if (!RC[k].W && alns[k].n > 1) {
      CU(launch_pair(PD[k], (alns[k].n + kTile - 1) / kTile, alns[k].n, st));
      ctx->launches++;
    }
  CU(cudaEventRecord(E[2], st));
  replay_batch_kernel<<<2 * ctx->sms, 256, 0, st>>>((const ReplayArgs *)bb[BB_RDESC].p, K);
  CU(cudaGetLastError());
  ctx->launches++;
  CU(cudaEventRecord(E[3], st));
  //------------------------------------------------------------------ rows
  const size_t NS = seg_base[K];
  TRY(ensure(ctx, bb[BB_SBYTES], NS * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_SOFF], NS * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_SLINKS], NS * sizeof(long long)));
  TRY(ensure(ctx, bb[BB_SSKIP], NS * sizeof(long long)));
  TRY(ensure(ctx, bb[BB_SMAX], NS * 3 * sizeof(double)));
  TRY(ensure(ctx, bb[BB_RSUM], NR * 3 * sizeof(double)));
  TRY(ensure(ctx, bb[BB_RW], NR * 3 * sizeof(double)));
  TRY(ensure(ctx, bb[BB_HIST], (size_t)K * 3 * kHistBins * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_TOTAL], sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_SCANTMP], (2 * (NS / kScanTile + 1) + 1) * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_RED], (size_t)K * 3 * sizeof(double)));
  TRY(ensure(ctx, bb[BB_REDC], (size_t)K * 2 * sizeof(long long)));
  TRY(ensure(ctx, bb[BB_FIRST], (size_t)K * sizeof(unsigned long long)));
  TRY(ensure(ctx, bb[BB_FIRSTIDX], (size_t)K * sizeof(long)));
  TRY(ensure(ctx, bb[BB_ROWDESC], K * sizeof(RowArgs)));
  CU(cudaMemsetAsync(bb[BB_HIST].p, 0, (size_t)K * 3 * kHistBins * sizeof(unsigned long long), st));
  std::vector<RowArgs> RA(K);
  std::vector<int2> blocks;
  long segmax = 1;
  std::vector<long> first_idx(K);
  for (int k = 0; k < K; k++) {
    RowArgs &a = RA[k];
    memset(&a, 0, sizeof a);
    a.rc = RC[k];
    a.dist = PD[k].dist;
    a.r0 = 0;
    a.r1 = alns[k].n;
    a.ncols = alns[k].n;
    a.colbase = 0;
    a.counts = (const long *)bb[BB_COUNTS].p + row_base[k];
    a.name_len = (const int32_t *)bb[BB_NAMELEN].p + row_base[k];
    a.name_off = (const uint64_t *)bb[BB_NAMEOFF].p + row_base[k];
    a.names = (const char *)bb[BB_NAMES].p;
    a.maxseg = maxseg[k];
    a.seg_cols = nullptr;
    a.nrows = alns[k].n;
    a.seg_bytes = (unsigned long long *)bb[BB_SBYTES].p + seg_base[k];
    a.seg_links = (long long *)bb[BB_SLINKS].p + seg_base[k];
    a.seg_skip = (long long *)bb[BB_SSKIP].p + seg_base[k];
    a.seg_max = (double *)bb[BB_SMAX].p + 3 * seg_base[k];
    a.row_sum = (double *)bb[BB_RSUM].p + 3 * row_base[k];
    a.row_w = (double *)bb[BB_RW].p + 3 * row_base[k];
    a.hist = (unsigned long long *)bb[BB_HIST].p + (size_t)k * 3 * kHistBins;
    a.seg_off = (const unsigned long long *)bb[BB_SOFF].p + seg_base[k];
    a.out = nullptr;
    a.hy = nullptr;
    a.err = (unsigned long long *)bb[BB_COUNTERS].p + 4 * k + 3;
    segmax = std::max(segmax, maxseg[k]);
    for (long bx = 0; bx < (alns[k].n + kWarps - 1) / kWarps; bx++) blocks.push_back(make_int2(k, (int)bx));
    first_idx[k] = (long)seg_base[k];
  }
  TRY(ensure(ctx, bb[BB_BLOCKS], blocks.size() * sizeof(int2)));
  CU(cudaMemcpyAsync(bb[BB_ROWDESC].p, RA.data(), K * sizeof(RowArgs), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(bb[BB_BLOCKS].p, blocks.data(), blocks.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(bb[BB_FIRSTIDX].p, first_idx.data(), K * sizeof(long), cudaMemcpyHostToDevice, st));
  const RowArgs *rd = (const RowArgs *)bb[BB_ROWDESC].p;
  const int2 *bp = (const int2 *)bb[BB_BLOCKS].p;
  unsigned long long total = 0, und = 0;
  std::vector<double> red((size_t)K * 3);
  std::vector<long long> redc((size_t)K * 2);
  std::vector<unsigned long long> first(K + 1), hist((size_t)K * 3 * kHistBins), counters((size_t)K * 4);
  auto rows_and_read = [&]() -> int {
    CU(cudaMemsetAsync(bb[BB_HIST].p, 0, (size_t)K * 3 * kHistBins * sizeof(unsigned long long), st));
    stats_batch_kernel<<<dim3((unsigned)blocks.size(), (unsigned)segmax), 256, 0, st>>>(rd, bp);
    CU(cudaGetLastError());
    sum_batch_kernel<<<(unsigned)blocks.size(), 256, 0, st>>>(rd, bp);
    CU(cudaGetLastError());
    CU(launch_scan((const unsigned long long *)bb[BB_SBYTES].p, (unsigned long long *)bb[BB_SOFF].p, (long)NS,
                   (unsigned long long *)bb[BB_TOTAL].p, (unsigned long long *)bb[BB_SCANTMP].p, st));
    aln_reduce_kernel<<<K, 256, 0, st>>>(rd, (double *)bb[BB_RED].p, (long long *)bb[BB_REDC].p);
    CU(cudaGetLastError());
    gather_u64_kernel<<<(K + 255) / 256, 256, 0, st>>>((const unsigned long long *)bb[BB_SOFF].p,
                                                       (const long *)bb[BB_FIRSTIDX].p,
                                                       (unsigned long long *)bb[BB_FIRST].p, K);
    CU(cudaGetLastError());
    ctx->launches += 5;
    CU(cudaEventRecord(E[4], st));
    CU(cudaMemcpyAsync(&total, bb[BB_TOTAL].p, sizeof total, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(red.data(), bb[BB_RED].p, red.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(redc.data(), bb[BB_REDC].p, redc.size() * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(first.data(), bb[BB_FIRST].p, K * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(hist.data(), bb[BB_HIST].p, hist.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       st));
    CU(cudaMemcpyAsync(&und, bb[BB_UNDN].p, sizeof und, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return TN93G_OK;
  };
  TRY(rows_and_read());
  long resolved = 0;
  // more undecided pairs than the list holds: the alignments that listed any run again alone below
  const bool overflow = und > und_cap;
  if (und && !overflow) {
    // pairs whose bytes or decisions depend on the C library's rounding of a logarithm: finished with its
    // logarithms, then the row stage runs again
    TRY(resolve_listed(ctx, (const ReplayArgs *)bb[BB_RDESC].p, (const unsigned long long *)bb[BB_UND].p,
                       (unsigned)und, st));
    resolved = (long)und;
    TRY(rows_and_read());
  }
  first[K] = total;
  bool any_emit = false;
  for (int k = 0; k < K; k++) any_emit |= RC[k].emit;
  if (any_emit && total) {
    if (bb[BB_OUT].n < total) TRY(ensure(ctx, bb[BB_OUT], total + total / 4));
    TRY(ensure_pinned(ctx, total));
    for (int k = 0; k < K; k++) RA[k].out = (char *)bb[BB_OUT].p;
    CU(cudaMemcpyAsync(bb[BB_ROWDESC].p, RA.data(), K * sizeof(RowArgs), cudaMemcpyHostToDevice, st));
    write_batch_kernel<<<dim3((unsigned)blocks.size(), (unsigned)segmax), 256, 0, st>>>(rd, bp);
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaEventRecord(E[5], st));
    CU(cudaMemcpyAsync(ctx->pinned, bb[BB_OUT].p, total, cudaMemcpyDeviceToHost, st));
  } else {
    CU(cudaEventRecord(E[5], st));
  }
  CU(cudaMemcpyAsync(counters.data(), bb[BB_COUNTERS].p, counters.size() * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, st));
  CU(cudaEventRecord(E[6], st));
  CU(cudaStreamSynchronize(st));
  const int pairs_e[7][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {0, 6}};
  for (int q = 0; q < 7; q++) {
    CU(cudaEventElapsedTime(&ms, E[pairs_e[q][0]], E[pairs_e[q][1]]));
    ctx->timings[q] = ms;
  }
  if (use_tc) {
    unsigned long long tcerr = 0;
    CU(cudaMemcpy(&tcerr, bb[BB_TCERR].p, sizeof tcerr, cudaMemcpyDeviceToHost));
    if (tcerr) {
      ctx->err = "the tensor-core count kernel timed out waiting for its pipeline";
      return TN93G_ETIMEOUT;
    }
  }
  for (int k = 0; k < K; k++) {
    if (counters[4 * k + 3]) {
      ctx->err = "internal error: a row's text did not match its counted length";
      return TN93G_ECUDA;
    }
    tn93g_summary &S = sums[k];
    memset(&S, 0, sizeof S);
    const unsigned long N = (unsigned long)alns[k].n;
    S.pairwise = N * (N - 1) / 2;
    S.links = (long)redc[2 * k];
    S.skipped = (long)redc[2 * k + 1];
    S.max[0] = red[3 * k];
    S.mean[0] = red[3 * k + 1];
    S.weighted[0] = red[3 * k + 2];
    for (int q = 0; q < 3; q++)
      for (int b = 0; b < kHistBins; b++) S.hist[q][b] = hist[((size_t)k * 3 + q) * kHistBins + b];
    S.logs_ambiguous = (long)counters[4 * k];
    S.logs_resolved = (long)counters[4 * k + 1];  // every listed pair was finished (resolved = the list's total)
    S.undecided = 0;
    S.pairs_replayed = (long)counters[4 * k + 2];
    S.output_bytes = RC[k].emit ? first[k + 1] - first[k] : 0;
  }
  (void)resolved;
  // After an overflow of the undecided list, every alignment that listed a pair runs again alone through
  // tn93g_run's path (which grows its list as needed): its text and summary replace the batch's.
  std::vector<std::string> redo_text(K);
  std::vector<char> redone(K, 0);
  if (overflow) {
    for (int k = 0; k < K; k++) {
      if (!counters[4 * k + 1]) continue;
      const tn93g_alignment &A = alns[k];
      tn93g_set *set = nullptr;
      TRY(tn93g_upload(ctx, &set, A.codes, A.n, A.L, A.copy_counts, A.names, A.name_off, A.name_len));
      tn93g_summary S2;
      const int r = run_impl(ctx, set, A.n, &opts[k], append_sink, &redo_text[k], &S2, false);
      tn93g_free_set(ctx, set);
      TRY(r);
      sums[k] = S2;
      redone[k] = 1;
    }
  }
  // Per alignment: the JSON numbers certain for every rounding of the C library's log, or the alignment runs
  // again alone through tn93g_run's path, whose exact-sums pass gives its maximum and mean (its text and counts
  // are certified pair by pair already).
  {
    std::vector<unsigned long long> ambw((size_t)K * 4);
    CU(cudaMemcpy(ambw.data(), bb[BB_AMB].p, ambw.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (int k = 0; k < K; k++) {
      if (redone[k]) continue;
      tn93g_summary &S = sums[k];
      amb_bounds(&ambw[(size_t)k * 4], S.amb_bounds[0]);
      if (summary_certified(&S, S.amb_bounds, 2 * alns[k].n + 2, 0)) continue;
      const tn93g_alignment &A = alns[k];
      tn93g_set *set = nullptr;
      TRY(tn93g_upload(ctx, &set, A.codes, A.n, A.L, A.copy_counts, A.names, A.name_off, A.name_len));
      tn93g_opts o = opts[k];
      o.count_only = 1;
      tn93g_summary S2;
      const int r = run_impl(ctx, set, A.n, &o, nullptr, nullptr, &S2, false, 0, -1, nullptr, kRunResolveAll);
      tn93g_free_set(ctx, set);
      TRY(r);
      S.max[0] = S2.max[0];
      S.mean[0] = S2.mean[0];
      S.logs_resolved += S2.logs_resolved;
      S.sums_repass = 1;
      memset(S.amb_bounds, 0, sizeof S.amb_bounds);
    }
  }
  if (any_emit && sink)
    for (int k = 0; k < K; k++) {
      if (!RC[k].emit) continue;
      const int r = redone[k] ? sink(user, k, redo_text[k].data(), redo_text[k].size())
                              : sink(user, k, (const char *)ctx->pinned + first[k], (size_t)(first[k + 1] - first[k]));
      if (r) return TN93G_ESINK;
    }
  return TN93G_OK;
}
