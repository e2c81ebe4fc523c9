// kernels.cuh -- device-side data layout and kernel declarations of the all-pairs TN93 engine.
//
// HBM layout of one run (N sequences, Lc variable columns after folding the constant ones, W = ceil(Lc/64)
// plane words, Npad = N rounded up to 32):
//   planes  u64 [W][NP][Npad]  per 64-column word: hi, lo (base = hi + 2 lo, set only at clean sites),
//                              clean, W (N, or N-or-gap under gapmm) and, under gapmm, gap. Sequence-minor,
//                              so the 32 lanes of a warp load 32 sequences' words in one coalesced access.
//   cc      u8  [N][Lc]        compressed codes, row-major (site-order replay, column-side events)
//   ccT     u8  [Lc][Npad]     the same, position-major (row-side events look up 32 columns at once)
//   ev      u32 [ev_off[N]]    per sequence, its sparse events (k << 5 | code) in site order
//   dist    f64 [rows][ncols]  raw distance of every pair of a band of rows (skip marker for -l skips)
#pragma once
#include <stdint.h>

#include "tables.h"
#include "tn93_math.cuh"

namespace tn93 {

// raw-distance slot of a pair skipped by the -l test (a signalling-NaN pattern no arithmetic produces)
constexpr uint64_t kSkipBits = 0x7FF4000000000BADull;

struct PackArgs {
  const uint8_t *codes;  // [N][L]
  long N, L, Lc, W, Npad;
  const int32_t *varcol;  // [Lc]
  int NP;                 // planes per word (4, or 5 under gapmm)
  bool wplane, gapmm;
  uint64_t *planes;
  uint8_t *cc;
  uint32_t *evcount;  // [N]
  const uint32_t *ev_off;
  uint32_t *ev;
};

struct RunConsts {
  long N, n1, Lc, W, Npad;
  int NP;
  int mode;
  bool wplane, gapmm, cross, fst, fallback_avg, emit;
  int format;
  char delim;
  bool report_self;
  double threshold, min_distance, resolve_fraction;
  long min_overlap;
  long constT, constNf[4], constCnt[4];
  double log_band, log_spread;  // the logarithm's ambiguity band and candidate distance in ulps (tlog)
  bool resolve_all;             // every pair with an ambiguous logarithm goes to the undecided list
  bool packed;                  // no sequence has more than kPackedMaxEvents events: the packed event sums apply
};

// The pair stage's tables in device memory: the x16 event table with the N-plane entries after it (Tables::ev,
// ew[4], eww) and its packed form (PackedTables, built for the run's N-plane setting).
struct PairTables {
  AggEntry agg[kEvEntries + 5];
  PackedTables packed;
};

// Where the pair stage reports exactness problems:
//   * the undecided list: pairs whose printed bytes, histogram bin or link decision depend on which candidate the
//     C library's log returns; entries are two words, (und_k, (i << 32) | j); the host takes those logarithms from
//     the C library and the pairs are finished again on the device;
//   * amb: per summary unit (a histogram bin of the run, or a query of a server batch) four words over the pairs
//     with an ambiguous logarithm: [0] the largest low candidate and [1] the largest high candidate (non-negative
//     doubles as ordered bit patterns), [2] the sum of (high - low) x copy weight (a double), [3] unused. The host
//     uses them to certify the maximum and the mean the JSON summary prints.
struct ExactSink {
  unsigned long long *und_list;  // nullptr: not listed (the allocation-free entry point)
  unsigned *und_n;
  unsigned und_cap;
  int und_k;                     // first word of this run's entries (the alignment of a batch)
  unsigned long long *amb;       // nullptr: not tracked
  const long *counts;            // copy numbers (the weights of the mean)
  const int *colunit;            // per column (from colbase): its summary unit; nullptr: the histogram bin
};

struct PairArgs {
  RunConsts rc;
  const uint64_t *planes;
  const uint8_t *cc, *ccT;
  const uint32_t *ev_off, *ev;
  const PairTables *tab;
  long r0, r1;          // band rows
  long ncols, colbase;  // row stride of dist and the first global column it holds
  long cstart;          // first column of the launch grid (a multiple of 32 past colbase)
  double *dist;
  unsigned long long *replay_q;  // (t << 63) | (i << 31) | j
  unsigned int *replay_n;
  unsigned long long replay_cap;
  unsigned long long *counters;  // [0] pairs with an ambiguous log, [1] undecided pairs
  const LogTable *logt;
  ExactSink ex;
  void *tcagg = nullptr;  // clean-site aggregates from the tensor-core kernel: one record per pair slot of
                          // [band rows][ncols], 8 uint16 (16 bytes) or 8 int32 (32 bytes), 7 used; with split, the
                          // pair kernel writes the pair's final x16 aggregates back into it
  int tc16 = 0;           // the records are uint16 (every final aggregate fits: 32 L < 65536), else int32
  int split = 0;          // tensor-core path only: the pair kernel stops before the formula, which formula_kernel
                          // finishes from the records
  // The nonzero words of each sequence's N plane (N sites, or N and gap sites under gapmm): sequence s owns
  // wl[wl_off[s] .. wl_off[s + 1]). With the tensor-core counts and packed events, the pair kernel's N-plane
  // cross terms visit only these words; nullptr: every word.
  const uint32_t *wl_off = nullptr, *wl = nullptr;
  long tcncols = 0, tccolbase = 0;  // row stride and first column of the aggregates when they hold a chunk of the
                                    // columns (0: the same as ncols and colbase)
};

struct ReplayArgs {
  RunConsts rc;
  const uint8_t *cc;
  const uint64_t *planes;
  const SiteEntry *site;  // [2][18*18]
  const unsigned long long *q;
  const unsigned int *qn;
  unsigned long long qcap;
  long r0, ncols, colbase;
  double *dist;
  unsigned long long *counters;
  const LogTable *logt;
  ExactSink ex;
};

// One undecided pair on its way through the host: the walk writes the formula's exact inputs and the arguments of
// its logarithms, the host writes the C library's log of each argument, and the finish kernel writes the distance.
struct UndEntry {
  double in[7];   // nf[4], diag, ag, ct
  double arg[3];  // arguments of the logarithms (Prep::arg)
  double lg[3];   // log(arg[q]) from the host's C library
  int nlog;       // logarithms the formula takes (0: the maximum distance)
  int state;      // 0 formula, 1 skipped by -l (nothing to write)
  long slot;      // index of the pair's raw distance in its run's dist
  int k, pad;     // run (alignment) of the pair
};

struct RowArgs {
  RunConsts rc;
  const double *dist;
  long r0, r1, ncols, colbase;
  const long *counts;
  const int32_t *name_len;
  const uint64_t *name_off;
  const char *names;
  long maxseg;  // segments per row ([row][segment] arrays below)
  // The resident-reference server's batches: query q spans the columns [seg_cols[q], seg_cols[q+1]); its
  // arrays are indexed [query][row] (so each query's text is contiguous), with per-query histograms.
  const long *seg_cols;  // nullptr outside the server
  long nrows;            // rows of the band (the query-major stride)
  unsigned long long *seg_bytes;
  long long *seg_links, *seg_skip;
  double *seg_max;                    // [row][segment][3]
  double *row_sum, *row_w;            // [row][3]
  unsigned long long *hist;           // [3][200] global
  const unsigned long long *seg_off;  // writer: byte offset of each segment in the band's output
  char *out;
  double *hy;               // hyphy: [N][N] reported distances (NaN = not reported)
  unsigned long long *err;  // set when a segment's text would exceed its counted length
  uint32_t *dcode = nullptr;  // [band rows][ncols] printed-distance codes (print_code): the stats kernel writes them,
                              // the writer formats from them; nullptr: the writer converts the distances itself
};

}  // namespace tn93
