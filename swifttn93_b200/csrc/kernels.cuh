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
};

struct PairArgs {
  RunConsts rc;
  const uint64_t *planes;
  const uint8_t *cc, *ccT;
  const uint32_t *ev_off, *ev;
  const AggEntry *agg;  // Tables::ev, then ew[4], eww
  long r0, r1;          // band rows
  long ncols, colbase;  // row stride of dist and the first global column it holds
  long cstart;          // first column of the launch grid (a multiple of 32 past colbase)
  double *dist;
  unsigned long long *replay_q;  // (t << 63) | (i << 31) | j
  unsigned int *replay_n;
  unsigned long long replay_cap;
  unsigned long long *counters;  // [0] pairs with an ambiguous log, [1] undecided pairs
  const LogTable *logt;
  const void *tcagg = nullptr;  // clean-site aggregates from the tensor-core kernel ([7][band rows][ncols])
  size_t tcplane = 0;           // (band rows) x ncols
  int tc16 = 0;                 // the aggregates are uint16 (every value fits: 2 Lc < 65536), else int32
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
};

}  // namespace tn93
