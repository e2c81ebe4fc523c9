// tables.h -- per-site contribution tables of tn93's ambiguity semantics, built on the host once per run and
// uploaded to the device.
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace tn93 {

constexpr int kCodes = 18;   // "ACGTURYSWKMBDHVN?-"
constexpr int kGap = 17;
constexpr int kN = 15;
constexpr int kSparse0 = 4;  // first non-clean code
constexpr int kSparseCodes = 13;  // codes 4..16

// Lanes of an aggregate entry (x16 integers, exact while every contribution is a multiple of 1/16):
//   0 T (total), 1 D (diagonal), 2 AG (A<->G), 3 CT (C<->T), 4 nfA, 5 nfC, 6 nfG  -- the main mode
//   7 ambiguity count (resolved events, for the -g test)
//   8 1 when the main-mode contribution is not a multiple of 1/16 (a pair with any such site takes the
//     site-order replay)
//   9..15 lanes 0..6 in AVERAGE mode (the -g fallback)
constexpr int kLanes = 16;
struct AggEntry {
  int32_t v[kLanes];
};

// One site of the site-order replay: the float contributions of tn93's handler to the 4x4 table (row = code of
// the first sequence), its integer diagonal increments and its ambiguity count.
struct SiteEntry {
  double fc[16];
  int32_t icd[4];
  int32_t amb;
  int32_t pad[3];
};

struct Tables {
  AggEntry ev[kSparseCodes * kCodes];  // [c - 4][o]: a sparse code c of one sequence facing code o
  AggEntry ew[4];                      // N (or, under gapmm, a gap) facing clean base b
  AggEntry eww;                        // N facing N
  SiteEntry site[2][kCodes * kCodes];  // [0 main mode, 1 AVERAGE][c1 * 18 + c2]
  // ev, ew and eww form one array of kSparseCodes * kCodes + 5 entries (copied to the device as one table)
  const AggEntry *agg() const { return ev; }
};
static_assert(offsetof(Tables, ew) == sizeof(AggEntry) * kSparseCodes * kCodes &&
                  offsetof(Tables, eww) == offsetof(Tables, ew) + 4 * sizeof(AggEntry),
              "the event tables are contiguous");

// mode: 0 resolve, 1 average, 2 skip, 3 gapmm, 4 subset; subset[c] = 1 for codes listed in -a LIST
void build_tables(Tables *T, int mode, const unsigned char subset[kCodes]);

// The pair kernel's copy of the event table, packed: per (sparse code c of one sequence, code o of the other) the
// main-mode x16 lanes two to a 32-bit word, w[0] = T | D << 16, w[1] = AG | CT << 16, w[2] = nfA | nfC << 16,
// w[3] = nfG | amb << 16, and a separate flag word (1: not a multiple of 1/16). No lane of an entry exceeds 32, so
// packed sums stay exact for fewer than 2048 events per pair; the engine packs when no sequence has more than
// kPackedMaxEvents events. col[] is row[] with zeros where o is itself a sparse event code (such a site is counted
// once, from the row's side), so the column side needs no test.
constexpr int kPackedMaxEvents = 1023;
constexpr int kEvEntries = kSparseCodes * kCodes;
struct PackedTables {
  uint32_t row[kEvEntries][4];
  uint32_t col[kEvEntries][4];
  uint32_t rowf[kEvEntries];
  uint32_t colf[kEvEntries];
};
void pack_tables(const Tables &T, bool w_plane, PackedTables *P);

// true if code c is a "sparse event" code: not clean, not a gap, and not N when N has its own plane
inline bool is_sparse_code(int c, bool w_plane) { return c >= kSparse0 && c < kGap && !(w_plane && c == kN); }

}  // namespace tn93
