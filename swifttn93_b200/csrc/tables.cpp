// tables.cpp -- tn93's per-site semantics for one pair of codes, tabulated.
//
// The semantics restated here (tn93 v1.1.0 as excerpted in swifttn93 solver/refkernel.cpp):
//   * a code stands for a set of bases: A C G T, U = T, the two-fold R Y S W K M, the three-fold B D H V,
//     and N ? = any base; a gap stands for none (refkernel.cpp:19-35). Its weight is 1 / |set|
//     (refkernel.cpp:38-51: 1, 1/2, 1/3, 1/4, and 0 for the gap);
//   * a clean site (both A/C/G/T) adds 1 to the integer table cell (c1, c2);
//   * a gap on either side contributes nothing; under -a gapmm a gap facing a non-gap counts as N
//     (refkernel.cpp:633-658);
//   * otherwise the ambiguity handler (refkernel.cpp:819-937):
//       - skip mode: nothing;
//       - one side clean (b), the other ambiguous (a): under resolve (or subset with a listed) and b in set(a):
//         one ambiguity, integer cell (b, b) += 1; else each base x of set(a) adds weight(a) to the float cell
//         pairing b with x (orientation kept: row = first sequence);
//       - both ambiguous with norm = weight(a) * weight(b) > 0: under resolve (or subset with both listed)
//         one ambiguity, and if the sets share m bases each shared base adds 1/m to its diagonal cell;
//         otherwise (no shared base, or averaging) every (x, y) of set(a) x set(b) adds norm.
#include "tables.h"

#include <math.h>
#include <string.h>

namespace tn93 {

namespace {

// set(code) as a 4-bit mask over A, C, G, T
const uint8_t kSet[kCodes] = {1, 2, 4, 8, 8, 1 | 4, 2 | 8, 2 | 4, 1 | 8, 4 | 8, 1 | 2, 2 | 4 | 8, 1 | 4 | 8,
                              1 | 2 | 8, 1 | 2 | 4, 15, 15, 0};

double weight(int c)
{
  const int n = __builtin_popcount(kSet[c]);
  if (n == 0) return 0.0;
  if (n == 3) return 1.0 / 3.0;
  return 1.0 / (double)n;
}

struct Site {
  double fc[4][4];
  long ic[4][4];
  long amb;
};

bool resolves(int mode, const unsigned char *subset, int c) { return mode == 0 || (mode == 4 && subset[c]); }

// the contribution of one site with codes (c1, c2) to a pair's counts
void site_contribution(int c1, int c2, int mode, const unsigned char *subset, Site &S)
{
  memset(&S, 0, sizeof S);
  if (c1 == kGap || c2 == kGap) {
    if (mode != 3 || (c1 == kGap && c2 == kGap)) return;
    if (c1 == kGap)
      c1 = kN;
    else
      c2 = kN;
  }
  if (c1 < 4 && c2 < 4) {
    S.ic[c1][c2] = 1;
    return;
  }
  if (mode == 2) return;
  if (c1 < 4 || c2 < 4) {
    const int b = c1 < 4 ? c1 : c2, a = c1 < 4 ? c2 : c1;
    const double w = weight(a);
    if (!(w > 0.)) return;
    if (resolves(mode, subset, a) && (kSet[a] >> b & 1)) {
      S.amb = 1;
      S.ic[b][b] = 1;
      return;
    }
    for (int x = 0; x < 4; x++)
      if (kSet[a] >> x & 1) {
        if (c1 < 4)
          S.fc[b][x] += w;
        else
          S.fc[x][b] += w;
      }
    return;
  }
  const double norm = weight(c1) * weight(c2);
  if (!(norm > 0.0)) return;
  if (resolves(mode, subset, c1) && resolves(mode, subset, c2)) {
    S.amb = 1;
    const int shared = kSet[c1] & kSet[c2];
    const int m = __builtin_popcount(shared);
    if (m > 0) {
      const double v = 1. / m;
      for (int x = 0; x < 4; x++)
        if (shared >> x & 1) S.fc[x][x] += v;
      return;
    }
  }
  for (int x = 0; x < 4; x++)
    if (kSet[c1] >> x & 1)
      for (int y = 0; y < 4; y++)
        if (kSet[c2] >> y & 1) S.fc[x][y] += norm;
}

// x16 aggregates of one site; returns false when a float contribution is not a multiple of 1/16
bool aggregate(const Site &S, int32_t out[8])
{
  double cell[4][4];
  bool dyadic = true;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      const double s = S.fc[a][b] * 16.0;
      if (s != floor(s)) dyadic = false;
      cell[a][b] = s + 16.0 * (double)S.ic[a][b];
    }
  for (int k = 0; k < 8; k++) out[k] = 0;
  out[7] = (int32_t)S.amb;
  if (!dyadic) return false;
  double T = 0, D = 0, nf[4] = {0, 0, 0, 0};
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      T += cell[a][b];
      nf[a] += cell[a][b];
      nf[b] += cell[a][b];
    }
  for (int a = 0; a < 4; a++) D += cell[a][a];
  out[0] = (int32_t)T;
  out[1] = (int32_t)D;
  out[2] = (int32_t)(cell[0][2] + cell[2][0]);
  out[3] = (int32_t)(cell[1][3] + cell[3][1]);
  out[4] = (int32_t)nf[0];
  out[5] = (int32_t)nf[1];
  out[6] = (int32_t)nf[2];
  return true;
}

AggEntry make_agg(int c1, int c2, int mode, const unsigned char *subset)
{
  AggEntry e;
  memset(&e, 0, sizeof e);
  Site S;
  int32_t m[8], a[8];
  site_contribution(c1, c2, mode, subset, S);
  const bool dm = aggregate(S, m);
  site_contribution(c1, c2, 1, subset, S);
  const bool da = aggregate(S, a);
  for (int k = 0; k < 7; k++) e.v[k] = m[k];
  e.v[7] = m[7];
  e.v[8] = dm ? 0 : 1;  // counts entries whose main-mode contribution is not a multiple of 1/16
  for (int k = 0; k < 7; k++) e.v[9 + k] = a[k];
  return e;
}

}  // namespace

void build_tables(Tables *T, int mode, const unsigned char subset[kCodes])
{
  memset(T, 0, sizeof *T);
  for (int c = kSparse0; c < kGap; c++)
    for (int o = 0; o < kCodes; o++) T->ev[(c - kSparse0) * kCodes + o] = make_agg(c, o, mode, subset);
  for (int b = 0; b < 4; b++) T->ew[b] = make_agg(kN, b, mode, subset);
  T->eww = make_agg(kN, kN, mode, subset);
  for (int t = 0; t < 2; t++) {
    const int m = t == 0 ? mode : 1;
    for (int c1 = 0; c1 < kCodes; c1++)
      for (int c2 = 0; c2 < kCodes; c2++) {
        SiteEntry &s = T->site[t][c1 * kCodes + c2];
        memset(&s, 0, sizeof s);
        if (c1 < 4 && c2 < 4) continue;  // clean sites are counted by the caller
        Site S;
        site_contribution(c1, c2, m, subset, S);
        for (int q = 0; q < 16; q++) s.fc[q] = S.fc[q >> 2][q & 3];
        for (int q = 0; q < 4; q++) s.icd[q] = (int32_t)S.ic[q][q];
        s.amb = (int32_t)S.amb;
      }
  }
}

void pack_tables(const Tables &T, bool w_plane, PackedTables *P)
{
  memset(P, 0, sizeof *P);
  for (int c = kSparse0; c < kGap; c++)
    for (int o = 0; o < kCodes; o++) {
      const int k = (c - kSparse0) * kCodes + o;
      const int32_t *v = T.ev[k].v;
      const uint32_t w[4] = {(uint32_t)v[0] | (uint32_t)v[1] << 16, (uint32_t)v[2] | (uint32_t)v[3] << 16,
                             (uint32_t)v[4] | (uint32_t)v[5] << 16, (uint32_t)v[6] | (uint32_t)v[7] << 16};
      const bool partner_sparse = is_sparse_code(o, w_plane);
      for (int q = 0; q < 4; q++) {
        P->row[k][q] = w[q];
        P->col[k][q] = partner_sparse ? 0u : w[q];
      }
      P->rowf[k] = (uint32_t)v[8];
      P->colf[k] = partner_sparse ? 0u : (uint32_t)v[8];
    }
}

}  // namespace tn93
