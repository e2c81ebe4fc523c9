// Host-side check of the product's scalar arithmetic (swifttn93_b200/csrc/tn93_math.cuh, compiled here for
// the CPU with -ffp-contract=off) against the C library: tlog against log(), fmt_g against printf("%g"),
// tn93_distance against the formula evaluated with log(). Prints one JSON line of counters; exits non-zero
// on any mismatch.   usage: math_check N SEED
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tn93_math.cuh"

namespace tn93 { void build_log_table(LogTable *T); }
using namespace tn93;

static uint64_t st;
static uint64_t rnd() { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return st; }
static double urand() { return (double)(rnd() >> 11) * 0x1p-53; }

static double ref_formula(const double nf[4], double diag, double ag_in, double ct_in)
{
  double s = nf[0] + nf[1] + nf[2] + nf[3];
  double tng = 2. / s, auxd = 1. / s, f[4], K1 = 0, K2 = 0, K3 = 0;
  for (int k = 0; k < 4; k++) f[k] = nf[k] * auxd;
  double fR = f[0] + f[2], fY = f[1] + f[3];
  int k2p = nf[0] == 0 || nf[1] == 0 || nf[2] == 0 || nf[3] == 0;
  if (!k2p) {
    K1 = 2. * f[0] * f[2] / fR;
    K2 = 2. * f[1] * f[3] / fY;
    K3 = 2. * (fR * fY - f[0] * f[2] * fY / fR - f[1] * f[3] * fR / fY);
  }
  double AG = ag_in * tng, CT = ct_in * tng, tv = 1. - (diag * tng + AG + CT);
  if (k2p) {
    double ti = AG + CT;
    AG = 1. - 2. * ti - tv;
    CT = 1. - 2. * tv;
    return (AG > 0. && CT > 0.) ? -0.5 * log(AG) - 0.25 * log(CT) : 1000.0;
  }
  AG = 1. - AG / K1 - 0.5 * tv / fR;
  CT = 1. - CT / K2 - 0.5 * tv / fY;
  tv = 1. - 0.5 * tv / fY / fR;
  return (AG > 0. && CT > 0. && tv > 0) ? -K1 * log(AG) - K2 * log(CT) - K3 * log(tv) : 1000.0;
}

int main(int argc, char **argv)
{
  long n = argc > 1 ? atol(argv[1]) : 1000000;
  st = argc > 2 ? strtoull(argv[2], 0, 10) * 2654435761ull + 0x9E3779B97F4A7C15ull : 1;
  static LogTable T;
  build_log_table(&T);
  long log_bad = 0, log_amb = 0, log_n = 0, g_bad = 0, g_n = 0, d_bad = 0, d_amb = 0, d_n = 0;
  // 1. log against the C library over (0, 1] and around 1 (the formula's inputs), and over all magnitudes
  for (long i = 0; i < n; i++) {
    double u = urand(), x;
    switch (i % 6) {
      case 0: x = 0.5 + 0.5 * u; break;
      case 1: x = 1.0 - u * 0x1p-7; break;
      case 2: x = 1.0 - u * 0x1p-30; break;
      case 3: x = u + 0x1p-1074; break;
      case 4: x = 1.0 + u * 0x1p-6; break;
      default: { uint64_t b = rnd() & 0x7FEFFFFFFFFFFFFFull; memcpy(&x, &b, 8); if (!(x > 0)) x = 1.5; }
    }
    LogR r = tlog(T, x);
    double g = log(x);
    log_n++;
    log_amb += r.amb;
    bool ok = r.amb ? (g == r.y || g == r.alt) : g == r.y;
    if (!ok) {
      if (log_bad < 5) fprintf(stderr, "log mismatch x=%a glibc=%a y=%a alt=%a amb=%d\n", x, g, r.y, r.alt, r.amb);
      log_bad++;
    }
  }
  // 2. %g against printf over random bit patterns, decades and rounding boundaries
  char a[64], b[64];
  for (long i = 0; i < n; i++) {
    double x;
    uint64_t bits = rnd();
    switch (i % 5) {
      case 0: memcpy(&x, &bits, 8); break;
      case 1: x = urand() * 1000.0; break;
      case 2: x = pow(10.0, (double)((int)(rnd() % 40) - 20)) * (1.0 + (urand() - 0.5) * 1e-6); break;
      case 3: { double k = (double)(rnd() % 2000000) + 0.5; x = k * pow(10.0, (double)((int)(rnd() % 16) - 12)); break; }
      default: x = urand() * 1e-4; break;
    }
    int la = fmt_g(x, a);
    if (fmt_g_len(x) != la) {
      if (g_bad < 5) fprintf(stderr, "fmt_g_len mismatch %a: %d vs %d\n", x, fmt_g_len(x), la);
      g_bad++;
    }
    a[la] = 0;
    snprintf(b, sizeof b, "%g", x);
    g_n++;
    if (strcmp(a, b)) {
      if (g_bad < 5) fprintf(stderr, "fmt mismatch %a: got '%s' want '%s'\n", x, a, b);
      g_bad++;
    }
  }
  // powers of ten and their neighbours a few ulps away (the decade estimate's edges)
  for (int e = -8; e <= 8; e++) {
    double x = pow(10.0, (double)e);
    for (int u = 0; u < 4; u++) x = nextafter(x, 0.0);
    for (int u = 0; u < 9; u++, x = nextafter(x, 1e300)) {
      const int la = fmt_g(x, a);
      a[la] = 0;
      snprintf(b, sizeof b, "%g", x);
      g_n++;
      if (strcmp(a, b) || fmt_g_len(x) != la) {
        if (g_bad < 5) fprintf(stderr, "fmt mismatch at a power of ten %a: got '%s' want '%s'\n", x, a, b);
        g_bad++;
      }
    }
  }
  // 3. the full formula over plausible count tables (x16 integer aggregates / 16)
  for (long i = 0; i < n; i++) {
    long L = 50 + (long)(rnd() % 30000);
    long T16 = L * 16 - (long)(rnd() % (L * 8));
    double div = urand() * (i % 3 == 0 ? 0.3 : 0.05);
    long mm = (long)(T16 * div), ts = (long)(mm * urand());
    long ct = (long)(ts * urand());
    double pa = 0.15 + 0.2 * urand(), pc = 0.1 + 0.2 * urand(), pg = 0.1 + 0.2 * urand();
    long nA = (long)(2 * T16 * pa), nC = (long)(2 * T16 * pc), nG = (long)(2 * T16 * pg);
    if (i % 17 == 0) nC = 0;  // K2P branch
    long nT = 2 * T16 - nA - nC - nG;
    double nf[4] = {nA / 16.0, nC / 16.0, nG / 16.0, nT / 16.0};
    double diag = (T16 - mm) / 16.0, agv = (ts - ct) / 16.0, ctv = ct / 16.0;
    Dist D = tn93_distance(T, nf, diag, agv, ctv);
    double ref = ref_formula(nf, diag, agv, ctv);
    // the resolution path: the formula's arguments, the C library's log of each, then the combination
    const Prep P = tn93_prep(nf, diag, agv, ctv);
    const double res = tn93_combine(P, P.nlog ? log(P.arg[0]) : 0., P.nlog ? log(P.arg[1]) : 0.,
                                    P.nlog == 3 ? log(P.arg[2]) : 0.);
    d_n++;
    d_amb += D.amb != 0;
    bool ok = D.amb ? (ref >= D.lo && ref <= D.hi) : (memcmp(&ref, &D.d, 8) == 0);
    ok = ok && memcmp(&ref, &res, 8) == 0;
    // with every logarithm ambiguous (band 0.5 ulp, candidates 2^20 ulps apart) the distance's range must equal the
    // smallest and largest of the eight combinations of candidates
    if (P.nlog) {
      const Dist W = tn93_distance(T, nf, diag, agv, ctv, 0.5, 1048576.0);
      const LogR la = tlog(T, P.arg[0], 0.5, 1048576.0), lc = tlog(T, P.arg[1], 0.5, 1048576.0);
      LogR lt;
      lt.y = lt.alt = 0.0;
      lt.amb = 0;
      if (P.nlog == 3) lt = tlog(T, P.arg[2], 0.5, 1048576.0);
      double lo = 1e300, hi = -1e300;
      for (int m = 0; m < 8; m++) {
        const double v = tn93_combine(P, (m & 1) ? la.alt : la.y, (m & 2) ? lc.alt : lc.y, (m & 4) ? lt.alt : lt.y);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
      }
      if (memcmp(&lo, &W.lo, 8) != 0 || memcmp(&hi, &W.hi, 8) != 0) {
        if (d_bad < 5) fprintf(stderr, "corner mismatch: [%a,%a] want [%a,%a]\n", W.lo, W.hi, lo, hi);
        ok = false;
      }
    }
    if (!ok) {
      if (d_bad < 5) fprintf(stderr, "dist mismatch: got %a [%a,%a] amb %d want %a\n", D.d, D.lo, D.hi, D.amb, ref);
      d_bad++;
    }
  }
  printf("{\"log_n\": %ld, \"log_bad\": %ld, \"log_amb\": %ld, \"fmt_n\": %ld, \"fmt_bad\": %ld, \"dist_n\": %ld, "
         "\"dist_bad\": %ld, \"dist_amb\": %ld}\n",
         log_n, log_bad, log_amb, g_n, g_bad, d_n, d_bad, d_amb);
  return (log_bad || g_bad || d_bad) ? 1 : 0;
}
