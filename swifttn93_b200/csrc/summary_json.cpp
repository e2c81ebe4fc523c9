// summary_json.cpp -- tn93's JSON summary (swifttn93.cpp:60-74, 2914-2958) as bytes: the same fields in the same
// order, each number printed as its iostream statement prints it (the default stream format of a double is
// printf's "%g"; integers in decimal).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <string>

#include "tn93g.h"

namespace {

void put(std::string &o, const char *fmt, ...)
{
  char b[256];
  va_list ap;
  va_start(ap, fmt);
  const int n = vsnprintf(b, sizeof b, fmt, ap);
  va_end(ap);
  o.append(b, (size_t)n);
}

void histogram(std::string &o, const char *tag, const unsigned long *h)
{
  if (tag)
    put(o, "\t\"Histogram %s\" : [", tag);
  else
    o += "\t\"Histogram\" : [";
  for (int k = 0; k < 200; k++) {
    if (k) o += ',';
    put(o, "[%g,%lu]", (k + 1.) / 200, h[k]);
  }
  o += "]\n";
}

}  // namespace

extern "C" size_t tn93g_summary_json(const tn93g_summary *s, unsigned long n1, unsigned long n2, int second_file,
                                     int fst, char *buf, size_t cap)
{
  std::string o;
  o += "{\n";
  put(o, "\t\"Actual comparisons performed\" :%lu,\n", s->pairwise - (unsigned long)s->skipped);
  put(o, "\t\"Comparisons accounting for copy numbers \" :%g,\n", s->weighted[0] + s->weighted[1] + s->weighted[2]);
  put(o, "\t\"Total comparisons possible\" : %lu,\n", s->pairwise);
  put(o, "\t\"Links found\" : %ld,\n", s->links);
  put(o, "\t\"Maximum distance\" : %g,\n", s->max[0]);
  if (!second_file)
    put(o, "\t\"Sequences\" : %lu,\n", n1);
  else {
    put(o, "\t\"Sequences in first file\" : %lu,\n", n1);
    put(o, "\t\"Sequences in second file\" : %lu,\n", n2);
  }
  unsigned long h0[200];
  for (int k = 0; k < 200; k++) h0[k] = s->hist[0][k];
  if (fst) {
    const char *keys[4] = {"File 1", "File 2", "Between", "Combined"};
    for (int k = 0; k < 3; k++) put(o, "\t\"Mean distance %s\" : %g,\n", keys[k], s->mean[k] / s->weighted[k]);
    const double meta = (s->mean[0] + s->mean[1] + s->mean[2]) / (s->weighted[0] + s->weighted[1] + s->weighted[2]),
                 intra = (s->mean[0] + s->mean[1]) / (s->weighted[0] + s->weighted[1]),
                 piD = s->mean[2] / s->weighted[2] - intra;
    put(o, "\t\"Mean distance [intra] \" : %g,\n", intra);
    put(o, "\t\"Mean distance [combined]\" : %g,\n", meta);
    put(o, "\t\"F_ST\" : %g,\n", piD / (intra + piD));
    for (int k = 0; k < 3; k++) {
      histogram(o, keys[k], s->hist[k]);
      o += ",\n";
    }
    for (int k = 0; k < 200; k++) h0[k] += s->hist[1][k] + s->hist[2][k];
    histogram(o, keys[3], h0);
  } else {
    put(o, "\t\"Mean distance\" : %g,\n", s->mean[0] / s->weighted[0]);
    histogram(o, nullptr, h0);
  }
  o += "}\n";
  if (buf && cap) {
    const size_t n = o.size() < cap ? o.size() : cap - 1;
    for (size_t k = 0; k < n; k++) buf[k] = o[k];
    buf[n] = 0;
  }
  return o.size();
}

//---------------------------------------------------------------------------------------------- certificate
// Every number the summary prints comes from the row-ordered sums of the distances and their maximum. The engine
// computes them from correctly rounded logarithms; tn93 uses the C library's log, which may round a logarithm the
// other way. Per summary unit u the engine reports, over the pairs with such an ambiguous logarithm, the largest
// low and high candidate distance and the sum of (high - low) x weight. With S = the engine's sum and n the length
// of the longest chain of additions a term goes through (a row, then the rows), the C library's run gives a sum
// S' with |S' - S| <= spread (1 + 2g) + 2g |S| (1 + 2g), g = n u / (1 - n u), u = 2^-53 (each sum is within g of
// its exact value, and the exact values differ by at most the spread). Its maximum lies in [largest low,
// max(largest high, M)] when some ambiguous pair reaches M, and is M otherwise. IEEE addition, subtraction and
// division are monotone in each operand, so the printed expressions evaluated at the ends of these intervals
// bound every value tn93 can print; when both ends print the same %g text, so does tn93.
namespace tn93 {

namespace {

struct Iv {
  double lo, hi;
};

Iv iv(double x) { return Iv{x, x}; }
Iv iv_add(Iv a, Iv b) { return Iv{a.lo + b.lo, a.hi + b.hi}; }
Iv iv_sub(Iv a, Iv b) { return Iv{a.lo - b.hi, a.hi - b.lo}; }
// quotient over the corners; an interval denominator must not contain 0
bool iv_div(Iv a, Iv b, Iv &out)
{
  if (!(b.lo > 0. || b.hi < 0.)) return false;
  const double c[4] = {a.lo / b.lo, a.lo / b.hi, a.hi / b.lo, a.hi / b.hi};
  out.lo = out.hi = c[0];
  for (double v : c) {
    if (v != v) return false;
    out.lo = v < out.lo ? v : out.lo;
    out.hi = v > out.hi ? v : out.hi;
  }
  return true;
}
bool same_text(Iv v)
{
  if (v.lo == v.hi) return true;
  char a[64], b[64];
  snprintf(a, sizeof a, "%g", v.lo);
  snprintf(b, sizeof b, "%g", v.hi);
  return strcmp(a, b) == 0;
}

}  // namespace

// bounds[u] = {largest low, largest high, spread, number of ambiguous pairs} of unit u (0..2: the histogram bins);
// chain = n above. True when every number printed by tn93g_summary_json is certain.
bool summary_certified(const tn93g_summary *s, const double bounds[3][4], long chain, int fst)
{
  bool any = false;
  for (int u = 0; u < 3; u++) any |= bounds[u][3] > 0;
  if (!any) return true;
  const double g = (double)chain * 0x1p-53 / (1. - (double)chain * 0x1p-53);
  Iv S[3], M[3];
  for (int u = 0; u < 3; u++) {
    const double sum = s->mean[u];
    if (bounds[u][3] > 0) {
      const double B = bounds[u][2] * (1. + 2. * g) * (1. + 0x1p-40) + 2. * g * fabs(sum) * (1. + 2. * g) + 1e-300;
      S[u] = Iv{nextafter(sum - B, -INFINITY), nextafter(sum + B, INFINITY)};
      M[u] = bounds[u][1] >= s->max[u] ? Iv{bounds[u][0] < s->max[u] ? bounds[u][0] : s->max[u], bounds[u][1]}
                                       : iv(s->max[u]);
    } else {
      S[u] = iv(sum);
      M[u] = iv(s->max[u]);
    }
  }
  if (!same_text(M[0])) return false;
  const Iv W[3] = {iv(s->weighted[0]), iv(s->weighted[1]), iv(s->weighted[2])};
  Iv q;
  if (!fst) return iv_div(S[0], W[0], q) ? same_text(q) : bounds[0][3] == 0;
  // the -m expressions of tn93g_summary_json, in the same order of operations
  Iv m[3];
  for (int k = 0; k < 3; k++) {
    if (!iv_div(S[k], W[k], m[k])) {
      if (bounds[k][3] > 0) return false;
      m[k] = iv(s->mean[k] / s->weighted[k]);
    }
    if (!same_text(m[k])) return false;
  }
  Iv meta, intra, piD, fst_v;
  if (!iv_div(iv_add(iv_add(S[0], S[1]), S[2]), iv_add(iv_add(W[0], W[1]), W[2]), meta)) return false;
  if (!iv_div(iv_add(S[0], S[1]), iv_add(W[0], W[1]), intra)) return false;
  piD = iv_sub(m[2], intra);
  if (!iv_div(piD, iv_add(intra, piD), fst_v)) return false;
  return same_text(intra) && same_text(meta) && same_text(fst_v);
}

}  // namespace tn93

extern "C" int tn93g_summary_certified(const tn93g_summary *s, long chain, int fst)
{
  return s && tn93::summary_certified(s, s->amb_bounds, chain, fst) ? 1 : 0;
}
