// summary_json.cpp -- tn93's JSON summary (swifttn93.cpp:60-74, 2914-2958) as bytes: the same fields in the same
// order, each number printed as its iostream statement prints it (the default stream format of a double is
// printf's "%g"; integers in decimal).
#include <stdarg.h>
#include <stdio.h>

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
