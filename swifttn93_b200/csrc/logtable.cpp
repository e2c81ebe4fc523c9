// logtable.cpp -- fills the reduction table of tlog (tn93_math.cuh) with quadruple-precision values.
#include <quadmath.h>
#include <string.h>

#include "tn93_math.cuh"

namespace tn93 {

static void split(__float128 v, double &hi, double &lo)
{
  hi = (double)v;
  lo = (double)(v - (__float128)hi);
}

void build_log_table(LogTable *T)
{
  for (int i = 0; i < kLogTab; i++) {
    double c;
    if (i == 0 || i == kLogTab - 1)
      c = 1.0;  // the intervals touching 1: f = x - 1 exactly
    else if (i < kLogFold)
      c = (257.0 + 2.0 * i) / 256.0;  // centre of [1 + i/128, 1 + (i+1)/128)
    else
      c = (257.0 + 2.0 * i) / 512.0;  // centre of the folded interval [(128+i)/256, (129+i)/256)
    T->c[i] = c;
    split((__float128)1 / (__float128)c, T->invc_hi[i], T->invc_lo[i]);
    split(logq((__float128)c), T->logc_hi[i], T->logc_lo[i]);
  }
  const __float128 ln2 = logq((__float128)2);
  double h = (double)ln2;
  uint64_t u;
  memcpy(&u, &h, 8);
  u &= ~((1ull << 11) - 1);  // keep 42 significant bits
  memcpy(&h, &u, 8);
  T->ln2_hi = h;
  T->ln2_lo = (double)(ln2 - (__float128)h);
}

}  // namespace tn93
