// tn93_math.cuh -- exact scalar arithmetic of the all-pairs TN93 path, compiled for the device and (for
// tests) for the host:
//   * tn93_distance: the TN93 / K2P formula in tn93's exact IEEE order of operations, with no fused
//     multiply-adds (swifttn93 solver/swifttn93.cpp:1954-2001, tn93 refkernel.cpp:752-803);
//   * tlog: a natural logarithm written from the mathematics (table-driven reduction after Tang, ACM TOMS
//     15(2), 1989, evaluated in double-double) that returns the correctly rounded result together with a
//     flag when the exact value lies so close to a rounding midpoint that the C library's log, whose
//     documented error is up to 0.52 ulp, may round the other way. The caller then evaluates both
//     candidates and checks that every printed byte and decision agrees (a decision-stability
//     certificate);
//   * hist_bin: the histogram index with x86 double->long semantics and tn93's unsigned clamp
//     (solver/swifttn93.cpp:2003-2014);
//   * fmt_g: printf("%g") at precision 6, exact for every double (round-half-even on the exact binary value,
//     as glibc does), used for every distance written to the output (solver/fastfmt.h:75-157).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define TN_HD __host__ __device__ __forceinline__
#define TN_HDI __host__ __device__
#else
#define TN_HD static inline
#define TN_HDI static
#endif

#if defined(__CUDA_ARCH__)
// explicit round-to-nearest operations: the compiler may not contract them into fused multiply-adds
#define TADD(a, b) __dadd_rn((a), (b))
#define TSUB(a, b) __dsub_rn((a), (b))
#define TMUL(a, b) __dmul_rn((a), (b))
#define TDIV(a, b) __ddiv_rn((a), (b))
#define TFMA(a, b, c) __fma_rn((a), (b), (c))
#define TFLOOR(a) floor(a)
#define TBITS(x) ((uint64_t)__double_as_longlong(x))
#define TDBL(u) __longlong_as_double((long long)(u))
#else
#include <math.h>
#include <string.h>
// host builds of this header are compiled with -ffp-contract=off
#define TADD(a, b) ((a) + (b))
#define TSUB(a, b) ((a) - (b))
#define TMUL(a, b) ((a) * (b))
#define TDIV(a, b) ((a) / (b))
#define TFMA(a, b, c) fma((a), (b), (c))
#define TFLOOR(a) floor(a)
static inline uint64_t tn_bits_host(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static inline double tn_dbl_host(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }
#define TBITS(x) tn_bits_host(x)
#define TDBL(u) tn_dbl_host(u)
#endif

namespace tn93 {

constexpr int kHistBins = 200;
constexpr double kMaxDist = 1000.0;

//---------------------------------------------------------------------------------------------- log tables
// Reduction: x = 2^k * m with m in [1, 2) split into 128 intervals by its top 7 fraction bits; intervals at
// and above 1 + 53/128 are folded down (m/2, k+1) so that m lies in [0.707, 1.414). Each interval has a
// centre c with at most 10 significant bits (c = 1 exactly for the two intervals touching 1), so f = m - c is
// exact; log x = k ln2 + log c + log1p(f / c). The table holds 1/c and log c as double-doubles; the host
// fills it once with quadruple-precision arithmetic (libquadmath) and uploads it.
constexpr int kLogTab = 128;
constexpr int kLogFold = 53;
struct LogTable {
  double c[kLogTab];
  double invc_hi[kLogTab], invc_lo[kLogTab];
  double logc_hi[kLogTab], logc_lo[kLogTab];
  double ln2_hi, ln2_lo;  // ln2_hi has 42 significant bits, so k * ln2_hi is exact for |k| < 2048
};

// The C library's log may differ from the correctly rounded value when the exact value lies within
// (0.519 - 0.5) ulp of a midpoint; values within this band (with a margin) are reported as ambiguous. The band
// is a run parameter (at least kLogBand, at most 0.5 ulp: every log ambiguous), and so is the distance of the
// other candidate (kLogSpread = 1 ulp, the most the C library can differ by). Tests widen both to drive pairs
// through the certificate's failure path; the defaults are what every run uses otherwise.
constexpr double kLogBand = 0.03;
constexpr double kLogSpread = 1.0;

struct LogR {
  double y;    // correctly rounded log (best estimate)
  double alt;  // the other candidate when amb
  int amb;     // 1 if the C library may return alt instead of y
};

TN_HD void two_sum(double a, double b, double &s, double &e)
{
  s = TADD(a, b);
  double bb = TSUB(s, a);
  e = TADD(TSUB(a, TSUB(s, bb)), TSUB(b, bb));
}
TN_HD void fast_two_sum(double a, double b, double &s, double &e)
{
  s = TADD(a, b);
  e = TSUB(b, TSUB(s, a));
}

// log of a positive finite x (callers never pass anything else); band and spread in ulps (see kLogBand)
TN_HD LogR tlog(const LogTable &T, double x, double band = kLogBand, double spread = kLogSpread)
{
  LogR R;
  R.amb = 0;
  if (x == 1.0) {
    R.y = R.alt = 0.0;
    return R;
  }
  uint64_t b = TBITS(x);
  int k = 0;
  if ((b >> 52) == 0) {  // subnormal: scale into the normal range
    x = TMUL(x, 18014398509481984.0);  // 2^54
    b = TBITS(x);
    k = -54;
  }
  k += (int)(b >> 52) - 1023;
  int idx = (int)((b >> 45) & 127);
  double m = TDBL((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  if (idx >= kLogFold) {
    m = TMUL(m, 0.5);
    k += 1;
  }
  const double c = T.c[idx];
  const double f = TSUB(m, c);  // exact (Sterbenz)
  // r = f / c as a double-double
  const double r_hi = TMUL(f, T.invc_hi[idx]);
  const double r_lo = TADD(TFMA(f, T.invc_hi[idx], -r_hi), TMUL(f, T.invc_lo[idx]));
  // log1p(r) = r - r^2/2 + r^3 P(r), P(r) = 1/3 - r/4 + ... + r^8/11 (|r| < 2^-7: the tail is below 2^-70 r)
  const double q = r_hi;
  const double t2h = TMUL(q, q), t2l = TFMA(q, q, -t2h);
  double P = 1.0 / 11.0;
  P = TFMA(P, q, -1.0 / 10.0);
  P = TFMA(P, q, 1.0 / 9.0);
  P = TFMA(P, q, -1.0 / 8.0);
  P = TFMA(P, q, 1.0 / 7.0);
  P = TFMA(P, q, -1.0 / 6.0);
  P = TFMA(P, q, 1.0 / 5.0);
  P = TFMA(P, q, -1.0 / 4.0);
  P = TFMA(P, q, 1.0 / 3.0);
  const double tail = TMUL(TMUL(t2h, q), P);
  double s_hi, s_lo;
  two_sum(q, TMUL(-0.5, t2h), s_hi, s_lo);
  // remaining small terms: -t2l/2 + tail + r_lo / (1 + q)
  s_lo = TADD(s_lo, TADD(TADD(TMUL(-0.5, t2l), tail), TSUB(r_lo, TMUL(r_lo, q))));
  // k ln2 + log c + (s_hi + s_lo)
  const double kd = (double)k;
  double u_hi, u_lo, v_hi, v_lo;
  two_sum(TMUL(kd, T.ln2_hi), T.logc_hi[idx], u_hi, u_lo);
  two_sum(u_hi, s_hi, v_hi, v_lo);
  const double lo = TADD(TADD(TADD(u_lo, v_lo), TADD(s_lo, T.logc_lo[idx])), TMUL(kd, T.ln2_lo));
  double hi, lo2;
  fast_two_sum(v_hi, lo, hi, lo2);
  // hi is the rounding of the double-double (hi + lo2); |exact - (hi + lo2)| <= 2^-69 |hi|
  R.y = hi;
  R.alt = hi;
  const uint64_t hb = TBITS(hi);
  const int hexp = (int)((hb >> 52) & 0x7ff);
  const double ulp = TDBL((uint64_t)(hexp > 52 ? hexp - 52 : 1) << 52);  // 2^(e-52)
  const bool pow2 = (hb & 0x000FFFFFFFFFFFFFull) == 0;
  const double E = TMUL(hi < 0 ? -hi : hi, 1.6940658945086007e-21);  // 2^-69 |hi|
  // e_away > 0: the remainder points away from zero
  const double e_away = hi < 0 ? -lo2 : lo2;
  const double half = (e_away >= 0 || !pow2) ? TMUL(0.5, ulp) : TMUL(0.25, ulp);
  const double margin = TSUB(TSUB(half, e_away < 0 ? -e_away : e_away), E);
  if (margin <= TMUL(band, ulp)) {
    R.amb = 1;
    // neighbour of hi on the side of the remainder (spread ulps away; 1 unless a test widens it)
    const bool away = e_away >= 0;
    const uint64_t sp = (uint64_t)spread;
    R.alt = TDBL(away ? hb + sp : hb - sp);
  }
  return R;
}

//---------------------------------------------------------------------------------------------- formula
// Formula inputs, all exact: nf[4] base totals over both sequences, diag = sum of the 4x4 diagonal,
// ag = fc[A][G] + fc[G][A], ct = fc[C][T] + fc[T][C].
struct Dist {
  double d;      // distance from the correctly rounded logarithms
  double lo, hi; // range of the distance over every candidate the C library's log may give
  int amb;       // number of ambiguous logarithms
};

// The formula up to its logarithms: whether it is K2P (a base absent from both sequences), its coefficients, and
// the arguments of its two (K2P) or three logarithms. nlog = 0 when an argument is not positive (tn93 then
// reports the maximum distance).
struct Prep {
  int nlog;
  bool k2p;
  double K1, K2, K3;
  double arg[3];
};

// x / b rounded to nearest, given y = RN(1 / b). On the device the quotient is corrected twice with fused
// multiply-adds (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000 processor", IBM J.
// Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point Arithmetic, ch. on FMA-based division):
// q0 = RN(x y) lies within 1.5 ulp of x / b; q1 = RN(q0 + r0 y) with r0 = RN(x - b q0) lies within 1 ulp; then
// r1 = x - b q1 is exact and RN(q1 + r1 y) = RN(x / b) by Markstein's theorem. It holds while no product or
// remainder underflows or overflows, which the formula cannot reach: base frequencies are at least 2^-31 (a
// sixteenth of a count over at most 2^26 sites), so every nonzero operand lies between 2^-200 and 2^200. Several
// quotients share one divisor, so one true division (the reciprocal) serves all of them. The host build divides.
TN_HD double div_by(double x, double b, double y)
{
#if defined(__CUDA_ARCH__)
  const double q0 = TMUL(x, y);
  const double r0 = TFMA(-q0, b, x);
  const double q1 = TFMA(r0, y, q0);
  const double r1 = TFMA(-q1, b, x);
  return TFMA(r1, y, q1);
#else
  (void)y;
  return x / b;
#endif
}

// tn93's formula (refkernel.cpp:752-803, swifttn93.cpp:1954-2001) with every IEEE operation in its order, split
// at the logarithms: tn93_prep computes their arguments, tn93_combine the distance from their values. Every
// quotient is the correctly rounded one (div_by with the divisor's reciprocal, or a true division).
TN_HD Prep tn93_prep(const double nf[4], double diag, double ag_in, double ct_in)
{
  Prep P;
  const double s = TADD(TADD(TADD(nf[0], nf[1]), nf[2]), nf[3]);
  // tn93 divides 2 by s and 1 by s; scaling by 2 commutes with rounding, so 2 x (1 / s) is the same double
  const double auxd = TDIV(1.0, s);
  const double tng = TMUL(2.0, auxd);
  double f0 = TMUL(nf[0], auxd), f1 = TMUL(nf[1], auxd), f2 = TMUL(nf[2], auxd), f3 = TMUL(nf[3], auxd);
  const double fR = TADD(f0, f2), fY = TADD(f1, f3);
  P.k2p = nf[0] == 0 || nf[1] == 0 || nf[2] == 0 || nf[3] == 0;
  P.K1 = P.K2 = P.K3 = 0;
  double rR = 0, rY = 0;  // RN(1 / fR), RN(1 / fY)
  if (!P.k2p) {
    rR = TDIV(1.0, fR);
    rY = TDIV(1.0, fY);
    P.K1 = div_by(TMUL(TMUL(2.0, f0), f2), fR, rR);
    P.K2 = div_by(TMUL(TMUL(2.0, f1), f3), fY, rY);
    P.K3 = TMUL(2.0, TSUB(TSUB(TMUL(fR, fY), div_by(TMUL(TMUL(f0, f2), fY), fR, rR)),
                          div_by(TMUL(TMUL(f1, f3), fR), fY, rY)));
  }
  double AG = TMUL(ag_in, tng), CT = TMUL(ct_in, tng);
  double tv = TSUB(1.0, TADD(TADD(TMUL(diag, tng), AG), CT));
  if (P.k2p) {
    const double ti = TADD(AG, CT);
    AG = TSUB(TSUB(1.0, TMUL(2.0, ti)), tv);
    CT = TSUB(1.0, TMUL(2.0, tv));
    P.arg[0] = AG;
    P.arg[1] = CT;
    P.arg[2] = 1.0;
    P.nlog = (AG > 0. && CT > 0.) ? 2 : 0;
  } else {
    const double htv = TMUL(0.5, tv), hY = div_by(htv, fY, rY);
    AG = TSUB(TSUB(1.0, TDIV(AG, P.K1)), div_by(htv, fR, rR));
    CT = TSUB(TSUB(1.0, TDIV(CT, P.K2)), hY);
    tv = TSUB(1.0, div_by(hY, fR, rR));
    P.arg[0] = AG;
    P.arg[1] = CT;
    P.arg[2] = tv;
    P.nlog = (AG > 0. && CT > 0. && tv > 0) ? 3 : 0;
  }
  return P;
}

// the distance from the logarithms of P's arguments (lg[0..nlog)); the maximum distance when nlog = 0
TN_HD double tn93_combine(const Prep &P, double la, double lc, double lt)
{
  if (P.nlog == 0) return kMaxDist;
  if (P.k2p) return TSUB(TMUL(-0.5, la), TMUL(0.25, lc));
  const double nK1 = -P.K1;
  return TSUB(TSUB(TMUL(nK1, la), TMUL(P.K2, lc)), TMUL(P.K3, lt));
}

TN_HD Dist tn93_distance(const LogTable &T, const double nf[4], double diag, double ag_in, double ct_in,
                         double band = kLogBand, double spread = kLogSpread)
{
  Dist D;
  D.amb = 0;
  const Prep P = tn93_prep(nf, diag, ag_in, ct_in);
  if (P.nlog == 0) {
    D.d = D.lo = D.hi = kMaxDist;
    return D;
  }
  const LogR a = tlog(T, P.arg[0], band, spread), c = tlog(T, P.arg[1], band, spread);
  LogR t;
  t.y = t.alt = 0.0;
  t.amb = 0;
  if (P.nlog == 3) t = tlog(T, P.arg[2], band, spread);
  D.d = tn93_combine(P, a.y, c.y, t.y);
  D.lo = D.hi = D.d;
  D.amb = a.amb + c.amb + t.amb;
  if (D.amb) {
    // The range over every combination of candidates. tn93_combine is monotone in each logarithm (IEEE products and
    // differences round monotonically): non-increasing in la, lc, lt when K1, K2, K3 >= 0 (always under K2P, whose
    // coefficients are -1/2 and -1/4), non-decreasing when negative. So the smallest distance is the combination
    // that takes, per logarithm, the larger candidate where its coefficient is >= 0 and the smaller elsewhere, and
    // the largest the opposite one: the same two values the eight corners would give.
    const bool da = P.k2p || P.K1 >= 0, dc = P.k2p || P.K2 >= 0, dt = P.k2p || P.K3 >= 0;
    const double a_hi = a.alt > a.y ? a.alt : a.y, a_lo = a.alt > a.y ? a.y : a.alt;
    const double c_hi = c.alt > c.y ? c.alt : c.y, c_lo = c.alt > c.y ? c.y : c.alt;
    const double t_hi = t.alt > t.y ? t.alt : t.y, t_lo = t.alt > t.y ? t.y : t.alt;
    D.lo = tn93_combine(P, da ? a_hi : a_lo, dc ? c_hi : c_lo, dt ? t_hi : t_lo);
    D.hi = tn93_combine(P, da ? a_lo : a_hi, dc ? c_lo : c_hi, dt ? t_lo : t_hi);
  }
  return D;
}

// histogram index of a raw distance: floor(d * 200) converted to a signed 64-bit integer (NaN and out-of-range
// values become INT64_MIN, as the x86 conversion does), then clamped to the last bin as an unsigned value
TN_HD int hist_bin(double d)
{
  const double f = TFLOOR(TMUL(d, 200.0));
  if (!(f >= 0.0 && f < (double)kHistBins)) return kHistBins - 1;
  return (int)f;
}

//---------------------------------------------------------------------------------------------- %g
// Decimal digits of a positive finite double: q in [100000, 999999] and exponent X with
// value ~= q * 10^(X-5), q rounded half-to-even on the exact binary value.
struct Dec {
  uint32_t q;
  int X;
};

// 64x64 -> 128 multiply
TN_HD void mul64(uint64_t a, uint64_t b, uint64_t &hi, uint64_t &lo)
{
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umul64hi(a, b);
#else
  unsigned __int128 p = (unsigned __int128)a * b;
  lo = (uint64_t)p;
  hi = (uint64_t)(p >> 64);
#endif
}

// Big-integer arithmetic for values outside [1e-5, 1e5): little-endian 32-bit limbs (up to 1280 bits).
constexpr int kBigLimbs = 40;
struct Big {
  uint32_t w[kBigLimbs];
  int n;
};
TN_HDI inline void big_set(Big &a, uint64_t v)
{
  for (int i = 0; i < kBigLimbs; i++) a.w[i] = 0;
  a.w[0] = (uint32_t)v;
  a.w[1] = (uint32_t)(v >> 32);
  a.n = a.w[1] ? 2 : (a.w[0] ? 1 : 0);
}
TN_HDI inline void big_mul_small(Big &a, uint32_t m)
{
  uint64_t carry = 0;
  for (int i = 0; i < a.n; i++) {
    const uint64_t t = (uint64_t)a.w[i] * m + carry;
    a.w[i] = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry) a.w[a.n++] = (uint32_t)carry;
}
// a /= d, returns the remainder
TN_HDI inline uint32_t big_div_small(Big &a, uint32_t d)
{
  uint64_t rem = 0;
  for (int i = a.n - 1; i >= 0; i--) {
    const uint64_t cur = (rem << 32) | a.w[i];
    a.w[i] = (uint32_t)(cur / d);
    rem = cur % d;
  }
  while (a.n && a.w[a.n - 1] == 0) a.n--;
  return (uint32_t)rem;
}
TN_HDI inline void big_shl(Big &a, int s)
{
  if (a.n == 0 || s == 0) return;
  const int limbs = s >> 5, bits = s & 31;
  for (int i = a.n - 1 + limbs + 1; i >= 0; i--) {
    const int src = i - limbs;
    uint32_t v = 0;
    if (src >= 0 && src < a.n) v = a.w[src] << bits;
    if (bits && src - 1 >= 0 && src - 1 < a.n) v |= a.w[src - 1] >> (32 - bits);
    if (i < kBigLimbs) a.w[i] = v;
  }
  a.n = a.n + limbs + 1;
  if (a.n > kBigLimbs) a.n = kBigLimbs;
  while (a.n && a.w[a.n - 1] == 0) a.n--;
}
// a >>= s (s >= 1); returns the discarded bits compared with 2^(s-1): -1 below, 0 equal, +1 above
TN_HDI inline int big_shr_cmp_half(Big &a, int s)
{
  const int hb = s - 1;
  const int hl = hb >> 5, hbit = hb & 31;
  const bool half = hl < a.n && ((a.w[hl] >> hbit) & 1);
  bool below = hl < a.n && (a.w[hl] & ((1u << hbit) - 1)) != 0;
  for (int i = 0; i < hl && i < a.n; i++)
    if (a.w[i]) below = true;
  const int limbs = s >> 5, bits = s & 31;
  for (int i = 0; i < a.n; i++) {
    const int src = i + limbs;
    uint32_t v = 0;
    if (src < a.n) v = a.w[src] >> bits;
    if (bits && src + 1 < a.n) v |= a.w[src + 1] << (32 - bits);
    a.w[i] = v;
  }
  a.n = a.n - limbs;
  if (a.n < 0) a.n = 0;
  while (a.n && a.w[a.n - 1] == 0) a.n--;
  return half ? (below ? 1 : 0) : -1;
}
TN_HDI inline uint64_t big_low64(const Big &a)
{
  return (a.n > 0 ? a.w[0] : 0) | ((a.n > 1 ? (uint64_t)a.w[1] : 0) << 32);
}
// a /= 5^k; returns true if any remainder along the way was non-zero (i.e. 5^k does not divide a)
TN_HDI inline bool big_div_pow5(Big &a, int k)
{
  bool rem = false;
  for (; k > 0; k -= 13) {
    uint32_t d = 1;
    for (int j = 0; j < (k < 13 ? k : 13); j++) d *= 5u;
    if (big_div_small(a, d)) rem = true;
  }
  return rem;
}
TN_HDI inline void big_mul_pow5(Big &a, int k)
{
  for (; k > 0; k -= 13) {
    uint32_t d = 1;
    for (int j = 0; j < (k < 13 ? k : 13); j++) d *= 5u;
    big_mul_small(a, d);
  }
}

// floor(m * 2^e2 * 10^s) (truncated to 64 bits; callers only use values below 10^7) and the comparison of
// the discarded fraction with 1/2 in cmp (-1 below, 0 exactly half, +1 above).
TN_HDI inline uint64_t dec_scale_big(uint64_t m, int e2, int s, int &cmp)
{
  Big A;
  big_set(A, m);
  const int t = e2 + s;  // net power of two once 10^s = 5^s 2^s
  if (s >= 0) {
    big_mul_pow5(A, s);
    if (t >= 0) {
      big_shl(A, t);
      cmp = -1;
    } else {
      cmp = big_shr_cmp_half(A, -t);
    }
    return big_low64(A);
  }
  const int a = -s;
  int u = 0;
  if (t >= 0)
    big_shl(A, t);
  else
    u = -t;
  if (u == 0) {
    // frac = (A mod 5^a) / 5^a, never exactly 1/2 (5^a is odd): floor(2A / 5^a) - 2 floor(A / 5^a) is 1 iff frac > 1/2
    Big A2 = A;
    big_mul_small(A2, 2);
    big_div_pow5(A, a);
    big_div_pow5(A2, a);
    const uint64_t q1 = big_low64(A), q2 = big_low64(A2);
    cmp = (q2 - 2 * q1) == 1 ? 1 : -1;
    return q1;
  }
  const bool rem5 = big_div_pow5(A, a);
  const int h = big_shr_cmp_half(A, u);
  cmp = (h == 0 && rem5) ? 1 : h;
  return big_low64(A);
}

// 10^s for 0 <= s <= 10
#if defined(__CUDACC__)
__constant__ uint64_t kPow10u[11] = {1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull, 1000000ull, 10000000ull,
                                     100000000ull, 1000000000ull, 10000000000ull};
#endif
TN_HD uint64_t pow10u(int s)
{
#if defined(__CUDA_ARCH__)
  return kPow10u[s];
#else
  uint64_t p = 1;
  for (int i = 0; i < s; i++) p *= 10u;
  return p;
#endif
}

// the same for 1e-5 <= d < 1e5, where m * 10^s < 2^87 and the binary shift is 26..68 bits (0 <= s <= 10)
TN_HD uint64_t dec_scale_fast(uint64_t m, int e2, int s, int &cmp)
{
  const uint64_t p10 = pow10u(s);
  uint64_t hi, lo;
  mul64(m, p10, hi, lo);
  const int u = -(e2);  // value = (hi:lo) * 2^e2, e2 < 0 here
  uint64_t q, rh, rl, halfh, halfl;  // remainder (rh:rl) and 2^(u-1) as 128-bit values
  if (u >= 64) {
    q = hi >> (u - 64);
    rh = u - 64 == 0 ? 0 : (hi & ((1ull << (u - 64)) - 1));
    rl = lo;
    halfh = 1ull << (u - 65);
    halfl = 0;
    if (u == 64) {  // 2^63 sits in the low word
      halfh = 0;
      halfl = 1ull << 63;
    }
  } else {
    q = (lo >> u) | (u ? (hi << (64 - u)) : 0);
    rh = 0;
    rl = lo & ((1ull << u) - 1);
    halfh = 0;
    halfl = 1ull << (u - 1);
  }
  cmp = rh > halfh ? 1 : (rh < halfh ? -1 : (rl > halfl ? 1 : (rl < halfl ? -1 : 0)));
  return q;
}

// six significant digits of d > 0 (finite), rounded half-to-even on the exact binary value
TN_HD Dec decimal6(double d)
{
  const uint64_t b = TBITS(d);
  const int be = (int)((b >> 52) & 0x7ff);
  uint64_t m = b & 0x000FFFFFFFFFFFFFull;
  int e2;
  if (be == 0) {
    e2 = -1074;
  } else {
    m |= 1ull << 52;
    e2 = be - 1075;
  }
  const bool fast = d >= 1e-5 && d < 1e5;
  // decimal exponent estimate: a comparison chain in the fast window (an estimate off by one near a power of ten
  // is corrected by the loop below, which checks that the scaled value has six digits), log10 elsewhere
  int X;
  if (fast) {
    const double p10[9] = {1e-4, 1e-3, 1e-2, 1e-1, 1e0, 1e1, 1e2, 1e3, 1e4};
    X = -5;
#pragma unroll
    for (int k = 0; k < 9; k++) X += d >= p10[k] ? 1 : 0;
  } else {
    X = (int)floor(log10(d));
  }
  uint64_t q = 0;
  int cmp = 0;
  for (int guard = 0; guard < 4; guard++) {
    const int s = 5 - X;
    // the fast path covers 1 <= s <= 10; an estimate that left the window takes the exact general path
    q = (fast && s >= 1 && s <= 10) ? dec_scale_fast(m, e2, s, cmp) : dec_scale_big(m, e2, s, cmp);
    if (q >= 1000000ull)
      X++;
    else if (q < 100000ull)
      X--;
    else
      break;
  }
  q += (cmp > 0 || (cmp == 0 && (q & 1))) ? 1 : 0;
  if (q == 1000000ull) {
    q = 100000ull;
    X++;
  }
  Dec r;
  r.q = (uint32_t)q;
  r.X = X;
  return r;
}

// the text of printf("%g") for a positive value with decimal digits D (after any sign); returns the length
TN_HD int fmt_dec(const Dec &D, char *out)
{
  int n = 0;
  char dg[6];
  uint32_t q = D.q;
  for (int i = 5; i >= 0; i--) {
    dg[i] = (char)('0' + q % 10u);
    q /= 10u;
  }
  int nd = 6;
  while (nd > 1 && dg[nd - 1] == '0') nd--;
  const int X = D.X;
  if (X < -4 || X >= 6) {
    out[n++] = dg[0];
    if (nd > 1) {
      out[n++] = '.';
      for (int i = 1; i < nd; i++) out[n++] = dg[i];
    }
    out[n++] = 'e';
    out[n++] = X < 0 ? '-' : '+';
    int ax = X < 0 ? -X : X;
    if (ax >= 100) {
      out[n++] = (char)('0' + ax / 100);
      ax %= 100;
    }
    out[n++] = (char)('0' + ax / 10);
    out[n++] = (char)('0' + ax % 10);
    return n;
  }
  if (X >= 0) {
    for (int i = 0; i <= X; i++) out[n++] = dg[i];
    if (nd > X + 1) {
      out[n++] = '.';
      for (int i = X + 1; i < nd; i++) out[n++] = dg[i];
    }
    return n;
  }
  out[n++] = '0';
  out[n++] = '.';
  for (int i = 0; i < -X - 1; i++) out[n++] = '0';
  for (int i = 0; i < nd; i++) out[n++] = dg[i];
  return n;
}

// printf("%g", d) at the default precision 6; out needs 24 bytes; returns the length
TN_HD int fmt_g(double d, char *out)
{
  int n = 0;
  const uint64_t b = TBITS(d);
  if (b >> 63) out[n++] = '-';
  const uint64_t a = b & 0x7FFFFFFFFFFFFFFFull;
  if (a > 0x7FF0000000000000ull) {
    out[n++] = 'n'; out[n++] = 'a'; out[n++] = 'n';
    return n;
  }
  if (a == 0x7FF0000000000000ull) {
    out[n++] = 'i'; out[n++] = 'n'; out[n++] = 'f';
    return n;
  }
  if (a == 0) {
    out[n++] = '0';
    return n;
  }
  return n + fmt_dec(decimal6(TDBL(a)), out + n);
}

// length of fmt_dec's text for digits D
TN_HD int dec_len(const Dec &D)
{
  uint32_t q = D.q;
  int nd = 6;
  while (nd > 1 && q % 10u == 0) {
    q /= 10u;
    nd--;
  }
  const int X = D.X;
  if (X < -4 || X >= 6) return nd + (nd > 1 ? 1 : 0) + 2 + ((X <= -100 || X >= 100) ? 3 : 2);
  if (X >= 0) return nd > X + 1 ? nd + 1 : X + 1;
  return 2 + (-X - 1) + nd;
}

// length of printf("%g", d) without building the text (the same rules as fmt_g)
TN_HD int fmt_g_len(double d)
{
  const uint64_t b = TBITS(d);
  const int neg = (int)(b >> 63);
  const uint64_t a = b & 0x7FFFFFFFFFFFFFFFull;
  if (a >= 0x7FF0000000000000ull) return neg + 3;  // nan, inf
  if (a == 0) return neg + 1;
  return neg + dec_len(decimal6(TDBL(a)));
}

// decimal digits of a non-negative integer below 10^18; returns the length
TN_HD int fmt_long(long v, char *out)
{
  char t[24];
  int n = 0;
  unsigned long u = v < 0 ? (unsigned long)(-(v + 1)) + 1ul : (unsigned long)v;
  do {
    t[n++] = (char)('0' + u % 10u);
    u /= 10u;
  } while (u);
  int k = 0;
  if (v < 0) out[k++] = '-';
  while (n) out[k++] = t[--n];
  return k;
}

}  // namespace tn93
