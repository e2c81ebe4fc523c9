/*
 * tn93_oracle.c -- TEST INFRASTRUCTURE ONLY. A plain-C restatement of the all-pairs TN93 path of
 * swifttn93 / tn93 v1.1.0, used as the CPU oracle by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py. Nothing in the product links, loads or calls this file.
 *
 * It is deliberately the slow, obvious form of the algorithm: every pair walks every alignment column
 * in site order and applies tn93's ambiguity semantics one site at a time, exactly as tn93's own
 * computeTN93 does, then evaluates the TN93 formula with the C library's log() and prints with printf.
 * Parity pins: tests/test_oracle.py checks this program byte for byte against the reference binary
 * built by oracle/build_ref.sh, and against the sha256 golden hashes the reference ships in
 * application/results/network.jsonl:1-5.
 *
 * Citations are to files of the reference (swifttn93 repository):
 *   CLI semantics        solver/argparse.cpp:138-446, solver/argparse.hpp:5-16
 *   FASTA reader         solver/swifttn93.cpp:259-406
 *   alphabet + tables    solver/refkernel.cpp:9-103
 *   ambiguity semantics  solver/refkernel.cpp:819-937
 *   per-pair walk        solver/refkernel.cpp:212-750 (site order, gap skipping, -g fallback)
 *   formula              solver/refkernel.cpp:752-815, solver/swifttn93.cpp:1954-2014
 *   row loop + output    solver/swifttn93.cpp:2222-2966
 *
 * Build: cc -O2 -fopenmp -ffp-contract=off -o tn93_oracle tn93_oracle.c -lm   (see oracle/Makefile)
 */
#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { M_RESOLVE = 0, M_AVERAGE = 1, M_SKIP = 2, M_GAPMM = 3, M_SUBSET = 4 };
enum { F_CSV = 0, F_CSVN = 1, F_HYPHY = 2 };
#define CODE_GAP 17
#define CODE_N 15
#define HBINS 200
#define MAX_DIST 1000.0

/* ------------------------------------------------------------------ alphabet (refkernel.cpp:9-51) */
static const char kValid[] = "ACGTURYSWKMBDHVN?-";
/* which of A,C,G,T each code stands for, and 1/(number of bases) (refkernel.cpp:19-51) */
static const int kRes[18][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}, {0, 0, 0, 1},
                                {1, 0, 1, 0}, {0, 1, 0, 1}, {0, 1, 1, 0}, {1, 0, 0, 1}, {0, 0, 1, 1},
                                {1, 1, 0, 0}, {0, 1, 1, 1}, {1, 0, 1, 1}, {1, 1, 0, 1}, {1, 1, 1, 0},
                                {1, 1, 1, 1}, {1, 1, 1, 1}, {0, 0, 0, 0}};
static double kResCount[18];
static signed char code_of[256];   /* validFlags[toupper(c)] */
static unsigned char resolve_these[18];

static void init_alphabet(const char *subset)
{
  for (int i = 0; i < 18; i++) {
    int n = kRes[i][0] + kRes[i][1] + kRes[i][2] + kRes[i][3];
    /* tn93 stores 1./2.f etc.: exact reciprocals 1, 1/2, 1/3 (as double), 1/4, and 0 for the gap */
    kResCount[i] = n == 0 ? 0.0 : (n == 3 ? 1.0 / 3.0f : 1.0 / (double)n);
  }
  signed char vf[256];
  for (int i = 0; i < 256; i++) vf[i] = -1;
  for (int i = 0; kValid[i]; i++) vf[(unsigned char)kValid[i]] = (signed char)i;
  for (int c = 0; c < 256; c++) code_of[c] = vf[(unsigned char)toupper(c)];
  memset(resolve_these, 0, sizeof resolve_these);
  if (subset)
    for (const char *p = subset; *p; p++) {
      int v = vf[(unsigned char)toupper((unsigned char)*p)];
      if (v > 3) resolve_these[v] = 1;
    }
}

/* ------------------------------------------------------------------ ambiguity handler (refkernel.cpp:819-937) */
typedef struct {
  double fc[4][4];
  long ic[4][4];
  unsigned long amb;
} Counts;

static void handle(unsigned c1, unsigned c2, int mode, Counts *C)
{
  if (mode == M_SKIP) return;
  if (c1 < 4) { /* c1 clean, c2 not */
    if (kResCount[c2] > 0.) {
      if ((mode == M_RESOLVE || (mode == M_SUBSET && resolve_these[c2])) && kRes[c2][c1]) {
        C->amb++;
        C->ic[c1][c1]++;
        return;
      }
      for (int b = 0; b < 4; b++)
        if (kRes[c2][b]) C->fc[c1][b] += kResCount[c2];
    }
    return;
  }
  if (c2 < 4) { /* c2 clean, c1 not */
    if (kResCount[c1] > 0.) {
      if ((mode == M_RESOLVE || (mode == M_SUBSET && resolve_these[c1])) && kRes[c1][c2]) {
        C->amb++;
        C->ic[c2][c2]++;
        return;
      }
      for (int a = 0; a < 4; a++)
        if (kRes[c1][a]) C->fc[a][c2] += kResCount[c1];
    }
    return;
  }
  /* both ambiguous */
  double norm = kResCount[c1] * kResCount[c2];
  if (!(norm > 0.0)) return;
  if (mode == M_RESOLVE || (mode == M_SUBSET && resolve_these[c1] && resolve_these[c2])) {
    C->amb++;
    int matched = 0, pm[4] = {0, 0, 0, 0};
    for (int b = 0; b < 4; b++)
      if (kRes[c1][b] && kRes[c2][b]) {
        matched++;
        pm[b] = 1;
      }
    if (matched > 0) {
      double v = 1. / matched;
      for (int b = 0; b < 4; b++)
        if (pm[b]) C->fc[b][b] += v;
      return;
    }
  }
  for (int a = 0; a < 4; a++)
    if (kRes[c1][a])
      for (int b = 0; b < 4; b++)
        if (kRes[c2][b]) C->fc[a][b] += norm;
}

/* ------------------------------------------------------------------ formula (refkernel.cpp:752-815) */
static double tn93_formula(const double nf[4], double diag, double ag_in, double ct_in)
{
  double s = nf[0] + nf[1] + nf[2] + nf[3];
  double tng = 2. / s, auxd = 1. / s, f[4], K1 = 0, K2 = 0, K3 = 0, dist;
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
    dist = (AG > 0. && CT > 0.) ? -0.5 * log(AG) - 0.25 * log(CT) : MAX_DIST;
  } else {
    AG = 1. - AG / K1 - 0.5 * tv / fR;
    CT = 1. - CT / K2 - 0.5 * tv / fY;
    tv = 1. - 0.5 * tv / fY / fR;
    dist = (AG > 0. && CT > 0. && tv > 0) ? -K1 * log(AG) - K2 * log(CT) - K3 * log(tv) : MAX_DIST;
  }
  return dist;
}

/* ------------------------------------------------------------------ one pair (refkernel.cpp:212-750)
 * Returns the raw distance (before the "<= 0 -> 0" clamp), or -1 for a pair below the overlap.
 * *computed is set when the distance formula ran (the histogram is updated only then). */
static double pair_distance(const unsigned char *s1, const unsigned char *s2, long L, int mode, long min_overlap,
                            double resolve_fraction, int *computed)
{
  Counts C;
  memset(&C, 0, sizeof C);
  for (long p = 0; p < L; p++) {
    unsigned c1 = s1[p], c2 = s2[p];
    if (c1 < 4 && c2 < 4) {
      C.ic[c1][c2]++;
      continue;
    }
    if (c1 == CODE_GAP || c2 == CODE_GAP) {
      /* a gap facing anything contributes nothing, except under gapmm where a gap facing a non-gap is an N */
      if (mode != M_GAPMM || (c1 == CODE_GAP && c2 == CODE_GAP)) continue;
      if (c1 == CODE_GAP)
        c1 = CODE_N;
      else
        c2 = CODE_N;
    }
    handle(c1, c2, mode, &C);
  }
  double tot = 0., nf[4] = {0., 0., 0., 0.};
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      double pc = (C.fc[a][b] += (double)C.ic[a][b]);
      tot += pc;
      nf[a] += pc;
      nf[b] += pc;
    }
  *computed = 0;
  if (tot <= min_overlap) return -1.;
  if ((mode == M_RESOLVE || mode == M_SUBSET) && resolve_fraction < 1. && tot * resolve_fraction <= C.amb)
    return pair_distance(s1, s2, L, M_AVERAGE, min_overlap, resolve_fraction, computed);
  *computed = 1;
  return tn93_formula(nf, C.fc[0][0] + C.fc[1][1] + C.fc[2][2] + C.fc[3][3], C.fc[0][2] + C.fc[2][0],
                      C.fc[1][3] + C.fc[3][1]);
}

/* ------------------------------------------------------------------ CLI (argparse.cpp:20-446) */
static const char kUsage[] =
    "usage: tn93 [-h] [-v] [-o OUTPUT] [-t THRESHOLD] [-w MIN_THRESHOLD] [-a AMBIGS] [-g FRACTION] [-l OVERLAP] "
    "[-d COUNTS_IN_NAME] [-f FORMAT] [-s SECOND_FASTA] [-b] [-r] [-c] [-n] [-0] [-q] [-H] [-S] [-D DELIMITER][FASTA]\n";

typedef struct {
  FILE *out, *in1, *in2;
  double distance, min_distance, resolve_fraction, include_prob;
  int ambig, format, boot, boot2, count, quiet, fst, no_header, self, hamming;
  unsigned long overlap;
  char counts_sep, delim;
  char *subset;
} Args;

static void die(const char *fmt, ...)
{
  va_list ap;
  fprintf(stderr, "%stn93: error: ", kUsage);
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
  exit(1);
}

static const char *next_arg(int *i, int argc, char **argv)
{
  if (++*i == argc) die("ran out of command line arguments");
  return argv[*i];
}

static void parse_args(Args *A, int argc, char **argv)
{
  memset(A, 0, sizeof *A);
  A->out = stdout;
  A->in1 = stdin;
  A->distance = 0.015;
  A->min_distance = -1.e-10;
  A->resolve_fraction = 1.0;
  A->include_prob = 1.0;
  A->overlap = 100;
  A->counts_sep = ':';
  A->delim = ',';
  for (int i = 1; i < argc; i++) {
    const char *a = argv[i];
    if (a[0] == '-' && a[1] == '-') {
      if (!strcmp(a + 2, "help")) {
        fprintf(stderr, "%s\n", kUsage);
        exit(1);
      } else if (!strcmp(a + 2, "version")) {
        fprintf(stderr, "v1.1.0\n");
        exit(0);
      } else if (!strcmp(a + 2, "hamming-skip"))
        A->hamming = 1;
      else if (!strcmp(a + 2, "subquadratic"))
        ;
      else
        die("unknown argument: %s", a);
    } else if (a[0] == '-') {
      const char *v;
      switch (a[1]) {
        case 'h':
          if (a[2]) die("unknown argument: %s", a);
          fprintf(stderr, "%s\n", kUsage);
          exit(1);
        case 'v': fprintf(stderr, "v1.1.0\n"); exit(0);
        case 'o':
          v = next_arg(&i, argc, argv);
          A->out = strcmp(v, "-") ? fopen(v, "wb") : stdout;
          if (!A->out) die("failed to open the OUTPUT file %s", v);
          break;
        case 't':
          v = next_arg(&i, argc, argv);
          A->distance = atof(v);
          if (A->distance < 0.0) die("genetic distance threshold must be >= 0, had: %s", v);
          break;
        case 'w':
          v = next_arg(&i, argc, argv);
          A->min_distance = atof(v);
          if (A->min_distance < 0.0 || A->min_distance > 1.0)
            die("genetic minimum distance threshold must be >= 0, had: %s", v);
          break;
        case 'l':
          v = next_arg(&i, argc, argv);
          A->overlap = (unsigned long)(long)atoi(v);
          if (A->overlap == 0) die("overlap must be positive, had: %s", v);
          break;
        case 'f':
          v = next_arg(&i, argc, argv);
          if (!strcmp(v, "csv"))
            A->format = F_CSV;
          else if (!strcmp(v, "csvn"))
            A->format = F_CSVN;
          else if (!strcmp(v, "hyphy"))
            A->format = F_HYPHY;
          else
            die("invalid output format: %s", v);
          break;
        case 'a':
          v = next_arg(&i, argc, argv);
          if (!strcmp(v, "resolve"))
            A->ambig = M_RESOLVE;
          else if (!strcmp(v, "average"))
            A->ambig = M_AVERAGE;
          else if (!strcmp(v, "skip"))
            A->ambig = M_SKIP;
          else if (!strcmp(v, "gapmm"))
            A->ambig = M_GAPMM;
          else {
            A->ambig = M_SUBSET;
            A->subset = strdup(v);
          }
          break;
        case 's':
          v = next_arg(&i, argc, argv);
          A->in2 = strcmp(v, "-") ? fopen(v, "rb") : stdin;
          if (!A->in2) die("failed to open the second INPUT file %s", v);
          if (A->in1 == A->in2) die("input FASTA files must not both be stdin %s", v);
          break;
        case 'd':
          v = next_arg(&i, argc, argv);
          A->counts_sep = v[0];
          if (!isprint((unsigned char)A->counts_sep)) die("count separator must be a printable character, had: %s", v);
          break;
        case 'u':
          v = next_arg(&i, argc, argv);
          A->include_prob = atof(v);
          if (A->include_prob < 0.0 || A->include_prob > 1.0)
            die("sequence inclusion probability must be >= 0, had: %s", v);
          break;
        case 'D':
          v = next_arg(&i, argc, argv);
          if (strlen(v) == 1)
            A->delim = v[0];
          else
            die("invalid output format: %s", v);
          break;
        case 'b': A->boot = 1; break;
        case 'r': A->boot2 = 1; break;
        case 'c': A->count = 1; break;
        case 'n': A->no_header = 1; break;
        case 'q': A->quiet = 1; break;
        case 'H': A->hamming = 1; break;
        case 'S': break;
        case 'm': A->fst = 1; break;
        case '0': A->self = 1; break;
        case 'g':
          v = next_arg(&i, argc, argv);
          A->resolve_fraction = atof(v);
          if (A->resolve_fraction < 0.0 || A->resolve_fraction > 1.0)
            die("resolve ambigous fraction must be >= 0, had: %s", v);
          break;
        default: die("unknown argument: %s", a);
      }
    } else if (i == argc - 1) {
      A->in1 = strcmp(a, "-") ? fopen(a, "rb") : stdin;
      if (!A->in1) die("failed to open the INPUT file %s", a);
      if (A->in1 == A->in2) die("input FASTA files must not both be stdin %s", a);
    } else
      die("unknown argument: %s", a);
  }
}

/* ------------------------------------------------------------------ FASTA (swifttn93.cpp:259-406) */
typedef struct {
  unsigned char *codes;
  size_t ncodes, cap;
  char **names;
  long *nlen, *counts;
  long N, ncap;
} Seqs;

static void push_code(Seqs *S, unsigned char c)
{
  if (S->ncodes == S->cap) {
    S->cap = S->cap ? 2 * S->cap : 4096;
    S->codes = (unsigned char *)realloc(S->codes, S->cap);
  }
  S->codes[S->ncodes++] = c;
}

static void finish_seq(Seqs *S, size_t begin, long *first_len)
{
  long len = (long)(S->ncodes - begin);
  if (S->N == 0) {
    *first_len = len;
    if (len <= 0) {
      fprintf(stderr, "First sequence length must be positive.\n");
      exit(1);
    }
  } else if (len != *first_len) {
    fprintf(stderr, "All sequences must have the same length (%ld), but sequence '%s' had length %ld", *first_len,
            S->names[S->N], len);
    exit(1);
  }
  S->N++;
}

/* returns 0 on success, 1 on a reader error (message printed) */
static int read_fasta(FILE *F, Seqs *S, long *first_len, char sep)
{
  size_t cap = 1 << 16, n = 0;
  unsigned char *buf = (unsigned char *)malloc(cap);
  for (;;) {
    if (n == cap) buf = (unsigned char *)realloc(buf, cap *= 2);
    size_t r = fread(buf + n, 1, cap - n, F);
    if (r == 0) break;
    n += r;
  }
  int state = 0;
  size_t begin = S->ncodes;
  const unsigned char *p = buf, *end = buf + n;
  while (p < end) {
    if (state == 0) {
      while (p < end && *p != '>' && *p != '#') p++;
      if (p == end) break;
      p++;
      state = 1;
      continue;
    }
    if (state == 1) {
      const unsigned char *q = p;
      while (q < end && *q != '\n' && *q != '\r') q++;
      if (S->N == S->ncap) {
        S->ncap = S->ncap ? 2 * S->ncap : 64;
        S->names = (char **)realloc(S->names, S->ncap * sizeof(char *));
        S->nlen = (long *)realloc(S->nlen, S->ncap * sizeof(long));
        S->counts = (long *)realloc(S->counts, S->ncap * sizeof(long));
      }
      long len = (long)(q - p);
      char *nm = (char *)malloc(len + 1);
      memcpy(nm, p, len);
      nm[len] = 0;
      S->names[S->N] = nm;
      S->nlen[S->N] = len;
      if (q == end) {
        p = q;
        break;
      }
      p = q + 1;
      if (len <= 0) {
        fprintf(stderr, "Sequence names must be non-empty.\n");
        free(buf);
        return 1;
      }
      /* copy number: digits after the last separator that is neither the first nor the last character */
      unsigned long count = 1;
      if (len >= 3) {
        long k;
        for (k = len - 2; k >= 1; k--)
          if (nm[k] == sep) break;
        if (k >= 1) count = (unsigned long)(long)(int)strtol(nm + k + 1, NULL, 10);
        if (count < 1) count = 1;
      }
      S->counts[S->N] = (long)count;
      state = 2;
      begin = S->ncodes;
      continue;
    }
    /* state 2: sequence bytes; other bytes are dropped; '>' or '#' starts the next record */
    while (p < end) {
      signed char v = code_of[*p];
      if (v >= 0) {
        push_code(S, (unsigned char)v);
        p++;
        continue;
      }
      if (*p == '>' || *p == '#') break;
      p++;
    }
    if (p == end) break;
    p++;
    finish_seq(S, begin, first_len);
    state = 1;
  }
  free(buf);
  if (state == 2) {
    finish_seq(S, begin, first_len);
    return 0;
  }
  fprintf(stderr, "Unexpected end of file: state %d\n", state);
  return 1;
}

/* ------------------------------------------------------------------ output helpers */
typedef struct {
  char *p;
  size_t n, cap;
} Buf;

static void bput(Buf *b, const char *s, size_t k)
{
  if (b->n + k > b->cap) {
    b->cap = (b->n + k) * 2 + 256;
    b->p = (char *)realloc(b->p, b->cap);
  }
  memcpy(b->p + b->n, s, k);
  b->n += k;
}

static void dump_hist(FILE *o, const char *tag, const unsigned long *h)
{
  if (tag)
    fprintf(o, "\t\"Histogram %s\" : [", tag);
  else
    fprintf(o, "\t\"Histogram\" : [");
  for (int k = 0; k < HBINS; k++) {
    if (k) fputc(',', o);
    fprintf(o, "[%g,%lu]", (k + 1.) / HBINS, h[k]);
  }
  fprintf(o, "]\n");
}

typedef struct {
  Buf out;
  double lsum[3], lw[3], lmax[3];
  long links, skipped;
  unsigned long hist[3][HBINS];
  long *hy_j;
  double *hy_d;
  long hy_n, hy_cap;
} Row;

/* ------------------------------------------------------------------ main (swifttn93.cpp:2222-2966) */
int main(int argc, char **argv)
{
  Args A;
  parse_args(&A, argc, argv);
  if (A.boot || A.boot2 || A.include_prob < 1.) {
    fprintf(stderr, "swifttn93: -b, -r and -u (random resampling) are not supported\n");
    return 1;
  }
  if (A.hamming) {
    fprintf(stderr, "swifttn93: -H (Hamming early exit) is not supported\n");
    return 1;
  }
  init_alphabet(A.subset);
  Seqs S;
  memset(&S, 0, sizeof S);
  long L = 0;
  if (read_fasta(A.in1, &S, &L, A.counts_sep)) return 1;
  unsigned long n1 = (unsigned long)S.N, n2 = 0;
  if (A.in2) {
    if (read_fasta(A.in2, &S, &L, A.counts_sep)) return 1;
    n2 = (unsigned long)S.N - n1;
  }
  /* test hook: TN93_ORACLE_DUMP=PATH writes the parsed alignment (name, copy number and codes of every sequence,
     one line each) to PATH and stops, so a reader can be compared with this one */
  const char *dump = getenv("TN93_ORACLE_DUMP");
  if (dump) {
    FILE *D = fopen(dump, "wb");
    if (!D) return 1;
    for (long i = 0; i < S.N; i++) {
      fprintf(D, "%s\t%ld\t", S.names[i], S.counts[i]);
      for (long k = 0; k < L; k++) fputc("ACGTURYSWKMBDHVN?-"[S.codes[(size_t)i * L + k]], D);
      fputc('\n', D);
    }
    fclose(D);
    return 0;
  }
  const int fst = A.in2 && A.fst, cross = A.in2 && !fst;
  const int report_self = !A.in2 && A.self && !A.count;
  const long N = S.N;
  unsigned long pairwise = cross ? n2 * n1 : (unsigned long)(N - 1) * (unsigned long)N / 2;
  if (!A.quiet) {
    if (!A.in2)
      fprintf(stderr, "Read %ld sequences of length %ld\nWill perform %lu pairwise distance calculations", N, L,
              pairwise);
    else {
      fprintf(stderr,
              "Read %lu sequences from file 1 and %lu sequences from file 2 of length %ld\nWill perform %lu pairwise "
              "distance calculations",
              n1, n2, L, pairwise);
      if (fst) fprintf(stderr, ". Running in F_ST mode");
    }
  }
  if (A.format != F_HYPHY && !A.count && !A.no_header) {
    if (A.format == F_CSV)
      fprintf(A.out, "ID1%cID2%cDistance\n", A.delim, A.delim);
    else
      fprintf(A.out, "Seq1%cSeq2%cDistance\n", A.delim, A.delim);
  }
  long upper = cross ? (long)n1 : N, row_b = 0;
  /* test hook: TN93_ORACLE_ROWS=B:E runs only the rows [B, E) of the pair triangle (a row band, as one rank of a
     sharded run computes it) and TN93_ORACLE_PARTIAL=PATH writes that band's counts, maxima, histograms and
     per-row sums (hex floats) to PATH, so the merge of bands can be checked against a whole run */
  const char *rows_env = getenv("TN93_ORACLE_ROWS");
  FILE *partial = NULL;
  if (rows_env) {
    long b = 0, e = 0;
    if (sscanf(rows_env, "%ld:%ld", &b, &e) != 2 || b < 0 || e < b || e > upper) return 1;
    row_b = b;
    upper = e;
    const char *pp = getenv("TN93_ORACLE_PARTIAL");
    if (pp) partial = fopen(pp, "wb");
    if (cross)
      pairwise = (unsigned long)(N - (long)n1) * (unsigned long)(e - b);
    else
      pairwise = (unsigned long)((e - b) * (2 * N - b - e - 1) / 2);
  }
  const int emit = !A.count, hy = A.format == F_HYPHY;
  double maxv[3] = {0, 0, 0}, mean[3] = {0, 0, 0}, wc[3] = {0, 0, 0};
  long links = 0, skipped = 0;
  unsigned long hist[3][HBINS];
  memset(hist, 0, sizeof hist);
  long **hyj = NULL;
  double **hyd = NULL;
  long *hyn = NULL, *hycap = NULL;
  if (hy && emit) {
    hyj = (long **)calloc(N, sizeof(long *));
    hyd = (double **)calloc(N, sizeof(double *));
    hyn = (long *)calloc(N, sizeof(long));
    hycap = (long *)calloc(N, sizeof(long));
  }
  const long BLK = 256;
  Row *rows = (Row *)calloc(BLK, sizeof(Row));
  for (long r0 = row_b; r0 < upper; r0 += BLK) {
    const long r1 = r0 + BLK < upper ? r0 + BLK : upper;
#pragma omp parallel for schedule(dynamic, 1)
    for (long i = r0; i < r1; i++) {
      Row *R = &rows[i - r0];
      R->out.n = 0;
      R->links = R->skipped = 0;
      R->hy_n = 0;
      memset(R->hist, 0, sizeof R->hist);
      for (int q = 0; q < 3; q++) R->lsum[q] = R->lw[q] = R->lmax[q] = 0.;
      const long c1 = S.counts[i];
      char tmp[512];
      if (!cross) {
        if (c1 > 1) {
          unsigned long svs = (unsigned long)(c1 * (c1 - 1L)) >> 1;
          int q = i < (long)n1 ? 0 : 1;
          R->lw[q] += svs;
          R->hist[q][0] += svs;
        }
        if (report_self) {
          if (A.format == F_CSV) {
            bput(&R->out, S.names[i], S.nlen[i]);
            bput(&R->out, &A.delim, 1);
            bput(&R->out, S.names[i], S.nlen[i]);
            bput(&R->out, &A.delim, 1);
            bput(&R->out, "0\n", 2);
          } else if (A.format == F_CSVN) {
            int k = snprintf(tmp, sizeof tmp, "%ld%c%ld%c0\n", i, A.delim, i, A.delim);
            bput(&R->out, tmp, k);
          }
        }
      }
      const long lb = cross ? (long)n1 : i + 1;
      for (long j = lb; j < N; j++) {
        int bin = 0;
        if (fst) {
          if (i < (long)n1) {
            if (j >= (long)n1) bin = 2;
          } else
            bin = 1;
        }
        const long w = c1 * S.counts[j];
        int computed = 0;
        double d = pair_distance(S.codes + i * L, S.codes + j * L, L, A.ambig, (long)A.overlap, A.resolve_fraction,
                                 &computed);
        double thisD = d;
        if (computed) {
          /* histogram index: floor(d * 200) as a long, clamped to the last bin as an unsigned value; NaN and
             out-of-range values convert to LONG_MIN on x86 (swifttn93.cpp:2003-2014) */
          double f = floor(d * 200.0);
          long idx = (f >= -9.2233720368547758e18 && f < 9.2233720368547758e18) ? (long)f : (long)0x8000000000000000UL;
          if ((unsigned long)idx >= (unsigned long)HBINS) idx = HBINS - 1;
          R->hist[bin][idx] += (unsigned long)w;
          thisD = d <= 0. ? 0. : d;
        }
        if (thisD >= A.min_distance && thisD <= A.distance) {
          R->links += w;
          if (emit) {
            if (A.format == F_CSV) {
              bput(&R->out, S.names[i], S.nlen[i]);
              bput(&R->out, &A.delim, 1);
              bput(&R->out, S.names[j], S.nlen[j]);
              int k = snprintf(tmp, sizeof tmp, "%c%g\n", A.delim, thisD);
              bput(&R->out, tmp, k);
            } else if (A.format == F_CSVN) {
              int k = snprintf(tmp, sizeof tmp, "%ld%c%ld%c%g\n", i, A.delim, j, A.delim, thisD);
              bput(&R->out, tmp, k);
            } else {
              if (R->hy_n == R->hy_cap) {
                R->hy_cap = R->hy_cap ? 2 * R->hy_cap : 16;
                R->hy_j = (long *)realloc(R->hy_j, R->hy_cap * sizeof(long));
                R->hy_d = (double *)realloc(R->hy_d, R->hy_cap * sizeof(double));
              }
              R->hy_j[R->hy_n] = j;
              R->hy_d[R->hy_n++] = thisD;
            }
          }
        }
        if (thisD <= -0.5)
          R->skipped += 1;
        else {
          R->lsum[bin] += thisD * (double)w;
          R->lw[bin] += (double)w;
          if (thisD > R->lmax[bin]) R->lmax[bin] = thisD;
        }
      }
    }
    /* rows in order: output, sums, links (swifttn93.cpp:2838-2853) */
    for (long i = r0; i < r1; i++) {
      Row *R = &rows[i - r0];
      if (R->out.n) fwrite(R->out.p, 1, R->out.n, A.out);
      links += R->links;
      skipped += R->skipped;
      for (int q = 0; q < 3; q++) {
        if (R->lmax[q] > maxv[q]) maxv[q] = R->lmax[q];
        mean[q] += R->lsum[q];
        wc[q] += R->lw[q];
        for (int k = 0; k < HBINS; k++) hist[q][k] += R->hist[q][k];
      }
      if (partial)
        fprintf(partial, "row %ld %a %a %a %a %a %a\n", i, R->lsum[0], R->lsum[1], R->lsum[2], R->lw[0], R->lw[1],
                R->lw[2]);
      for (long t = 0; t < R->hy_n; t++) {
        long js[2] = {i, R->hy_j[t]}, other[2] = {R->hy_j[t], i};
        for (int e = 0; e < 2; e++) {
          long r = js[e];
          if (hyn[r] == hycap[r]) {
            hycap[r] = hycap[r] ? 2 * hycap[r] : 16;
            hyj[r] = (long *)realloc(hyj[r], hycap[r] * sizeof(long));
            hyd[r] = (double *)realloc(hyd[r], hycap[r] * sizeof(double));
          }
          hyj[r][hyn[r]] = other[e];
          hyd[r][hyn[r]++] = R->hy_d[t];
        }
      }
    }
  }
  if (emit && hy) {
    /* tn93's -f hyphy matrix: 0 on the diagonal, the reported distance where linked, 100 elsewhere
       (swifttn93.cpp:2869-2897) */
    fputc('{', A.out);
    for (long r = 0; r < N; r++) {
      fputs("\n{", A.out);
      long li = 0;
      for (long c = 0; c < N; c++) {
        if (c) fputc(',', A.out);
        if (c == r)
          fputc('0', A.out);
        else if (li < hyn[r] && hyj[r][li] == c)
          fprintf(A.out, "%g", hyd[r][li++]);
        else
          fputs("100", A.out);
      }
      fputc('}', A.out);
    }
    fputs("\n}", A.out);
  }
  fflush(A.out);
  if (partial) {
    fprintf(partial, "pairwise %lu\nskipped %ld\nlinks %ld\nmax %a %a %a\n", pairwise, skipped, links, maxv[0], maxv[1],
            maxv[2]);
    for (int q = 0; q < 3; q++) {
      fprintf(partial, "hist%d", q);
      for (int k = 0; k < HBINS; k++) fprintf(partial, " %lu", hist[q][k]);
      fputc('\n', partial);
    }
    fclose(partial);
  }
  if (!A.quiet)
    fprintf(stderr, "\nProgress:%8g%% (%8ld links found, %12.3g evals)", 100., links, (double)pairwise);
  fprintf(stderr, "\n");
  FILE *js = A.out == stdout ? stderr : stdout;
  fprintf(js, "{\n");
  fprintf(js, "\t\"Actual comparisons performed\" :%lu,\n", pairwise - (unsigned long)skipped);
  fprintf(js, "\t\"Comparisons accounting for copy numbers \" :%g,\n", wc[0] + wc[1] + wc[2]);
  fprintf(js, "\t\"Total comparisons possible\" : %lu,\n", pairwise);
  fprintf(js, "\t\"Links found\" : %ld,\n", links);
  fprintf(js, "\t\"Maximum distance\" : %g,\n", maxv[0]);
  if (!A.in2)
    fprintf(js, "\t\"Sequences\" : %lu,\n", (unsigned long)N);
  else {
    fprintf(js, "\t\"Sequences in first file\" : %lu,\n", n1);
    fprintf(js, "\t\"Sequences in second file\" : %lu,\n", n2);
  }
  if (fst) {
    const char *keys[4] = {"File 1", "File 2", "Between", "Combined"};
    for (int k = 0; k < 3; k++) fprintf(js, "\t\"Mean distance %s\" : %g,\n", keys[k], mean[k] / wc[k]);
    double meta = (mean[0] + mean[1] + mean[2]) / (wc[0] + wc[1] + wc[2]);
    double intra = (mean[0] + mean[1]) / (wc[0] + wc[1]);
    double piD = mean[2] / wc[2] - intra;
    fprintf(js, "\t\"Mean distance [intra] \" : %g,\n", intra);
    fprintf(js, "\t\"Mean distance [combined]\" : %g,\n", meta);
    fprintf(js, "\t\"F_ST\" : %g,\n", piD / (intra + piD));
    for (int k = 0; k < 3; k++) {
      dump_hist(js, keys[k], hist[k]);
      fprintf(js, ",\n");
    }
    for (int k = 0; k < HBINS; k++) hist[0][k] += hist[1][k] + hist[2][k];
    dump_hist(js, keys[3], hist[0]);
  } else {
    fprintf(js, "\t\"Mean distance\" : %g,\n", mean[0] / wc[0]);
    dump_hist(js, NULL, hist[0]);
  }
  fprintf(js, "}\n");
  fflush(js);
  if (A.count) fprintf(A.out, "Found %ld links among %ld pairwise comparisons\n", links, (long)(pairwise - skipped));
  if (A.out != stdout) fclose(A.out);
  return 0;
}
