// cli.cpp -- the tn93 v1.1.0 command line on top of the B200 engine (libtn93g.so).
//
// Host side, as in the reference: option parsing with tn93's semantics and messages (argparse.cpp:20-446),
// the FASTA reader (tn93g_read_fasta, swifttn93.cpp:259-406), the unsupported-option
// guard (swifttn93.cpp:2226-2233), the header line (swifttn93.cpp:2307-2316) and the JSON summary printed
// with the same iostream statements as tn93 (swifttn93.cpp:2900-2963), so the bytes on stdout match. The
// pair engine, its reductions and the distance-file text run on the GPU through include/tn93g.h.
#include <ctype.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <iomanip>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "tn93g.h"

namespace {

const char kValid[] = "ACGTURYSWKMBDHVN?-";

const char kUsage[] =
    "usage: tn93 [-h] [-v] [-o OUTPUT] [-t THRESHOLD] [-w MIN_THRESHOLD] [-a AMBIGS] [-g FRACTION] [-l OVERLAP] "
    "[-d COUNTS_IN_NAME] [-f FORMAT] [-s SECOND_FASTA] [-b] [-r] [-c] [-n] [-0] [-q] [-H] [-S] [-D DELIMITER][FASTA]\n";

// tn93's help text after the usage line (argparse.cpp:41-100), printed by -h and --help; kept byte for byte, since
// callers compare the command line's output with tn93's
const char kHelp[] =
    "compute Tamura Nei 93 distances between aligned sequences (version v1.1.0)\n"
    "\n"
    "optional arguments:\n"
    "  -h, --help               show this help message and exit\n"
    "  -v, --version            show tn93 version (v1.1.0)\n"
    "  -o OUTPUT                direct the output to a file named OUTPUT (default=stdout)\n"
    "  -t THRESHOLD             only report (count) distances below this threshold (>=0, default=0.015)\n"
    "  -w MINIMUM THRESHOLD     report distances above minimum threshold \n"
    "  -a AMBIGS                handle ambigous nucleotides using one of the following strategies (default=resolve)\n"
    "                           resolve: resolve ambiguities to minimize distance (e.g.R matches A);\n"
    "                           average: average ambiguities (e.g.R-A is 0.5 A-A and 0.5 G-A);\n"
    "                           skip: do not include sites with ambiguous nucleotides in distance calculations;\n"
    "                           gapmm: a gap ('-') matched to anything other than another gap is like matching an N (4-fold ambig) to it;\n"
    "                           a string (e.g. RY): any ambiguity in the list is RESOLVED; any ambiguitiy NOT in the list is averaged (LIST-NOT LIST will also be averaged);\n"
    "  -g FRACTION              in combination with AMBIGS, works to limit (for resolve and string options to AMBIG)\n"
    "                           the maximum tolerated FRACTION of ambiguous characters; sequences whose pairwise comparisons\n"
    "                           include no more than FRACTION [0,1] of sites with resolvable ambiguities will be resolved\n"
    "                           while all others will be AVERAGED (default = 1.0)\n"
    "  -f FORMAT                controls the format of the output unless -c is set (default=csv)\n"
    "                           csv: seqname1, seqname2, distance;\n"
    "                           csvn: 1, 2, distance;\n"
    "                           hyphy: {{d11,d12,..,d1n}...{dn1,dn2,...,dnn}}, where distances above THRESHOLD are set to 100;\n"
    "  -l OVERLAP               only process pairs of sequences that overlap over at least OVERLAP nucleotides (an integer >0, default=100):\n"
    "  -d COUNTS_IN_NAME        if sequence name is of the form 'somethingCOUNTS_IN_NAMEinteger' then treat the integer as a copy number\n"
    "                           when computing distance histograms (a character, default=':'):\n"
    "  -s SECOND_FASTA          if specified, read another FASTA file from SECOND_FASTA and perform pairwise comparison BETWEEN the files (default=NULL)\n"
    "  -b                       bootstrap alignment columns before computing distances (default = false)\n"
    "                           when -s is supplied, permutes the assigment of sequences to files\n"
    "                           interacts with -r option\n"
    "  -r                       if -b is specified AND -s is supplied, using -r will bootstrap across sites\n"
    "                           instead of allocating sequences to 'compartments' randomly\n"
    "  -c                       only count the pairs below a threshold, do not write out all the pairs \n"
    "  -n                       if set, do NOT write out headers for delimited files (default is to write) \n"
    "  -m                       compute inter- and intra-population means suitable for FST caclulations\n"
    "                           only applied when -s is used to provide a second file\n"
    "  -u PROBABILITY           subsample sequences with specified probability (a value between 0 and 1, default = 1.0)\n"
    "  -D DELIMITER             use this character as a delimiter in the output column-file (a character, default = ',')\n"
    "  -0                       report distances between each sequence and itself (as 0); this is useful to ensure every sequence\n"
    "                           in the input file appears in the output, e.g. for network construction to contrast clustered/unclustered\n"
    "  -q                       do not report progress updates and other diagnostics to stderr \n"
    "  -H                       use Hamming distance early exit to speed up distance calculations \n"
    "  -S, --subquadratic       perform subquadratic pairwise distance calculations (default = false)\n"
    "  FASTA                    read sequences to compare from this file (default=stdin)\n";

struct Options {
  FILE *out = stdout, *in1 = stdin, *in2 = nullptr;
  double distance = 0.015, min_distance = -1.e-10, resolve_fraction = 1.0, include_prob = 1.0;
  int ambig = TN93G_RESOLVE, format = TN93G_CSV;
  unsigned long overlap = 100;
  bool bootstrap = false, bootstrap2 = false, count = false, quiet = false, fst = false, no_header = false,
       report_self = false, hamming = false;
  char counts_sep = ':', delimiter = ',';
  std::string subset;
};

[[noreturn]] void fail(const char *fmt, ...)
{
  va_list ap;
  fprintf(stderr, "%stn93: error: ", kUsage);
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
  exit(1);
}

// tn93's parser: options are matched on their second character, every non-option argument but the last is
// an error, and the last one is the input FASTA (argparse.cpp:138-226)
Options parse(int argc, char **argv)
{
  Options o;
  auto value = [&](int &i) -> const char * {
    if (++i == argc) fail("ran out of command line arguments");
    return argv[i];
  };
  auto open_in = [&](const char *v, const char *what) -> FILE * {
    FILE *f = strcmp(v, "-") ? fopen(v, "rb") : stdin;
    if (!f) fail("failed to open the %s %s", what, v);
    return f;
  };
  for (int i = 1; i < argc; i++) {
    const char *a = argv[i];
    if (a[0] == '-' && a[1] == '-') {
      const char *l = a + 2;
      if (!strcmp(l, "help")) {
        fprintf(stderr, "%s\n%s", kUsage, kHelp);
        exit(1);
      } else if (!strcmp(l, "version")) {
        fprintf(stderr, "v1.1.0\n");
        exit(0);
      } else if (!strcmp(l, "hamming-skip"))
        o.hamming = true;
      else if (strcmp(l, "subquadratic"))
        fail("unknown argument: %s", a);
      continue;
    }
    if (a[0] != '-') {
      if (i != argc - 1) fail("unknown argument: %s", a);
      o.in1 = open_in(a, "INPUT file");
      if (o.in1 == o.in2) fail("input FASTA files must not both be stdin %s", a);
      continue;
    }
    const char *v;
    switch (a[1]) {
      case 'h':
        if (a[2]) fail("unknown argument: %s", a);
        fprintf(stderr, "%s\n%s", kUsage, kHelp);
        exit(1);
      case 'v': fprintf(stderr, "v1.1.0\n"); exit(0);
      case 'o':
        v = value(i);
        o.out = strcmp(v, "-") ? fopen(v, "wb") : stdout;
        if (!o.out) fail("failed to open the OUTPUT file %s", v);
        break;
      case 't':
        v = value(i);
        o.distance = atof(v);
        if (o.distance < 0.0) fail("genetic distance threshold must be >= 0, had: %s", v);
        break;
      case 'w':
        v = value(i);
        o.min_distance = atof(v);
        if (o.min_distance < 0.0 || o.min_distance > 1.0) fail("genetic minimum distance threshold must be >= 0, had: %s", v);
        break;
      case 'l':
        v = value(i);
        o.overlap = (unsigned long)(long)atoi(v);
        if (o.overlap == 0) fail("overlap must be positive, had: %s", v);
        break;
      case 'f':
        v = value(i);
        if (!strcmp(v, "csv"))
          o.format = TN93G_CSV;
        else if (!strcmp(v, "csvn"))
          o.format = TN93G_CSVN;
        else if (!strcmp(v, "hyphy"))
          o.format = TN93G_HYPHY;
        else
          fail("invalid output format: %s", v);
        break;
      case 'a':
        v = value(i);
        if (!strcmp(v, "resolve"))
          o.ambig = TN93G_RESOLVE;
        else if (!strcmp(v, "average"))
          o.ambig = TN93G_AVERAGE;
        else if (!strcmp(v, "skip"))
          o.ambig = TN93G_SKIP;
        else if (!strcmp(v, "gapmm"))
          o.ambig = TN93G_GAPMM;
        else {
          o.ambig = TN93G_SUBSET;
          o.subset = v;
        }
        break;
      case 's':
        v = value(i);
        o.in2 = open_in(v, "second INPUT file");
        if (o.in1 == o.in2) fail("input FASTA files must not both be stdin %s", v);
        break;
      case 'd':
        v = value(i);
        o.counts_sep = v[0];
        if (!isprint((unsigned char)o.counts_sep)) fail("count separator must be a printable character, had: %s", v);
        break;
      case 'u':
        v = value(i);
        o.include_prob = atof(v);
        if (o.include_prob < 0.0 || o.include_prob > 1.0) fail("sequence inclusion probability must be >= 0, had: %s", v);
        break;
      case 'D':
        v = value(i);
        if (strlen(v) != 1) fail("invalid output format: %s", v);
        o.delimiter = v[0];
        break;
      case 'b': o.bootstrap = true; break;
      case 'r': o.bootstrap2 = true; break;
      case 'c': o.count = true; break;
      case 'n': o.no_header = true; break;
      case 'q': o.quiet = true; break;
      case 'H': o.hamming = true; break;
      case 'S': break;
      case 'm': o.fst = true; break;
      case '0': o.report_self = true; break;
      case 'g':
        v = value(i);
        o.resolve_fraction = atof(v);
        if (o.resolve_fraction < 0.0 || o.resolve_fraction > 1.0) fail("resolve ambigous fraction must be >= 0, had: %s", v);
        break;
      default: fail("unknown argument: %s", a);
    }
  }
  return o;
}

// parsed alignment: codes 0..17 row-major, names, copy numbers
struct Alignment {
  std::vector<uint8_t> codes;
  std::vector<char> names;
  std::vector<size_t> name_off;
  std::vector<long> name_len, counts;
  long N = 0;
};

// Reads one FASTA with tn93's reader (tn93g_read_fasta) and appends it to A; every file after the first must
// have the first one's sequence length. Returns false after printing tn93's message (tn93 then exits with 1).
bool read_fasta(FILE *F, Alignment &A, long &first_len, char sep)
{
  std::vector<char> buf;
  {
    char tmp[1 << 16];
    size_t r;
    while ((r = fread(tmp, 1, sizeof tmp, F)) > 0) buf.insert(buf.end(), tmp, tmp + r);
  }
  tn93g_alignment R;
  char msg[512];
  const int rc = tn93g_read_fasta(buf.data(), buf.size(), A.N ? first_len : 0, sep, &R, msg, sizeof msg);
  if (rc != TN93G_OK) {
    std::cerr << (rc == TN93G_EFASTA ? msg : tn93g_strerror(rc));
    return false;
  }
  if (!A.N) first_len = R.L;
  const size_t base = A.names.size();
  size_t nb = 0;
  for (long k = 0; k < R.n; k++) nb = std::max(nb, R.name_off[k] + (size_t)R.name_len[k] + 1);
  A.names.insert(A.names.end(), R.names, R.names + nb);
  A.codes.insert(A.codes.end(), R.codes, R.codes + (size_t)R.n * R.L);
  for (long k = 0; k < R.n; k++) {
    A.name_off.push_back(base + R.name_off[k]);
    A.name_len.push_back(R.name_len[k]);
    A.counts.push_back(R.copy_counts[k]);
  }
  A.N += R.n;
  tn93g_alignment_free(&R);
  return true;
}

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// the distance file's sink: the text of each band, in order, with the time spent writing it
struct OutFile {
  FILE *f;
  double seconds = 0;
};

int write_sink(void *user, const char *bytes, size_t n)
{
  OutFile *o = (OutFile *)user;
  const double t0 = now_s();
  const bool ok = fwrite(bytes, 1, n, o->f) == n;
  o->seconds += now_s() - t0;
  return ok ? 0 : 1;
}

}  // namespace

int main(int argc, char **argv)
{
  const double t_start = now_s();
  Options o = parse(argc, argv);
  if (o.bootstrap || o.bootstrap2 || o.include_prob < 1.) {
    std::cerr << "swifttn93: -b, -r and -u (random resampling) are not supported" << std::endl;
    return 1;
  }
  if (o.hamming) {
    std::cerr << "swifttn93: -H (Hamming early exit) is not supported" << std::endl;
    return 1;
  }
  unsigned char subset[18] = {0};
  for (unsigned char ch : o.subset) {
    const char *f = strchr(kValid, toupper(ch));
    if (f && toupper(ch) && f - kValid > 3) subset[f - kValid] = 1;
  }
  // the device context is set up on a second thread while the input is parsed
  tn93g_ctx *ctx = nullptr;
  int rc = TN93G_OK;
  double t_ctx = 0;
  std::thread init([&] {
    const double t0 = now_s();
    rc = tn93g_create(&ctx, 0, 0);
    t_ctx = now_s() - t0;
  });
  struct Joiner {
    std::thread &t;
    ~Joiner()
    {
      if (t.joinable()) t.join();
    }
  } joiner{init};
  const double t_read0 = now_s();
  Alignment A;
  long L = 0;
  if (!read_fasta(o.in1, A, L, o.counts_sep)) return 1;
  const unsigned long n1 = (unsigned long)A.N;
  unsigned long n2 = 0;
  if (o.in2) {
    if (!read_fasta(o.in2, A, L, o.counts_sep)) return 1;
    n2 = (unsigned long)A.N - n1;
  }
  const double t_read = now_s() - t_read0;
  const bool fst = o.in2 && o.fst;
  const bool report_self = !o.in2 && o.report_self && !o.count;
  const unsigned long N = (unsigned long)A.N;
  const unsigned long pairwise = (o.in2 && !fst) ? n2 * n1 : (N - 1) * N / 2;
  if (!o.quiet) {
    if (!o.in2)
      std::cerr << "Read " << N << " sequences of length " << L << std::endl
                << "Will perform " << pairwise << " pairwise distance calculations";
    else {
      std::cerr << "Read " << n1 << " sequences from file 1 and " << n2 << " sequences from file 2 of length " << L
                << std::endl
                << "Will perform " << pairwise << " pairwise distance calculations";
      if (fst) std::cerr << ". Running in F_ST mode";
    }
  }
  if (o.format != TN93G_HYPHY && !o.count && !o.no_header) {
    if (o.format == TN93G_CSV)
      fprintf(o.out, "ID1%cID2%cDistance\n", o.delimiter, o.delimiter);
    else
      fprintf(o.out, "Seq1%cSeq2%cDistance\n", o.delimiter, o.delimiter);
  }
  const double t_wait0 = now_s();
  init.join();
  const double t_wait = now_s() - t_wait0;
  if (rc != TN93G_OK) {
    std::cerr << "tn93g: " << tn93g_strerror(rc) << std::endl;
    return 2;
  }
  tn93g_set *set = nullptr;
  if (A.names.empty()) A.names.push_back('\0');
  rc = tn93g_upload(ctx, &set, A.codes.data(), A.N, L, A.counts.data(), A.names.data(), A.name_off.data(),
                    A.name_len.data());
  if (rc != TN93G_OK) {
    std::cerr << "tn93g: " << tn93g_strerror(rc) << " " << tn93g_last_cuda_error(ctx) << std::endl;
    return 2;
  }
  tn93g_opts op;
  memset(&op, 0, sizeof op);
  op.mode = o.ambig;
  op.threshold = o.distance;
  op.min_distance = o.min_distance;
  op.resolve_fraction = o.resolve_fraction;
  op.min_overlap = (long)o.overlap;
  op.format = o.format;
  op.delimiter = o.delimiter;
  op.report_self = report_self;
  op.count_only = o.count;
  op.do_fst = fst;
  memcpy(op.subset, subset, sizeof subset);
  tn93g_summary S;
  OutFile of{o.out};
  const double t_run0 = now_s();
  rc = tn93g_run(ctx, set, (long)n1, &op, write_sink, &of, &S);
  const double t_run = now_s() - t_run0;
  if (rc != TN93G_OK) {
    // a run that could not make every printed byte exact fails loudly (exit 3), like any engine error (exit 2)
    std::cerr << "tn93g: " << tn93g_strerror(rc) << " " << tn93g_last_cuda_error(ctx) << std::endl;
    return rc == TN93G_EUNDECIDED ? 3 : 2;
  }
  const double t_free0 = now_s();
  tn93g_free_set(ctx, set);
  tn93g_destroy(ctx);
  fflush(o.out);
  const double t_free = now_s() - t_free0;
  if (getenv("TN93G_STATS")) {
    fprintf(stderr,
            "tn93g: replayed %ld, ambiguous-log pairs %ld, finished with the C library's log %ld, undecided %ld, "
            "exact-sums pass %d\n",
            S.pairs_replayed, S.logs_ambiguous, S.logs_resolved, S.undecided, S.sums_repass);
    fprintf(stderr,
            "tn93g: seconds: read %.3f, context %.3f (waited %.3f), run %.3f (writing %.3f), release %.3f, "
            "to here %.3f\n",
            t_read, t_ctx, t_wait, t_run, of.seconds, t_free, now_s() - t_start);
  }
  if (!o.quiet)
    std::cerr << std::endl << "Progress:" << std::setw(8) << 100. << "% (" << std::setw(8) << S.links
              << " links found, " << std::setw(12) << std::setprecision(3) << (double)pairwise << " evals)";
  std::cerr << std::endl;
  std::ostream *os = o.out == stdout ? &std::cerr : &std::cout;
  // tn93's summary (swifttn93.cpp:2914-2958), printed by the library's formatter
  {
    const size_t len = tn93g_summary_json(&S, o.in2 ? n1 : N, n2, o.in2 != nullptr, fst, nullptr, 0);
    std::string js(len + 1, '\0');
    tn93g_summary_json(&S, o.in2 ? n1 : N, n2, o.in2 != nullptr, fst, &js[0], js.size());
    os->write(js.data(), (std::streamsize)len);
    os->flush();
  }
  if (o.count)
    fprintf(o.out, "Found %ld links among %ld pairwise comparisons\n", S.links, (long)(pairwise - S.skipped));
  if (o.out != stdout) fclose(o.out);
  return 0;
}
