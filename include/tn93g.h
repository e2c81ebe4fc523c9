/*
 * tn93g.h -- C ABI of the B200 all-pairs TN93 engine (libtn93g.so).
 *
 * The reference (swifttn93, a drop-in for tn93 v1.1.0) has no plugin or FFI layer: its pair engine is linked
 * into main (solver/swifttn93.cpp:2299-2301) and consumes the parsed alignment (struct SeqSet,
 * solver/swifttn93.cpp:140-147) plus the scalar options of args_t (solver/argparse.hpp:41-65). This header is
 * that seam made explicit: the command-line front end parses options and FASTA on the host exactly as tn93
 * does, hands the codes to the engine, and receives the distance file bytes (in row order, through a
 * callback) and the numbers of the JSON summary. Plain pointers and sizes only; no CUDA or C++ types.
 *
 * Errors: every function returns TN93G_OK (0) or a negative TN93G_E* code; tn93g_strerror names it. Nothing
 * here exits the process. Threading: one host thread uses a context at a time.
 */
#ifndef TN93G_H
#define TN93G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TN93G_OK 0
#define TN93G_EINVAL (-1)   /* bad argument (null pointer, bad size, bad option value) */
#define TN93G_ECUDA (-2)    /* a CUDA runtime call failed (see tn93g_last_cuda_error) */
#define TN93G_ENOMEM (-3)   /* device or pinned host memory exhausted, or over the context's HBM budget */
#define TN93G_ESINK (-4)    /* the output callback returned non-zero */
#define TN93G_ENODEV (-5)   /* no usable CUDA device */
#define TN93G_ETIMEOUT (-6) /* a bounded device wait gave up (device error word set) */
#define TN93G_ETOOBIG (-7)  /* alignment too long for the 32-bit x16 count lanes (L >= 2^25) */
#define TN93G_ESCRATCH (-8) /* input beyond the fixed limits of tn93g_pair_distances_noalloc */
#define TN93G_EFASTA (-9)   /* tn93g_read_fasta refused the file (tn93's message is returned with it) */
#define TN93G_EUNDECIDED (-10) /* a printed distance or decision could not be made exact (see tn93g_summary) */

/* Fault injection for tests of the bounded device waits (tn93g_inject_fault). */
#define TN93G_FAULT_NONE 0
#define TN93G_FAULT_SKIP_FILL 1 /* the first tile of the next run's tensor-core count launch never receives its
                                   first operand stage, so its bounded wait runs out (TN93G_ETIMEOUT) */

/* Ambiguity modes, numbered as tn93's RESOLVE/AVERAGE/SKIP/GAPMM/SUBSET (solver/refkernel.h:14-18). */
#define TN93G_RESOLVE 0
#define TN93G_AVERAGE 1
#define TN93G_SKIP 2
#define TN93G_GAPMM 3
#define TN93G_SUBSET 4

/* Output formats, numbered as tn93's format_t (solver/argparse.hpp:25-30). */
#define TN93G_CSV 0
#define TN93G_CSVN 1
#define TN93G_HYPHY 2

/* Options of one run; the fields are args_t's (solver/argparse.hpp:46-63) after main's derivations
 * (solver/swifttn93.cpp:2256-2257, 2275-2294). */
typedef struct tn93g_opts {
  int mode;                    /* TN93G_RESOLVE .. TN93G_SUBSET (-a) */
  double threshold;            /* -t: a pair is reported when min_distance <= d <= threshold */
  double min_distance;         /* -w (default -1e-10) */
  double resolve_fraction;     /* -g (default 1.0) */
  long min_overlap;            /* -l, as the long tn93 passes to computeTN93 */
  int format;                  /* TN93G_CSV, TN93G_CSVN or TN93G_HYPHY (-f) */
  char delimiter;              /* -D (default ',') */
  int report_self;             /* -0, already combined with "one input file and not -c" */
  int count_only;              /* -c: no pair lines, only counts */
  int do_fst;                  /* -m with a second file: all pairs over both files, three histograms */
  unsigned char subset[18];    /* -a LIST: codes (index in "ACGTURYSWKMBDHVN?-") resolved under SUBSET */
} tn93g_opts;

/* Receives the distance file in order, in chunks (the header line is the caller's). The bytes are valid only
 * during the call. Return 0 to continue, non-zero to abort the run with TN93G_ESINK. */
typedef int (*tn93g_sink)(void *user, const char *bytes, size_t n);

/* The numbers of tn93's JSON summary (solver/swifttn93.cpp:2327-2330, 2914-2958). mean[] and weighted[] are
 * the row-ordered sums, not yet divided; the caller prints them with tn93's own iostream statements. */
typedef struct tn93g_summary {
  unsigned long pairwise;         /* Total comparisons possible */
  long skipped;                   /* pairs below the overlap (-l) */
  long links;                     /* weighted count of reported pairs */
  double max[3], mean[3], weighted[3];
  unsigned long hist[3][200];
  /* engine counters */
  long pairs_replayed;            /* pairs that took the site-order (non-dyadic) path */
  long logs_ambiguous;            /* pairs with a logarithm inside the C library's rounding band */
  long undecided;                 /* pairs whose printed bytes or decisions still depend on that rounding (0 unless
                                     the run failed with TN93G_EUNDECIDED) */
  size_t output_bytes;
  long logs_resolved;             /* pairs finished with the C library's own logarithms: those whose bytes or
                                     decisions depended on its rounding, and, when the JSON numbers needed it
                                     (sums_repass), every pair with an ambiguous logarithm */
  int sums_repass;                /* 1 when the maximum and means came from that second, exact pass */
  /* per histogram bin (units of a row band's partial sums): over the pairs with an ambiguous logarithm, the
   * largest low and largest high candidate distance, the sum of (high - low) x copy weight, and their number;
   * tn93g_summary_certified turns these into a certificate of the printed JSON numbers */
  double amb_bounds[3][4];
} tn93g_summary;

typedef struct tn93g_ctx tn93g_ctx;
typedef struct tn93g_set tn93g_set;

/* Creates a context on CUDA device `device`. hbm_budget (bytes, 0 = no limit) caps the engine's device
 * allocations. Replaces: Engine construction and its buffers (solver/swifttn93.cpp:490-569). */
int tn93g_create(tn93g_ctx **out, int device, size_t hbm_budget);
void tn93g_destroy(tn93g_ctx *ctx);
const char *tn93g_strerror(int code);
/* the message of the last failed CUDA call in this context */
const char *tn93g_last_cuda_error(tn93g_ctx *ctx);

/* Uploads an alignment: N sequences of L codes (0..17, the index of the character in "ACGTURYSWKMBDHVN?-",
 * as read_fasta produces them, solver/swifttn93.cpp:292-406), row-major; copy numbers (>= 1, or as tn93
 * parsed them); names as one byte buffer with per-sequence offsets and lengths (not NUL-terminated).
 * The caller keeps ownership of its buffers; they may be freed when the call returns.
 * Replaces: the SeqSet handed to Engine::prepare (solver/swifttn93.cpp:140-147, 2300). */
int tn93g_upload(tn93g_ctx *ctx, tn93g_set **out, const uint8_t *codes, long N, long L, const long *copy_counts,
                 const char *names, const size_t *name_off, const long *name_len);
void tn93g_free_set(tn93g_ctx *ctx, tn93g_set *set);

/* All pairs of one uploaded set. n1 = number of sequences that came from the first file (n1 = N for one file).
 * When n1 < N and !opts->do_fst, only the cross pairs (rows 0..n1-1 against columns n1..N-1) are computed,
 * as tn93's -s mode does (solver/swifttn93.cpp:2321-2322, 2392). The distance file (after the header line)
 * is delivered to sink in order; the summary is written to *out.
 * Replaces: the pair loop, its reductions and writer (solver/swifttn93.cpp:2339-2866). */
int tn93g_run(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, tn93g_sink sink, void *user,
              tn93g_summary *out);

/* The same run with the distance file left in device memory instead of being copied to the host: *dev_out
 * (device pointer owned by the context, valid until the next run or tn93g_destroy) receives *nbytes bytes.
 * For consumers that post-process on the GPU, and to time the engine with its inputs and outputs in HBM. */
int tn93g_run_to_device(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, void **dev_out,
                        size_t *nbytes, tn93g_summary *out);

/* The context's CUDA stream (a cudaStream_t), on which every kernel and copy of a run is issued. */
void *tn93g_stream(tn93g_ctx *ctx);

/* Number of kernel launches of the last run. */
long tn93g_last_launches(tn93g_ctx *ctx);

/* Device time of the last run's stages in milliseconds (CUDA events on the engine's stream):
 * [0] pack, [1] pair stage, [2] site-order replay, [3] row reductions, [4] output formatting,
 * [5] device->host copies, [6] whole run, [7] the tensor-core count kernel (part of [1]; 0 on the popcount
 * path). Returns the number of entries written (<= n). */
int tn93g_last_timings(tn93g_ctx *ctx, double *ms, int n);

/* Selects how the pair stage counts clean-site base combinations in tn93g_run / tn93g_run_rows: 0 = AND/XOR + POPC
 * over bit planes on the CUDA cores, 1 = one-hot INT8 matrix products on the tensor cores (tcgen05.mma kind::i8,
 * counts in tensor memory; the default, measured faster). Both give the same integers, so every output is
 * identical; the environment variable TN93G_COUNT=popc selects 0 when a context is created. Replaces: nothing
 * (the reference has one CPU counting path). */
int tn93g_set_count_path(tn93g_ctx *ctx, int path);

/* ---- row bands (one alignment split over several GPUs) ----
 * tn93g_run restricted to the rows [row_begin, row_end) of the pair triangle (pairs (i, j > i) with i in the
 * range; under -s the rows of the first file): the sink receives those rows' lines in order, the summary covers
 * those pairs only (its mean and weights are the rows' sums added in row order from 0), and row_sums, when not
 * NULL, receives 6 doubles per row: the row's sums for bins 0-2, then its weights for bins 0-2. Concatenating the
 * texts of consecutive bands and adding all bands' row sums in row order gives tn93g_run's bytes and summary
 * exactly (integer counts and histograms add, maxima take the maximum). -f hyphy (one matrix over all pairs) is
 * refused with TN93G_EINVAL. Replaces: the row range of swifttn93.cpp:2322, 2354, 2384 (one process runs every
 * row there). */
int tn93g_run_rows(tn93g_ctx *ctx, const tn93g_set *set, long n1, const tn93g_opts *opts, long row_begin,
                   long row_end, tn93g_sink sink, void *user, double *row_sums, tn93g_summary *summary);

/* An alignment in host memory: n sequences of length L, codes 0..17 in the order "ACGTURYSWKMBDHVN?-" (row-major),
 * copy numbers, and names (name k is names[name_off[k] .. name_off[k] + name_len[k])). */
typedef struct tn93g_alignment {
  uint8_t *codes;
  long n, L;
  long *copy_counts;
  char *names;
  size_t *name_off;
  long *name_len;
} tn93g_alignment;

/* Receives the whole distance file body of query (or batch alignment) number `query` (bytes valid only during the
 * call); non-zero aborts the call with TN93G_ESINK. */
typedef int (*tn93g_query_sink)(void *user, int query, const char *bytes, size_t n);

/* ---- batches of independent alignments ----
 * Runs K alignments (each with its own options; csv or csvn, no -m) in one pass: packing per alignment, one
 * persistent pair launch per kernel class over a queue of every alignment's tiles (longest alignments first), then
 * batched replay, statistics, sums, scan, per-alignment reduction and text. sink(user, k, bytes, n) receives
 * alignment k's whole distance file body and sums[k] its summary, exactly as tn93g_run on that alignment alone
 * would give them. rows_per_warp (NULL: 4) picks each alignment's pair-tile height (8 x 1, 2 or 4 rows by 32
 * columns) and pair_blocks (0: 2) the resident blocks per SM of the pair kernel (2 or 3); neither changes a result.
 * Replaces: one tn93 process per alignment (swifttn93.cpp:2222-2966 runs one file). */
int tn93g_batch_run(tn93g_ctx *ctx, int K, const tn93g_alignment *alignments, const tn93g_opts *opts,
                    const int *rows_per_warp, int pair_blocks, tn93g_query_sink sink, void *user,
                    tn93g_summary *sums);

/* ---- FASTA ----
 * tn93's reader (swifttn93.cpp:259-406) on a file held in memory: out receives malloc'ed codes (0..17 in the order
 * "ACGTURYSWKMBDHVN?-", row-major n x L), copy numbers (parsed after the last counts_sep), names and their offsets
 * and lengths, in the layout tn93g_upload takes. expect_len > 0 requires that sequence length (a second file, as
 * tn93 -s reads it after the first). On a refusal it returns TN93G_EFASTA with the message tn93 prints in msg.
 * Replaces: read_fasta (swifttn93.cpp:292-406), which tn93 runs on a FILE*. */
int tn93g_read_fasta(const char *bytes, size_t nbytes, long expect_len, char counts_sep, tn93g_alignment *out,
                     char *msg, size_t msg_cap);
void tn93g_alignment_free(tn93g_alignment *a);

/* FASTA ingest on the device: the work of tn93g_read_fasta followed by tn93g_upload, with the per-byte work on the
 * GPU. The host finds the records (names, and the byte range of each sequence up to the next '>' or '#') with
 * vectorised byte searches; the file's bytes go to the device once, where one kernel counts each sequence's letters
 * and another maps and compresses them, in file order, into the new set's codes. The same acceptance rules, checks
 * and messages as tn93g_read_fasta (TN93G_EFASTA, with the message in msg); expect_len > 0 requires that length.
 * On success *out is a set as tn93g_upload makes it, of *n_out sequences of *L_out columns.
 * Replaces: the byte map and compression of the FASTA reader, swifttn93.cpp:259-406 (345-369 in AVX-512). */
int tn93g_upload_fasta(tn93g_ctx *ctx, tn93g_set **out, const char *bytes, size_t nbytes, long expect_len,
                       char counts_sep, long *n_out, long *L_out, char *msg, size_t msg_cap);
/* The host half of tn93g_upload_fasta (its record scan and the reader's checks) with the letters counted on the
 * host: the same result and message as tn93g_upload_fasta without a device, for tests. Replaces: nothing in the
 * reference. */
int tn93g_fasta_check(const char *bytes, size_t nbytes, long expect_len, char counts_sep, long *n_out, long *L_out,
                      char *msg, size_t msg_cap);

/* ---- the -s mode as a service: a resident reference and batches of queries ----
 * A server keeps one reference alignment packed on the device and runs batches of query alignments against it.
 * Each query's result is exactly the distance file body and summary of `tn93 -s QUERY.fa REF.fa` with the
 * server's options: rows are the reference's sequences and columns the query's (swifttn93.cpp:2321-2322, 2392),
 * and csvn indices are global (reference first, then the query). Replaces: nothing in the reference, which reads
 * both files on every call (swifttn93.cpp:2243-2254); the per-query semantics are its -s mode. */
typedef struct tn93g_server tn93g_server;

/* Packs the reference (arguments as tn93g_upload) and allocates, within the context's HBM budget, every per-batch
 * buffer for batches of up to max_batch_sequences query sequences in up to max_batch_queries queries (about
 * 16 bytes per reference x query-sequence pair and 104 bytes per reference sequence x query); only the text
 * buffer grows later. opts->format must be csv or csvn; the server's options apply to every batch. */
int tn93g_server_create(tn93g_ctx *ctx, tn93g_server **out, const uint8_t *codes, long N, long L,
                        const long *copy_counts, const char *names, const size_t *name_off, const long *name_len,
                        const tn93g_opts *opts, long max_batch_sequences, int max_batch_queries);
/* Runs nq query alignments (each of the reference's length L, as tn93g_read_fasta returns them; at most the
 * server's capacity) in one batch; sums[q] receives query q's summary (its pairwise count is reference N x query
 * n; engine counters are reported in sums[0]). */
int tn93g_server_batch(tn93g_server *srv, int nq, const tn93g_alignment *queries, tn93g_query_sink sink, void *user,
                       tn93g_summary *sums);
/* Frees the server's device buffers; call it before tn93g_destroy of the server's context. */
void tn93g_server_destroy(tn93g_server *srv);

/* The JSON summary tn93 prints for one run (swifttn93.cpp:2914-2958), byte for byte; n2 = 0 and second_file = 0
 * for a single input file. Returns the length (the text is NUL-terminated when it fits in cap). */
size_t tn93g_summary_json(const tn93g_summary *s, unsigned long n1, unsigned long n2, int second_file, int fst,
                          char *buf, size_t cap);

/* 1 when every number tn93g_summary_json prints from s is the same for every way the C library's log may round
 * the ambiguous logarithms that s->amb_bounds describes; chain = the longest chain of additions behind a sum (the
 * longest row plus the number of rows). tn93g_run certifies its own summary (and makes a second, exact pass when
 * this fails); callers that merge row bands (tn93g_run_rows) call it on the merged summary, whose amb_bounds
 * combine the bands' (maximum of the largest candidates, sum of the spreads and counts). Replaces: nothing (the
 * reference computes every logarithm with the C library). */
int tn93g_summary_certified(const tn93g_summary *s, long chain, int fst);

/* ---- exactness and failure-detection knobs (tests and diagnostics) ----
 * tn93g_set_log_band: the rounding band (in ulps, kLogBand = 0.03 to 0.5) within which a logarithm counts as
 * ambiguous, and the distance of its other candidate (1 ulp, or more to exaggerate it). Widening them drives pairs
 * through the undecided path; every result stays exact. Defaults also from TN93G_LOG_BAND / TN93G_LOG_SPREAD.
 * tn93g_set_exact_sums: when on, every pair with an ambiguous logarithm is finished with the C library's log, so
 * the sums need no certificate (row bands whose merged summary failed tn93g_summary_certified run again so).
 * tn93g_set_wait_limit: the limit of each bounded device wait, in seconds (default 0.2).
 * tn93g_inject_fault: TN93G_FAULT_* for the next run only. Replaces: nothing in the reference. */
int tn93g_set_log_band(tn93g_ctx *ctx, double band_ulps, double spread_ulps);
int tn93g_set_exact_sums(tn93g_ctx *ctx, int on);
int tn93g_set_wait_limit(tn93g_ctx *ctx, double seconds);
int tn93g_inject_fault(tn93g_ctx *ctx, int fault);

/* Self-test of the device formula's division scheme (tests). n random pairs of counts go through the formula up
 * to its logarithms on the device and on the host (IEEE division), and n random quotients x / b through the
 * device's reciprocal-sharing division against its own correctly rounded division. mismatches[0] receives the
 * formula inputs whose results differ in any bit, mismatches[1] the quotients. Replaces: nothing in the
 * reference. */
int tn93g_selftest_division(tn93g_ctx *ctx, long n, unsigned long long seed, long mismatches[2]);

/* Allocation-free pair distances. This entry point has no counterpart in the reference; it exists for callers
 * that cannot allocate device memory: plugin hosts whose own allocator owns the whole device (a second
 * allocator would fail or fragment it), and latency-critical loops that must not enter the driver's allocator.
 * It runs the same pack, pair and site-order replay kernels as tn93g_run on one alignment, but every
 * intermediate buffer lives in one fixed array inside this library (about 16 MB of device memory, held on
 * every GPU that loads the library until the process exits), so it calls no cudaMalloc, cudaFree or other
 * allocating routine. Limits: N <= 512 sequences, L <= 4096 columns; larger inputs return TN93G_ESCRATCH.
 *   d_codes  device pointer, N x L codes 0..17 (row-major), the caller's
 *   d_dist   device pointer, N x N doubles (row-major), the caller's; for every j > i, d_dist[i*N + j] receives
 *            the raw distance of pair (i, j) as tn93g_run computes it (before tn93's "<= 0 -> 0"), or the bit
 *            pattern 0x7FF4000000000BAD for a pair below the overlap (-l); other entries are not written
 *   stream   a cudaStream_t, or NULL for the default stream
 * Each call copies a few small arrays between host and device to plan its launches and synchronises the given
 * stream before it returns. The first call on a device (with that device current) also looks up the array's
 * device address and writes its logarithm table into it. All calls share the array and it keeps the last
 * call's contents (each call clears what must start at zero), so two calls whose GPU work overlaps would race:
 * the library serialises calls from one process with a lock and returns only after the stream has drained; do
 * not overlap them by other means. */
int tn93g_pair_distances_noalloc(const uint8_t *d_codes, long N, long L, const tn93g_opts *opts, double *d_dist,
                                 void *stream);
/* message of the last failed tn93g_pair_distances_noalloc call made by the calling thread ("" after a success) */
const char *tn93g_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TN93G_H */
