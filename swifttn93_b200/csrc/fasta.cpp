// fasta.cpp -- tn93's FASTA reader as a library call (the acceptance rules and messages of swifttn93.cpp:259-406):
// '>' or '#' opens a record whose name runs to the end of the line; sequence bytes map through the alphabet
// "ACGTURYSWKMBDHVN?-" case-insensitively and every other byte is dropped; a record ends at the next '>' or '#';
// every sequence must have the first one's length; the copy number is the integer after the last separator that
// is neither the name's first nor its last character (at least 1). Shared by the command line and the
// resident-reference server, so a query file is accepted or refused exactly as tn93 -s would.
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "tn93g.h"

namespace {

struct CodeMap {
  signed char v[256];
  CodeMap()
  {
    static const char kValid[] = "ACGTURYSWKMBDHVN?-";
    for (int c = 0; c < 256; c++) {
      v[c] = -1;
      const int u = (c >= 'a' && c <= 'z') ? c - 32 : c;
      if (!u) continue;
      const char *f = strchr(kValid, u);
      if (f) v[c] = (signed char)(f - kValid);
    }
  }
};
const CodeMap kMap;

struct Reader {
  uint8_t *codes = nullptr;  // every input byte may be a code: sized to the input, written through a pointer
  size_t ncodes = 0;
  ~Reader() { free(codes); }
  std::vector<char> names;
  std::vector<size_t> name_off;
  std::vector<long> name_len, counts;
};

template <class T>
T *dup(const std::vector<T> &v)
{
  T *p = (T *)malloc(v.size() * sizeof(T) + 1);
  if (p && !v.empty()) memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

}  // namespace

extern "C" int tn93g_read_fasta(const char *bytes, size_t nbytes, long expect_len, char counts_sep,
                                tn93g_alignment *out, char *msg, size_t msg_cap)
{
  if (!out || (!bytes && nbytes)) return TN93G_EINVAL;
  memset(out, 0, sizeof *out);
  std::string err;
  Reader A;
  A.codes = (uint8_t *)malloc(nbytes + 1);
  if (!A.codes) return TN93G_ENOMEM;
  long N = 0, first_len = expect_len > 0 ? expect_len : 0;
  const bool have_len = expect_len > 0;
  const unsigned char *p = (const unsigned char *)bytes, *end = p + nbytes;
  int state = 0;
  size_t seq_begin = 0;
  auto close_sequence = [&]() -> bool {
    const long len = (long)(A.ncodes - seq_begin);
    if (N == 0 && !have_len) {
      first_len = len;
      if (first_len <= 0) {
        err = "First sequence length must be positive.\n";
        return false;
      }
    } else if (len != first_len) {
      err = "All sequences must have the same length (" + std::to_string(first_len) + "), but sequence '" +
            std::string(A.names.data() + A.name_off.back()) + "' had length " + std::to_string(len);
      return false;
    }
    N++;
    return true;
  };
  bool ok = true;
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
      const size_t begin = A.names.size();
      A.names.insert(A.names.end(), p, q);
      if (q == end) {
        p = q;
        break;
      }
      p = q + 1;
      const long len = (long)(A.names.size() - begin);
      A.names.push_back('\0');
      if (len <= 0) {
        err = "Sequence names must be non-empty.\n";
        ok = false;
        break;
      }
      unsigned long count = 1;
      if (len >= 3) {
        const char *nm = A.names.data() + begin;
        long k = len - 2;
        while (k >= 1 && nm[k] != counts_sep) k--;
        if (k >= 1) count = (unsigned long)(long)(int)strtol(nm + k + 1, nullptr, 10);
        if (count < 1) count = 1;
      }
      A.counts.push_back((long)count);
      A.name_off.push_back(begin);
      A.name_len.push_back(len);
      state = 2;
      seq_begin = A.ncodes;
      continue;
    }
    uint8_t *dst = A.codes + A.ncodes;
    while (p < end) {
      const signed char v = kMap.v[*p];
      if (v >= 0) {
        *dst++ = (uint8_t)v;
        p++;
        continue;
      }
      if (*p == '>' || *p == '#') break;
      p++;
    }
    A.ncodes = (size_t)(dst - A.codes);
    if (p == end) break;
    p++;
    if (!close_sequence()) {
      ok = false;
      break;
    }
    state = 1;
  }
  if (ok) {
    if (state == 2)
      ok = close_sequence();
    else {
      err = "Unexpected end of file: state " + std::to_string(state) + "\n";
      ok = false;
    }
  }
  if (!ok) {
    if (msg && msg_cap) {
      const size_t k = err.size() < msg_cap ? err.size() : msg_cap - 1;
      memcpy(msg, err.data(), k);
      msg[k] = 0;
    }
    return TN93G_EFASTA;
  }
  if (msg && msg_cap) msg[0] = 0;
  if (A.names.empty()) A.names.push_back('\0');
  out->n = N;
  out->L = first_len;
  out->codes = A.codes;  // the input-sized buffer (its first n x L bytes are the codes)
  A.codes = nullptr;
  out->copy_counts = dup(A.counts);
  out->names = dup(A.names);
  out->name_off = dup(A.name_off);
  out->name_len = dup(A.name_len);
  if (!out->codes || !out->copy_counts || !out->names || !out->name_off || !out->name_len) {
    tn93g_alignment_free(out);
    return TN93G_ENOMEM;
  }
  return TN93G_OK;
}

extern "C" void tn93g_alignment_free(tn93g_alignment *a)
{
  if (!a) return;
  free(a->codes);
  free(a->copy_counts);
  free(a->names);
  free(a->name_off);
  free(a->name_len);
  memset(a, 0, sizeof *a);
}
