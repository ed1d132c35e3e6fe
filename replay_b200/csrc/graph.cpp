// Contact-file ingest and the device interval index.
//
// Replaces tool/temporal_contact_matrix.c (parse_edgelist_build_intervals
// :148-321, count_valid_edges :122-143, parse_iso8601_to_unix :95-120,
// get_or_create_node_index :328-356); the index itself is built on the
// device (ingest.cu).
//
// The file format and its acceptance rules are the reference's:
//  * line 1 starts with "NODE_LIST" + blank; its tokens are non-negative
//    base-10 ids without duplicates; N = token count;
//  * the contact lines a line-counting pass accepts with the pattern
//    " %d, %d, %63[^,], %63[^;];" bound the number of contacts; the parse
//    pass reads " %d , %d , %63[^,] , %63[^;\r\n] ;" and skips (and counts
//    as malformed) lines it cannot read; lines starting with '#' are
//    comments; lines are read in fgets chunks of at most 99,999 chars;
//  * timestamps are "%d-%d-%dT%d:%d:%d" in UTC with timegm's normalisation
//    of out-of-range fields; a timestamp equal to -1 rejects the line;
//  * node index = order of first appearance in contact lines.
// Lines of the exact form "id, id, YYYY-MM-DDTHH:MM:SSZ, YYYY-MM-DDTHH:MM:SSZ;"
// (what the network generator writes) are read at fixed offsets; other
// lines both patterns read alike take a hand-written scanning path; every
// other line goes through sscanf with the reference's two patterns.  The
// file is split into one range per thread.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "rp_internal.h"

namespace rp {
namespace {

constexpr size_t kFgetsChunk = 99999;  // fgets(buf, 100000, fp)

int64_t floor_div64(int64_t a, int64_t b) {
  int64_t q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return q;
}

// Proleptic Gregorian day number of y-m-d relative to 1970-01-01
// (H. Hinnant's days_from_civil).
int64_t days_from_civil(int64_t y, int64_t m, int64_t d) {
  y -= m <= 2;
  const int64_t era = (y >= 0 ? y : y - 399) / 400;
  const int64_t yoe = y - era * 400;
  const int64_t doy = (153 * (m > 2 ? m - 3 : m + 9) + 2) / 5 + d - 1;
  const int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + doe - 719468;
}

int64_t utc_seconds(int64_t year, int64_t month, int64_t day, int64_t hour,
                    int64_t minute, int64_t second) {
  const int64_t m0 = month - 1;
  const int64_t y = year + floor_div64(m0, 12);
  const int64_t m = m0 - floor_div64(m0, 12) * 12;
  return (days_from_civil(y, m + 1, 1) + day - 1) * 86400 + hour * 3600 +
         minute * 60 + second;
}

int64_t iso8601_slow(const char *s) {
  int year, month, day, hour, min, sec;
  char extra[10];
  if (sscanf(s, "%d-%d-%dT%d:%d:%d%9s", &year, &month, &day, &hour, &min, &sec,
             extra) < 6)
    return -1;
  return utc_seconds(year, month, day, hour, min, sec);
}

struct IdMap {
  std::vector<int32_t> keys, vals;
  std::vector<uint8_t> used;
  size_t mask = 0, count = 0;
  explicit IdMap(size_t expect) {
    size_t cap = 1024;
    while (cap < 2 * expect + 2) cap <<= 1;
    keys.resize(cap);
    vals.resize(cap);
    used.assign(cap, 0);
    mask = cap - 1;
  }
  static size_t h(int32_t k) {
    uint64_t x = (uint32_t)k * 0x9E3779B97F4A7C15ull;
    return (size_t)(x ^ (x >> 31));
  }
  void grow() {
    IdMap big(keys.size());
    for (size_t i = 0; i < keys.size(); ++i)
      if (used[i]) big.put(keys[i], vals[i]);
    *this = std::move(big);
  }
  void put(int32_t k, int32_t v) {
    size_t i = h(k) & mask;
    while (used[i]) i = (i + 1) & mask;
    used[i] = 1;
    keys[i] = k;
    vals[i] = v;
    ++count;
  }
  int32_t get(int32_t k) const {
    size_t i = h(k) & mask;
    while (used[i]) {
      if (keys[i] == k) return vals[i];
      i = (i + 1) & mask;
    }
    return -1;
  }
  int32_t get_or_add(int32_t k) {
    int32_t v = get(k);
    if (v >= 0) return v;
    if (2 * (count + 1) > keys.size()) grow();
    v = (int32_t)count;
    put(k, v);
    return v;
  }
};

struct Contact {
  int64_t s, e;
  int32_t a, b;  // ids numbered by first appearance within the chunk's range
};

// One thread's share of the file: its contacts, and the raw ids in the order
// they first appear there (first[j] is the raw id of local number j), so
// that the file-wide first-appearance numbering is a merge of the ranges in
// file order.
struct ChunkResult {
  std::vector<Contact> contacts;
  IdMap ids{1024};
  std::vector<int32_t> dense;  // local number of raw id i (< dense.size()), -1 if none yet
  std::vector<int32_t> first;
  int64_t counted = 0;
  int64_t malformed = 0;
  int32_t local(int32_t raw) {
    if ((uint32_t)raw < dense.size()) {
      int32_t &d = dense[(uint32_t)raw];
      if (d < 0) {
        d = (int32_t)first.size();
        first.push_back(raw);
      }
      return d;
    }
    int32_t j = ids.get(raw);
    if (j < 0) {
      j = (int32_t)first.size();
      if (2 * (ids.count + 1) > ids.keys.size()) ids.grow();
      ids.put(raw, j);
      first.push_back(raw);
    }
    return j;
  }
  void add(int64_t ts, int64_t te, int32_t a, int32_t b) {
    const int32_t la = local(a);  // a before b: the reference indexes the
    const int32_t lb = local(b);  // first endpoint first
    contacts.push_back(Contact{ts, te, la, lb});
  }
};

inline bool is_blank(char c) { return c == ' ' || c == '\t'; }
inline bool is_digit(char c) { return c >= '0' && c <= '9'; }

// Parses [-]digits (1..9 digits) at p.
inline bool fast_int(const char *&p, const char *end, int64_t &out) {
  bool neg = false;
  if (p < end && *p == '-') {
    neg = true;
    ++p;
  }
  int n = 0;
  int64_t v = 0;
  while (p < end && is_digit(*p) && n < 10) {
    v = v * 10 + (*p - '0');
    ++p;
    ++n;
  }
  if (n == 0 || n > 9) return false;
  out = neg ? -v : v;
  return true;
}

// digits-digits-digitsTdigits:digits:digits[Z] followed by blanks up to `end`
inline bool fast_ts(const char *p, const char *end, int64_t &out) {
  int64_t f[6];
  const char seps[6] = {'-', '-', 'T', ':', ':', 0};
  for (int i = 0; i < 6; ++i) {
    int n = 0;
    int64_t v = 0;
    while (p < end && is_digit(*p) && n < 10) {
      v = v * 10 + (*p - '0');
      ++p;
      ++n;
    }
    if (n == 0 || n > 9) return false;
    f[i] = v;
    if (i < 5) {
      if (p >= end || *p != seps[i]) return false;
      ++p;
    }
  }
  if (p < end && *p == 'Z') ++p;
  while (p < end && is_blank(*p)) ++p;
  if (p != end) return false;
  out = utc_seconds(f[0], f[1], f[2], f[3], f[4], f[5]);
  return true;
}

// Canonical line: [blanks]id,[blanks]id,[blanks]TS[blanks],[blanks]TS[blanks];...
// Returns false when the line is not canonical (caller falls back).
inline bool fast_line(const char *p, const char *end, Contact &c) {
  while (p < end && is_blank(*p)) ++p;
  int64_t a, b;
  if (!fast_int(p, end, a) || p >= end || *p != ',') return false;
  ++p;
  while (p < end && is_blank(*p)) ++p;
  if (!fast_int(p, end, b) || p >= end || *p != ',') return false;
  ++p;
  while (p < end && is_blank(*p)) ++p;
  const char *s0 = p;
  while (p < end && *p != ',' && *p != '\n' && *p != '\r' && *p != ';') ++p;
  if (p >= end || *p != ',' || p == s0 || p - s0 > 63) return false;
  const char *s1 = p;
  ++p;
  while (p < end && is_blank(*p)) ++p;
  const char *e0 = p;
  while (p < end && *p != ';' && *p != '\n' && *p != '\r' && *p != ',') ++p;
  if (p >= end || *p != ';' || p == e0 || p - e0 > 63) return false;
  const char *e1 = p;
  int64_t ts, te;
  if (!fast_ts(s0, s1, ts) || !fast_ts(e0, e1, te)) return false;
  c.s = ts;
  c.e = te;
  c.a = (int32_t)a;
  c.b = (int32_t)b;
  return true;
}

// One fgets chunk through the reference's two sscanf patterns.
void slow_chunk(const char *p, size_t len, ChunkResult &r) {
  std::string line(p, len);
  if (!line.empty() && line[0] == '#') return;
  int d1, d2;
  char s[64], e[64];
  if (sscanf(line.c_str(), " %d, %d, %63[^,], %63[^;];", &d1, &d2, s, e) == 4)
    r.counted++;
  int a, b;
  if (sscanf(line.c_str(), " %d , %d , %63[^,] , %63[^;\r\n] ;", &a, &b, s, e) != 4) {
    r.malformed++;
    return;
  }
  const int64_t ts = iso8601_slow(s), te = iso8601_slow(e);
  if (ts == -1 || te == -1) return;
  r.add(ts, te, a, b);
}

// "DDDD-DD-DDTDD:DD:DDZ" exactly (the generator's and most files' form).
inline bool canon_ts(const char *p, int64_t &out) {
  static const char kSep[20] = {0, 0, 0, 0, '-', 0, 0, '-', 0, 0, 'T', 0, 0, ':', 0, 0, ':', 0, 0, 'Z'};
  uint32_t dg[20];
  bool ok = true;
#pragma GCC unroll 20
  for (int i = 0; i < 20; ++i) {
    if (kSep[i]) {
      ok &= p[i] == kSep[i];
    } else {
      dg[i] = (uint32_t)(unsigned char)p[i] - (uint32_t)'0';
      ok &= dg[i] <= 9u;
    }
  }
  if (!ok) return false;
  out = utc_seconds(dg[0] * 1000 + dg[1] * 100 + dg[2] * 10 + dg[3], dg[5] * 10 + dg[6],
                    dg[8] * 10 + dg[9], dg[11] * 10 + dg[12], dg[14] * 10 + dg[15],
                    dg[17] * 10 + dg[18]);
  return true;
}

// "id, id, TS, TS;" with ids of 1-9 digits and TS in canon_ts form; returns
// the position just past ';', or nullptr for any other shape.
inline const char *canon_line(const char *p, const char *end, Contact &c) {
  int64_t v[2];
  for (int k = 0; k < 2; ++k) {
    int n = 0;
    int64_t x = 0;
    while (p < end && is_digit(*p) && n < 10) {
      x = x * 10 + (*p - '0');
      ++p;
      ++n;
    }
    if (n == 0 || n > 9 || end - p < 2 || p[0] != ',' || p[1] != ' ') return nullptr;
    p += 2;
    v[k] = x;
  }
  if (end - p < 43 || p[20] != ',' || p[21] != ' ' || p[42] != ';') return nullptr;
  int64_t ts, te;
  if (!canon_ts(p, ts) || !canon_ts(p + 22, te)) return nullptr;
  c.s = ts;
  c.e = te;
  c.a = (int32_t)v[0];
  c.b = (int32_t)v[1];
  return p + 43;
}

void parse_range(const char *p, const char *end, ChunkResult &r) {
  r.contacts.reserve((size_t)(end - p) / 60 + 16);
  while (p < end) {
    if (*p != '#') {
      Contact c;
      const char *q = canon_line(p, end, c);
      if (q) {
        const char *nl = (const char *)memchr(q, '\n', (size_t)(end - q));
        const char *le = nl ? nl + 1 : end;
        if ((size_t)(le - p) <= kFgetsChunk) {
          r.counted++;
          if (c.s != -1 && c.e != -1) r.add(c.s, c.e, c.a, c.b);
          p = le;
          continue;
        }
      }
    }
    const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
    const char *le = nl ? nl + 1 : end;  // line including '\n'
    const size_t len = (size_t)(le - p);
    if (len <= kFgetsChunk) {
      if (p[0] != '#') {
        Contact c;
        if (fast_line(p, le, c)) {
          r.counted++;
          if (c.s != -1 && c.e != -1) r.add(c.s, c.e, c.a, c.b);
        } else {
          slow_chunk(p, len, r);
        }
      }
    } else {
      for (size_t off = 0; off < len; off += kFgetsChunk)
        slow_chunk(p + off, std::min(kFgetsChunk, len - off), r);
    }
    p = le;
  }
}



}  // namespace

// ---------------------------------------------------------------------------
rp_status parse_contact_file(const char *path, ParsedContacts &out) {
  out.release_all();
  out.n = 0;
  int fd = open(path, O_RDONLY);
  if (fd < 0) {
    set_error("could not open file '%s'", path);
    return RP_ERR_IO;
  }
  struct stat stt;
  if (fstat(fd, &stt) != 0) {
    close(fd);
    set_error("could not stat '%s'", path);
    return RP_ERR_IO;
  }
  const size_t size = (size_t)stt.st_size;
  const char *data = nullptr;
  if (size > 0) {
    data = (const char *)mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (data == MAP_FAILED) {
      close(fd);
      set_error("could not map '%s'", path);
      return RP_ERR_IO;
    }
  }
  close(fd);
  struct Unmap {
    const char *d;
    size_t n;
    ~Unmap() {
      if (d) munmap((void *)d, n);
    }
  } unmap{data, size};

  // ---- header ----
  if (size == 0) {
    set_error("unable to read first line from file");
    return RP_ERR_PARSE;
  }
  const char *hl_end = (const char *)memchr(data, '\n', size);
  const size_t hlen = hl_end ? (size_t)(hl_end - data) + 1 : size;
  std::string header(data, hlen);
  if (header.compare(0, 9, "NODE_LIST") != 0 || header.size() < 10 ||
      (header[9] != ' ' && header[9] != '\t')) {
    set_error("first line must begin with 'NODE_LIST'");
    return RP_ERR_PARSE;
  }
  std::vector<long> ids;
  {
    char *save = nullptr;
    for (char *tok = strtok_r(&header[9], " \t\r\n", &save); tok;
         tok = strtok_r(nullptr, " \t\r\n", &save)) {
      errno = 0;
      char *endp = nullptr;
      long id = strtol(tok, &endp, 10);
      if (errno != 0 || *endp != '\0' || id < 0) {
        set_error("invalid node ID in NODE_LIST: '%s'", tok);
        return RP_ERR_PARSE;
      }
      ids.push_back((long)(int)id);
    }
  }
  if (ids.empty()) {
    set_error("no valid node IDs found in NODE_LIST");
    return RP_ERR_PARSE;
  }
  {
    std::vector<long> sorted = ids;
    std::sort(sorted.begin(), sorted.end());
    for (size_t i = 1; i < sorted.size(); ++i)
      if (sorted[i] == sorted[i - 1]) {
        set_error("duplicate node ID detected in NODE_LIST: %ld", sorted[i]);
        return RP_ERR_PARSE;
      }
  }
  if (ids.size() > (size_t)INT32_MAX) {
    set_error("NODE_LIST too long");
    return RP_ERR_RANGE;
  }
  const int32_t n_nodes = (int32_t)ids.size();
  out.n_nodes = n_nodes;

  // ---- contact lines (the header's own fgets chunks are malformed lines) ----
  int64_t header_chunks = 0;
  for (size_t off = 0; off < hlen; off += kFgetsChunk) ++header_chunks;
  unsigned nthreads = std::thread::hardware_concurrency();
  if (nthreads == 0) nthreads = 1;
  if (nthreads > 32) nthreads = 32;
  const char *body = data + hlen, *body_end = data + size;
  const size_t body_len = (size_t)(body_end - body);
  if (body_len < (size_t)1 << 20) nthreads = 1;
  std::vector<const char *> cuts(nthreads + 1);
  cuts[0] = body;
  cuts[nthreads] = body_end;
  for (unsigned t = 1; t < nthreads; ++t) {
    const char *p = body + body_len * t / nthreads;
    if (p < cuts[t - 1]) p = cuts[t - 1];
    const char *nl = (const char *)memchr(p, '\n', (size_t)(body_end - p));
    cuts[t] = nl ? nl + 1 : body_end;
  }
  std::vector<ChunkResult> parts(nthreads);
  // ids in [0, max NODE_LIST id] are numbered through a dense table per
  // thread when all tables together stay within 64M entries (256 MB)
  size_t dense_n = 0;
  {
    long max_id = 0;
    for (long id : ids) max_id = id > max_id ? id : max_id;
    if ((size_t)(max_id + 1) * nthreads <= ((size_t)1 << 26)) dense_n = (size_t)max_id + 1;
  }
  {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nthreads; ++t)
      pool.emplace_back([&, t] {
        parts[t].dense.assign(dense_n, -1);
        parse_range(cuts[t], cuts[t + 1], parts[t]);
      });
    for (auto &th : pool) th.join();
  }
  int64_t counted = 0, valid = 0;
  out.n_malformed = header_chunks;
  for (auto &pr : parts) {
    counted += pr.counted;
    valid += (int64_t)pr.contacts.size();
    out.n_malformed += pr.malformed;
  }
  if (counted <= 0) {
    set_error("no valid edge lines found in %s", path);
    return RP_ERR_PARSE;
  }
  if (valid > counted) {
    set_error("more edges parsed than expected (%lld > %lld)", (long long)valid,
              (long long)counted);
    return RP_ERR_PARSE;
  }
  if (valid == 0) {
    set_error("no intervals read or parse error");
    return RP_ERR_PARSE;
  }
  if (valid > (int64_t)INT32_MAX) {
    set_error("too many contacts (%lld)", (long long)valid);
    return RP_ERR_RANGE;
  }

  // ---- node index: first appearance over the ranges in file order ----
  std::vector<std::vector<int32_t>> to_global(nthreads);
  {
    IdMap map((size_t)n_nodes);
    for (unsigned t = 0; t < nthreads; ++t) {
      to_global[t].resize(parts[t].first.size());
      for (size_t j = 0; j < parts[t].first.size(); ++j)
        to_global[t][j] = map.get_or_add(parts[t].first[j]);
    }
    out.n_index = (int32_t)map.count;
  }
  if (out.n_index > n_nodes) {
    set_error("contact lines name %d distinct nodes but NODE_LIST declares %d",
              out.n_index, n_nodes);
    return RP_ERR_PARSE;
  }
  out.start = (int64_t *)malloc(sizeof(int64_t) * (size_t)valid);
  out.end = (int64_t *)malloc(sizeof(int64_t) * (size_t)valid);
  out.u = (int32_t *)malloc(sizeof(int32_t) * (size_t)valid);
  out.v = (int32_t *)malloc(sizeof(int32_t) * (size_t)valid);
  if (!out.start || !out.end || !out.u || !out.v) {
    out.release_all();
    set_error("out of host memory for %lld contacts", (long long)valid);
    return RP_ERR_NOMEM;
  }
  {
    std::vector<int64_t> base(nthreads + 1, 0);
    for (unsigned t = 0; t < nthreads; ++t)
      base[t + 1] = base[t] + (int64_t)parts[t].contacts.size();
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nthreads; ++t)
      pool.emplace_back([&, t] {
        int64_t k = base[t];
        const int32_t *g = to_global[t].data();
        for (const Contact &c : parts[t].contacts) {
          const int32_t ia = g[c.a], ib = g[c.b];
          out.start[k] = c.s;
          out.end[k] = c.e;
          out.u[k] = ia < ib ? ia : ib;
          out.v[k] = ia < ib ? ib : ia;
          ++k;
        }
        std::vector<Contact>().swap(parts[t].contacts);
      });
    for (auto &th : pool) th.join();
  }
  out.n = valid;
  return RP_OK;
}

// ---------------------------------------------------------------------------
static int64_t sat_sub(int64_t a, int64_t b) {  // a - b, b >= 0, saturating
  if (a < INT64_MIN + b) return INT64_MIN;
  return a - b;
}

int32_t plan_window_ranges(const Graph &g, int64_t ws, int64_t we, float scale, int64_t cap,
                           CandRange *ranges, WinDesc &out) {
  out.ws = ws;
  out.we = we;
  out.scale = scale;
  // The reference mirrors a query whose start is negative (intervaldb.c:437-444).
  if (ws < 0) {
    out.qs = -we;
    out.qe = -ws;
  } else {
    out.qs = ws;
    out.qe = we;
  }
  out.range_off = 0;
  out.n_ranges = 0;
  out.n_candidates = 0;
  for (int c = 0; c < kClasses; ++c) {
    const int64_t b0 = g.class_off[c], b1 = g.class_off[c + 1];
    if (b1 <= b0) continue;
    // candidates: stored start in (qs - 2^c, qe)
    const int64_t span = c >= 63 ? INT64_MAX : ((int64_t)1 << c);
    const int64_t lo_key = sat_sub(out.qs, span);  // start > lo_key
    auto first = g.h_cs.begin() + b0, last = g.h_cs.begin() + b1;
    auto lo = std::upper_bound(first, last, lo_key);
    auto hi = std::lower_bound(lo, last, out.qe);
    const int64_t count = hi - lo;
    if (count <= 0) continue;
    ranges[out.n_ranges++] = CandRange{(int64_t)(lo - g.h_cs.begin()), count, out.n_candidates};
    out.n_candidates += count;
  }
  out.may_truncate = out.n_candidates > cap ? 1 : 0;
  return out.n_ranges;
}

void plan_window(const Graph &g, int64_t ws, int64_t we, float scale,
                 int64_t cap, std::vector<CandRange> &ranges, WinDesc &out) {
  CandRange r[kClasses];
  const int32_t n = plan_window_ranges(g, ws, we, scale, cap, r, out);
  out.range_off = (int32_t)ranges.size();
  ranges.insert(ranges.end(), r, r + n);
}

}  // namespace rp
