/* CPU oracle for the replay hot path -- TEST INFRASTRUCTURE ONLY (see
 * replay_oracle.h).  Compiled with -ffp-contract=off so that every float
 * operation rounds exactly as the CUDA kernels' explicit __f*_rn intrinsics.
 *
 * Reference behaviour restated here, with the reference location each
 * function follows (paths relative to the HarrisonGreenlee/Replay tree):
 *   orc_parse_file      tool/temporal_contact_matrix.c:122-321 (two passes,
 *                       sscanf patterns, '#' comments, NODE_LIST rules) and
 *                       :328-356 (index = order of first appearance)
 *   orc_parse_iso8601   tool/temporal_contact_matrix.c:95-120 (timegm, with
 *                       its normalisation of out-of-range fields)
 *   orc_sort_order      tool/ncls/ncls/src/intervaldb.c:30-46,240 (qsort by
 *                       start asc, end desc; glibc's qsort is a stable merge
 *                       sort, so ties keep file order)
 *   orc_nlists          tool/ncls/ncls/src/intervaldb.c:243-320
 *   orc_window_hits     tool/ncls/ncls/src/intervaldb.c:426-485 called with
 *                       nbuf = nlists by tool/gpu_cpu_temporal_sim.cu:973-991
 *   orc_csr_f32         tool/gpu_cpu_temporal_sim.cu:238-350
 *   orc_spmm_f32        tool/gpu_cpu_temporal_sim.cu:403-433 (Eigen row-major
 *                       sparse x dense: sequential row sums)
 *   orc_schedule        tool/gpu_cpu_temporal_sim.cu:859-959
 *   countdown rules     tool/gpu_cpu_temporal_sim.cu:73-176, 505-568
 */
#include "replay_oracle.h"

#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Philox4x32-10: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11.  Two 32x32->64 multiplies per round, Weyl key
 * schedule. */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                       uint32_t out[4]) {
  uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; round++) {
    uint64_t p0 = (uint64_t)PHILOX_M0 * x0;
    uint64_t p1 = (uint64_t)PHILOX_M1 * x2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ x1 ^ k0;
    uint32_t n2 = hi0 ^ x3 ^ k1;
    x0 = n0;
    x1 = lo1;
    x2 = n2;
    x3 = lo0;
    k0 += PHILOX_W0;
    k1 += PHILOX_W1;
  }
  out[0] = x0;
  out[1] = x1;
  out[2] = x2;
  out[3] = x3;
}

float orc_unit(uint32_t x) {
  /* 24-bit grid: exact in float, never 0, may be 1. */
  return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

float orc_uniform(uint64_t seed, uint32_t node, uint32_t step,
                  uint32_t replica, uint32_t stream) {
  uint32_t ctr[4] = {node, step, replica >> 2, stream};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  orc_philox4x32_10(ctr, key, out);
  return orc_unit(out[replica & 3u]);
}

/* Fixed-point threshold floor(p * 2^64) of a per-step probability, with
 * p >= 1 flagged as certain. */
uint64_t orc_threshold64(float p, int *always) {
  *always = p >= 1.0f;
  if (!(p > 0.0f) || p >= 1.0f) return 0;
  return (uint64_t)ldexp((double)p, 64);
}

/* Flow decision of replica r (E->I, I->R, R->S): its per-step uniform U is
 * bit (r % 32) of successive random planes; plane k (k = 0 is 2^-1) is
 * output k % 4 of Philox(key = seed, counter = (node, step, r / 32,
 * (k / 4) << 4)).  Event iff U < T on the first 64 bits. */
int orc_flow_event(uint64_t seed, uint32_t node, uint32_t step, uint32_t replica,
                   uint64_t T, int always) {
  if (always) return 1;
  if (T == 0) return 0;
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t bit = replica & 31u;
  for (int j = 0; j < 16; j++) {
    uint32_t ctr[4] = {node, step, replica >> 5, (uint32_t)j << 4};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    for (int q = 0; q < 4; q++) {
      const int k = 4 * j + q;
      const uint32_t wb = (x[q] >> bit) & 1u;
      const uint32_t tb = (uint32_t)(T >> (63 - k)) & 1u;
      if (wb != tb) return wb < tb;
    }
  }
  return 0;
}

/* Geometric infection uniform U_r of replica r (64 bits, k = 0 is 2^-1)
 * compared with T = floor(P 2^64): its top 8 bits are bit-sliced -- bit k is
 * bit (r % 32) of output k % 4 of Philox(key = seed, counter = (node, step,
 * r / 32, 4 | (k / 4) << 4)), k < 8 -- and its low 56 bits are the top 56
 * bits of outputs 0-1 (output 0 high) of Philox(counter = (node, step, r,
 * 12)). */
static int infect_less(uint64_t seed, uint32_t node, uint32_t step, uint32_t replica,
                       uint64_t T) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t bit = replica & 31u;
  uint32_t u8 = 0;
  for (int j = 0; j < 2; j++) {
    uint32_t ctr[4] = {node, step, replica >> 5, 4u | ((uint32_t)j << 4)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    for (int q = 0; q < 4; q++) u8 = (u8 << 1) | ((x[q] >> bit) & 1u);
  }
  const uint32_t t8 = (uint32_t)(T >> 56);
  if (u8 != t8) return u8 < t8;
  uint32_t ctr[4] = {node, step, replica, 12u};
  uint32_t x[4];
  orc_philox4x32_10(ctr, key, x);
  const uint64_t low = (((uint64_t)x[0] << 32) | x[1]) >> 8;
  return low < (T & 0x00FFFFFFFFFFFFFFull);
}

/* Infection decision of replica r (geometric mode): event iff
 * U_r < floor(P 2^64) (infect_less); P >= 1 always infects, P <= 0 (or NaN)
 * never. */
int orc_infect_event(uint64_t seed, uint32_t node, uint32_t step, uint32_t replica, float P) {
  if (!(P > 0.0f)) return 0;
  if (P >= 1.0f) return 1;
  return infect_less(seed, node, step, replica, (uint64_t)ldexp((double)P, 64));
}

/* 1 - exp(-x) for x >= 0 using only correctly rounded +,-,*: Cody-Waite
 * reduction x = k ln2 + r, |r| <= ln2/2, and the Taylor series of expm1(-r)
 * through r^9/9!.  The device code performs the identical sequence with
 * __fmul_rn/__fadd_rn, so both sides round identically. */
float orc_one_minus_exp_neg(float x) {
  if (x != x) return x;
  if (!(x > 0.0f)) return 0.0f;
  if (x >= 87.0f) return 1.0f;
  const float inv_ln2 = 0x1.715476p+0f;
  const float ln2_hi = 0x1.62e4p-1f; /* 15 significant bits: k*ln2_hi exact */
  const float ln2_lo = 0x1.7f7d1cp-20f;
  int k = (int)(x * inv_ln2 + 0.5f);
  float kf = (float)k;
  float r = (x - kf * ln2_hi) - kf * ln2_lo;
  float y = -r;
  float p = 0x1.71de3ap-19f;        /* 1/9! */
  p = p * y + 0x1.a01a02p-16f;      /* 1/8! */
  p = p * y + 0x1.a01a02p-13f;      /* 1/7! */
  p = p * y + 0x1.6c16c2p-10f;      /* 1/6! */
  p = p * y + 0x1.111112p-7f;       /* 1/5! */
  p = p * y + 0x1.555556p-5f;       /* 1/4! */
  p = p * y + 0x1.555556p-3f;       /* 1/3! */
  p = p * y + 0.5f;                 /* 1/2! */
  float em1 = y + (y * y) * p; /* expm1(-r) */
  if (k == 0) return -em1;
  union {
    uint32_t u;
    float f;
  } scale;
  scale.u = (uint32_t)(127 - k) << 23; /* 2^-k, k in [1,126] */
  float e = (1.0f + em1) * scale.f;
  return 1.0f - e;
}

/* ------------------------------------------------------------------------ */
/* Days from the civil date (proleptic Gregorian), H. Hinnant's published
 * algorithm "days_from_civil". */
static int64_t days_from_civil(int64_t y, int64_t m, int64_t d) {
  y -= m <= 2;
  int64_t era = (y >= 0 ? y : y - 399) / 400;
  int64_t yoe = y - era * 400;
  int64_t doy = (153 * (m > 2 ? m - 3 : m + 9) + 2) / 5 + d - 1;
  int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + doe - 719468;
}

static int64_t floor_div(int64_t a, int64_t b) {
  int64_t q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) q--;
  return q;
}

int64_t orc_timegm(int year, int month0, int mday, int hour, int min, int sec) {
  /* timegm() normalises every field; months fold into years, the rest is
   * linear in seconds. */
  int64_t y = (int64_t)year + floor_div(month0, 12);
  int64_t m = (int64_t)month0 - floor_div(month0, 12) * 12;
  int64_t days = days_from_civil(y, m + 1, 1) + (int64_t)mday - 1;
  return days * 86400 + (int64_t)hour * 3600 + (int64_t)min * 60 + (int64_t)sec;
}

int64_t orc_parse_iso8601(const char *s) {
  if (!s) return -1;
  int year, month, day, hour, min, sec;
  char extra[10];
  if (sscanf(s, "%d-%d-%dT%d:%d:%d%9s", &year, &month, &day, &hour, &min, &sec,
             extra) < 6)
    return -1;
  return orc_timegm(year, month - 1, day, hour, min, sec);
}

static int cmpl(const void *a, const void *b) {
  long x = *(const long *)a, y = *(const long *)b;
  return x < y ? -1 : (x > y);
}

/* ---- node map: int id -> first-appearance index (open addressing) ---- */
typedef struct {
  int32_t *keys;
  int32_t *vals;
  uint8_t *used;
  int64_t cap, count;
} idmap;

static void idmap_init(idmap *m) {
  m->cap = 1024;
  m->count = 0;
  m->keys = (int32_t *)malloc(sizeof(int32_t) * m->cap);
  m->vals = (int32_t *)malloc(sizeof(int32_t) * m->cap);
  m->used = (uint8_t *)calloc(m->cap, 1);
}
static void idmap_free(idmap *m) {
  free(m->keys);
  free(m->vals);
  free(m->used);
}
static uint64_t hash32(uint32_t x) {
  uint64_t h = x * 0x9E3779B97F4A7C15ull;
  return h ^ (h >> 29);
}
static int32_t idmap_get_or_add(idmap *m, int32_t key);
static void idmap_grow(idmap *m) {
  idmap old = *m;
  m->cap *= 2;
  m->count = 0;
  m->keys = (int32_t *)malloc(sizeof(int32_t) * m->cap);
  m->vals = (int32_t *)malloc(sizeof(int32_t) * m->cap);
  m->used = (uint8_t *)calloc(m->cap, 1);
  for (int64_t i = 0; i < old.cap; i++) {
    if (!old.used[i]) continue;
    uint64_t h = hash32((uint32_t)old.keys[i]) & (m->cap - 1);
    while (m->used[h]) h = (h + 1) & (m->cap - 1);
    m->used[h] = 1;
    m->keys[h] = old.keys[i];
    m->vals[h] = old.vals[i];
    m->count++;
  }
  idmap_free(&old);
}
static int32_t idmap_get_or_add(idmap *m, int32_t key) {
  if (2 * (m->count + 1) > m->cap) idmap_grow(m);
  uint64_t h = hash32((uint32_t)key) & (m->cap - 1);
  while (m->used[h]) {
    if (m->keys[h] == key) return m->vals[h];
    h = (h + 1) & (m->cap - 1);
  }
  m->used[h] = 1;
  m->keys[h] = key;
  m->vals[h] = (int32_t)m->count;
  m->count++;
  return m->vals[h];
}

#define ORC_MAX_LINE 100000

static char *read_first_line(FILE *fp) {
  size_t cap = 128, n = 0;
  char *buf = (char *)malloc(cap);
  int c = 0;
  while ((c = fgetc(fp)) != EOF) {
    if (n + 1 >= cap) {
      cap *= 2;
      buf = (char *)realloc(buf, cap);
    }
    buf[n++] = (char)c;
    if (c == '\n') break;
  }
  if (n == 0 && c == EOF) {
    free(buf);
    return NULL;
  }
  buf[n] = 0;
  return buf;
}

int orc_parse_file(const char *path, int32_t *n_nodes, int32_t *n_index,
                   int64_t *n_contacts, int64_t **start, int64_t **end,
                   int32_t **u, int32_t **v, int64_t *n_malformed) {
  *n_nodes = 0;
  *n_index = 0;
  *n_contacts = 0;
  *n_malformed = 0;
  *start = NULL;
  *end = NULL;
  *u = NULL;
  *v = NULL;
  FILE *fp = fopen(path, "r");
  if (!fp) return 1;
  char *header = read_first_line(fp);
  fclose(fp);
  if (!header) return 2;
  if (strncmp(header, "NODE_LIST", 9) != 0 ||
      (header[9] != ' ' && header[9] != '\t')) {
    free(header);
    return 2;
  }
  /* NODE_LIST tokens: non-negative base-10 integers, no duplicates. */
  int64_t ntok = 0, tcap = 1024;
  long *ids = (long *)malloc(sizeof(long) * tcap);
  char *save = NULL;
  for (char *tok = strtok_r(header + 9, " \t\r\n", &save); tok;
       tok = strtok_r(NULL, " \t\r\n", &save)) {
    errno = 0;
    char *endp = NULL;
    long id = strtol(tok, &endp, 10);
    if (errno != 0 || *endp != '\0' || id < 0) {
      free(ids);
      free(header);
      return 3;
    }
    if (ntok == tcap) {
      tcap *= 2;
      ids = (long *)realloc(ids, sizeof(long) * tcap);
    }
    ids[ntok++] = (long)(int)id;
  }
  free(header);
  /* duplicate check on the int-truncated ids, as the reference compares */
  {
    long *sorted = (long *)malloc(sizeof(long) * (ntok ? ntok : 1));
    memcpy(sorted, ids, sizeof(long) * ntok);
    qsort(sorted, ntok, sizeof(long), cmpl);
    for (int64_t i = 1; i < ntok; i++)
      if (sorted[i] == sorted[i - 1]) {
        free(sorted);
        free(ids);
        return 3;
      }
    free(sorted);
  }
  free(ids);
  if (ntok <= 0) return 3;
  *n_nodes = (int32_t)ntok;

  /* pass 1: count lines matching the counting pattern */
  fp = fopen(path, "r");
  if (!fp) return 1;
  char *line = (char *)malloc(ORC_MAX_LINE);
  int64_t counted = 0;
  while (fgets(line, ORC_MAX_LINE, fp)) {
    if (line[0] == '#') continue;
    int d1, d2;
    char s[64], e[64];
    if (sscanf(line, " %d, %d, %63[^,], %63[^;];", &d1, &d2, s, e) == 4)
      counted++;
  }
  fclose(fp);
  if (counted <= 0) {
    free(line);
    return 4;
  }
  /* pass 2: parse */
  fp = fopen(path, "r");
  if (!fp) {
    free(line);
    return 1;
  }
  int64_t cap = counted;
  int64_t *st = (int64_t *)malloc(sizeof(int64_t) * cap);
  int64_t *en = (int64_t *)malloc(sizeof(int64_t) * cap);
  int32_t *uu = (int32_t *)malloc(sizeof(int32_t) * cap);
  int32_t *vv = (int32_t *)malloc(sizeof(int32_t) * cap);
  idmap map;
  idmap_init(&map);
  int64_t n = 0;
  int rc = 0;
  while (fgets(line, ORC_MAX_LINE, fp)) {
    if (line[0] == '#') continue;
    int a, b;
    char s[64], e[64];
    if (sscanf(line, " %d , %d , %63[^,] , %63[^;\r\n] ;", &a, &b, s, e) != 4) {
      (*n_malformed)++;
      continue;
    }
    int64_t ts = orc_parse_iso8601(s), te = orc_parse_iso8601(e);
    if (ts == -1 || te == -1) continue;
    int32_t ia = idmap_get_or_add(&map, a);
    int32_t ib = idmap_get_or_add(&map, b);
    if (n >= cap) {
      rc = 5;
      break;
    }
    st[n] = ts;
    en[n] = te;
    uu[n] = ia < ib ? ia : ib;
    vv[n] = ia < ib ? ib : ia;
    n++;
  }
  fclose(fp);
  free(line);
  *n_index = (int32_t)map.count;
  idmap_free(&map);
  if (rc) {
    free(st);
    free(en);
    free(uu);
    free(vv);
    return rc;
  }
  if (n == 0) {
    free(st);
    free(en);
    free(uu);
    free(vv);
    return 4;
  }
  *n_contacts = n;
  *start = st;
  *end = en;
  *u = uu;
  *v = vv;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Stable merge sort of positions by (start asc, end desc). */
static const int64_t *g_sort_start, *g_sort_end;
static int before(int64_t a, int64_t b) {
  if (g_sort_start[a] != g_sort_start[b]) return g_sort_start[a] < g_sort_start[b];
  return g_sort_end[a] > g_sort_end[b];
}
static void merge_sort(int64_t *a, int64_t *tmp, int64_t n) {
  if (n < 2) return;
  int64_t h = n / 2;
  merge_sort(a, tmp, h);
  merge_sort(a + h, tmp, n - h);
  int64_t i = 0, j = h, k = 0;
  while (i < h && j < n) {
    if (before(a[j], a[i]))
      tmp[k++] = a[j++];
    else
      tmp[k++] = a[i++];
  }
  while (i < h) tmp[k++] = a[i++];
  while (j < n) tmp[k++] = a[j++];
  memcpy(a, tmp, sizeof(int64_t) * n);
}

void orc_sort_order(const int64_t *start, const int64_t *end, int64_t n,
                    int64_t *perm) {
  for (int64_t i = 0; i < n; i++) perm[i] = i;
  int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * (n ? n : 1));
  g_sort_start = start;
  g_sort_end = end;
  merge_sort(perm, tmp, n);
  free(tmp);
}

/* The nested containment list nests interval i under the nearest open
 * ancestor that contains it, where "contains" excludes identical intervals
 * (intervaldb.c:247-256).  Its nlists counts one header per interval with a
 * child plus one per restart of the parent chain (intervaldb.c:258-261),
 * which happens before every top-level interval but the first.  Computed
 * here with the same stack walk, over contacts already in sorted order. */
int64_t orc_nlists(const int64_t *s, const int64_t *e, int64_t n) {
  if (n <= 0) return 0;
  int64_t *chain = (int64_t *)malloc(sizeof(int64_t) * n);
  uint8_t *has_child = (uint8_t *)calloc(n, 1);
  int64_t depth = 0, n_top = 0;
  for (int64_t i = 0; i < n; i++) {
    while (depth > 0) {
      int64_t p = chain[depth - 1];
      int outside = e[i] > e[p] || (e[i] == e[p] && s[i] == s[p]);
      if (!outside) break;
      depth--;
    }
    if (depth == 0)
      n_top++;
    else
      has_child[chain[depth - 1]] = 1;
    chain[depth++] = i;
  }
  int64_t parents = 0;
  for (int64_t i = 0; i < n; i++) parents += has_child[i];
  free(chain);
  free(has_child);
  return (n_top - 1) + parents;
}

/* The reference's interval database is compiled with ALL_POSITIVE_ORIENTATION
 * (intervaldb.h:191): at build time every interval with start < 0 is stored
 * mirrored as (-end, -(int)start) (intervaldb.c:233-235, 412-424; the int
 * temporary truncates), a query whose start is negative is mirrored the same
 * way (intervaldb.c:437-444), and returned hits whose stored orientation
 * differs from the query's are mirrored back (intervaldb.c:475-478). */
void orc_store_coords(const int64_t *start, const int64_t *end, int64_t n,
                      int64_t *out_s, int64_t *out_e) {
  for (int64_t i = 0; i < n; i++) {
    if (start[i] < 0) {
      out_s[i] = -end[i];
      out_e[i] = -(int64_t)(int32_t)start[i];
    } else {
      out_s[i] = start[i];
      out_e[i] = end[i];
    }
  }
}

void orc_hit_coords(int64_t s, int64_t e, int64_t ws, int64_t *hs,
                    int64_t *he) {
  int query_sign = ws < 0 ? -1 : 1;
  int hit_sign = s >= 0 ? 1 : -1;
  if (hit_sign != query_sign) {
    *hs = -e;
    *he = -(int64_t)(int32_t)s;
  } else {
    *hs = s;
    *he = e;
  }
}

/* The NCLS returns the stored intervals overlapping the (possibly mirrored)
 * query (start < qe && qs < end) in a depth-first walk of the nesting forest;
 * every list is ordered by start and a subtree follows its root, so that walk
 * visits hits in sorted order.  The driver passes nbuf = nlists, so the query
 * stops after max(nlists, 1) hits (intervaldb.c:465-467).  Arrays hold stored
 * coordinates in sorted order. */
int64_t orc_window_hits(const int64_t *s, const int64_t *e, int64_t n,
                        int64_t nlists, int64_t ws, int64_t we,
                        int64_t *out_rank) {
  int64_t cap = nlists > 0 ? nlists : 1;
  int64_t qs = ws, qe = we;
  if (ws < 0) {
    qs = -we;
    qe = -ws;
  }
  int64_t k = 0;
  for (int64_t i = 0; i < n && k < cap; i++) {
    if (s[i] < qe && qs < e[i]) out_rank[k++] = i;
  }
  return k;
}

/* ------------------------------------------------------------------------ */
typedef struct {
  int32_t row, col;
  int64_t order; /* emission order: hit index * 2 + direction */
  float wf;
  int32_t wi;
} edge_item;

static int cmp_edge(const void *a, const void *b) {
  const edge_item *x = (const edge_item *)a, *y = (const edge_item *)b;
  if (x->row != y->row) return x->row < y->row ? -1 : 1;
  if (x->col != y->col) return x->col < y->col ? -1 : 1;
  return x->order < y->order ? -1 : (x->order > y->order);
}

static int64_t emit_edges(const int64_t *s, const int64_t *e, const int32_t *u,
                          const int32_t *v, const int64_t *hit_rank,
                          int64_t n_hits, int64_t ws, int64_t we, float scale,
                          edge_item *items) {
  int64_t cnt = 0;
  for (int64_t h = 0; h < n_hits; h++) {
    int64_t r = hit_rank[h];
    int64_t hs, he;
    orc_hit_coords(s[r], e[r], ws, &hs, &he);
    int64_t os = hs > ws ? hs : ws;
    int64_t oe = he < we ? he : we;
    if (oe <= os) continue;
    int64_t ov = oe - os;
    float wf = (float)ov * scale;
    items[cnt].row = u[r];
    items[cnt].col = v[r];
    items[cnt].order = 2 * h;
    items[cnt].wf = wf;
    items[cnt].wi = (int32_t)ov;
    cnt++;
    items[cnt].row = v[r];
    items[cnt].col = u[r];
    items[cnt].order = 2 * h + 1;
    items[cnt].wf = wf;
    items[cnt].wi = (int32_t)ov;
    cnt++;
  }
  qsort(items, cnt, sizeof(edge_item), cmp_edge);
  return cnt;
}

int64_t orc_csr_f32(const int64_t *s, const int64_t *e, const int32_t *u,
                    const int32_t *v, const int64_t *hit_rank, int64_t n_hits,
                    int32_t n_nodes, int64_t ws, int64_t we, float scale,
                    int32_t *row_ptr, int32_t *col, float *val) {
  edge_item *items =
      (edge_item *)malloc(sizeof(edge_item) * (2 * n_hits > 0 ? 2 * n_hits : 1));
  int64_t cnt = emit_edges(s, e, u, v, hit_rank, n_hits, ws, we, scale, items);
  int64_t nnz = 0;
  for (int64_t i = 0; i < cnt; i++) {
    if (nnz > 0 && items[i].row == items[nnz - 1].row &&
        items[i].col == items[nnz - 1].col)
      items[nnz - 1].wf = items[nnz - 1].wf + items[i].wf;
    else
      items[nnz++] = items[i];
  }
  for (int32_t i = 0; i <= n_nodes; i++) row_ptr[i] = 0;
  for (int64_t i = 0; i < nnz; i++) row_ptr[items[i].row + 1]++;
  for (int32_t i = 0; i < n_nodes; i++) row_ptr[i + 1] += row_ptr[i];
  for (int64_t i = 0; i < nnz; i++) {
    col[i] = items[i].col;
    val[i] = items[i].wf;
  }
  free(items);
  return nnz;
}

int64_t orc_csr_i32(const int64_t *s, const int64_t *e, const int32_t *u,
                    const int32_t *v, const int64_t *hit_rank, int64_t n_hits,
                    int32_t n_nodes, int64_t ws, int64_t we, int32_t *row_ptr,
                    int32_t *col, int32_t *val) {
  edge_item *items =
      (edge_item *)malloc(sizeof(edge_item) * (2 * n_hits > 0 ? 2 * n_hits : 1));
  int64_t cnt = emit_edges(s, e, u, v, hit_rank, n_hits, ws, we, 1.0f, items);
  int64_t nnz = 0;
  for (int64_t i = 0; i < cnt; i++) {
    if (nnz > 0 && items[i].row == items[nnz - 1].row &&
        items[i].col == items[nnz - 1].col)
      items[nnz - 1].wi += items[i].wi;
    else
      items[nnz++] = items[i];
  }
  for (int32_t i = 0; i <= n_nodes; i++) row_ptr[i] = 0;
  for (int64_t i = 0; i < nnz; i++) row_ptr[items[i].row + 1]++;
  for (int32_t i = 0; i < n_nodes; i++) row_ptr[i + 1] += row_ptr[i];
  for (int64_t i = 0; i < nnz; i++) {
    col[i] = items[i].col;
    val[i] = items[i].wi;
  }
  free(items);
  return nnz;
}

void orc_spmm_f32(const int32_t *row_ptr, const int32_t *col, const float *val,
                  int32_t n, const float *b, float *c, int32_t m) {
  for (int32_t r = 0; r < m; r++) {
    const float *bc = b + (int64_t)r * n;
    float *cc = c + (int64_t)r * n;
    for (int32_t i = 0; i < n; i++) {
      float acc = 0.0f;
      for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; k++)
        acc = acc + val[k] * bc[col[k]];
      cc[i] = acc;
    }
  }
}

void orc_spmm_i64(const int32_t *row_ptr, const int32_t *col,
                  const int32_t *val, int32_t n, const uint8_t *b, int64_t *c,
                  int32_t m) {
  for (int32_t r = 0; r < m; r++) {
    const uint8_t *bc = b + (int64_t)r * n;
    int64_t *cc = c + (int64_t)r * n;
    for (int32_t i = 0; i < n; i++) {
      int64_t acc = 0;
      for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; k++)
        acc += bc[col[k]] ? (int64_t)val[k] : 0;
      cc[i] = acc;
    }
  }
}

/* ------------------------------------------------------------------------ */
static int add_overflows(int64_t a, int64_t b) {
  return (b > 0 && a > INT64_MAX - b) || (b < 0 && a < INT64_MIN - b);
}

static int slice_start(int64_t start, float step, int64_t window, int32_t it,
                       int64_t *ws, int64_t *ts) {
  double raw = (double)it * (double)step;
  if (raw > (double)INT64_MAX || raw < (double)INT64_MIN) return 1;
  int64_t off = (int64_t)llround(raw);
  if (add_overflows(start, off)) return 1;
  int64_t net = (off / window) * window;
  if (off < 0 && (off % window)) net -= window;
  if (add_overflows(start, net)) return 1;
  *ws = start + net;
  *ts = start + off;
  return 0;
}

int orc_schedule(int64_t start_time, float step_size, int64_t window,
                 int32_t n_steps, int64_t *ws, int64_t *we, float *scale,
                 int64_t *ts) {
  if (window <= 0 || !(step_size > 0.0f)) return 1;
  int64_t cached = 0;
  int valid = 0;
  int32_t steps = 1;
  for (int32_t it = 0; it < n_steps; it++) {
    int64_t cs, t;
    if (slice_start(start_time, step_size, window, it, &cs, &t)) return 1;
    if (add_overflows(cs, window)) return 1;
    if (!valid || cs != cached) {
      steps = 0;
      for (int32_t f = it; f < n_steps; f++) {
        int64_t fs, ft;
        if (slice_start(start_time, step_size, window, f, &fs, &ft)) return 1;
        if (fs != cs) break;
        steps++;
      }
      if (steps <= 0) return 1;
      cached = cs;
      valid = 1;
    }
    ws[it] = cs;
    we[it] = cs + window;
    scale[it] = 1.0f / (float)steps;
    ts[it] = t;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
int orc_countdown_class(int32_t c, int32_t E, int32_t I, int32_t R) {
  int32_t upper = E + I + R;
  int32_t elapsed = (c <= 0 || c > upper) ? 0 : (upper - c);
  if (c == 0) return 0;
  if (E > 0 && elapsed < E) return 1;
  if (I > 0 && elapsed < E + I) return 2;
  if (R > 0 && elapsed < E + I + R) return 3;
  return 0;
}

/* Floyd's algorithm: k distinct nodes out of n for replica r of network
 * `net` (node indices within the network; stream 2 + 4 net). */
static void exact_k(uint64_t seed, uint32_t r, uint32_t net, int32_t n, int32_t k,
                    int32_t *chosen) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  int32_t cnt = 0;
  for (int32_t j = n - k; j < n; j++) {
    uint32_t ctr[4] = {(uint32_t)j, 0xFFFFFFFEu, r, 2u + 4u * net};
    uint32_t out[4];
    orc_philox4x32_10(ctr, key, out);
    uint64_t r64 = (uint64_t)out[0] | ((uint64_t)out[1] << 32);
    int32_t t = (int32_t)(((unsigned __int128)r64 * (uint64_t)(j + 1)) >> 64);
    int dup = 0;
    for (int32_t q = 0; q < cnt; q++)
      if (chosen[q] == t) {
        dup = 1;
        break;
      }
    chosen[cnt++] = dup ? j : t;
  }
}

int orc_run(const int64_t *start, const int64_t *end, const int32_t *u,
            const int32_t *v, int64_t n_contacts, int32_t n_nodes,
            const orc_params *p, int32_t *counts, uint8_t *node_states) {
  const int32_t N = n_nodes, M = p->n_replicas, T = p->n_steps;
  if (N <= 0 || M <= 0 || T < 0) return 1;
  int64_t *stored_s = (int64_t *)malloc(sizeof(int64_t) * (n_contacts ? n_contacts : 1));
  int64_t *stored_e = (int64_t *)malloc(sizeof(int64_t) * (n_contacts ? n_contacts : 1));
  orc_store_coords(start, end, n_contacts, stored_s, stored_e);
  start = stored_s;
  end = stored_e;
  int64_t *perm = (int64_t *)malloc(sizeof(int64_t) * (n_contacts ? n_contacts : 1));
  orc_sort_order(start, end, n_contacts, perm);
  int64_t *ss = (int64_t *)malloc(sizeof(int64_t) * (n_contacts ? n_contacts : 1));
  int64_t *se = (int64_t *)malloc(sizeof(int64_t) * (n_contacts ? n_contacts : 1));
  int32_t *su = (int32_t *)malloc(sizeof(int32_t) * (n_contacts ? n_contacts : 1));
  int32_t *sv = (int32_t *)malloc(sizeof(int32_t) * (n_contacts ? n_contacts : 1));
  for (int64_t i = 0; i < n_contacts; i++) {
    ss[i] = start[perm[i]];
    se[i] = end[perm[i]];
    su[i] = u[perm[i]];
    sv[i] = v[perm[i]];
  }
  free(perm);
  free(stored_s);
  free(stored_e);
  int64_t nlists = p->ncls_cap ? orc_nlists(ss, se, n_contacts) : n_contacts;

  int64_t *ws = (int64_t *)malloc(sizeof(int64_t) * (T ? T : 1));
  int64_t *we = (int64_t *)malloc(sizeof(int64_t) * (T ? T : 1));
  int64_t *ts = (int64_t *)malloc(sizeof(int64_t) * (T ? T : 1));
  float *scale = (float *)malloc(sizeof(float) * (T ? T : 1));
  if (orc_schedule(p->start_time, p->step_size, p->window, T, ws, we, scale, ts)) {
    free(ss); free(se); free(su); free(sv); free(ws); free(we); free(ts); free(scale);
    return 2;
  }
  const int64_t NM = (int64_t)N * M;
  int32_t *cd = (int32_t *)calloc(NM, sizeof(int32_t)); /* countdown or code */
  int32_t *row_ptr = (int32_t *)malloc(sizeof(int32_t) * (N + 1));
  int64_t *hits = (int64_t *)malloc(sizeof(int64_t) * (n_contacts ? n_contacts : 1));
  int32_t *col = (int32_t *)malloc(sizeof(int32_t) * (2 * n_contacts + 1));
  float *valf = (float *)malloc(sizeof(float) * (2 * n_contacts + 1));
  int32_t *vali = (int32_t *)malloc(sizeof(int32_t) * (2 * n_contacts + 1));
  float *expf_ = (float *)malloc(sizeof(float) * NM);
  int64_t *expi = (int64_t *)malloc(sizeof(int64_t) * NM);
  float *bf = (float *)malloc(sizeof(float) * NM);
  uint8_t *bi = (uint8_t *)malloc(NM);
  int32_t *chosen = (int32_t *)malloc(sizeof(int32_t) * (p->initial_count > 0 ? p->initial_count : 1));

  const int countdown = p->transition == 0;
  const int32_t Ed = p->exposed_duration, Id = p->infectious_duration,
                Rd = p->resistant_duration;
  const int32_t upper = Ed + Id + Rd, medium = Id + Rd, lower = Rd;
  const float neg_log_base = -logf(1.0f - p->infect_prob);
  int te_all, ti_all, tr_all;
  const uint64_t te = orc_threshold64(p->p_ei, &te_all);
  const uint64_t ti = orc_threshold64(p->p_ir, &ti_all);
  const uint64_t tr = orc_threshold64(p->p_rs, &tr_all);

  /* replicas r of this run are replicas r + roff of the stream layout */
  const int32_t roff = p->replica_offset;
  if (roff < 0 || roff % 32) return 4;
  /* network partition (one network spanning all nodes without a batch) */
  const int32_t n_nets = p->net_first ? p->n_nets : 1;
  int32_t one_net[2] = {0, N};
  const int32_t *nf = p->net_first ? p->net_first : one_net;
  /* initial state */
  for (int32_t k = 0; k < n_nets; k++)
    if (p->initial_count > 0 && p->initial_count > nf[k + 1] - nf[k]) return 3;
  for (int32_t r = 0; r < M; r++) {
    if (p->initial_count > 0) {
      for (int32_t k = 0; k < n_nets; k++) {
        exact_k(p->seed, (uint32_t)(r + roff), (uint32_t)k, nf[k + 1] - nf[k], p->initial_count, chosen);
        for (int32_t q = 0; q < p->initial_count; q++) {
          int64_t idx = nf[k] + chosen[q] + (int64_t)r * N;
          cd[idx] = countdown ? (int32_t)((float)medium + p->step_size) : 2;
        }
      }
    } else {
      for (int32_t i = 0; i < N; i++) {
        float uu = orc_uniform(p->seed, (uint32_t)i, 0xFFFFFFFFu, (uint32_t)(r + roff), 1u);
        if (uu < p->initial_infected)
          cd[i + (int64_t)r * N] = countdown ? (int32_t)((float)medium + p->step_size) : 2;
      }
    }
  }

#define ORC_RECORD(tidx)                                                      \
  do {                                                                        \
    for (int32_t k = 0; k < n_nets; k++)                                      \
      for (int32_t r = 0; r < M; r++) {                                       \
        int32_t cnt4[4] = {0, 0, 0, 0};                                       \
        for (int32_t i = nf[k]; i < nf[k + 1]; i++) {                         \
          int32_t c = cd[i + (int64_t)r * N];                                 \
          int cls = countdown ? orc_countdown_class(c, Ed, Id, Rd) : c;       \
          cnt4[cls]++;                                                        \
          if (node_states)                                                    \
            node_states[((int64_t)(tidx) * M + r) * N + i] = (uint8_t)cls;    \
        }                                                                     \
        int32_t *row = counts + (((int64_t)(tidx) * n_nets + k) * M + r) * 4; \
        row[0] = cnt4[1];                                                     \
        row[1] = cnt4[2];                                                     \
        row[2] = cnt4[3];                                                     \
        row[3] = cnt4[0];                                                     \
      }                                                                       \
  } while (0)

  ORC_RECORD(0);
  for (int32_t t = 0; t < T; t++) {
    int64_t nh = p->ncls_cap
                     ? orc_window_hits(ss, se, n_contacts, nlists, ws[t], we[t], hits)
                     : orc_window_hits(ss, se, n_contacts, n_contacts, ws[t], we[t], hits);
    if (countdown) {
      orc_csr_f32(ss, se, su, sv, hits, nh, N, ws[t], we[t], scale[t], row_ptr, col, valf);
      for (int64_t idx = 0; idx < NM; idx++)
        bf[idx] = (cd[idx] > lower && cd[idx] <= medium) ? 1.0f : 0.0f;
      orc_spmm_f32(row_ptr, col, valf, N, bf, expf_, M);
      for (int32_t r = 0; r < M; r++)
        for (int32_t i = 0; i < N; i++) {
          int64_t idx = i + (int64_t)r * N;
          if (cd[idx] == 0) {
            float e = expf_[idx] / 3600.0f;
            float P = orc_one_minus_exp_neg(neg_log_base * e);
            float uu = orc_uniform(p->seed, (uint32_t)i, (uint32_t)t, (uint32_t)(r + roff), 3u);
            if (P > uu) cd[idx] = (int32_t)((float)upper + p->step_size);
          }
        }
      for (int64_t idx = 0; idx < NM; idx++) {
        if (cd[idx] > 0) cd[idx] = (int32_t)((float)cd[idx] - p->step_size);
        if (cd[idx] < 0) cd[idx] = 0;
      }
    } else {
      orc_csr_i32(ss, se, su, sv, hits, nh, N, ws[t], we[t], row_ptr, col, vali);
      for (int64_t idx = 0; idx < NM; idx++) bi[idx] = cd[idx] == 2;
      orc_spmm_i64(row_ptr, col, vali, N, bi, expi, M);
      for (int32_t r = 0; r < M; r++) {
        float beta = p->beta_per_replica ? p->beta_per_replica[r] : p->beta;
        for (int32_t i = 0; i < N; i++) {
          int64_t idx = i + (int64_t)r * N;
          int32_t st = cd[idx];
          if (st == 0) {
            if (expi[idx] > 0) {
              float sus = p->susceptibility ? p->susceptibility[i] : 1.0f;
              float bs = beta * sus;
              float ef = (float)expi[idx];
              if (scale[t] != 1.0f) ef = ef * scale[t];
              float P = orc_one_minus_exp_neg(bs * ef);
              if (orc_infect_event(p->seed, (uint32_t)i, (uint32_t)t, (uint32_t)(r + roff), P))
                cd[idx] = p->has_exposed ? 1 : 2;
            }
          } else if (st == 1) {
            if (orc_flow_event(p->seed, (uint32_t)i, (uint32_t)t, (uint32_t)(r + roff), te, te_all))
              cd[idx] = 2;
          } else if (st == 2) {
            if (orc_flow_event(p->seed, (uint32_t)i, (uint32_t)t, (uint32_t)(r + roff), ti, ti_all))
              cd[idx] = p->ir_to_s ? 0 : 3;
          } else {
            if (orc_flow_event(p->seed, (uint32_t)i, (uint32_t)t, (uint32_t)(r + roff), tr, tr_all))
              cd[idx] = 0;
          }
        }
      }
    }
    ORC_RECORD(t + 1);
  }
#undef ORC_RECORD
  free(ss); free(se); free(su); free(sv); free(ws); free(we); free(ts); free(scale);
  free(cd); free(row_ptr); free(hits); free(col); free(valf); free(vali);
  free(expf_); free(expi); free(bf); free(bi); free(chosen);
  return 0;
}
