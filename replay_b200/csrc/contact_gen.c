/* contact_network: synthetic temporal contact networks of the reference's
 * group model, byte for byte.
 *
 *   contact_network <start_datetime> <steps> <step_size> <population_size>
 *                   <num_groups> <prob_inner> <prob_inter> <output_file> <seed>
 *
 * Restates generate_networks/graph_generator.c:41-157 and main.c:8-66 of the
 * reference: nodes 1..N are assigned to groups round-robin; for every step
 * and every pair i < j one uniform rand()/RAND_MAX decides a contact (prob_inner
 * within a group, prob_inter across), and a contact draws two timestamps
 * base + step*step_size + rand() % step_size, ordered so that start <= end,
 * written as "i, j, YYYY-MM-DDTHH:MM:SSZ, YYYY-MM-DDTHH:MM:SSZ;" after a
 * "NODE_LIST 1 .. N" header.  The start datetime is read as local time
 * (mktime), as the reference does.
 *
 * rand() is glibc's default generator (TYPE_3, an additive lagged Fibonacci
 * generator r[i] = r[i-31] + r[i-3] seeded through the Park-Miller LCG
 * 16807 x mod 2^31-1, first 310 outputs discarded, results r >> 1),
 * implemented here without locks so that the stream matches srand/rand of
 * glibc exactly.  Timestamps are formatted from the civil calendar directly.
 */
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
  int32_t r[34];
  int i; /* next position (mod 34) */
} glibc_rand;

static void grand_seed(glibc_rand *g, unsigned int seed) {
  int32_t *r = g->r;
  r[0] = seed == 0 ? 1 : (int32_t)seed;
  for (int i = 1; i < 31; ++i) {
    /* 16807 * r[i-1] % (2^31 - 1) without overflow (Schrage) */
    const int32_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
    int32_t w = 16807 * lo - 2836 * hi;
    if (w < 0) w += 2147483647;
    r[i] = w;
  }
  for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
  g->i = 34 % 34;
  /* r[k] for k >= 34 lives at k % 34; discard outputs 34 .. 343 */
  for (int k = 34; k < 344; ++k)
    r[k % 34] = (int32_t)((uint32_t)r[(k - 31) % 34] + (uint32_t)r[(k - 3) % 34]);
  g->i = 344 % 34;
}

static inline int grand_next(glibc_rand *g) {
  const int k = g->i;
  const int a = k >= 31 ? k - 31 : k + 3; /* (k - 31) mod 34 */
  const int b = k >= 3 ? k - 3 : k + 31;  /* (k - 3) mod 34 */
  const uint32_t v = (uint32_t)g->r[a] + (uint32_t)g->r[b];
  g->r[k] = (int32_t)v;
  g->i = k == 33 ? 0 : k + 1;
  return (int)(v >> 1);
}

/* days since 1970-01-01 -> civil date (H. Hinnant's days_from_civil inverse) */
static void civil_from_days(int64_t z, int64_t *y, int *m, int *d) {
  z += 719468;
  const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
  const int64_t doe = z - era * 146097;
  const int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  const int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const int64_t mp = (5 * doy + 2) / 153;
  *d = (int)(doy - (153 * mp + 2) / 5 + 1);
  *m = (int)(mp < 10 ? mp + 3 : mp - 9);
  *y = yoe + era * 400 + (*m <= 2);
}

static char *put_2(char *p, int v) {
  *p++ = (char)('0' + v / 10);
  *p++ = (char)('0' + v % 10);
  return p;
}

/* "YYYY-MM-DDTHH:MM:SSZ" of a UTC time (years 0..9999) */
static char *put_iso(char *p, int64_t t) {
  int64_t days = t / 86400, sec = t % 86400;
  if (sec < 0) {
    sec += 86400;
    --days;
  }
  int64_t y;
  int m, d;
  civil_from_days(days, &y, &m, &d);
  const int yy = (int)y;
  *p++ = (char)('0' + yy / 1000 % 10);
  *p++ = (char)('0' + yy / 100 % 10);
  *p++ = (char)('0' + yy / 10 % 10);
  *p++ = (char)('0' + yy % 10);
  *p++ = '-';
  p = put_2(p, m);
  *p++ = '-';
  p = put_2(p, d);
  *p++ = 'T';
  p = put_2(p, (int)(sec / 3600));
  *p++ = ':';
  p = put_2(p, (int)(sec / 60 % 60));
  *p++ = ':';
  p = put_2(p, (int)(sec % 60));
  *p++ = 'Z';
  return p;
}

static char *put_int(char *p, long long v) {
  char tmp[24];
  int n = 0;
  unsigned long long u = v < 0 ? 0ull - (unsigned long long)v : (unsigned long long)v;
  if (v < 0) *p++ = '-';
  do {
    tmp[n++] = (char)('0' + (int)(u % 10));
    u /= 10;
  } while (u);
  while (n) *p++ = tmp[--n];
  return p;
}

static time_t parse_datetime(const char *s) {
  int year, month, day, hour, minute, second;
  if (sscanf(s, "%d-%d-%dT%d:%d:%d", &year, &month, &day, &hour, &minute, &second) != 6) {
    fprintf(stderr, "Error parsing datetime string: %s\n", s);
    exit(EXIT_FAILURE);
  }
  struct tm tm_info;
  memset(&tm_info, 0, sizeof(tm_info));
  tm_info.tm_year = year - 1900;
  tm_info.tm_mon = month - 1;
  tm_info.tm_mday = day;
  tm_info.tm_hour = hour;
  tm_info.tm_min = minute;
  tm_info.tm_sec = second;
  return mktime(&tm_info); /* local time, as the reference */
}

int main(int argc, char **argv) {
  if (argc != 10) {
    printf("Usage: %s <start_datetime> <steps> <step_size> <population_size> <num_groups> "
           "<prob_inner> <prob_inter> <output_file> <seed>\n",
           argv[0]);
    return 1;
  }
  const time_t base = parse_datetime(argv[1]);
  const int steps = atoi(argv[2]);
  const int step_size = atoi(argv[3]);
  const int n = atoi(argv[4]);
  const int groups = atoi(argv[5]);
  const double p_in = atof(argv[6]), p_out = atof(argv[7]);
  const char *out_path = argv[8];
  const int seed = atoi(argv[9]);
  if (seed < 0) {
    fprintf(stderr, "Seed must be a non-negative integer.\n");
    return 0;
  }
  if (step_size <= 0 || groups <= 0) {
    fprintf(stderr, "step_size and num_groups must be positive.\n");
    return 1;
  }
  FILE *fp = fopen(out_path, "w");
  if (!fp) {
    fprintf(stderr, "Error: Could not open output file '%s' for writing: %s\n", out_path,
            strerror(errno));
    return 0;
  }
  const size_t cap = 1 << 22;
  char *buf = (char *)malloc(cap);
  if (!buf) return 1;
  char *p = buf;
  memcpy(p, "NODE_LIST", 9);
  p += 9;
  for (int i = 1; i <= n; ++i) {
    if ((size_t)(p - buf) + 32 > cap) {
      fwrite(buf, 1, (size_t)(p - buf), fp);
      p = buf;
    }
    *p++ = ' ';
    p = put_int(p, i);
  }
  *p++ = '\n';
  glibc_rand g;
  grand_seed(&g, (unsigned int)seed);
  const double rmax = (double)RAND_MAX;
  for (int step = 0; step < steps; ++step) {
    printf("Generating step %d/%d...\n", step + 1, steps);
    const int64_t t0 = (int64_t)base + (int64_t)step * step_size;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) {
        const double prob = (i % groups == j % groups) ? p_in : p_out;
        if (((double)grand_next(&g) / rmax) < prob) {
          int64_t a = t0 + grand_next(&g) % step_size;
          int64_t b = t0 + grand_next(&g) % step_size;
          if (a > b) {
            const int64_t t = a;
            a = b;
            b = t;
          }
          if ((size_t)(p - buf) + 96 > cap) {
            fwrite(buf, 1, (size_t)(p - buf), fp);
            p = buf;
          }
          p = put_int(p, i + 1);
          *p++ = ',';
          *p++ = ' ';
          p = put_int(p, j + 1);
          *p++ = ',';
          *p++ = ' ';
          p = put_iso(p, a);
          *p++ = ',';
          *p++ = ' ';
          p = put_iso(p, b);
          *p++ = ';';
          *p++ = '\n';
        }
      }
  }
  fwrite(buf, 1, (size_t)(p - buf), fp);
  free(buf);
  fclose(fp);
  printf("Temporal graph file generated: %s\n", out_path);
  return 0;
}
