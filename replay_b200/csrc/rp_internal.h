// Internal types shared by the host driver and the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <cstdlib>
#include <vector>

#include "../../include/replay.h"

namespace rp {

struct FlowThresholds {
  unsigned long long te, ti, tr;
  int te_all, ti_all, tr_all;
};

// ---- errors ---------------------------------------------------------------
void set_error(const char *fmt, ...);
rp_status cuda_fail(cudaError_t e, const char *what);
#define RP_TRY_CUDA(call)                                  \
  do {                                                     \
    cudaError_t _e = (call);                               \
    if (_e != cudaSuccess) return ::rp::cuda_fail(_e, #call); \
  } while (0)
#define RP_TRY(call)                 \
  do {                               \
    rp_status _s = (call);           \
    if (_s != RP_OK) return _s;      \
  } while (0)

// ---- device buffer ----------------------------------------------------------
// Device blocks released while no device work can touch them are kept for
// reuse instead of going back through cudaFree, whose device-wide wait and
// unmapping dominate closing a simulation or a graph and whose matching
// cudaMalloc calls dominate creating the next one.  An owner parks its
// buffers (ParkGuard) after synchronizing the device; DevBuf::alloc takes
// the smallest kept block of the current device that fits (at most twice
// the request); a failing cudaMalloc returns that device's kept blocks and
// retries.  At most kCacheBytes stay kept per device (the oldest go first);
// rp_release_cached_memory returns them all.
constexpr size_t kCacheBytes = size_t(8) << 30;
void *cache_take(int device, size_t n, size_t *cap);
void cache_put(int device, void *p, size_t cap);
void cache_trim(int device);  // -1: every device
extern thread_local int g_park;  // > 0: releases on this thread keep their blocks

// Declared before the buffers it covers (so it is destroyed after them) and
// armed once the device work that used them has completed: from then on the
// buffers released on this thread are kept instead of freed.
struct ParkGuard {
  bool armed = false;
  ParkGuard() = default;
  ParkGuard(const ParkGuard &) = delete;
  ParkGuard &operator=(const ParkGuard &) = delete;
  void arm() {
    if (!armed) {
      armed = true;
      ++g_park;
    }
  }
  // Waits for all work on `device` (the wait cudaFree would have made: work
  // a caller enqueued on its own streams may still read the buffers), then
  // arms; the caller's current device is left as it was.
  void arm_after_sync(int device) {
    int cur = 0;
    const bool have_cur = cudaGetDevice(&cur) == cudaSuccess;
    if (cudaSetDevice(device) == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess) arm();
    if (have_cur) cudaSetDevice(cur);
    (void)cudaGetLastError();
  }
  ~ParkGuard() {
    if (armed) --g_park;
  }
};

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  size_t cap = 0;     // bytes of the block behind ptr (>= bytes)
  int dev = 0;        // device of the block
  bool owned = true;  // false: a view of memory this buffer must not free
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  rp_status alloc(size_t n) {
    release();
    if (n == 0) n = 16;
    int d = 0;
    cudaGetDevice(&d);
    size_t c = 0;
    if (void *p = cache_take(d, n, &c)) {
      ptr = p;
      bytes = n;
      cap = c;
      dev = d;
      return RP_OK;
    }
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      cache_trim(d);
      e = cudaMalloc(&ptr, n);
    }
    if (e != cudaSuccess) {
      ptr = nullptr;
      (void)cudaGetLastError();
      set_error("cudaMalloc of %zu bytes failed: %s", n, cudaGetErrorString(e));
      return RP_ERR_NOMEM;
    }
    bytes = n;
    cap = n;
    dev = d;
    return RP_OK;
  }
  void release() {
    if (ptr && owned) {
      if (g_park > 0)
        cache_put(dev, ptr, cap);
      else
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
    cap = 0;
    owned = true;
  }
  // Exchanges the blocks of two buffers (pointer, sizes, device, ownership:
  // a block's size must travel with it, or it would be kept under the wrong
  // size).
  void swap(DevBuf &o) {
    std::swap(ptr, o.ptr);
    std::swap(bytes, o.bytes);
    std::swap(cap, o.cap);
    std::swap(dev, o.dev);
    std::swap(owned, o.owned);
  }
  // Points at memory owned elsewhere (no allocation; release() won't free it).
  void borrow(void *p, size_t n) {
    release();
    ptr = p;
    bytes = n;
    owned = false;
  }
  template <typename T>
  T *as() const {
    return static_cast<T *>(ptr);
  }
};

// ---- interval index -----------------------------------------------------------
// Contacts live in "stored coordinates" (the reference interval database's
// orientation rule, see graph.cpp) and are partitioned into duration classes:
// class 0 holds durations <= 1 s (including empty and inverted intervals),
// class c >= 1 holds durations in (2^(c-1), 2^c].  Inside a class contacts
// are ordered by start, so the candidates of a query [qs, qe) in class c are
// the contiguous run with start in (qs - 2^c, qe): two binary searches.
constexpr int kClasses = 64;

struct CandRange {
  int64_t lo;     // first candidate, index into the class-ordered arrays
  int64_t count;  // candidates in this class
  int64_t prefix; // candidates in earlier ranges of the same window
};

struct WinDesc {
  int64_t ws, we;        // window [ws, we)
  int64_t qs, qe;        // query actually run (mirrored when ws < 0)
  int64_t n_candidates;  // sum of range counts
  float scale;           // 1 / steps in the window (reference weight scale)
  int32_t range_off;     // first CandRange of this window
  int32_t n_ranges;
  int32_t may_truncate;  // candidates exceed the hit cap
};

struct Graph {
  int device = 0;
  int32_t n_nodes = 0, n_index = 0;
  int64_t n_contacts = 0, nlists = 0, n_malformed = 0;
  int64_t t_min = 0, t_max = 0;
  int32_t n_classes_used = 0;
  std::vector<int64_t> class_off;  // kClasses + 1 offsets
  std::vector<int64_t> h_cs;       // class-ordered stored starts
  DevBuf cs, ce;                   // int64 stored start / end, class order
  DevBuf cu, cv;                   // int32 endpoints (u <= v)
  DevBuf crank;                    // int32 position in (start asc, end desc) order
};

// Contacts read from a text file: malloc'd arrays of n entries in file
// order (u <= v, compressed indices), owned by this object until release().
struct ParsedContacts {
  int32_t n_nodes = 0, n_index = 0;
  int64_t n_malformed = 0, n = 0;
  int64_t *start = nullptr, *end = nullptr;
  int32_t *u = nullptr, *v = nullptr;
  ParsedContacts() = default;
  ParsedContacts(const ParsedContacts &) = delete;
  ParsedContacts &operator=(const ParsedContacts &) = delete;
  ~ParsedContacts() { release_all(); }
  void release_all() {
    free(start), free(end), free(u), free(v);
    start = end = nullptr;
    u = v = nullptr;
  }
  void release() { start = end = nullptr, u = v = nullptr; }  // ownership passed on
};
rp_status parse_contact_file(const char *path, ParsedContacts &out);
// Builds the device interval index of n contacts given in host memory
// (u[k] <= v[k]); ingest.cu.
rp_status graph_build_device(Graph &g, const int64_t *start, const int64_t *end,
                             const int32_t *u, const int32_t *v, int64_t n, int32_t n_nodes);

// Plans the query of one window: candidate ranges appended to `ranges`.
// Candidate ranges of window [ws, we) (at most kClasses, written to `ranges`,
// range_off = 0); returns their number.  plan_window appends them to a list.
int32_t plan_window_ranges(const Graph &g, int64_t ws, int64_t we, float scale, int64_t cap,
                           CandRange *ranges, WinDesc &out);
void plan_window(const Graph &g, int64_t ws, int64_t we, float scale,
                 int64_t cap, std::vector<CandRange> &ranges, WinDesc &out);

// ---- window builder ----------------------------------------------------------
struct Hit {
  int32_t rank;  // position in (start asc, end desc) order
  int32_t u;     // < 0: counts toward the hit cap but carries no weight
  int32_t v;
  int32_t w;     // int32 seconds or float bits
};

struct WindowWorkspace {
  int32_t n_nodes = 0;
  int64_t cap_hits = 0, cap_entries = 0;
  int32_t n_tiles = 0;
  DevBuf hits;      // Hit[cap_hits]
  DevBuf entries;   // int2 {col, weight}[cap_entries]
  DevBuf erank;     // int32[cap_entries]
  DevBuf tmp_e;     // int2[cap_entries]  radix ping-pong for hub rows
  DevBuf tmp_r;     // int32[cap_entries]
  DevBuf row_ptr;   // int32[n+1]
  DevBuf deg;       // int32[n] degree, then fill cursor
  DevBuf tiles;     // int32[n_tiles]
  DevBuf counters;  // u64[4]: recorded hits, long rows, spare, predicate hits
  DevBuf long_rows; // int32[n]
  DevBuf win;       // WinDesc[n_windows]
  DevBuf ranges;    // CandRange[...]
};

rp_status window_workspace_alloc(WindowWorkspace &w, int32_t n_nodes,
                                 int64_t cap_hits, int64_t n_windows,
                                 const std::vector<WinDesc> &wins,
                                 const std::vector<CandRange> &ranges);

// ---- mean-field replay (meanfield.cu) ----
struct MfRates {
  float beta, p_ei, p_ir, p_rs;
  int32_t has_exposed, ir_to_s;
};
int32_t mf_blocks(int32_t n);
void mf_step(const int32_t *rp, const int2 *ent, int32_t n, float scale, const MfRates *r,
             const float *sus, const float *x, float *xo, float *q_out, float *e_out,
             float *inc_part, cudaStream_t st);
void mf_incidence(const float *part, int32_t nblk, int32_t T, float *inc, cudaStream_t st);
void mf_adjoint(int32_t n, const int32_t *rp_c, const int2 *ent_c, const float *z_in,
                const float *a_in, const float *x, const float *q, const float *e,
                const float *ginc, int32_t tl, float scale, const MfRates *r, const float *sus,
                float *a_out, float *z_out, float *gsus, double *gpart, cudaStream_t st);
void mf_finish(const double *gpart, int32_t nblk, double *out, cudaStream_t st);

// ---- node-state text (text.cu) ----
int64_t text_line_bound(int32_t n_nodes);  // bytes of one line at most
void enqueue_states_text(const uint8_t *cls, int32_t n, int32_t r0, int32_t r1, int64_t ts,
                         int64_t node_digits, int64_t *rowlen, int64_t *rowoff, char *out,
                         cudaStream_t st);

// Scan tiles the window builder uses for n_nodes rows.
int32_t window_scan_tiles(int32_t n_nodes);

enum WeightKind { kWeightF32 = 0, kWeightI32 = 1 };

// Enqueues the CSR build of window `wi` into ws.row_ptr / ws.entries.
// sort_rows: order each row by (col, rank) and merge duplicates in place
// (merged-away entries keep their column with weight 0).
void enqueue_window_build(const Graph &g, WindowWorkspace &ws, int wi,
                          const WinDesc &desc, int64_t cap, int weight_kind,
                          bool sort_rows, cudaStream_t st);
// Compacts the sorted, merged CSR in ws into (row_ptr_out, entries_out):
// drops merged-away entries.  tmp_rows: int32[n+1] scratch.
void enqueue_window_compact(WindowWorkspace &ws, int32_t *row_ptr_out,
                            int2 *entries_out, cudaStream_t st);

// ---- kernels of the step loop -------------------------------------------------
struct StepConsts {
  uint32_t key0, key1;
  uint32_t rk[20];    // Philox round keys of (key0, key1)
  FlowThresholds th;  // p_ei, p_ir, p_rs as 64-bit fixed point
  float step_size;
  float neg_log_base;  // -logf(1 - infect_prob), countdown mode
  int32_t upper, medium, lower, E, I, R;  // countdown ranges / durations
  float p_ei, p_ir, p_rs;
  int32_t has_exposed, ir_to_s;
  float beta;
  const float *beta_r;  // device, may be null
  const float *sus;     // device, may be null
  uint32_t roff;        // replica offset of the stream layout (multiple of 32)
  int32_t *err;         // device flag set by a kernel that gave up a bounded wait
  int32_t hints;        // batched path: keep and use the per-item hint bytes
};

// Plain path (column-major N x M state, per-replica SpMV + elementwise).
void plain_init(int transition, void *state, int32_t n, int32_t m,
                float p0, int32_t k_exact, const StepConsts &c,
                cudaStream_t st);
void plain_spmv(int transition, const int32_t *row_ptr, const int2 *entries,
                const void *state, void *exposure, int32_t n, int32_t m,
                const StepConsts &c, cudaStream_t st);
void plain_transition(int transition, void *state, const void *exposure,
                      int32_t n, int32_t m, uint32_t step, float scale,
                      int32_t *counts_row, const StepConsts &c,
                      cudaStream_t st);
void plain_count(int transition, const void *state, int32_t n, int32_t m,
                 int32_t *counts_row, const StepConsts &c, cudaStream_t st);
void plain_classify(int transition, const void *state, int32_t n, int32_t m,
                    uint8_t *out, const StepConsts &c, cudaStream_t st);

// Batched path (bit-packed replica words).
struct PackedTask {
  int32_t row_begin, row_end;  // rows of one network
  int32_t slice;               // 32 four-word columns (128 words) per slice
  int32_t count_base;          // index of replica 0 of this network in counts
  int32_t stage;               // k_infect: CSR pairs staged per chunk (<= 768)
};
constexpr int32_t kStageDefault = 768;  // k_infect's staging buffer, in pairs
struct PackedLayout {
  int32_t n_nodes;
  int32_t words;      // words per node row, padded to a multiple of 4
  int32_t vwords;     // words holding replicas: ceil(m / 32)
  int32_t q4;         // four-word columns per row (words / 4)
  int32_t m;          // replicas per network
  uint32_t last_mask; // valid bits of word vwords - 1
  int32_t lpr;        // lanes per row (power of 2, <= 32)
  int32_t n_tasks;
  int32_t max_task_rows;  // rows of the tallest task
};
rp_status packed_prepare();  // kernel attributes, once per device
void packed_init(const PackedLayout &L, uint32_t *sa, uint32_t *sb,
                 uint32_t *mask, uint8_t *flag, float p0, int32_t k_exact,
                 const int32_t *net_first_row, const int32_t *net_rows,
                 int32_t n_nets, const StepConsts &c, cudaStream_t st);
// One step: exposure + infection draws (k_infect), then transitions, counts
// and the next infectious mask (k_flow).
void packed_infect(const PackedLayout &L, const PackedTask *tasks,
                   const int32_t *row_ptr, const int2 *entries,
                   const uint32_t *mask, const uint32_t *sa, const uint32_t *sb,
                   uint32_t *evs, uint8_t *flag, uint32_t step, float scale,
                   const StepConsts &c, cudaStream_t st);
void packed_flow(const PackedLayout &L, const PackedTask *tasks,
                 const int32_t *row_ptr, uint32_t *mask, uint32_t *sa,
                 uint32_t *sb, const uint32_t *evs, uint8_t *flag,
                 unsigned long long *ev_row, unsigned long long *rs_row,
                 uint32_t step, const StepConsts &c, cudaStream_t st);
// Batched countdown mode (countdown.cu): per-replica codes into the host's
// countdown table (next | class << 16 | infectious << 18), 1 or 2 bytes each.
rp_status cd_prepare();
void cd_init(const PackedLayout &L, const PackedTask *tasks, const uint32_t *infected,
             void *codes, int code_bytes, uint32_t *mask, const uint32_t *tab,
             uint32_t init_code, unsigned long long *init_counts, cudaStream_t st);
void cd_step(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
             const int2 *entries, const uint32_t *mask_in, uint32_t *mask_out, void *codes,
             int code_bytes, const uint32_t *tab, int32_t n_codes, uint32_t infect_code,
             unsigned long long *ev_row, uint32_t step, const StepConsts &c, cudaStream_t st);
void cd_finalize(const unsigned long long *init, const unsigned long long *ev, int32_t steps,
                 int32_t per_row, const int32_t *net_size, int32_t m, int32_t *counts,
                 cudaStream_t st);
void cd_classify(const PackedLayout &L, const void *codes, int code_bytes, const uint32_t *tab,
                 uint8_t *out, cudaStream_t st);
void packed_count(const PackedLayout &L, const PackedTask *tasks,
                  const uint32_t *sa, const uint32_t *sb,
                  unsigned long long *counts_row, cudaStream_t st);
void packed_finalize_events(const unsigned long long *init,
                            const unsigned long long *ev,
                            const unsigned long long *rs, int32_t steps,
                            int32_t per_row, const int32_t *net_size,
                            int32_t m, int32_t has_exposed, int32_t ir_to_s,
                            int32_t *counts, cudaStream_t st);
void packed_classify(const PackedLayout &L, const uint32_t *sa,
                     const uint32_t *sb, uint8_t *out, cudaStream_t st);
void packed_exposure(const int32_t *row_ptr, const int2 *entries, int32_t n,
                     const uint32_t *masks, int32_t words, int32_t m,
                     int64_t *exposure, cudaStream_t st);
void plain_spmv_f32_raw(const int32_t *row_ptr, const int32_t *col,
                        const float *val, int32_t n, const float *b, float *c,
                        int32_t m, cudaStream_t st);

}  // namespace rp

struct rp_graph {
  rp::ParkGuard park;  // destroyed after g: its blocks are kept for reuse
  rp::Graph g;
  double prep_ms = 0.0, build_ms = 0.0;  // creation phases (rp_graph_info)
  ~rp_graph() { park.arm_after_sync(g.device); }
};
