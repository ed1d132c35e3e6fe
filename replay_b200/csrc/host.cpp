// libreplay host driver: the C ABI of include/replay.h.
//
// Replaces the reference driver (tool/gpu_cpu_temporal_sim.cu:570-1185):
// schedule arithmetic, per-step window queries, CSR construction, the
// exposure product, transitions and count output -- with all per-step work
// enqueued on the device and captured once into a CUDA graph, so one replay
// is one graph launch.  No host synchronisation inside the step loop; only
// the (n_steps+1) x M x 4 counts leave the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "contact_prep.h"
#include "rp_internal.h"

namespace rp {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

rp_status cuda_fail(cudaError_t e, const char *what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  (void)cudaGetLastError();
  return RP_ERR_CUDA;
}

// ---- kept device blocks ------------------------------------------------------
thread_local int g_park = 0;

namespace {
struct KeptBlock {
  int device;
  size_t cap;
  void *ptr;
};
std::mutex g_cache_mu;
std::vector<KeptBlock> g_cache;  // oldest first

// cudaFree on the block's own device, restoring the caller's device
void free_on(int device, void *p) {
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  cudaFree(p);
  if (cur != device) cudaSetDevice(cur);
}
}  // namespace

void *cache_take(int device, size_t n, size_t *cap) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  size_t best = g_cache.size();
  for (size_t i = 0; i < g_cache.size(); ++i) {
    const KeptBlock &b = g_cache[i];
    if (b.device != device || b.cap < n || b.cap / 2 > n) continue;
    if (best == g_cache.size() || b.cap < g_cache[best].cap) best = i;
  }
  if (best == g_cache.size()) return nullptr;
  void *p = g_cache[best].ptr;
  *cap = g_cache[best].cap;
  g_cache.erase(g_cache.begin() + (std::ptrdiff_t)best);
  return p;
}

void cache_put(int device, void *p, size_t cap) {
  std::vector<KeptBlock> evict;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache.push_back(KeptBlock{device, cap, p});
    size_t kept = 0;
    for (const KeptBlock &b : g_cache)
      if (b.device == device) kept += b.cap;
    for (size_t i = 0; i < g_cache.size() && kept > kCacheBytes;) {
      if (g_cache[i].device == device) {
        kept -= g_cache[i].cap;
        evict.push_back(g_cache[i]);
        g_cache.erase(g_cache.begin() + (std::ptrdiff_t)i);
      } else {
        ++i;
      }
    }
  }
  for (const KeptBlock &b : evict) free_on(b.device, b.ptr);
}

void cache_trim(int device) {
  std::vector<KeptBlock> out;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (size_t i = 0; i < g_cache.size();) {
      if (device < 0 || g_cache[i].device == device) {
        out.push_back(g_cache[i]);
        g_cache.erase(g_cache.begin() + (std::ptrdiff_t)i);
      } else {
        ++i;
      }
    }
  }
  for (const KeptBlock &b : out) free_on(b.device, b.ptr);
}

namespace {

bool add_overflows(int64_t a, int64_t b) {
  return (b > 0 && a > INT64_MAX - b) || (b < 0 && a < INT64_MIN - b);
}

// Window start and timestamp of iteration `it` (gpu_cpu_temporal_sim.cu:860-902).
bool slice_start(int64_t start, float step, int64_t window, int32_t it, int64_t &ws,
                 int64_t &ts) {
  const double raw = (double)it * (double)step;
  if (raw > (double)INT64_MAX || raw < (double)INT64_MIN) return false;
  const int64_t off = (int64_t)llround(raw);
  if (add_overflows(start, off)) return false;
  int64_t net = (off / window) * window;
  if (off < 0 && (off % window)) net -= window;
  if (add_overflows(start, net)) return false;
  ws = start + net;
  ts = start + off;
  return true;
}

// Per-step windows, weight scales and timestamps (:859-959).
rp_status make_schedule(const rp_params &p, std::vector<int64_t> &ws,
                        std::vector<float> &scale, std::vector<int64_t> &ts) {
  const int32_t T = p.n_steps;
  ws.resize(T);
  scale.resize(T);
  ts.resize(T);
  if (p.window <= 0) {
    set_error("static network duration must be positive");
    return RP_ERR_ARG;
  }
  if (!(p.step_size > 0.0f)) {
    set_error("step size must be positive");
    return RP_ERR_ARG;
  }
  int64_t cached = 0;
  bool valid = false;
  int32_t steps = 1;
  for (int32_t it = 0; it < T; ++it) {
    int64_t cs, t;
    if (!slice_start(p.start_time, p.step_size, p.window, it, cs, t) ||
        add_overflows(cs, p.window)) {
      set_error("overflow computing the simulation time of step %d", it);
      return RP_ERR_RANGE;
    }
    if (!valid || cs != cached) {
      steps = 0;
      for (int32_t f = it; f < T; ++f) {
        int64_t fs, ft;
        if (!slice_start(p.start_time, p.step_size, p.window, f, fs, ft)) {
          set_error("overflow computing a future simulation time");
          return RP_ERR_RANGE;
        }
        if (fs != cs) break;
        ++steps;
      }
      cached = cs;
      valid = true;
    }
    ws[it] = cs;
    scale[it] = 1.0f / (float)steps;
    ts[it] = t;
  }
  return RP_OK;
}

// Countdown arithmetic of the reference, on the host (IEEE single
// precision, no contraction): c = (int)((float)c - step), c = (int)((float)base + step).
int32_t host_cd_sub(int32_t c, float step) { return (int32_t)((float)c - step); }
int32_t host_cd_add(int32_t base, float step) { return (int32_t)((float)base + step); }

// Summary class of a countdown value (tool/gpu_cpu_temporal_sim.cu:530-550).
uint32_t host_cd_class(int32_t c, int32_t E, int32_t I, int32_t R) {
  const int32_t upper = E + I + R;
  const int32_t elapsed = (c <= 0 || c > upper) ? 0 : (upper - c);
  if (c == 0) return 0;
  if (E > 0 && elapsed < E) return 1;
  if (I > 0 && elapsed < E + I) return 2;
  if (R > 0 && elapsed < E + I + R) return 3;
  return 0;
}

// The countdown values a replica can hold within n_steps steps, as codes
// (countdown.cu): code 0 is c == 0; the sequence from an infection (base
// E + I + R) and from an initial infection (base I + R) follow, each cut
// after n_steps + 2 values.  Entry: next code | class << 16 | infectious << 18.
struct CdTable {
  std::vector<uint32_t> tab;
  uint32_t infect_code = 0;  // code of a replica infected this step, after the step's decrement
  uint32_t init_code = 0;    // code of an initially infected replica at t0
  int code_bytes = 0;        // 1 or 2; 0 when the table is too large
};

void build_cd_table(const rp_params &p, CdTable &t) {
  const int32_t E = p.exposed_duration, I = p.infectious_duration, R = p.resistant_duration;
  const int32_t upper = E + I + R, medium = I + R, lower = R;
  const float step = p.step_size;
  const int64_t cap = (int64_t)(p.n_steps > 0 ? p.n_steps : 0) + 2;
  t.tab.assign(1, 0u);  // code 0: susceptible, stays
  auto entry = [&](int32_t c) {
    const uint32_t inf = (c > lower && c <= medium) ? 1u : 0u;
    return host_cd_class(c, E, I, R) << 16 | inf << 18;
  };
  auto sequence = [&](int32_t c) -> uint32_t {  // returns the first value's code
    const uint32_t first = (uint32_t)t.tab.size();
    for (int64_t k = 0; k < cap && c > 0 && t.tab.size() <= 65536; ++k) {
      const uint32_t code = (uint32_t)t.tab.size();
      t.tab.push_back(entry(c));
      int32_t nx = host_cd_sub(c, step);
      if (nx < 0) nx = 0;
      // next code: 0 when the countdown ends, itself at the cut (never
      // reached within the replay)
      const uint32_t next = nx == 0 ? 0u : (k + 1 < cap ? code + 1 : code);
      t.tab.back() |= next & 0xFFFFu;
      c = nx;
    }
    return t.tab.size() > first ? first : 0u;
  };
  const int32_t c_inf = host_cd_add(upper, step);
  const uint32_t inf_first = c_inf > 0 ? sequence(c_inf) : 0u;
  // the infection's value takes its first decrement in the same step
  t.infect_code = inf_first ? (t.tab[inf_first] & 0xFFFFu) : 0u;
  const int32_t c_init = host_cd_add(medium, step);
  t.init_code = c_init > 0 ? sequence(c_init) : 0u;
  t.code_bytes = t.tab.size() <= 256 ? 1 : (t.tab.size() <= 65536 ? 2 : 0);
}

int resolve_path(const rp_params &p) {
  if (p.path != RP_PATH_AUTO) return p.path;
  if (p.transition == RP_TRANSITION_GEOMETRIC) return RP_PATH_BATCHED;
  CdTable t;
  build_cd_table(p, t);
  return t.code_bytes ? RP_PATH_BATCHED : RP_PATH_PLAIN;
}

}  // namespace
}  // namespace rp

using namespace rp;

namespace {
double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

struct rp_sim {
  // destroyed after every buffer below: armed by the destructor once the
  // device is idle, so that the buffers are kept for reuse
  ParkGuard park;
  const Graph *g = nullptr;
  rp_params p{};
  int path = RP_PATH_PLAIN;
  int weight_kind = kWeightF32;
  int32_t N = 0, M = 0, T = 0;
  int64_t cap = 0;
  std::vector<int64_t> step_ws, step_ts;
  std::vector<float> step_scale;
  std::vector<int32_t> step_win;  // window index per step
  std::vector<WinDesc> wins;
  std::vector<CandRange> ranges;
  WindowWorkspace wsp;
  // per-step mode: window w + 1 is built on a side stream into the other
  // workspace while window w's steps run
  WindowWorkspace wsp2;
  bool overlap = false;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_built[2] = {nullptr, nullptr}, ev_free = nullptr, ev_join = nullptr;
  bool prebuilt = false;
  std::vector<int64_t> arena_rp_off, arena_ent_off;
  DevBuf arena_rp, arena_ent;
  int64_t prebuilt_nnz = 0;
  // plain state
  DevBuf state, exposure;
  // batched state
  DevBuf sa, sb, mask, evs, flag, tasks, ev, rs, init_counts;
  DevBuf mask2;  // countdown mode: the infectious masks alternate between steps
  DevBuf err;  // int32: set by a kernel that gave up a bounded wait
  // batched countdown state: per-replica codes into the countdown table
  DevBuf codes, cd_tab;
  CdTable cd;
  PackedLayout L{};
  DevBuf net_size, net_first, net_rows;
  int32_t n_nets = 1;
  std::vector<int32_t> net_bounds;  // n_nets + 1 node offsets (empty: one network)
  std::vector<int32_t> h_first, h_rows;  // per network: first row, rows
  std::vector<int32_t> task_rows;        // per network: rows of one task
  std::vector<int32_t> task_stage;       // per network: CSR pairs staged per chunk
  int32_t n_slices = 1;
  // node-state text mode (rp_sim_run_text)
  rp_text_cb text_cb = nullptr;
  void *text_user = nullptr;
  int32_t text_rows = 0;  // replica rows per text chunk
  int64_t node_digits = 0;
  DevBuf text_dev[2], text_rowlen, text_rowoff;
  char *text_host[2] = {nullptr, nullptr};
  int64_t *text_len_host = nullptr;
  cudaEvent_t text_ev[2] = {nullptr, nullptr};
  // shared
  DevBuf counts, beta_r, sus, classes;
  StepConsts c{};
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernels_per_run = 0;
  int64_t nnz_total = 0;
  double setup_ms = 0.0, alloc_ms = 0.0, prebuild_ms = 0.0, capture_ms = 0.0;

  ~rp_sim() {
    if (exec) cudaGraphExecDestroy(exec);
    if (stream) cudaStreamSynchronize(stream);
    if (side) {
      cudaStreamSynchronize(side);
      cudaStreamDestroy(side);
    }
    for (cudaEvent_t e : {ev_built[0], ev_built[1], ev_free, ev_join})
      if (e) cudaEventDestroy(e);
    for (int b = 0; b < 2; ++b) {
      if (text_host[b]) cudaFreeHost(text_host[b]);
      if (text_ev[b]) cudaEventDestroy(text_ev[b]);
    }
    if (text_len_host) cudaFreeHost(text_len_host);
    if (stream) cudaStreamDestroy(stream);
    if (g) park.arm_after_sync(g->device);
  }

  // Node-state CSV lines of one recorded step, formatted on the device in
  // chunks of replica rows; the host callback writes chunk k while the
  // device formats chunk k+1.
  rp_status emit_text(cudaStream_t st, int32_t step_index, int64_t ts) {
    int prev = -1;
    int64_t prev_len = 0;
    for (int32_t r0 = 0, k = 0; r0 < M; r0 += text_rows, ++k) {
      const int32_t r1 = std::min(M, r0 + text_rows);
      const int b = k & 1;
      enqueue_states_text(classes.as<uint8_t>(), N, r0, r1, ts, node_digits,
                          text_rowlen.as<int64_t>(), text_rowoff.as<int64_t>(),
                          text_dev[b].as<char>(), st);
      RP_TRY_CUDA(cudaMemcpyAsync(text_len_host + b, text_rowoff.as<int64_t>() + (r1 - r0),
                                  sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      if (prev >= 0) {
        RP_TRY_CUDA(cudaEventSynchronize(text_ev[prev]));
        if (text_cb(text_user, step_index, ts, text_host[prev], (size_t)prev_len) != 0) {
          set_error("text callback aborted the run");
          return RP_ERR_ARG;
        }
      }
      RP_TRY_CUDA(cudaStreamSynchronize(st));
      const int64_t len = text_len_host[b];
      RP_TRY_CUDA(cudaMemcpyAsync(text_host[b], text_dev[b].ptr, (size_t)len,
                                  cudaMemcpyDeviceToHost, st));
      RP_TRY_CUDA(cudaEventRecord(text_ev[b], st));
      prev = b;
      prev_len = len;
    }
    if (prev >= 0) {
      RP_TRY_CUDA(cudaEventSynchronize(text_ev[prev]));
      if (text_cb(text_user, step_index, ts, text_host[prev], (size_t)prev_len) != 0) {
        set_error("text callback aborted the run");
        return RP_ERR_ARG;
      }
    }
    return RP_OK;
  }

  WindowWorkspace &ws_of(int w) { return overlap && (w & 1) ? wsp2 : wsp; }
  const WindowWorkspace &ws_of(int w) const { return overlap && (w & 1) ? wsp2 : wsp; }
  const int32_t *rp_of(int t) const {
    if (prebuilt) return arena_rp.as<int32_t>() + arena_rp_off[step_win[t]];
    return ws_of(step_win[t]).row_ptr.as<int32_t>();
  }
  const int2 *ent_of(int t) const {
    if (prebuilt) return arena_ent.as<int2>() + arena_ent_off[step_win[t]];
    return ws_of(step_win[t]).entries.as<int2>();
  }

  // Optional event marks around kernel groups (rp_sim_profile).
  struct Marks {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;  // group kind of the interval ending at ev[i]
    cudaStream_t st;
    void mark(int k) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      cudaEventRecord(e, st);
      ev.push_back(e);
      kind.push_back(k);
    }
    ~Marks() {
      for (auto e : ev) cudaEventDestroy(e);
    }
  };
  enum { kMarkStart = 0, kMarkOther = 1, kMarkBuild = 2, kMarkSpmv = 3, kMarkStep = 4 };

  // Enqueues one whole replay.  With `cb`, per-step node states are copied
  // out and handed to the callback (not capturable).
  rp_status enqueue(cudaStream_t st, rp_state_cb cb, void *user, int *n_kernels,
                    Marks *mk = nullptr) {
    int k = 0;
    auto mark = [&](int kind) {
      if (mk) mk->mark(kind);
    };
    mark(kMarkStart);
    const int32_t rows = T + 1;
    std::vector<uint8_t> host_states;
    if (cb && !text_cb) host_states.resize((size_t)N * M);
    auto emit_states = [&](int32_t step_index, int64_t tstamp) -> rp_status {
      if (!cb && !text_cb) return RP_OK;
      if (path == RP_PATH_BATCHED && cd.code_bytes)
        cd_classify(L, codes.ptr, cd.code_bytes, cd_tab.as<uint32_t>(), classes.as<uint8_t>(),
                    st);
      else if (path == RP_PATH_BATCHED)
        packed_classify(L, sa.as<uint32_t>(), sb.as<uint32_t>(), classes.as<uint8_t>(), st);
      else
        plain_classify(p.transition, state.ptr, N, M, classes.as<uint8_t>(), c, st);
      if (text_cb) return emit_text(st, step_index, tstamp);
      RP_TRY_CUDA(cudaMemcpyAsync(host_states.data(), classes.ptr, host_states.size(),
                                  cudaMemcpyDeviceToHost, st));
      RP_TRY_CUDA(cudaStreamSynchronize(st));
      if (cb(user, step_index, tstamp, host_states.data(), N, M) != 0) {
        set_error("state callback aborted the run");
        return RP_ERR_ARG;
      }
      return RP_OK;
    };
    if (path == RP_PATH_PLAIN) {
      RP_TRY_CUDA(cudaMemsetAsync(counts.ptr, 0, counts.bytes, st));
      plain_init(p.transition, state.ptr, N, M, p.initial_infected, p.initial_count, c, st);
      plain_count(p.transition, state.ptr, N, M, counts.as<int32_t>(), c, st);
      k += 2 + (p.initial_count > 0);
    } else {
      RP_TRY_CUDA(cudaMemsetAsync(ev.ptr, 0, ev.bytes, st));
      // k_infect writes event words one by one; k_flow reads whole items
      if (evs.ptr) RP_TRY_CUDA(cudaMemsetAsync(evs.ptr, 0, evs.bytes, st));
      if (rs.ptr && p.p_rs > 0.0f) RP_TRY_CUDA(cudaMemsetAsync(rs.ptr, 0, rs.bytes, st));
      RP_TRY_CUDA(cudaMemsetAsync(init_counts.ptr, 0, init_counts.bytes, st));
      packed_init(L, sa.as<uint32_t>(), sb.as<uint32_t>(), mask.as<uint32_t>(),
                  flag.as<uint8_t>(), p.initial_infected, p.initial_count, net_first.as<int32_t>(),
                  net_rows.as<int32_t>(), n_nets, c, st);
      if (cd.code_bytes)  // countdown codes from the initial-infection plane
        cd_init(L, tasks.as<PackedTask>(), sa.as<uint32_t>(), codes.ptr, cd.code_bytes,
                mask.as<uint32_t>(), cd_tab.as<uint32_t>(), cd.init_code,
                init_counts.as<unsigned long long>(), st);
      else
        packed_count(L, tasks.as<PackedTask>(), sa.as<uint32_t>(), sb.as<uint32_t>(),
                     init_counts.as<unsigned long long>(), st);
      k += 2 + 2 * (p.initial_count > 0);
    }
    mark(kMarkOther);
    RP_TRY(emit_states(0, p.start_time));
    const int per_row = n_nets * M;
    const int n_win = (int)wins.size();
    auto build = [&](int w, cudaStream_t bs) {
      enqueue_window_build(*g, ws_of(w), w, wins[w], cap, weight_kind,
                           weight_kind == kWeightF32, bs);
      // k_hits, k_scan_tiles, k_scan_apply, k_fill (+ k_trunc, + the two row sorts)
      k += 4 + (wins[w].may_truncate ? 1 : 0) + (weight_kind == kWeightF32 ? 2 : 0);
    };
    bool side_used = false;
    if (!prebuilt && overlap && T > 0) {
      build(step_win[0], st);
      mark(kMarkBuild);
    }
    for (int32_t t = 0; t < T; ++t) {
      const int w = step_win[t];
      if (!prebuilt && (t == 0 || w != step_win[t - 1])) {
        if (!overlap) {
          build(w, st);
          mark(kMarkBuild);
        } else {
          if (t > 0) RP_TRY_CUDA(cudaStreamWaitEvent(st, ev_built[w & 1], 0));
          if (w + 1 < n_win) {
            // window w-1's steps, the last users of the other workspace, are
            // all enqueued before this point
            RP_TRY_CUDA(cudaEventRecord(ev_free, st));
            RP_TRY_CUDA(cudaStreamWaitEvent(side, ev_free, 0));
            build(w + 1, side);
            RP_TRY_CUDA(cudaEventRecord(ev_built[(w + 1) & 1], side));
            side_used = true;
          }
        }
      }
      if (path == RP_PATH_PLAIN) {
        plain_spmv(p.transition, rp_of(t), ent_of(t), state.ptr, exposure.ptr, N, M, c, st);
        mark(kMarkSpmv);
        plain_transition(p.transition, state.ptr, exposure.ptr, N, M, (uint32_t)t,
                         step_scale[t], counts.as<int32_t>() + (int64_t)(t + 1) * M * 4, c,
                         st);
        mark(kMarkStep);
        k += 2;
      } else {
        if (cd.code_bytes) {
          // countdown codes: the infectious masks alternate, step t reads
          // buffer t & 1 and writes every word of the other
          const uint32_t *m_in = (t & 1) ? mask2.as<uint32_t>() : mask.as<uint32_t>();
          uint32_t *m_out = (t & 1) ? mask.as<uint32_t>() : mask2.as<uint32_t>();
          cd_step(L, tasks.as<PackedTask>(), rp_of(t), ent_of(t), m_in, m_out, codes.ptr,
                  cd.code_bytes, cd_tab.as<uint32_t>(), (int32_t)cd.tab.size(), cd.infect_code,
                  ev.as<unsigned long long>() + (int64_t)t * per_row, (uint32_t)t, c, st);
          mark(kMarkStep);
          k += 1;
        } else {
          packed_infect(L, tasks.as<PackedTask>(), rp_of(t), ent_of(t), mask.as<uint32_t>(),
                        sa.as<uint32_t>(), sb.as<uint32_t>(), evs.as<uint32_t>(),
                        flag.as<uint8_t>(), (uint32_t)t, step_scale[t], c, st);
          mark(kMarkSpmv);
          packed_flow(L, tasks.as<PackedTask>(), rp_of(t), mask.as<uint32_t>(),
                      sa.as<uint32_t>(), sb.as<uint32_t>(), evs.as<uint32_t>(),
                      flag.as<uint8_t>(), ev.as<unsigned long long>() + (int64_t)t * per_row,
                      p.p_rs > 0.0f ? rs.as<unsigned long long>() + (int64_t)t * per_row
                                    : nullptr,
                      (uint32_t)t, c, st);
          mark(kMarkStep);
          k += 2;
        }
      }
      RP_TRY(emit_states(t + 1, step_ts[t]));
    }
    if (side_used) {  // join the side stream (required to end a capture)
      RP_TRY_CUDA(cudaEventRecord(ev_join, side));
      RP_TRY_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    }
    if (path == RP_PATH_BATCHED && cd.code_bytes) {
      cd_finalize(init_counts.as<unsigned long long>(), ev.as<unsigned long long>(), T, per_row,
                  net_size.as<int32_t>(), M, counts.as<int32_t>(), st);
      k += 1;
      mark(kMarkOther);
    } else if (path == RP_PATH_BATCHED) {
      packed_finalize_events(init_counts.as<unsigned long long>(),
                             ev.as<unsigned long long>(),
                             p.p_rs > 0.0f ? rs.as<unsigned long long>() : nullptr, T,
                             per_row, net_size.as<int32_t>(), M, p.has_exposed, p.ir_to_s,
                             counts.as<int32_t>(), st);
      k += 1;
      mark(kMarkOther);
    }
    (void)rows;
    RP_TRY_CUDA(cudaGetLastError());
    if (n_kernels) *n_kernels = k;
    return RP_OK;
  }
};

// Mean-field replay: the schedule and prebuilt window CSRs of a geometric
// simulation, FP32 probability planes, checkpoints every K steps.
struct rp_meanfield {
  ParkGuard park;  // destroyed last (see rp_sim)
  rp_sim base;
  int32_t N = 0, T = 0, K = 24, nblk = 0, n_ckpt = 0;
  MfRates rates{};
  bool have_forward = false, has_sus = false;
  DevBuf ckpt;                 // n_ckpt x 4N: x_0, x_K, x_2K, ...
  DevBuf xa, xb;               // 4N ping-pong
  DevBuf seg_x, seg_q, seg_e;  // recomputed segment: K x 4N, K x N, K x N
  DevBuf inc_part;             // T x blocks incidence partials
  DevBuf a0, a1, z0, z1;       // adjoint ping-pong (4N), coupling terms (N)
  DevBuf gpart;                // blocks x 4 FP64 scalar-gradient partials
  DevBuf sus;                  // copy of the forward's susceptibility (ones when none)
  DevBuf ones;                 // N x 1.0f
  DevBuf d_rates;              // MfRates read by the kernels
  DevBuf inc, ginc;            // T incidences; T incidence gradients
  DevBuf gx0, gsus, grates;    // adjoint outputs
  // the whole forward and the whole adjoint, captured once on `cap` (all
  // pointers internal) and replayed on the caller's stream
  cudaStream_t cap = nullptr;
  cudaGraphExec_t fwd = nullptr, bwd = nullptr;
  const float *final_x = nullptr;  // x_T inside the forward's buffers
  ~rp_meanfield() {
    if (fwd) cudaGraphExecDestroy(fwd);
    if (bwd) cudaGraphExecDestroy(bwd);
    if (cap) cudaStreamDestroy(cap);
    if (base.g) park.arm_after_sync(base.g->device);
  }
};

namespace {

// Builds every window's canonical CSR once into the arena.
rp_status prebuild(rp_sim &s) {
  const int nw = (int)s.wins.size();
  const int32_t N = s.N;
  std::vector<int64_t> nnz(nw, 0);
  DevBuf tmp_rp, tmp_ent;
  RP_TRY(tmp_rp.alloc(sizeof(int32_t) * ((size_t)N + 1)));
  RP_TRY(tmp_ent.alloc(sizeof(int2) * (size_t)s.wsp.cap_entries));
  cudaStream_t st = s.stream;
  for (int w = 0; w < nw; ++w) {
    enqueue_window_build(*s.g, s.wsp, w, s.wins[w], s.cap, s.weight_kind, true, st);
    enqueue_window_compact(s.wsp, tmp_rp.as<int32_t>(), tmp_ent.as<int2>(), st);
    int32_t total = 0;
    RP_TRY_CUDA(cudaMemcpyAsync(&total, tmp_rp.as<int32_t>() + N, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, st));
    RP_TRY_CUDA(cudaStreamSynchronize(st));
    nnz[w] = total;
  }
  s.arena_rp_off.resize(nw);
  s.arena_ent_off.resize(nw);
  int64_t ent = 0;
  for (int w = 0; w < nw; ++w) {
    s.arena_rp_off[w] = (int64_t)w * (N + 1);
    s.arena_ent_off[w] = ent;
    ent += nnz[w];
  }
  s.prebuilt_nnz = ent;
  RP_TRY(s.arena_rp.alloc(sizeof(int32_t) * (size_t)nw * ((size_t)N + 1)));
  // two spare pairs for the step kernel's 16-byte bulk staging
  RP_TRY(s.arena_ent.alloc(sizeof(int2) * (size_t)(ent + 2)));
  for (int w = 0; w < nw; ++w) {
    enqueue_window_build(*s.g, s.wsp, w, s.wins[w], s.cap, s.weight_kind, true, st);
    enqueue_window_compact(s.wsp, s.arena_rp.as<int32_t>() + s.arena_rp_off[w],
                           s.arena_ent.as<int2>() + s.arena_ent_off[w], st);
  }
  RP_TRY_CUDA(cudaStreamSynchronize(st));
  return RP_OK;
}

rp_status sim_setup(rp_sim &s, const Graph &g, const rp_params &p) {
  s.g = &g;
  s.p = p;
  s.N = g.n_nodes;
  s.M = p.n_replicas;
  s.T = p.n_steps;
  if (s.M <= 0 || s.T < 0) {
    set_error("n_replicas must be positive and n_steps non-negative");
    return RP_ERR_ARG;
  }
  if (p.transition != RP_TRANSITION_COUNTDOWN && p.transition != RP_TRANSITION_GEOMETRIC) {
    set_error("unknown transition mode %d", p.transition);
    return RP_ERR_ARG;
  }
  s.path = resolve_path(p);
  if (s.path != RP_PATH_PLAIN && s.path != RP_PATH_BATCHED) {
    set_error("unknown path %d", p.path);
    return RP_ERR_ARG;
  }
  if (s.path == RP_PATH_BATCHED && p.transition == RP_TRANSITION_COUNTDOWN) {
    build_cd_table(p, s.cd);
    if (!s.cd.code_bytes) {
      set_error("countdown values of this replay need more than 65536 codes; the batched "
                "path stores at most 65536 (use the plain path)");
      return RP_ERR_RANGE;
    }
  }
  if (p.initial_count > s.N) {
    set_error("initial_count %d exceeds the %d nodes", p.initial_count, s.N);
    return RP_ERR_ARG;
  }
  if (s.path == RP_PATH_PLAIN && (int64_t)s.M > 4 * 65535) {
    set_error("the plain path supports at most 262140 replicas");
    return RP_ERR_RANGE;
  }
  // per-(network, replica) event counters hold 21-bit fields
  int32_t largest = s.N;
  if (!s.net_bounds.empty()) {
    largest = 0;
    for (size_t k = 0; k + 1 < s.net_bounds.size(); ++k)
      largest = std::max(largest, s.net_bounds[k + 1] - s.net_bounds[k]);
  }
  if (s.path == RP_PATH_BATCHED && largest >= (1 << 21)) {
    set_error("batched path counts networks of fewer than 2^21 nodes");
    return RP_ERR_RANGE;
  }
  s.weight_kind = p.transition == RP_TRANSITION_COUNTDOWN ? kWeightF32 : kWeightI32;
  if (s.weight_kind == kWeightI32 && p.window > INT32_MAX) {
    set_error("integer contact-second weights need a window of at most 2^31-1 s");
    return RP_ERR_RANGE;
  }
  RP_TRY_CUDA(cudaSetDevice(g.device));
  RP_TRY_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));

  // ---- schedule and windows ----
  RP_TRY(make_schedule(p, s.step_ws, s.step_scale, s.step_ts));
  s.cap = p.ncls_cap ? (g.nlists > 0 ? g.nlists : 1) : INT64_MAX;
  s.step_win.resize(s.T);
  int64_t max_cand = 0;
  for (int32_t t = 0; t < s.T; ++t) {
    if (t == 0 || s.step_ws[t] != s.step_ws[t - 1]) {
      WinDesc d{};
      plan_window(g, s.step_ws[t], s.step_ws[t] + p.window, s.step_scale[t], s.cap, s.ranges,
                  d);
      s.wins.push_back(d);
      if (d.n_candidates > max_cand) max_cand = d.n_candidates;
    }
    s.step_win[t] = (int32_t)s.wins.size() - 1;
  }
  // per-item hint bytes pay off on windows with many pairs per row (two per
  // hit; a window's candidates bound its hits from above): at least 4 N
  // candidates
  s.c.hints = 0;
  for (const WinDesc &d : s.wins)
    if (d.n_candidates >= 4 * (int64_t)s.N) s.c.hints = 1;
  if (max_cand > (int64_t)INT32_MAX / 2) {
    set_error("a window has %lld candidate contacts; at most 2^30 are supported",
              (long long)max_cand);
    return RP_ERR_RANGE;
  }
  RP_TRY(window_workspace_alloc(s.wsp, s.N, max_cand, (int64_t)s.wins.size(), s.wins,
                                s.ranges));

  // ---- constants ----
  s.c.key0 = (uint32_t)p.seed;
  s.c.key1 = (uint32_t)(p.seed >> 32);
  for (int r = 0; r < 10; ++r) {
    s.c.rk[2 * r] = s.c.key0 + (uint32_t)r * 0x9E3779B9u;
    s.c.rk[2 * r + 1] = s.c.key1 + (uint32_t)r * 0xBB67AE85u;
  }
  s.c.step_size = p.step_size;
  s.c.neg_log_base = -logf(1.0f - p.infect_prob);
  s.c.E = p.exposed_duration;
  s.c.I = p.infectious_duration;
  s.c.R = p.resistant_duration;
  s.c.upper = p.exposed_duration + p.infectious_duration + p.resistant_duration;
  s.c.medium = p.infectious_duration + p.resistant_duration;
  s.c.lower = p.resistant_duration;
  auto thr = [](float pr, int &all) -> unsigned long long {
    all = pr >= 1.0f;
    if (!(pr > 0.0f) || pr >= 1.0f) return 0ull;
    return (unsigned long long)ldexp((double)pr, 64);
  };
  s.c.th.te = thr(p.p_ei, s.c.th.te_all);
  s.c.th.ti = thr(p.p_ir, s.c.th.ti_all);
  s.c.th.tr = thr(p.p_rs, s.c.th.tr_all);
  s.c.p_ei = p.p_ei;
  s.c.p_ir = p.p_ir;
  s.c.p_rs = p.p_rs;
  if (p.replica_offset < 0 || p.replica_offset % 32 != 0) {
    set_error("replica_offset must be a non-negative multiple of 32");
    return RP_ERR_ARG;
  }
  s.c.roff = (uint32_t)p.replica_offset;
  s.c.has_exposed = p.has_exposed;
  s.c.ir_to_s = p.ir_to_s;
  s.c.beta = p.beta;
  if (p.beta_per_replica) {
    RP_TRY(s.beta_r.alloc(sizeof(float) * s.M));
    RP_TRY_CUDA(cudaMemcpy(s.beta_r.ptr, p.beta_per_replica, sizeof(float) * s.M,
                           cudaMemcpyHostToDevice));
    s.c.beta_r = s.beta_r.as<float>();
  }
  if (p.susceptibility) {
    RP_TRY(s.sus.alloc(sizeof(float) * (size_t)s.N));
    RP_TRY_CUDA(cudaMemcpy(s.sus.ptr, p.susceptibility, sizeof(float) * s.N,
                           cudaMemcpyHostToDevice));
    s.c.sus = s.sus.as<float>();
  }
  return RP_OK;
}

// Rows per batched task: about one wave of CTAs (148 SMs x 3), between 32
// and 4,096 rows (a task stages its row pointers in shared memory).  Sparse
// batches of many networks reach the cap: there a task is a short chain of
// global round trips, and fewer, taller tasks shorten the step.
constexpr int64_t kTaskRowsDefaultMax = 4096;
int32_t rows_per_task(int32_t n_rows, int32_t n_slices) {
  const int64_t target_tasks = 148 * 3;
  int64_t rows = ((int64_t)n_rows * n_slices + target_tasks - 1) / target_tasks;
  if (rows < 32) rows = 32;
  if (rows > kTaskRowsDefaultMax) rows = kTaskRowsDefaultMax;
  return (int32_t)rows;
}

// Tiles every network's rows into tasks of s.task_rows[net] rows x one
// 32-column slice (a task never spans two networks: its counters flush to
// the network's count row) and uploads them.
rp_status upload_tasks(rp_sim &s) {
  std::vector<PackedTask> tasks;
  const int32_t M = s.M;
  for (int net = 0; net < s.n_nets; ++net) {
    const int32_t rpt = s.task_rows[net];
    const int32_t f = s.h_first[net], e = f + s.h_rows[net];
    for (int32_t r0 = f; r0 < e; r0 += rpt)
      for (int32_t sl = 0; sl < s.n_slices; ++sl)
        tasks.push_back(PackedTask{r0, std::min(r0 + rpt, e), sl, net * M, s.task_stage[net]});
  }
  if (s.tasks.bytes < sizeof(PackedTask) * tasks.size())
    RP_TRY(s.tasks.alloc(sizeof(PackedTask) * tasks.size()));
  RP_TRY_CUDA(cudaMemcpy(s.tasks.ptr, tasks.data(), sizeof(PackedTask) * tasks.size(),
                         cudaMemcpyHostToDevice));
  s.L.n_tasks = (int32_t)tasks.size();
  s.L.max_task_rows = 0;
  for (const PackedTask &t : tasks)
    s.L.max_task_rows = std::max(s.L.max_task_rows, t.row_end - t.row_begin);
  return RP_OK;
}

rp_status alloc_state(rp_sim &s) {
  const int32_t N = s.N, M = s.M, T = s.T;
  const int64_t NM = (int64_t)N * M;
  RP_TRY(s.err.alloc(sizeof(int32_t)));
  RP_TRY_CUDA(cudaMemset(s.err.ptr, 0, sizeof(int32_t)));
  s.c.err = s.err.as<int32_t>();
  RP_TRY(s.counts.alloc(sizeof(int32_t) * (size_t)(T + 1) * (size_t)M * 4 * s.n_nets));
  if (s.p.record_node_states) RP_TRY(s.classes.alloc((size_t)NM));
  if (s.path == RP_PATH_PLAIN) {
    const size_t sb = s.p.transition == RP_TRANSITION_COUNTDOWN ? 4 : 1;
    const size_t eb = s.p.transition == RP_TRANSITION_COUNTDOWN ? 4 : 8;
    RP_TRY(s.state.alloc(sb * (size_t)NM));
    RP_TRY(s.exposure.alloc(eb * (size_t)NM));
    return RP_OK;
  }
  // batched layout: rows padded to 4-word columns, 32 columns per slice
  PackedLayout &L = s.L;
  L.n_nodes = N;
  L.m = M;
  L.vwords = (M + 31) / 32;
  L.words = (L.vwords + 3) / 4 * 4;
  L.q4 = L.words / 4;
  L.last_mask = (M % 32) ? ((1u << (M % 32)) - 1u) : 0xFFFFFFFFu;
  int lpr = 1;
  while (lpr < L.q4 && lpr < 32) lpr <<= 1;
  L.lpr = lpr;
  const int32_t n_slices = (L.q4 + 31) / 32;
  s.n_slices = n_slices;
  std::vector<int32_t> first, rows, size;
  if (s.net_bounds.empty()) {  // one network: rows [0, N)
    first.push_back(0);
    rows.push_back(N);
    size.push_back(N);
  } else {
    for (int net = 0; net < s.n_nets; ++net) {
      first.push_back(s.net_bounds[net]);
      rows.push_back(s.net_bounds[net + 1] - s.net_bounds[net]);
      size.push_back(s.net_bounds[net + 1] - s.net_bounds[net]);
    }
  }
  s.h_first = first;
  s.h_rows = rows;
  // default tiles: about 3 tasks per SM over the whole batch's rows (a
  // network smaller than a task is one task); rp_sim_autotune refines them
  s.task_rows.assign(s.n_nets, rows_per_task(N, n_slices));
  s.task_stage.assign(s.n_nets, kStageDefault);
  RP_TRY(packed_prepare());
  RP_TRY(cd_prepare());
  const size_t plane = sizeof(uint32_t) * (size_t)N * L.words;
  RP_TRY(s.sa.alloc(plane));
  RP_TRY(s.sb.alloc(plane));
  RP_TRY(s.mask.alloc(plane));
  RP_TRY(s.flag.alloc(((size_t)N * L.q4 + 3) / 4 * 4));
  if (!s.cd.code_bytes) RP_TRY(s.evs.alloc(plane));
  if (s.cd.code_bytes) {
    RP_TRY(s.mask2.alloc(plane));
    RP_TRY(s.codes.alloc((size_t)s.cd.code_bytes * 32 * (size_t)N * L.words));
    RP_TRY(s.cd_tab.alloc(sizeof(uint32_t) * s.cd.tab.size()));
    RP_TRY_CUDA(cudaMemcpy(s.cd_tab.ptr, s.cd.tab.data(), sizeof(uint32_t) * s.cd.tab.size(),
                           cudaMemcpyHostToDevice));
  }
  RP_TRY(upload_tasks(s));
  const size_t per_row = (size_t)s.n_nets * M;
  RP_TRY(s.ev.alloc(sizeof(unsigned long long) * per_row * (size_t)(T > 0 ? T : 1)));
  if (s.p.p_rs > 0.0f)
    RP_TRY(s.rs.alloc(sizeof(unsigned long long) * per_row * (size_t)(T > 0 ? T : 1)));
  RP_TRY(s.init_counts.alloc(sizeof(unsigned long long) * per_row));
  RP_TRY(s.net_first.alloc(sizeof(int32_t) * first.size()));
  RP_TRY(s.net_rows.alloc(sizeof(int32_t) * rows.size()));
  RP_TRY(s.net_size.alloc(sizeof(int32_t) * size.size()));
  RP_TRY_CUDA(cudaMemcpy(s.net_first.ptr, first.data(), sizeof(int32_t) * first.size(),
                         cudaMemcpyHostToDevice));
  RP_TRY_CUDA(cudaMemcpy(s.net_rows.ptr, rows.data(), sizeof(int32_t) * rows.size(),
                         cudaMemcpyHostToDevice));
  RP_TRY_CUDA(cudaMemcpy(s.net_size.ptr, size.data(), sizeof(int32_t) * size.size(),
                         cudaMemcpyHostToDevice));
  return RP_OK;
}

rp_status capture(rp_sim &s) {
  cudaGraph_t graph = nullptr;
  RP_TRY_CUDA(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
  rp_status st = s.enqueue(s.stream, nullptr, nullptr, &s.kernels_per_run);
  cudaError_t e = cudaStreamEndCapture(s.stream, &graph);
  if (st != RP_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&s.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  return RP_OK;
}

}  // namespace

// Captures stream work enqueued by `body` on m.cap into an executable graph.
template <typename F>
rp_status mf_capture(rp_meanfield &m, cudaGraphExec_t &exec, F body) {
  cudaGraph_t graph = nullptr;
  RP_TRY_CUDA(cudaStreamBeginCapture(m.cap, cudaStreamCaptureModeThreadLocal));
  rp_status st = body(m.cap);
  cudaError_t e = cudaStreamEndCapture(m.cap, &graph);
  if (st != RP_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (mean-field)");
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate (mean-field)");
  return RP_OK;
}

// The forward over every step from ckpt[0]: states ping-pong in xa/xb,
// checkpoints every K steps, per-step incidence into m.inc.
rp_status mf_capture_forward(rp_meanfield &m) {
  const int32_t N = m.N, T = m.T;
  const size_t plane = sizeof(float) * 4 * (size_t)N;
  float *ck = m.ckpt.as<float>();
  float *pp[2] = {m.xa.as<float>(), m.xb.as<float>()};
  m.final_x = T > 0 ? pp[(T - 1) & 1] : ck;
  return mf_capture(m, m.fwd, [&](cudaStream_t st) -> rp_status {
    const float *x = ck;
    for (int32_t t = 0; t < T; ++t) {
      float *nxt = pp[t & 1];
      mf_step(m.base.rp_of(t), m.base.ent_of(t), N, m.base.step_scale[t],
              m.d_rates.as<MfRates>(), m.sus.as<float>(), x, nxt, nullptr, nullptr,
              m.inc_part.as<float>() + (size_t)t * m.nblk, st);
      if ((t + 1) % m.K == 0 && t + 1 < T)
        RP_TRY_CUDA(cudaMemcpyAsync(ck + (size_t)((t + 1) / m.K) * 4 * N, nxt, plane,
                                    cudaMemcpyDeviceToDevice, st));
      x = nxt;
    }
    mf_incidence(m.inc_part.as<float>(), m.nblk, T, m.inc.as<float>(), st);
    return RP_OK;
  });
}

// The adjoint from y = a0 (dL/dx_T) and m.ginc (dL/dincidence) back to
// dL/dx_0 (gx0), with dL/ds (gsus) and the FP64 rate gradients (grates):
// per checkpoint segment the states, exp(-beta s e) and scaled exposures
// are recomputed, then one kernel per reverse step.
rp_status mf_capture_backward(rp_meanfield &m) {
  const int32_t N = m.N, T = m.T, K = m.K;
  const size_t plane = sizeof(float) * 4 * (size_t)N;
  return mf_capture(m, m.bwd, [&](cudaStream_t st) -> rp_status {
    const float *sus = m.sus.as<float>();
    const MfRates *r = m.d_rates.as<MfRates>();
    RP_TRY_CUDA(cudaMemsetAsync(m.gpart.ptr, 0, m.gpart.bytes, st));
    RP_TRY_CUDA(cudaMemsetAsync(m.gsus.ptr, 0, sizeof(float) * (size_t)N, st));
    float *a[2] = {m.a0.as<float>(), m.a1.as<float>()};
    float *z[2] = {m.z0.as<float>(), m.z1.as<float>()};
    int ai = 0;
    const float *ck = m.ckpt.as<float>();
    float *sx = m.seg_x.as<float>(), *sq = m.seg_q.as<float>(), *se = m.seg_e.as<float>();
    // x of step t within the recomputed segment starting at c0
    auto seg_state = [&](int32_t c0, int32_t t) -> const float * {
      return t == c0 ? ck + (size_t)(c0 / K) * 4 * N : sx + (size_t)(t - c0) * 4 * N;
    };
    for (int32_t t = T - 1; t >= 0; --t) {
      const int32_t c0 = (t / K) * K;
      if (t == T - 1 || t == c0 + K - 1) {
        for (int32_t u = c0; u <= t; ++u) {
          float *xo = u + 1 <= t ? sx + (size_t)(u + 1 - c0) * 4 * N : m.xa.as<float>();
          mf_step(m.base.rp_of(u), m.base.ent_of(u), N, m.base.step_scale[u], r, sus,
                  seg_state(c0, u), xo, sq + (size_t)(u - c0) * N, se + (size_t)(u - c0) * N,
                  m.inc_part.as<float>() + (size_t)u * m.nblk, st);
        }
      }
      const bool couple = t + 1 < T;
      mf_adjoint(N, couple ? m.base.rp_of(t + 1) : nullptr,
                 couple ? m.base.ent_of(t + 1) : nullptr, z[(t + 1) & 1], a[ai],
                 seg_state(c0, t), sq + (size_t)(t - c0) * N, se + (size_t)(t - c0) * N,
                 m.ginc.as<float>(), t, m.base.step_scale[t], r, sus, a[ai ^ 1], z[t & 1],
                 m.gsus.as<float>(), m.gpart.as<double>(), st);
      ai ^= 1;
    }
    if (T > 0)
      mf_adjoint(N, m.base.rp_of(0), m.base.ent_of(0), z[0], a[ai], nullptr, nullptr, nullptr,
                 nullptr, 0, 1.0f, r, sus, m.gx0.as<float>(), nullptr, nullptr, nullptr, st);
    else
      RP_TRY_CUDA(cudaMemcpyAsync(m.gx0.ptr, a[ai], plane, cudaMemcpyDeviceToDevice, st));
    mf_finish(m.gpart.as<double>(), m.nblk, m.grates.as<double>(), st);
    return RP_OK;
  });
}

// Fails when a kernel of the last replay gave up a bounded wait (the flag is
// sticky until read here).
rp_status check_kernel_flag(rp_sim &s, cudaStream_t st) {
  int32_t flag = 0;
  RP_TRY_CUDA(cudaMemcpyAsync(&flag, s.err.ptr, sizeof(flag), cudaMemcpyDeviceToHost, st));
  RP_TRY_CUDA(cudaStreamSynchronize(st));
  if (flag) {
    RP_TRY_CUDA(cudaMemsetAsync(s.err.ptr, 0, sizeof(int32_t), st));
    set_error("a step kernel gave up waiting for its staged copies; results are invalid");
    return RP_ERR_DEVICE;
  }
  return RP_OK;
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

RP_API const char *rp_last_error(void) { return g_err; }
RP_API const char *rp_version(void) { return "replay-b200 0.1 (sm_100a)"; }
RP_API void rp_release_cached_memory(void) { cache_trim(-1); }

RP_API rp_status rp_graph_load_text(const char *path, int device, rp_graph **out) {
  if (!path || !out) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  *out = nullptr;
  std::unique_ptr<rp_graph> h(new rp_graph());
  ParsedContacts pc;
  const auto t0 = std::chrono::steady_clock::now();
  {
    // The device's context (a few hundred milliseconds to create, and
    // needing no input) is created on a helper thread while the file is
    // parsed; errors surface at the first device call below.
    struct Joined {
      std::thread t;
      ~Joined() {
        if (t.joinable()) t.join();
      }
    } warm{std::thread([device] {
      if (cudaSetDevice(device) == cudaSuccess) cudaFree(nullptr);
    })};
    RP_TRY(parse_contact_file(path, pc));
  }
  h->g.device = device;
  h->g.n_index = pc.n_index;
  h->g.n_malformed = pc.n_malformed;
  h->prep_ms = ms_since(t0);
  const auto t1 = std::chrono::steady_clock::now();
  RP_TRY(graph_build_device(h->g, pc.start, pc.end, pc.u, pc.v, pc.n, pc.n_nodes));
  RP_TRY_CUDA(cudaDeviceSynchronize());
  h->build_ms = ms_since(t1);
  *out = h.release();
  return RP_OK;
}

RP_API rp_status rp_parse_contacts(const char *path, int32_t *n_nodes, int32_t *n_index,
                                   int64_t *n_contacts, int64_t *n_malformed, int64_t **start,
                                   int64_t **end, int32_t **u, int32_t **v) {
  if (!path || !n_nodes || !n_index || !n_contacts || !n_malformed || !start || !end || !u || !v) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  *start = *end = nullptr;
  *u = *v = nullptr;
  *n_contacts = 0;
  ParsedContacts pc;
  RP_TRY(parse_contact_file(path, pc));
  *n_nodes = pc.n_nodes;
  *n_index = pc.n_index;
  *n_malformed = pc.n_malformed;
  *start = pc.start, *end = pc.end, *u = pc.u, *v = pc.v;
  *n_contacts = pc.n;
  pc.release();  // the caller frees the arrays with rp_free
  return RP_OK;
}

RP_API void rp_free(void *p) { free(p); }

RP_API rp_status rp_graph_from_arrays(const int64_t *start, const int64_t *end,
                                      const int32_t *u, const int32_t *v, int64_t n_contacts,
                                      int32_t n_nodes, int device, rp_graph **out) {
  if (!out || n_contacts < 0 || n_nodes <= 0 ||
      (n_contacts > 0 && (!start || !end || !u || !v))) {
    set_error("invalid graph arrays");
    return RP_ERR_ARG;
  }
  *out = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<int32_t> uu(n_contacts), vv(n_contacts);
  int32_t n_index = 0;
  const int threads = (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  const int64_t bad = prep_contacts(u, v, n_contacts, n_nodes, uu.data(), vv.data(), &n_index,
                                    threads);
  if (bad >= 0) {
    set_error("contact %lld joins node outside [0, %d)", (long long)bad, n_nodes);
    return RP_ERR_ARG;
  }
  std::unique_ptr<rp_graph> h(new rp_graph());
  h->g.device = device;
  h->g.n_index = n_index;
  h->prep_ms = ms_since(t0);
  const auto t1 = std::chrono::steady_clock::now();
  RP_TRY(graph_build_device(h->g, start, end, uu.data(), vv.data(), n_contacts, n_nodes));
  RP_TRY_CUDA(cudaDeviceSynchronize());
  h->build_ms = ms_since(t1);
  *out = h.release();
  return RP_OK;
}

RP_API rp_status rp_graph_get_info(const rp_graph *h, rp_graph_info *o) {
  if (!h || !o) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  const Graph &g = h->g;
  o->n_nodes = g.n_nodes;
  o->n_index = g.n_index;
  o->n_contacts = g.n_contacts;
  o->nlists = g.nlists;
  o->n_malformed = g.n_malformed;
  o->t_min = g.t_min;
  o->t_max = g.t_max;
  o->n_classes = g.n_classes_used;
  o->device = g.device;
  o->prep_ms = h->prep_ms;
  o->build_ms = h->build_ms;
  return RP_OK;
}

RP_API void rp_graph_free(rp_graph *h) { delete h; }

RP_API rp_status rp_window_csr(rp_graph *h, int64_t ws, int64_t we, float scale,
                               int32_t weight_kind, int32_t ncls_cap, int32_t *row_ptr,
                               int32_t *col, void *val, int64_t capacity, int64_t *nnz,
                               int64_t *n_hits) {
  if (!h || !row_ptr || !nnz || !n_hits || we <= ws ||
      (weight_kind != kWeightF32 && weight_kind != kWeightI32)) {
    set_error("invalid window CSR request");
    return RP_ERR_ARG;
  }
  const Graph &g = h->g;
  if (weight_kind == kWeightI32 && we - ws > INT32_MAX) {
    set_error("integer weights need a window of at most 2^31-1 s");
    return RP_ERR_RANGE;
  }
  RP_TRY_CUDA(cudaSetDevice(g.device));
  const int64_t cap = ncls_cap ? (g.nlists > 0 ? g.nlists : 1) : INT64_MAX;
  std::vector<WinDesc> wins(1);
  std::vector<CandRange> ranges;
  plan_window(g, ws, we, scale, cap, ranges, wins[0]);
  WindowWorkspace w;
  RP_TRY(window_workspace_alloc(w, g.n_nodes, wins[0].n_candidates, 1, wins, ranges));
  DevBuf out_rp, out_ent;
  RP_TRY(out_rp.alloc(sizeof(int32_t) * ((size_t)g.n_nodes + 1)));
  RP_TRY(out_ent.alloc(sizeof(int2) * (size_t)w.cap_entries));
  cudaStream_t st = nullptr;
  enqueue_window_build(g, w, 0, wins[0], cap, weight_kind, true, st);
  unsigned long long hits_raw = 0;
  RP_TRY_CUDA(cudaMemcpyAsync(&hits_raw, w.counters.as<unsigned long long>() + 3,
                              sizeof(hits_raw), cudaMemcpyDeviceToHost, st));
  enqueue_window_compact(w, out_rp.as<int32_t>(), out_ent.as<int2>(), st);
  RP_TRY_CUDA(cudaMemcpyAsync(row_ptr, out_rp.ptr, sizeof(int32_t) * ((size_t)g.n_nodes + 1),
                              cudaMemcpyDeviceToHost, st));
  RP_TRY_CUDA(cudaStreamSynchronize(st));
  const int64_t total = row_ptr[g.n_nodes];
  *nnz = total;
  *n_hits = (int64_t)hits_raw < cap ? (int64_t)hits_raw : cap;
  if (total > capacity) {
    set_error("CSR has %lld entries, capacity %lld", (long long)total, (long long)capacity);
    return RP_ERR_RANGE;
  }
  if (total > 0) {
    std::vector<int2> ent((size_t)total);
    RP_TRY_CUDA(cudaMemcpy(ent.data(), out_ent.ptr, sizeof(int2) * (size_t)total,
                           cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < total; ++k) {
      if (col) col[k] = ent[k].x;
      if (val) static_cast<int32_t *>(val)[k] = ent[k].y;
    }
  }
  return RP_OK;
}

RP_API void rp_params_default(rp_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->struct_size = sizeof(rp_params);
  p->n_replicas = 1000;
  p->n_steps = 42;
  p->step_size = 3600.0f;
  p->start_time = 946713600;
  p->window = 3600;
  p->transition = RP_TRANSITION_COUNTDOWN;
  p->path = RP_PATH_AUTO;
  p->csr_mode = RP_CSR_PER_STEP;
  p->ncls_cap = 1;
  p->seed = 1;
  p->has_exposed = 1;
}

RP_API rp_status rp_sim_create(const rp_graph *h, const rp_params *p, rp_sim **out) {
  return rp_sim_create_batch(h, p, nullptr, 1, out);
}

RP_API rp_status rp_sim_create_batch(const rp_graph *h, const rp_params *p,
                                     const int32_t *net_first, int32_t n_networks,
                                     rp_sim **out) {
  if (!h || !p || !out) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  if (p->struct_size != sizeof(rp_params)) {
    set_error("rp_params.struct_size mismatch (%u, expected %zu)", p->struct_size,
              sizeof(rp_params));
    return RP_ERR_ARG;
  }
  *out = nullptr;
  std::unique_ptr<rp_sim> s(new rp_sim());
  if (net_first) {
    const int32_t N = h->g.n_nodes;
    if (n_networks < 1 || net_first[0] != 0 || net_first[n_networks] != N) {
      set_error("network offsets must start at 0 and end at the graph's %d nodes", N);
      return RP_ERR_ARG;
    }
    int32_t smallest = N;
    for (int32_t k = 0; k < n_networks; ++k) {
      const int32_t nk = net_first[k + 1] - net_first[k];
      if (nk <= 0) {
        set_error("network %d has no nodes (offsets must increase)", k);
        return RP_ERR_ARG;
      }
      smallest = nk < smallest ? nk : smallest;
    }
    if (n_networks > 1) {
      if (resolve_path(*p) != RP_PATH_BATCHED) {
        set_error("a multi-network batch runs on the batched path");
        return RP_ERR_ARG;
      }
      if (p->ncls_cap) {
        set_error("the reference's hit cap belongs to one network's index; set ncls_cap = 0 "
                  "for a multi-network batch");
        return RP_ERR_ARG;
      }
      if (p->initial_count > smallest) {
        set_error("initial_count %d exceeds the smallest network (%d nodes)", p->initial_count,
                  smallest);
        return RP_ERR_ARG;
      }
    }
    s->n_nets = n_networks;
    s->net_bounds.assign(net_first, net_first + n_networks + 1);
  } else if (n_networks != 1) {
    set_error("network offsets missing");
    return RP_ERR_ARG;
  }
  auto t0 = std::chrono::steady_clock::now();
  RP_TRY(sim_setup(*s, h->g, *p));
  s->setup_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  RP_TRY(alloc_state(*s));
  s->alloc_ms = ms_since(t0);
  s->prebuilt = p->csr_mode == RP_CSR_PREBUILT;
  t0 = std::chrono::steady_clock::now();
  if (s->prebuilt) {
    RP_TRY(prebuild(*s));
    s->prebuild_ms = ms_since(t0);
  } else if (s->wins.size() > 1) {
    int64_t max_cand = 0;
    for (const WinDesc &d : s->wins) max_cand = std::max(max_cand, d.n_candidates);
    RP_TRY(window_workspace_alloc(s->wsp2, s->N, max_cand, (int64_t)s->wins.size(), s->wins,
                                  s->ranges));
    RP_TRY_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&s->ev_built[0], &s->ev_built[1], &s->ev_free, &s->ev_join})
      RP_TRY_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    s->overlap = true;
    s->setup_ms += ms_since(t0);
  }
  for (int32_t t = 0; t < s->T; ++t) {
    // nnz multiplied per step (for the roofline); per-step mode counts the
    // candidate bound, replaced by exact values when prebuilt.
    if (s->prebuilt) {
      const int w = s->step_win[t];
      const int64_t next = (w + 1 < (int)s->wins.size()) ? s->arena_ent_off[w + 1]
                                                         : s->prebuilt_nnz;
      s->nnz_total += next - s->arena_ent_off[w];
    }
  }
  t0 = std::chrono::steady_clock::now();
  if (!p->record_node_states) RP_TRY(capture(*s));
  s->capture_ms = ms_since(t0);
  *out = s.release();
  return RP_OK;
}

RP_API void rp_sim_free(rp_sim *s) { delete s; }

RP_API rp_status rp_sim_enqueue(rp_sim *s, void *stream) {
  if (!s) {
    set_error("null simulation");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (s->exec) {
    RP_TRY_CUDA(cudaGraphLaunch(s->exec, st));
    return RP_OK;
  }
  return s->enqueue(st, nullptr, nullptr, nullptr);
}

RP_API rp_status rp_sim_counts(rp_sim *s, int32_t *counts) {
  if (!s || !counts) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  RP_TRY_CUDA(cudaDeviceSynchronize());
  RP_TRY(check_kernel_flag(*s, s->stream));
  RP_TRY_CUDA(cudaMemcpy(counts, s->counts.ptr, s->counts.bytes, cudaMemcpyDeviceToHost));
  return RP_OK;
}

RP_API rp_status rp_sim_run(rp_sim *s, int32_t *counts, rp_state_cb cb, void *user) {
  if (!s || !counts) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  if (s->p.record_node_states && cb) {
    RP_TRY(s->enqueue(s->stream, cb, user, nullptr));
  } else if (s->exec) {
    RP_TRY_CUDA(cudaGraphLaunch(s->exec, s->stream));
  } else {
    RP_TRY(s->enqueue(s->stream, nullptr, nullptr, nullptr));
  }
  RP_TRY_CUDA(cudaMemcpyAsync(counts, s->counts.ptr, s->counts.bytes, cudaMemcpyDeviceToHost,
                              s->stream));
  RP_TRY(check_kernel_flag(*s, s->stream));
  return RP_OK;
}

RP_API rp_status rp_sim_run_text(rp_sim *s, int32_t *counts, rp_text_cb cb, void *user) {
  if (!s || !counts || !cb) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  if (!s->p.record_node_states) {
    set_error("rp_sim_run_text needs a simulation created with record_node_states");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  if (!s->text_host[0]) {  // chunk buffers: about 64 MB of text per chunk
    const int64_t line = text_line_bound(s->N);
    const int64_t per_row = line * (int64_t)s->N;
    s->text_rows = (int32_t)std::max<int64_t>(1, std::min<int64_t>(s->M, (64ll << 20) / per_row));
    const size_t bytes = (size_t)(per_row * s->text_rows);
    for (int b = 0; b < 2; ++b) {
      RP_TRY(s->text_dev[b].alloc(bytes));
      RP_TRY_CUDA(cudaMallocHost(&s->text_host[b], bytes));
      RP_TRY_CUDA(cudaEventCreateWithFlags(&s->text_ev[b], cudaEventDisableTiming));
    }
    RP_TRY_CUDA(cudaMallocHost(&s->text_len_host, 2 * sizeof(int64_t)));
    RP_TRY(s->text_rowlen.alloc(sizeof(int64_t) * (size_t)s->text_rows));
    RP_TRY(s->text_rowoff.alloc(sizeof(int64_t) * ((size_t)s->text_rows + 1)));
    int64_t d = 0;
    for (int64_t i = 0, p10 = 10, nd = 1; i < s->N; ++i) {
      if (i == p10) {
        p10 *= 10;
        ++nd;
      }
      d += nd;
    }
    s->node_digits = d;
  }
  s->text_cb = cb;
  s->text_user = user;
  rp_status st = s->enqueue(s->stream, nullptr, nullptr, nullptr);
  s->text_cb = nullptr;
  s->text_user = nullptr;
  RP_TRY(st);
  RP_TRY_CUDA(cudaMemcpyAsync(counts, s->counts.ptr, s->counts.bytes, cudaMemcpyDeviceToHost,
                              s->stream));
  RP_TRY(check_kernel_flag(*s, s->stream));
  return RP_OK;
}

RP_API rp_status rp_sim_timestamps(rp_sim *s, int64_t *ts) {
  if (!s || !ts) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  ts[0] = s->p.start_time;
  for (int32_t t = 0; t < s->T; ++t) ts[t + 1] = s->step_ts[t];
  return RP_OK;
}

RP_API rp_status rp_sim_get_info(const rp_sim *s, rp_sim_info *o) {
  if (!s || !o) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  o->path = s->path;
  o->words = s->path == RP_PATH_BATCHED ? s->L.words : 0;
  o->n_windows = (int32_t)s->wins.size();
  o->kernels_per_run = s->kernels_per_run;
  int64_t mc = 0;
  for (auto &w : s->wins) mc = w.n_candidates > mc ? w.n_candidates : mc;
  o->max_candidates = mc;
  o->prebuilt_nnz = s->prebuilt_nnz;
  int64_t bytes = 0;
  const DevBuf *bufs[] = {&s->arena_rp, &s->arena_ent, &s->state, &s->exposure, &s->sa,
                          &s->sb, &s->mask, &s->mask2, &s->evs, &s->flag, &s->err,
                          &s->codes, &s->cd_tab,
                          &s->tasks, &s->ev, &s->rs,
                          &s->init_counts, &s->counts, &s->beta_r, &s->sus, &s->classes,
                          &s->wsp.hits, &s->wsp.entries, &s->wsp.erank, &s->wsp.tmp_e,
                          &s->wsp.tmp_r, &s->wsp.row_ptr, &s->wsp.deg, &s->wsp.tiles,
                          &s->wsp.long_rows};
  for (auto b : bufs) bytes += (int64_t)b->bytes;
  o->device_bytes = bytes;
  o->nnz_total = s->nnz_total;
  o->setup_ms = s->setup_ms;
  o->alloc_ms = s->alloc_ms;
  o->prebuild_ms = s->prebuild_ms;
  o->capture_ms = s->capture_ms;
  return RP_OK;
}

RP_API rp_status rp_sim_profile(rp_sim *s, rp_profile *out) {
  if (!s || !out) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  RP_TRY_CUDA(cudaStreamSynchronize(s->stream));
  rp_sim::Marks mk;
  mk.st = s->stream;
  int nk = 0;
  RP_TRY(s->enqueue(s->stream, nullptr, nullptr, &nk, &mk));
  RP_TRY_CUDA(cudaStreamSynchronize(s->stream));
  memset(out, 0, sizeof(*out));
  for (size_t i = 1; i < mk.ev.size(); ++i) {
    float ms = 0.0f;
    RP_TRY_CUDA(cudaEventElapsedTime(&ms, mk.ev[i - 1], mk.ev[i]));
    out->total_ms += ms;
    switch (mk.kind[i]) {
      case rp_sim::kMarkBuild: out->build_ms += ms; out->build_launches++; break;
      case rp_sim::kMarkSpmv: out->spmv_ms += ms; out->spmv_launches++; break;
      case rp_sim::kMarkStep: out->step_ms += ms; out->step_launches++; break;
      default: out->other_ms += ms; break;
    }
  }
  out->kernels = nk;
  return RP_OK;
}

RP_API rp_status rp_sim_profile_steps(rp_sim *s, float *step_ms) {
  if (!s || !step_ms) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  RP_TRY_CUDA(cudaStreamSynchronize(s->stream));
  rp_sim::Marks mk;
  mk.st = s->stream;
  int nk = 0;
  RP_TRY(s->enqueue(s->stream, nullptr, nullptr, &nk, &mk));
  RP_TRY_CUDA(cudaStreamSynchronize(s->stream));
  int t = 0;
  for (size_t i = 1; i < mk.ev.size(); ++i) {
    float ms = 0.0f;
    RP_TRY_CUDA(cudaEventElapsedTime(&ms, mk.ev[i - 1], mk.ev[i]));
    if (mk.kind[i] == rp_sim::kMarkSpmv && t < s->T) step_ms[t] = ms;
    if (mk.kind[i] == rp_sim::kMarkStep && t < s->T) {
      step_ms[t] += ms;
      ++t;
    }
  }
  return RP_OK;
}

RP_API rp_status rp_exposure_spmv_f32(const int32_t *d_row_ptr, const int32_t *d_col,
                                      const float *d_val, int32_t n_nodes,
                                      const float *d_infectious, float *d_exposure,
                                      int32_t n_replicas, void *stream) {
  if (!d_row_ptr || n_nodes <= 0 || n_replicas <= 0 || !d_infectious || !d_exposure) {
    set_error("invalid SpMV arguments");
    return RP_ERR_ARG;
  }
  plain_spmv_f32_raw(d_row_ptr, d_col, d_val, n_nodes, d_infectious, d_exposure, n_replicas,
                     static_cast<cudaStream_t>(stream));
  RP_TRY_CUDA(cudaGetLastError());
  return RP_OK;
}

RP_API rp_status rp_exposure_spmm_packed(const int32_t *d_row_ptr, const int32_t *d_entries,
                                         int32_t n_nodes, const uint32_t *d_masks,
                                         int32_t words, int32_t n_replicas,
                                         int64_t *d_exposure, void *stream) {
  if (!d_row_ptr || n_nodes <= 0 || n_replicas <= 0 || words != (n_replicas + 31) / 32 ||
      !d_masks || !d_exposure) {
    set_error("invalid packed SpMM arguments");
    return RP_ERR_ARG;
  }
  packed_exposure(d_row_ptr, reinterpret_cast<const int2 *>(d_entries), n_nodes, d_masks,
                  words, n_replicas, d_exposure, static_cast<cudaStream_t>(stream));
  RP_TRY_CUDA(cudaGetLastError());
  return RP_OK;
}

// ---- tile autotuner --------------------------------------------------------

RP_API rp_status rp_sim_autotune(rp_sim *s, int32_t probe_steps, rp_tune_result *out) {
  if (!s || !out) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  if (s->path != RP_PATH_BATCHED) {
    set_error("the autotuner tiles the batched path");
    return RP_ERR_ARG;
  }
  if (s->p.record_node_states) {
    set_error("autotune a simulation created without record_node_states");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(s->g->device));
  const int32_t T_full = s->T;
  const int32_t probe = probe_steps < 1 ? 1 : (probe_steps > T_full ? T_full : probe_steps);
  cudaEvent_t e0, e1;
  RP_TRY_CUDA(cudaEventCreate(&e0));
  RP_TRY_CUDA(cudaEventCreate(&e1));
  int probes = 0;
  // device time of the replay's first `probe` steps (second of two eager runs)
  auto time_probe = [&](double &ms) -> rp_status {
    s->T = probe;
    rp_status st = RP_OK;
    for (int rep = 0; rep < 2 && st == RP_OK; ++rep) {
      if (rep == 1) cudaEventRecord(e0, s->stream);
      st = s->enqueue(s->stream, nullptr, nullptr, nullptr);
    }
    s->T = T_full;
    RP_TRY(st);
    RP_TRY_CUDA(cudaEventRecord(e1, s->stream));
    RP_TRY_CUDA(cudaEventSynchronize(e1));
    float f = 0.0f;
    RP_TRY_CUDA(cudaEventElapsedTime(&f, e0, e1));
    ms = f;
    ++probes;
    return RP_OK;
  };
  // size buckets: floor(log2 rows) of each network
  std::vector<int32_t> bucket(s->n_nets), blist;
  for (int k = 0; k < s->n_nets; ++k) {
    int32_t b = 0;
    while ((2 << b) <= s->h_rows[k]) ++b;
    bucket[k] = b;
    if (std::find(blist.begin(), blist.end(), b) == blist.end()) blist.push_back(b);
  }
  std::sort(blist.begin(), blist.end(), [](int a, int b) { return a > b; });
  if (blist.size() > 32) {
    set_error("more than 32 network-size buckets");
    return RP_ERR_RANGE;
  }
  double best = 0.0;
  rp_status st = time_probe(best);
  const double ms_default = best;
  static const int32_t kCand[] = {32, 64, 128, 256, 512, 1024, 2048, 4096};
  static const int32_t kStageCand[] = {192, 384};
  std::vector<int32_t> chosen(blist.size(), 0), chosen_stage(blist.size(), 0);
  for (size_t bi = 0; bi < blist.size() && st == RP_OK; ++bi) {
    std::vector<int32_t> keep = s->task_rows;
    for (int32_t cand : kCand) {
      std::vector<int32_t> saved = s->task_rows;
      for (int k = 0; k < s->n_nets; ++k)
        if (bucket[k] == blist[bi]) s->task_rows[k] = cand;
      double ms = 0.0;
      st = upload_tasks(*s);
      if (st == RP_OK) st = time_probe(ms);
      if (st != RP_OK) break;
      if (ms < best * 0.98) {
        best = ms;
        keep = s->task_rows;
        chosen[bi] = cand;
      }
      s->task_rows = saved;
    }
    s->task_rows = keep;
    // then the staging depth, with the bucket's chosen task height
    std::vector<int32_t> keep_stage = s->task_stage;
    for (int32_t cand : kStageCand) {
      if (st != RP_OK) break;
      std::vector<int32_t> saved = s->task_stage;
      for (int k = 0; k < s->n_nets; ++k)
        if (bucket[k] == blist[bi]) s->task_stage[k] = cand;
      double ms = 0.0;
      st = upload_tasks(*s);
      if (st == RP_OK) st = time_probe(ms);
      if (st != RP_OK) break;
      if (ms < best * 0.98) {
        best = ms;
        keep_stage = s->task_stage;
        chosen_stage[bi] = cand;
      }
      s->task_stage = saved;
    }
    s->task_stage = keep_stage;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  RP_TRY(st);
  RP_TRY(upload_tasks(*s));
  if (s->exec) {
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
  }
  RP_TRY(capture(*s));
  memset(out, 0, sizeof(*out));
  out->n_buckets = (int32_t)blist.size();
  for (size_t bi = 0; bi < blist.size(); ++bi) {
    out->bucket_log2[bi] = blist[bi];
    out->rows_per_task[bi] = chosen[bi];
    out->stage_pairs[bi] = chosen_stage[bi];
  }
  out->probe_steps = probe;
  out->probes = probes;
  out->ms_default = ms_default;
  out->ms_tuned = best;
  return RP_OK;
}

// ---- mean-field replay --------------------------------------------------

RP_API rp_status rp_meanfield_create(const rp_graph *h, const rp_params *p,
                                     int32_t checkpoint_every, rp_meanfield **out) {
  if (!h || !p || !out) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  if (p->struct_size != sizeof(rp_params)) {
    set_error("rp_params.struct_size mismatch (%u, expected %zu)", p->struct_size,
              sizeof(rp_params));
    return RP_ERR_ARG;
  }
  if (checkpoint_every <= 0) {
    set_error("checkpoint interval must be positive");
    return RP_ERR_ARG;
  }
  *out = nullptr;
  std::unique_ptr<rp_meanfield> m(new rp_meanfield());
  rp_params q = *p;
  q.n_replicas = 32;
  q.transition = RP_TRANSITION_GEOMETRIC;
  q.path = RP_PATH_BATCHED;
  q.csr_mode = RP_CSR_PREBUILT;
  q.initial_count = 0;
  q.beta_per_replica = nullptr;
  q.susceptibility = nullptr;
  rp_sim &b = m->base;
  RP_TRY(sim_setup(b, h->g, q));
  b.prebuilt = true;
  RP_TRY(prebuild(b));
  const int32_t N = b.N, T = b.T;
  m->N = N;
  m->T = T;
  m->K = checkpoint_every < (T > 0 ? T : 1) ? checkpoint_every : (T > 0 ? T : 1);
  m->nblk = mf_blocks(N);
  m->n_ckpt = T > 0 ? (T + m->K - 1) / m->K : 1;
  const size_t plane = sizeof(float) * 4 * (size_t)N;
  RP_TRY(m->ckpt.alloc(plane * m->n_ckpt));
  RP_TRY(m->xa.alloc(plane));
  RP_TRY(m->xb.alloc(plane));
  RP_TRY(m->seg_x.alloc(plane * m->K));
  RP_TRY(m->seg_q.alloc(sizeof(float) * (size_t)N * m->K));
  RP_TRY(m->seg_e.alloc(sizeof(float) * (size_t)N * m->K));
  RP_TRY(m->inc_part.alloc(sizeof(float) * (size_t)m->nblk * (T > 0 ? T : 1)));
  RP_TRY(m->a0.alloc(plane));
  RP_TRY(m->a1.alloc(plane));
  RP_TRY(m->z0.alloc(sizeof(float) * (size_t)N));
  RP_TRY(m->z1.alloc(sizeof(float) * (size_t)N));
  RP_TRY(m->gpart.alloc(sizeof(double) * 4 * (size_t)m->nblk));
  RP_TRY(m->sus.alloc(sizeof(float) * (size_t)N));
  RP_TRY(m->ones.alloc(sizeof(float) * (size_t)N));
  {
    std::vector<float> one((size_t)N, 1.0f);
    RP_TRY_CUDA(cudaMemcpy(m->ones.ptr, one.data(), sizeof(float) * (size_t)N,
                           cudaMemcpyHostToDevice));
  }
  RP_TRY(m->d_rates.alloc(sizeof(MfRates)));
  RP_TRY(m->inc.alloc(sizeof(float) * (size_t)(T > 0 ? T : 1)));
  RP_TRY(m->ginc.alloc(sizeof(float) * (size_t)(T > 0 ? T : 1)));
  RP_TRY(m->gx0.alloc(plane));
  RP_TRY(m->gsus.alloc(sizeof(float) * (size_t)N));
  RP_TRY(m->grates.alloc(sizeof(double) * 4));
  RP_TRY_CUDA(cudaStreamCreateWithFlags(&m->cap, cudaStreamNonBlocking));
  m->rates.has_exposed = p->has_exposed;
  m->rates.ir_to_s = p->ir_to_s;
  *out = m.release();
  return RP_OK;
}

RP_API void rp_meanfield_free(rp_meanfield *m) { delete m; }

RP_API rp_status rp_meanfield_forward(rp_meanfield *m, const float *d_x0, float beta,
                                      const float *d_sus, float p_ei, float p_ir, float p_rs,
                                      float *d_incidence, float *d_xT, void *stream) {
  if (!m || !d_x0) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  auto unit = [](float v) { return v >= 0.0f && v <= 1.0f; };
  if (!(beta >= 0.0f) || !unit(p_ei) || !unit(p_ir) || !unit(p_rs)) {
    set_error("beta must be >= 0 and the rates in [0, 1]");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(m->base.g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int32_t N = m->N, T = m->T;
  const size_t plane = sizeof(float) * 4 * (size_t)N;
  m->rates.beta = beta;
  m->rates.p_ei = p_ei;
  m->rates.p_ir = p_ir;
  m->rates.p_rs = p_rs;
  m->has_sus = d_sus != nullptr;
  if (!m->fwd) RP_TRY(mf_capture_forward(*m));
  // inputs into the graph's fixed buffers (a missing susceptibility is a
  // vector of ones: the products it enters are then exact)
  RP_TRY_CUDA(cudaMemcpyAsync(m->d_rates.ptr, &m->rates, sizeof(MfRates), cudaMemcpyHostToDevice,
                              st));
  RP_TRY_CUDA(cudaMemcpyAsync(m->sus.ptr, d_sus ? d_sus : m->ones.as<float>(),
                              sizeof(float) * (size_t)N, cudaMemcpyDeviceToDevice, st));
  RP_TRY_CUDA(cudaMemcpyAsync(m->ckpt.ptr, d_x0, plane, cudaMemcpyDeviceToDevice, st));
  RP_TRY_CUDA(cudaGraphLaunch(m->fwd, st));
  if (d_incidence && T > 0)
    RP_TRY_CUDA(cudaMemcpyAsync(d_incidence, m->inc.ptr, sizeof(float) * (size_t)T,
                                cudaMemcpyDeviceToDevice, st));
  if (d_xT) RP_TRY_CUDA(cudaMemcpyAsync(d_xT, m->final_x, plane, cudaMemcpyDeviceToDevice, st));
  RP_TRY_CUDA(cudaGetLastError());
  m->have_forward = true;
  return RP_OK;
}

RP_API rp_status rp_meanfield_backward(rp_meanfield *m, const float *d_grad_incidence,
                                       const float *d_grad_xT, float *d_grad_x0,
                                       float *d_grad_sus, double *d_grad_rates, void *stream) {
  if (!m || !d_grad_x0) {
    set_error("null argument");
    return RP_ERR_ARG;
  }
  if (!m->have_forward) {
    set_error("rp_meanfield_backward needs a preceding rp_meanfield_forward");
    return RP_ERR_ARG;
  }
  RP_TRY_CUDA(cudaSetDevice(m->base.g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int32_t N = m->N, T = m->T;
  const size_t plane = sizeof(float) * 4 * (size_t)N;
  if (!m->bwd) RP_TRY(mf_capture_backward(*m));
  // inputs into the graph's fixed buffers: a missing gradient is zero
  if (d_grad_xT)
    RP_TRY_CUDA(cudaMemcpyAsync(m->a0.ptr, d_grad_xT, plane, cudaMemcpyDeviceToDevice, st));
  else
    RP_TRY_CUDA(cudaMemsetAsync(m->a0.ptr, 0, plane, st));
  if (T > 0) {
    if (d_grad_incidence)
      RP_TRY_CUDA(cudaMemcpyAsync(m->ginc.ptr, d_grad_incidence, sizeof(float) * (size_t)T,
                                  cudaMemcpyDeviceToDevice, st));
    else
      RP_TRY_CUDA(cudaMemsetAsync(m->ginc.ptr, 0, sizeof(float) * (size_t)T, st));
  }
  RP_TRY_CUDA(cudaGraphLaunch(m->bwd, st));
  RP_TRY_CUDA(cudaMemcpyAsync(d_grad_x0, m->gx0.ptr, plane, cudaMemcpyDeviceToDevice, st));
  if (d_grad_sus)
    RP_TRY_CUDA(cudaMemcpyAsync(d_grad_sus, m->gsus.ptr, sizeof(float) * (size_t)N,
                                cudaMemcpyDeviceToDevice, st));
  if (d_grad_rates)
    RP_TRY_CUDA(cudaMemcpyAsync(d_grad_rates, m->grates.ptr, sizeof(double) * 4,
                                cudaMemcpyDeviceToDevice, st));
  RP_TRY_CUDA(cudaGetLastError());
  return RP_OK;
}

}  // extern "C"
