// Host preparation of caller-given contact arrays before the device index
// build (rp_graph_from_arrays): endpoints ordered u <= v (the reference's
// pair packing, tool/temporal_contact_matrix.c:80-90), range checks, and the
// number of distinct nodes that appear.  Header-only so that a host-side
// test can compile it without the CUDA runtime.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace rp {

// Writes uu[k] = min(u[k], v[k]) and vv[k] = max(u[k], v[k]) for every
// contact, and *n_index = the number of distinct nodes among them.  Returns
// -1, or the first contact k with an endpoint outside [0, n_nodes) (then the
// outputs are unspecified).  Ranges of at least kPrepChunk contacts run on
// up to `threads` host threads.
constexpr int64_t kPrepChunk = int64_t(1) << 20;

inline int64_t prep_contacts(const int32_t *u, const int32_t *v, int64_t n, int32_t n_nodes,
                             int32_t *uu, int32_t *vv, int32_t *n_index, int threads) {
  std::vector<uint8_t> seen((size_t)n_nodes, 0);
  int nt = (int)std::min<int64_t>(threads < 1 ? 1 : threads, (n + kPrepChunk - 1) / kPrepChunk);
  if (nt < 1) nt = 1;
  std::vector<int64_t> bad((size_t)nt, -1);
  auto range = [&](int t) {
    const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
    for (int64_t k = lo; k < hi; ++k) {
      const int32_t a = u[k], b = v[k];
      if (a < 0 || b < 0 || a >= n_nodes || b >= n_nodes) {
        bad[(size_t)t] = k;
        return;
      }
      uu[k] = a < b ? a : b;
      vv[k] = a < b ? b : a;
      // several threads may mark one node: relaxed atomic bytes, stored
      // only when not yet set (a marked line then stays shared between the
      // threads' caches instead of bouncing); one thread stores directly
      if (nt == 1 || !__atomic_load_n(&seen[(size_t)a], __ATOMIC_RELAXED))
        __atomic_store_n(&seen[(size_t)a], (uint8_t)1, __ATOMIC_RELAXED);
      if (nt == 1 || !__atomic_load_n(&seen[(size_t)b], __ATOMIC_RELAXED))
        __atomic_store_n(&seen[(size_t)b], (uint8_t)1, __ATOMIC_RELAXED);
    }
  };
  if (nt == 1) {
    range(0);
  } else {
    std::vector<std::thread> pool;
    pool.reserve((size_t)nt - 1);
    for (int t = 1; t < nt; ++t) {
      try {
        pool.emplace_back(range, t);
      } catch (...) {  // no thread to spare: this thread takes the range
        range(t);
      }
    }
    range(0);
    for (std::thread &th : pool) th.join();
  }
  for (int t = 0; t < nt; ++t)
    if (bad[(size_t)t] >= 0) return bad[(size_t)t];  // ranges are in contact order
  int64_t count = 0;
  for (uint8_t s : seen) count += s;
  *n_index = (int32_t)count;
  return -1;
}

}  // namespace rp
