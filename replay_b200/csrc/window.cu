// Per-window symmetric CSR builder on the device.
//
// Replaces the reference's per-step host path: find_intervals over the NCLS
// (tool/ncls/ncls/src/intervaldb.c:426-485, called with nbuf = nlists from
// tool/gpu_cpu_temporal_sim.cu:973-991) and build_csr_from_intervals
// (tool/gpu_cpu_temporal_sim.cu:238-350: overlap weights, symmetric
// emission, qsort by (row, col), FP32 duplicate merge, counting sort).
//
// Kernels, in launch order for one window:
//   k_hits      candidates of the duration-class index -> hit list (+degrees)
//   k_trunc     only when the reference's hit cap can bind: keep the cap
//               smallest ranks (radix select), then count degrees
//   k_scan_*    degrees -> row_ptr (exclusive scan), cursors reset
//   k_fill      hits -> row segments {col, weight} + rank
//   k_rowsort_* rows ordered by (col, rank), duplicates merged in rank order
#include <cstdio>

#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanTile = 4 * kScanThreads;
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ int block_excl_scan(int v, int *warp_tot,
                                               int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  const int off = warp ? warp_tot[warp - 1] : 0;
  total = warp_tot[(blockDim.x >> 5) - 1];
  __syncthreads();
  return off + x - v;
}

__device__ __forceinline__ int block_sum(int v, int *warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = __reduce_add_sync(kFull, v);
  if (lane == 0) warp_tot[warp] = v;
  __syncthreads();
  int t = 0;
  if (warp == 0) {
    t = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
    t = __reduce_add_sync(kFull, t);
    if (lane == 0) warp_tot[0] = t;
  }
  __syncthreads();
  t = warp_tot[0];
  __syncthreads();
  return t;
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_hits(const WinDesc *__restrict__ wins, int wi,
           const CandRange *__restrict__ ranges, const int64_t *__restrict__ cs,
           const int64_t *__restrict__ ce, const int32_t *__restrict__ cu,
           const int32_t *__restrict__ cv, const int32_t *__restrict__ crank,
           Hit *__restrict__ hits, unsigned long long *__restrict__ counters,
           int32_t *__restrict__ deg, int weight_f32) {
  __shared__ CandRange sr[kClasses];
  __shared__ WinDesc sw;
  if (threadIdx.x == 0) sw = wins[wi];
  __syncthreads();
  if ((int)threadIdx.x < sw.n_ranges) sr[threadIdx.x] = ranges[sw.range_off + threadIdx.x];
  __syncthreads();
  const int nr = sw.n_ranges;
  const int64_t total = sw.n_candidates;
  const int count_deg = !sw.may_truncate;
  const int query_neg = sw.ws < 0;
  const unsigned lane = threadIdx.x & 31;
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) - lane;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = warp0; base < total; base += stride) {
    const int64_t t = base + lane;
    bool rec = false, pred = false;
    Hit h;
    if (t < total) {
      int k = 0;
      for (int step = 32; step > 0; step >>= 1)
        if (k + step < nr && sr[k + step].prefix <= t) k += step;
      const int64_t idx = sr[k].lo + (t - sr[k].prefix);
      const int64_t s = cs[idx], e = ce[idx];
      if (s < sw.qe && sw.qs < e) {
        pred = true;
        // Coordinates handed to the CSR builder: mirrored back when the
        // stored orientation differs from the query's.
        int64_t hs = s, he = e;
        if ((s < 0) != query_neg) {
          hs = -e;
          he = -(int64_t)(int32_t)s;
        }
        const int64_t os = hs > sw.ws ? hs : sw.ws;
        const int64_t oe = he < sw.we ? he : sw.we;
        const int64_t ov = oe - os;
        h.rank = crank[idx];
        h.v = cv[idx];
        if (ov > 0) {
          h.u = cu[idx];
          h.w = weight_f32 ? __float_as_int(__fmul_rn(__ll2float_rn(ov), sw.scale))
                           : (int32_t)ov;
          rec = true;
          if (count_deg) {
            atomicAdd(&deg[h.u], 1);
            atomicAdd(&deg[h.v], 1);
          }
        } else if (!count_deg) {
          h.u = -1;
          h.w = 0;
          rec = true;
        }
      }
    }
    const unsigned pmask = __ballot_sync(kFull, pred);
    if (pmask && lane == 0) atomicAdd(&counters[3], (unsigned long long)__popc(pmask));
    const unsigned mask = __ballot_sync(kFull, rec);
    if (mask) {
      unsigned long long pos0 = 0;
      if (lane == 0) pos0 = atomicAdd(&counters[0], (unsigned long long)__popc(mask));
      pos0 = __shfl_sync(kFull, pos0, 0);
      if (rec) hits[pos0 + __popc(mask & ((1u << lane) - 1u))] = h;
    }
  }
}

// The reference query stops after max(nlists,1) hits taken in sorted order
// (the NCLS depth-first order), i.e. it keeps the cap smallest ranks.
__global__ void __launch_bounds__(1024)
    k_trunc(Hit *__restrict__ hits, const unsigned long long *__restrict__ counters,
            int64_t cap, int32_t *__restrict__ deg) {
  __shared__ unsigned hist[256];
  __shared__ unsigned s_prefix, s_k;
  const int64_t n = (int64_t)counters[0];
  uint32_t thr = 0xFFFFFFFFu;
  if (n > cap) {
    if (threadIdx.x == 0) {
      s_prefix = 0;
      s_k = (unsigned)cap;  // 1-based rank of the last kept hit
    }
    __syncthreads();
    for (int d = 3; d >= 0; --d) {
      for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
      __syncthreads();
      const unsigned pre = s_prefix;
      const unsigned hi_mask = (d == 3) ? 0u : (0xFFFFFFFFu << (8 * (d + 1)));
      for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned r = (unsigned)hits[i].rank;
        if ((r & hi_mask) == (pre & hi_mask)) atomicAdd(&hist[(r >> (8 * d)) & 255u], 1u);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned k = s_k, acc = 0;
        int b = 0;
        for (; b < 256; ++b) {
          if (acc + hist[b] >= k) break;
          acc += hist[b];
        }
        s_k = k - acc;
        s_prefix = pre | ((unsigned)b << (8 * d));
      }
      __syncthreads();
    }
    thr = s_prefix;
  }
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    Hit h = hits[i];
    if ((uint32_t)h.rank > thr) {
      hits[i].u = -2;
      continue;
    }
    if (h.u >= 0) {
      atomicAdd(&deg[h.u], 1);
      atomicAdd(&deg[h.v], 1);
    }
  }
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_tiles(const int32_t *__restrict__ in, int32_t n, int32_t *__restrict__ tiles) {
  __shared__ int wt[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + 4 * threadIdx.x;
  int s = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (base + j < n) s += in[base + j];
  s = block_sum(s, wt);
  if (threadIdx.x == 0) tiles[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_apply(int32_t *__restrict__ in, int32_t n,
                 const int32_t *__restrict__ tiles, int32_t *__restrict__ out,
                 int zero_in) {
  __shared__ int wt[32];
  int off = 0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) off += tiles[b];
  off = block_sum(off, wt);
  const int64_t base = (int64_t)blockIdx.x * kScanTile + 4 * threadIdx.x;
  int v[4], s = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    v[j] = (base + j < n) ? in[base + j] : 0;
    s += v[j];
  }
  int total;
  int ex = block_excl_scan(s, wt, total) + off;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (base + j < n) {
      out[base + j] = ex;
      if (zero_in) in[base + j] = 0;
    }
    ex += v[j];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = off + total;
}

__global__ void __launch_bounds__(256)
    k_fill(const Hit *__restrict__ hits, const unsigned long long *__restrict__ counters,
           const int32_t *__restrict__ row_ptr, int32_t *__restrict__ cursor,
           int2 *__restrict__ entries, int32_t *__restrict__ erank) {
  const int64_t n = (int64_t)counters[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const Hit h = hits[i];
    if (h.u < 0) continue;
    const int32_t pu = row_ptr[h.u] + atomicAdd(&cursor[h.u], 1);
    entries[pu] = make_int2(h.v, h.w);
    erank[pu] = h.rank;
    const int32_t pv = row_ptr[h.v] + atomicAdd(&cursor[h.v], 1);
    entries[pv] = make_int2(h.u, h.w);
    erank[pv] = h.rank;
  }
}

// ---- row sort + merge -----------------------------------------------------------
// The leader of a peer group is its lowest lane.
__device__ __forceinline__ bool before_leader(unsigned peers, unsigned lane) {
  return (unsigned)(__ffs(peers) - 1) == lane;
}

__device__ __forceinline__ uint64_t make_key(int32_t col, int32_t rank) {
  return ((uint64_t)(uint32_t)col << 32) | (uint32_t)rank;
}

__device__ __forceinline__ int32_t merge_add(int32_t acc, int32_t w, int f32) {
  return f32 ? __float_as_int(__fadd_rn(__int_as_float(acc), __int_as_float(w)))
             : acc + w;
}

constexpr int kWarpCap = 512;       // rows up to this length sort in a warp
constexpr int kRowsortWarps = 4;

// Merges runs of equal columns in a sorted segment held in shared memory:
// the first entry of a run receives the sequential sum, the rest weight 0.
__device__ void merge_runs_smem(const uint64_t *key, int32_t *val, int L, int f32,
                                int tid, int nthreads) {
  for (int i = tid; i < L; i += nthreads) {
    const uint32_t c = (uint32_t)(key[i] >> 32);
    const bool head = (i == 0) || ((uint32_t)(key[i - 1] >> 32) != c);
    if (!head) continue;
    int32_t acc = val[i];
    int j = i + 1;
    for (; j < L && (uint32_t)(key[j] >> 32) == c; ++j) acc = merge_add(acc, val[j], f32);
    val[i] = acc;
    for (int q = i + 1; q < j; ++q) val[q] = 0;
  }
}

__global__ void __launch_bounds__(32 * kRowsortWarps)
    k_rowsort_warp(int32_t n, const int32_t *__restrict__ row_ptr,
                   int2 *__restrict__ entries, int32_t *__restrict__ erank,
                   unsigned long long *__restrict__ counters,
                   int32_t *__restrict__ long_rows, int f32) {
  __shared__ uint64_t skey[kRowsortWarps][kWarpCap];
  __shared__ int32_t sval[kRowsortWarps][kWarpCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = gw; row < n; row += nw) {
    const int32_t beg = row_ptr[row], L = row_ptr[row + 1] - beg;
    if (L <= 1) continue;
    if (L > kWarpCap) {
      if (lane == 0) {
        unsigned long long p = atomicAdd(&counters[1], 1ull);
        long_rows[p] = (int32_t)row;
      }
      continue;
    }
    if (L <= 32) {
      uint64_t k = ~0ull;
      int32_t w = 0;
      if (lane < L) {
        const int2 en = entries[beg + lane];
        k = make_key(en.x, erank[beg + lane]);
        w = en.y;
      }
      // bitonic sort of 32 keys across the warp, ascending
#pragma unroll
      for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          const uint64_t ok = __shfl_xor_sync(kFull, k, stride);
          const int32_t ow = __shfl_xor_sync(kFull, w, stride);
          const bool up = ((lane & size) == 0);
          const bool lower = ((lane & stride) == 0);
          const bool take = (lower == up) ? (ok < k) : (ok > k);
          if (take) {
            k = ok;
            w = ow;
          }
        }
      }
      const uint32_t c = (uint32_t)(k >> 32);
      const uint32_t cprev = __shfl_up_sync(kFull, c, 1);
      const bool head = lane < L && (lane == 0 || cprev != c);
      int32_t acc = w;
      bool active = head;
      for (int d = 1; d < 32; ++d) {
        const int32_t ow = __shfl_down_sync(kFull, w, d);
        const uint32_t oc = __shfl_down_sync(kFull, c, d);
        if (active) {
          if (lane + d < L && oc == c)
            acc = merge_add(acc, ow, f32);
          else
            active = false;
        }
        if (!__any_sync(kFull, active)) break;
      }
      if (lane < L) {
        entries[beg + lane] = make_int2((int32_t)c, head ? acc : 0);
        erank[beg + lane] = (int32_t)(uint32_t)k;
      }
      continue;
    }
    // 32 < L <= kWarpCap: bitonic sort in this warp's shared-memory slot
    int P = 64;
    while (P < L) P <<= 1;
    uint64_t *key = skey[wib];
    int32_t *val = sval[wib];
    for (int i = lane; i < P; i += 32) {
      if (i < L) {
        const int2 en = entries[beg + i];
        key[i] = make_key(en.x, erank[beg + i]);
        val[i] = en.y;
      } else {
        key[i] = ~0ull;
        val[i] = 0;
      }
    }
    __syncwarp();
    for (int size = 2; size <= P; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int i = lane; i < P; i += 32) {
          const int j = i ^ stride;
          if (j > i) {
            const bool up = ((i & size) == 0);
            const uint64_t a = key[i], b = key[j];
            if ((a > b) == up) {
              key[i] = b;
              key[j] = a;
              const int32_t t = val[i];
              val[i] = val[j];
              val[j] = t;
            }
          }
        }
        __syncwarp();
      }
    }
    merge_runs_smem(key, val, L, f32, lane, 32);
    __syncwarp();
    for (int i = lane; i < L; i += 32) {
      entries[beg + i] = make_int2((int32_t)(key[i] >> 32), val[i]);
      erank[beg + i] = (int32_t)(uint32_t)key[i];
    }
    __syncwarp();
  }
}

// Rows longer than a warp slot: one CTA per row, stable LSD radix sort on
// (rank, then col) between the row segment and a scratch segment, then the
// sequential merge.  Only reached by hub rows of FP32-weight windows.
__global__ void __launch_bounds__(256)
    k_rowsort_long(const int32_t *__restrict__ row_ptr, int2 *__restrict__ entries,
                   int32_t *__restrict__ erank, int2 *__restrict__ tmp_e,
                   int32_t *__restrict__ tmp_r,
                   const unsigned long long *__restrict__ counters,
                   const int32_t *__restrict__ long_rows, int rank_bits,
                   int col_bits, int f32) {
  __shared__ unsigned hist[256];
  __shared__ unsigned offs[256];
  const int64_t nl = (int64_t)counters[1];
  for (int64_t li = blockIdx.x; li < nl; li += gridDim.x) {
    const int32_t row = long_rows[li];
    const int32_t beg = row_ptr[row], L = row_ptr[row + 1] - beg;
    int2 *ea = entries + beg, *eb = tmp_e + beg;
    int32_t *ra = erank + beg, *rb = tmp_r + beg;
    int npass = 0;
    for (int field = 0; field < 2; ++field) {
      const int bits = field == 0 ? rank_bits : col_bits;
      for (int sh = 0; sh < bits; sh += 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < L; i += blockDim.x) {
          const uint32_t key = field == 0 ? (uint32_t)ra[i] : (uint32_t)ea[i].x;
          atomicAdd(&hist[(key >> sh) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          unsigned acc = 0;
          for (int b = 0; b < 256; ++b) {
            offs[b] = acc;
            acc += hist[b];
          }
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // stable scatter by one warp, in order
          const unsigned lane = threadIdx.x;
          for (int base = 0; base < L; base += 32) {
            const int i = base + lane;
            const bool ok = i < L;
            uint32_t dig = 0;
            if (ok) {
              const uint32_t key = field == 0 ? (uint32_t)ra[i] : (uint32_t)ea[i].x;
              dig = (key >> sh) & 255u;
            }
            const unsigned act = __ballot_sync(kFull, ok);
            const unsigned peers = __match_any_sync(kFull, ok ? dig : 0xFFFFu) & act;
            if (ok) {
              const unsigned before = __popc(peers & ((1u << lane) - 1u));
              const unsigned pos = offs[dig] + before;
              eb[pos] = ea[i];
              rb[pos] = ra[i];
            }
            __syncwarp();
            if (ok && before_leader(peers, lane)) offs[dig] += __popc(peers);
            __syncwarp();
          }
        }
        __syncthreads();
        int2 *te = ea; ea = eb; eb = te;
        int32_t *tr = ra; ra = rb; rb = tr;
        ++npass;
      }
    }
    if (npass & 1) {  // result lives in the scratch segment: copy back
      for (int i = threadIdx.x; i < L; i += blockDim.x) {
        entries[beg + i] = ea[i];
        erank[beg + i] = ra[i];
      }
      __syncthreads();
    }
    // sequential merge of equal-column runs
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      const int32_t c = entries[beg + i].x;
      const bool head = (i == 0) || entries[beg + i - 1].x != c;
      if (!head) continue;
      int32_t acc = entries[beg + i].y;
      int j = i + 1;
      for (; j < L && entries[beg + j].x == c; ++j) acc = merge_add(acc, entries[beg + j].y, f32);
      entries[beg + i].y = acc;
      for (int q = i + 1; q < j; ++q) entries[beg + q].y = 0;
    }
    __syncthreads();
  }
}

__global__ void k_count_kept(int32_t n, const int32_t *__restrict__ row_ptr,
                             const int2 *__restrict__ entries, int32_t *__restrict__ len) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    int c = 0;
    for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) c += entries[k].y != 0;
    len[r] = c;
  }
}

__global__ void k_compact(int32_t n, const int32_t *__restrict__ row_ptr,
                          const int2 *__restrict__ entries,
                          const int32_t *__restrict__ out_ptr, int2 *__restrict__ out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    int32_t o = out_ptr[r];
    for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
      const int2 en = entries[k];
      if (en.y != 0) out[o++] = en;
    }
  }
}

int grid_for(int64_t work, int threads, int cap) {
  int64_t b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

int bits_for(int64_t maxval) {
  int b = 0;
  while (b < 63 && (int64_t(1) << b) <= maxval) ++b;
  return b < 1 ? 1 : b;
}

}  // namespace

int32_t window_scan_tiles(int32_t n_nodes) {
  const int32_t t = (int32_t)((n_nodes + kScanTile - 1) / kScanTile);
  return t < 1 ? 1 : t;
}

rp_status window_workspace_alloc(WindowWorkspace &w, int32_t n_nodes,
                                 int64_t cap_hits, int64_t n_windows,
                                 const std::vector<WinDesc> &wins,
                                 const std::vector<CandRange> &ranges) {
  w.n_nodes = n_nodes;
  w.cap_hits = cap_hits < 1 ? 1 : cap_hits;
  w.cap_entries = 2 * w.cap_hits;
  w.n_tiles = (int32_t)((n_nodes + kScanTile - 1) / kScanTile);
  if (w.n_tiles < 1) w.n_tiles = 1;
  RP_TRY(w.hits.alloc(sizeof(Hit) * w.cap_hits));
  // two spare pairs: the step kernel stages entry ranges with 16-byte bulk
  // copies that may read 8 bytes past the last pair
  RP_TRY(w.entries.alloc(sizeof(int2) * (w.cap_entries + 2)));
  RP_TRY(w.erank.alloc(sizeof(int32_t) * w.cap_entries));
  RP_TRY(w.tmp_e.alloc(sizeof(int2) * w.cap_entries));
  RP_TRY(w.tmp_r.alloc(sizeof(int32_t) * w.cap_entries));
  RP_TRY(w.row_ptr.alloc(sizeof(int32_t) * ((size_t)n_nodes + 1)));
  RP_TRY(w.deg.alloc(sizeof(int32_t) * ((size_t)n_nodes + 1)));
  RP_TRY(w.tiles.alloc(sizeof(int32_t) * (size_t)w.n_tiles));
  RP_TRY(w.counters.alloc(sizeof(unsigned long long) * 4));
  RP_TRY(w.long_rows.alloc(sizeof(int32_t) * ((size_t)n_nodes + 1)));
  RP_TRY(w.win.alloc(sizeof(WinDesc) * (n_windows > 0 ? n_windows : 1)));
  RP_TRY(w.ranges.alloc(sizeof(CandRange) * (ranges.empty() ? 1 : ranges.size())));
  RP_TRY_CUDA(cudaMemset(w.deg.ptr, 0, w.deg.bytes));
  if (!wins.empty())
    RP_TRY_CUDA(cudaMemcpy(w.win.ptr, wins.data(), sizeof(WinDesc) * wins.size(),
                           cudaMemcpyHostToDevice));
  if (!ranges.empty())
    RP_TRY_CUDA(cudaMemcpy(w.ranges.ptr, ranges.data(),
                           sizeof(CandRange) * ranges.size(), cudaMemcpyHostToDevice));
  return RP_OK;
}

void enqueue_window_build(const Graph &g, WindowWorkspace &ws, int wi,
                          const WinDesc &desc, int64_t cap, int weight_kind,
                          bool sort_rows, cudaStream_t st) {
  const int32_t n = ws.n_nodes;
  unsigned long long *ctr = ws.counters.as<unsigned long long>();
  cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * 4, st);
  // degrees start at zero (the previous window left its fill cursors here)
  cudaMemsetAsync(ws.deg.ptr, 0, sizeof(int32_t) * (size_t)n, st);
  const int f32 = weight_kind == kWeightF32;
  k_hits<<<grid_for(desc.n_candidates, 256, 148 * 16), 256, 0, st>>>(
      ws.win.as<WinDesc>(), wi, ws.ranges.as<CandRange>(), g.cs.as<int64_t>(),
      g.ce.as<int64_t>(), g.cu.as<int32_t>(), g.cv.as<int32_t>(), g.crank.as<int32_t>(),
      ws.hits.as<Hit>(), ctr, ws.deg.as<int32_t>(), f32);
  if (desc.may_truncate)
    k_trunc<<<1, 1024, 0, st>>>(ws.hits.as<Hit>(), ctr, cap, ws.deg.as<int32_t>());
  k_scan_tiles<<<ws.n_tiles, kScanThreads, 0, st>>>(ws.deg.as<int32_t>(), n,
                                                   ws.tiles.as<int32_t>());
  k_scan_apply<<<ws.n_tiles, kScanThreads, 0, st>>>(ws.deg.as<int32_t>(), n,
                                                   ws.tiles.as<int32_t>(),
                                                   ws.row_ptr.as<int32_t>(), 1);
  k_fill<<<grid_for(desc.n_candidates, 256, 148 * 8), 256, 0, st>>>(
      ws.hits.as<Hit>(), ctr, ws.row_ptr.as<int32_t>(), ws.deg.as<int32_t>(),
      ws.entries.as<int2>(), ws.erank.as<int32_t>());
  if (sort_rows) {
    k_rowsort_warp<<<grid_for(n, 32 * kRowsortWarps / 32, 148 * 16), 32 * kRowsortWarps, 0,
                     st>>>(n, ws.row_ptr.as<int32_t>(), ws.entries.as<int2>(),
                           ws.erank.as<int32_t>(), ctr, ws.long_rows.as<int32_t>(), f32);
    k_rowsort_long<<<148, 256, 0, st>>>(ws.row_ptr.as<int32_t>(), ws.entries.as<int2>(),
                                        ws.erank.as<int32_t>(), ws.tmp_e.as<int2>(),
                                        ws.tmp_r.as<int32_t>(), ctr,
                                        ws.long_rows.as<int32_t>(), bits_for(g.n_contacts),
                                        bits_for(n), f32);
  }
}

void enqueue_window_compact(WindowWorkspace &ws, int32_t *row_ptr_out,
                            int2 *entries_out, cudaStream_t st) {
  const int32_t n = ws.n_nodes;
  int32_t *len = ws.deg.as<int32_t>();
  k_count_kept<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(n, ws.row_ptr.as<int32_t>(),
                                                        ws.entries.as<int2>(), len);
  k_scan_tiles<<<ws.n_tiles, kScanThreads, 0, st>>>(len, n, ws.tiles.as<int32_t>());
  k_scan_apply<<<ws.n_tiles, kScanThreads, 0, st>>>(len, n, ws.tiles.as<int32_t>(),
                                                   row_ptr_out, 1);
  k_compact<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(n, ws.row_ptr.as<int32_t>(),
                                                     ws.entries.as<int2>(), row_ptr_out,
                                                     entries_out);
}

}  // namespace rp
