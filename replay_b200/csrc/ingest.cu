// Device build of the interval index (the ingest step after parsing).
//
// Replaces the reference's NCLS build (tool/ncls/ncls/src/intervaldb.c:
// 227-326, imstart_qsort_cmp :30-46) with data-parallel passes over the
// contacts on the GPU:
//   1. stored coordinates: a negative start is mirrored to (-end, -(int32)
//      start), as the reference database stores it (:233-235, :412-424);
//   2. order by (start asc, end desc), ties in file order (the reference's
//      qsort is glibc's stable merge sort): a stable LSD radix sort, 8-bit
//      digits over the significant bits of the key only;
//   3. the sublist count nlists = (top-level intervals - 1) + (intervals
//      with a child).  In sorted order interval i has a child iff i+1 nests
//      in it, and i is top-level iff it lies outside the root of the
//      current nesting chain, which is the interval where the running
//      maximum end was first reached -- a prefix scan;
//   4. duration classes (class 0: duration <= 1, class c: (2^(c-1), 2^c]),
//      a stable partition: one more radix pass on the class.
// The host keeps only the class-ordered starts (window planning).
#include <algorithm>

#include "rp_internal.h"

namespace rp {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per tile
constexpr int kBins = 256;
constexpr int kWarpsPerBlock = kSortThreads / 32;
constexpr int kScanChunk = 4096;  // counts per block of the offset scan

__device__ __forceinline__ unsigned long long ordered(int64_t x) {
  return (unsigned long long)x ^ 0x8000000000000000ull;
}

__global__ void k_store_coords(int64_t *__restrict__ s, int64_t *__restrict__ e, int64_t n,
                               unsigned long long *__restrict__ mm) {
  unsigned long long smin = ~0ull, smax = 0, emin = ~0ull, emax = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = s[i], b = e[i];
    if (a < 0) {
      const int64_t m = -b;
      b = -(int64_t)(int32_t)a;
      a = m;
      s[i] = a;
      e[i] = b;
    }
    smin = min(smin, ordered(a));
    smax = max(smax, ordered(a));
    emin = min(emin, ordered(b));
    emax = max(emax, ordered(b));
  }
  for (int o = 16; o > 0; o >>= 1) {
    smin = min(smin, __shfl_xor_sync(0xFFFFFFFFu, smin, o));
    smax = max(smax, __shfl_xor_sync(0xFFFFFFFFu, smax, o));
    emin = min(emin, __shfl_xor_sync(0xFFFFFFFFu, emin, o));
    emax = max(emax, __shfl_xor_sync(0xFFFFFFFFu, emax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], smin);
    atomicMax(&mm[1], smax);
    atomicMin(&mm[2], emin);
    atomicMax(&mm[3], emax);
  }
}

// key = (start - smin) << eb | (emax - end) when both fit in 64 bits
// (mode 0); else mode 1: end key only, mode 2: start key only.
__global__ void k_make_keys(const int64_t *__restrict__ s, const int64_t *__restrict__ e,
                            const uint32_t *__restrict__ perm, int64_t n,
                            const unsigned long long *__restrict__ mm, int eb, int mode,
                            unsigned long long *__restrict__ key) {
  const int64_t smin = (int64_t)(mm[0] ^ 0x8000000000000000ull);
  const int64_t emax = (int64_t)(mm[3] ^ 0x8000000000000000ull);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = perm ? perm[i] : i;
    const unsigned long long ks = (unsigned long long)s[j] - (unsigned long long)smin;
    const unsigned long long ke = (unsigned long long)emax - (unsigned long long)e[j];
    key[i] = mode == 0 ? ((eb == 64 ? 0ull : (ks << eb)) | ke) : (mode == 1 ? ke : ks);
  }
}

__global__ void k_iota(uint32_t *__restrict__ v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

// ---- stable radix sort pass over 8 bits of a 64-bit key --------------------
__global__ void __launch_bounds__(kSortThreads)
    k_digit_hist(const unsigned long long *__restrict__ key, int64_t n, int shift,
                 int32_t n_tiles, int32_t *__restrict__ counts) {
  __shared__ int32_t h[kBins];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile;
  for (int j = 0; j < kSortItems; ++j) {
    const int64_t i = base + (int64_t)j * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(key[i] >> shift) & 0xFF], 1);
  }
  __syncthreads();
  counts[(int64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];  // digit-major
}

// Exclusive scan of int32 counts (total < 2^31), three steps.
__global__ void __launch_bounds__(1024)
    k_scan_chunks(const int32_t *__restrict__ in, int64_t n, int32_t *__restrict__ sums) {
  __shared__ int32_t ws[32];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + 4 * threadIdx.x;
  int32_t v = 0;
  for (int k = 0; k < 4; ++k)
    if (base + k < n) v += in[base + k];
  v = __reduce_add_sync(0xFFFFFFFFu, v);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    int32_t t = ws[threadIdx.x];
    t = __reduce_add_sync(0xFFFFFFFFu, t);
    if (threadIdx.x == 0) sums[blockIdx.x] = t;
  }
}

__global__ void k_scan_sums(int32_t *__restrict__ sums, int32_t n) {
  if (threadIdx.x != 0) return;
  int32_t run = 0;
  for (int32_t i = 0; i < n; ++i) {
    const int32_t v = sums[i];
    sums[i] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(1024)
    k_scan_apply(const int32_t *__restrict__ in, int64_t n, const int32_t *__restrict__ sums,
                 int32_t *__restrict__ out) {
  __shared__ int32_t ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + 4 * threadIdx.x;
  int32_t v[4], t = 0;
  for (int k = 0; k < 4; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    t += v[k];
  }
  int32_t x = t;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int32_t w = ws[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    ws[lane] = w;
  }
  __syncthreads();
  int32_t run = sums[blockIdx.x] + (warp ? ws[warp - 1] : 0) + x - t;
  for (int k = 0; k < 4; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

// Stable scatter: the tile's keys are ranked in index order, round by round
// (round j holds keys j*256 .. j*256+255 of the tile, one per thread).
__global__ void __launch_bounds__(kSortThreads)
    k_digit_scatter(const unsigned long long *__restrict__ key, const uint32_t *__restrict__ val,
                    int64_t n, int shift, int32_t n_tiles, const int32_t *__restrict__ offs,
                    unsigned long long *__restrict__ key_out, uint32_t *__restrict__ val_out) {
  __shared__ int32_t s_base[kBins];
  __shared__ int32_t s_wcnt[kWarpsPerBlock][kBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  s_base[threadIdx.x] = offs[(int64_t)threadIdx.x * n_tiles + blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kSortTile;
  for (int j = 0; j < kSortItems; ++j) {
    for (int w = 0; w < kWarpsPerBlock; ++w) s_wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = base + (int64_t)j * kSortThreads + threadIdx.x;
    const bool ok = i < n;
    const unsigned long long k = ok ? key[i] : 0ull;
    const uint32_t d = ok ? (uint32_t)((k >> shift) & 0xFF) : kBins;  // kBins: no key
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (ok && rank == 0) s_wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (ok) {
      int32_t pos = s_base[d] + rank;
      for (int w = 0; w < warp; ++w) pos += s_wcnt[w][d];
      key_out[pos] = k;
      val_out[pos] = val[i];
    }
    __syncthreads();
    int32_t add = 0;
    for (int w = 0; w < kWarpsPerBlock; ++w) add += s_wcnt[w][threadIdx.x];
    s_base[threadIdx.x] += add;
  }
}

// ---- nesting counts ---------------------------------------------------------
template <typename T>
__global__ void k_gather(const T *__restrict__ src, const uint32_t *__restrict__ perm, int64_t n,
                         T *__restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

struct MaxFirst {  // running maximum end and the first index reaching it
  int64_t v;
  int64_t at;
};
__device__ __forceinline__ MaxFirst combine(MaxFirst a, MaxFirst b) { return b.v > a.v ? b : a; }

constexpr int kNestChunk = 4096;

__global__ void __launch_bounds__(256)
    k_nest_chunks(const int64_t *__restrict__ se, int64_t n, MaxFirst *__restrict__ agg) {
  // sequential per chunk is enough here: one thread per chunk
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t b = c * kNestChunk;
  if (b >= n) return;
  const int64_t e = min(n, b + kNestChunk);
  MaxFirst m{se[b], b};
  for (int64_t i = b + 1; i < e; ++i) m = combine(m, MaxFirst{se[i], i});
  agg[c] = m;
}

__global__ void k_nest_prefix(MaxFirst *__restrict__ agg, int64_t n_chunks) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  MaxFirst run{INT64_MIN, -1};
  for (int64_t c = 0; c < n_chunks; ++c) {
    const MaxFirst v = agg[c];
    agg[c] = run;  // exclusive
    run = c == 0 ? v : combine(run, v);
  }
}

__global__ void __launch_bounds__(256)
    k_nest_count(const int64_t *__restrict__ ss, const int64_t *__restrict__ se, int64_t n,
                 const MaxFirst *__restrict__ agg, unsigned long long *__restrict__ counters) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t b = c * kNestChunk;
  if (b >= n) return;
  const int64_t e = min(n, b + kNestChunk);
  MaxFirst run = agg[c];
  unsigned long long top = 0, parents = 0;
  for (int64_t i = b; i < e; ++i) {
    // i is top-level iff outside the chain root R = run.at (none for i = 0)
    bool is_top = run.at < 0;
    if (!is_top) {
      const int64_t r = run.at;
      is_top = se[i] > se[r] || (se[i] == se[r] && ss[i] == ss[r]);
    }
    top += is_top;
    // i has a child iff i+1 is not outside i
    if (i + 1 < n) parents += !(se[i + 1] > se[i] || (se[i + 1] == se[i] && ss[i + 1] == ss[i]));
    run = run.at < 0 ? MaxFirst{se[i], i} : combine(run, MaxFirst{se[i], i});
  }
  atomicAdd(&counters[0], top);
  atomicAdd(&counters[1], parents);
}

// duration class keys (sorted order) and per-class counts
__global__ void k_class_keys(const int64_t *__restrict__ ss, const int64_t *__restrict__ se,
                             int64_t n, unsigned long long *__restrict__ key,
                             unsigned long long *__restrict__ class_cnt) {
  __shared__ unsigned int h[kClasses];
  for (int c = threadIdx.x; c < kClasses; c += blockDim.x) h[c] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = se[i] - ss[i];
    const int c = d > 1 ? 64 - __clzll((long long)(d - 1)) : 0;
    key[i] = (unsigned long long)c;
    atomicAdd(&h[c], 1u);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < kClasses; c += blockDim.x)
    if (h[c]) atomicAdd(&class_cnt[c], (unsigned long long)h[c]);
}

int grid_of(int64_t n, int threads) {
  const int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

int bit_width(uint64_t x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

// Stable LSD sort of (key, val) over bits [0, bits) of key; results end in
// (key, val) (the buffers ping-pong with (k2, v2)).
rp_status radix_sort(DevBuf &key, DevBuf &val, DevBuf &k2, DevBuf &v2, int64_t n, int bits,
                     DevBuf &counts, DevBuf &offs, DevBuf &sums, cudaStream_t st) {
  const int32_t n_tiles = (int32_t)((n + kSortTile - 1) / kSortTile);
  const int64_t nc = (int64_t)kBins * n_tiles;
  const int32_t n_chunks = (int32_t)((nc + kScanChunk - 1) / kScanChunk);
  for (int shift = 0; shift < bits; shift += 8) {
    k_digit_hist<<<n_tiles, kSortThreads, 0, st>>>(key.as<unsigned long long>(), n, shift, n_tiles,
                                                   counts.as<int32_t>());
    k_scan_chunks<<<n_chunks, 1024, 0, st>>>(counts.as<int32_t>(), nc, sums.as<int32_t>());
    k_scan_sums<<<1, 32, 0, st>>>(sums.as<int32_t>(), n_chunks);
    k_scan_apply<<<n_chunks, 1024, 0, st>>>(counts.as<int32_t>(), nc, sums.as<int32_t>(),
                                            offs.as<int32_t>());
    k_digit_scatter<<<n_tiles, kSortThreads, 0, st>>>(
        key.as<unsigned long long>(), val.as<uint32_t>(), n, shift, n_tiles, offs.as<int32_t>(),
        k2.as<unsigned long long>(), v2.as<uint32_t>());
    key.swap(k2);
    val.swap(v2);
  }
  RP_TRY_CUDA(cudaGetLastError());
  return RP_OK;
}

}  // namespace

rp_status graph_build_device(Graph &g, const int64_t *start, const int64_t *end, const int32_t *u,
                             const int32_t *v, int64_t n, int32_t n_nodes) {
  g.n_nodes = n_nodes;
  g.n_contacts = n;
  if (n > (int64_t)INT32_MAX) {
    set_error("too many contacts");
    return RP_ERR_RANGE;
  }
  RP_TRY_CUDA(cudaSetDevice(g.device));
  g.class_off.assign(kClasses + 1, 0);
  g.n_classes_used = 0;
  g.nlists = 0;
  RP_TRY(g.cs.alloc(sizeof(int64_t) * n));
  RP_TRY(g.ce.alloc(sizeof(int64_t) * n));
  RP_TRY(g.cu.alloc(sizeof(int32_t) * n));
  RP_TRY(g.cv.alloc(sizeof(int32_t) * n));
  RP_TRY(g.crank.alloc(sizeof(int32_t) * n));
  g.h_cs.clear();
  if (n == 0) return RP_OK;
  cudaStream_t st = nullptr;
  // the scratch below is kept for the next build once the stream is idle
  ParkGuard park;
  DevBuf s, e, uu, vv, key, val, k2, v2, counts, offs, sums, mm, ctr, agg, ss, se, su, sv;
  RP_TRY(s.alloc(sizeof(int64_t) * n));
  RP_TRY(e.alloc(sizeof(int64_t) * n));
  RP_TRY(uu.alloc(sizeof(int32_t) * n));
  RP_TRY(vv.alloc(sizeof(int32_t) * n));
  RP_TRY_CUDA(cudaMemcpyAsync(s.ptr, start, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
  RP_TRY_CUDA(cudaMemcpyAsync(e.ptr, end, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
  RP_TRY_CUDA(cudaMemcpyAsync(uu.ptr, u, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  RP_TRY_CUDA(cudaMemcpyAsync(vv.ptr, v, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));

  // 1. stored coordinates and the key ranges
  RP_TRY(mm.alloc(sizeof(unsigned long long) * 4));
  const unsigned long long init[4] = {~0ull, 0ull, ~0ull, 0ull};
  RP_TRY_CUDA(cudaMemcpyAsync(mm.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_store_coords<<<grid_of(n, 256), 256, 0, st>>>(s.as<int64_t>(), e.as<int64_t>(), n,
                                                  mm.as<unsigned long long>());
  unsigned long long hmm[4];
  RP_TRY_CUDA(cudaMemcpyAsync(hmm, mm.ptr, sizeof(hmm), cudaMemcpyDeviceToHost, st));
  RP_TRY_CUDA(cudaStreamSynchronize(st));
  const int64_t smin = (int64_t)(hmm[0] ^ 0x8000000000000000ull);
  const int64_t smax = (int64_t)(hmm[1] ^ 0x8000000000000000ull);
  const int64_t emin = (int64_t)(hmm[2] ^ 0x8000000000000000ull);
  const int64_t emax = (int64_t)(hmm[3] ^ 0x8000000000000000ull);
  g.t_min = smin;
  g.t_max = emax;
  const int sb = bit_width((uint64_t)smax - (uint64_t)smin);
  const int eb = bit_width((uint64_t)emax - (uint64_t)emin);

  // 2. (start asc, end desc, file order): stable radix sort of the index
  const int32_t n_tiles = (int32_t)((n + kSortTile - 1) / kSortTile);
  const int64_t nc = (int64_t)kBins * n_tiles;
  RP_TRY(key.alloc(sizeof(unsigned long long) * n));
  RP_TRY(k2.alloc(sizeof(unsigned long long) * n));
  RP_TRY(val.alloc(sizeof(uint32_t) * n));
  RP_TRY(v2.alloc(sizeof(uint32_t) * n));
  RP_TRY(counts.alloc(sizeof(int32_t) * nc));
  RP_TRY(offs.alloc(sizeof(int32_t) * nc));
  RP_TRY(sums.alloc(sizeof(int32_t) * ((nc + kScanChunk - 1) / kScanChunk)));
  k_iota<<<grid_of(n, 256), 256, 0, st>>>(val.as<uint32_t>(), n);
  if (sb + eb <= 64) {
    k_make_keys<<<grid_of(n, 256), 256, 0, st>>>(s.as<int64_t>(), e.as<int64_t>(), nullptr, n,
                                                 mm.as<unsigned long long>(), eb, 0,
                                                 key.as<unsigned long long>());
    RP_TRY(radix_sort(key, val, k2, v2, n, sb + eb, counts, offs, sums, st));
  } else {
    k_make_keys<<<grid_of(n, 256), 256, 0, st>>>(s.as<int64_t>(), e.as<int64_t>(), nullptr, n,
                                                 mm.as<unsigned long long>(), eb, 1,
                                                 key.as<unsigned long long>());
    RP_TRY(radix_sort(key, val, k2, v2, n, eb, counts, offs, sums, st));
    k_make_keys<<<grid_of(n, 256), 256, 0, st>>>(s.as<int64_t>(), e.as<int64_t>(),
                                                 val.as<uint32_t>(), n,
                                                 mm.as<unsigned long long>(), eb, 2,
                                                 key.as<unsigned long long>());
    RP_TRY(radix_sort(key, val, k2, v2, n, sb, counts, offs, sums, st));
  }
  RP_TRY(ss.alloc(sizeof(int64_t) * n));
  RP_TRY(se.alloc(sizeof(int64_t) * n));
  RP_TRY(su.alloc(sizeof(int32_t) * n));
  RP_TRY(sv.alloc(sizeof(int32_t) * n));
  const uint32_t *perm = val.as<uint32_t>();
  k_gather<int64_t><<<grid_of(n, 256), 256, 0, st>>>(s.as<int64_t>(), perm, n, ss.as<int64_t>());
  k_gather<int64_t><<<grid_of(n, 256), 256, 0, st>>>(e.as<int64_t>(), perm, n, se.as<int64_t>());
  k_gather<int32_t><<<grid_of(n, 256), 256, 0, st>>>(uu.as<int32_t>(), perm, n, su.as<int32_t>());
  k_gather<int32_t><<<grid_of(n, 256), 256, 0, st>>>(vv.as<int32_t>(), perm, n, sv.as<int32_t>());

  // 3. nlists
  const int64_t n_chunks = (n + kNestChunk - 1) / kNestChunk;
  RP_TRY(agg.alloc(sizeof(MaxFirst) * n_chunks));
  RP_TRY(ctr.alloc(sizeof(unsigned long long) * (2 + kClasses)));
  RP_TRY_CUDA(cudaMemsetAsync(ctr.ptr, 0, ctr.bytes, st));
  const int nb = (int)((n_chunks + 255) / 256);
  k_nest_chunks<<<nb, 256, 0, st>>>(se.as<int64_t>(), n, agg.as<MaxFirst>());
  k_nest_prefix<<<1, 32, 0, st>>>(agg.as<MaxFirst>(), n_chunks);
  k_nest_count<<<nb, 256, 0, st>>>(ss.as<int64_t>(), se.as<int64_t>(), n, agg.as<MaxFirst>(),
                                   ctr.as<unsigned long long>());

  // 4. stable partition by duration class; class c's rank in (start, end)
  // order is the sorted position
  k_class_keys<<<grid_of(n, 256), 256, 0, st>>>(ss.as<int64_t>(), se.as<int64_t>(), n,
                                                key.as<unsigned long long>(),
                                                ctr.as<unsigned long long>() + 2);
  k_iota<<<grid_of(n, 256), 256, 0, st>>>(val.as<uint32_t>(), n);
  RP_TRY(radix_sort(key, val, k2, v2, n, 8, counts, offs, sums, st));
  const uint32_t *order = val.as<uint32_t>();
  k_gather<int64_t><<<grid_of(n, 256), 256, 0, st>>>(ss.as<int64_t>(), order, n, g.cs.as<int64_t>());
  k_gather<int64_t><<<grid_of(n, 256), 256, 0, st>>>(se.as<int64_t>(), order, n, g.ce.as<int64_t>());
  k_gather<int32_t><<<grid_of(n, 256), 256, 0, st>>>(su.as<int32_t>(), order, n, g.cu.as<int32_t>());
  k_gather<int32_t><<<grid_of(n, 256), 256, 0, st>>>(sv.as<int32_t>(), order, n, g.cv.as<int32_t>());
  RP_TRY_CUDA(cudaMemcpyAsync(g.crank.ptr, order, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));

  unsigned long long hc[2 + kClasses];
  RP_TRY_CUDA(cudaMemcpyAsync(hc, ctr.ptr, sizeof(hc), cudaMemcpyDeviceToHost, st));
  g.h_cs.resize(n);
  RP_TRY_CUDA(cudaMemcpyAsync(g.h_cs.data(), g.cs.ptr, sizeof(int64_t) * n, cudaMemcpyDeviceToHost,
                              st));
  RP_TRY_CUDA(cudaStreamSynchronize(st));
  park.arm();
  g.nlists = ((int64_t)hc[0] - 1) + (int64_t)hc[1];
  for (int c = 0; c < kClasses; ++c) {
    g.class_off[c + 1] = g.class_off[c] + (int64_t)hc[2 + c];
    g.n_classes_used += hc[2 + c] > 0;
  }
  return RP_OK;
}

}  // namespace rp
