// Allocation-free window CSR build (rp_window_csr_noalloc).
//
// The same device builder as rp_window_csr (interval-index candidate scan,
// hit cap, row fill, per-row sort and duplicate merge, compaction), with
// every scratch buffer carved out of one file-scope device array instead of
// cudaMalloc'd workspaces, and the result left in caller-owned device
// buffers.  It exists for callers that must not allocate or free device
// memory on this path: cudaFree waits for the whole device, so a process that
// keeps other streams busy (or hands all device memory to its own pool) cannot
// afford it per window.
//
// Limits: at most kNoAllocMaxNodes nodes in the graph and kNoAllocMaxCandidates
// candidate contacts in one window (contacts whose stored start falls inside
// the window's scan range); larger requests fail with RP_ERR_RANGE.  The
// scratch array is shared by all calls on a device, so calls must not
// overlap: issue them from one thread on one stream at a time.  Every call
// looks up the array's address (cudaGetSymbolAddress; the first call in a
// context may load this module), copies small descriptors from the host
// stack and synchronizes the stream before it returns, so a call cannot be
// made while the stream is being captured.  The caller's current device is
// restored on return.
#include "rp_internal.h"

namespace rp {
namespace {

constexpr int32_t kNoAllocMaxNodes = 65536;
constexpr int64_t kNoAllocMaxCandidates = 131072;
constexpr int32_t kNoAllocMaxTiles = 64;

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Byte offsets of the scratch regions.
constexpr size_t kHitsOff = 0;
constexpr size_t kEntOff = kHitsOff + align256(sizeof(Hit) * kNoAllocMaxCandidates);
constexpr size_t kErankOff = kEntOff + align256(sizeof(int2) * 2 * kNoAllocMaxCandidates);
constexpr size_t kTmpEOff = kErankOff + align256(sizeof(int32_t) * 2 * kNoAllocMaxCandidates);
constexpr size_t kTmpROff = kTmpEOff + align256(sizeof(int2) * 2 * kNoAllocMaxCandidates);
constexpr size_t kRowPtrOff = kTmpROff + align256(sizeof(int32_t) * 2 * kNoAllocMaxCandidates);
constexpr size_t kNodeBytes = align256(sizeof(int32_t) * (kNoAllocMaxNodes + 1));
constexpr size_t kDegOff = kRowPtrOff + kNodeBytes;
constexpr size_t kLongOff = kDegOff + kNodeBytes;
constexpr size_t kTilesOff = kLongOff + kNodeBytes;
constexpr size_t kCtrOff = kTilesOff + align256(sizeof(int32_t) * kNoAllocMaxTiles);
constexpr size_t kWinOff = kCtrOff + align256(sizeof(unsigned long long) * 4);
constexpr size_t kRangeOff = kWinOff + align256(sizeof(WinDesc));
constexpr size_t kScratchBytes = kRangeOff + align256(sizeof(CandRange) * kClasses);  // ~8.8 MB

static __device__ __align__(256) unsigned char g_window_scratch[kScratchBytes];

// Address of the scratch array in the current device's context.  Looked up
// on every call (no allocation, and cheap): a cached address would go stale
// if the primary context were reset and the module reloaded elsewhere.
rp_status scratch_address(unsigned char **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_window_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(window scratch)");
  *out = static_cast<unsigned char *>(p);
  return RP_OK;
}

// Makes `device` current for the scope and restores the caller's device.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int device) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

rp_status window_csr_noalloc(const Graph &g, int64_t ws, int64_t we, float scale, int weight_kind,
                             int ncls_cap, int32_t *d_row_ptr, int32_t *d_entries,
                             int64_t capacity, int64_t *nnz, int64_t *n_hits, cudaStream_t st) {
  if (!d_row_ptr || !nnz || !n_hits || capacity < 0 || (capacity > 0 && !d_entries) || we <= ws ||
      (weight_kind != kWeightF32 && weight_kind != kWeightI32)) {
    set_error("invalid window CSR request");
    return RP_ERR_ARG;
  }
  if (weight_kind == kWeightI32 && we - ws > INT32_MAX) {
    set_error("integer weights need a window of at most 2^31-1 s");
    return RP_ERR_RANGE;
  }
  if (g.n_nodes > kNoAllocMaxNodes) {
    set_error("graph has %d nodes; the allocation-free window build takes at most %d", g.n_nodes,
              kNoAllocMaxNodes);
    return RP_ERR_RANGE;
  }
  DeviceScope scope(g.device);
  if (scope.err != cudaSuccess) return cuda_fail(scope.err, "cudaSetDevice");
  unsigned char *base = nullptr;
  RP_TRY(scratch_address(&base));

  const int64_t cap = ncls_cap ? (g.nlists > 0 ? g.nlists : 1) : INT64_MAX;
  CandRange ranges[kClasses];
  WinDesc desc{};
  plan_window_ranges(g, ws, we, scale, cap, ranges, desc);
  if (desc.n_candidates > kNoAllocMaxCandidates) {
    set_error("window [%lld, %lld) scans %lld candidate contacts; the allocation-free window "
              "build takes at most %lld", (long long)ws, (long long)we,
              (long long)desc.n_candidates, (long long)kNoAllocMaxCandidates);
    return RP_ERR_RANGE;
  }
  const int32_t n = g.n_nodes;
  if (window_scan_tiles(n) > kNoAllocMaxTiles) {
    set_error("internal: scan tiles exceed the scratch layout");
    return RP_ERR_RANGE;
  }

  WindowWorkspace w;
  w.n_nodes = n;
  w.cap_hits = desc.n_candidates < 1 ? 1 : desc.n_candidates;
  w.cap_entries = 2 * w.cap_hits;
  w.n_tiles = window_scan_tiles(n);
  w.hits.borrow(base + kHitsOff, sizeof(Hit) * w.cap_hits);
  w.entries.borrow(base + kEntOff, sizeof(int2) * w.cap_entries);
  w.erank.borrow(base + kErankOff, sizeof(int32_t) * w.cap_entries);
  w.tmp_e.borrow(base + kTmpEOff, sizeof(int2) * w.cap_entries);
  w.tmp_r.borrow(base + kTmpROff, sizeof(int32_t) * w.cap_entries);
  w.row_ptr.borrow(base + kRowPtrOff, sizeof(int32_t) * ((size_t)n + 1));
  w.deg.borrow(base + kDegOff, sizeof(int32_t) * ((size_t)n + 1));
  w.long_rows.borrow(base + kLongOff, sizeof(int32_t) * ((size_t)n + 1));
  w.tiles.borrow(base + kTilesOff, sizeof(int32_t) * (size_t)w.n_tiles);
  w.counters.borrow(base + kCtrOff, sizeof(unsigned long long) * 4);
  w.win.borrow(base + kWinOff, sizeof(WinDesc));
  w.ranges.borrow(base + kRangeOff, sizeof(CandRange) * kClasses);

  // The builder zeroes its hit counters and degree cursors itself; the
  // window descriptor and candidate ranges are uploaded from the stack
  // (pageable source: the copy is staged before cudaMemcpyAsync returns).
  RP_TRY_CUDA(cudaMemcpyAsync(w.win.ptr, &desc, sizeof(WinDesc), cudaMemcpyHostToDevice, st));
  if (desc.n_ranges > 0)
    RP_TRY_CUDA(cudaMemcpyAsync(w.ranges.ptr, ranges, sizeof(CandRange) * desc.n_ranges,
                                cudaMemcpyHostToDevice, st));
  enqueue_window_build(g, w, 0, desc, cap, weight_kind, true, st);
  unsigned long long hits_raw = 0;
  RP_TRY_CUDA(cudaMemcpyAsync(&hits_raw, w.counters.as<unsigned long long>() + 3,
                              sizeof(hits_raw), cudaMemcpyDeviceToHost, st));
  // compacted pairs go to tmp_e (free once the rows are sorted), the row
  // pointers straight to the caller
  enqueue_window_compact(w, d_row_ptr, w.tmp_e.as<int2>(), st);
  int32_t total = 0;
  RP_TRY_CUDA(cudaMemcpyAsync(&total, d_row_ptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RP_TRY_CUDA(cudaStreamSynchronize(st));
  *nnz = total;
  *n_hits = (int64_t)hits_raw < cap ? (int64_t)hits_raw : cap;
  if (total > capacity) {
    set_error("CSR has %d entries, capacity %lld", total, (long long)capacity);
    return RP_ERR_RANGE;
  }
  if (total > 0) {
    RP_TRY_CUDA(cudaMemcpyAsync(d_entries, w.tmp_e.ptr, sizeof(int2) * (size_t)total,
                                cudaMemcpyDeviceToDevice, st));
    RP_TRY_CUDA(cudaStreamSynchronize(st));
  }
  return RP_OK;
}

}  // namespace
}  // namespace rp

extern "C" RP_API rp_status rp_window_csr_noalloc(rp_graph *g, int64_t ws, int64_t we,
                                                  float scale, int32_t weight_kind,
                                                  int32_t ncls_cap, int32_t *d_row_ptr,
                                                  int32_t *d_entries, int64_t capacity,
                                                  int64_t *nnz, int64_t *n_hits, void *stream) {
  if (!g) {
    rp::set_error("null graph");
    return RP_ERR_ARG;
  }
  return rp::window_csr_noalloc(g->g, ws, we, scale, weight_kind, ncls_cap, d_row_ptr, d_entries,
                                capacity, nnz, n_hits, static_cast<cudaStream_t>(stream));
}
