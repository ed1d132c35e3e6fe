// Node-state CSV text formatted on the device.
//
// The reference writes one line per (replica, node) and recorded step,
// "time,simulation_id,node_id,state\n" with state in {susceptible,
// incubating, infectious, resistant}, replicas outer and nodes inner
// (write_simulation_state, tool/gpu_cpu_temporal_sim.cu:505-568).  Here a
// chunk of replica rows [r0, r1) of one step is formatted in two passes:
//   k_text_rows   per replica row (one block): its byte length;
//   k_text_scan   exclusive scan of the row lengths (one block);
//   k_text_write  per replica row: threads own contiguous node segments,
//                 a block scan of segment lengths gives each thread's
//                 offset, and every thread writes its lines.
// The node-index digit count sum_i digits(i) is the same for every row and
// is computed on the host.
#include "rp_internal.h"

namespace rp {
namespace {

constexpr int kTextThreads = 256;

__device__ __constant__ char kNames[4][12] = {"susceptible", "incubating", "infectious",
                                              "resistant"};
__device__ __constant__ int kNameLen[4] = {11, 10, 10, 9};

__device__ __forceinline__ int digits_u64(unsigned long long x) {
  int d = 1;
  while (x >= 10ull) {
    x /= 10ull;
    ++d;
  }
  return d;
}

__device__ __forceinline__ int len_i64(long long x) {
  return x < 0 ? 1 + digits_u64(0ull - (unsigned long long)x) : digits_u64((unsigned long long)x);
}

// Writes x in decimal at p; returns the end.
__device__ __forceinline__ char *put_i64(char *p, long long x) {
  unsigned long long u = (unsigned long long)x;
  if (x < 0) {
    *p++ = '-';
    u = 0ull - u;
  }
  char tmp[20];
  int n = 0;
  do {
    tmp[n++] = (char)('0' + (int)(u % 10ull));
    u /= 10ull;
  } while (u);
  while (n) *p++ = tmp[--n];
  return p;
}

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *sh, T &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (int)(blockDim.x >> 5) ? sh[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;
  }
  __syncthreads();
  const T off = warp ? sh[warp - 1] : T(0);
  total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return off + x - v;
}

// Byte length of each replica row of the chunk.
__global__ void __launch_bounds__(kTextThreads)
    k_text_rows(const uint8_t *__restrict__ cls, int32_t n, int32_t r0, long long ts,
                long long node_digits, long long *__restrict__ rowlen) {
  __shared__ long long sh[32];
  const int32_t r = r0 + blockIdx.x;
  const uint8_t *row = cls + (int64_t)r * n;
  long long names = 0;
  for (int32_t i = threadIdx.x; i < n; i += blockDim.x) names += kNameLen[row[i] & 3];
  long long total;
  block_excl_scan(names, sh, total);
  if (threadIdx.x == 0)
    rowlen[blockIdx.x] = total + node_digits + (long long)n * (len_i64(ts) + len_i64(r) + 4);
}

// Exclusive scan of the chunk's row lengths (one block); total at [rows].
__global__ void __launch_bounds__(1024)
    k_text_scan(const long long *__restrict__ rowlen, int32_t rows, long long *__restrict__ rowoff) {
  __shared__ long long sh[32];
  const int32_t per = (rows + blockDim.x - 1) / blockDim.x;
  const int32_t b = threadIdx.x * per, e = min(rows, b + per);
  long long s = 0;
  for (int32_t k = b; k < e; ++k) s += rowlen[k];
  long long total;
  long long run = block_excl_scan(s, sh, total);
  for (int32_t k = b; k < e; ++k) {
    rowoff[k] = run;
    run += rowlen[k];
  }
  if (threadIdx.x == 0) rowoff[rows] = total;
}

__global__ void __launch_bounds__(kTextThreads)
    k_text_write(const uint8_t *__restrict__ cls, int32_t n, int32_t r0, long long ts,
                 const long long *__restrict__ rowoff, char *__restrict__ out) {
  __shared__ long long sh[32];
  const int32_t r = r0 + blockIdx.x;
  const uint8_t *row = cls + (int64_t)r * n;
  const int32_t per = (n + blockDim.x - 1) / blockDim.x;
  const int32_t b = threadIdx.x * per, e = min(n, b + per);
  const int fixed = len_i64(ts) + len_i64(r) + 4;  // three commas and the newline
  long long seg = 0;
  for (int32_t i = b; i < e; ++i) seg += fixed + len_i64(i) + kNameLen[row[i] & 3];
  long long total;
  const long long off = block_excl_scan(seg, sh, total);
  char *p = out + rowoff[blockIdx.x] + off;
  for (int32_t i = b; i < e; ++i) {
    p = put_i64(p, ts);
    *p++ = ',';
    p = put_i64(p, r);
    *p++ = ',';
    p = put_i64(p, i);
    *p++ = ',';
    const int c = row[i] & 3;
    for (int k = 0; k < kNameLen[c]; ++k) *p++ = kNames[c][k];
    *p++ = '\n';
  }
}

}  // namespace

int64_t text_line_bound(int32_t n_nodes) {
  // 20 chars of timestamp, 11 of replica, 11 of node, 11 of state, 4 separators
  (void)n_nodes;
  return 57;
}

void enqueue_states_text(const uint8_t *cls, int32_t n, int32_t r0, int32_t r1, int64_t ts,
                         int64_t node_digits, int64_t *rowlen, int64_t *rowoff, char *out,
                         cudaStream_t st) {
  const int32_t rows = r1 - r0;
  if (rows <= 0) return;
  k_text_rows<<<rows, kTextThreads, 0, st>>>(cls, n, r0, (long long)ts, (long long)node_digits,
                                             reinterpret_cast<long long *>(rowlen));
  k_text_scan<<<1, 1024, 0, st>>>(reinterpret_cast<const long long *>(rowlen), rows,
                                  reinterpret_cast<long long *>(rowoff));
  k_text_write<<<rows, kTextThreads, 0, st>>>(cls, n, r0, (long long)ts,
                                              reinterpret_cast<const long long *>(rowoff), out);
}

}  // namespace rp
