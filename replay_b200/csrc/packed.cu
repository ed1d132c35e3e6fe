// Batched path, set-up and read-out kernels: initial conditions (Bernoulli
// and exact-k seeding), full E/I/R counts of the planes, per-step counts
// from the event rows, per-replica node classes, and the exposure test hook.
// The per-step kernel is in step.cu.
//
// Layout in HBM, node-major, 32 replicas per uint32 word; every node row is
// padded to a multiple of 4 words (W words per node):
//   sa, sb    state planes; replica bit (a, b): S (0,0), E (0,1), I (1,0),
//             R (1,1)
//   mask      infectious bits (a & ~b), two buffers alternating per step
//   ev (+rs)  per-replica event counters of every step: S->E | ->I | I->
//             in 21-bit fields (+ R->S), summed into counts by k_finalize
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kFieldBits = 21;  // global event fields: S->E | ->I | I->
constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t word_mask(const PackedLayout &L, int word) {
  return word < L.vwords - 1 ? kFull : (word == L.vwords - 1 ? L.last_mask : 0u);
}

__device__ __forceinline__ void count_bits(unsigned long long *s_ev, int wl, uint32_t t,
                                           unsigned long long inc) {
  while (t) {
    const int r = __ffs(t) - 1;
    atomicAdd(&s_ev[wl * 32 + r], inc);
    t &= t - 1;
  }
}

// Full E/I/R counts of the planes (initial state): one shared atomic per
// set bit, E | I << 21 | R << 42 per replica.
__global__ void __launch_bounds__(kThreads)
    k_packed_count(PackedLayout L, const PackedTask *__restrict__ tasks,
                   const uint32_t *__restrict__ sa, const uint32_t *__restrict__ sb,
                   unsigned long long *__restrict__ out) {
  __shared__ unsigned long long s_ev[128 * 32];
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int wbase = T.slice * 128;
    const int nw = min(128, L.words - wbase);
    for (int j = threadIdx.x; j < 128 * 32; j += blockDim.x) s_ev[j] = 0;
    __syncthreads();
    const int64_t items = (int64_t)(T.row_end - T.row_begin) * nw;
    for (int64_t it = threadIdx.x; it < items; it += blockDim.x) {
      const int row = T.row_begin + (int)(it / nw);
      const int wl = (int)(it % nw);
      const int word = wbase + wl;
      const uint32_t vm = word_mask(L, word);
      const int64_t idx = (int64_t)row * L.words + word;
      const uint32_t a = sa[idx] & vm, b = sb[idx] & vm;
      count_bits(s_ev, wl, ~a & b, 1ull);
      count_bits(s_ev, wl, a & ~b, 1ull << kFieldBits);
      count_bits(s_ev, wl, a & b, 1ull << (2 * kFieldBits));
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) {
      const int rep = wbase * 32 + j;
      if (rep < L.m && s_ev[j]) atomicAdd(&out[T.count_base + rep], s_ev[j]);
    }
    __syncthreads();
  }
}

// Bernoulli(p0) initial infection per (node, replica), stream 1, the plain
// path's uniforms.  Writes planes and the step-0 mask.
__global__ void __launch_bounds__(256)
    k_packed_init(PackedLayout L, uint32_t *__restrict__ sa, uint32_t *__restrict__ sb,
                  uint32_t *__restrict__ mask, float p0, StepConsts c) {
  const int64_t total = (int64_t)L.n_nodes * L.words;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int32_t row = (int32_t)(idx / L.words);
    const int32_t word = (int32_t)(idx % L.words);
    const uint32_t vmask = word_mask(L, word);
    uint32_t inf = 0;
    if (p0 > 0.0f && vmask) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint32_t x[4];
        philox4x32_10((uint32_t)row, kStepInit, (uint32_t)((word + (c.roff >> 5)) * 8 + q), kStreamInit, c.key0,
                      c.key1, x);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc)
          if (unit24(x[cc]) < p0) inf |= 1u << (4 * q + cc);
      }
    }
    inf &= vmask;
    sa[idx] = inf;
    sb[idx] = 0;
    mask[idx] = inf;
  }
}

// Exactly k infected per (network, replica) by Floyd's sampling, stream 2,
// node = index within the network.
__global__ void k_packed_pick(PackedLayout L, uint32_t *__restrict__ sa,
                              const int32_t *__restrict__ net_first_row,
                              const int32_t *__restrict__ net_rows, int32_t n_nets, int32_t k,
                              StepConsts c) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)n_nets * L.m) return;
  const int32_t net = (int32_t)(gid / L.m), r = (int32_t)(gid % L.m);
  const int32_t n = net_rows[net], first = net_first_row[net];
  const uint32_t bit = 1u << (r & 31);
  const int32_t word = r >> 5;
  const int32_t kk = k < n ? k : n;
  for (int32_t j = n - kk; j < n; ++j) {
    uint32_t x[4];
    philox4x32_10((uint32_t)j, kStepPick, (uint32_t)r + c.roff, kStreamPick + 4u * (uint32_t)net, c.key0,
                  c.key1, x);
    const uint64_t r64 = (uint64_t)x[0] | ((uint64_t)x[1] << 32);
    const int32_t t = (int32_t)__umul64hi(r64, (uint64_t)(j + 1));
    const uint32_t old = atomicOr(&sa[(int64_t)(first + t) * L.words + word], bit);
    if (old & bit) atomicOr(&sa[(int64_t)(first + j) * L.words + word], bit);
  }
}

__global__ void k_mask_from_planes(int64_t total, const uint32_t *__restrict__ sa,
                                   const uint32_t *__restrict__ sb, uint32_t *__restrict__ mask) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    mask[i] = sa[i] & ~sb[i];
}

// counts[t][net][r][4] from the initial counts and the per-step events.
__global__ void k_finalize(const unsigned long long *__restrict__ init,
                           const unsigned long long *__restrict__ ev,
                           const unsigned long long *__restrict__ rs, int32_t steps,
                           int32_t per_row, const int32_t *__restrict__ net_size, int32_t m,
                           int32_t has_exposed, int32_t ir_to_s, int32_t *__restrict__ counts) {
  const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= per_row) return;
  const unsigned long long fm = (1ull << kFieldBits) - 1;
  const int64_t N = net_size[j / m];
  const unsigned long long p = init[j];
  int64_t E = (int64_t)(p & fm), I = (int64_t)((p >> kFieldBits) & fm),
          R = (int64_t)((p >> (2 * kFieldBits)) & fm);
  int32_t *o = counts + (int64_t)j * 4;
  o[0] = (int32_t)E;
  o[1] = (int32_t)I;
  o[2] = (int32_t)R;
  o[3] = (int32_t)(N - E - I - R);
  for (int32_t t = 0; t < steps; ++t) {
    const unsigned long long e = ev[(int64_t)t * per_row + j];
    const int64_t se = (int64_t)(e & fm), xi = (int64_t)((e >> kFieldBits) & fm),
                  ix = (int64_t)((e >> (2 * kFieldBits)) & fm);
    const int64_t rsv = rs ? (int64_t)rs[(int64_t)t * per_row + j] : 0;
    E += se - (has_exposed ? xi : 0);
    I += xi - ix;
    R += (ir_to_s ? 0 : ix) - rsv;
    o = counts + ((int64_t)(t + 1) * per_row + j) * 4;
    o[0] = (int32_t)E;
    o[1] = (int32_t)I;
    o[2] = (int32_t)R;
    o[3] = (int32_t)(N - E - I - R);
  }
}

__global__ void k_packed_classify(PackedLayout L, const uint32_t *__restrict__ sa,
                                  const uint32_t *__restrict__ sb, uint8_t *__restrict__ out) {
  const int64_t total = (int64_t)L.n_nodes * L.m;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = (int32_t)(g / L.n_nodes), i = (int32_t)(g % L.n_nodes);
    const int64_t idx = (int64_t)i * L.words + (r >> 5);
    const uint32_t a = (sa[idx] >> (r & 31)) & 1u, b = (sb[idx] >> (r & 31)) & 1u;
    out[g] = (uint8_t)(a ? (b ? 3 : 2) : (b ? 1 : 0));
  }
}

// Exposure only (test hook): exposure[i * m + r] exact int64, masks with
// `W` words per node.
__global__ void __launch_bounds__(256)
    k_packed_exposure(const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
                      int32_t n, const uint32_t *__restrict__ masks, int32_t W, int32_t m,
                      int64_t *__restrict__ exposure) {
  const int64_t total = (int64_t)n * m;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = (int32_t)(g / m), r = (int32_t)(g % m);
    int64_t acc = 0;
    for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
      const int2 en = ent[k];
      if ((masks[(int64_t)en.x * W + (r >> 5)] >> (r & 31)) & 1u) acc += en.y;
    }
    exposure[g] = acc;
  }
}

int task_grid(int n_tasks, int per_sm) {
  int g = n_tasks < 148 * per_sm ? n_tasks : 148 * per_sm;
  return g < 1 ? 1 : g;
}

}  // namespace

rp_status packed_prepare() { return RP_OK; }

void packed_init(const PackedLayout &L, uint32_t *sa, uint32_t *sb, uint32_t *mask,
                 float p0, int32_t k_exact, const int32_t *net_first_row,
                 const int32_t *net_rows, int32_t n_nets, const StepConsts &c,
                 cudaStream_t st) {
  const int64_t total = (int64_t)L.n_nodes * L.words;
  k_packed_init<<<1184, 256, 0, st>>>(L, sa, sb, mask, k_exact > 0 ? 0.0f : p0, c);
  if (k_exact > 0) {
    const int64_t nt = (int64_t)n_nets * L.m;
    k_packed_pick<<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(L, sa, net_first_row, net_rows,
                                                                n_nets, k_exact, c);
    k_mask_from_planes<<<1184, 256, 0, st>>>(total, sa, sb, mask);
  }
}

void packed_count(const PackedLayout &L, const PackedTask *tasks, const uint32_t *sa,
                  const uint32_t *sb, unsigned long long *counts_row, cudaStream_t st) {
  k_packed_count<<<task_grid(L.n_tasks, 2), kThreads, 0, st>>>(L, tasks, sa, sb, counts_row);
}

void packed_finalize_events(const unsigned long long *init, const unsigned long long *ev,
                            const unsigned long long *rs, int32_t steps, int32_t per_row,
                            const int32_t *net_size, int32_t m, int32_t has_exposed,
                            int32_t ir_to_s, int32_t *counts, cudaStream_t st) {
  k_finalize<<<(per_row + 127) / 128, 128, 0, st>>>(init, ev, rs, steps, per_row, net_size, m,
                                                   has_exposed, ir_to_s, counts);
}

void packed_classify(const PackedLayout &L, const uint32_t *sa, const uint32_t *sb,
                     uint8_t *out, cudaStream_t st) {
  k_packed_classify<<<1184, 256, 0, st>>>(L, sa, sb, out);
}

void packed_exposure(const int32_t *row_ptr, const int2 *entries, int32_t n,
                     const uint32_t *masks, int32_t words, int32_t m, int64_t *exposure,
                     cudaStream_t st) {
  k_packed_exposure<<<1184, 256, 0, st>>>(row_ptr, entries, n, masks, words, m, exposure);
}

}  // namespace rp
