// Batched path, countdown mode: the reference's own transition rules
// (initialize_countdown_vector, generate_infectious_vector,
// compute_infection_probability, monte_carlo_simulation and
// update_countdown_vector, tool/gpu_cpu_temporal_sim.cu:73-176) for every
// replica of the batch in one kernel per step.
//
// A replica's countdown is deterministic between infections: after the
// reference sets c = (int)((float)base + step) it only ever applies
// c = max(0, (int)((float)c - step)).  So the host enumerates the values a
// replica can take within the replay -- the sequence from an infection
// (base = E + I + R) and the one from an initial infection (base = I + R),
// each cut after n_steps + 2 values -- and the device stores per (node,
// replica) a code into that table: code 0 is c == 0 (susceptible), and
// table entry k holds the code after one more decrement, the summary class
// of the value (0 S, 1 E, 2 I, 3 R: countdown_class) and whether the value
// is infectious (R < c <= I + R).  Codes are 8 bits when the table has at
// most 256 entries, else 16 bits.
//
// Layout in HBM, node-major like the geometric planes: every node row holds
// W words x 32 replica codes (W padded to a multiple of 4), and the
// infectious bits of the codes are kept bit-packed (mask_in / mask_out,
// alternating per step) for the exposure gather.
//
// k_cd_step, one lane per (node, 32-replica word):
//   1. S = replicas with code 0; inf = OR of the neighbours' mask_in words
//      (the CSR's rows are sorted in the reference's merge order);
//   2. exposed replicas (inf & S) draw their uniform (the plain path's
//      stream: Philox counter (node, step, replica / 4, 3), output
//      replica % 4, on the 24-bit grid) and are candidates when
//      u < x_max = -log(1 - p) * (e_max / 3600), e_max the row's total
//      weight (every FP32 in-order partial sum of a subset is at most the
//      full one, and P <= x);
//   3. candidates accumulate their exposure in the reference's order (one
//      FP32 add per infectious neighbour, in CSR order, as Eigen's row-major
//      product does), then P = 1 - exp(-x) with
//      x = -log(1 - p) * (e / 3600), and infect iff P > u;
//   4. every code advances one decrement (an infection enters the infection
//      sequence and takes its first decrement in the same step), the new
//      codes and the new infectious word are written, and class changes are
//      counted per replica (signed E, I, R deltas).
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kCdThreads = 256;
constexpr int kCdWarps = kCdThreads / 32;
constexpr int kCdTabSmem = 8192;  // table entries kept in shared memory

// Table entry: next code (16 bits) | class << 16 | infectious << 18.
__device__ __forceinline__ uint32_t tab_next(uint32_t e) { return e & 0xFFFFu; }
__device__ __forceinline__ uint32_t tab_cls(uint32_t e) { return (e >> 16) & 3u; }
__device__ __forceinline__ uint32_t tab_inf(uint32_t e) { return (e >> 18) & 1u; }

// Signed per-replica class deltas in a 64-bit word: E, I, R in 16-bit
// fields (shared-memory counters of one task) or 21-bit fields (the step's
// event row), added modulo 2^64.
__device__ __forceinline__ unsigned long long cls_enc(uint32_t cls, int bits) {
  return cls == 0 ? 0ull : (1ull << (bits * (int)(cls - 1)));
}
__device__ __forceinline__ int64_t sext(unsigned long long v, int bits) {
  const unsigned long long m = (1ull << bits) - 1ull;
  const unsigned long long x = v & m;
  return (x >> (bits - 1)) ? (int64_t)x - (int64_t)(1ull << bits) : (int64_t)x;
}
// Splits a modular sum of three signed fields of `bits` bits each.
__device__ __forceinline__ void dec3(unsigned long long v, int bits, int64_t d[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d[k] = sext(v, bits);
    v = (v - (unsigned long long)d[k]) >> bits;
  }
}

template <typename CodeT>
struct CodeVec;  // 32 codes of one word, loaded and stored as 16-byte vectors
template <>
struct CodeVec<uint8_t> {
  static constexpr int kVec = 2;
  __device__ static uint32_t get(const uint4 (&v)[kVec], int r) {
    const uint4 &q = v[r >> 4];
    const int k = (r >> 2) & 3;
    const uint32_t w = k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
    return (w >> (8 * (r & 3))) & 0xFFu;
  }
  __device__ static void set(uint4 (&v)[kVec], int r, uint32_t code) {
    uint4 &q = v[r >> 4];
    const int k = (r >> 2) & 3, sh = 8 * (r & 3);
    uint32_t &w = k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
    w = (w & ~(0xFFu << sh)) | (code << sh);
  }
};
template <>
struct CodeVec<uint16_t> {
  static constexpr int kVec = 4;
  __device__ static uint32_t get(const uint4 (&v)[kVec], int r) {
    const uint4 &q = v[r >> 3];
    const int k = (r >> 1) & 3;
    const uint32_t w = k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
    return (w >> (16 * (r & 1))) & 0xFFFFu;
  }
  __device__ static void set(uint4 (&v)[kVec], int r, uint32_t code) {
    uint4 &q = v[r >> 3];
    const int k = (r >> 1) & 3, sh = 16 * (r & 1);
    uint32_t &w = k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
    w = (w & ~(0xFFFFu << sh)) | (code << sh);
  }
};

__device__ __forceinline__ uint32_t word_mask(const PackedLayout &L, int word) {
  return word < L.vwords - 1 ? kFull : (word == L.vwords - 1 ? L.last_mask : 0u);
}

template <typename CodeT>
__global__ void __launch_bounds__(kCdThreads)
    k_cd_step(PackedLayout L, const PackedTask *__restrict__ tasks,
              const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
              const uint32_t *__restrict__ mask_in, uint32_t *__restrict__ mask_out,
              CodeT *__restrict__ codes, const uint32_t *__restrict__ tab, int32_t n_codes,
              uint32_t infect_code, unsigned long long *__restrict__ ev_row, uint32_t step,
              StepConsts c) {
  using V = CodeVec<CodeT>;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  unsigned long long *s_ev = reinterpret_cast<unsigned long long *>(s_dyn);  // 128 x 32
  float *s_acc = reinterpret_cast<float *>(s_ev + 128 * 32);  // [warp][replica][lane]
  uint32_t *s_tab = reinterpret_cast<uint32_t *>(s_acc + kCdWarps * 32 * 32);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float *acc = s_acc + warp * 32 * 32;
  const bool tab_smem = n_codes <= kCdTabSmem;
  if (tab_smem)
    for (int j = threadIdx.x; j < n_codes; j += blockDim.x) s_tab[j] = tab[j];
  const uint32_t *tb = tab_smem ? s_tab : tab;
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int wbase = T.slice * 128;
    const int nw = min(128, L.words - wbase);
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) s_ev[j] = 0;
    __syncthreads();
    const int64_t items = (int64_t)(T.row_end - T.row_begin) * nw;
    // warp-uniform trip count
    for (int64_t it0 = (int64_t)warp * 32; it0 < items; it0 += (int64_t)kCdWarps * 32) {
      const int64_t it = it0 + lane;
      const bool valid = it < items;
      const int row = T.row_begin + (valid ? (int)(it / nw) : 0);
      const int wl = valid ? (int)(it % nw) : 0;
      const int word = wbase + wl;
      const uint32_t vm = valid ? word_mask(L, word) : 0u;
      const int64_t wi = (int64_t)row * L.words + word;
      uint4 cv[V::kVec];
      const uint4 *src = reinterpret_cast<const uint4 *>(codes + wi * 32);
#pragma unroll
      for (int k = 0; k < V::kVec; ++k) cv[k] = vm ? src[k] : make_uint4(0, 0, 0, 0);
      uint32_t S = 0;
#pragma unroll
      for (int r = 0; r < 32; ++r) S |= (V::get(cv, r) == 0u ? 1u : 0u) << r;
      S &= vm;
      uint32_t X = 0;
      float efmax = 0.0f;
      int32_t beg = 0, npr = 0;
      if (S) {
        beg = row_ptr[row];
        npr = row_ptr[row + 1] - beg;
        uint32_t inf = 0;
        int k = 0;
        for (; k + 4 <= npr; k += 4) {
          const int2 q0 = ent[beg + k], q1 = ent[beg + k + 1], q2 = ent[beg + k + 2],
                     q3 = ent[beg + k + 3];
          inf |= mask_in[(int64_t)q0.x * L.words + word] | mask_in[(int64_t)q1.x * L.words + word] |
                 mask_in[(int64_t)q2.x * L.words + word] | mask_in[(int64_t)q3.x * L.words + word];
          efmax = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(efmax, __int_as_float(q0.y)),
                                                __int_as_float(q1.y)),
                                      __int_as_float(q2.y)),
                            __int_as_float(q3.y));
        }
        for (; k < npr; ++k) {
          const int2 q0 = ent[beg + k];
          inf |= mask_in[(int64_t)q0.x * L.words + word];
          efmax = __fadd_rn(efmax, __int_as_float(q0.y));
        }
        X = inf & S;
      }
      uint32_t evS = 0;
      if (X) {
        // candidates: u < x_max (P <= x <= x_max)
        const float xmax = __fmul_rn(c.neg_log_base, __fdiv_rn(efmax, 3600.0f));
        const uint32_t gq = (uint32_t)(word * 8) + (c.roff >> 2);  // global quad of replica 0
        uint32_t cand = 0;
        uint32_t ub[32];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (!((X >> (4 * q)) & 0xFu)) continue;
          uint32_t x[4];
          philox4x32_10((uint32_t)row, step, gq + (uint32_t)q, kStreamInfect, c.key0, c.key1, x);
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) {
            const int r = 4 * q + cc;
            ub[r] = x[cc];
            if (((X >> r) & 1u) && unit24(x[cc]) < xmax) cand |= 1u << r;
          }
        }
        if (cand) {
          // exposure of each candidate in CSR order (FP32 adds, as the
          // reference's SpMM accumulates a row)
          for (uint32_t t = cand; t; t &= t - 1) acc[(__ffs(t) - 1) * 32 + lane] = 0.0f;
          for (int k = 0; k < npr; ++k) {
            const int2 q0 = ent[beg + k];
            uint32_t hit = mask_in[(int64_t)q0.x * L.words + word] & cand;
            while (hit) {
              const int r = __ffs(hit) - 1;
              acc[r * 32 + lane] = __fadd_rn(acc[r * 32 + lane], __int_as_float(q0.y));
              hit &= hit - 1;
            }
          }
          for (uint32_t t = cand; t; t &= t - 1) {
            const int r = __ffs(t) - 1;
            const float e = __fdiv_rn(acc[r * 32 + lane], 3600.0f);
            const float P = one_minus_exp_neg(__fmul_rn(c.neg_log_base, e));
            if (P > unit24(ub[r])) evS |= 1u << r;
          }
        }
      }
      // ---- advance every code; infectious word; class changes ----
      uint32_t minf = 0;
      bool changed = false;
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        if (!((vm >> r) & 1u)) continue;
        const uint32_t code = V::get(cv, r);
        const uint32_t e0 = tb[code];
        const uint32_t nc = code == 0u ? (((evS >> r) & 1u) ? infect_code : 0u) : tab_next(e0);
        if (nc == code) {
          minf |= tab_inf(e0) << r;
          continue;
        }
        const uint32_t e1 = tb[nc];
        minf |= tab_inf(e1) << r;
        V::set(cv, r, nc);
        changed = true;
        const uint32_t c0 = tab_cls(e0), c1 = tab_cls(e1);
        if (c0 != c1) atomicAdd(&s_ev[wl * 32 + r], cls_enc(c1, 16) - cls_enc(c0, 16));
      }
      if (changed) {
        uint4 *dst = reinterpret_cast<uint4 *>(codes + wi * 32);
#pragma unroll
        for (int k = 0; k < V::kVec; ++k) dst[k] = cv[k];
      }
      if (valid) mask_out[wi] = minf;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) {
      const unsigned long long v = s_ev[j];
      const int rep = wbase * 32 + j;
      if (!v || rep >= L.m) continue;
      int64_t d[3];
      dec3(v, 16, d);
      const unsigned long long g = (unsigned long long)d[0] +
                                   ((unsigned long long)d[1] << 21) +
                                   ((unsigned long long)d[2] << 42);
      if (g) atomicAdd(&ev_row[T.count_base + rep], g);
    }
    __syncthreads();
  }
}

// Initial codes from the initial-infection bit plane (sa after packed_init):
// infected replicas take `init_code`, the rest code 0; the infectious words
// and the initial class counts (E | I << 21 | R << 42 per replica).
template <typename CodeT>
__global__ void __launch_bounds__(kCdThreads)
    k_cd_init(PackedLayout L, const PackedTask *__restrict__ tasks,
              const uint32_t *__restrict__ infected, CodeT *__restrict__ codes,
              uint32_t *__restrict__ mask, const uint32_t *__restrict__ tab, uint32_t init_code,
              unsigned long long *__restrict__ init_counts) {
  __shared__ unsigned long long s_cnt[128 * 32];
  const uint32_t e = tab[init_code];
  const uint32_t cls = tab_cls(e), inf = tab_inf(e);
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int wbase = T.slice * 128;
    const int nw = min(128, L.words - wbase);
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) s_cnt[j] = 0;
    __syncthreads();
    const int64_t items = (int64_t)(T.row_end - T.row_begin) * nw * 32;
    for (int64_t it = threadIdx.x; it < items; it += blockDim.x) {
      const int row = T.row_begin + (int)(it / (nw * 32));
      const int rem = (int)(it % (nw * 32));
      const int wl = rem >> 5, r = rem & 31;
      const int word = wbase + wl;
      const int64_t wi = (int64_t)row * L.words + word;
      const uint32_t bits = infected[wi] & word_mask(L, word);
      const bool on = (bits >> r) & 1u;
      codes[wi * 32 + r] = (CodeT)(on ? init_code : 0u);
      if (r == 0) mask[wi] = inf ? bits : 0u;
      if (on && cls) atomicAdd(&s_cnt[wl * 32 + r], 1ull << (21 * (cls - 1)));
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) {
      const int rep = wbase * 32 + j;
      if (rep < L.m && s_cnt[j]) atomicAdd(&init_counts[T.count_base + rep], s_cnt[j]);
    }
    __syncthreads();
  }
}

// counts[t][net][r][4] (E, I, R, S) from the initial counts and the per-step
// signed class deltas.
__global__ void k_cd_finalize(const unsigned long long *__restrict__ init,
                              const unsigned long long *__restrict__ ev, int32_t steps,
                              int32_t per_row, const int32_t *__restrict__ net_size, int32_t m,
                              int32_t *__restrict__ counts) {
  const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= per_row) return;
  const unsigned long long fm = (1ull << 21) - 1;
  const int64_t N = net_size[j / m];
  const unsigned long long p = init[j];
  int64_t E = (int64_t)(p & fm), I = (int64_t)((p >> 21) & fm), R = (int64_t)((p >> 42) & fm);
  int32_t *o = counts + (int64_t)j * 4;
  o[0] = (int32_t)E;
  o[1] = (int32_t)I;
  o[2] = (int32_t)R;
  o[3] = (int32_t)(N - E - I - R);
  for (int32_t t = 0; t < steps; ++t) {
    int64_t d[3];
    dec3(ev[(int64_t)t * per_row + j], 21, d);
    E += d[0];
    I += d[1];
    R += d[2];
    o = counts + ((int64_t)(t + 1) * per_row + j) * 4;
    o[0] = (int32_t)E;
    o[1] = (int32_t)I;
    o[2] = (int32_t)R;
    o[3] = (int32_t)(N - E - I - R);
  }
}

// Node classes (replica-major, as the node-state output wants them).
template <typename CodeT>
__global__ void __launch_bounds__(256)
    k_cd_classify(PackedLayout L, const CodeT *__restrict__ codes, const uint32_t *__restrict__ tab,
                  uint8_t *__restrict__ out) {
  const int64_t total = (int64_t)L.n_nodes * L.m;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = (int32_t)(g / L.n_nodes), i = (int32_t)(g % L.n_nodes);
    out[g] = (uint8_t)tab_cls(tab[codes[((int64_t)i * L.words + (r >> 5)) * 32 + (r & 31)]]);
  }
}

int cd_grid(int n_tasks) {
  int g = n_tasks < 148 * 4 ? n_tasks : 148 * 4;
  return g < 1 ? 1 : g;
}

size_t cd_smem(int32_t n_codes) {
  return sizeof(unsigned long long) * 128 * 32 + sizeof(float) * kCdWarps * 32 * 32 +
         (n_codes <= kCdTabSmem ? sizeof(uint32_t) * (size_t)n_codes : 0);
}

}  // namespace

rp_status cd_prepare() {
  const int max_smem = (int)cd_smem(kCdTabSmem);
  cudaError_t e = cudaFuncSetAttribute(k_cd_step<uint8_t>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_cd_step<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             max_smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_cd_step)");
  return RP_OK;
}

void cd_init(const PackedLayout &L, const PackedTask *tasks, const uint32_t *infected,
             void *codes, int code_bytes, uint32_t *mask, const uint32_t *tab,
             uint32_t init_code, unsigned long long *init_counts, cudaStream_t st) {
  const int g = cd_grid(L.n_tasks);
  if (code_bytes == 1)
    k_cd_init<uint8_t><<<g, kCdThreads, 0, st>>>(L, tasks, infected, static_cast<uint8_t *>(codes),
                                                 mask, tab, init_code, init_counts);
  else
    k_cd_init<uint16_t><<<g, kCdThreads, 0, st>>>(
        L, tasks, infected, static_cast<uint16_t *>(codes), mask, tab, init_code, init_counts);
}

void cd_step(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
             const int2 *entries, const uint32_t *mask_in, uint32_t *mask_out, void *codes,
             int code_bytes, const uint32_t *tab, int32_t n_codes, uint32_t infect_code,
             unsigned long long *ev_row, uint32_t step, const StepConsts &c, cudaStream_t st) {
  const int g = cd_grid(L.n_tasks);
  const size_t smem = cd_smem(n_codes);
  if (code_bytes == 1)
    k_cd_step<uint8_t><<<g, kCdThreads, smem, st>>>(L, tasks, row_ptr, entries, mask_in, mask_out,
                                                    static_cast<uint8_t *>(codes), tab, n_codes,
                                                    infect_code, ev_row, step, c);
  else
    k_cd_step<uint16_t><<<g, kCdThreads, smem, st>>>(L, tasks, row_ptr, entries, mask_in, mask_out,
                                                     static_cast<uint16_t *>(codes), tab, n_codes,
                                                     infect_code, ev_row, step, c);
}

void cd_finalize(const unsigned long long *init, const unsigned long long *ev, int32_t steps,
                 int32_t per_row, const int32_t *net_size, int32_t m, int32_t *counts,
                 cudaStream_t st) {
  k_cd_finalize<<<(per_row + 127) / 128, 128, 0, st>>>(init, ev, steps, per_row, net_size, m,
                                                      counts);
}

void cd_classify(const PackedLayout &L, const void *codes, int code_bytes, const uint32_t *tab,
                 uint8_t *out, cudaStream_t st) {
  if (code_bytes == 1)
    k_cd_classify<uint8_t><<<1184, 256, 0, st>>>(L, static_cast<const uint8_t *>(codes), tab, out);
  else
    k_cd_classify<uint16_t><<<1184, 256, 0, st>>>(L, static_cast<const uint16_t *>(codes), tab,
                                                  out);
}

}  // namespace rp
