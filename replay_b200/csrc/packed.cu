// Batched path: replica-bit-packed state, one fused kernel per step.
//
// Layout in HBM, node-major with replicas packed 32 per uint32 word
// (words = ceil(M / 32) per node):
//   sa, sb    state planes; replica bit (a, b): S (0,0), E (0,1), I (1,0),
//             R (1,1)
//   mask_t    infectious bits of step t (= a & ~b), double-buffered: step t
//             reads mask_t of the neighbours and writes mask_{t+1}
// The CSR of the step's window is {col, weight} pairs (int32 contact-seconds).
//
// k_packed_step, per (row, word) lane:
//   1. read the state planes, decode S/E/I/R masks;
//   2. exposure: for every neighbour j, m = mask_t[j, word] & S; replicas
//      with a set bit accumulate the edge weight (exact integer sums, the
//      replacement of cusparseSpMM, tool/gpu_cpu_temporal_sim.cu:1062);
//   3. transition: one Philox uniform per replica that can move, keyed
//      (seed, replica, node, step), same rules and same uniforms as the
//      plain path's k_transition_geometric;
//   4. write changed planes and mask_{t+1};
//   5. count transition events per replica in bit-sliced (vertical)
//      counters, reduce them per CTA and add them to the step's event row;
//      counts(t+1) = counts(t) + events(t) is resolved by k_finalize.
// A warp covers `ws` words of 32/ws rows at a time; a task is a run of rows
// of one network for one 32-word slice.
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kPlanes = 8;  // vertical counters hold up to 255 events/lane

// Event fields of one u64: S->E | ->I | I-> , 21 bits each.
constexpr int kFieldBits = 21;

__device__ __forceinline__ void vc_add(uint32_t (&P)[kPlanes], uint32_t m) {
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) {
    const uint32_t t = P[k] & m;
    P[k] ^= m;
    m = t;
    if (!m) break;
  }
}

__device__ __forceinline__ uint32_t vc_count(const uint32_t (&P)[kPlanes], int r) {
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) c |= ((P[k] >> r) & 1u) << k;
  return c;
}

__device__ __forceinline__ uint32_t vc_any(const uint32_t (&P)[kPlanes]) {
  uint32_t o = 0;
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) o |= P[k];
  return o;
}

template <int WS>
__device__ __forceinline__ unsigned long long group_sum(unsigned long long v) {
  // sum over lanes with the same word offset (lane % WS)
#pragma unroll
  for (int o = WS; o < 32; o <<= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Flushes the lane's vertical counters into the CTA's shared event rows.
template <int WS>
__device__ void flush_events(uint32_t (&cSE)[kPlanes], uint32_t (&cXI)[kPlanes],
                             uint32_t (&cIX)[kPlanes], uint32_t (&cRS)[kPlanes],
                             unsigned long long *s_ev, unsigned long long *s_rs,
                             int wsub, int rsub) {
  const uint32_t any = vc_any(cSE) | vc_any(cXI) | vc_any(cIX);
  const uint32_t any_rs = vc_any(cRS);
  const uint32_t any_w = __reduce_or_sync(kFull, any | any_rs);
  if (!any_w) return;
#pragma unroll 1
  for (int r = 0; r < 32; ++r) {
    if (!((any_w >> r) & 1u)) continue;
    unsigned long long v = (unsigned long long)vc_count(cSE, r) |
                           ((unsigned long long)vc_count(cXI, r) << kFieldBits) |
                           ((unsigned long long)vc_count(cIX, r) << (2 * kFieldBits));
    unsigned long long w = vc_count(cRS, r);
    v = group_sum<WS>(v);
    w = group_sum<WS>(w);
    if (rsub == 0) {
      if (v) atomicAdd(&s_ev[wsub * 32 + r], v);
      if (w) atomicAdd(&s_rs[wsub * 32 + r], w);
    }
  }
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) cSE[k] = cXI[k] = cIX[k] = cRS[k] = 0;
}

template <int WS, typename Acc>
__global__ void __launch_bounds__(256, 2)
    k_packed_step(PackedLayout L, const PackedTask *__restrict__ tasks,
                  const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
                  const uint32_t *__restrict__ mask_in, uint32_t *__restrict__ mask_out,
                  uint32_t *__restrict__ sa, uint32_t *__restrict__ sb,
                  unsigned long long *__restrict__ ev_row,
                  unsigned long long *__restrict__ rs_row, uint32_t step, float scale,
                  StepConsts c) {
  constexpr int RG = 32 / WS;
  __shared__ unsigned long long s_ev[WS * 32];
  __shared__ unsigned long long s_rs[WS * 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int rsub = lane / WS, wsub = lane % WS;
  const int W = L.words;
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    for (int j = threadIdx.x; j < WS * 32; j += blockDim.x) {
      s_ev[j] = 0;
      s_rs[j] = 0;
    }
    __syncthreads();
    const int word = T.slice * WS + wsub;
    const bool word_ok = word < W;
    const uint32_t vmask = word_ok ? (word == W - 1 ? L.last_mask : kFull) : 0u;
    uint32_t cSE[kPlanes], cXI[kPlanes], cIX[kPlanes], cRS[kPlanes];
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) cSE[k] = cXI[k] = cIX[k] = cRS[k] = 0;
    int ev_rows = 0;
    for (int base = T.row_begin + warp * RG; base < T.row_end; base += nwarps * RG) {
      const int row = base + rsub;
      const bool active = word_ok && row < T.row_end;
      uint32_t tSE = 0, tXI = 0, tIX = 0, tRS = 0;
      if (active) {
        const int64_t idx = (int64_t)row * W + word;
        const uint32_t a = sa[idx], b = sb[idx];
        const uint32_t S = ~a & ~b & vmask, E = ~a & b, I = a & ~b, R = a & b;
        Acc acc[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) acc[r] = 0;
        uint32_t exposed = 0;
        if (S) {
          const int32_t beg = row_ptr[row], end = row_ptr[row + 1];
          for (int32_t k = beg; k < end; ++k) {
            const int2 en = ent[k];
            const uint32_t mm = mask_in[(int64_t)en.x * W + word] & S;
            if (mm) {
              exposed |= mm;
#pragma unroll
              for (int r = 0; r < 32; ++r) acc[r] += ((mm >> r) & 1u) ? (Acc)en.y : (Acc)0;
            }
          }
        }
        const uint32_t need = exposed | E | I | (c.p_rs > 0.0f ? R : 0u);
        uint32_t na = a, nb = b;
        if (need) {
          const float sus = c.sus ? c.sus[row] : 1.0f;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if ((need >> (4 * q)) & 0xFu) {
              uint32_t x[4];
              philox4x32_10((uint32_t)row, step, (uint32_t)(word * 8 + q), kStreamStep,
                            c.key0, c.key1, x);
#pragma unroll
              for (int cc = 0; cc < 4; ++cc) {
                const int r = 4 * q + cc;
                const uint32_t bit = 1u << r;
                if (!(need & bit)) continue;
                const float u = unit24(x[cc]);
                if (S & bit) {
                  const float br = c.beta_r ? c.beta_r[word * 32 + r] : c.beta;
                  const float bs = c.sus ? __fmul_rn(br, sus) : br;
                  float ef = (sizeof(Acc) == 8) ? __ll2float_rn((long long)acc[r])
                                                : __int2float_rn((int)acc[r]);
                  if (scale != 1.0f) ef = __fmul_rn(ef, scale);
                  const float P = one_minus_exp_neg(__fmul_rn(bs, ef));
                  if (P > u) {
                    if (c.has_exposed)
                      nb |= bit;
                    else
                      na |= bit;
                  }
                } else if (E & bit) {
                  if (u < c.p_ei) {
                    na |= bit;
                    nb &= ~bit;
                  }
                } else if (I & bit) {
                  if (u < c.p_ir) {
                    if (c.ir_to_s)
                      na &= ~bit;
                    else
                      nb |= bit;
                  }
                } else {
                  if (u < c.p_rs) {
                    na &= ~bit;
                    nb &= ~bit;
                  }
                }
              }
            }
          }
          const uint32_t nI = na & ~nb;
          tSE = S & ~na & nb;
          tXI = (S | E) & nI;
          tIX = I & ~nI;
          tRS = R & ~na & ~nb;
          if (na != a) sa[idx] = na;
          if (nb != b) sb[idx] = nb;
        }
        mask_out[idx] = na & ~nb;
      }
      if (tSE | tXI | tIX | tRS) {
        if (tSE) vc_add(cSE, tSE);
        if (tXI) vc_add(cXI, tXI);
        if (tIX) vc_add(cIX, tIX);
        if (tRS) vc_add(cRS, tRS);
        ++ev_rows;
      }
      if (__any_sync(kFull, ev_rows == (1 << kPlanes) - 1)) {
        flush_events<WS>(cSE, cXI, cIX, cRS, s_ev, s_rs, wsub, rsub);
        ev_rows = 0;
      }
    }
    flush_events<WS>(cSE, cXI, cIX, cRS, s_ev, s_rs, wsub, rsub);
    __syncthreads();
    for (int j = threadIdx.x; j < WS * 32; j += blockDim.x) {
      const int rep = (T.slice * WS + (j >> 5)) * 32 + (j & 31);
      if (rep >= L.m) continue;
      if (s_ev[j]) atomicAdd(&ev_row[T.count_base + rep], s_ev[j]);
      if (rs_row && s_rs[j]) atomicAdd(&rs_row[T.count_base + rep], s_rs[j]);
    }
    __syncthreads();
  }
}

// Full E/I/R counts of the current planes (initial state), same reduction
// with the state masks in place of the event masks.
template <int WS>
__global__ void __launch_bounds__(256)
    k_packed_count(PackedLayout L, const PackedTask *__restrict__ tasks,
                   const uint32_t *__restrict__ sa, const uint32_t *__restrict__ sb,
                   unsigned long long *__restrict__ out) {
  constexpr int RG = 32 / WS;
  __shared__ unsigned long long s_ev[WS * 32];
  __shared__ unsigned long long s_rs[WS * 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int rsub = lane / WS, wsub = lane % WS;
  const int W = L.words;
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    for (int j = threadIdx.x; j < WS * 32; j += blockDim.x) s_ev[j] = s_rs[j] = 0;
    __syncthreads();
    const int word = T.slice * WS + wsub;
    const bool word_ok = word < W;
    uint32_t cE[kPlanes], cI[kPlanes], cR[kPlanes], cZ[kPlanes];
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) cE[k] = cI[k] = cR[k] = cZ[k] = 0;
    int rows = 0;
    for (int base = T.row_begin + warp * RG; base < T.row_end; base += nwarps * RG) {
      const int row = base + rsub;
      if (word_ok && row < T.row_end) {
        const int64_t idx = (int64_t)row * W + word;
        const uint32_t a = sa[idx], b = sb[idx];
        vc_add(cE, ~a & b);
        vc_add(cI, a & ~b);
        vc_add(cR, a & b);
      }
      ++rows;
      if (__any_sync(kFull, rows == (1 << kPlanes) - 1)) {
        flush_events<WS>(cE, cI, cR, cZ, s_ev, s_rs, wsub, rsub);
        rows = 0;
      }
    }
    flush_events<WS>(cE, cI, cR, cZ, s_ev, s_rs, wsub, rsub);
    __syncthreads();
    for (int j = threadIdx.x; j < WS * 32; j += blockDim.x) {
      const int rep = (T.slice * WS + (j >> 5)) * 32 + (j & 31);
      if (rep < L.m && s_ev[j]) atomicAdd(&out[T.count_base + rep], s_ev[j]);
    }
    __syncthreads();
  }
}

// Bernoulli(p0) initial infection per (node, replica), stream 1, same
// uniforms as the plain path.  Writes planes and the step-0 mask.
__global__ void __launch_bounds__(256)
    k_packed_init(PackedLayout L, uint32_t *__restrict__ sa, uint32_t *__restrict__ sb,
                  uint32_t *__restrict__ mask, float p0, StepConsts c) {
  const int64_t total = (int64_t)L.n_nodes * L.words;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int32_t row = (int32_t)(idx / L.words);
    const int32_t word = (int32_t)(idx % L.words);
    const uint32_t vmask = word == L.words - 1 ? L.last_mask : kFull;
    uint32_t inf = 0;
    if (p0 > 0.0f) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint32_t x[4];
        philox4x32_10((uint32_t)row, kStepInit, (uint32_t)(word * 8 + q), kStreamInit,
                      c.key0, c.key1, x);
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
    philox4x32_10((uint32_t)j, kStepPick, (uint32_t)r, kStreamPick + 4u * (uint32_t)net,
                  c.key0, c.key1, x);
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

// Exposure only (test hook): exposure[i * m + r] exact int64.
__global__ void __launch_bounds__(256)
    k_packed_exposure(const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
                      int32_t n, const uint32_t *__restrict__ masks, int32_t W, int32_t m,
                      int64_t *__restrict__ exposure) {
  const int64_t total = (int64_t)n * W;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = (int32_t)(g / W), w = (int32_t)(g % W);
    int64_t acc[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) acc[r] = 0;
    for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
      const int2 en = ent[k];
      const uint32_t mm = masks[(int64_t)en.x * W + w];
#pragma unroll
      for (int r = 0; r < 32; ++r) acc[r] += ((mm >> r) & 1u) ? (int64_t)en.y : 0;
    }
#pragma unroll
    for (int r = 0; r < 32; ++r)
      if (w * 32 + r < m) exposure[(int64_t)i * m + w * 32 + r] = acc[r];
  }
}

template <int WS>
void launch_step_ws(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
                    const int2 *entries, const uint32_t *mask_in, uint32_t *mask_out,
                    uint32_t *sa, uint32_t *sb, unsigned long long *ev_row,
                    unsigned long long *rs_row, uint32_t step, float scale, bool wide,
                    const StepConsts &c, int grid, cudaStream_t st) {
  if (wide)
    k_packed_step<WS, long long><<<grid, 256, 0, st>>>(L, tasks, row_ptr, entries, mask_in,
                                                       mask_out, sa, sb, ev_row, rs_row, step,
                                                       scale, c);
  else
    k_packed_step<WS, int><<<grid, 256, 0, st>>>(L, tasks, row_ptr, entries, mask_in, mask_out,
                                                 sa, sb, ev_row, rs_row, step, scale, c);
}

int task_grid(int n_tasks) {
  int g = n_tasks < 148 * 2 ? n_tasks : 148 * 2;
  return g < 1 ? 1 : g;
}

}  // namespace

void packed_init(const PackedLayout &L, uint32_t *sa, uint32_t *sb, uint32_t *mask, float p0,
                 int32_t k_exact, const int32_t *net_of_row, const int32_t *net_first_row,
                 const int32_t *net_rows, int32_t n_nets, const StepConsts &c,
                 cudaStream_t st) {
  (void)net_of_row;
  const int64_t total = (int64_t)L.n_nodes * L.words;
  k_packed_init<<<1184, 256, 0, st>>>(L, sa, sb, mask, k_exact > 0 ? 0.0f : p0, c);
  if (k_exact > 0) {
    const int64_t nt = (int64_t)n_nets * L.m;
    k_packed_pick<<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(L, sa, net_first_row, net_rows,
                                                                n_nets, k_exact, c);
    k_mask_from_planes<<<1184, 256, 0, st>>>(total, sa, sb, mask);
  }
}

void packed_step(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
                 const int2 *entries, const uint32_t *mask_in, uint32_t *mask_out,
                 uint32_t *sa, uint32_t *sb, unsigned long long *ev_row,
                 unsigned long long *rs_row, uint32_t step, float scale, bool wide_acc,
                 const StepConsts &c, cudaStream_t st) {
  const int grid = task_grid(L.n_tasks);
  switch (L.ws) {
    case 1: launch_step_ws<1>(L, tasks, row_ptr, entries, mask_in, mask_out, sa, sb, ev_row, rs_row, step, scale, wide_acc, c, grid, st); break;
    case 2: launch_step_ws<2>(L, tasks, row_ptr, entries, mask_in, mask_out, sa, sb, ev_row, rs_row, step, scale, wide_acc, c, grid, st); break;
    case 4: launch_step_ws<4>(L, tasks, row_ptr, entries, mask_in, mask_out, sa, sb, ev_row, rs_row, step, scale, wide_acc, c, grid, st); break;
    case 8: launch_step_ws<8>(L, tasks, row_ptr, entries, mask_in, mask_out, sa, sb, ev_row, rs_row, step, scale, wide_acc, c, grid, st); break;
    case 16: launch_step_ws<16>(L, tasks, row_ptr, entries, mask_in, mask_out, sa, sb, ev_row, rs_row, step, scale, wide_acc, c, grid, st); break;
    default: launch_step_ws<32>(L, tasks, row_ptr, entries, mask_in, mask_out, sa, sb, ev_row, rs_row, step, scale, wide_acc, c, grid, st); break;
  }
}

void packed_count(const PackedLayout &L, const PackedTask *tasks, const uint32_t *sa,
                  const uint32_t *sb, unsigned long long *counts_row, cudaStream_t st) {
  const int grid = task_grid(L.n_tasks);
  switch (L.ws) {
    case 1: k_packed_count<1><<<grid, 256, 0, st>>>(L, tasks, sa, sb, counts_row); break;
    case 2: k_packed_count<2><<<grid, 256, 0, st>>>(L, tasks, sa, sb, counts_row); break;
    case 4: k_packed_count<4><<<grid, 256, 0, st>>>(L, tasks, sa, sb, counts_row); break;
    case 8: k_packed_count<8><<<grid, 256, 0, st>>>(L, tasks, sa, sb, counts_row); break;
    case 16: k_packed_count<16><<<grid, 256, 0, st>>>(L, tasks, sa, sb, counts_row); break;
    default: k_packed_count<32><<<grid, 256, 0, st>>>(L, tasks, sa, sb, counts_row); break;
  }
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
