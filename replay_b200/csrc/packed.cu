// Batched path: replica-bit-packed state, two kernels per step.
//
// Layout in HBM, node-major, 32 replicas per uint32 word; every node row is
// padded to a multiple of 4 words so that a lane moves 128 replicas with one
// 16-byte access:
//   sa, sb    state planes; replica bit (a, b): S (0,0), E (0,1), I (1,0),
//             R (1,1)
//   mask_t    infectious bits of step t (a & ~b), double-buffered: step t
//             reads mask_t and writes mask_{t+1}
//   evs       infection events of the step, written for rows with contacts
// The window CSR holds {col, weight} pairs (int32 contact-seconds).
//
// k_infect (exposure SpMM + infection draws), per row with contacts, lanes
// over 4-word columns (the replacement of cusparseSpMM,
// tool/gpu_cpu_temporal_sim.cu:1062, and monte_carlo_simulation, :137-159):
//   1. inf = OR over neighbours j of mask_t[j] (16 B per lane per entry);
//   2. exposed = inf & S; the quads (4 replicas) holding exposed replicas are
//      compacted across the warp so every lane draws: exact int64 exposure
//      sums of the quad's replicas over the row's entries, one Philox call,
//      P = 1 - exp(-beta_r s_i e) > u (the replica's infection uniform);
//   3. events go to evs.
// k_flow (transitions + count reduction), every (row, 4-word column):
//   reads the planes and the row's infection events, draws the bit-sliced
//   flow uniforms of the E, I (and waning R) replicas, 32 replicas per random
//   plane (flow_events), applies all moves with bitwise operations, writes the
//   planes and mask_{t+1}, and adds every transition event to per-replica
//   counters in shared memory, flushed once per task to the step's event
//   row; k_finalize turns initial counts + events into per-step counts.
// Every decision uses the state at the start of the step: k_infect reads the
// planes before k_flow rewrites them.
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kFieldBits = 21;  // global event fields: S->E | ->I | I->
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ uint32_t word_mask(const PackedLayout &L, int word) {
  return word < L.vwords - 1 ? kFull : (word == L.vwords - 1 ? L.last_mask : 0u);
}

__device__ __forceinline__ uint32_t get4(const uint4 &v, int w) {
  return w == 0 ? v.x : (w == 1 ? v.y : (w == 2 ? v.z : v.w));
}

// 8-bit mask of the non-empty nibbles of x.
__device__ __forceinline__ uint32_t nibble_any(uint32_t x) {
  x |= x >> 1;
  x |= x >> 2;
  x &= 0x11111111u;
  uint32_t o = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) o |= ((x >> (4 * q)) & 1u) << q;
  return o;
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
    k_infect(PackedLayout L, const PackedTask *__restrict__ tasks,
             const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
             const uint4 *__restrict__ mask_in, const uint4 *__restrict__ sa,
             const uint4 *__restrict__ sb, uint4 *__restrict__ evs, uint32_t step, float scale,
             StepConsts c) {
  __shared__ uint32_t s_exp[kWarps][32][4];
  __shared__ uint32_t s_ev[kWarps][32][4];
  __shared__ int32_t s_off[kWarps][32];
  __shared__ uint32_t s_qm[kWarps][32];
  __shared__ int32_t s_row[kWarps][32];
  __shared__ int32_t s_col[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lpr = L.lpr, rpw = 32 / lpr;
  const int rsub = lane / lpr, csub = lane % lpr;
  const uint32_t *mask_w = reinterpret_cast<const uint32_t *>(mask_in);
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int cbase = T.slice * 32;
    const int ncols = min(32, L.q4 - cbase);
    for (int base = T.row_begin + warp * rpw; base < T.row_end; base += kWarps * rpw) {
      const int row = base + rsub;
      const bool row_ok = row < T.row_end;
      int32_t beg = 0, end = 0;
      if (row_ok) {
        beg = row_ptr[row];
        end = row_ptr[row + 1];
      }
      const bool nonempty = row_ok && end > beg;
      // ---- OR of the neighbours' infectious words, 4 columns per lane ----
      // (warp-uniform trip count: the compaction below shuffles)
      for (int cc0 = 0; cc0 < ncols; cc0 += lpr) {
        const int cc = cc0 + csub;
        const bool col_ok = cc < ncols;
        const int col = cbase + (col_ok ? cc : 0);
        uint4 inf = make_uint4(0, 0, 0, 0);
        if (nonempty && col_ok) {
          int32_t k = beg;
          for (; k + 2 <= end; k += 2) {
            const int2 e0 = ent[k], e1 = ent[k + 1];
            const uint4 m0 = mask_in[(int64_t)e0.x * L.q4 + col];
            const uint4 m1 = mask_in[(int64_t)e1.x * L.q4 + col];
            inf.x |= m0.x | m1.x;
            inf.y |= m0.y | m1.y;
            inf.z |= m0.z | m1.z;
            inf.w |= m0.w | m1.w;
          }
          if (k < end) {
            const int2 e0 = ent[k];
            const uint4 m0 = mask_in[(int64_t)e0.x * L.q4 + col];
            inf.x |= m0.x;
            inf.y |= m0.y;
            inf.z |= m0.z;
            inf.w |= m0.w;
          }
        }
        uint32_t ex[4] = {0, 0, 0, 0};
        if (inf.x | inf.y | inf.z | inf.w) {
          const int64_t idx = (int64_t)row * L.q4 + col;
          const uint4 a = sa[idx], b = sb[idx];
#pragma unroll
          for (int w = 0; w < 4; ++w)
            ex[w] = get4(inf, w) & ~get4(a, w) & ~get4(b, w) & word_mask(L, 4 * col + w);
        }
        uint32_t qm = 0;
#pragma unroll
        for (int w = 0; w < 4; ++w) qm |= nibble_any(ex[w]) << (8 * w);
        // ---- compact the exposed quads of the warp ----
        const int cnt = __popc(qm);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        if (total) {
          s_off[warp][lane] = incl - cnt;
          s_qm[warp][lane] = qm;
          s_row[warp][lane] = row;
          s_col[warp][lane] = col;
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            s_exp[warp][lane][w] = ex[w];
            s_ev[warp][lane][w] = 0;
          }
          __syncwarp();
          for (int p = lane; p < total; p += 32) {
            int owner = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1)
              if (owner + st < 32 && s_off[warp][owner + st] <= p) owner += st;
            uint32_t m = s_qm[warp][owner];
            for (int k = p - s_off[warp][owner]; k > 0; --k) m &= m - 1;
            const int slot = __ffs(m) - 1;
            const int w = slot >> 3, q = slot & 7;
            const int orow = s_row[warp][owner];
            const int word = 4 * s_col[warp][owner] + w;
            const uint32_t bits = (s_exp[warp][owner][w] >> (4 * q)) & 0xFu;
            long long e0 = 0, e1 = 0, e2 = 0, e3 = 0;
            const int32_t ob = row_ptr[orow], oe = row_ptr[orow + 1];
            for (int32_t k = ob; k < oe; ++k) {
              const int2 en = ent[k];
              const uint32_t mw = mask_w[(int64_t)en.x * L.words + word] >> (4 * q);
              e0 += (mw & 1u) ? en.y : 0;
              e1 += (mw & 2u) ? en.y : 0;
              e2 += (mw & 4u) ? en.y : 0;
              e3 += (mw & 8u) ? en.y : 0;
            }
            uint32_t x[4];
            philox4x32_10((uint32_t)orow, step, (uint32_t)(word * 8 + q), kStreamInfect, c.key0,
                          c.key1, x);
            const float sus = c.sus ? c.sus[orow] : 1.0f;
            const long long ev4[4] = {e0, e1, e2, e3};
            uint32_t ev = 0;
#pragma unroll
            for (int cq = 0; cq < 4; ++cq) {
              if ((bits >> cq) & 1u) {
                const int r = word * 32 + 4 * q + cq;
                const float br = c.beta_r ? c.beta_r[r] : c.beta;
                const float bs = c.sus ? __fmul_rn(br, sus) : br;
                float ef = __ll2float_rn(ev4[cq]);
                if (scale != 1.0f) ef = __fmul_rn(ef, scale);
                if (one_minus_exp_neg(__fmul_rn(bs, ef)) > unit24(x[cq]))
                  ev |= 1u << (4 * q + cq);
              }
            }
            if (ev) atomicOr(&s_ev[warp][owner][w], ev);
          }
          __syncwarp();
#pragma unroll
          for (int w = 0; w < 4; ++w) ex[w] = s_ev[warp][lane][w];
          __syncwarp();
        }
        if (nonempty && col_ok)
          evs[(int64_t)row * L.q4 + col] = make_uint4(ex[0], ex[1], ex[2], ex[3]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void count_bits(unsigned long long *s_ev, int wl, uint32_t t,
                                           unsigned long long inc) {
  while (t) {
    const int r = __ffs(t) - 1;
    atomicAdd(&s_ev[wl * 32 + r], inc);
    t &= t - 1;
  }
}

__global__ void __launch_bounds__(kThreads)
    k_flow(PackedLayout L, const PackedTask *__restrict__ tasks,
           const int32_t *__restrict__ row_ptr, const uint4 *__restrict__ evs,
           uint4 *__restrict__ mask_out, uint4 *__restrict__ sa, uint4 *__restrict__ sb,
           unsigned long long *__restrict__ ev_row, unsigned long long *__restrict__ rs_row,
           uint32_t step, StepConsts c) {
  // per task: 128 words x 32 replicas of 4 x 16-bit event counters
  __shared__ unsigned long long s_ev[128 * 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lpr = L.lpr, rpw = 32 / lpr;
  const int rsub = lane / lpr, csub = lane % lpr;
  const bool waning = c.th.tr_all || c.th.tr != 0;
  const unsigned long long kSE = 1ull, kXI = 1ull << 16, kIX = 1ull << 32, kRS = 1ull << 48;
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int cbase = T.slice * 32;
    const int ncols = min(32, L.q4 - cbase);
    for (int j = threadIdx.x; j < 128 * 32; j += blockDim.x) s_ev[j] = 0;
    __syncthreads();
    for (int base = T.row_begin + warp * rpw; base < T.row_end; base += kWarps * rpw) {
      const int row = base + rsub;
      if (row >= T.row_end) continue;
      const bool nonempty = row_ptr[row + 1] > row_ptr[row];
      for (int cc = csub; cc < ncols; cc += lpr) {
        const int col = cbase + cc;
        const int64_t idx = (int64_t)row * L.q4 + col;
        const uint4 a4 = sa[idx], b4 = sb[idx];
        const uint4 e4 = nonempty ? evs[idx] : make_uint4(0, 0, 0, 0);
        uint32_t na[4], nb[4], mo[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const int word = 4 * col + w;
          const uint32_t a = get4(a4, w), b = get4(b4, w);
          na[w] = a;
          nb[w] = b;
          mo[w] = 0;
          if (!word_mask(L, word)) continue;
          const uint32_t E = ~a & b, I = a & ~b, R = a & b;
          const uint32_t evS = get4(e4, w);
          const uint32_t Rw = waning ? R : 0u;
          const uint32_t evF =
              (E | I | Rw) ? flow_events(E, I, Rw, c.th, c.key0, c.key1, (uint32_t)row, step,
                                         (uint32_t)word)
                           : 0u;
          const uint32_t evE = evF & E, evI = evF & I, evR = evF & Rw;
          uint32_t xa = a, xb = b;
          if (c.has_exposed)
            xb |= evS;
          else
            xa |= evS;
          xa |= evE;
          xb &= ~evE;
          if (c.ir_to_s)
            xa &= ~evI;
          else
            xb |= evI;
          xa &= ~evR;
          xb &= ~evR;
          na[w] = xa;
          nb[w] = xb;
          mo[w] = xa & ~xb;
          const int wl = 4 * cc + w;
          if (evS | evE | evI | evR) {
            count_bits(s_ev, wl, c.has_exposed ? evS : 0u, kSE);
            count_bits(s_ev, wl, evE | (c.has_exposed ? 0u : evS), kXI);
            count_bits(s_ev, wl, evI, kIX);
            count_bits(s_ev, wl, evR, kRS);
          }
        }
        const uint4 oa = make_uint4(na[0], na[1], na[2], na[3]);
        const uint4 ob = make_uint4(nb[0], nb[1], nb[2], nb[3]);
        if (oa.x != a4.x || oa.y != a4.y || oa.z != a4.z || oa.w != a4.w) sa[idx] = oa;
        if (ob.x != b4.x || ob.y != b4.y || ob.z != b4.z || ob.w != b4.w) sb[idx] = ob;
        mask_out[idx] = make_uint4(mo[0], mo[1], mo[2], mo[3]);
      }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < ncols * 128; j += blockDim.x) {
      const unsigned long long v = s_ev[j];
      if (!v) continue;
      const int rep = cbase * 128 + j;
      if (rep >= L.m) continue;
      const unsigned long long f = 0xFFFFull;
      const unsigned long long g = (v & f) | (((v >> 16) & f) << kFieldBits) |
                                   (((v >> 32) & f) << (2 * kFieldBits));
      if (g) atomicAdd(&ev_row[T.count_base + rep], g);
      if (rs_row && (v >> 48)) atomicAdd(&rs_row[T.count_base + rep], v >> 48);
    }
    __syncthreads();
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
        philox4x32_10((uint32_t)row, kStepInit, (uint32_t)(word * 8 + q), kStreamInit, c.key0,
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
    philox4x32_10((uint32_t)j, kStepPick, (uint32_t)r, kStreamPick + 4u * (uint32_t)net, c.key0,
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

void packed_init(const PackedLayout &L, uint32_t *sa, uint32_t *sb, uint32_t *mask, float p0,
                 int32_t k_exact, const int32_t *net_first_row, const int32_t *net_rows,
                 int32_t n_nets, const StepConsts &c, cudaStream_t st) {
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
                 const int2 *entries, const uint32_t *mask_in, uint32_t *mask_out, uint32_t *sa,
                 uint32_t *sb, uint32_t *evs, unsigned long long *ev_row,
                 unsigned long long *rs_row, uint32_t step, float scale, const StepConsts &c,
                 cudaStream_t st) {
  k_infect<<<task_grid(L.n_tasks, 4), kThreads, 0, st>>>(
      L, tasks, row_ptr, entries, reinterpret_cast<const uint4 *>(mask_in),
      reinterpret_cast<const uint4 *>(sa), reinterpret_cast<const uint4 *>(sb),
      reinterpret_cast<uint4 *>(evs), step, scale, c);
  k_flow<<<task_grid(L.n_tasks, 4), kThreads, 0, st>>>(
      L, tasks, row_ptr, reinterpret_cast<const uint4 *>(evs), reinterpret_cast<uint4 *>(mask_out),
      reinterpret_cast<uint4 *>(sa), reinterpret_cast<uint4 *>(sb), ev_row, rs_row, step, c);
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
