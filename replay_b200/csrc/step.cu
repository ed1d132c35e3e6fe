// Batched path, geometric mode: one fused kernel per step (k_step).
//
// It replaces, for every replica of the batch at once, the reference's
// per-step sequence generate_infectious_vector -> cusparseSpMM ->
// compute_infection_probability -> monte_carlo_simulation ->
// update_countdown_vector (tool/gpu_cpu_temporal_sim.cu:1053-1084) with the
// geometric transition rules and the per-replica S/E/I/R count reduction
// that feeds --summary-out (:181-202).
//
// Layout in HBM, node-major, 32 replicas per uint32 word; every node row is
// padded to a multiple of 4 words so that a lane moves 128 replicas with one
// 16-byte access (an "item" = one node x one 4-word column):
//   sa, sb      state planes, updated in place; replica bit (a, b):
//               S (0,0), E (0,1), I (1,0), R (1,1)
//   mask_in     infectious bits at the start of the step (read by the gather)
//   mask_out    infectious bits after the step (every item written): the two
//               mask buffers alternate between steps, so that every
//               infection decision reads start-of-step neighbour states
// The window CSR holds {col, weight} pairs (int32 contact-seconds).
//
// One CTA of 16 warps per SM walks tasks (rows x a 32-column slice).  Inside
// a task every warp runs its own pipeline over warp chunks of up to 64 items
// (2 rows of a 4,096-replica slice), fetched from a shared counter: lane 0
// stages chunk k+1's two plane tiles and its CSR pairs into the warp's other
// shared-memory stage with bulk asynchronous copies (cp.async.bulk, mbarrier
// completion, no multicast) while the warp works on chunk k.  Per chunk:
//   1. each lane gathers, for its items, the OR of the neighbours' mask_in
//      words (16 B per entry, a row's lanes read one 512-byte line) and the
//      row's total contact-seconds e_max;
//   2. exposed words (inf & S) go to an infection queue and words with E or
//      I (R when immunity wanes) replicas to a flow queue, decided 32 words
//      at a time so that lanes work on dense lists:
//        infection: the exposed replicas of a word compare the top byte of
//        their infection uniforms (8 bit-sliced planes, two Philox calls per
//        word) with that of the bound B = max beta_r s_i e_max >= every P;
//        the survivors compute their exact int64 exposure -- one batch of 32
//        candidates spreads its (candidate, CSR pair) products over all 32
//        lanes, every pair an independent load -- then P = 1 - exp(-x) and
//        U < floor(P 2^64);
//        flows: bit-sliced uniforms, 32 replicas per random plane;
//   3. the owner lane applies the events to its items (all decisions use
//      the start-of-step planes), writes changed planes and mask_out, and
//      counts every transition per replica in shared memory (flushed once
//      per task to the step's event row).
// Every wait on a staged copy is bounded: a warp that gives up sets the
// simulation's error flag (the host fails the run) and skips the chunk.
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kFieldBits = 21;   // global event fields: S->E | ->I | I->
constexpr int kStepWarps = 16;
constexpr int kStepThreads = kStepWarps * 32;
constexpr int kMaxTaskRows = 1024;
constexpr int kWItems = 64;      // items per warp chunk (2 per lane)
constexpr int kWEnt = 128;       // staged CSR pairs per warp chunk
constexpr int kQueue = 160;      // 31 left over + 4 words x 32 lanes of one pass
constexpr long long kSpinLimit = 1ll << 22;

__device__ __forceinline__ uint32_t word_mask(const PackedLayout &L, int word) {
  return word < L.vwords - 1 ? kFull : (word == L.vwords - 1 ? L.last_mask : 0u);
}
__device__ __forceinline__ uint32_t get4(const uint4 &v, int w) {
  return w == 0 ? v.x : (w == 1 ? v.y : (w == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set4(uint4 &v, int w, uint32_t x) {
  if (w == 0) v.x = x; else if (w == 1) v.y = x; else if (w == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ void or4(uint4 &a, const uint4 b) {
  a.x |= b.x;
  a.y |= b.y;
  a.z |= b.z;
  a.w |= b.w;
}

// Fast division of an item index by the columns of a task (ncols <= 32):
// q = umulhi(i, ceil(2^32 / d)).
struct Div {
  uint32_t d, mag;
  __device__ explicit Div(uint32_t dd) : d(dd), mag(dd > 1 ? 0xFFFFFFFFu / dd + 1u : 0u) {}
  __device__ uint32_t div(uint32_t i) const { return d > 1 ? __umulhi(i, mag) : i; }
};

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int &total) {
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  total = __shfl_sync(kFull, incl, 31);
  return incl - v;
}

// Position of the k-th (from 0) set bit of t (k < popc(t)), by halving.
__device__ __forceinline__ int nth_set_bit(uint32_t t, int k) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const int c = __popc(t & ((1u << w) - 1u));
    if (k >= c) {
      k -= c;
      pos += w;
      t >>= w;
    }
  }
  return pos;
}

// Largest owner with off[owner] <= p over 32 non-decreasing offsets.
__device__ __forceinline__ int find_owner(const int32_t *off, int p) {
  int owner = 0;
#pragma unroll
  for (int st = 16; st > 0; st >>= 1)
    if (off[owner + st] <= p) owner += st;
  return owner;
}

// ---- bulk asynchronous copies (global -> this CTA's shared memory) ----------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Waits for the phase with the given parity to complete; false after
// kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// `bytes` (a multiple of 16) from 16-byte aligned global `src` to 16-byte
// aligned shared `dst`; completion is signalled on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- shared memory ------------------------------------------------------------
struct alignas(16) WarpStage {
  uint4 pa[kWItems];
  uint4 pb[kWItems];
  int2 ent[kWEnt + 2];  // staged pairs; the copy starts up to one pair early
};

struct alignas(16) WarpSmem {
  WarpStage st[2];
  unsigned long long bar[2];
  uint4 pl[32][2];            // infection planes of the round's words
  uint32_t evs[kWItems * 4];  // infection events of the chunk's words
  uint32_t fl[kWItems * 4];   // flow events of the chunk's words
  float ief[kWItems];         // ef(e_max) of each chunk item's row
  long long esum[32];         // exact exposures of a candidate batch
  uint32_t qX[kQueue];        // infection queue: exposed replicas
  uint16_t qsw[kQueue];       //   chunk item * 4 + word in item
  uint16_t fq[kQueue];        // flow queue: chunk item * 4 + word
  uint32_t C[32];             // candidates after the bound test
  int32_t off[32];            // scan offsets of the round's candidates
  int32_t poff[32];           // scan offsets of a batch's CSR pairs
  int32_t ksw[32];            // candidates carried to the next batch: sw << 5 | bit
  uint8_t ku8[32];            //   top byte of the replica's uniform
  int32_t cbeg[32];           // batch candidates: first CSR pair (absolute)
  int32_t cword[32];          //   word index in the row, << 5 | bit
  int32_t n, nk, fn, pad;
};

constexpr size_t kStepSmem = sizeof(WarpSmem) * kStepWarps;
static_assert(kStepSmem + 37 * 1024 <= 227 * 1024, "step kernel shared memory");

// Per-chunk context of a warp.
struct Chunk {
  int r0, r1;         // task-relative rows
  int items;
  int32_t e0;         // first CSR pair of the chunk (absolute)
  int shift;          // staged pair index of e0 (the copy starts 16-byte aligned)
  bool staged;
};

__device__ __forceinline__ Chunk chunk_desc(int k, int rpc, int nrows, int ncols,
                                            const int32_t *s_rp, const int2 *ent) {
  Chunk ch;
  ch.r0 = k * rpc;
  ch.r1 = min(ch.r0 + rpc, nrows);
  ch.items = (ch.r1 - ch.r0) * ncols;
  ch.e0 = s_rp[ch.r0];
  ch.staged = s_rp[ch.r1] - ch.e0 <= kWEnt;
  const uintptr_t src = reinterpret_cast<uintptr_t>(ent + ch.e0);
  ch.shift = (int)((src & 15u) >> 3);
  return ch;
}

// Issued by lane 0: bulk copies of a chunk's plane tiles and (when they fit)
// its CSR pairs into a stage.
__device__ __forceinline__ void chunk_issue(const Chunk &ch, WarpStage &st,
                                            unsigned long long *bar, const PackedLayout &L,
                                            const PackedTask &T, int cbase, int ncols,
                                            const uint4 *sa, const uint4 *sb, const int2 *ent,
                                            const int32_t *s_rp) {
  const int nr = ch.r1 - ch.r0;
  const uint32_t row_bytes = (uint32_t)ncols * 16u;
  uint32_t pair_bytes = 0;
  const int32_t npairs = s_rp[ch.r1] - ch.e0;
  if (ch.staged && npairs > 0) pair_bytes = ((uint32_t)(npairs + ch.shift) * 8u + 15u) & ~15u;
  fence_proxy_async();
  mbar_expect_tx(bar, 2u * row_bytes * (uint32_t)nr + pair_bytes);
  const int64_t row0 = (int64_t)(T.row_begin + ch.r0);
  if (ncols == L.q4) {  // the slice is the whole row: one tile per plane
    bulk_g2s(st.pa, sa + row0 * L.q4, row_bytes * (uint32_t)nr, bar);
    bulk_g2s(st.pb, sb + row0 * L.q4, row_bytes * (uint32_t)nr, bar);
  } else {
    for (int r = 0; r < nr; ++r) {
      bulk_g2s(st.pa + r * ncols, sa + (row0 + r) * L.q4 + cbase, row_bytes, bar);
      bulk_g2s(st.pb + r * ncols, sb + (row0 + r) * L.q4 + cbase, row_bytes, bar);
    }
  }
  if (pair_bytes) bulk_g2s(st.ent, ent + ch.e0 - ch.shift, pair_bytes, bar);
}

__device__ __forceinline__ void count_bits(unsigned long long *s_ev, int wl, uint32_t t,
                                           unsigned long long inc) {
  while (t) {
    const int r = __ffs(t) - 1;
    atomicAdd(&s_ev[wl * 32 + r], inc);
    t &= t - 1;
  }
}

// Applies one word's moves from its start-of-step planes; counts the events
// (4 x 16-bit fields per replica: S->E | ->I | I-> | R->S).
__device__ __forceinline__ void apply_word(uint32_t A, uint32_t B, uint32_t evS, uint32_t f,
                                           bool waning, const StepConsts &c,
                                           unsigned long long *s_ev, int wl, uint32_t &na,
                                           uint32_t &nb) {
  const uint32_t E = ~A & B, I = A & ~B, Rw = waning ? (A & B) : 0u;
  const uint32_t evE = f & E, evI = f & I, evR = f & Rw;
  uint32_t xa = A, xb = B;
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
  na = xa;
  nb = xb;
  if (evS | evE | evI | evR) {
    count_bits(s_ev, wl, c.has_exposed ? evS : 0u, 1ull);
    count_bits(s_ev, wl, evE | (c.has_exposed ? 0u : evS), 1ull << 16);
    count_bits(s_ev, wl, evI, 1ull << 32);
    count_bits(s_ev, wl, evR, 1ull << 48);
  }
}

// Flow round: queued words [base, base + cnt) one per lane, planes from the
// chunk's stage; results to W.fl.
__device__ __forceinline__ void flow_round(WarpSmem &W, const WarpStage &st, int base, int cnt,
                                           int lane, bool waning, const StepConsts &c,
                                           uint32_t step, int row0, int r0, int cbase,
                                           const Div &dv, int ncols) {
  if (lane < cnt) {
    const int sw = W.fq[base + lane];
    const int item = sw >> 2, w = sw & 3;
    const uint32_t A = get4(st.pa[item], w), B = get4(st.pb[item], w);
    const int rl = (int)dv.div((uint32_t)item);
    const int col = cbase + item - rl * ncols;
    const uint32_t E = ~A & B, I = A & ~B, R = waning ? (A & B) : 0u;
    W.fl[sw] = flow_events(E, I, R, c.th, c.rk, (uint32_t)(row0 + r0 + rl), step,
                           (uint32_t)(4 * col + w) + (c.roff >> 5));
  }
}

// Infection round over queue entries [0, n): the bound test one word per
// lane, then the exact test of the surviving candidates in full batches of
// 32 together with those carried from earlier rounds (fewer than 32 are
// carried unless `drain`).  Events are OR-ed into W.evs.
__device__ __forceinline__ void infect_round(WarpSmem &W, const WarpStage &st, const Chunk &ch,
                                             int n, bool drain, int lane, const PackedLayout &L,
                                             int row0, int cbase, const Div &dv, int ncols,
                                             const int32_t *s_rp, const int2 *ent,
                                             const float *s_bw, const uint32_t *mask_w,
                                             uint32_t step, float scale, const StepConsts &c) {
  // ---- bound test, one word per lane ----
  uint32_t Cw = 0;
  if (lane < n) {
    const int sw = W.qsw[lane];
    const int item = sw >> 2, w = sw & 3;
    const int rl = (int)dv.div((uint32_t)item);
    const int word = 4 * (cbase + item - rl * ncols) + w;
    const int orow = row0 + ch.r0 + rl;
    // every exposed replica has P <= x <= |bs_r| ef(e_max) =: B; replicas
    // whose uniform's top byte is above B's cannot infect
    float bsmax = c.beta_r ? s_bw[word - 4 * cbase] : fabsf(c.beta);
    if (c.sus) bsmax = __fmul_rn(bsmax, fabsf(__ldg(c.sus + orow)));
    const float B = __fmul_rn(bsmax, W.ief[item]);
    if (B > 0.0f) {
      uint32_t pl[8];
      infect_planes(c.rk, (uint32_t)orow, step, (uint32_t)word + (c.roff >> 5), pl);
      Cw = B >= 1.0f ? W.qX[lane] : top8_le(W.qX[lane], fixed64(B), pl);
      W.pl[lane][0] = make_uint4(pl[0], pl[1], pl[2], pl[3]);
      W.pl[lane][1] = make_uint4(pl[4], pl[5], pl[6], pl[7]);
    }
  }
  int ctotal;
  const int coff = warp_excl_scan(__popc(Cw), lane, ctotal);
  W.C[lane] = Cw;
  W.off[lane] = coff;
  __syncwarp();
  const int nk = W.nk;
  const int total = nk + ctotal;
  // candidate p of this round: carried (p < nk) or the (p - nk)-th new one
  auto candidate = [&](int p, int &sw, int &b, uint32_t &u8) {
    if (p < nk) {
      sw = W.ksw[p] >> 5;
      b = W.ksw[p] & 31;
      u8 = W.ku8[p];
    } else {
      const int o = find_owner(W.off, p - nk);
      b = nth_set_bit(W.C[o], p - nk - W.off[o]);
      sw = W.qsw[o];
      const uint4 a = W.pl[o][0], d = W.pl[o][1];
      const uint32_t pl[8] = {a.x, a.y, a.z, a.w, d.x, d.y, d.z, d.w};
      u8 = top8_of(pl, (uint32_t)b);
    }
  };
  // ---- exact test, in batches of 32 candidates ----
  int base = 0;
  for (; total - base >= 32 || (drain && base < total); base += 32) {
    const int p = base + lane;
    int sw = 0, b = 0, npairs = 0;
    uint32_t u8 = 0;
    int32_t beg = 0;
    if (p < total) {
      candidate(p, sw, b, u8);
      const int rlc = (int)dv.div((uint32_t)(sw >> 2));
      beg = s_rp[ch.r0 + rlc];
      npairs = s_rp[ch.r0 + rlc + 1] - beg;
    }
    const int item = sw >> 2, w = sw & 3;
    const int rl = (int)dv.div((uint32_t)item);
    const int word = 4 * (cbase + item - rl * ncols) + w;
    // the batch's (candidate, CSR pair) products spread over the lanes:
    // every pair is one independent mask-word load
    int ptotal;
    const int poff = warp_excl_scan(npairs, lane, ptotal);
    W.poff[lane] = poff;
    W.cbeg[lane] = beg;
    W.cword[lane] = word << 5 | b;
    W.esum[lane] = 0;
    __syncwarp();
    for (int q0 = 0; q0 < ptotal; q0 += 64) {
      int32_t pc[2], pw[2], cw[2], own[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = q0 + 32 * h + lane;
        own[h] = -1;
        pc[h] = pw[h] = cw[h] = 0;
        if (q < ptotal) {
          const int o = find_owner(W.poff, q);
          const int32_t k = W.cbeg[o] + (q - W.poff[o]);
          const int2 e = ch.staged ? st.ent[k - ch.e0 + ch.shift] : __ldg(ent + k);
          pc[h] = e.x;
          pw[h] = e.y;
          cw[h] = W.cword[o];
          own[h] = o;
        }
      }
      uint32_t mw[2];
#pragma unroll
      for (int h = 0; h < 2; ++h)
        mw[h] = own[h] >= 0 ? mask_w[(int64_t)pc[h] * L.words + (cw[h] >> 5)] : 0u;
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (own[h] >= 0 && ((mw[h] >> (cw[h] & 31)) & 1u))
          atomicAdd(reinterpret_cast<unsigned long long *>(&W.esum[own[h]]),
                    (unsigned long long)(long long)pw[h]);
    }
    __syncwarp();
    if (p < total) {
      const long long e = W.esum[lane];
      const int orow = row0 + ch.r0 + rl;
      const float br = c.beta_r ? __ldg(c.beta_r + word * 32 + b) : c.beta;
      const float bs = c.sus ? __fmul_rn(br, __ldg(c.sus + orow)) : br;
      float ef = __ll2float_rn(e);
      if (scale != 1.0f) ef = __fmul_rn(ef, scale);
      const float xx = __fmul_rn(bs, ef);
      // P <= x: a uniform whose top byte is above x's cannot infect (no
      // exponential)
      if (xx > 0.0f && !(xx < 1.0f && u8 > (uint32_t)(fixed64(xx) >> 56))) {
        const uint32_t gword = (uint32_t)word + (c.roff >> 5);
        if (infect_event(one_minus_exp_neg(xx), u8, c.rk, (uint32_t)orow, step,
                         gword * 32u + (uint32_t)b))
          atomicOr(&W.evs[sw], 1u << b);
      }
    }
    __syncwarp();
  }
  // carry the rest (fewer than 32) to the next round
  const int rest = total - base;
  int kv = 0;
  uint32_t ku = 0;
  if (rest > 0 && base + lane < total) {
    int sw, b;
    candidate(base + lane, sw, b, ku);
    kv = sw << 5 | b;
  }
  __syncwarp();
  if (rest > 0 && lane < rest) {
    W.ksw[lane] = kv;
    W.ku8[lane] = (uint8_t)ku;
  }
  if (lane == 0) W.nk = rest > 0 ? rest : 0;
  __syncwarp();
}

// The step kernel (see the file comment).  One CTA per SM; tasks are
// assigned round-robin, warp chunks inside a task dynamically.
__global__ void __launch_bounds__(kStepThreads, 1)
    k_step(PackedLayout L, const PackedTask *__restrict__ tasks,
           const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
           const uint4 *__restrict__ mask_in, uint4 *__restrict__ mask_out,
           uint4 *__restrict__ sa, uint4 *__restrict__ sb,
           unsigned long long *__restrict__ ev_row, unsigned long long *__restrict__ rs_row,
           uint32_t step, float scale, StepConsts c) {
  __shared__ int32_t s_rp[kMaxTaskRows + 1];
  __shared__ float s_bw[128];  // max |beta_r| of each word of the slice
  __shared__ unsigned long long s_ev[128 * 32];
  __shared__ int32_t s_next;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  WarpSmem &W = reinterpret_cast<WarpSmem *>(s_dyn)[warp];
  const uint32_t *mask_w = reinterpret_cast<const uint32_t *>(mask_in);
  const bool waning = c.th.tr_all || c.th.tr != 0;
  const bool fe = c.th.te_all || c.th.te != 0, fi = c.th.ti_all || c.th.ti != 0;
  if (lane == 0) {
    mbar_init(&W.bar[0], 1);
    mbar_init(&W.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  uint32_t phase = 0;
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int cbase = T.slice * 32;
    const int ncols = min(32, L.q4 - cbase);
    const Div dv((uint32_t)ncols);
    const int nrows = T.row_end - T.row_begin;
    const int row0 = T.row_begin;
    __syncthreads();  // the previous task's flush is done with s_ev
    for (int i = threadIdx.x; i <= nrows; i += blockDim.x) s_rp[i] = row_ptr[row0 + i];
    for (int j = threadIdx.x; j < ncols * 128; j += blockDim.x) s_ev[j] = 0;
    if (c.beta_r)
      for (int wl = threadIdx.x; wl < ncols * 4; wl += blockDim.x) {
        float mx = 0.0f;
        for (int r = 0; r < 32; ++r) {
          const int rep = cbase * 128 + wl * 32 + r;
          if (rep < L.m) mx = fmaxf(mx, fabsf(__ldg(c.beta_r + rep)));
        }
        s_bw[wl] = mx;
      }
    if (threadIdx.x == 0) s_next = 0;
    __syncthreads();
    const int rpc = max(1, kWItems / ncols);
    const int nchunks = (nrows + rpc - 1) / rpc;
    auto grab = [&]() {
      int k = 0;
      if (lane == 0) k = atomicAdd(&s_next, 1);
      return __shfl_sync(kFull, k, 0);
    };
    int cur = grab();
    int s = 0;
    if (cur < nchunks && lane == 0) {
      const Chunk ch = chunk_desc(cur, rpc, nrows, ncols, s_rp, ent);
      chunk_issue(ch, W.st[0], &W.bar[0], L, T, cbase, ncols, sa, sb, ent, s_rp);
    }
    while (cur < nchunks) {
      const int nxt = grab();
      if (nxt < nchunks && lane == 0) {
        const Chunk chn = chunk_desc(nxt, rpc, nrows, ncols, s_rp, ent);
        chunk_issue(chn, W.st[s ^ 1], &W.bar[s ^ 1], L, T, cbase, ncols, sa, sb, ent, s_rp);
      }
      const bool ready = mbar_wait(&W.bar[s], (phase >> s) & 1u);
      phase ^= 1u << s;
      if (!ready) {
        if (lane == 0 && c.err) atomicExch(c.err, 1);
        cur = nxt;
        s ^= 1;
        continue;
      }
      const Chunk ch = chunk_desc(cur, rpc, nrows, ncols, s_rp, ent);
      const WarpStage &st = W.st[s];
      for (int j = lane; j < kWItems * 4; j += 32) {
        W.evs[j] = 0;
        W.fl[j] = 0;
      }
      if (lane == 0) {
        W.n = 0;
        W.nk = 0;
        W.fn = 0;
      }
      __syncwarp();
      // the lane's two items: planes kept in registers for the apply step
      // (one pass per item, not unrolled: one call site of each round)
      uint4 A0 = make_uint4(0, 0, 0, 0), B0 = A0, A1 = A0, B1 = A0;
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        const bool valid = i < ch.items;
        const int rl = valid ? (int)dv.div((uint32_t)i) : 0;
        const int col = cbase + (valid ? i - rl * ncols : 0);
        const int rloc = ch.r0 + rl;
        const uint4 a4 = valid ? st.pa[i] : make_uint4(0, 0, 0, 0);
        const uint4 b4 = valid ? st.pb[i] : make_uint4(0, 0, 0, 0);
        if (h == 0) {
          A0 = a4;
          B0 = b4;
        } else {
          A1 = a4;
          B1 = b4;
        }
        uint32_t S[4], F[4];
        bool anyS = false;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const uint32_t vm = valid ? word_mask(L, 4 * col + w) : 0u;
          const uint32_t a = get4(a4, w), b = get4(b4, w);
          S[w] = ~a & ~b & vm;
          F[w] = ((fe ? ~a & b : 0u) | (fi ? a & ~b : 0u) | (waning ? a & b : 0u)) & vm;
          anyS |= S[w] != 0u;
        }
        // ---- gather: OR of the neighbours' start-of-step masks ----
        uint32_t X[4] = {0, 0, 0, 0};
        float efmax = 0.0f;
        const int32_t beg = valid ? s_rp[rloc] : 0;
        const int npr = valid ? s_rp[rloc + 1] - beg : 0;
        if (npr > 0 && anyS) {
          const int2 *er = ch.staged ? st.ent + (beg - ch.e0 + ch.shift) : ent + beg;
          uint4 inf = make_uint4(0, 0, 0, 0);
          long long emax = 0;
          int k = 0;
          for (; k + 4 <= npr; k += 4) {
            const int2 q0 = er[k], q1 = er[k + 1], q2 = er[k + 2], q3 = er[k + 3];
            const uint4 m0 = mask_in[(int64_t)q0.x * L.q4 + col];
            const uint4 m1 = mask_in[(int64_t)q1.x * L.q4 + col];
            const uint4 m2 = mask_in[(int64_t)q2.x * L.q4 + col];
            const uint4 m3 = mask_in[(int64_t)q3.x * L.q4 + col];
            or4(inf, m0);
            or4(inf, m1);
            or4(inf, m2);
            or4(inf, m3);
            emax += (long long)q0.y + q1.y + q2.y + q3.y;
          }
          for (; k < npr; ++k) {
            const int2 q0 = er[k];
            or4(inf, mask_in[(int64_t)q0.x * L.q4 + col]);
            emax += q0.y;
          }
#pragma unroll
          for (int w = 0; w < 4; ++w) X[w] = get4(inf, w) & S[w];
          efmax = __ll2float_rn(emax);
          if (scale != 1.0f) efmax = __fmul_rn(efmax, scale);
        }
        if (valid) W.ief[i] = efmax;
        // ---- queue exposed and flow words ----
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const unsigned qm = __ballot_sync(kFull, X[w] != 0u);
          if (qm) {
            const int pos = W.n + __popc(qm & ((1u << lane) - 1u));
            if (X[w]) {
              W.qsw[pos] = (uint16_t)(i * 4 + w);
              W.qX[pos] = X[w];
            }
            __syncwarp();
            if (lane == 0) W.n += __popc(qm);
          }
          const unsigned fm = __ballot_sync(kFull, F[w] != 0u);
          if (fm) {
            const int pos = W.fn + __popc(fm & ((1u << lane) - 1u));
            if (F[w]) W.fq[pos] = (uint16_t)(i * 4 + w);
            __syncwarp();
            if (lane == 0) W.fn += __popc(fm);
          }
          __syncwarp();
        }
        // ---- full rounds (the last pass drains the queues) ----
        const bool last = h == 1;
        while (W.n >= 32 || (last && (W.n > 0 || W.nk > 0))) {
          const int n = W.n;
          const int take = n < 32 ? n : 32;
          infect_round(W, st, ch, take, last && take == n, lane, L, row0, cbase, dv, ncols, s_rp,
                       ent, s_bw, mask_w, step, scale, c);
          const int rest = n - take;
          uint16_t qs = 0;
          uint32_t qx = 0;
          for (int j0 = 0; j0 < rest; j0 += 32) {
            const int j = j0 + lane;
            if (j < rest) {
              qs = W.qsw[take + j];
              qx = W.qX[take + j];
            }
            __syncwarp();
            if (j < rest) {
              W.qsw[j] = qs;
              W.qX[j] = qx;
            }
            __syncwarp();
          }
          if (lane == 0) W.n = rest;
          __syncwarp();
        }
        const int fnq = W.fn;
        int f0 = 0;
        for (; fnq - f0 >= 32 || (last && f0 < fnq); f0 += 32)
          flow_round(W, st, f0, min(32, fnq - f0), lane, waning, c, step, row0, ch.r0, cbase, dv,
                     ncols);
        __syncwarp();
        const int frest = fnq - f0;
        if (f0 > 0 && frest > 0) {  // move the remainder (< 32 words) to the front
          const uint16_t v = lane < frest ? W.fq[f0 + lane] : 0;
          __syncwarp();
          if (lane < frest) W.fq[lane] = v;
        }
        if (lane == 0) W.fn = frest > 0 ? frest : 0;
        __syncwarp();
      }
      // ---- apply every item's events, write its planes and next mask ----
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        if (i >= ch.items) continue;
        const int rl = (int)dv.div((uint32_t)i);
        const int cc = i - rl * ncols;
        const int64_t idx = (int64_t)(row0 + ch.r0 + rl) * L.q4 + cbase + cc;
        const uint4 a4 = h ? A1 : A0, b4 = h ? B1 : B0;
        uint4 na4 = a4, nb4 = b4;
        bool changed = false;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const uint32_t evS = W.evs[i * 4 + w], f = W.fl[i * 4 + w];
          if (!(evS | f)) continue;
          uint32_t na, nb;
          apply_word(get4(a4, w), get4(b4, w), evS, f, waning, c, s_ev, 4 * cc + w, na, nb);
          set4(na4, w, na);
          set4(nb4, w, nb);
          changed = true;
        }
        if (changed) {
          sa[idx] = na4;
          sb[idx] = nb4;
        }
        mask_out[idx] = make_uint4(na4.x & ~nb4.x, na4.y & ~nb4.y, na4.z & ~nb4.z,
                                   na4.w & ~nb4.w);
      }
      __syncwarp();
      cur = nxt;
      s ^= 1;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < ncols * 128; j += blockDim.x) {
      const unsigned long long v = s_ev[j];
      if (!v) continue;
      const int rep = cbase * 128 + j;
      if (rep >= L.m) continue;
      const unsigned long long f16 = 0xFFFFull;
      const unsigned long long g = (v & f16) | (((v >> 16) & f16) << kFieldBits) |
                                   (((v >> 32) & f16) << (2 * kFieldBits));
      if (g) atomicAdd(&ev_row[T.count_base + rep], g);
      if (rs_row && (v >> 48)) atomicAdd(&rs_row[T.count_base + rep], v >> 48);
    }
  }
}

}  // namespace

rp_status step_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kStepSmem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_step)");
  return RP_OK;
}

void packed_step_fused(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
                       const int2 *entries, const uint32_t *mask_in, uint32_t *mask_out,
                       uint32_t *sa, uint32_t *sb, unsigned long long *ev_row,
                       unsigned long long *rs_row, uint32_t step, float scale,
                       const StepConsts &c, cudaStream_t st) {
  const int grid = L.n_tasks < 148 ? (L.n_tasks > 0 ? L.n_tasks : 1) : 148;
  k_step<<<grid, kStepThreads, kStepSmem, st>>>(
      L, tasks, row_ptr, entries, reinterpret_cast<const uint4 *>(mask_in),
      reinterpret_cast<uint4 *>(mask_out), reinterpret_cast<uint4 *>(sa),
      reinterpret_cast<uint4 *>(sb), ev_row, rs_row, step, scale, c);
}

}  // namespace rp
