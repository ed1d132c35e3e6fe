// Batched path: replica-bit-packed state, two kernels per step.
//
// Layout in HBM, node-major, 32 replicas per uint32 word; every node row is
// padded to a multiple of 4 words so that a lane moves 128 replicas with one
// 16-byte access:
//   sa, sb    state planes; replica bit (a, b): S (0,0), E (0,1), I (1,0),
//             R (1,1)
//   mask      infectious bits (a & ~b); k_infect reads it, then k_flow
//             rewrites the words whose state changed
//   evs       infection events of the step (items with events only; a
//             per-item flag byte tells k_flow which ones)
// The window CSR holds {col, weight} pairs (int32 contact-seconds).
//
// k_infect (exposure SpMM + infection draws), per row with contacts, lanes
// over 4-word columns (the replacement of cusparseSpMM,
// tool/gpu_cpu_temporal_sim.cu:1062, and monte_carlo_simulation, :137-159):
//   1. inf = OR over neighbours j of mask_t[j] (16 B per lane per entry);
//   2. exposed = inf & S; the exposed replicas of a word compare the top
//      byte of their infection uniforms (8 bit-sliced planes, two Philox
//      calls per word) with that of the word bound B = max bs_r * e_max
//      (e_max = the row's total contact-seconds, so every P <= B); only
//      replicas at or below it compute their exact int64 exposure and
//      P = 1 - exp(-beta_r s_i e) and finish the comparison against
//      floor(P 2^64) (infect_event; the uniform's low 56 bits are drawn
//      only on a tie of the top byte);
//   3. events are OR-ed into evs and flag their item.
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

__device__ __forceinline__ void set4(uint4 &v, int w, uint32_t x) {
  if (w == 0) v.x = x; else if (w == 1) v.y = x; else if (w == 2) v.z = x; else v.w = x;
}

__device__ __forceinline__ void or4(uint4 &a, const uint4 b) {
  a.x |= b.x;
  a.y |= b.y;
  a.z |= b.z;
  a.w |= b.w;
}

// Fast division of an item index by the columns of a task (ncols <= 32,
// items < 2^27): q = umulhi(i, ceil(2^32 / d)).
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

__device__ __forceinline__ int find_owner(const int32_t *off, int p) {
  int owner = 0;
#pragma unroll
  for (int st = 16; st > 0; st >>= 1)
    if (off[owner + st] <= p) owner += st;
  return owner;
}

constexpr int kMaxTaskRows = 4096;  // rows of one task (host-side limit)

// Per-item hint byte (item = node x 4-word column): bit 0 an infection event
// of this step (k_infect), bit 1 replicas that may move (E, I, waning R),
// bit 2 replicas that may be susceptible.  k_flow rewrites bits 1-2 of every
// item from its start-of-step planes and events, as a superset of the next
// step's state; k_infect skips the neighbours of items without bit 2 where
// rows are long enough for the extra load to pay.  The hints are kept only
// for graphs whose windows average at least 8 pairs per row (StepConsts
// hints); elsewhere the extra work would not pay.
constexpr uint8_t kFlagEvent = 1, kFlagActive = 2, kFlagSusceptible = 4;

constexpr int kEntCap = kStageDefault;  // staging buffer capacity, CSR pairs
constexpr int kEntBuf = kEntCap + 4; // a staging buffer (the copy may start one pair early)
constexpr int kPiece = kEntBuf / 2 - 2;  // pairs per piece of a long row (a half buffer)
constexpr long long kSpinLimit = 1ll << 22;

// ---- bulk asynchronous copies (global -> this CTA's shared memory) ----------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
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
// Stages pairs [k0, k1) of `ent` (k1 - k0 <= kEntBuf - 2) into `dst` with one
// bulk copy (cp.async.bulk, no multicast) completing on `bar`; the copy
// starts on the 16-byte boundary at or below pair k0, so pair k lands at
// dst[k - k0 + shift].  Returns shift.  Issued by one thread.
__device__ __forceinline__ int stage_pairs(int2 *dst, const int2 *ent, int32_t k0, int32_t k1,
                                           unsigned long long *bar) {
  const uintptr_t src = reinterpret_cast<uintptr_t>(ent + k0);
  const int shift = (int)((src & 15u) >> 3);
  const uint32_t bytes = ((uint32_t)(k1 - k0 + shift) * 8u + 15u) & ~15u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(ent + k0 - shift), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
  return shift;
}
__device__ __forceinline__ int pair_shift(const int2 *ent, int32_t k0) {
  return (int)((reinterpret_cast<uintptr_t>(ent + k0) & 15u) >> 3);
}

// ---------------------------------------------------------------------------
// Per-warp queue of exposed words of k_infect (dynamic shared memory):
// entries accumulate over rows and are decided 32 at a time.
constexpr int kInfectQueue = 160;  // 31 left over + 4 words x 32 lanes of one pass
constexpr int kWordExact = 4;      // candidates of a word (long row) for the one-pass exact test
struct InfectQueue {
  uint4 pl[32][2];               // the 8 random planes of each word (round scratch)
  int32_t rloc[kInfectQueue];    // task-relative row
  int32_t word[kInfectQueue];    // word index within the row
  uint32_t X[kInfectQueue];      // exposed replicas of the word
  float efmax[kInfectQueue];     // ef(e_max) of the row
  uint32_t C[32];      // candidates after the bound test (round scratch)
  int32_t off[32];     // warp scan offsets of the candidates
  // candidates carried to the next round (fewer than 32), self-contained
  int32_t krloc[32];
  int32_t kwb[32];  // word << 5 | replica bit
  uint8_t ku8[32];  // top 8 bits of the replica's uniform
  // exact-test batch: per candidate lane, its row's first CSR pair, its
  // word << 5 | bit, the scan offsets of the batch's (candidate, pair)
  // products and the exposure sums
  int32_t cbeg[32];
  int32_t cword[32];
  int32_t poff[32];
  long long esum[32];
  int32_t n;
  int32_t nk;
};

// k_infect's dynamic shared memory, sized per launch: two staging buffers
// and the warps' queues at fixed offsets, then the task's row pointers (max
// task rows + 1), then a long row's per-replica exposures (int32,
// min(32, q4) columns x 128 replicas).  Sized for the launch, so that tall
// tasks or wide rows cost only where they occur (three CTAs per SM need at
// most about 74 KB each).
constexpr int kInfectQueueOff = 2 * kEntBuf * 8;
constexpr int kInfectRpOff = kInfectQueueOff + kWarps * (int)sizeof(InfectQueue);
__host__ __device__ constexpr int infect_acc_off(int max_rows) {
  return (kInfectRpOff + 4 * (max_rows + 1) + 15) / 16 * 16;
}
__host__ __device__ constexpr int infect_smem(int q4, int max_rows) {
  return infect_acc_off(max_rows) + (q4 < 32 ? q4 : 32) * 128 * 4;
}
constexpr int kInfectDynSmemMax = infect_smem(32, kMaxTaskRows);

// Top 8 uniform bits of replica bit b from a queued word's planes.
__device__ __forceinline__ uint32_t queued_top8(const uint4 (&q)[2], uint32_t b) {
  const uint4 a = q[0], c = q[1];
  const uint32_t pl[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
  return top8_of(pl, b);
}

// What an infection decision reads besides the candidate (values, so that
// the out-of-line word_exact_pass takes them in registers).
struct DecideArgs {
  const uint32_t *rk;     // Philox round keys
  const float *beta_r;    // per-replica beta, or null
  const float *sus;       // per-node susceptibility, or null
  float beta, scale;
  uint32_t roff, step;
  int32_t words, q4, row_begin;
};

// Decides candidate replica b of task-relative row orl, word `word`, from
// its exact exposure e (contact-seconds) and its uniform's top byte u8.
__device__ __forceinline__ void decide(const DecideArgs &d, int orl, int word, int b,
                                       long long e, uint32_t u8, uint32_t *evs_w,
                                       uint32_t *flag32) {
  const int orow = d.row_begin + orl;
  const float br = d.beta_r ? __ldg(d.beta_r + word * 32 + b) : d.beta;
  const float bs = d.sus ? __fmul_rn(br, d.sus[orow]) : br;
  float ef = __ll2float_rn(e);
  if (d.scale != 1.0f) ef = __fmul_rn(ef, d.scale);
  const float xx = __fmul_rn(bs, ef);
  if (!(xx > 0.0f)) return;
  // P <= x: a uniform whose top byte is above x's cannot infect (no
  // exponential)
  if (xx < 1.0f && u8 > (uint32_t)(fixed64(xx) >> 56)) return;
  const uint32_t gword = (uint32_t)word + (d.roff >> 5);
  if (infect_event(one_minus_exp_neg(xx), u8, d.rk, (uint32_t)orow, d.step,
                   gword * 32u + (uint32_t)b)) {
    atomicOr(&evs_w[(int64_t)orow * d.words + word], 1u << b);
    const int64_t idx = (int64_t)orow * d.q4 + (word >> 2);
    atomicOr(&flag32[idx >> 2], 1u << (8 * (idx & 3)));
  }
}

// The exact test of the queued words in `wlist` (lane o's word holds
// candidates Cw of lane o): one pass over each word's row with lane =
// replica, so that each pair's mask word is one broadcast load shared by all
// the word's candidates.  For words with many candidates on rows of more
// than 32 pairs (a dense neighbourhood, whose bound test lets most exposed
// replicas through); on other words the per-replica test costs less.  Kept
// out of line: the busy steps of sparse graphs rarely take it.
__device__ __noinline__ void word_exact_pass(const InfectQueue &Q, unsigned wlist, uint32_t Cw,
                                             int lane, const int32_t *s_rp, const int2 *s_ent,
                                             const int2 *__restrict__ ent, bool staged, int32_t e0,
                                             const uint32_t *mask_w, uint32_t *evs_w,
                                             uint32_t *flag32, DecideArgs d) {
  for (unsigned t = wlist; t; t &= t - 1) {
    const int o = __ffs(t) - 1;
    const uint32_t Co = __shfl_sync(kFull, Cw, o);
    const int orl = Q.rloc[o], word = Q.word[o];
    const int32_t kend = s_rp[orl + 1];
    int32_t k = s_rp[orl];
    long long e = 0;
    for (; k + 4 <= kend; k += 4) {
      int2 q[4];
      uint32_t m[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) q[j] = staged ? s_ent[k + j - e0] : __ldg(ent + k + j);
#pragma unroll
      for (int j = 0; j < 4; ++j) m[j] = mask_w[(int64_t)q[j].x * d.words + word];
#pragma unroll
      for (int j = 0; j < 4; ++j) e += ((m[j] >> lane) & 1u) ? q[j].y : 0;
    }
    for (; k < kend; ++k) {
      const int2 q0 = staged ? s_ent[k - e0] : __ldg(ent + k);
      e += ((mask_w[(int64_t)q0.x * d.words + word] >> lane) & 1u) ? q0.y : 0;
    }
    if ((Co >> lane) & 1u)
      decide(d, orl, word, lane, e, queued_top8(Q.pl[o], (uint32_t)lane), evs_w, flag32);
  }
}

// Decides up to 32 queued exposed words: the bound test one word per lane
// (phase 2), then the exact test of the surviving candidates: a word with
// at least kWordExact of them in one pass over its row (phase 3a), the
// others one replica per lane (phase 3), in full batches of 32 together with
// the candidates carried from earlier rounds; fewer than 32 left over are
// carried to the next round unless `drain` is set.  Events are OR-ed into
// their words and flag their items.
__device__ __forceinline__ void infect_round(InfectQueue &Q, int n, bool drain, int lane,
                                             const PackedLayout &L, const PackedTask &T,
                                             int cbase, const int32_t *s_rp, const int2 *s_ent,
                                             const int2 *__restrict__ ent, bool staged,
                                             int32_t e0, const float *s_bw,
                                             const uint32_t *mask_w, uint32_t *evs_w,
                                             uint32_t *flag32, uint32_t step, float scale,
                                             const StepConsts &c) {
  // ---- phase 2: bound test, one word per lane ----
  uint32_t Cw = 0;
  if (lane < n) {
    const int orow = T.row_begin + Q.rloc[lane];
    const int word = Q.word[lane];
    // every exposed replica has P <= x <= |bs_r| ef(e_max) =: B; replicas
    // whose uniform's top byte is above B's cannot infect
    float bsmax = c.beta_r ? s_bw[word - 4 * cbase] : fabsf(c.beta);
    if (c.sus) bsmax = __fmul_rn(bsmax, fabsf(c.sus[orow]));
    const float B = __fmul_rn(bsmax, Q.efmax[lane]);
    if (B > 0.0f) {
      uint32_t pl[8];
      infect_planes(c.rk, (uint32_t)orow, step, (uint32_t)word + (c.roff >> 5), pl);
      Cw = B >= 1.0f ? Q.X[lane] : top8_le(Q.X[lane], fixed64(B), pl);
      Q.pl[lane][0] = make_uint4(pl[0], pl[1], pl[2], pl[3]);
      Q.pl[lane][1] = make_uint4(pl[4], pl[5], pl[6], pl[7]);
    }
  }
  // ---- phase 3a: a word with many candidates on a row of more than 32
  // pairs takes one pass over its row (word_exact_pass) ----
  const unsigned wlist = __ballot_sync(
      kFull, __popc(Cw) >= kWordExact && s_rp[Q.rloc[lane] + 1] - s_rp[Q.rloc[lane]] > 32);
  const DecideArgs d{c.rk, c.beta_r, c.sus, c.beta, scale, c.roff, step, L.words, L.q4,
                     T.row_begin};
  if (wlist) word_exact_pass(Q, wlist, Cw, lane, s_rp, s_ent, ent, staged, e0, mask_w, evs_w, flag32, d);
  if ((wlist >> lane) & 1u) Cw = 0;
  Q.C[lane] = Cw;
  int ctotal;
  Q.off[lane] = warp_excl_scan(__popc(Cw), lane, ctotal);
  __syncwarp();
  // ---- phase 3: exact test of 32 candidates at a time ----
  // When every candidate's row is short, each lane sums its own row.
  // Otherwise the batch's (candidate, CSR pair) products are spread over the
  // lanes: every pair is one independent mask-word load (a long row is
  // shared by all 32 lanes), and the exposures sum in shared memory (exact
  // int64).
  const int nk = Q.nk;
  const int total = nk + ctotal;
  int base = 0;
  for (; total - base >= 32 || (drain && base < total); base += 32) {
    const int p = base + lane;
    int orl = 0, word = 0, b = 0, npairs = 0;
    int32_t beg = 0;
    uint32_t u8 = 0;
    if (p < total) {
      if (p < nk) {
        const int wb = Q.kwb[p];
        orl = Q.krloc[p];
        word = wb >> 5;
        b = wb & 31;
        u8 = Q.ku8[p];
      } else {
        const int o = find_owner(Q.off, p - nk);
        b = nth_set_bit(Q.C[o], p - nk - Q.off[o]);
        orl = Q.rloc[o];
        word = Q.word[o];
        u8 = queued_top8(Q.pl[o], (uint32_t)b);
      }
      beg = s_rp[orl];
      npairs = s_rp[orl + 1] - beg;
    }
    long long e = 0;
    if (__reduce_max_sync(kFull, (unsigned)npairs) <= 32u) {
      // short rows: each lane sums its own row (loads two pairs ahead)
      int32_t k = beg;
      const int32_t kend = beg + npairs;
      for (; k + 1 < kend; k += 2) {
        const int2 q0 = staged ? s_ent[k - e0] : __ldg(ent + k);
        const int2 q1 = staged ? s_ent[k + 1 - e0] : __ldg(ent + k + 1);
        const uint32_t m0 = mask_w[(int64_t)q0.x * L.words + word];
        const uint32_t m1 = mask_w[(int64_t)q1.x * L.words + word];
        e += ((m0 >> b) & 1u) ? q0.y : 0;
        e += ((m1 >> b) & 1u) ? q1.y : 0;
      }
      if (k < kend) {
        const int2 q0 = staged ? s_ent[k - e0] : __ldg(ent + k);
        e += ((mask_w[(int64_t)q0.x * L.words + word] >> b) & 1u) ? q0.y : 0;
      }
    } else {
    int ptotal;
    const int poff = warp_excl_scan(npairs, lane, ptotal);
    __syncwarp();
    Q.poff[lane] = poff;
    Q.cbeg[lane] = beg;
    Q.cword[lane] = word << 5 | b;
    Q.esum[lane] = 0;
    __syncwarp();
    for (int q0 = 0; q0 < ptotal; q0 += 64) {
      int32_t pc[2], pw[2], cw[2], own[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = q0 + 32 * h + lane;
        own[h] = -1;
        pc[h] = pw[h] = cw[h] = 0;
        if (q < ptotal) {
          const int o = find_owner(Q.poff, q);
          const int32_t k = Q.cbeg[o] + (q - Q.poff[o]);
          const int2 e = staged ? s_ent[k - e0] : __ldg(ent + k);
          pc[h] = e.x;
          pw[h] = e.y;
          cw[h] = Q.cword[o];
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
          atomicAdd(reinterpret_cast<unsigned long long *>(&Q.esum[own[h]]),
                    (unsigned long long)(long long)pw[h]);
    }
    __syncwarp();
    e = Q.esum[lane];
    }
    if (p < total) decide(d, orl, word, b, e, u8, evs_w, flag32);
  }
  __syncwarp();
  // carry the rest: slots below nk keep their entries when no batch ran
  const int rest = total - base;
  if (rest > 0) {
    const int p = base + lane;
    if (p < total && p >= nk) {
      const int o = find_owner(Q.off, p - nk);
      const int b = nth_set_bit(Q.C[o], p - nk - Q.off[o]);
      Q.kwb[lane] = Q.word[o] << 5 | b;
      Q.krloc[lane] = Q.rloc[o];
      Q.ku8[lane] = (uint8_t)queued_top8(Q.pl[o], (uint32_t)b);
    }
  }
  __syncwarp();
  if (lane == 0) Q.nk = rest > 0 ? rest : 0;
  __syncwarp();
}

// One item (row, 4-word column) per lane gathers the OR of the neighbours'
// mask words (its loads issued together) and queues its exposed words;
// infect_round decides the queue 32 words at a time, so that every lane
// works on a dense list of words and then of candidate replicas.
__global__ void __launch_bounds__(kThreads, 3)
    k_infect(PackedLayout L, const PackedTask *__restrict__ tasks,
             const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
             const uint4 *__restrict__ mask_in, const uint4 *__restrict__ sa,
             const uint4 *__restrict__ sb, uint4 *__restrict__ evs,
             uint32_t *__restrict__ flag32, uint32_t step, float scale,
             const __grid_constant__ StepConsts c) {
  __shared__ float s_bw[128];  // max |beta_r| of each word of the slice
  __shared__ uint4 s_lor[32];  // long row: OR of the neighbours' masks per column
  __shared__ long long s_lemax;
  __shared__ int32_t s_stage;  // the task's staging depth (CSR pairs per chunk)
  __shared__ unsigned long long s_bar[4];  // chunk buffers 0, 1; long-row halves 0, 1
  extern __shared__ __align__(16) unsigned char s_dyn[];
  int2 *const s_buf0 = reinterpret_cast<int2 *>(s_dyn);  // two staging buffers of kEntBuf pairs
  auto bufp = [&](int b) { return s_buf0 + b * kEntBuf; };
  InfectQueue &Q = reinterpret_cast<InfectQueue *>(s_dyn + kInfectQueueOff)[threadIdx.x >> 5];
  // the task's row pointers (rows of a task <= L.max_task_rows)
  int32_t *const s_rp = reinterpret_cast<int32_t *>(s_dyn + kInfectRpOff);
  // a long row's per-replica exposures (int32, ncols x 128 replicas)
  int32_t *const s_acc = reinterpret_cast<int32_t *>(s_dyn + infect_acc_off(L.max_task_rows));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t *mask_w = reinterpret_cast<const uint32_t *>(mask_in);
  uint32_t *evs_w = reinterpret_cast<uint32_t *>(evs);
  const uint8_t *flag8 = reinterpret_cast<const uint8_t *>(flag32);
  if (lane == 0) {
    Q.n = 0;
    Q.nk = 0;
  }
  if (threadIdx.x < 4) mbar_init(&s_bar[threadIdx.x]);
  if (threadIdx.x == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  uint32_t cph = 0, pph = 0;  // phase parity of each chunk buffer / half barrier
  int buf = 0;
  // every thread waits on the same barriers in the same order; a wait that
  // gives up raises the error flag (the host fails the run)
  auto wait_bar = [&](int b, uint32_t &ph, int bit) {
    const bool ready = mbar_wait(&s_bar[b], (ph >> bit) & 1u);
    ph ^= 1u << bit;
    if (!ready && c.err) atomicExch(c.err, 1);
  };
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int cbase = T.slice * 32;
    const int ncols = min(32, L.q4 - cbase);
    const Div dv((uint32_t)ncols);
    const int nrows = T.row_end - T.row_begin;
    for (int i = threadIdx.x; i <= nrows; i += blockDim.x) s_rp[i] = row_ptr[T.row_begin + i];
    if (threadIdx.x == 0) s_stage = T.stage < 1 || T.stage > kEntCap ? kEntCap : T.stage;
    if (c.beta_r)
      for (int wl = threadIdx.x; wl < ncols * 4; wl += blockDim.x) {
        float mx = 0.0f;
        for (int r = 0; r < 32; ++r) {
          const int rep = cbase * 128 + wl * 32 + r;
          if (rep < L.m) mx = fmaxf(mx, fabsf(__ldg(c.beta_r + rep)));
        }
        s_bw[wl] = mx;
      }
    __syncthreads();
    // chunk of rows [r0, end) of at most s_stage CSR pairs (>= 1 row; the
    // task's staging depth, at most a buffer; read from shared memory so
    // that it holds no register across the task)
    auto chunk_end = [&](int r0) {
      const int32_t stage = s_stage;
      int lo = r0 + 1, hi = nrows;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_rp[mid] - s_rp[r0] <= stage) lo = mid; else hi = mid - 1;
      }
      return lo;
    };
    // the chunk's pairs go to buffer b with one bulk copy (thread 0)
    auto stage_chunk = [&](int ra, int rb, int b) {
      const int32_t k0 = s_rp[ra], k1 = s_rp[rb];
      if (threadIdx.x == 0 && k1 > k0 && k1 - k0 <= kEntCap)
        stage_pairs(bufp(b), ent, k0, k1, &s_bar[b]);
    };
    int r0 = 0, r1 = nrows > 0 ? chunk_end(0) : 0;
    if (nrows > 0) stage_chunk(0, r1, buf);
    while (r0 < nrows) {
      const int r2 = r1 < nrows ? chunk_end(r1) : nrows;
      if (r1 < nrows) stage_chunk(r1, r2, buf ^ 1);  // prefetch the next chunk's pairs
      const int32_t e0 = s_rp[r0], e1 = s_rp[r1];
      const bool staged = e1 - e0 <= kEntCap;
      if (staged && e1 > e0) wait_bar(buf, cph, buf);
      const int2 *s_ent = bufp(buf) + pair_shift(ent, e0);
      // one row with more pairs than a buffer; streamed only when one of
      // its items may hold susceptible replicas
      const bool long_row =
          !staged && (!c.hints ||
                      __syncthreads_or(threadIdx.x < ncols &&
                                       (flag8[(int64_t)(T.row_begin + r0) * L.q4 + cbase +
                                              threadIdx.x] & kFlagSusceptible)));
      const bool skip_row = !staged && !long_row;
      const bool use_hint = c.hints && e1 - e0 >= 8 * (r1 - r0);  // at least 8 pairs per row
      bool dense_done = false;
      if (long_row) {
        // A hub of the window graph.  Its pairs stream through the two halves
        // of this chunk's buffer, one piece ahead; every warp takes a share
        // of each piece (lane = column: a pair costs one 512-byte line of mask
        // words) and, for the susceptible replicas of the row, adds the
        // pair's contact-seconds to each infectious neighbour replica's exact
        // exposure in shared memory.  Every exposed replica is then decided
        // from its exposure directly (no bound test, no per-candidate scan).
        const int64_t row = T.row_begin + r0;
        uint4 S4 = make_uint4(0, 0, 0, 0);
        if (lane < ncols) {
          const uint4 a4 = sa[row * L.q4 + cbase + lane], b4 = sb[row * L.q4 + cbase + lane];
#pragma unroll
          for (int w = 0; w < 4; ++w)
            set4(S4, w, ~get4(a4, w) & ~get4(b4, w) & word_mask(L, 4 * (cbase + lane) + w));
        }
        for (int j = threadIdx.x; j < ncols * 128; j += blockDim.x) s_acc[j] = 0;
        int2 *const half0 = bufp(buf);
        auto half = [&](int h) { return half0 + h * (kEntBuf / 2); };
        if (threadIdx.x < 32) s_lor[threadIdx.x] = make_uint4(0, 0, 0, 0);
        if (threadIdx.x == 0) {
          s_lemax = 0;
          stage_pairs(half(0), ent, e0, min(e0 + kPiece, e1), &s_bar[2]);
        }
        __syncthreads();
        uint4 linf = make_uint4(0, 0, 0, 0);
        long long lemax = 0;
        auto add_pair = [&](int2 q, uint4 m) {
          m = make_uint4(m.x & S4.x, m.y & S4.y, m.z & S4.z, m.w & S4.w);
          or4(linf, m);
#pragma unroll
          for (int w = 0; w < 4; ++w)
            for (uint32_t t = get4(m, w); t; t &= t - 1)
              atomicAdd(&s_acc[(lane * 4 + w) * 32 + __ffs(t) - 1], q.y);
        };
        const int npieces = (e1 - e0 + kPiece - 1) / kPiece;
        for (int pk = 0; pk < npieces; ++pk) {
          const int hb = pk & 1;
          const int32_t p0 = e0 + pk * kPiece, p1 = min(p0 + kPiece, e1);
          if (threadIdx.x == 0 && pk + 1 < npieces)
            stage_pairs(half(hb ^ 1), ent, p1, min(p1 + kPiece, e1), &s_bar[2 + (hb ^ 1)]);
          wait_bar(2 + hb, pph, hb);
          const int2 *pc = half(hb) + pair_shift(ent, p0);
          int32_t k = p0 + warp;
          for (; k + kWarps < p1; k += 2 * kWarps) {
            const int2 q0 = pc[k - p0], q1 = pc[k - p0 + kWarps];
            lemax += (long long)q0.y + q1.y;
            if (lane < ncols) {
              const uint4 m0 = mask_in[(int64_t)q0.x * L.q4 + cbase + lane];
              const uint4 m1 = mask_in[(int64_t)q1.x * L.q4 + cbase + lane];
              add_pair(q0, m0);
              add_pair(q1, m1);
            }
          }
          for (; k < p1; k += kWarps) {
            const int2 q0 = pc[k - p0];
            lemax += q0.y;
            if (lane < ncols) add_pair(q0, mask_in[(int64_t)q0.x * L.q4 + cbase + lane]);
          }
          __syncthreads();  // the half is free to restage
        }
        if (lane < ncols) {
          atomicOr(&s_lor[lane].x, linf.x);
          atomicOr(&s_lor[lane].y, linf.y);
          atomicOr(&s_lor[lane].z, linf.z);
          atomicOr(&s_lor[lane].w, linf.w);
        }
        if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long *>(&s_lemax),
                                 (unsigned long long)lemax);
        __syncthreads();
        // int32 sums are exact while the row's total fits; otherwise its
        // items take the per-candidate exact test below
        dense_done = s_lemax <= 0x7FFFFFFFll;
        if (dense_done) {
          const uint32_t *lor = reinterpret_cast<const uint32_t *>(s_lor);
          const float bs_row = c.sus ? __ldg(c.sus + row) : 1.0f;
          for (int wl = threadIdx.x; wl < ncols * 4; wl += blockDim.x) {
            const uint32_t X = lor[wl];  // exposed replicas of the word
            if (!X) continue;
            const int word = 4 * cbase + wl;
            uint32_t pl[8];
            infect_planes(c.rk, (uint32_t)row, step, (uint32_t)word + (c.roff >> 5), pl);
            uint32_t ev = 0;
            for (uint32_t t = X; t; t &= t - 1) {
              const int b = __ffs(t) - 1;
              const float br = c.beta_r ? __ldg(c.beta_r + word * 32 + b) : c.beta;
              const float bs = c.sus ? __fmul_rn(br, bs_row) : br;
              float ef = __int2float_rn(s_acc[wl * 32 + b]);
              if (scale != 1.0f) ef = __fmul_rn(ef, scale);
              const float xx = __fmul_rn(bs, ef);
              if (!(xx > 0.0f)) continue;
              const uint32_t u8 = top8_of(pl, (uint32_t)b);
              if (xx < 1.0f && u8 > (uint32_t)(fixed64(xx) >> 56)) continue;
              const uint32_t gword = (uint32_t)word + (c.roff >> 5);
              if (infect_event(one_minus_exp_neg(xx), u8, c.rk, (uint32_t)row, step,
                               gword * 32u + (uint32_t)b))
                ev |= 1u << b;
            }
            if (ev) {
              atomicOr(&evs_w[row * L.words + word], ev);
              const int64_t idx = row * L.q4 + (word >> 2);
              atomicOr(&flag32[idx >> 2], 1u << (8 * (idx & 3)));
            }
          }
        }
        __syncthreads();
      }
      const int nitems = skip_row || dense_done ? 0 : (r1 - r0) * ncols;
      // warp-uniform passes; one pass past the items decides what is left
      // queued (the staged pairs change with the next chunk)
      int blk = warp * 32;  // this warp's next block of 32 items
      // a chunk with fewer pairs than half its rows compacts its items
      // (most of its rows have no pairs)
      const bool sparse = 2 * (e1 - e0) < r1 - r0;
      for (;;) {
        // ---- phase 1a: in a sparse chunk, up to 32 items with CSR pairs
        // from the warp's next blocks (many blocks fold into one pass; items
        // without pairs have nothing to gather).  Their indices pass through
        // Q.off, the rounds' scratch, which is free until the rounds ----
        int got, it;
        if (sparse) {
          got = 0;
          while (blk < nitems) {
            const int itb = blk + lane;
            bool has = false;
            if (itb < nitems) {
              const int rlb = (int)dv.div((uint32_t)itb);
              has = s_rp[r0 + rlb + 1] > s_rp[r0 + rlb];
            }
            const unsigned hm = __ballot_sync(kFull, has);
            if (got + __popc(hm) > 32) break;
            if (has) Q.off[got + __popc(hm & ((1u << lane) - 1u))] = itb;
            got += __popc(hm);
            blk += kWarps * 32;
          }
          __syncwarp();
          it = lane < got ? Q.off[lane] : 0;
          __syncwarp();
        } else {  // one block per pass
          got = blk < nitems ? min(32, nitems - blk) : 0;
          it = blk + lane;
          blk += kWarps * 32;
        }
        const bool flushing = got == 0;
        // ---- phase 1: gather, per lane ----
        const bool ok = lane < got;
        const int rl = ok ? (int)dv.div((uint32_t)it) : 0;
        const int cc = ok ? it - rl * ncols : 0;
        const int rloc = r0 + rl;
        const int col = cbase + cc;
        const int row = T.row_begin + rloc;
        const int32_t beg = s_rp[rloc], end = s_rp[rloc + 1];
        const int64_t idx = (int64_t)row * L.q4 + col;
        // an item without susceptible replicas cannot be infected: on
        // pair-heavy chunks the hint byte saves the item's whole gather
        const int n = ok && (!use_hint || (flag8[idx] & kFlagSusceptible)) ? end - beg : 0;
        uint32_t X[4] = {0, 0, 0, 0};
        float efmax = 0.0f;
        if (n > 0) {
          const uint4 a4 = sa[idx], b4 = sb[idx];
          const int2 *er = s_ent + (beg - e0);
          uint4 inf = make_uint4(0, 0, 0, 0);
          long long emax = 0;
          int k = 0;
          if (long_row) {  // gathered by the whole CTA above
            inf = s_lor[cc];
            emax = s_lemax;
            k = n;
          }
          for (; k + 4 <= n; k += 4) {
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
          for (; k < n; ++k) {
            const int2 q0 = er[k];
            or4(inf, mask_in[(int64_t)q0.x * L.q4 + col]);
            emax += q0.y;
          }
#pragma unroll
          for (int w = 0; w < 4; ++w)
            X[w] = get4(inf, w) & ~get4(a4, w) & ~get4(b4, w) & word_mask(L, 4 * col + w);
          efmax = __ll2float_rn(emax);
          if (scale != 1.0f) efmax = __fmul_rn(efmax, scale);
        }
        // ---- queue the exposed words ----
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const unsigned qm = __ballot_sync(kFull, X[w] != 0u);
          if (!qm) continue;
          const int base = Q.n;
          if (X[w]) {
            const int pos = base + __popc(qm & ((1u << lane) - 1u));
            Q.rloc[pos] = rloc;
            Q.word[pos] = 4 * col + w;
            Q.X[pos] = X[w];
            Q.efmax[pos] = efmax;
          }
          __syncwarp();
          if (lane == 0) Q.n = base + __popc(qm);
          __syncwarp();
        }
        // ---- decide full rounds (and, past the items, the remainder and
        // the carried candidates: the staged pairs change with the chunk) ----
        while (Q.n >= 32 || (flushing && (Q.n > 0 || Q.nk > 0))) {
          const int take = Q.n < 32 ? Q.n : 32;
          infect_round(Q, take, flushing && take == Q.n, lane, L, T, cbase, s_rp, s_ent, ent,
                       staged, e0, s_bw, mask_w, evs_w, flag32, step, scale, c);
          const int rest = Q.n - take;
          for (int i = lane; i < rest; i += 32) {
            Q.rloc[i] = Q.rloc[take + i];
            Q.word[i] = Q.word[take + i];
            Q.X[i] = Q.X[take + i];
            Q.efmax[i] = Q.efmax[take + i];
          }
          __syncwarp();
          if (lane == 0) Q.n = rest;
          __syncwarp();
        }
        if (flushing) break;
      }
      __syncthreads();
      r0 = r1;
      r1 = r2;
      buf ^= 1;
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

// Applies one word's moves; returns the new planes and counts the events.
// Per-replica event counters of a task slice in shared memory, two 32-bit
// words per replica (32-bit shared atomics): c0 = S->E | ->I << 16,
// c1 = I-> | R->S << 16 (a task has at most 4,096 rows).
__device__ __forceinline__ void count_bits32(uint32_t *s_c, int wl, uint32_t t, uint32_t inc) {
  while (t) {
    const int r = __ffs(t) - 1;
    atomicAdd(&s_c[wl * 32 + r], inc);
    t &= t - 1;
  }
}

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
    uint32_t *c0 = reinterpret_cast<uint32_t *>(s_ev), *c1 = c0 + 128 * 32;
    count_bits32(c0, wl, c.has_exposed ? evS : 0u, 1u);
    count_bits32(c0, wl, evE | (c.has_exposed ? 0u : evS), 1u << 16);
    count_bits32(c1, wl, evI, 1u);
    count_bits32(c1, wl, evR, 1u << 16);
  }
}

// Per-warp queue of words with flow candidates (dynamic shared memory):
// words are queued while the warp streams its items and drawn in full
// 32-lane rounds, so sparse candidates do not leave lanes idle.
constexpr int kFlowIPL = 4;      // items per lane per pass (loads in flight)
constexpr int kFlowQueue = 576;  // 31 left over + 4 words x kFlowIPL items x 32 lanes (+ pad)
struct FlowQueue {
  int32_t row[kFlowQueue];
  uint16_t word[kFlowQueue];  // word index within the row
  int32_t n;
};
constexpr int kFlowDynSmem = 128 * 32 * 8 + kWarps * (int)sizeof(FlowQueue);

// Draws the flows of queue entries [0, cnt) (cnt <= 32, one per lane) and
// writes the words: infection events and flows act on disjoint state bits,
// so both are applied here from the start-of-step planes.
__device__ __forceinline__ void flow_round(const FlowQueue &Q, int base, int cnt, int lane,
                                           bool waning, const StepConsts &c, uint32_t step,
                                           unsigned long long *s_ev, uint32_t *sa_w,
                                           uint32_t *sb_w, uint32_t *mask_w, uint32_t *evs_w,
                                           int words, int cbase) {
  if (lane < cnt) {
    const int q = base + lane;
    const int row = Q.row[q], word = Q.word[q];
    const int64_t wi = (int64_t)row * words + word;
    const uint32_t A = sa_w[wi], B = sb_w[wi], ev = evs_w[wi];
    if (ev) evs_w[wi] = 0u;
    const uint32_t E = ~A & B, I = A & ~B, R = waning ? (A & B) : 0u;
    const uint32_t f =
        flow_events(E, I, R, c.th, c.rk, (uint32_t)row, step, (uint32_t)word + (c.roff >> 5));
    uint32_t na, nb;
    apply_word(A, B, ev, f, waning, c, s_ev, word - 4 * cbase, na, nb);
    if (na != A || nb != B) {
      sa_w[wi] = na;
      sb_w[wi] = nb;
      mask_w[wi] = na & ~nb;
    }
  }
}

// Streams the items of each task: infection events of words without flow
// candidates are applied on the spot, words with candidates are queued.
__global__ void __launch_bounds__(kThreads, 3)
    k_flow(PackedLayout L, const PackedTask *__restrict__ tasks,
           const int32_t *__restrict__ row_ptr, uint4 *__restrict__ evs,
           uint4 *__restrict__ mask, uint4 *__restrict__ sa, uint4 *__restrict__ sb,
           uint8_t *__restrict__ flag, unsigned long long *__restrict__ ev_row,
           unsigned long long *__restrict__ rs_row, uint32_t step, StepConsts c) {
  extern __shared__ __align__(16) unsigned char s_dynf[];
  // 4 x 16-bit event counters per replica of the slice
  unsigned long long *s_ev = reinterpret_cast<unsigned long long *>(s_dynf);
  FlowQueue &Q = reinterpret_cast<FlowQueue *>(s_dynf + 128 * 32 * 8)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool waning = c.th.tr_all || c.th.tr != 0;
  uint32_t *sa_w = reinterpret_cast<uint32_t *>(sa);
  uint32_t *sb_w = reinterpret_cast<uint32_t *>(sb);
  uint32_t *mask_w = reinterpret_cast<uint32_t *>(mask);
  for (int ti = blockIdx.x; ti < L.n_tasks; ti += gridDim.x) {
    const PackedTask T = tasks[ti];
    const int cbase = T.slice * 32;
    const int ncols = min(32, L.q4 - cbase);
    const Div dv((uint32_t)ncols);
    const int nrows = T.row_end - T.row_begin;
    {  // the task's counters: two 32-bit words for each of its ncols x 128 replicas
      uint32_t *c0 = reinterpret_cast<uint32_t *>(s_ev);
      for (int j = threadIdx.x; j < ncols * 128; j += blockDim.x) {
        c0[j] = 0;
        c0[128 * 32 + j] = 0;
      }
    }
    if (lane == 0) Q.n = 0;
    __syncthreads();
    const int nitems = nrows * ncols;
    uint32_t *evs_w = reinterpret_cast<uint32_t *>(evs);
    // warp-uniform passes of kFlowIPL items per lane, all loads issued
    // first; candidate words are queued, and full rounds of 32 decided after
    // the pass (one pass past the items decides the rest; one call site of
    // flow_round keeps the kernel small)
    for (int it0 = warp * 32 * kFlowIPL;; it0 += kWarps * 32 * kFlowIPL) {
      const bool flushing = it0 >= nitems;
      int rl[kFlowIPL], cl[kFlowIPL];
      bool in[kFlowIPL];
      uint8_t st[kFlowIPL];
      uint4 a4[kFlowIPL], b4[kFlowIPL];
#pragma unroll
      for (int h = 0; h < kFlowIPL; ++h) {
        const int itv = it0 + 32 * h + lane;
        in[h] = itv < nitems;
        rl[h] = in[h] ? (int)dv.div((uint32_t)itv) : 0;
        cl[h] = in[h] ? itv - rl[h] * ncols : 0;
        const int64_t idx = (int64_t)(T.row_begin + rl[h]) * L.q4 + cbase + cl[h];
        a4[h] = b4[h] = make_uint4(0, 0, 0, 0);
        st[h] = 0;
        if (in[h]) {
          st[h] = flag[idx];
          a4[h] = sa[idx];
          b4[h] = sb[idx];
        }
      }
      // quiet items (every replica susceptible, or recovered without waning,
      // and no infection event) need no work: skip them a warp at a time
      bool busy = false;
      uint32_t cm[kFlowIPL];
      int cnt = 0;
#pragma unroll
      for (int h = 0; h < kFlowIPL; ++h) {
        cm[h] = 0;
#pragma unroll
        for (int w = 0; w < 4; ++w) {  // padding replicas are S: no replica mask needed
          const uint32_t A = get4(a4[h], w), B = get4(b4[h], w);
          if ((waning ? (A | B) : (A ^ B)) != 0u) cm[h] |= 1u << w;
        }
        cnt += __popc(cm[h]);
        busy |= (st[h] & kFlagEvent) != 0 || cm[h] != 0;
        // next step's hint byte, from this step's planes and events: a
        // superset of the items with susceptible replicas (and of those
        // that can move: E, I, waning R, or newly infected)
        if (c.hints && in[h]) {
          // E, I or waning R (the words of cm), or an infection event
          const bool act = (st[h] & kFlagEvent) != 0 || cm[h] != 0u;
          uint32_t s4 = 0;
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            const uint32_t A = get4(a4[h], w), B = get4(b4[h], w);
            // S now, or back to S this step (waning R, or I -> S); padding
            // replicas are S, so only a row's last item needs the mask
            uint32_t sw = (~A & ~B) | (waning ? (A & B) : 0u) | (c.ir_to_s ? (A & ~B) : 0u);
            if (4 * (cbase + cl[h]) + 4 > L.vwords) sw &= word_mask(L, 4 * (cbase + cl[h]) + w);
            s4 |= sw;
          }
          const uint8_t nb = (uint8_t)((act ? kFlagActive : 0) | (s4 ? kFlagSusceptible : 0));
          if (nb != st[h]) flag[(int64_t)(T.row_begin + rl[h]) * L.q4 + cbase + cl[h]] = nb;
        }
      }
      if (!flushing && !__any_sync(kFull, busy)) continue;
      // infection events: words without flow candidates are applied here;
      // the queued words' events are read (and cleared) by their round
#pragma unroll
      for (int h = 0; h < kFlowIPL; ++h) {
        if (!(st[h] & kFlagEvent)) continue;
        const int64_t idx = (int64_t)(T.row_begin + rl[h]) * L.q4 + cbase + cl[h];
        const uint4 e4 = evs[idx];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const uint32_t ev = get4(e4, w);
          if (!ev || ((cm[h] >> w) & 1u)) continue;
          const int word = 4 * (cbase + cl[h]) + w;
          const int64_t wi = (int64_t)(T.row_begin + rl[h]) * L.words + word;
          uint32_t na, nb;
          apply_word(get4(a4[h], w), get4(b4[h], w), ev, 0u, waning, c, s_ev, 4 * cl[h] + w, na,
                     nb);
          sa_w[wi] = na;
          sb_w[wi] = nb;
          mask_w[wi] = na & ~nb;
          evs_w[wi] = 0u;
        }
      }
      // queue the candidate words of the pass (one scan)
      int total;
      int pos = warp_excl_scan(cnt, lane, total);
      if (total > 0) {  // warp-uniform
        pos += Q.n;
        // one iteration per candidate word of the lane (most lanes have none)
        uint32_t all = 0;
#pragma unroll
        for (int h = 0; h < kFlowIPL; ++h) all |= cm[h] << (4 * h);
        while (all) {
          const int bit = __ffs(all) - 1;
          all &= all - 1;
          const int h = bit >> 2;
          int r = rl[0], cc = cl[0];
#pragma unroll
          for (int hh = 1; hh < kFlowIPL; ++hh)
            if (h == hh) {
              r = rl[hh];
              cc = cl[hh];
            }
          Q.row[pos] = T.row_begin + r;
          Q.word[pos] = (uint16_t)(4 * (cbase + cc) + (bit & 3));
          ++pos;
        }
        __syncwarp();
      }
      const int n = Q.n + total;
      int start = 0;
      for (; n - start >= 32 || (flushing && n - start > 0); start += 32)
        flow_round(Q, start, min(32, n - start), lane, waning, c, step, s_ev, sa_w, sb_w, mask_w,
                   evs_w, L.words, cbase);
      __syncwarp();
      const int rest = max(n - start, 0);
      if (start > 0 && rest > 0) {  // move the remainder (< 32 words) to the front
        const int q = start + lane;
        int32_t r0 = 0;
        uint16_t w0 = 0;
        if (lane < rest) {
          r0 = Q.row[q];
          w0 = Q.word[q];
        }
        __syncwarp();
        if (lane < rest) {
          Q.row[lane] = r0;
          Q.word[lane] = w0;
        }
      }
      __syncwarp();
      if (lane == 0) Q.n = rest;
      __syncwarp();
      if (flushing) break;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < ncols * 128; j += blockDim.x) {
      const uint32_t *c0 = reinterpret_cast<const uint32_t *>(s_ev), *c1 = c0 + 128 * 32;
      const unsigned long long v = (unsigned long long)c0[j] | ((unsigned long long)c1[j] << 32);
      if (!v) continue;
      const int rep = cbase * 128 + j;
      if (rep >= L.m) continue;
      const unsigned long long f16 = 0xFFFFull;
      const unsigned long long g = (v & f16) | (((v >> 16) & f16) << kFieldBits) |
                                   (((v >> 32) & f16) << (2 * kFieldBits));
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
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) s_ev[j] = 0;
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

// Hint bytes of every item from the initial planes (kFlagActive: E, I or
// waning R replicas; kFlagSusceptible: S replicas).
__global__ void k_flag_from_planes(PackedLayout L, const uint4 *__restrict__ sa,
                                   const uint4 *__restrict__ sb, uint8_t *__restrict__ flag,
                                   bool waning) {
  const int64_t total = (int64_t)L.n_nodes * L.q4;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint4 a4 = sa[i], b4 = sb[i];
    const int col = (int)(i % L.q4);
    bool act = false, sus = false;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const uint32_t A = get4(a4, w), B = get4(b4, w), vm = word_mask(L, 4 * col + w);
      act |= (((A ^ B) | (waning ? (A & B) : 0u)) & vm) != 0u;
      sus |= ((~A & ~B) & vm) != 0u;
    }
    flag[i] = (uint8_t)((act ? kFlagActive : 0) | (sus ? kFlagSusceptible : 0));
  }
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

rp_status packed_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_flow, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kFlowDynSmem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_flow)");
  e = cudaFuncSetAttribute(k_infect, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kInfectDynSmemMax);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_infect)");
  return RP_OK;
}

void packed_init(const PackedLayout &L, uint32_t *sa, uint32_t *sb, uint32_t *mask,
                 uint8_t *flag, float p0, int32_t k_exact, const int32_t *net_first_row,
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
  cudaMemsetAsync(flag, 0, ((size_t)L.n_nodes * L.q4 + 3) / 4 * 4, st);
  k_flag_from_planes<<<1184, 256, 0, st>>>(L, reinterpret_cast<const uint4 *>(sa),
                                           reinterpret_cast<const uint4 *>(sb), flag,
                                           c.th.tr_all || c.th.tr != 0);
}

void packed_step(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
                 const int2 *entries, uint32_t *mask, uint32_t *sa, uint32_t *sb, uint32_t *evs,
                 uint8_t *flag, unsigned long long *ev_row, unsigned long long *rs_row,
                 uint32_t step, float scale, const StepConsts &c, cudaStream_t st) {
  packed_infect(L, tasks, row_ptr, entries, mask, sa, sb, evs, flag, step, scale, c, st);
  packed_flow(L, tasks, row_ptr, mask, sa, sb, evs, flag, ev_row, rs_row, step, c, st);
}

void packed_infect(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
                   const int2 *entries, const uint32_t *mask, const uint32_t *sa,
                   const uint32_t *sb, uint32_t *evs, uint8_t *flag, uint32_t step, float scale,
                   const StepConsts &c, cudaStream_t st) {
  k_infect<<<task_grid(L.n_tasks, 3), kThreads, infect_smem(L.q4, L.max_task_rows), st>>>(
      L, tasks, row_ptr, entries, reinterpret_cast<const uint4 *>(mask),
      reinterpret_cast<const uint4 *>(sa), reinterpret_cast<const uint4 *>(sb),
      reinterpret_cast<uint4 *>(evs), reinterpret_cast<uint32_t *>(flag), step, scale, c);
}

void packed_flow(const PackedLayout &L, const PackedTask *tasks, const int32_t *row_ptr,
                 uint32_t *mask, uint32_t *sa, uint32_t *sb, const uint32_t *evs, uint8_t *flag,
                 unsigned long long *ev_row, unsigned long long *rs_row, uint32_t step,
                 const StepConsts &c, cudaStream_t st) {
  k_flow<<<task_grid(L.n_tasks, 3), kThreads, kFlowDynSmem, st>>>(
      L, tasks, row_ptr, reinterpret_cast<uint4 *>(const_cast<uint32_t *>(evs)),
      reinterpret_cast<uint4 *>(mask), reinterpret_cast<uint4 *>(sa),
      reinterpret_cast<uint4 *>(sb), flag, ev_row, rs_row, step, c);
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
