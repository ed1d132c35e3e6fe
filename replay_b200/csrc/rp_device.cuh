// Device helpers shared by the replay kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rp_internal.h"

namespace rp {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of two
// 32x32->64 multiplies with a Weyl key schedule.  Counter-based: every
// (key, counter) pair is an independent draw, so any thread can produce the
// uniform of any (replica, node, step) without state.
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1,
                                              uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1,
                                              uint32_t out[4]) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint32_t lo0 = 0xD2511F53u * c0;
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Same generator with the 10 round keys precomputed (key schedule hoisted
// out of the per-call work): rk[2 i], rk[2 i + 1] are round i's key words.
__device__ __forceinline__ void philox4x32_10_rk(uint32_t c0, uint32_t c1, uint32_t c2,
                                                 uint32_t c3, const uint32_t *rk,
                                                 uint32_t out[4]) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint32_t lo0 = 0xD2511F53u * c0;
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ rk[2 * round];
    const uint32_t n2 = hi0 ^ c3 ^ rk[2 * round + 1];
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Two independent calls of philox4x32_10_rk on counters (c0, c1, c2, c3a)
// and (c0, c1, c2, c3b), interleaved round by round so that the two
// dependency chains overlap (twice the instruction-level parallelism).
__device__ __forceinline__ void philox4x32_10_rk_x2(uint32_t c0, uint32_t c1, uint32_t c2,
                                                    uint32_t c3a, uint32_t c3b,
                                                    const uint32_t *rk, uint32_t a[4],
                                                    uint32_t b[4]) {
  uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3a;
  uint32_t y0 = c0, y1 = c1, y2 = c2, y3 = c3b;
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint32_t xl0 = 0xD2511F53u * x0, xh0 = __umulhi(0xD2511F53u, x0);
    const uint32_t yl0 = 0xD2511F53u * y0, yh0 = __umulhi(0xD2511F53u, y0);
    const uint32_t xl1 = 0xCD9E8D57u * x2, xh1 = __umulhi(0xCD9E8D57u, x2);
    const uint32_t yl1 = 0xCD9E8D57u * y2, yh1 = __umulhi(0xCD9E8D57u, y2);
    const uint32_t k0 = rk[2 * round], k1 = rk[2 * round + 1];
    x0 = xh1 ^ x1 ^ k0;
    y0 = yh1 ^ y1 ^ k0;
    x2 = xh0 ^ x3 ^ k1;
    y2 = yh0 ^ y3 ^ k1;
    x1 = xl1;
    y1 = yl1;
    x3 = xl0;
    y3 = yl0;
  }
  a[0] = x0; a[1] = x1; a[2] = x2; a[3] = x3;
  b[0] = y0; b[1] = y1; b[2] = y2; b[3] = y3;
}

// Uniform on the 24-bit grid ((x >> 8) + 1) * 2^-24, in (0, 1]; exact in
// float, so host and device agree bit for bit.
__device__ __forceinline__ float unit24(uint32_t x) {
  return __fmul_rn(__uint2float_rn((x >> 8) + 1u), 0x1p-24f);
}

// Random stream layout, key = seed, counter = (node, step, c2, c3):
//  * countdown-mode infection (S->E / S->I) uniform of replica r:
//    c2 = r / 4, c3 = 3, output r % 4 on the 24-bit grid; event iff P > u;
//  * flow (E->I, I->R, R->S) uniform of replica r: bit-sliced -- bit k of
//    U_r (k = 0 is 2^-1) is bit r % 32 of output k % 4 of counter
//    (node, step, r / 32, (k / 4) << 4); event iff U_r < floor(p 2^64)
//    over the first 64 bits (flow_events);
//  * geometric-mode infection uniform: top 8 bits bit-sliced on
//    c3 = 4 | j << 4 (c2 = r / 32), low 56 bits on c2 = r, c3 = 12
//    (infect_event);
//  * Bernoulli initial condition: step 0xFFFFFFFF, c2 = r / 4, c3 = 1;
//  * exact-count initial condition (Floyd): node = draw j, step
//    0xFFFFFFFE, c2 = r, c3 = 2 (+ 4 x network index).
constexpr uint32_t kStreamFlow = 0u;    // bit-sliced flow uniforms, c3 = plane/4 << 4
constexpr uint32_t kStreamInit = 1u;
constexpr uint32_t kStreamPick = 2u;
constexpr uint32_t kStreamInfect = 3u;  // scalar infection uniforms
constexpr uint32_t kStepInit = 0xFFFFFFFFu;
constexpr uint32_t kStepPick = 0xFFFFFFFEu;

// 1 - exp(-x) for x >= 0 from correctly rounded multiplies and adds only
// (no FMA contraction): Cody-Waite reduction x = k ln2 + r with ln2 split in
// a 15-bit head and a tail, then the Taylor series of expm1(-r) through
// r^9/9! in Horner form.  Max error about 1 ulp; NaN propagates (the
// reference's p = 1, zero-exposure case), +inf gives 1.
__device__ __forceinline__ float one_minus_exp_neg(float x) {
  if (x != x) return x;
  if (!(x > 0.0f)) return 0.0f;
  if (x >= 87.0f) return 1.0f;
  const float inv_ln2 = 0x1.715476p+0f;
  const float ln2_hi = 0x1.62e4p-1f;
  const float ln2_lo = 0x1.7f7d1cp-20f;
  const int k = __float2int_rz(__fadd_rn(__fmul_rn(x, inv_ln2), 0.5f));
  const float kf = __int2float_rn(k);
  const float r =
      __fsub_rn(__fsub_rn(x, __fmul_rn(kf, ln2_hi)), __fmul_rn(kf, ln2_lo));
  const float y = -r;
  float p = 0x1.71de3ap-19f;
  p = __fadd_rn(__fmul_rn(p, y), 0x1.a01a02p-16f);
  p = __fadd_rn(__fmul_rn(p, y), 0x1.a01a02p-13f);
  p = __fadd_rn(__fmul_rn(p, y), 0x1.6c16c2p-10f);
  p = __fadd_rn(__fmul_rn(p, y), 0x1.111112p-7f);
  p = __fadd_rn(__fmul_rn(p, y), 0x1.555556p-5f);
  p = __fadd_rn(__fmul_rn(p, y), 0x1.555556p-3f);
  p = __fadd_rn(__fmul_rn(p, y), 0.5f);
  const float em1 = __fadd_rn(y, __fmul_rn(__fmul_rn(y, y), p));
  if (k == 0) return -em1;
  const float scale = __int_as_float((127 - k) << 23);
  const float e = __fmul_rn(__fadd_rn(1.0f, em1), scale);
  return __fsub_rn(1.0f, e);
}

// Per-step flow thresholds (FlowThresholds, rp_internal.h) hold
// floor(p 2^64); p >= 1 is a certain event, p <= 0 none.
// Flow events of the replicas selected by E, I, R (disjoint masks of one
// 32-replica word of `node`): replica r moves iff its bit-sliced uniform is
// below its state's threshold.  All 32 replicas are compared at once, one
// random plane per bit, stopping when every candidate is decided (about
// log2(candidates) + 2 planes).  Returns the event mask.
__device__ __forceinline__ uint32_t flow_events(uint32_t E, uint32_t I, uint32_t R,
                                                const FlowThresholds &th, const uint32_t *rk,
                                                uint32_t node, uint32_t step, uint32_t word) {
  uint32_t lt = (th.te_all ? E : 0u) | (th.ti_all ? I : 0u) | (th.tr_all ? R : 0u);
  const uint32_t e2 = (th.te_all || th.te == 0) ? 0u : E;
  const uint32_t i2 = (th.ti_all || th.ti == 0) ? 0u : I;
  const uint32_t r2 = (th.tr_all || th.tr == 0) ? 0u : R;
  uint32_t und = e2 | i2 | r2;
  if (und == 0u) return lt;  // every candidate's threshold is 0 or 1: no draw
  // one random call decides 4 planes for all 32 replicas of the word
  auto planes = [&](const uint32_t (&x)[4], int j) {
    const int sh = 60 - 4 * j;
    const uint32_t ce = (uint32_t)(th.te >> sh) & 0xFu;
    const uint32_t ci = (uint32_t)(th.ti >> sh) & 0xFu;
    const uint32_t cr = (uint32_t)(th.tr >> sh) & 0xFu;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t b = 3 - q;
      const uint32_t T = (((ce >> b) & 1u) ? e2 : 0u) | (((ci >> b) & 1u) ? i2 : 0u) |
                         (((cr >> b) & 1u) ? r2 : 0u);
      const uint32_t w = x[q];
      lt |= und & T & ~w;
      und &= ~(T ^ w);
    }
  };
  // the first two calls (8 planes) run together, unconditionally; later
  // planes only while some replica is undecided
  uint32_t x0[4], x1[4];
  philox4x32_10_rk_x2(node, step, word, 0u, 1u << 4, rk, x0, x1);
  planes(x0, 0);
  planes(x1, 1);
  for (int j = 2; j < 16 && und != 0u; ++j) {
    uint32_t x[4];
    philox4x32_10_rk(node, step, word, (uint32_t)j << 4, rk, x);
    planes(x, j);
  }
  return lt;
}

// floor(p 2^64) for 0 < p < 1 (exact: p 2^64 is exact in float, then
// truncated).
__device__ __forceinline__ unsigned long long fixed64(float p) {
  return __float2ull_rz(__fmul_rn(p, 0x1p64f));
}

// Geometric infection uniform U_r of replica r, 64 bits, compared with
// floor(P 2^64).  Its top 8 bits are bit-sliced: bit k (k = 0 is 2^-1) is bit
// r % 32 of output k % 4 of counter (node, step, r / 32, 4 | (k / 4) << 4),
// so that two calls screen all 32 replicas of a word at once.  Its low 56
// bits are the top 56 bits of outputs 0-1 (output 0 high) of counter
// (node, step, r, 12), drawn only when the top 8 bits tie with the
// threshold's.
constexpr uint32_t kTagInfect = 4u;
constexpr uint32_t kTagInfectTail = 12u;

// The 8 planes of a word's infection uniforms.
__device__ __forceinline__ void infect_planes(const uint32_t *rk, uint32_t node, uint32_t step,
                                              uint32_t word, uint32_t pl[8]) {
  philox4x32_10_rk_x2(node, step, word, kTagInfect, kTagInfect | 16u, rk, pl, pl + 4);
}

// Top 8 bits of the uniform of replica bit b from its word's planes.
__device__ __forceinline__ uint32_t top8_of(const uint32_t pl[8], uint32_t b) {
  uint32_t u = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) u = (u << 1) | ((pl[k] >> b) & 1u);
  return u;
}

// Replicas of `cand` whose top 8 uniform bits are at most T's: a superset of
// those with U < T.
__device__ __forceinline__ uint32_t top8_le(uint32_t cand, unsigned long long T,
                                            const uint32_t pl[8]) {
  const uint32_t t8 = (uint32_t)(T >> 56);
  uint32_t lt = 0, und = cand;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t t = ((t8 >> (7 - k)) & 1u) ? 0xFFFFFFFFu : 0u;
    lt |= und & t & ~pl[k];
    und &= ~(t ^ pl[k]);
  }
  return lt | und;
}

// Low 56 bits of the infection uniform of (global) replica `replica`.
__device__ __forceinline__ unsigned long long infect_tail56(const uint32_t *rk, uint32_t node,
                                                            uint32_t step, uint32_t replica) {
  uint32_t x[4];
  philox4x32_10_rk(node, step, replica, kTagInfectTail, rk, x);
  return (((unsigned long long)x[0] << 32) | x[1]) >> 8;
}

// Infection event of a replica whose uniform's top 8 bits are u8: event iff
// U < floor(P 2^64); P >= 1 always, P <= 0 or NaN never.
__device__ __forceinline__ bool infect_event(float P, uint32_t u8, const uint32_t *rk,
                                             uint32_t node, uint32_t step, uint32_t replica) {
  if (!(P > 0.0f)) return false;
  if (P >= 1.0f) return true;
  const unsigned long long T = fixed64(P);
  const uint32_t t8 = (uint32_t)(T >> 56);
  if (u8 != t8) return u8 < t8;
  return infect_tail56(rk, node, step, replica) < (T & 0x00FFFFFFFFFFFFFFull);
}

// Countdown arithmetic of the reference (int op float, truncated back to
// int): c = (int)((float)c - step) and c = (int)((float)base + step).
__device__ __forceinline__ int32_t cd_sub(int32_t c, float step) {
  return __float2int_rz(__fsub_rn(__int2float_rn(c), step));
}
__device__ __forceinline__ int32_t cd_add(int32_t base, float step) {
  return __float2int_rz(__fadd_rn(__int2float_rn(base), step));
}

// Summary classification of a countdown value
// (tool/gpu_cpu_temporal_sim.cu:530-550): 0 S, 1 E, 2 I, 3 R.
__device__ __forceinline__ int countdown_class(int32_t c, int32_t E, int32_t I,
                                               int32_t R) {
  const int32_t upper = E + I + R;
  const int32_t elapsed = (c <= 0 || c > upper) ? 0 : (upper - c);
  if (c == 0) return 0;
  if (E > 0 && elapsed < E) return 1;
  if (I > 0 && elapsed < E + I) return 2;
  if (R > 0 && elapsed < E + I + R) return 3;
  return 0;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

}  // namespace rp
