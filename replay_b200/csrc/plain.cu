// Plain path: the drop-in structure of the reference step loop
// (tool/gpu_cpu_temporal_sim.cu:1053-1084) without cuSPARSE: one
// per-replica SpMV over the window CSR, then one elementwise transition
// kernel that also reduces the per-replica S/E/I/R counts.
//
// State is column-major N x M (index = node + replica * N) as in the
// reference: int32 countdowns (countdown mode) or uint8 codes (geometric
// mode: 0 S, 1 E, 2 I, 3 R).  The infectious vector of
// generate_infectious_vector (:92-111) is read straight from the
// neighbours' states inside the SpMV.
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

// ---- exposure -----------------------------------------------------------------
// Countdown mode: FP32 row sums in CSR order, as Eigen's row-major
// sparse x dense product (CPUComputeSpMM, :403-433) accumulates them.
__global__ void __launch_bounds__(256)
    k_spmv_countdown(const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
                     const int32_t *__restrict__ cd, float *__restrict__ expo, int32_t n,
                     int32_t m, int32_t lower, int32_t medium) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t beg = row_ptr[i], end = row_ptr[i + 1];
  for (int32_t r = blockIdx.y; r < m; r += gridDim.y) {
    const int32_t *col_state = cd + (int64_t)r * n;
    float acc = 0.0f;
    for (int32_t k = beg; k < end; ++k) {
      const int2 en = ent[k];
      const int32_t c = col_state[en.x];
      if (c > lower && c <= medium) acc = __fadd_rn(acc, __int_as_float(en.y));
    }
    expo[i + (int64_t)r * n] = acc;
  }
}

// Geometric mode: exact int64 contact-second sums.
__global__ void __launch_bounds__(256)
    k_spmv_geometric(const int32_t *__restrict__ row_ptr, const int2 *__restrict__ ent,
                     const uint8_t *__restrict__ st, int64_t *__restrict__ expo,
                     int32_t n, int32_t m) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t beg = row_ptr[i], end = row_ptr[i + 1];
  for (int32_t r = blockIdx.y; r < m; r += gridDim.y) {
    const uint8_t *col_state = st + (int64_t)r * n;
    int64_t acc = 0;
    for (int32_t k = beg; k < end; ++k) {
      const int2 en = ent[k];
      if (col_state[en.x] == 2) acc += en.y;
    }
    expo[i + (int64_t)r * n] = acc;
  }
}

// Raw FP32 SpMV on a float infectious matrix (test hook).
__global__ void __launch_bounds__(256)
    k_spmv_raw(const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col,
               const float *__restrict__ val, const float *__restrict__ b,
               float *__restrict__ c, int32_t n, int32_t m) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int32_t r = blockIdx.y; r < m; r += gridDim.y) {
    const float *bc = b + (int64_t)r * n;
    float acc = 0.0f;
    for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
      acc = __fadd_rn(acc, __fmul_rn(val[k], bc[col[k]]));
    c[i + (int64_t)r * n] = acc;
  }
}

// ---- count reduction ------------------------------------------------------------
// Each thread holds classes of up to 4 replicas (a quad) of one node; the
// block (256 consecutive nodes, same quad) reduces 16 counters and adds them
// to counts_row[replica][slot], slot 0 E, 1 I, 2 R, 3 S.
__device__ __forceinline__ void reduce_quad_counts(const int cls[4], int32_t q, int32_t m,
                                                   int32_t *counts_row) {
  __shared__ int part[8][16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c4 = 0; c4 < 4; ++c4) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int v = __reduce_add_sync(kFull, cls[c4] == k ? 1 : 0);
      if (lane == 0) part[warp][c4 * 4 + k] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w][threadIdx.x];
    const int c4 = threadIdx.x >> 2, k = threadIdx.x & 3;
    const int32_t r = 4 * q + c4;
    const int slot = (k + 3) & 3;  // S->3, E->0, I->1, R->2
    if (r < m && s) atomicAdd(&counts_row[r * 4 + slot], s);
  }
}

// ---- transitions -------------------------------------------------------------
// Countdown mode, rules of compute_infection_probability (:113-135),
// monte_carlo_simulation (:137-159) and update_countdown_vector (:161-176)
// with the counter-based uniform of (seed, replica, node, step).
__global__ void __launch_bounds__(256)
    k_transition_countdown(int32_t *__restrict__ cd, const float *__restrict__ expo,
                           int32_t n, int32_t m, uint32_t step, StepConsts c,
                           int32_t *__restrict__ counts_row) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t q = blockIdx.y;
  int cls[4] = {-1, -1, -1, -1};
  if (i < n) {
    int32_t v[4];
    bool any_s = false;
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {
      const int32_t r = 4 * q + c4;
      v[c4] = r < m ? cd[i + (int64_t)r * n] : -1;
      any_s |= v[c4] == 0;
    }
    uint32_t x[4] = {0, 0, 0, 0};
    if (any_s)
      philox4x32_10((uint32_t)i, step, (uint32_t)q + (c.roff >> 2), kStreamInfect, c.key0, c.key1, x);
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {
      const int32_t r = 4 * q + c4;
      if (r >= m) continue;
      int32_t cv = v[c4];
      const int64_t idx = i + (int64_t)r * n;
      if (cv == 0) {
        const float e = __fdiv_rn(expo[idx], 3600.0f);
        const float P = one_minus_exp_neg(__fmul_rn(c.neg_log_base, e));
        if (P > unit24(x[c4])) cv = cd_add(c.upper, c.step_size);
      }
      if (cv > 0) cv = cd_sub(cv, c.step_size);
      if (cv < 0) cv = 0;
      if (cv != v[c4]) cd[idx] = cv;
      cls[c4] = countdown_class(cv, c.E, c.I, c.R);
    }
  }
  reduce_quad_counts(cls, q, m, counts_row);
}

__device__ __forceinline__ float infection_x(const StepConsts &c, int32_t r, int32_t i,
                                             int64_t e, float scale) {
  const float br = c.beta_r ? c.beta_r[r] : c.beta;
  const float bs = c.sus ? __fmul_rn(br, c.sus[i]) : br;
  float ef = __ll2float_rn(e);
  if (scale != 1.0f) ef = __fmul_rn(ef, scale);
  return __fmul_rn(bs, ef);
}

// Geometric mode: S->E with P = 1 - exp(-beta_r * s_i * exposure) against
// the replica's infection uniform; E->I, I->R (or I->S), R->S with fixed
// per-step probabilities against its bit-sliced flow uniform (flow_events on
// this quad's bits of the replica word).
__global__ void __launch_bounds__(256)
    k_transition_geometric(uint8_t *__restrict__ st, const int64_t *__restrict__ expo,
                           int32_t n, int32_t m, uint32_t step, float scale,
                           StepConsts c, int32_t *__restrict__ counts_row) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t q = blockIdx.y;
  int cls[4] = {-1, -1, -1, -1};
  if (i < n) {
    uint8_t v[4];
    int64_t e[4];
    uint32_t Em = 0, Im = 0, Rm = 0;
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {
      const int32_t r = 4 * q + c4;
      v[c4] = 0;
      e[c4] = 0;
      if (r < m) {
        const int64_t idx = i + (int64_t)r * n;
        v[c4] = st[idx];
        if (v[c4] == 0) e[c4] = expo[idx];
        const uint32_t bit = 1u << (r & 31);
        Em |= v[c4] == 1 ? bit : 0u;
        Im |= v[c4] == 2 ? bit : 0u;
        Rm |= v[c4] == 3 ? bit : 0u;
      }
    }
    const uint32_t word = (uint32_t)(q >> 3) + (c.roff >> 5);  // stream word of the replicas
    uint32_t pl[8];  // the word's infection planes, drawn once if needed
    bool have_pl = false;
    const uint32_t ev = (Em | Im | Rm)
                            ? flow_events(Em, Im, Rm, c.th, c.rk, (uint32_t)i, step, word)
                            : 0u;
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {
      const int32_t r = 4 * q + c4;
      if (r >= m) continue;
      uint8_t nv = v[c4];
      const bool fired = (ev >> (r & 31)) & 1u;
      if (v[c4] == 0) {
        if (e[c4] > 0) {
          const float P = one_minus_exp_neg(infection_x(c, r, i, e[c4], scale));
          if (P > 0.0f && P < 1.0f && !have_pl) {
            infect_planes(c.rk, (uint32_t)i, step, word, pl);
            have_pl = true;
          }
          const uint32_t u8 = have_pl ? top8_of(pl, (uint32_t)(r & 31)) : 0u;
          if (infect_event(P, u8, c.rk, (uint32_t)i, step, word * 32u + (uint32_t)(r & 31)))
            nv = c.has_exposed ? 1 : 2;
        }
      } else if (v[c4] == 1) {
        if (fired) nv = 2;
      } else if (v[c4] == 2) {
        if (fired) nv = c.ir_to_s ? 0 : 3;
      } else {
        if (fired) nv = 0;
      }
      if (nv != v[c4]) st[i + (int64_t)r * n] = nv;
      cls[c4] = nv;
    }
  }
  reduce_quad_counts(cls, q, m, counts_row);
}

// ---- initial state -----------------------------------------------------------
// Bernoulli(p0) per (node, replica) from stream 1 (initialize_countdown_vector,
// :73-90: infected start at medium + step, i.e. infectious after one step).
__global__ void __launch_bounds__(256)
    k_init(int transition, void *__restrict__ state, int32_t n, int32_t m, float p0,
           StepConsts c) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t q = blockIdx.y;
  if (i >= n) return;
  uint32_t x[4];
  philox4x32_10((uint32_t)i, kStepInit, (uint32_t)q + (c.roff >> 2), kStreamInit, c.key0, c.key1, x);
#pragma unroll
  for (int c4 = 0; c4 < 4; ++c4) {
    const int32_t r = 4 * q + c4;
    if (r >= m) continue;
    const bool inf = unit24(x[c4]) < p0;
    const int64_t idx = i + (int64_t)r * n;
    if (transition == RP_TRANSITION_COUNTDOWN)
      static_cast<int32_t *>(state)[idx] = inf ? cd_add(c.medium, c.step_size) : 0;
    else
      static_cast<uint8_t *>(state)[idx] = inf ? 2 : 0;
  }
}

// Exactly k distinct nodes per replica (Floyd's sampling) from stream 2.
// The state already holds zeros; a chosen node is non-zero.
__global__ void k_pick(int transition, void *__restrict__ state, int32_t n, int32_t m,
                       int32_t k, StepConsts c) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int32_t val = cd_add(c.medium, c.step_size);
  for (int32_t j = n - k; j < n; ++j) {
    uint32_t x[4];
    philox4x32_10((uint32_t)j, kStepPick, (uint32_t)r + c.roff, kStreamPick, c.key0, c.key1, x);
    const uint64_t r64 = (uint64_t)x[0] | ((uint64_t)x[1] << 32);
    const int32_t t = (int32_t)__umul64hi(r64, (uint64_t)(j + 1));
    int64_t idx = t + (int64_t)r * n;
    bool taken;
    if (transition == RP_TRANSITION_COUNTDOWN)
      taken = static_cast<int32_t *>(state)[idx] != 0;
    else
      taken = static_cast<uint8_t *>(state)[idx] != 0;
    if (taken) idx = j + (int64_t)r * n;
    if (transition == RP_TRANSITION_COUNTDOWN)
      static_cast<int32_t *>(state)[idx] = val;
    else
      static_cast<uint8_t *>(state)[idx] = 2;
  }
}

__global__ void __launch_bounds__(256)
    k_count(int transition, const void *__restrict__ state, int32_t n, int32_t m,
            StepConsts c, int32_t *__restrict__ counts_row) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t q = blockIdx.y;
  int cls[4] = {-1, -1, -1, -1};
  if (i < n) {
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {
      const int32_t r = 4 * q + c4;
      if (r >= m) continue;
      const int64_t idx = i + (int64_t)r * n;
      cls[c4] = transition == RP_TRANSITION_COUNTDOWN
                    ? countdown_class(static_cast<const int32_t *>(state)[idx], c.E, c.I, c.R)
                    : static_cast<const uint8_t *>(state)[idx];
    }
  }
  reduce_quad_counts(cls, q, m, counts_row);
}

__global__ void k_classify(int transition, const void *__restrict__ state, int32_t n,
                           int32_t m, StepConsts c, uint8_t *__restrict__ out) {
  const int64_t total = (int64_t)n * m;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    out[idx] = transition == RP_TRANSITION_COUNTDOWN
                   ? (uint8_t)countdown_class(static_cast<const int32_t *>(state)[idx], c.E,
                                              c.I, c.R)
                   : static_cast<const uint8_t *>(state)[idx];
  }
}

dim3 node_quad_grid(int32_t n, int32_t m) {
  return dim3((unsigned)((n + 255) / 256), (unsigned)((m + 3) / 4));
}

}  // namespace

void plain_init(int transition, void *state, int32_t n, int32_t m, float p0,
                int32_t k_exact, const StepConsts &c, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  k_init<<<node_quad_grid(n, m), 256, 0, st>>>(transition, state, n, m,
                                                k_exact > 0 ? 0.0f : p0, c);
  if (k_exact > 0) k_pick<<<(m + 127) / 128, 128, 0, st>>>(transition, state, n, m, k_exact, c);
}

void plain_spmv(int transition, const int32_t *row_ptr, const int2 *entries,
                const void *state, void *exposure, int32_t n, int32_t m,
                const StepConsts &c, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  dim3 grid((unsigned)((n + 255) / 256), (unsigned)(m < 65535 ? m : 65535));
  if (transition == RP_TRANSITION_COUNTDOWN)
    k_spmv_countdown<<<grid, 256, 0, st>>>(row_ptr, entries,
                                           static_cast<const int32_t *>(state),
                                           static_cast<float *>(exposure), n, m, c.lower,
                                           c.medium);
  else
    k_spmv_geometric<<<grid, 256, 0, st>>>(row_ptr, entries,
                                           static_cast<const uint8_t *>(state),
                                           static_cast<int64_t *>(exposure), n, m);
}

void plain_transition(int transition, void *state, const void *exposure, int32_t n,
                      int32_t m, uint32_t step, float scale, int32_t *counts_row,
                      const StepConsts &c, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  if (transition == RP_TRANSITION_COUNTDOWN)
    k_transition_countdown<<<node_quad_grid(n, m), 256, 0, st>>>(
        static_cast<int32_t *>(state), static_cast<const float *>(exposure), n, m, step, c,
        counts_row);
  else
    k_transition_geometric<<<node_quad_grid(n, m), 256, 0, st>>>(
        static_cast<uint8_t *>(state), static_cast<const int64_t *>(exposure), n, m, step,
        scale, c, counts_row);
}

void plain_count(int transition, const void *state, int32_t n, int32_t m,
                 int32_t *counts_row, const StepConsts &c, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  k_count<<<node_quad_grid(n, m), 256, 0, st>>>(transition, state, n, m, c, counts_row);
}

void plain_classify(int transition, const void *state, int32_t n, int32_t m,
                    uint8_t *out, const StepConsts &c, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  k_classify<<<1184, 256, 0, st>>>(transition, state, n, m, c, out);
}

void plain_spmv_f32_raw(const int32_t *row_ptr, const int32_t *col, const float *val,
                        int32_t n, const float *b, float *c, int32_t m, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  dim3 grid((unsigned)((n + 255) / 256), (unsigned)(m < 65535 ? m : 65535));
  k_spmv_raw<<<grid, 256, 0, st>>>(row_ptr, col, val, b, c, n, m);
}

}  // namespace rp
