// Expected-value (individual-based mean-field) replay and its adjoint.
//
// Same per-step window CSRs as the Monte Carlo replay (int32 contact-second
// weights w_ij, weight scale 1/steps-in-window), FP32 node probabilities
// x = (S, E, I, R), four planes of N floats.  One step t, with
// e_i = scale_t * sum_j w_ij I_j and P_i = 1 - exp(-beta s_i e_i):
//   new_i = S_i P_i                     (to E, or to I without an exposed state)
//   S' = S (1 - P) + p_rs R [+ p_ir I when I -> S]
//   E' = E (1 - p_ei) + new             (exposed state only)
//   I' = I (1 - p_ir) + p_ei E          (+ new without an exposed state)
//   R' = R (1 - p_rs) [+ p_ir I when I -> R]
// and the step's expected incidence is sum_i new_i.  This is the
// expectation of the geometric Monte Carlo step with every indicator
// replaced by its probability (p_S <- p_S exp(-beta s_i sum_j w_ij p_I,j)).
//
// The adjoint runs backwards over the same CSRs: with y = dL/dx_{t+1} and
// g_t = dL/dincidence_t, u_i = y_X,i - y_S,i + g_t (X the infection target),
//   dL/dS_i = y_S + P u,  dL/dE_i = y_E + p_ei (y_I - y_E),
//   dL/dR_i = y_R + p_rs (y_S - y_R),
//   dL/dI_j = y_I + p_ir (y_Y - y_I) + sum_i w_ij z_i,
//   z_i = scale S_i u_i exp(-beta s_i e_i) beta s_i
// (the transpose SpMV is the same CSR: the window graph is symmetric), and
// the parameter gradients
//   dL/dbeta += sum_i S u q s e,  dL/ds_i += S u q beta e,
//   dL/dp_ei += sum E (y_I - y_E), dL/dp_ir += sum I (y_Y - y_I),
//   dL/dp_rs += sum R (y_S - y_R).
// One kernel per reverse step finishes dL/dx_t of a row (gather of z_t over
// its neighbours) and immediately takes the local part of step t-1 for the
// same row.  Scalar gradients accumulate in FP64, per block, in fixed order.
// The kernels read the rates from device memory, so that the host captures
// a whole forward (and a whole adjoint) once as a CUDA graph and replays it
// for any beta and rates.
#include "rp_device.cuh"
#include "rp_internal.h"

namespace rp {
namespace {

constexpr int kMfThreads = 256;

template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  T t = 0;
  if (warp == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xFFFFFFFFu, t, o);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

__device__ __forceinline__ float row_exposure(const int32_t *__restrict__ rp,
                                              const int2 *__restrict__ ent,
                                              const float *__restrict__ v, int32_t i) {
  float e = 0.0f;
  const int32_t b = rp[i], en = rp[i + 1];
  for (int32_t k = b; k < en; ++k) {
    const int2 q = ent[k];
    e = fmaf((float)q.y, v[q.x], e);
  }
  return e;
}

__global__ void __launch_bounds__(kMfThreads)
    k_mf_step(const int32_t *__restrict__ rp, const int2 *__restrict__ ent, int32_t n, float scale,
              const MfRates *__restrict__ rates, const float *__restrict__ sus, const float *__restrict__ x,
              float *__restrict__ xo, float *__restrict__ q_out, float *__restrict__ e_out,
              float *__restrict__ inc_part) {
  __shared__ float sh[32];
  const MfRates r = *rates;
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float newinf = 0.0f;
  if (i < n) {
    const float S = x[i], E = x[n + i], I = x[2 * (size_t)n + i], R = x[3 * (size_t)n + i];
    const float es = row_exposure(rp, ent, x + 2 * (size_t)n, i) * scale;
    const float si = sus ? sus[i] : 1.0f;
    const float a = r.beta * si * es;
    const float P = -expm1f(-a), q = expf(-a);
    newinf = S * P;
    const float f_ei = r.has_exposed ? E * r.p_ei : 0.0f;
    const float f_i = I * r.p_ir, f_rs = R * r.p_rs;
    float S2 = S * q + f_rs, E2 = E - f_ei, I2 = I - f_i + f_ei, R2 = R - f_rs;
    if (r.has_exposed) E2 += newinf; else I2 += newinf;
    if (r.ir_to_s) S2 += f_i; else R2 += f_i;
    xo[i] = S2;
    xo[n + i] = E2;
    xo[2 * (size_t)n + i] = I2;
    xo[3 * (size_t)n + i] = R2;
    if (q_out) q_out[i] = q;
    if (e_out) e_out[i] = es;
  }
  const float tot = block_sum(newinf, sh);
  if (threadIdx.x == 0) inc_part[blockIdx.x] = tot;
}

// Incidence of each step: sum of the step's block partials, in block order.
__global__ void k_mf_incidence(const float *__restrict__ part, int32_t nblk, int32_t T,
                               float *__restrict__ inc) {
  const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  float s = 0.0f;
  for (int32_t b = 0; b < nblk; ++b) s += part[(size_t)t * nblk + b];
  inc[t] = s;
}

// One reverse step.  Coupling part (when rp_c != nullptr): the full adjoint
// of x_tc is a_loc + (0, 0, sum_j w_ij z_j, 0).  Local part (when x != nullptr):
// from that adjoint y (of x_{tl+1}) and the step tl data, the local adjoint
// of x_tl goes to a_out and z_tl to z_out; parameter gradients accumulate.
// Without a local part the full adjoint goes to a_out.
__global__ void __launch_bounds__(kMfThreads)
    k_mf_adjoint(int32_t n, const int32_t *__restrict__ rp_c, const int2 *__restrict__ ent_c,
                 const float *__restrict__ z_in, const float *__restrict__ a_in,
                 const float *__restrict__ x, const float *__restrict__ qv,
                 const float *__restrict__ ev, const float *__restrict__ ginc, int32_t tl,
                 float scale, const MfRates *__restrict__ rates,
                 const float *__restrict__ sus,
                 float *__restrict__ a_out, float *__restrict__ z_out, float *__restrict__ gsus,
                 double *__restrict__ gpart) {
  __shared__ double sh[32];
  const MfRates r = *rates;
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double gb = 0.0, ge = 0.0, gi = 0.0, gr = 0.0;
  if (i < n) {
    const float yS = a_in[i], yE = a_in[n + i], yR = a_in[3 * (size_t)n + i];
    float yI = a_in[2 * (size_t)n + i];
    if (rp_c) yI += row_exposure(rp_c, ent_c, z_in, i);
    if (!x) {
      a_out[i] = yS;
      a_out[n + i] = yE;
      a_out[2 * (size_t)n + i] = yI;
      a_out[3 * (size_t)n + i] = yR;
    } else {
      const float S = x[i], E = x[n + i], I = x[2 * (size_t)n + i], R = x[3 * (size_t)n + i];
      const float q = qv[i], P = 1.0f - q, es = ev[i];
      const float si = sus ? sus[i] : 1.0f;
      const float yX = r.has_exposed ? yE : yI;
      const float yY = r.ir_to_s ? yS : yR;
      const float g = ginc ? ginc[tl] : 0.0f;  // dL/dincidence of step tl
      const float u = yX - yS + g;
      const float suq = S * u * q;
      a_out[i] = yS + P * u;
      a_out[n + i] = r.has_exposed ? yE + r.p_ei * (yI - yE) : yE;
      a_out[2 * (size_t)n + i] = yI + r.p_ir * (yY - yI);
      a_out[3 * (size_t)n + i] = yR + r.p_rs * (yS - yR);
      // d(es_i)/dI_j = scale w_ij, so z_i = scale * S u q beta s_i
      z_out[i] = suq * r.beta * si * scale;
      if (gsus) gsus[i] += suq * r.beta * es;
      gb = (double)suq * (double)si * (double)es;
      if (r.has_exposed) ge = (double)E * ((double)yI - (double)yE);
      gi = (double)I * ((double)yY - (double)yI);
      gr = (double)R * ((double)yS - (double)yR);
    }
  }
  if (!x) return;
  const double tb = block_sum(gb, sh);
  const double te = block_sum(ge, sh);
  const double ti = block_sum(gi, sh);
  const double tr = block_sum(gr, sh);
  if (threadIdx.x == 0) {
    double *p = gpart + 4 * (size_t)blockIdx.x;
    p[0] += tb;
    p[1] += te;
    p[2] += ti;
    p[3] += tr;
  }
}

__global__ void k_mf_finish(const double *__restrict__ gpart, int32_t nblk,
                            double *__restrict__ out) {
  const int k = threadIdx.x;
  if (k >= 4) return;
  double s = 0.0;
  for (int32_t b = 0; b < nblk; ++b) s += gpart[4 * (size_t)b + k];
  out[k] = s;
}

}  // namespace

int32_t mf_blocks(int32_t n) { return (n + kMfThreads - 1) / kMfThreads; }

void mf_step(const int32_t *rp, const int2 *ent, int32_t n, float scale, const MfRates *r,
             const float *sus, const float *x, float *xo, float *q_out, float *e_out,
             float *inc_part, cudaStream_t st) {
  k_mf_step<<<mf_blocks(n), kMfThreads, 0, st>>>(rp, ent, n, scale, r, sus, x, xo, q_out, e_out,
                                                inc_part);
}

void mf_incidence(const float *part, int32_t nblk, int32_t T, float *inc, cudaStream_t st) {
  if (T <= 0) return;
  k_mf_incidence<<<(T + 127) / 128, 128, 0, st>>>(part, nblk, T, inc);
}

void mf_adjoint(int32_t n, const int32_t *rp_c, const int2 *ent_c, const float *z_in,
                const float *a_in, const float *x, const float *q, const float *e,
                const float *ginc, int32_t tl, float scale, const MfRates *r, const float *sus,
                float *a_out, float *z_out, float *gsus, double *gpart, cudaStream_t st) {
  k_mf_adjoint<<<mf_blocks(n), kMfThreads, 0, st>>>(n, rp_c, ent_c, z_in, a_in, x, q, e, ginc, tl,
                                                   scale, r, sus, a_out, z_out, gsus, gpart);
}

void mf_finish(const double *gpart, int32_t nblk, double *out, cudaStream_t st) {
  k_mf_finish<<<1, 32, 0, st>>>(gpart, nblk, out);
}

}  // namespace rp
