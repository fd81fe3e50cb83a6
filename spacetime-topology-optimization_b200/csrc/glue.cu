// The production loop's stage glue on the device, for any stage mask: the rows of the
// one batched whole + self-weight solve (compliance.batched_whole_and_gravity_compliance,
// _gravity_load and gravity_compliance, sttopt/compliance.py:137-253), with the smooth
// stage indicator time_mask (:33-46) evaluated in the kernel or a caller's mask rows,
// and the adjoint of those rows; the per-row SIMP-weighted strain energy reduction is
// stt_element_sens + stt_vec_dots.  Also the adjoint of the lumped reaction
// (sttopt/torch_fem.py:117-132).
//
// Row layout: with a whole-structure row (F0 != NULL / has_row0), row 0 is the whole
// structure and stage s is row s + 1; xt and the mask rows hold the stages only.
#include <cmath>

#include "common.cuh"
#include "errors.h"

namespace stt {

constexpr int kMaxGlueStages = 128;

// Per stage: the time ti, tanh(beta ti) and the denominator
// tanh(beta ti) + tanh(beta (1 - ti)), evaluated on the host as the reference does
// (math.tanh); only tanh(beta (t - ti)) depends on the element.
struct StageTimes {
  double ti[kMaxGlueStages];
  double a[kMaxGlueStages];
  double den[kMaxGlueStages];
};

STT_DEV double simp_pow_g(double x, double p) { return p == 3.0 ? x * x * x : pow(x, p); }
STT_DEV double simp_dpow(double x, double p) { return p == 3.0 ? 3.0 * (x * x) : p * pow(x, p - 1.0); }

// m = max(0, 1 - (a + tanh(beta (t - ti))) / den); the derivative passes where the
// unclamped value is >= 0 (torch.clamp's gradient mask).
STT_DEV double smooth_mask(double t, double beta, double ti, double a, double den, double* dmdt) {
  const double th = tanh(beta * (t - ti));
  const double v = 1.0 - (a + th) / den;
  if (dmdt) *dmdt = v >= 0.0 ? -beta * (1.0 - th * th) / den : 0.0;
  return v >= 0.0 ? v : 0.0;
}

// One thread per (element, row): row y < has_row0 is the whole structure.
__global__ void glue_rows_kernel(const double* __restrict__ x, const double* __restrict__ t,
                                 const double* __restrict__ M, double* __restrict__ M_out,
                                 double* __restrict__ xt_out, double* __restrict__ rho, int nel,
                                 int n_stage, int has_row0, double beta, double Emin, double Emax,
                                 double penal, const StageTimes st) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (e >= nel) return;
  const double xe = x[e];
  if (row < has_row0) {
    if (rho) rho[e] = Emin + simp_pow_g(xe, penal) * (Emax - Emin);
    return;
  }
  const int s = row - has_row0;
  const size_t o = (size_t)s * nel + e;
  const double m = M ? M[o] : smooth_mask(t[e], beta, st.ti[s], st.a[s], st.den[s], nullptr);
  if (M_out) M_out[o] = m;
  const double xte = xe * m;
  if (xt_out) xt_out[o] = xte;
  if (rho) rho[(size_t)row * nel + e] = Emin + simp_pow_g(xte, penal) * (Emax - Emin);
}

// One thread per (node, row): F[2n] = 0, F[2n+1] = -(fe/4) sum of xt over the node's
// elements (the self-weight, sttopt/gravity.py:15-36), row 0 a copy of F0.
__global__ void glue_load_kernel(const double* __restrict__ xt, const double* __restrict__ F0,
                                 double* __restrict__ F, int nelx, int nely, int has_row0) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (n >= nnx * nny) return;
  const long long ndof = 2LL * nnx * nny;
  double* Fr = F + (size_t)row * ndof;
  if (row < has_row0) {
    Fr[2 * (size_t)n] = F0[2 * (size_t)n];
    Fr[2 * (size_t)n + 1] = F0[2 * (size_t)n + 1];
    return;
  }
  const int nel = nelx * nely;
  const double* xs = xt + (size_t)(row - has_row0) * nel;
  const int r = n / nnx, c = n - r * nnx;
  const double fe4 = (1.0 / ((double)nelx * nely)) / 4;
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int er = r - 1 + a, ec = c - 1 + b;
      if (er < 0 || er >= nely || ec < 0 || ec >= nelx) continue;
      acc += fe4 * xs[er * nelx + ec];
    }
  Fr[2 * (size_t)n] = 0.0;
  Fr[2 * (size_t)n + 1] = -acc;
}

// One thread per element, looping over the stages: the gradient reaching a stage's xt
// (from xt itself, from its SIMP density row and from its self-weight load) is split
// into the x and mask (or t, for the smooth indicator) parts.
__global__ void glue_adjoint_kernel(const double* __restrict__ x, const double* __restrict__ t,
                                    const double* __restrict__ M, const double* __restrict__ g_xt,
                                    const double* __restrict__ g_rho, const double* __restrict__ g_F,
                                    int nelx, int nely, int n_stage, int has_row0, double beta,
                                    double Emin, double Emax, double penal, const StageTimes st,
                                    double* __restrict__ gx, double* __restrict__ gt,
                                    double* __restrict__ gM) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int nel = nelx * nely;
  if (e >= nel) return;
  const int er = e / nelx, ec = e - er * nelx, nnx = nelx + 1;
  const long long ndof = 2LL * nnx * (nely + 1);
  const double fe4 = (1.0 / ((double)nelx * nely)) / 4;
  const double xe = x[e];
  const double te = t ? t[e] : 0.0;
  const double dE = Emax - Emin;
  double ax = 0.0, at = 0.0;
  if (has_row0 && g_rho) ax += g_rho[e] * simp_dpow(xe, penal) * dE;
  for (int s = 0; s < n_stage; ++s) {
    const int row = s + has_row0;
    const size_t o = (size_t)s * nel + e;
    double dmdt = 0.0;
    const double m = t ? smooth_mask(te, beta, st.ti[s], st.a[s], st.den[s], gt ? &dmdt : nullptr) : M[o];
    const double xte = xe * m;
    double g = g_xt ? g_xt[o] : 0.0;
    if (g_rho) g += g_rho[(size_t)row * nel + e] * simp_dpow(xte, penal) * dE;
    if (g_F) {
      const double* gr = g_F + (size_t)row * ndof;
      double load = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long node = (long long)(er + corner_dr(q)) * nnx + ec + corner_dc(q);
        load += gr[2 * node + 1];
      }
      g -= fe4 * load;
    }
    ax += m * g;
    if (gt) at += xe * g * dmdt;
    if (gM) gM[o] = xe * g;
  }
  gx[e] = ax;
  if (gt) gt[e] = at;
}

// The adjoint of the lumped reaction: out[e] = (1/4) sum over e's corners and their d
// dofs of g (each element value reaches its 4 d dofs with weight 1/4).
template <int D>
__global__ void lumped_reaction_adjoint_kernel(const double* __restrict__ g, long long g_rs,
                                               double* __restrict__ out, long long o_rs, int nelx,
                                               int nely) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (e >= nelx * nely) return;
  const int er = e / nelx, ec = e - er * nelx, nnx = nelx + 1;
  const double* gr = g + (size_t)row * g_rs;
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long node = (long long)(er + corner_dr(q)) * nnx + ec + corner_dc(q);
#pragma unroll
    for (int i = 0; i < D; ++i) acc += gr[node * D + i];
  }
  out[(size_t)row * o_rs + e] = acc / 4;
}

static int grid_of(long long n) { return (int)((n + 255) / 256); }

static int fill_times(int n_stage, const double* times, double beta, StageTimes* st) {
  if (n_stage > kMaxGlueStages) return set_error(STT_ERR_INVALID, "stage glue: more than 128 stages");
  for (int s = 0; s < n_stage; ++s) {
    const double ti = times ? times[s] : 0.0;
    st->ti[s] = ti;
    st->a[s] = std::tanh(beta * ti);
    st->den[s] = std::tanh(beta * ti) + std::tanh(beta * (1.0 - ti));
  }
  return STT_OK;
}

}  // namespace stt

using namespace stt;

extern "C" int stt_stage_glue_rows(int nelx, int nely, int n_stage, int has_row0, const double* x,
                                   const double* t, const double* times, double beta, const double* M,
                                   double* M_out, const double* F0, double Emin, double Emax, double penal,
                                   double* xt, double* rho, double* F, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || n_stage < 0 || !x || (n_stage > 0 && !M && (!t || !times)) ||
      (F && n_stage > 0 && !xt) || (F && has_row0 && !F0))
    return set_error(STT_ERR_INVALID, "stt_stage_glue_rows: bad sizes or null pointer");
  has_row0 = has_row0 ? 1 : 0;
  const int rows = n_stage + has_row0;
  if (rows <= 0 || rows > 65535) return set_error(STT_ERR_INVALID, "stt_stage_glue_rows: bad row count");
  StageTimes st;
  STT_TRY(fill_times(M ? 0 : n_stage, times, beta, &st));
  const int nel = nelx * nely, nnode = (nelx + 1) * (nely + 1);
  cudaStream_t s = (cudaStream_t)stream;
  glue_rows_kernel<<<dim3(grid_of(nel), rows), 256, 0, s>>>(x, t, M, M_out, xt, rho, nel, n_stage, has_row0, beta,
                                                            Emin, Emax, penal, st);
  STT_TRY(check_launch("stage_glue_rows"));
  if (F) {
    glue_load_kernel<<<dim3(grid_of(nnode), rows), 256, 0, s>>>(xt, F0, F, nelx, nely, has_row0);
    STT_TRY(check_launch("stage_glue_load"));
  }
  return STT_OK;
}

extern "C" int stt_stage_glue_adjoint(int nelx, int nely, int n_stage, int has_row0, const double* x,
                                      const double* t, const double* times, double beta, const double* M,
                                      const double* g_xt, const double* g_rho, const double* g_F, double Emin,
                                      double Emax, double penal, double* gx, double* gt, double* gM,
                                      stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || n_stage < 0 || n_stage + has_row0 <= 0 || !x || !gx)
    return set_error(STT_ERR_INVALID, "stt_stage_glue_adjoint: bad sizes or null pointer");
  if ((gt && !t) || (t && !times) || (!t && n_stage > 0 && !M))
    return set_error(STT_ERR_INVALID, "stt_stage_glue_adjoint: the smooth mask needs t and times, else M");
  StageTimes st;
  STT_TRY(fill_times(t ? n_stage : 0, times, beta, &st));
  glue_adjoint_kernel<<<grid_of((long long)nelx * nely), 256, 0, (cudaStream_t)stream>>>(
      x, t, M, g_xt, g_rho, g_F, nelx, nely, n_stage, has_row0 ? 1 : 0, beta, Emin, Emax, penal, st, gx, gt, gM);
  return check_launch("stage_glue_adjoint");
}

extern "C" int stt_lumped_reaction_adjoint(int d, int nelx, int nely, int nrows, const double* g, long long g_rs,
                                           double* out, long long o_rs, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !g || !out)
    return set_error(STT_ERR_INVALID, "stt_lumped_reaction_adjoint: bad sizes or null pointer");
  dim3 grid(grid_of((long long)nelx * nely), nrows);
  cudaStream_t st = (cudaStream_t)stream;
  if (d == 2)
    lumped_reaction_adjoint_kernel<2><<<grid, 256, 0, st>>>(g, g_rs, out, o_rs, nelx, nely);
  else if (d == 1)
    lumped_reaction_adjoint_kernel<1><<<grid, 256, 0, st>>>(g, g_rs, out, o_rs, nelx, nely);
  else
    return set_error(STT_ERR_INVALID, "stt_lumped_reaction_adjoint: d must be 1 or 2");
  return check_launch("lumped_reaction_adjoint");
}
