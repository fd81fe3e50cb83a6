// Element terms of the adjoint (FemSolve.backward, sttopt/torch_solve.py:144-152), the
// element strain energy (compliance._element_strain_energy, sttopt/compliance.py:49-59),
// the space-time stage glue with a hard stage threshold (compliance._gravity_load and
// batched_whole_and_gravity_compliance, sttopt/compliance.py:137-161,198-253; gravity
// load matrix sttopt/gravity.py:15-36), the virtual-heat element means
// (sttopt/virtual_heat.py:162-166) and the PCG vector steps for arbitrary operators.
#include <algorithm>

#include <cooperative_groups.h>

#include "common.cuh"
#include "errors.h"
#include "modal.h"

namespace cg = cooperative_groups;

namespace stt {

static int grid1(long long n, int bs = 256) {
  long long g = (n + bs - 1) / bs;
  if (g > (1 << 30)) g = 1 << 30;
  return (int)(g < 1 ? 1 : g);
}

template <int D>
struct KEd {
  double v[16 * D * D];
};

// Element e's dofs in the reference's local order (BL, BR, TR, TL; d interleaved).
template <int D>
STT_DEV void element_dofs(int e, int nelx, long long (&dofs)[4 * D]) {
  const int er = e / nelx, ec = e - er * nelx;
  const int nnx = nelx + 1;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long node = (long long)(er + corner_dr(q)) * nnx + ec + corner_dc(q);
#pragma unroll
    for (int i = 0; i < D; ++i) dofs[q * D + i] = node * D + i;
  }
}

template <int D>
__global__ void element_sens_kernel(const double* __restrict__ U, long long U_rs,
                                    const double* __restrict__ lam, long long lam_rs,
                                    double* __restrict__ ce, double* __restrict__ gd,
                                    double* __restrict__ gr, long long e_rs, int nelx, int nel,
                                    KEd<D> ke) {
  constexpr int NK = 4 * D;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= nel) return;
  long long dofs[NK];
  element_dofs<D>(e, nelx, dofs);
  double u[NK], l[NK];
  const double* Us = U + (size_t)s * U_rs;
#pragma unroll
  for (int k = 0; k < NK; ++k) u[k] = __ldg(Us + dofs[k]);
  if (lam) {
    const double* ls = lam + (size_t)s * lam_rs;
#pragma unroll
    for (int k = 0; k < NK; ++k) l[k] = __ldg(ls + dofs[k]);
  }
  // (Ue @ KE)[col] and (lam_e @ KE)[col]
  double c = 0.0, g = 0.0, q = 0.0;
#pragma unroll
  for (int col = 0; col < NK; ++col) {
    double uk = 0.0, lk = 0.0;
#pragma unroll
    for (int row = 0; row < NK; ++row) {
      uk = fma(u[row], ke.v[row * NK + col], uk);
      if (lam) lk = fma(l[row], ke.v[row * NK + col], lk);
    }
    c = fma(uk, u[col], c);
    if (lam) {
      g = fma(lk, u[col], g);
      q = fma(l[col], u[col], q);
    }
  }
  const size_t o = (size_t)s * e_rs + e;
  if (ce) ce[o] = c;
  if (gd) gd[o] = -g;
  if (gr) gr[o] = -q / 4;
}

__global__ void stage_membership_kernel(const double* __restrict__ t, int nel, int n_stage,
                                        uint8_t* __restrict__ member) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  const double te = t[e];
  for (int s = 0; s < n_stage; ++s) member[(size_t)s * nel + e] = te <= (double)(s + 1) / n_stage ? 1 : 0;
}

STT_DEV double simp_pow(double x, double p) { return p == 3.0 ? x * x * x : pow(x, p); }

// One thread per (node, stage): density rows of the elements handled by this node's
// top-left role, and the y load of the node.
__global__ void stage_rho_kernel(const double* __restrict__ x, const uint8_t* __restrict__ member,
                                 int nel, int n_stage, double Emin, double Emax, double penal,
                                 double* __restrict__ rho) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= nel) return;
  const double xt = x[e] * (double)member[(size_t)s * nel + e];
  rho[(size_t)s * nel + e] = Emin + simp_pow(xt, penal) * (Emax - Emin);
}

__global__ void stage_load_kernel(const double* __restrict__ x, const uint8_t* __restrict__ member,
                                  int nelx, int nely, const uint8_t* __restrict__ fixed,
                                  double* __restrict__ F) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (n >= nnx * nny) return;
  const int r = n / nnx, c = n - r * nnx;
  const int nel = nelx * nely;
  const double fe4 = (1.0 / ((double)nelx * nely)) / 4;
  // elements around the node in ascending element index (the CSR column order)
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int er = r - 1 + a, ec = c - 1 + b;
      if (er < 0 || er >= nely || ec < 0 || ec >= nelx) continue;
      const int e = er * nelx + ec;
      const double xt = x[e] * (double)member[(size_t)s * nel + e];
      acc += fe4 * xt;
    }
  double* Fs = F + (size_t)s * 2 * nnx * nny;
  const uint8_t fl = fixed ? fixed[n] : 0;
  Fs[2 * (size_t)n] = 0.0;
  Fs[2 * (size_t)n + 1] = (fl & 2) ? 0.0 : -acc;
}

__global__ void stage_gradient_kernel(const double* __restrict__ x, const uint8_t* __restrict__ member,
                                      const double* __restrict__ ce, const double* __restrict__ gd,
                                      const double* __restrict__ gF, int nelx, int nely, int n_stage,
                                      double Emin, double Emax, double penal, double* __restrict__ grad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int nel = nelx * nely;
  if (e >= nel) return;
  const int er = e / nelx, ec = e - er * nelx, nnx = nelx + 1;
  const long long nnode = (long long)nnx * (nely + 1);
  const double fe4 = (1.0 / ((double)nelx * nely)) / 4;
  double acc = 0.0;
  for (int s = 0; s < n_stage; ++s) {
    if (!member[(size_t)s * nel + e]) continue;
    const double xt = x[e];
    const double dsimp = penal * (penal == 3.0 ? xt * xt : pow(xt, penal - 1)) * (Emax - Emin);
    const size_t o = (size_t)s * nel + e;
    double load = 0.0;
    const double* g = gF + (size_t)s * 2 * nnode;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long node = (long long)(er + corner_dr(q)) * nnx + ec + corner_dc(q);
      load += g[2 * node + 1];
    }
    acc += (ce[o] + gd[o]) * dsimp - fe4 * load;
  }
  grad[e] += acc;
}

__global__ void heat_means_kernel(const double* __restrict__ T, int nelx, int nel, double* __restrict__ te) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  long long dofs[4];
  element_dofs<1>(e, nelx, dofs);
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) s += 1.0 - T[dofs[q]];
  te[e] = s / 4;
}

__global__ void heat_adjoint_load_kernel(const double* __restrict__ w, double scale, int nelx, int nely,
                                         double* __restrict__ g) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nnx * nny) return;
  const int r = n / nnx, c = n - r * nnx;
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int er = r - 1 + a, ec = c - 1 + b;
      if (er < 0 || er >= nely || ec < 0 || ec >= nelx) continue;
      acc += (w[er * nelx + ec] / scale) / 4;
    }
  g[n] = -acc;
}

// ce and gdens of plane-stress elements whose KE has the modal form KE = T^T M T (the
// level-0 kernels' edge modes Gx, Gy, H per component): U^T KE U = (T U) . M (T U), about
// 20 flops an element instead of the 8 x 8 product.  A warp marches down a strip of 31
// element columns (lane c holds node column c, the right neighbour's values come by
// shuffle), a row of nodes loaded once and coalesced per step; ce / gdens stores are
// coalesced.  Grid: (strips / 4, bands, rows).
struct ModalE {
  double m00, m01, m11, m22, m44, m55;
};

constexpr int kSensCols = 31;

STT_DEV void modal_modes(const double (&t)[2], const double (&b)[2], double (&md)[6]) {
  // t, b: this lane's top / bottom node; the right neighbour's by shuffle
  double tr[2], br[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    tr[d] = __shfl_down_sync(0xffffffffu, t[d], 1);
    br[d] = __shfl_down_sync(0xffffffffu, b[d], 1);
  }
  double Gx[2], Gy[2], H[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const double dB = br[d] - b[d], dT = tr[d] - t[d];
    Gx[d] = dB + dT;
    Gy[d] = (t[d] + tr[d]) - (b[d] + br[d]);
    H[d] = dT - dB;
  }
  md[0] = Gx[0];
  md[1] = Gy[1];
  md[2] = Gy[0] + Gx[1];  // the shear pair enters M once
  md[3] = H[0];
  md[4] = H[1];
  md[5] = 0.0;
}

template <bool LAM>
__global__ void __launch_bounds__(128) element_sens_modal_kernel(
    const double* __restrict__ U, long long U_rs, const double* __restrict__ lam, long long lam_rs,
    double* __restrict__ ce, double* __restrict__ gdens, double* __restrict__ greac, long long e_rs, int nelx,
    int nely, ModalE q) {
  const int s = blockIdx.z;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * 4 + warp;
  const int c = strip * kSensCols + lane;  // node column; element column when lane < 31
  const int nnx = nelx + 1;
  const bool col_ok = c < nnx;
  const bool el_ok = lane < kSensCols && c < nelx;
  const int band = (nely + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * band, r1 = min(r0 + band, nely);
  if (r0 >= r1) return;
  const double* us = U + (size_t)s * U_rs;
  const double* ls = LAM ? lam + (size_t)s * lam_rs : nullptr;
  auto load = [&](const double* v, int r, double(&o)[2]) {
    o[0] = o[1] = 0.0;
    if (col_ok) {
      const double2 t = __ldg(reinterpret_cast<const double2*>(v) + (size_t)r * nnx + c);
      o[0] = t.x;
      o[1] = t.y;
    }
  };
  double ut[2], lt[2] = {0.0, 0.0};
  load(us, r0, ut);
  if (LAM) load(ls, r0, lt);
  for (int r = r0; r < r1; ++r) {
    double ub[2], lb[2] = {0.0, 0.0};
    load(us, r + 1, ub);
    if (LAM) load(ls, r + 1, lb);
    double mu[6];
    modal_modes(ut, ub, mu);
    // q = M (T u): normal pair, shear, hourglass
    const double q0 = fma(q.m01, mu[1], q.m00 * mu[0]);
    const double q1 = fma(q.m01, mu[0], q.m11 * mu[1]);
    const double q2 = q.m22 * mu[2], q3 = q.m44 * mu[3], q4 = q.m55 * mu[4];
    const size_t e = (size_t)s * e_rs + (size_t)r * nelx + c;
    if (ce && el_ok) ce[e] = mu[0] * q0 + mu[1] * q1 + mu[2] * q2 + mu[3] * q3 + mu[4] * q4;
    if (LAM) {
      double ml[6];
      modal_modes(lt, lb, ml);
      if (gdens && el_ok) gdens[e] = -(ml[0] * q0 + ml[1] * q1 + ml[2] * q2 + ml[3] * q3 + ml[4] * q4);
      if (greac) {  // -lam_e . U_e / 4: this node column's two nodes and the right neighbour's
        const double pl = fma(ut[0], lt[0], fma(ut[1], lt[1], fma(ub[0], lb[0], ub[1] * lb[1])));
        const double pr = __shfl_down_sync(0xffffffffu, pl, 1);
        if (el_ok) greac[e] = -(pl + pr) * 0.25;
      }
#pragma unroll
      for (int d = 0; d < 2; ++d) lt[d] = lb[d];
    }
#pragma unroll
    for (int d = 0; d < 2; ++d) ut[d] = ub[d];
  }
}

// ---- PCG vector steps (arbitrary operator path) -----------------------------------

// Dot products of up to three vector pairs per row.  One thread-block cluster of
// kDotCluster CTAs per row: each CTA reduces a fixed contiguous chunk in a fixed order,
// and CTA 0 of the cluster sums the CTAs' partials in rank order through distributed
// shared memory -- deterministic, and no global scratch.
constexpr int kDotCluster = 8;
constexpr int kDotThreads = 512;

// K pairs, U strided loads of each in flight per thread (U kDotThreads apart): the
// accumulators are summed in a fixed order, so the result stays deterministic.
template <int K>
__global__ void __cluster_dims__(kDotCluster, 1, 1) __launch_bounds__(kDotThreads)
    vec_dots_kernel(long long n, const double* __restrict__ a0, const double* __restrict__ b0,
                    const double* __restrict__ a1, const double* __restrict__ b1,
                    const double* __restrict__ a2, const double* __restrict__ b2, long long rs,
                    double* __restrict__ dots) {
  constexpr int U = 4;
  __shared__ double scratch[kDotThreads / 32];
  __shared__ double part[3];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int s = blockIdx.y;
  const long long lo = n * rank / kDotCluster, hi = n * (rank + 1) / kDotCluster;
  const double* A[3] = {a0 + (size_t)s * rs, K > 1 ? a1 + (size_t)s * rs : nullptr,
                        K > 2 ? a2 + (size_t)s * rs : nullptr};
  const double* Bv[3] = {b0 + (size_t)s * rs, K > 1 ? b1 + (size_t)s * rs : nullptr,
                         K > 2 ? b2 + (size_t)s * rs : nullptr};
  // one pair after the other (a pass over each pair's chunk), U loads of each in flight
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double acc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) acc[u] = 0.0;
    long long i = lo + threadIdx.x;
    for (; i + (U - 1) * kDotThreads < hi; i += U * kDotThreads) {
      double va[U], vb[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        va[u] = __ldg(A[j] + i + u * kDotThreads);
        vb[u] = __ldg(Bv[j] + i + u * kDotThreads);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) acc[u] = fma(va[u], vb[u], acc[u]);
    }
    for (; i < hi; i += kDotThreads) acc[0] = fma(__ldg(A[j] + i), __ldg(Bv[j] + i), acc[0]);
    const double t = block_sum<kDotThreads>((acc[0] + acc[1]) + (acc[2] + acc[3]), scratch);
    if (threadIdx.x == 0) part[j] = t;
  }
  cluster.sync();
  if (rank == 0 && threadIdx.x < K) {
    double t = 0.0;
    for (int r = 0; r < kDotCluster; ++r) t += cluster.map_shared_rank(part, r)[threadIdx.x];
    dots[(size_t)s * K + threadIdx.x] = t;
  }
  cluster.sync();
}

// The two dots a.b0 and a.b1 of one first operand (k = 2, a0 == a1: U.gK and U.F of the
// stage adjoint's warm start, and the heat adjoint's) in one pass over a: 128-bit loads of
// the three vectors, U pairs in flight per thread (every row 16-byte aligned: an even
// stride or a single row; an odd length's last value is added by one fixed thread); the
// accumulators are summed in a fixed order, so the result stays deterministic.
__global__ void __cluster_dims__(kDotCluster, 1, 1) __launch_bounds__(kDotThreads)
    vec_dots_shared_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b0,
                           const double* __restrict__ b1, long long rs, double* __restrict__ dots) {
  constexpr int U = 4;
  __shared__ double scratch[kDotThreads / 32];
  __shared__ double part[2];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int s = blockIdx.y;
  const long long n2 = n / 2;
  const long long lo = n2 * rank / kDotCluster, hi = n2 * (rank + 1) / kDotCluster;
  const double2* A = reinterpret_cast<const double2*>(a + (size_t)s * rs);
  const double2* B0 = reinterpret_cast<const double2*>(b0 + (size_t)s * rs);
  const double2* B1 = reinterpret_cast<const double2*>(b1 + (size_t)s * rs);
  double acc0[U], acc1[U];
#pragma unroll
  for (int u = 0; u < U; ++u) acc0[u] = acc1[u] = 0.0;
  long long i = lo + threadIdx.x;
  for (; i + (U - 1) * kDotThreads < hi; i += U * kDotThreads) {
    double2 va[U], v0[U], v1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      va[u] = __ldg(A + i + u * kDotThreads);
      v0[u] = __ldg(B0 + i + u * kDotThreads);
      v1[u] = __ldg(B1 + i + u * kDotThreads);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      acc0[u] = fma(va[u].y, v0[u].y, fma(va[u].x, v0[u].x, acc0[u]));
      acc1[u] = fma(va[u].y, v1[u].y, fma(va[u].x, v1[u].x, acc1[u]));
    }
  }
  for (; i < hi; i += kDotThreads) {
    const double2 va = __ldg(A + i), v0 = __ldg(B0 + i), v1 = __ldg(B1 + i);
    acc0[0] = fma(va.y, v0.y, fma(va.x, v0.x, acc0[0]));
    acc1[0] = fma(va.y, v1.y, fma(va.x, v1.x, acc1[0]));
  }
  if ((n & 1) && rank == 0 && threadIdx.x == 0) {
    const size_t last = (size_t)s * rs + n - 1;
    acc0[0] = fma(__ldg(a + last), __ldg(b0 + last), acc0[0]);
    acc1[0] = fma(__ldg(a + last), __ldg(b1 + last), acc1[0]);
  }
  const double t0 = block_sum<kDotThreads>((acc0[0] + acc0[1]) + (acc0[2] + acc0[3]), scratch);
  if (threadIdx.x == 0) part[0] = t0;
  const double t1 = block_sum<kDotThreads>((acc1[0] + acc1[1]) + (acc1[2] + acc1[3]), scratch);
  if (threadIdx.x == 0) part[1] = t1;
  cluster.sync();
  if (rank == 0 && threadIdx.x < 2) {
    double t = 0.0;
    for (int r = 0; r < kDotCluster; ++r) t += cluster.map_shared_rank(part, r)[threadIdx.x];
    dots[(size_t)s * 2 + threadIdx.x] = t;
  }
  cluster.sync();
}

__global__ void vec_cg_update_kernel(long long n, const double* __restrict__ alpha, double* __restrict__ x,
                                     double* __restrict__ r, const double* __restrict__ p,
                                     const double* __restrict__ Ap, long long rs, double* __restrict__ rr) {
  __shared__ double scratch[8];
  const int s = blockIdx.x;
  const double a = alpha[s];
  double acc = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const size_t o = (size_t)s * rs + i;
    x[o] = x[o] + a * p[o];
    const double rv = r[o] - a * Ap[o];
    r[o] = rv;
    acc = fma(rv, rv, acc);
  }
  acc = block_sum<256>(acc, scratch);
  if (threadIdx.x == 0) rr[s] = acc;
}

__global__ void vec_xpay_kernel(long long n, const double* __restrict__ z, const double* __restrict__ beta,
                                double* __restrict__ p, long long rs) {
  const int s = blockIdx.y;
  const double b = beta[s];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const size_t o = (size_t)s * rs + i;
    p[o] = p[o] * b + z[o];
  }
}

}  // namespace stt

using namespace stt;

extern "C" int stt_element_sens(int d, int nelx, int nely, int nrows, const double* U, long long U_rs,
                                const double* lam, long long lam_rs, const double* KE, double* ce,
                                double* gdens, double* greac, long long e_rs, stt_stream_t stream) {
  if (!U || !KE || nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || ((gdens || greac) && !lam))
    return set_error(STT_ERR_INVALID, "stt_element_sens: bad arguments");
  const int nel = nelx * nely;
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid(grid1(nel), nrows);
  double m[8];
  if (d == 2 && (((uintptr_t)U | (uintptr_t)lam) & 15) == 0 && (U_rs & 1) == 0 && (lam_rs & 1) == 0 &&
      modal_from_ke(2, KE, m)) {
    // the modal form: a column-marching pass (16-byte node loads need aligned rows)
    const int strips = (nelx + kSensCols - 1) / kSensCols;
    int band = 32;
    while (band > 4 && (long long)((strips + 3) / 4) * ((nely + band - 1) / band) * nrows < 4 * 148) band /= 2;
    const dim3 g((strips + 3) / 4, (nely + band - 1) / band, nrows);
    const ModalE q{m[0], m[1], m[2], m[3], m[4], m[5]};
    if (lam)
      element_sens_modal_kernel<true><<<g, 128, 0, st>>>(U, U_rs, lam, lam_rs, ce, gdens, greac, e_rs, nelx, nely,
                                                         q);
    else
      element_sens_modal_kernel<false><<<g, 128, 0, st>>>(U, U_rs, nullptr, 0, ce, nullptr, nullptr, e_rs, nelx,
                                                          nely, q);
  } else if (d == 2) {
    KEd<2> k;
    for (int i = 0; i < 64; ++i) k.v[i] = KE[i];
    element_sens_kernel<2><<<grid, 256, 0, st>>>(U, U_rs, lam, lam_rs, ce, gdens, greac, e_rs, nelx, nel, k);
  } else if (d == 1) {
    KEd<1> k;
    for (int i = 0; i < 16; ++i) k.v[i] = KE[i];
    element_sens_kernel<1><<<grid, 256, 0, st>>>(U, U_rs, lam, lam_rs, ce, gdens, greac, e_rs, nelx, nel, k);
  } else {
    return set_error(STT_ERR_INVALID, "stt_element_sens: d must be 1 or 2");
  }
  return check_launch("element_sens");
}

extern "C" int stt_stage_membership(int nel, int n_stage, const double* tPhys, uint8_t* member,
                                    stt_stream_t stream) {
  if (nel <= 0 || n_stage <= 0 || !tPhys || !member) return set_error(STT_ERR_INVALID, "stt_stage_membership: bad arguments");
  stage_membership_kernel<<<grid1(nel), 256, 0, (cudaStream_t)stream>>>(tPhys, nel, n_stage, member);
  return check_launch("stage_membership");
}

extern "C" int stt_stage_rows(int nelx, int nely, int n_stage, const double* x, const uint8_t* member,
                              double Emin, double Emax, double penal, const uint8_t* fixed, double* rho,
                              double* F, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || n_stage <= 0 || n_stage > 65535 || !x || !member)
    return set_error(STT_ERR_INVALID, "stt_stage_rows: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int nel = nelx * nely, nnode = (nelx + 1) * (nely + 1);
  if (rho) stage_rho_kernel<<<dim3(grid1(nel), n_stage), 256, 0, st>>>(x, member, nel, n_stage, Emin, Emax, penal, rho);
  if (F) stage_load_kernel<<<dim3(grid1(nnode), n_stage), 256, 0, st>>>(x, member, nelx, nely, fixed, F);
  return check_launch("stage_rows");
}

extern "C" int stt_stage_gradient(int nelx, int nely, int n_stage, const double* x, const uint8_t* member,
                                  const double* ce, const double* gdens, const double* gF, double Emin,
                                  double Emax, double penal, double* grad, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || n_stage <= 0 || !x || !member || !ce || !gdens || !gF || !grad)
    return set_error(STT_ERR_INVALID, "stt_stage_gradient: bad arguments");
  stage_gradient_kernel<<<grid1(nelx * nely), 256, 0, (cudaStream_t)stream>>>(
      x, member, ce, gdens, gF, nelx, nely, n_stage, Emin, Emax, penal, grad);
  return check_launch("stage_gradient");
}

extern "C" int stt_heat_element_means(int nelx, int nely, const double* T, double* t_e, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || !T || !t_e) return set_error(STT_ERR_INVALID, "stt_heat_element_means: bad arguments");
  heat_means_kernel<<<grid1(nelx * nely), 256, 0, (cudaStream_t)stream>>>(T, nelx, nelx * nely, t_e);
  return check_launch("heat_means");
}

extern "C" int stt_heat_adjoint_load(int nelx, int nely, const double* w, double scale, double* g,
                                     stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || !w || !g) return set_error(STT_ERR_INVALID, "stt_heat_adjoint_load: bad arguments");
  heat_adjoint_load_kernel<<<grid1((nelx + 1) * (nely + 1)), 256, 0, (cudaStream_t)stream>>>(w, scale, nelx, nely, g);
  return check_launch("heat_adjoint_load");
}

extern "C" int stt_vec_dots(int nrows, long long n, const double* a0, const double* b0, const double* a1,
                            const double* b1, const double* a2, const double* b2, long long rs, double* dots,
                            stt_stream_t stream) {
  if (nrows <= 0 || n <= 0 || !a0 || !b0 || !dots) return set_error(STT_ERR_INVALID, "stt_vec_dots: bad arguments");
  if (nrows > 65535) return set_error(STT_ERR_INVALID, "stt_vec_dots: too many rows");
  const int k = (a1 && b1) ? ((a2 && b2) ? 3 : 2) : 1;
  const dim3 g(kDotCluster, nrows);
  cudaStream_t st = (cudaStream_t)stream;
  if (k == 2 && a0 == a1 && ((rs & 1) == 0 || nrows == 1) &&
      (((uintptr_t)a0 | (uintptr_t)b0 | (uintptr_t)b1) & 15) == 0) {
    vec_dots_shared_kernel<<<g, kDotThreads, 0, st>>>(n, a0, b0, b1, rs, dots);
    return check_launch("vec_dots");
  }
  if (k == 1)
    vec_dots_kernel<1><<<g, kDotThreads, 0, st>>>(n, a0, b0, a1, b1, a2, b2, rs, dots);
  else if (k == 2)
    vec_dots_kernel<2><<<g, kDotThreads, 0, st>>>(n, a0, b0, a1, b1, a2, b2, rs, dots);
  else
    vec_dots_kernel<3><<<g, kDotThreads, 0, st>>>(n, a0, b0, a1, b1, a2, b2, rs, dots);
  return check_launch("vec_dots");
}

extern "C" int stt_vec_cg_update(int nrows, long long n, const double* alpha, double* x, double* r,
                                 const double* p, const double* Ap, long long rs, double* rr,
                                 stt_stream_t stream) {
  if (nrows <= 0 || n <= 0 || !alpha || !x || !r || !p || !Ap || !rr)
    return set_error(STT_ERR_INVALID, "stt_vec_cg_update: bad arguments");
  vec_cg_update_kernel<<<nrows, 256, 0, (cudaStream_t)stream>>>(n, alpha, x, r, p, Ap, rs, rr);
  return check_launch("vec_cg_update");
}

extern "C" int stt_vec_xpay(int nrows, long long n, const double* z, const double* beta, double* p,
                            long long rs, stt_stream_t stream) {
  if (nrows <= 0 || n <= 0 || !z || !beta || !p) return set_error(STT_ERR_INVALID, "stt_vec_xpay: bad arguments");
  vec_xpay_kernel<<<dim3(std::min<long long>((n + 255) / 256, 1024), nrows), 256, 0, (cudaStream_t)stream>>>(n, z, beta, p, rs);
  return check_launch("vec_xpay");
}
