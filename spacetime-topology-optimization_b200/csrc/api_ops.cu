// Stand-alone level operators of the multigrid module's public helpers, on caller
// vectors (FP64):
//   * the grid transfers of torch_mg._on_node_grid with _interp_axis / _restrict_axis
//     (sttopt/torch_mg.py:75-109): the x pass then the y pass, every dof component alike,
//     with no projection (the hierarchy's own transfers project);
//   * keff_matvec (sttopt/torch_mg.py:179-193), the apply of explicit per-element matrices
//     (U_e^T keff_e, as the reference contracts them), as a node-centric gather: node n
//     sums, over its (up to four) elements, the element's dof values times the matrix
//     columns of n's corner, so each column is read once and the sum needs no atomics
//     (deterministic).
#include "common.cuh"
#include "errors.h"
#include "mg.cuh"

namespace stt {

static int api_grid(long long n, int bs = 256) {
  long long g = (n + bs - 1) / bs;
  if (g > (1 << 30)) g = 1 << 30;
  return (int)(g < 1 ? 1 : g);
}

// out[s][n*D + i] = sum over elements e of n, corner q of n in e:
//   sum_j U[s][dof_j(e)] keff[s][e][j][q*D + i]
template <int D>
__global__ void keff_apply_kernel(const double* __restrict__ U, long long u_rs, const double* __restrict__ keff,
                                  long long k_rs, double* __restrict__ out, long long o_rs, int nelx, int nely) {
  constexpr int NK = 4 * D;
  const int nnx = nelx + 1;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= (long long)nnx * (nely + 1)) return;
  const int s = blockIdx.y;
  const int r = (int)(n / nnx), c = (int)(n - (long long)r * nnx);
  const double* us = U + (size_t)s * u_rs;
  const double* ks = keff + (size_t)s * k_rs;
  double acc[D];
#pragma unroll
  for (int i = 0; i < D; ++i) acc[i] = 0.0;
  // elements (r - 1 + a, c - 1 + b); n is their corner corner_of(a, b)
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int er = r - 1 + a, ec = c - 1 + b;
      if (er < 0 || er >= nely || ec < 0 || ec >= nelx) continue;
      const long long e = (long long)er * nelx + ec;
      const int q = corner_of(a, b);
      double ue[NK];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const long long node = (long long)(er + corner_dr(k)) * nnx + ec + corner_dc(k);
#pragma unroll
        for (int j = 0; j < D; ++j) ue[k * D + j] = __ldg(us + node * D + j);
      }
      // the reference contracts U_e with the matrix's first index: (U_e^T keff_e)[q D + i]
      const double* ke = ks + (size_t)e * NK * NK;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < NK; ++j) acc[i] = fma(ue[j], __ldg(ke + (size_t)j * NK + q * D + i), acc[i]);
    }
  double* os = out + (size_t)s * o_rs;
#pragma unroll
  for (int i = 0; i < D; ++i) os[n * D + i] = acc[i];
}

}  // namespace stt

using namespace stt;

extern "C" int stt_grid_transfer(int d, int kx, int ky, int cnnx, int cnny, int nrows, int restrict_,
                                 const double* in, long long in_rs, double* out, long long out_rs,
                                 stt_stream_t stream) {
  if ((d != 1 && d != 2) || kx < 1 || kx > 3 || ky < 1 || ky > 3 || cnnx < 1 || cnny < 1 || nrows <= 0 ||
      nrows > 65535 || !in || !out)
    return set_error(STT_ERR_INVALID, "stt_grid_transfer: bad arguments");
  if (d == 2 && ((((uintptr_t)in | (uintptr_t)out) & 15) || (in_rs & 1) || (out_rs & 1)))
    return set_error(STT_ERR_INVALID, "stt_grid_transfer: 2-dof vectors must be 16-byte aligned with even strides");
  const int fnnx = kx * (cnnx - 1) + 1, fnny = ky * (cnny - 1) + 1;
  cudaStream_t st = (cudaStream_t)stream;
  if (restrict_) {
    const dim3 g = coarse_grid(cnnx - 1, cnny - 1, nrows);
    if (d == 2)
      restrict_kernel<2, double><<<g, kQThreads, 0, st>>>(in, in_rs, fnnx, fnny, out, out_rs, cnnx, cnny, kx, ky,
                                                          nullptr, nullptr);
    else
      restrict_kernel<1, double><<<g, kQThreads, 0, st>>>(in, in_rs, fnnx, fnny, out, out_rs, cnnx, cnny, kx, ky,
                                                          nullptr, nullptr);
  } else {
    if (fnny > 65535) return set_error(STT_ERR_INVALID, "stt_grid_transfer: more than 65535 fine rows");
    // out = P in: zero, then the prolongation adds
    STT_TRY(check_cuda(cudaMemset2DAsync(out, out_rs * sizeof(double), 0, (size_t)d * fnnx * fnny * sizeof(double),
                                         nrows, st),
                       "zero out"));
    const dim3 g((fnnx + kProlongThreads - 1) / kProlongThreads, fnny, nrows);
    if (d == 2)
      prolong_kernel<2, double><<<g, kProlongThreads, 0, st>>>(in, in_rs, cnnx, cnny, out, out_rs, fnnx, fnny, kx,
                                                               ky, nullptr, nullptr);
    else
      prolong_kernel<1, double><<<g, kProlongThreads, 0, st>>>(in, in_rs, cnnx, cnny, out, out_rs, fnnx, fnny, kx,
                                                               ky, nullptr, nullptr);
  }
  return check_launch("grid transfer");
}

extern "C" int stt_keff_apply(int d, int nelx, int nely, int nrows, const double* U, long long u_rs,
                              const double* keff, long long k_rs, double* out, long long o_rs, stt_stream_t stream) {
  if ((d != 1 && d != 2) || nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !U || !keff || !out)
    return set_error(STT_ERR_INVALID, "stt_keff_apply: bad arguments");
  const long long nnode = (long long)(nelx + 1) * (nely + 1);
  const dim3 g(api_grid(nnode), nrows);
  if (d == 2)
    keff_apply_kernel<2><<<g, 256, 0, (cudaStream_t)stream>>>(U, u_rs, keff, k_rs, out, o_rs, nelx, nely);
  else
    keff_apply_kernel<1><<<g, 256, 0, (cudaStream_t)stream>>>(U, u_rs, keff, k_rs, out, o_rs, nelx, nely);
  return check_launch("keff apply");
}
