// Shared device helpers for the sm_100a FEM solve kernels.
//
// Layout conventions (identical to the reference's tensors, so the Python boundary
// passes torch storage straight through):
//   node n = row * (nelx + 1) + col, row 0 at the top;
//   dof = d * n + i (d = 2 for plane stress, 1 for the scalar heat problem);
//   element e = row * nelx + col, local corners BL, BR, TR, TL.
// A "batch row" is one independent linear system; a "hierarchy row" is one operator
// (density field).  Several batch rows may share one hierarchy row (broadcast).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sttb200.h"

#define STT_DEV __device__ __forceinline__

namespace stt {

constexpr int kTX = 32;  // node tile width (threads in x)
constexpr int kTY = 8;   // node tile height (threads in y)
constexpr int kNT = kTX * kTY;

// Element matrix of the level-0 operator, carried in kernel parameter space so every
// access with a compile-time index is a uniform constant-bank load.
template <int D>
struct KEParam {
  double v[(4 * D) * (4 * D)];
};

// Per-batch-row PCG scalars, resident on the device for the whole solve.
struct RowState {
  double rz;          // r . z of the current iteration
  double rz_mix;      // r_new . z_old (flexible beta)
  double pAp;
  double alpha;
  double beta;
  double bnorm_safe;  // ||b|| or 1 where ||b|| == 0
  double rel;         // ||r|| / ||b||
  int active;         // 1 while the row iterates
  int conv_iter;      // iteration at which the row converged (-1 while active)
  int status;         // STT_OK, or STT_ERR_BREAKDOWN on a non-finite scalar
  int xpend;          // alpha p of the last update is not yet added to x
  int pbuf;           // which p buffer holds this row's last p (0 or 1)
  int conv;           // rel <= rtol at the last check (the reference's retirement schedule)
};

// Coefficients a node in an FP32 stored stencil (node-major): the 5 D^2 of the half
// stencil rounded up to a multiple of 4 (16-byte aligned node records).
template <int D>
__host__ __device__ constexpr int st32_nsp() {
  return (5 * D * D + 3) & ~3;
}

STT_DEV int hier_row(const int* row_map, int hrows, int s) {
  return row_map ? row_map[s] : (hrows == 1 ? 0 : s);
}

// Node (r, c)'s local corner index in the element (r - 1 + a, c - 1 + b).
// a = 0: the element above-left/above-right, node is on its bottom edge.
__host__ __device__ constexpr int corner_of(int a, int b) {
  return a == 0 ? (b == 0 ? 1 : 0) : (b == 0 ? 2 : 3);
}
// Offset (dr, dc) of corner k of the element whose top-left node is (0, 0).
__host__ __device__ constexpr int corner_dr(int k) { return (k == 0 || k == 1) ? 1 : 0; }
__host__ __device__ constexpr int corner_dc(int k) { return (k == 1 || k == 2) ? 1 : 0; }

template <typename T>
STT_DEV T ldg(const T* p) {
  return __ldg(p);
}

// ---- block reductions (kNT threads) ---------------------------------------------

STT_DEV double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over a block of NT threads; the result is valid in every thread.
template <int NT>
STT_DEV double block_sum(double v, double* scratch /* >= NT/32 doubles */) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) t += scratch[w];
  return t;
}

// Deterministic grid reduction of K values per batch row: every block stores its
// partial sums, the last block to arrive sums them in block order and runs `fin`.
// `counters[row]` is reset by that last block, so the buffer is reusable at once.
struct GridRed {
  double* partials;    // [rows][nblk][K]
  unsigned* counters;  // [rows]
  int nblk;
};

template <int K, int NT, typename Fin>
STT_DEV void grid_reduce(const GridRed& g, int row, int bid, const double (&v)[K], Fin fin) {
  __shared__ double scratch[NT / 32];
  __shared__ bool is_last;
  double s[K];
#pragma unroll
  for (int k = 0; k < K; ++k) s[k] = block_sum<NT>(v[k], scratch);
  const int tid = threadIdx.x;
  if (tid == 0) {
    double* dst = g.partials + ((size_t)row * g.nblk + bid) * K;
#pragma unroll
    for (int k = 0; k < K; ++k) dst[k] = s[k];
    __threadfence();
    unsigned prev = atomicAdd(&g.counters[row], 1u);
    is_last = (prev == (unsigned)g.nblk - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double t[K];
#pragma unroll
  for (int k = 0; k < K; ++k) t[k] = 0.0;
  const volatile double* src = g.partials + (size_t)row * g.nblk * K;
  for (int b = tid; b < g.nblk; b += NT) {
#pragma unroll
    for (int k = 0; k < K; ++k) t[k] += src[(size_t)b * K + k];
  }
#pragma unroll
  for (int k = 0; k < K; ++k) t[k] = block_sum<NT>(t[k], scratch);
  if (tid == 0) {
    fin(t);
    g.counters[row] = 0u;
  }
}

STT_DEV double safe_div(double num, double den) { return den != 0.0 ? num / den : 0.0; }

// Signs of the six plane-stress edge modes (Gx(ux), Gy(uy), Gy(ux), Gx(uy), H(ux), H(uy))
// under the x and the y reflection of an element: the Gx and H patterns change sign under
// x, Gy and H under y, and so do ux under x and uy under y.
__host__ __device__ constexpr int mode_dx(int i) { return (i == 2 || i == 3 || i == 5) ? -1 : 1; }
__host__ __device__ constexpr int mode_dy(int i) { return (i == 2 || i == 3 || i == 4) ? -1 : 1; }
constexpr double kModeDX[6] = {1, 1, -1, -1, 1, -1};
constexpr double kModeDY[6] = {1, 1, -1, -1, -1, 1};

// n / k and n % k for the coarsening factors k in {1, 2, 3} and 0 <= n < 2^30, without
// an integer division (0x55555556 = ceil(2^32 / 3) gives floor(n / 3) exactly there).
STT_DEV int div_k(int n, int k) {
  return k == 2 ? (n >> 1) : (k == 3 ? (int)__umulhi((unsigned)n, 0x55555556u) : n);
}

// The sweep update x0 + (omega * res) / diag: exact division in FP64 (the reference's
// arithmetic), the fast division in the FP32 V-cycle (a preconditioner, no reference).
STT_DEV double sweep_div(double num, double den) { return num / den; }
STT_DEV float sweep_div(float num, float den) { return __fdividef(num, den); }

}  // namespace stt
