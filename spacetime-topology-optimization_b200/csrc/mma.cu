// The MMA subproblem (sttopt/mma.py:150-557, Svanberg's method of moving asymptotes)
// on the device: mmasub's asymptotes and separable approximation, and subsolv's
// primal-dual interior-point Newton loop along the barrier path epsi = 1, 0.1, ... .
//
// Every n-sized or m x n-sized quantity stays in HBM and is touched only by the fused
// per-variable passes below; everything m-sized (y, z, lam, mu, zet, s, the bordered
// (m+1) x (m+1) Newton system, the line search's decisions) lives on the host, as the
// reference also solves that system on the host.  For mmasub the constraint
// approximation P, Q (m x n) is never stored: each pass rebuilds P_ij, Q_ij from dfdx_ij
// and three per-variable numbers, so a pass reads one m x n array instead of two.
//
// One Newton step is three passes over the variables: assemble (the residual at the
// current point, the Newton right-hand side and the m x m matrix GG diag(1/diagx) GG^T,
// formed on the FP64 tensor cores from a shared-memory tile of GG), step (dx and the
// fraction-to-the-boundary limits) and one search pass per line-search candidate.  The
// accepted step is applied by the next pass's prologue.  Reductions are deterministic:
// one partial a block, folded in block order (by the step and search passes' last block,
// and for the assemble pass's larger product by a separate fold kernel).
//
// The file is compiled with -fmad=false, so that a * b + c rounds twice as in the
// reference's tensor arithmetic; the dot products use fma() explicitly.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "errors.h"

namespace stt {

constexpr int kMmaThreads = 256;  // a tile is kMmaThreads variables, one a thread
constexpr int kMmaMaxM = 64;

// A per-variable parameter of mmasub: a vector (p) or one value for all (v).
struct VarParam {
  const double* p;
  double v;
};
STT_DEV double vp(const VarParam& q, long long j) { return q.p ? q.p[j] : q.v; }

// An m-vector passed by value as a kernel parameter.
struct MVec {
  double v[kMmaMaxM];
};

// The subproblem's per-variable data (fixed through subsolv).  With P / Q given (the
// subsolv entry) p0, q0, P, Q are read; otherwise (the mmasub entry) they are rebuilt
// from xval, df0dx, dfdx and rxm = raa0 / max(xmax - xmin, 1e-5).
struct MmaCols {
  long long n, ld;  // ld: row stride of P, Q or dfdx
  int m;
  const double *low, *upp, *alfa, *beta;
  const double *p0, *q0, *P, *Q;
  const double *xval, *df0dx, *dfdx, *rxm;
};

STT_DEV double nanmax(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

// The separable approximation of one gradient entry g (sttopt/mma.py:263-284), factored
// as P = P' ux2 and Q = Q' xl2 with P' = max(g, 0) + (0.001 |g| + r) and
// Q' = max(-g, 0) + (0.001 |g| + r): the reference's own operations before its
// multiplication by ux2 / xl2, which the passes fold into per-variable constants.
STT_DEV void approx_pq1(double g, double r, double& p1, double& q1) {
  const double pp = fmax(g, 0.0), qq = fmax(-g, 0.0);
  const double pq = 0.001 * (pp + qq) + r;
  p1 = pp + pq;
  q1 = qq + pq;
}

// A variable's fixed data; P = P' sp and Q = Q' sq (sp = sq = 1 when P, Q are given).
struct ColFixed {
  double low, upp, alfa, beta, p0, q0, sp, sq, r;
};

template <bool G>
STT_DEV ColFixed load_fixed(const MmaCols& c, long long j) {
  ColFixed f;
  f.low = c.low[j];
  f.upp = c.upp[j];
  f.alfa = c.alfa[j];
  f.beta = c.beta[j];
  if constexpr (G) {
    const double xv = c.xval[j];
    const double ux1 = f.upp - xv, xl1 = xv - f.low;
    f.sp = ux1 * ux1;
    f.sq = xl1 * xl1;
    f.r = c.rxm[j];
    double p1, q1;
    approx_pq1(c.df0dx[j], f.r, p1, q1);
    f.p0 = p1 * f.sp;
    f.q0 = q1 * f.sq;
  } else {
    f.p0 = c.p0[j];
    f.q0 = c.q0[j];
    f.sp = f.sq = 1.0;
    f.r = 0.0;
  }
  return f;
}

// Rows are read in chunks: the CH entries of column j in rows [i0, i0 + CH), all loads
// issued before any is used (a load guarded together with its use would wait out one
// memory latency a row).  Rows past m - 1 read as 0.
// The step and search passes take smaller chunks, for three blocks an SM.
template <int MB, bool G>
constexpr int pass_chunk() {
  if constexpr (G) {
    return MB <= 12 ? MB : (MB % 10 == 0 ? 10 : 8);
  } else {
    return MB <= 8 ? MB : 4;
  }
}
template <int MB, bool G>
constexpr int row_chunk() {
  if constexpr (G) {
    return MB <= 20 ? MB : (MB % 16 == 0 ? 16 : 8);
  } else {
    return MB <= 12 ? MB : (MB % 8 == 0 ? 8 : 4);  // two loads an entry
  }
}
template <int CH, bool G>
STT_DEV void load_rows(const MmaCols& c, int i0, long long j, double (&a)[CH], double (&b)[CH]) {
  const int nv = c.m - i0;
  long long o = (long long)i0 * c.ld + j;
#pragma unroll
  for (int u = 0; u < CH; ++u) {
    a[u] = b[u] = 0.0;
    if (u < nv) {
      if constexpr (G) {
        a[u] = __ldg(c.dfdx + o);
      } else {
        a[u] = __ldg(c.P + o);
        b[u] = __ldg(c.Q + o);
      }
    }
    o += c.ld;
  }
}
// P', Q' of one entry from what load_rows read.
template <bool G>
STT_DEV void rows_pq1(const ColFixed& f, double a, double b, double& p1, double& q1) {
  if constexpr (G) {
    approx_pq1(a, f.r, p1, q1);
  } else {
    p1 = a;
    q1 = b;
  }
}

// The per-variable factors of a gradient entry's terms at a point: gvec's
// P / ux1 + Q / xl1 = P' A + Q' B and GG's P / ux2 - Q / xl2 = P' C - Q' D.
struct ColFactors {
  double A, B, C, D;
};

// Divisions by the point's four distances are multiplications by these reciprocals (one
// division each), which rounds within an ulp of the reference's quotients.
struct ColPoint {
  double ux1, xl1, ux2, xl2, uxinv1, xlinv1, uxinv2, xlinv2, xa, bx, xainv, bxinv;
};
STT_DEV ColPoint point_of(const ColFixed& f, double x) {
  ColPoint p;
  p.ux1 = f.upp - x;
  p.xl1 = x - f.low;
  p.ux2 = p.ux1 * p.ux1;
  p.xl2 = p.xl1 * p.xl1;
  p.uxinv1 = 1.0 / p.ux1;
  p.xlinv1 = 1.0 / p.xl1;
  p.uxinv2 = 1.0 / p.ux2;
  p.xlinv2 = 1.0 / p.xl2;
  p.xa = x - f.alfa;
  p.bx = f.beta - x;
  p.xainv = 1.0 / p.xa;
  p.bxinv = 1.0 / p.bx;
  return p;
}
STT_DEV ColFactors factors_of(const ColFixed& f, const ColPoint& p) {
  return {f.sp * p.uxinv1, f.sq * p.xlinv1, f.sp * p.uxinv2, f.sq * p.xlinv2};
}

// old + t * d for x, xsi, eta, with dxsi / deta formed from dx as subsolv does
// (sttopt/mma.py:520-521).
STT_DEV void step_point(double& x, double& xsi, double& eta, double dx, double t, double epsi, double alfa,
                        double beta) {
  const double xainv = 1.0 / (x - alfa), bxinv = 1.0 / (beta - x);
  const double dxsi = -xsi + epsi * xainv - (xsi * dx) * xainv;
  const double deta = -eta + epsi * bxinv + (eta * dx) * bxinv;
  x = x + t * dx;
  xsi = xsi + t * dxsi;
  eta = eta + t * deta;
}

// The Newton terms of one variable (sttopt/mma.py:453-465): delx and diagx.
STT_DEV void newton_col(double plam, double qlam, const ColPoint& p, double xsi, double eta, double epsi,
                        double& delx, double& diagx) {
  const double dpsidx = plam * p.uxinv2 - qlam * p.xlinv2;
  delx = dpsidx - epsi * p.xainv + epsi * p.bxinv;
  diagx = 2.0 * (plam * p.uxinv2 * p.uxinv1 + qlam * p.xlinv2 * p.xlinv1) + xsi * p.xainv + eta * p.bxinv;
}

// The n-sized parts of the barrier residual (rex, rexsi, reeta; sttopt/mma.py:409-417):
// their sum of squares and largest magnitude.  A NaN part makes the sum of squares NaN,
// from which the host restores the NaN maximum the reference's max would give.
STT_DEV void resid_n(double plam, double qlam, const ColPoint& p, double xsi, double eta, double epsi, double& ss,
                     double& mx) {
  const double dpsidx = plam * p.uxinv2 - qlam * p.xlinv2;
  const double rex = dpsidx - xsi + eta;
  const double rexsi = xsi * p.xa - epsi;
  const double reeta = eta * p.bx - epsi;
  ss = fma(rex, rex, ss);
  ss = fma(rexsi, rexsi, ss);
  ss = fma(reeta, reeta, ss);
  mx = fmax(mx, fmax(fabs(rex), fmax(fabs(rexsi), fabs(reeta))));
}

// ---- deterministic block partials and the last block's finalisation --------------------

// Warp-then-block sum of one value a thread; every thread gets the result.
STT_DEV double block_total(double v, double* red /* >= kMmaThreads/32 */) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < kMmaThreads / 32; ++w) t += red[w];
  return t;
}
STT_DEV double block_nanmax(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = -INFINITY;
#pragma unroll
  for (int w = 0; w < kMmaThreads / 32; ++w) t = nanmax(t, red[w]);
  return t;
}

// Block partials are stored entry-major: entry e of block b at partials[e * grid + b].
STT_DEV double* part(double* partials, int e) { return partials + (size_t)e * gridDim.x + blockIdx.x; }

constexpr int kFoldMax = 16;  // a lane folds up to 16 blocks: grids of at most 512 blocks

// One partial entry over all nb blocks (p: its nb values): lane l takes blocks l, l + 32,
// ... with every load issued before the first is used, then the lanes combine in a fixed
// butterfly.  The result does not depend on the order the blocks ran in.
STT_DEV double fold_entry(const double* p, int nb, bool sum, int lane) {
  double v[kFoldMax];
#pragma unroll
  for (int q = 0; q < kFoldMax; ++q) {
    const int b = lane + 32 * q;
    v[q] = b < nb ? __ldcg(p + b) : (sum ? 0.0 : -INFINITY);
  }
  double t = v[0];
#pragma unroll
  for (int q = 1; q < kFoldMax; ++q) t = sum ? t + v[q] : nanmax(t, v[q]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_xor_sync(0xffffffffu, t, o);
    t = sum ? t + u : nanmax(t, u);
  }
  return t;
}

// After this block wrote its kp partials (the first ks summed, the rest max-reduced):
// the last block to arrive folds every entry over all blocks into fin[kp] (shared
// memory), a warp an entry, and returns true.
STT_DEV bool finish_blocks(const double* partials, unsigned* counter, int kp, int ks, double* fin) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  const int lane = threadIdx.x & 31, nb = gridDim.x;
  for (int e = threadIdx.x >> 5; e < kp; e += kMmaThreads / 32) {
    const double t = fold_entry(partials + (size_t)e * nb, nb, e < ks, lane);
    if (lane == 0) fin[e] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// ---- mmasub's per-variable setup ---------------------------------------------------------

// The moving asymptotes (sttopt/mma.py:226-247: from scratch while iteration < 2, else
// widened by asyincr where x moved monotonically and narrowed by asydecr where it
// oscillated, clamped to [asyclamp_min, asyclamp_max] times the range) and the move
// limits alfa / beta (:249-253).  low / upp are read and rewritten in place; rxm is
// raa0 / max(xmax - xmin, 1e-5), the curvature floor of the approximation (:255-284).
__global__ void __launch_bounds__(kMmaThreads) mma_setup_kernel(
    long long n, int iteration, const double* __restrict__ xval, const double* __restrict__ xmin,
    const double* __restrict__ xmax, const double* __restrict__ xold1, const double* __restrict__ xold2,
    double* __restrict__ low, double* __restrict__ upp, VarParam asyinit, VarParam clmin, VarParam clmax,
    VarParam move, double raa0, double albefa, double asyincr, double asydecr, double* __restrict__ alfa,
    double* __restrict__ beta, double* __restrict__ rxm) {
  for (long long j = blockIdx.x * (long long)kMmaThreads + threadIdx.x; j < n;
       j += (long long)gridDim.x * kMmaThreads) {
    const double xv = xval[j], xr = xmax[j] - xmin[j];
    double lo, up;
    if (iteration < 2) {
      lo = xv - vp(asyinit, j) * xr;
      up = xv + vp(asyinit, j) * xr;
    } else {
      const double x1 = xold1[j], zzz = (xv - x1) * (x1 - xold2[j]);
      const double factor = zzz > 0 ? asyincr : (zzz < 0 ? asydecr : 1.0);
      lo = xv - factor * (x1 - low[j]);
      up = xv + factor * (upp[j] - x1);
      lo = fmin(fmax(lo, xv - vp(clmax, j) * xr), xv - vp(clmin, j) * xr);
      up = fmax(fmin(up, xv + vp(clmax, j) * xr), xv + vp(clmin, j) * xr);
    }
    low[j] = lo;
    upp[j] = up;
    alfa[j] = fmax(fmax(lo + albefa * (xv - lo), xv - vp(move, j) * xr), xmin[j]);
    beta[j] = fmin(fmin(up - albefa * (up - xv), xv + vp(move, j) * xr), xmax[j]);
    rxm[j] = raa0 * (1.0 / fmax(xr, 1e-5));
  }
}

// subsolv's starting point (sttopt/mma.py:384-389): x the middle of [alfa, beta],
// xsi / eta = max(1 / distance to the bound, 1).
__global__ void __launch_bounds__(kMmaThreads) mma_init_kernel(long long n, const double* __restrict__ alfa,
                                                               const double* __restrict__ beta, double* __restrict__ x,
                                                               double* __restrict__ xsi, double* __restrict__ eta) {
  for (long long j = blockIdx.x * (long long)kMmaThreads + threadIdx.x; j < n;
       j += (long long)gridDim.x * kMmaThreads) {
    const double xv = 0.5 * (alfa[j] + beta[j]);
    x[j] = xv;
    xsi[j] = fmax(1.0 / (xv - alfa[j]), 1.0);
    eta[j] = fmax(1.0 / (beta[j] - xv), 1.0);
  }
}

// The accepted line-search step, applied where no later pass does it.
__global__ void __launch_bounds__(kMmaThreads) mma_apply_kernel(long long n, const double* __restrict__ alfa,
                                                                const double* __restrict__ beta,
                                                                const double* __restrict__ dx, double t, double epsi,
                                                                double* __restrict__ x, double* __restrict__ xsi,
                                                                double* __restrict__ eta) {
  for (long long j = blockIdx.x * (long long)kMmaThreads + threadIdx.x; j < n;
       j += (long long)gridDim.x * kMmaThreads) {
    double xv = x[j], xs = xsi[j], et = eta[j];
    step_point(xv, xs, et, dx[j], t, epsi, alfa[j], beta[j]);
    x[j] = xv;
    xsi[j] = xs;
    eta[j] = et;
  }
}

// ---- subsolv's Newton passes ---------------------------------------------------------------

// A warp's sum in a fixed butterfly order; every lane gets it.
STT_DEV double warp_allsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Per-row sums over all variables without a register a row: for row i the warp sums
// its 32 variables' terms and lane i mod 32 keeps the running total in acc[i / 32].
// Called by whole warps (lanes past n add zeros).
template <int MB>
struct RowSums {
  static constexpr int K = (MB + 31) / 32;
  double acc[K];
  STT_DEV void zero() {
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
  }
  STT_DEV void add(int i, double v) {
    v = warp_allsum(v);
    if ((threadIdx.x & 31) == (i & 31)) acc[i >> 5] += v;
  }
  // The block's row sums (warp by warp, in warp order) into its partial entries
  // e0 .. e0 + m - 1; sh holds kMmaThreads / 32 x kMmaMaxM doubles.
  STT_DEV void write(int m, double* partials, int e0, double* sh) const {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int i = k * 32 + lane;
      if (i < m) sh[warp * kMmaMaxM + i] = acc[k];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += kMmaThreads) {
      double t = 0.0;
      for (int w = 0; w < kMmaThreads / 32; ++w) t += sh[w * kMmaMaxM + i];
      *part(partials, e0 + i) = t;
    }
    __syncthreads();
  }
};

// The same row sums kept in shared memory, one slot a row and thread: a thread adds its
// own variables' terms to its slots (no synchronisation, no shuffles) and the block
// folds the slots once at the end.  slots: [MB][kMmaThreads] doubles.
template <int MB>
struct SlotSums {
  double* slots;
  STT_DEV void zero() {
#pragma unroll
    for (int i = 0; i < MB; ++i) slots[i * kMmaThreads + threadIdx.x] = 0.0;
  }
  STT_DEV void add(int i, double v) { slots[i * kMmaThreads + threadIdx.x] += v; }
  STT_DEV void write(int m, double* partials, int e0, double*) const {
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < m; i += kMmaThreads / 32) {
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < kMmaThreads / 32; ++k) t += slots[i * kMmaThreads + k * 32 + lane];
      t = warp_allsum(t);
      if (lane == 0) *part(partials, e0 + i) = t;
    }
    __syncthreads();
  }
};
// Slots where they fit beside the assemble pass's tile at two blocks an SM.
template <int MB>
constexpr bool use_slots() {
  return MB <= 24;
}
template <int MB>
using RowAcc = std::conditional_t<use_slots<MB>(), SlotSums<MB>, RowSums<MB>>;

// The m x m product GG diag(1/diagx) GG^T is formed on the FP64 tensor cores: tcgen05 has
// no FP64 kind, so this is mma.sync m8n8k4 (DMMA), 8 x 8 tiles of the (m + 1)-row tile of
// GG with delx appended (row m, which gives h), k running over a tile's variables.
constexpr int kMmaLd8 = kMmaThreads + 4;  // row stride of the GG tile: fragment loads hit distinct banks

STT_DEV void dmma_f64(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Upper-triangular 8 x 8 tiles (I <= K) of the (m + 1) x (m + 1) product, t8 a side.
__host__ __device__ inline int gram_side(int m) { return (m + 8) >> 3; }
__host__ __device__ inline int gram_tiles(int m) { return gram_side(m) * (gram_side(m) + 1) / 2; }
__host__ __device__ inline int tile_index(int I, int K, int t8) { return I * t8 - I * (I - 1) / 2 + (K - I); }
// The product's upper triangle (i <= k <= m, row m being delx), packed row by row.
__host__ __device__ inline int packed_index(int i, int k, int m1) { return i * m1 - i * (i - 1) / 2 + (k - i); }
// Partial entries of the assemble pass: [gvec (m) | sum of squares | packed product | max].
__host__ __device__ inline int assemble_kp(int m) { return m + 2 + (m + 1) * (m + 2) / 2; }
// Its dynamic shared memory: the GG tile (or, later, the folded entries), 1/diagx, a
// block-sum scratch, and when it forms gvec the row-sum slots or shuffle scratch.
inline size_t assemble_smem(int m, int mb, bool need_g) {
  const size_t rows = (size_t)gram_side(m) * 8;
  const size_t tail = !need_g ? 0 : mb <= 24 ? (size_t)mb * kMmaThreads : (size_t)(kMmaThreads / 32) * kMmaMaxM;
  return 8 * (std::max(rows * kMmaLd8, (size_t)assemble_kp(m)) + kMmaThreads + 8 + tail);
}
inline int mma_bucket(int m) {
  return m <= 4 ? 4 : m <= 8 ? 8 : m <= 12 ? 12 : m <= 16 ? 16 : m <= 20 ? 20 : m <= 24 ? 24 : m <= 32 ? 32
         : m <= 48 ? 48 : 64;
}

// The assemble pass (sttopt/mma.py:399-489, m < n): applies a pending accepted step,
// then at the point (x, lam, xsi, eta) and barrier epsi forms, over all variables,
//   gvec = P (1/ux1) + Q (1/xl1),  h = GG (delx / diagx),  A = GG diag(1/diagx) GG^T
// with GG = P diag(1/ux2) - Q diag(1/xl2), and the sum of squares and largest magnitude
// of the residual's n-sized parts.  A block's 256 variables write their GG column and
// delx into a shared tile; A and h come from DMMA tiles of that tile.  Up to 31
// constraints each warp takes 32 of the tile's variables for every 8 x 8 tile and the
// warps' sums are folded in warp order; above that the tiles are split among the warps.
// gvec is formed only with need_g: after a line search it is the accepted candidate's,
// which the search pass formed at this same point.
// res = [gvec (m), or zeros | h (m) | A (m x m) | sum of squares | max].
template <int MB, bool G>
__global__ void __launch_bounds__(kMmaThreads, 2) mma_assemble_kernel(
    MmaCols c, double* __restrict__ x, double* __restrict__ xsi, double* __restrict__ eta,
    const double* __restrict__ dx, int pend, double t_pend, double eps_pend, MVec lam, double epsi, int need_g,
    double* __restrict__ partials) {
  extern __shared__ double sm[];
  constexpr int T8 = (MB + 8) / 8;  // tile side for the largest m of the bucket
  constexpr int NT = T8 * (T8 + 1) / 2;
  constexpr bool KSPLIT = T8 <= 4;
  constexpr int TPW = KSPLIT ? NT : (NT + 7) / 8;  // tiles a warp accumulates
  const int m = c.m, t8 = gram_side(m), rows = t8 * 8, ntile = gram_tiles(m);
  const int head = max(rows * kMmaLd8, assemble_kp(m));
  double* gs = sm;                 // [rows][kMmaLd8]
  double* ws = sm + head;          // [kMmaThreads]: 1 / diagx
  double* wred = ws + kMmaThreads; // [8]
  double* tail = wred + 8;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int fr = lane >> 2, fc = lane & 3;  // DMMA fragment row and column
  double acc[TPW][2];
#pragma unroll
  for (int q = 0; q < TPW; ++q) acc[q][0] = acc[q][1] = 0.0;
  RowAcc<MB> gv;
  if (need_g) {
    if constexpr (use_slots<MB>()) gv.slots = tail;
    gv.zero();
  }
  double ss = 0.0, mx = 0.0;
  for (int r = m + 1; r < rows; ++r) gs[r * kMmaLd8 + tid] = 0.0;

  const long long ntiles = (c.n + kMmaThreads - 1) / kMmaThreads;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long j = tile * kMmaThreads + tid;
    const bool ok = j < c.n;
    ColFixed f{};
    ColPoint p{};
    double xs = 0.0, et = 0.0;
    if (ok) {
      f = load_fixed<G>(c, j);
      double xv = x[j];
      xs = xsi[j];
      et = eta[j];
      if (pend) {
        step_point(xv, xs, et, dx[j], t_pend, eps_pend, f.alfa, f.beta);
        x[j] = xv;
        xsi[j] = xs;
        eta[j] = et;
      }
      p = point_of(f, xv);
    }
    const ColFactors k = factors_of(f, p);
    double lp = 0.0, lq = 0.0;  // sum of lam_i P'_i, lam_i Q'_i
    constexpr int CH = row_chunk<MB, G>();
#pragma unroll
    for (int i0 = 0; i0 < MB; i0 += CH) {
      if (i0 < m) {
        double ra[CH], rb[CH];
        if (ok) {
          load_rows<CH, G>(c, i0, j, ra, rb);
        } else {
#pragma unroll
          for (int u = 0; u < CH; ++u) ra[u] = rb[u] = 0.0;
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          const int i = i0 + u;
          if (i < m) {
            double p1, q1;
            rows_pq1<G>(f, ra[u], rb[u], p1, q1);
            lp = fma(lam.v[i], p1, lp);
            lq = fma(lam.v[i], q1, lq);
            if (need_g) gv.add(i, fma(p1, k.A, q1 * k.B));
            gs[i * kMmaLd8 + tid] = fma(p1, k.C, -(q1 * k.D));
          }
        }
      }
    }
    double w = 0.0, delx = 0.0;
    if (ok) {
      const double plam = f.p0 + f.sp * lp;
      const double qlam = f.q0 + f.sq * lq;
      resid_n(plam, qlam, p, xs, et, epsi, ss, mx);
      double diagx;
      newton_col(plam, qlam, p, xs, et, epsi, delx, diagx);
      w = 1.0 / diagx;
    }
    gs[m * kMmaLd8 + tid] = delx;
    ws[tid] = w;
    // Up to 31 constraints a warp's tiles read only the 32 variables the warp wrote, so
    // the warps need not wait for one another.
    if constexpr (KSPLIT) {
      __syncwarp();
    } else {
      __syncthreads();
    }
    if constexpr (KSPLIT) {
#pragma unroll 2
      for (int k4 = 0; k4 < 8; ++k4) {
        const int col = warp * 32 + k4 * 4 + fc;
        const double wc = ws[col];
        double a[T8], b[T8];
#pragma unroll
        for (int I = 0; I < T8; ++I) {
          a[I] = I < t8 ? gs[(8 * I + fr) * kMmaLd8 + col] : 0.0;
          b[I] = a[I] * wc;
        }
        int q = 0;
#pragma unroll
        for (int I = 0; I < T8; ++I)
#pragma unroll
          for (int K = I; K < T8; ++K, ++q)
            if (K < t8) dmma_f64(acc[q], a[I], b[K]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < TPW; ++q) {
        const int t = warp + 8 * q;
        if (t < ntile) {
          int I = 0, rem = t;
          while (rem >= t8 - I) {
            rem -= t8 - I;
            ++I;
          }
          const int K = I + rem;
          const double* ga = gs + (8 * I + fr) * kMmaLd8 + fc;
          const double* gb = gs + (8 * K + fr) * kMmaLd8 + fc;
#pragma unroll 4
          for (int k4 = 0; k4 < kMmaThreads / 4; ++k4)
            dmma_f64(acc[q], ga[4 * k4], gb[4 * k4] * ws[4 * k4 + fc]);
        }
      }
    }
    if constexpr (KSPLIT) {
      __syncwarp();
    } else {
      __syncthreads();
    }
  }

  // Product partials: entry m + 1 + packed_index(i, k) holds (i, k), i <= k <= m; tile
  // t = (I, K) holds (8 I + r, 8 K + c) at r * 8 + c.
  const int m1 = m + 1;
  if constexpr (KSPLIT) {
    __syncthreads();    // every warp's tiles are done before the tile memory is reused
    double* red8 = sm;  // [8 warps][ntile][64]
    int q = 0;
#pragma unroll
    for (int I = 0; I < T8; ++I)
#pragma unroll
      for (int K = I; K < T8; ++K, ++q)
        if (K < t8) {
          double* d = red8 + ((size_t)warp * ntile + tile_index(I, K, t8)) * 64 + fr * 8 + fc * 2;
          d[0] = acc[q][0];
          d[1] = acc[q][1];
        }
    __syncthreads();
    for (int e = tid; e < m1 * m1; e += kMmaThreads) {
      const int i = e / m1, k = e % m1;
      if (i > k) continue;
      const size_t at = (size_t)tile_index(i >> 3, k >> 3, t8) * 64 + (i & 7) * 8 + (k & 7);
      double t = 0.0;
      for (int w8 = 0; w8 < kMmaThreads / 32; ++w8) t += red8[(size_t)w8 * ntile * 64 + at];
      *part(partials, m + 1 + packed_index(i, k, m1)) = t;
    }
  } else {
#pragma unroll
    for (int q = 0; q < TPW; ++q) {
      const int t = warp + 8 * q;
      if (t < ntile) {
        int I = 0, rem = t;
        while (rem >= t8 - I) {
          rem -= t8 - I;
          ++I;
        }
        const int K = I + rem;
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int i = 8 * I + fr, k = 8 * K + fc * 2 + v;
          if (i <= k && k <= m) *part(partials, m + 1 + packed_index(i, k, m1)) = acc[q][v];
        }
      }
    }
  }
  const int ks = assemble_kp(m) - 1;
  if (need_g) {
    gv.write(m, partials, 0, tail);
  } else {
    for (int i = tid; i < m; i += kMmaThreads) *part(partials, i) = 0.0;
  }
  const double t = block_total(ss, wred);
  if (tid == 0) *part(partials, m) = t;
  const double u = block_nanmax(mx, wred);
  if (tid == 0) *part(partials, ks) = u;
}

// Folds the assemble pass's block partials (entry-major, nb blocks) in block order, a
// warp an entry on as many SMs as there are entries / 8, and writes
// res = [gvec (m) | h (m) | A (m x m) | sum of squares | max].
__global__ void __launch_bounds__(kMmaThreads) mma_fold_kernel(const double* __restrict__ partials, int nb, int m,
                                                               double* __restrict__ res) {
  const int kp = assemble_kp(m), ks = kp - 1, m1 = m + 1, lane = threadIdx.x & 31;
  const int e = blockIdx.x * (kMmaThreads / 32) + (threadIdx.x >> 5);
  if (e >= kp) return;
  const double t = fold_entry(partials + (size_t)e * nb, nb, e < ks, lane);
  if (lane != 0) return;
  if (e < m) {
    res[e] = t;
  } else if (e == m) {
    res[2 * m + m * m] = t;
  } else if (e == ks) {
    res[2 * m + m * m + 1] = t;
  } else {
    int i = 0, pe = e - m - 1;
    while (pe >= m1 - i) {
      pe -= m1 - i;
      ++i;
    }
    const int k = i + pe;
    if (k == m) {
      if (i < m) res[m + i] = t;  // (m, m), delx' diag(1/diagx) delx, is not needed
    } else {
      res[2 * m + i * m + k] = t;
      res[2 * m + k * m + i] = t;
    }
  }
}

// The step pass (sttopt/mma.py:490-535, m < n): with the Newton step's dlam from the
// host, dx = -delx / diagx - (GG^T dlam) / diagx (stored), dxsi and deta, and the
// fraction-to-the-boundary limits max(-1.01 dx / (x - alfa)), max(1.01 dx / (beta - x))
// and max(-1.01 dxsi / xsi, -1.01 deta / eta).  res = those three maxima and the step
// length steg = 1 / max(them, stm_host (the m-sized variables' limit), 1), formed as the
// host forms it, for a search pass launched right behind this one.
template <int MB, bool G>
__global__ void __launch_bounds__(kMmaThreads, 3) mma_step_kernel(
    MmaCols c, const double* __restrict__ x, const double* __restrict__ xsi, const double* __restrict__ eta,
    MVec lam, MVec dlam, double epsi, double stm_host, double* __restrict__ dx, double* __restrict__ partials,
    unsigned* __restrict__ counter, double* __restrict__ res) {
  __shared__ double red[kMmaThreads / 32];
  __shared__ double fin[3];
  const int m = c.m;
  double m1 = -INFINITY, m2 = -INFINITY, m3 = -INFINITY;
  for (long long j = blockIdx.x * (long long)kMmaThreads + threadIdx.x; j < c.n;
       j += (long long)gridDim.x * kMmaThreads) {
    const ColFixed f = load_fixed<G>(c, j);
    const double xv = x[j], xs = xsi[j], et = eta[j];
    const ColPoint p = point_of(f, xv);
    double lp = 0.0, lq = 0.0, dp = 0.0, dq = 0.0;  // lam . P', lam . Q', dlam . P', dlam . Q'
    constexpr int CH = pass_chunk<MB, G>();
#pragma unroll
    for (int i0 = 0; i0 < MB; i0 += CH) {
      if (i0 < m) {
        double ra[CH], rb[CH];
        load_rows<CH, G>(c, i0, j, ra, rb);
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          const int i = i0 + u;
          if (i < m) {
            double p1, q1;
            rows_pq1<G>(f, ra[u], rb[u], p1, q1);
            lp = fma(lam.v[i], p1, lp);
            lq = fma(lam.v[i], q1, lq);
            dp = fma(dlam.v[i], p1, dp);
            dq = fma(dlam.v[i], q1, dq);
          }
        }
      }
    }
    const ColFactors k = factors_of(f, p);
    const double plam = f.p0 + f.sp * lp, qlam = f.q0 + f.sq * lq;
    const double gd = fma(dp, k.C, -(dq * k.D));  // GG^T dlam
    double delx, diagx;
    newton_col(plam, qlam, p, xs, et, epsi, delx, diagx);
    const double w = 1.0 / diagx;
    const double d = -delx * w - gd * w;
    dx[j] = d;
    const double dxsi = -xs + epsi * p.xainv - (xs * d) * p.xainv;
    const double deta = -et + epsi * p.bxinv + (et * d) * p.bxinv;
    m1 = nanmax(m1, (-1.01 * d) * p.xainv);
    m2 = nanmax(m2, (1.01 * d) * p.bxinv);
    m3 = nanmax(m3, nanmax((-1.01 * dxsi) / xs, (-1.01 * deta) / et));
  }
  const double b1 = block_nanmax(m1, red);
  const double b2 = block_nanmax(m2, red);
  const double b3 = block_nanmax(m3, red);
  if (threadIdx.x == 0) {
    *part(partials, 0) = b1;
    *part(partials, 1) = b2;
    *part(partials, 2) = b3;
  }
  if (!finish_blocks(partials, counter, 3, 0, fin)) return;
  if (threadIdx.x < 3) res[threadIdx.x] = fin[threadIdx.x];
  if (threadIdx.x == 0) res[3] = 1.0 / nanmax(nanmax(nanmax(fin[0], fin[1]), nanmax(fin[2], stm_host)), 1.0);
}

// The search pass: at the point (x, xsi, eta) + t (dx, dxsi, deta) (when dx is given)
// and multipliers lam + t dlam, gvec = P (1/ux1) + Q (1/xl1) and, when resid, the sum of
// squares and largest magnitude of the residual's n-sized parts (sttopt/mma.py:399-434).
// t is read from tdev when given (the step pass's steg, the line search's first
// candidate).  With x = xval and no step it gives mmasub's b + fval (:285).
// res = [gvec (m) | sum of squares | max].
template <int MB, bool G>
__global__ void __launch_bounds__(kMmaThreads, 3) mma_search_kernel(
    MmaCols c, const double* __restrict__ x, const double* __restrict__ xsi, const double* __restrict__ eta,
    const double* __restrict__ dx, double t_arg, const double* tdev, MVec lam0, MVec dlam, double epsi, int resid,
    double* __restrict__ partials, unsigned* __restrict__ counter, double* __restrict__ res) {
  __shared__ double red[kMmaThreads / 32 * (kMmaMaxM + 1)];
  __shared__ double fin[kMmaMaxM + 2];
  __shared__ MVec lam;  // the candidate's multipliers, lam0 + t dlam as the host forms them
  const double t = tdev ? *tdev : t_arg;
  for (int i = threadIdx.x; i < c.m; i += kMmaThreads) lam.v[i] = lam0.v[i] + t * dlam.v[i];
  __syncthreads();
  constexpr bool kSlots = MB <= 20;  // static shared memory stays under 48 KB
  __shared__ double slots[kSlots ? MB * kMmaThreads : 1];
  const int m = c.m;
  std::conditional_t<kSlots, SlotSums<MB>, RowSums<MB>> gv;
  if constexpr (kSlots) gv.slots = slots;
  gv.zero();
  double ss = 0.0, mx = 0.0;
  for (long long base = blockIdx.x * (long long)kMmaThreads; base < c.n; base += (long long)gridDim.x * kMmaThreads) {
    const long long j = base + threadIdx.x;
    const bool ok = j < c.n;
    ColFixed f{};
    ColPoint p{};
    double xs = 0.0, et = 0.0;
    if (ok) {
      f = load_fixed<G>(c, j);
      double xv = x[j];
      if (resid) {
        xs = xsi[j];
        et = eta[j];
      }
      if (dx) step_point(xv, xs, et, dx[j], t, epsi, f.alfa, f.beta);
      p = point_of(f, xv);
    }
    const ColFactors k = factors_of(f, p);
    double lp = 0.0, lq = 0.0;
    constexpr int CH = pass_chunk<MB, G>();
#pragma unroll
    for (int i0 = 0; i0 < MB; i0 += CH) {
      if (i0 < m) {
        double ra[CH], rb[CH];
        if (ok) {
          load_rows<CH, G>(c, i0, j, ra, rb);
        } else {
#pragma unroll
          for (int u = 0; u < CH; ++u) ra[u] = rb[u] = 0.0;
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          const int i = i0 + u;
          if (i < m) {
            double p1, q1;
            rows_pq1<G>(f, ra[u], rb[u], p1, q1);
            lp = fma(lam.v[i], p1, lp);
            lq = fma(lam.v[i], q1, lq);
            gv.add(i, fma(p1, k.A, q1 * k.B));
          }
        }
      }
    }
    if (ok && resid) resid_n(f.p0 + f.sp * lp, f.q0 + f.sq * lq, p, xs, et, epsi, ss, mx);
  }
  const int kp = m + 2, ks = m + 1;
  gv.write(m, partials, 0, red + kMmaThreads / 32);
  const double v = block_total(ss, red);
  const double u = block_nanmax(mx, red);
  if (threadIdx.x == 0) {
    *part(partials, m) = v;
    *part(partials, ks) = u;
  }
  if (!finish_blocks(partials, counter, kp, ks, fin)) return;
  for (int e = threadIdx.x; e < kp; e += kMmaThreads) res[e] = fin[e];
}

// ---- host side ------------------------------------------------------------------------------

namespace {

constexpr int kAsmBlocks = 2 * 148, kPassBlocks = 3 * 148;  // the resident blocks: 2 and 3 an SM
static_assert(kAsmBlocks <= 32 * kFoldMax && kPassBlocks <= 32 * kFoldMax, "a fold lane takes at most kFoldMax blocks");
constexpr int kMaxHalvings = 50;   // sttopt/mma.py:289
constexpr int kMaxNewton = 200;    // sttopt/mma.py:442

using AsmFn = void (*)(MmaCols, double*, double*, double*, const double*, int, double, double, MVec, double, int,
                       double*);
using StepFn = void (*)(MmaCols, const double*, const double*, const double*, MVec, MVec, double, double, double*,
                        double*, unsigned*, double*);
using SearchFn = void (*)(MmaCols, const double*, const double*, const double*, const double*, double, const double*,
                          MVec, MVec, double, int, double*, unsigned*, double*);
struct Kernels {
  AsmFn assemble;
  StepFn step;
  SearchFn search;
};
template <int MB, bool G>
Kernels kernels_of() {
  return {mma_assemble_kernel<MB, G>, mma_step_kernel<MB, G>, mma_search_kernel<MB, G>};
}
template <bool G>
Kernels pick_kernels(int m) {
  switch (mma_bucket(m)) {
    case 4: return kernels_of<4, G>();
    case 8: return kernels_of<8, G>();
    case 12: return kernels_of<12, G>();
    case 16: return kernels_of<16, G>();
    case 20: return kernels_of<20, G>();
    case 24: return kernels_of<24, G>();
    case 32: return kernels_of<32, G>();
    case 48: return kernels_of<48, G>();
    default: return kernels_of<64, G>();
  }
}

// Workspace: [alfa | beta | rxm | dx] (n each), block partials, results, counters.
struct MmaWs {
  double *alfa, *beta, *rxm, *dx, *partials, *res;
  unsigned* counters;
};
size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }
size_t partial_doubles(int m) {
  return std::max({(size_t)kAsmBlocks * assemble_kp(m), (size_t)kPassBlocks * (m + 2), (size_t)kPassBlocks * 3});
}
size_t carve(int m, long long n, char* base, MmaWs* w) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += round256(bytes);
    return p;
  };
  double* v[4];
  for (auto& p : v) p = reinterpret_cast<double*>(take(8 * (size_t)n));
  double* parts = reinterpret_cast<double*>(take(8 * partial_doubles(m)));
  double* res = reinterpret_cast<double*>(take(8 * ((size_t)m * m + 2 * m + 8)));
  unsigned* cnt = reinterpret_cast<unsigned*>(take(4 * sizeof(unsigned)));
  if (w) *w = {v[0], v[1], v[2], v[3], parts, res, cnt};
  return off;
}

double hmax(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

// A x = b for dense row-major A (N x N) by LU with partial pivoting (the first largest
// pivot, as LAPACK's getrf chooses).  Returns false on an exactly singular pivot.
bool dense_solve(std::vector<double>& A, std::vector<double>& b, int N) {
  for (int k = 0; k < N; ++k) {
    int piv = k;
    double best = std::fabs(A[(size_t)k * N + k]);
    for (int r = k + 1; r < N; ++r) {
      const double v = std::fabs(A[(size_t)r * N + k]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (best == 0.0) return false;
    if (piv != k) {
      for (int cidx = 0; cidx < N; ++cidx) std::swap(A[(size_t)k * N + cidx], A[(size_t)piv * N + cidx]);
      std::swap(b[k], b[piv]);
    }
    const double inv = 1.0 / A[(size_t)k * N + k];
    for (int r = k + 1; r < N; ++r) {
      const double l = A[(size_t)r * N + k] * inv;
      if (l == 0.0) continue;
      A[(size_t)r * N + k] = l;
      for (int cidx = k + 1; cidx < N; ++cidx) A[(size_t)r * N + cidx] -= l * A[(size_t)k * N + cidx];
      b[r] -= l * b[k];
    }
  }
  for (int k = N - 1; k >= 0; --k) {
    double s = b[k];
    for (int cidx = k + 1; cidx < N; ++cidx) s -= A[(size_t)k * N + cidx] * b[cidx];
    b[k] = s / A[(size_t)k * N + k];
  }
  return true;
}

// The subproblem's m-sized data and state (host).
struct MState {
  std::vector<double> y, lam, mu, s;
  double z = 1.0, zet = 1.0;
};
struct MData {
  int m;
  double a0;
  const double *a, *b, *c, *d;
};

// The m-sized parts of the residual (rey, rez, relam, remu, rezet, res;
// sttopt/mma.py:413-420) given gvec at the point: sum of squares and max magnitude.
void resid_m(const MData& D, const MState& S, const double* gvec, double epsi, double& ss, double& mx) {
  const int m = D.m;
  double dot = 0.0;
  for (int i = 0; i < m; ++i) dot += S.lam[i] * D.a[i];
  auto add = [&](double r) {
    ss += r * r;
    mx = hmax(mx, std::fabs(r));
  };
  for (int i = 0; i < m; ++i) add(D.c[i] + D.d[i] * S.y[i] - S.mu[i] - S.lam[i]);
  add(D.a0 - S.zet - dot);
  for (int i = 0; i < m; ++i) add(gvec[i] - D.a[i] * S.z - S.y[i] + S.s[i] - D.b[i]);
  for (int i = 0; i < m; ++i) add(S.mu[i] * S.y[i] - epsi);
  add(S.zet * S.z - epsi);
  for (int i = 0; i < m; ++i) add(S.lam[i] * S.s[i] - epsi);
}

void init_state(const MData& D, MState& S) {
  const int m = D.m;
  S.y.assign(m, 1.0);
  S.lam.assign(m, 1.0);
  S.s.assign(m, 1.0);
  S.mu.resize(m);
  for (int i = 0; i < m; ++i) S.mu[i] = std::max(1.0, 0.5 * D.c[i]);
  S.z = S.zet = 1.0;
}

// The m-sized Newton terms shared by both eliminations (sttopt/mma.py:454-467).
struct MNewton {
  std::vector<double> dely, dellam, diagy, diaglamyi;
  double delz;
};
MNewton newton_m(const MData& D, const MState& S, const double* gvec, double epsi) {
  const int m = D.m;
  MNewton N;
  N.dely.resize(m);
  N.dellam.resize(m);
  N.diagy.resize(m);
  N.diaglamyi.resize(m);
  double dot = 0.0;
  for (int i = 0; i < m; ++i) dot += D.a[i] * S.lam[i];
  N.delz = D.a0 - dot - epsi / S.z;
  for (int i = 0; i < m; ++i) {
    N.dely[i] = D.c[i] + D.d[i] * S.y[i] - S.lam[i] - epsi / S.y[i];
    N.dellam[i] = gvec[i] - D.a[i] * S.z - S.y[i] - D.b[i] + epsi / S.lam[i];
    N.diagy[i] = D.d[i] + S.mu[i] / S.y[i];
    N.diaglamyi[i] = S.s[i] / S.lam[i] + 1.0 / N.diagy[i];
  }
  return N;
}

// The m-sized step (dy, dmu, dzet, ds; sttopt/mma.py:518-526) and their share of the
// step limit, max(-1.01 dxx / xx) over y, z, lam, mu, zet, s.
struct MStep {
  std::vector<double> dy, dlam, dmu, ds;
  double dz, dzet;
};
double step_m(const MData& D, const MState& S, const MNewton& N, double epsi, MStep& T) {
  const int m = D.m;
  T.dy.resize(m);
  T.dmu.resize(m);
  T.ds.resize(m);
  for (int i = 0; i < m; ++i) {
    T.dy[i] = -N.dely[i] / N.diagy[i] + T.dlam[i] / N.diagy[i];
    T.dmu[i] = -S.mu[i] + epsi / S.y[i] - (S.mu[i] * T.dy[i]) / S.y[i];
    T.ds[i] = -S.s[i] + epsi / S.lam[i] - (S.s[i] * T.dlam[i]) / S.lam[i];
  }
  T.dzet = -S.zet + epsi / S.z - S.zet * T.dz / S.z;
  double st = -INFINITY;
  auto lim = [&](double d, double v) { st = hmax(st, (-1.01 * d) / v); };
  for (int i = 0; i < m; ++i) lim(T.dy[i], S.y[i]);
  lim(T.dz, S.z);
  for (int i = 0; i < m; ++i) lim(T.dlam[i], S.lam[i]);
  for (int i = 0; i < m; ++i) lim(T.dmu[i], S.mu[i]);
  lim(T.dzet, S.zet);
  for (int i = 0; i < m; ++i) lim(T.ds[i], S.s[i]);
  return st;
}

MState moved(const MState& S, const MStep& T, double t) {
  MState C = S;
  for (size_t i = 0; i < S.y.size(); ++i) {
    C.y[i] = S.y[i] + t * T.dy[i];
    C.lam[i] = S.lam[i] + t * T.dlam[i];
    C.mu[i] = S.mu[i] + t * T.dmu[i];
    C.s[i] = S.s[i] + t * T.ds[i];
  }
  C.z = S.z + t * T.dz;
  C.zet = S.zet + t * T.dzet;
  return C;
}

MVec mvec(const std::vector<double>& v) {
  MVec r;
  for (int i = 0; i < kMmaMaxM; ++i) r.v[i] = i < (int)v.size() ? v[i] : 0.0;
  return r;
}

// Counts of one solve: barrier levels stopped at the Newton cap (and the last such
// epsi), Newton steps, line-search candidates tried.
struct CapStats {
  int hits = 0, steps = 0, tries = 0;
  double epsi = 0.0;
};

}  // namespace

namespace {

// subsolv's barrier path and Newton loop for m < n (sttopt/mma.py:346-557) with the
// per-variable work on the device.  x, xsi, eta (device) receive the solution; S the
// m-sized part.
template <bool G>
int device_subsolv(const MmaCols& c, const MData& D, double epsimin, const MmaWs& w, double* x, double* xsi,
                   double* eta, cudaStream_t st, MState& S, CapStats& cap) {
  const int m = c.m;
  const long long tiles = (c.n + kMmaThreads - 1) / kMmaThreads;
  const int ga = (int)std::min<long long>(tiles, kAsmBlocks), gp = (int)std::min<long long>(tiles, kPassBlocks);
  const Kernels k = pick_kernels<G>(m);
  const size_t smem_g = assemble_smem(m, mma_bucket(m), true), smem = assemble_smem(m, mma_bucket(m), false);
  STT_TRY(check_cuda(cudaFuncSetAttribute((const void*)k.assemble, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_g),
                     "mma: assemble shared memory"));
  STT_TRY(check_cuda(cudaMemsetAsync(w.counters, 0, 4 * sizeof(unsigned), st), "mma: counters"));
  mma_init_kernel<<<gp, kMmaThreads, 0, st>>>(c.n, c.alfa, c.beta, x, xsi, eta);
  STT_TRY(check_launch("mma_init_kernel"));
  init_state(D, S);

  // results of one fetch: the assemble's [gvec | h | A | ss | mx] or the search's
  // [gvec | ss | mx] with the step's [3 maxima | steg] behind it
  const size_t nres = (size_t)m * m + 2 * m + 2;
  std::vector<double> R(std::max(nres, (size_t)m + 6)), gvec(m), h(m), A((size_t)m * m);
  auto fetch = [&](size_t count, const char* what) -> int {
    STT_TRY(check_cuda(cudaMemcpyAsync(R.data(), w.res, 8 * count, cudaMemcpyDeviceToHost, st), what));
    return check_cuda(cudaStreamSynchronize(st), what);
  };
  int pend = 0;
  double t_pend = 0.0, eps_pend = 0.0;
  // gvec at the current point: formed by the first assemble, then taken from each
  // accepted line-search candidate, whose point the next assemble starts from
  bool have_g = false;
  auto assemble = [&](double epsi, double& ssn, double& mxn) -> int {
    const int need_g = have_g ? 0 : 1;
    k.assemble<<<ga, kMmaThreads, need_g ? smem_g : smem, st>>>(c, x, xsi, eta, w.dx, pend, t_pend, eps_pend,
                                                                mvec(S.lam), epsi, need_g, w.partials);
    pend = 0;
    STT_TRY(check_launch("mma_assemble_kernel"));
    const int kp = assemble_kp(m), per = kMmaThreads / 32;
    mma_fold_kernel<<<(kp + per - 1) / per, kMmaThreads, 0, st>>>(w.partials, ga, m, w.res);
    STT_TRY(check_launch("mma_fold_kernel"));
    STT_TRY(fetch(nres, "mma: assemble"));
    if (!have_g) std::copy(R.begin(), R.begin() + m, gvec.begin());
    have_g = true;
    std::copy(R.begin() + m, R.begin() + 2 * m, h.begin());
    std::copy(R.begin() + 2 * m, R.begin() + 2 * m + (size_t)m * m, A.begin());
    ssn = R[nres - 2];
    mxn = ssn != ssn ? NAN : R[nres - 1];
    return STT_OK;
  };

  double epsi = 1.0;
  while (epsi > epsimin) {
    double ssn, mxn;
    STT_TRY(assemble(epsi, ssn, mxn));
    double ssm = 0.0, mxm = -INFINITY;
    resid_m(D, S, gvec.data(), epsi, ssm, mxm);
    double residunorm = std::sqrt(ssn + ssm), residumax = hmax(mxn, mxm);
    int ittt = 0;
    bool fresh = true;
    while (residumax > 0.9 * epsi && ittt < kMaxNewton) {
      ++ittt;
      ++cap.steps;
      if (!fresh) STT_TRY(assemble(epsi, ssn, mxn));
      fresh = false;
      // The bordered system [[diag(diaglamyi) + A, a], [a^T, -zet/z]] [dlam; dz] =
      // [dellam + dely/diagy - h; delz] (sttopt/mma.py:474-489).
      const MNewton N = newton_m(D, S, gvec.data(), epsi);
      const int M1 = m + 1;
      std::vector<double> AA((size_t)M1 * M1), bb(M1);
      for (int i = 0; i < m; ++i) {
        for (int kk = 0; kk < m; ++kk) AA[(size_t)i * M1 + kk] = A[(size_t)i * m + kk];
        AA[(size_t)i * M1 + i] = N.diaglamyi[i] + A[(size_t)i * m + i];
        AA[(size_t)i * M1 + m] = D.a[i];
        AA[(size_t)m * M1 + i] = D.a[i];
        bb[i] = N.dellam[i] + N.dely[i] / N.diagy[i] - h[i];
      }
      AA[(size_t)m * M1 + m] = -S.zet / S.z;
      bb[m] = N.delz;
      if (!dense_solve(AA, bb, M1)) return set_error(STT_ERR_BREAKDOWN, "mma: singular Newton system in subsolv");
      MStep T;
      T.dlam.assign(bb.begin(), bb.begin() + m);
      T.dz = bb[m];
      // The step pass forms steg on the device and the line search's first candidate
      // (t = steg) is evaluated right behind it: one sync for both.  The step's results sit
      // behind the search's in res: [search (m + 2) | step maxima (3) | steg].
      const double stm_m = step_m(D, S, N, epsi, T);
      const MVec lam_now = mvec(S.lam), dlam = mvec(T.dlam);
      double* const res_step = w.res + m + 2;
      k.step<<<gp, kMmaThreads, 0, st>>>(c, x, xsi, eta, lam_now, dlam, epsi, stm_m, w.dx, w.partials,
                                         w.counters + 1, res_step);
      STT_TRY(check_launch("mma_step_kernel"));
      k.search<<<gp, kMmaThreads, 0, st>>>(c, x, xsi, eta, w.dx, 0.0, res_step + 3, lam_now, dlam, epsi, 1,
                                           w.partials, w.counters + 2, w.res);
      STT_TRY(check_launch("mma_search_kernel"));
      STT_TRY(fetch((size_t)m + 6, "mma: step and first candidate"));
      const double steg = R[m + 5];  // 1 / max(stmalfa, stmbeta, stmxx, 1), as formed on the device
      // Backtracking on the residual norm: the first halving whose norm does not exceed
      // the current one, else the last (sttopt/mma.py:297-343).
      MState C;
      double resinew = 0.0, mxc = 0.0, t = 0.0;
      for (int jj = 0; jj < kMaxHalvings; ++jj) {
        t = steg / std::ldexp(1.0, jj);
        C = moved(S, T, t);
        ++cap.tries;
        if (jj > 0) {
          k.search<<<gp, kMmaThreads, 0, st>>>(c, x, xsi, eta, w.dx, t, nullptr, lam_now, dlam, epsi, 1, w.partials,
                                               w.counters + 2, w.res);
          STT_TRY(check_launch("mma_search_kernel"));
          STT_TRY(fetch((size_t)m + 2, "mma: line search"));
        }
        double ssc = R[m], mxcn = ssc != ssc ? NAN : R[m + 1], ssmc = 0.0, mxmc = -INFINITY;
        resid_m(D, C, R.data(), epsi, ssmc, mxmc);
        resinew = std::sqrt(ssc + ssmc);
        mxc = hmax(mxcn, mxmc);
        if (!(resinew > residunorm)) break;
      }
      S = C;
      std::copy(R.begin(), R.begin() + m, gvec.begin());  // the accepted candidate's gvec
      pend = 1;
      t_pend = t;
      eps_pend = epsi;
      residunorm = resinew;
      residumax = mxc;
    }
    if (ittt > kMaxNewton - 2) {
      ++cap.hits;
      cap.epsi = epsi;
    }
    epsi = 0.1 * epsi;
  }
  if (pend) {
    mma_apply_kernel<<<gp, kMmaThreads, 0, st>>>(c.n, c.alfa, c.beta, w.dx, t_pend, eps_pend, x, xsi, eta);
    STT_TRY(check_launch("mma_apply_kernel"));
  }
  return STT_OK;
}

// subsolv for m >= n (sttopt/mma.py:490-516, the elimination onto dx): n <= m variables,
// so the whole solve runs in the library's host code on host copies of the subproblem.
int host_subsolv(int m, int n, double epsimin, const std::vector<double>& low, const std::vector<double>& upp,
                 const std::vector<double>& alfa, const std::vector<double>& beta, const std::vector<double>& p0,
                 const std::vector<double>& q0, const std::vector<double>& P, const std::vector<double>& Q,
                 const MData& D, std::vector<double>& x, std::vector<double>& xsi, std::vector<double>& eta,
                 MState& S, CapStats& cap) {
  x.resize(n);
  xsi.resize(n);
  eta.resize(n);
  for (int j = 0; j < n; ++j) {
    x[j] = 0.5 * (alfa[j] + beta[j]);
    xsi[j] = std::max(1.0 / (x[j] - alfa[j]), 1.0);
    eta[j] = std::max(1.0 / (beta[j] - x[j]), 1.0);
  }
  init_state(D, S);
  std::vector<double> gvec(m);
  // The full residual's sum of squares and max at a point, with gvec left in gvec.
  auto residual = [&](const std::vector<double>& xx, const std::vector<double>& xs, const std::vector<double>& et,
                      const MState& St, double epsi, double& norm, double& mx) {
    double ss = 0.0;
    mx = -INFINITY;
    for (int i = 0; i < m; ++i) gvec[i] = 0.0;
    for (int j = 0; j < n; ++j) {
      const double ux1 = upp[j] - xx[j], xl1 = xx[j] - low[j];
      double plam = p0[j], qlam = q0[j];
      for (int i = 0; i < m; ++i) {
        plam += St.lam[i] * P[(size_t)i * n + j];
        qlam += St.lam[i] * Q[(size_t)i * n + j];
        gvec[i] += P[(size_t)i * n + j] * (1.0 / ux1) + Q[(size_t)i * n + j] * (1.0 / xl1);
      }
      const double rex = plam / (ux1 * ux1) - qlam / (xl1 * xl1) - xs[j] + et[j];
      const double r1 = xs[j] * (xx[j] - alfa[j]) - epsi, r2 = et[j] * (beta[j] - xx[j]) - epsi;
      ss += rex * rex + r1 * r1 + r2 * r2;
      mx = hmax(mx, hmax(std::fabs(rex), hmax(std::fabs(r1), std::fabs(r2))));
    }
    double ssm = 0.0, mxm = -INFINITY;
    resid_m(D, St, gvec.data(), epsi, ssm, mxm);
    norm = std::sqrt(ss + ssm);
    mx = hmax(mx, mxm);
  };
  double epsi = 1.0;
  std::vector<double> GG((size_t)m * n), delx(n), diagx(n), dx(n), dxsi(n), deta(n);
  while (epsi > epsimin) {
    double residunorm, residumax;
    residual(x, xsi, eta, S, epsi, residunorm, residumax);
    int ittt = 0;
    while (residumax > 0.9 * epsi && ittt < kMaxNewton) {
      ++ittt;
      ++cap.steps;
      for (int i = 0; i < m; ++i) gvec[i] = 0.0;
      for (int j = 0; j < n; ++j) {
        const double ux1 = upp[j] - x[j], xl1 = x[j] - low[j];
        const double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
        double plam = 0.0, qlam = 0.0;
        for (int i = 0; i < m; ++i) {
          const double Pij = P[(size_t)i * n + j], Qij = Q[(size_t)i * n + j];
          plam += S.lam[i] * Pij;
          qlam += S.lam[i] * Qij;
          gvec[i] += Pij * (1.0 / ux1) + Qij * (1.0 / xl1);
          GG[(size_t)i * n + j] = Pij * (1.0 / ux2) - Qij * (1.0 / xl2);
        }
        plam = p0[j] + plam;
        qlam = q0[j] + qlam;
        const double dpsidx = plam / ux2 - qlam / xl2;
        delx[j] = dpsidx - epsi / (x[j] - alfa[j]) + epsi / (beta[j] - x[j]);
        diagx[j] = 2.0 * (plam / (ux1 * ux2) + qlam / (xl1 * xl2)) + xsi[j] / (x[j] - alfa[j]) +
                   eta[j] / (beta[j] - x[j]);
      }
      const MNewton N = newton_m(D, S, gvec.data(), epsi);
      std::vector<double> dellamyi(m), ainv(m);
      for (int i = 0; i < m; ++i) {
        dellamyi[i] = N.dellam[i] + N.dely[i] / N.diagy[i];
        ainv[i] = 1.0 / N.diaglamyi[i];
      }
      // [[diag(diagx) + GG^T diag(1/diaglamyi) GG, axz], [axz^T, azz]] [dx; dz] = [-bx; -bz]
      const int N1 = n + 1;
      std::vector<double> AA((size_t)N1 * N1, 0.0), bb(N1);
      double azz = S.zet / S.z, bz = N.delz;
      for (int i = 0; i < m; ++i) {
        azz += D.a[i] * (D.a[i] / N.diaglamyi[i]);
        bz -= D.a[i] * (dellamyi[i] / N.diaglamyi[i]);
      }
      for (int p = 0; p < n; ++p) {
        double axz = 0.0, bx = delx[p];
        for (int i = 0; i < m; ++i) {
          axz -= GG[(size_t)i * n + p] * (D.a[i] / N.diaglamyi[i]);
          bx += GG[(size_t)i * n + p] * (dellamyi[i] / N.diaglamyi[i]);
        }
        for (int q = 0; q < n; ++q) {
          double v = p == q ? diagx[p] : 0.0;
          for (int i = 0; i < m; ++i) v += GG[(size_t)i * n + p] * ainv[i] * GG[(size_t)i * n + q];
          AA[(size_t)p * N1 + q] = v;
        }
        AA[(size_t)p * N1 + n] = axz;
        AA[(size_t)n * N1 + p] = axz;
        bb[p] = -bx;
      }
      AA[(size_t)n * N1 + n] = azz;
      bb[n] = -bz;
      if (!dense_solve(AA, bb, N1)) return set_error(STT_ERR_BREAKDOWN, "mma: singular Newton system in subsolv");
      MStep T;
      for (int j = 0; j < n; ++j) dx[j] = bb[j];
      T.dz = bb[n];
      T.dlam.resize(m);
      for (int i = 0; i < m; ++i) {
        double g = 0.0;
        for (int j = 0; j < n; ++j) g += GG[(size_t)i * n + j] * dx[j];
        T.dlam[i] = g / N.diaglamyi[i] - T.dz * (D.a[i] / N.diaglamyi[i]) + dellamyi[i] / N.diaglamyi[i];
      }
      double stmalfa = -INFINITY, stmbeta = -INFINITY, stmxx = step_m(D, S, N, epsi, T);
      for (int j = 0; j < n; ++j) {
        const double xa = x[j] - alfa[j], bx = beta[j] - x[j];
        dxsi[j] = -xsi[j] + epsi / xa - (xsi[j] * dx[j]) / xa;
        deta[j] = -eta[j] + epsi / bx + (eta[j] * dx[j]) / bx;
        stmalfa = hmax(stmalfa, (-1.01 * dx[j]) / xa);
        stmbeta = hmax(stmbeta, (1.01 * dx[j]) / bx);
        stmxx = hmax(stmxx, hmax((-1.01 * dxsi[j]) / xsi[j], (-1.01 * deta[j]) / eta[j]));
      }
      const double steg = 1.0 / hmax(hmax(hmax(stmalfa, stmbeta), stmxx), 1.0);
      MState C;
      std::vector<double> xc(n), xsc(n), etc(n);
      double resinew = 0.0, mxc = 0.0;
      for (int jj = 0; jj < kMaxHalvings; ++jj) {
        const double t = steg / std::ldexp(1.0, jj);
        C = moved(S, T, t);
        ++cap.tries;
        for (int j = 0; j < n; ++j) {
          xc[j] = x[j] + t * dx[j];
          xsc[j] = xsi[j] + t * dxsi[j];
          etc[j] = eta[j] + t * deta[j];
        }
        residual(xc, xsc, etc, C, epsi, resinew, mxc);
        if (!(resinew > residunorm)) break;
      }
      S = C;
      x = xc;
      xsi = xsc;
      eta = etc;
      residunorm = resinew;
      residumax = mxc;
    }
    if (ittt > kMaxNewton - 2) {
      ++cap.hits;
      cap.epsi = epsi;
    }
    epsi = 0.1 * epsi;
  }
  return STT_OK;
}

}  // namespace
}  // namespace stt

// ---- C ABI ------------------------------------------------------------------------------

namespace stt {
namespace {

int d2h(std::vector<double>& dst, const double* src, size_t count, cudaStream_t st) {
  dst.resize(count);
  if (!count) return STT_OK;
  return check_cuda(cudaMemcpyAsync(dst.data(), src, 8 * count, cudaMemcpyDeviceToHost, st), "mma: copy to host");
}
int h2d(double* dst, const std::vector<double>& src, cudaStream_t st) {
  if (src.empty()) return STT_OK;
  return check_cuda(cudaMemcpyAsync(dst, src.data(), 8 * src.size(), cudaMemcpyHostToDevice, st), "mma: copy to device");
}
// Rows of an m x n matrix with row stride ld, gathered to a dense host m x n.
int d2h_rows(std::vector<double>& dst, const double* src, int m, long long n, long long ld, cudaStream_t st) {
  dst.resize((size_t)m * n);
  for (int i = 0; i < m; ++i)
    STT_TRY(check_cuda(cudaMemcpyAsync(dst.data() + (size_t)i * n, src + (size_t)i * ld, 8 * (size_t)n,
                                       cudaMemcpyDeviceToHost, st),
                       "mma: copy to host"));
  return STT_OK;
}

void write_m(const MState& S, int m, double* y, double* z, double* lam, double* mu, double* zet, double* s) {
  std::copy(S.y.begin(), S.y.end(), y);
  std::copy(S.lam.begin(), S.lam.end(), lam);
  std::copy(S.mu.begin(), S.mu.end(), mu);
  std::copy(S.s.begin(), S.s.end(), s);
  *z = S.z;
  *zet = S.zet;
  (void)m;
}

int check_sizes(int m, long long n, size_t ws_bytes) {
  if (m < 1 || n < 1) return set_error(STT_ERR_INVALID, "mma: m and n must be positive");
  if (m < n && m > kMmaMaxM) return set_error(STT_ERR_INVALID, "mma: at most 64 constraints when m < n");
  if (n > (1LL << 40)) return set_error(STT_ERR_INVALID, "mma: n too large");
  if (ws_bytes < carve(m, n, nullptr, nullptr)) return set_error(STT_ERR_WORKSPACE, "mma: workspace too small");
  return STT_OK;
}

}  // namespace
}  // namespace stt

using namespace stt;

extern "C" size_t stt_mma_workspace_bytes(int m, long long n) {
  if (m < 1 || n < 1) return 0;
  return carve(m, n, nullptr, nullptr);
}

extern "C" int stt_mma_sub(int m, long long n, int iteration, const double* xval, const double* xmin,
                           const double* xmax, const double* xold1, const double* xold2, const double* df0dx,
                           const double* fval, const double* dfdx, long long dfdx_ld, double* low, double* upp,
                           double a0, const double* a, const double* c, const double* d, const double* asyinit,
                           double asyinit_v, const double* asyclamp_min, double asyclamp_min_v,
                           const double* asyclamp_max, double asyclamp_max_v, const double* move, double move_v,
                           double raa0, double albefa, double asyincr, double asydecr, double* xmma, double* xsi,
                           double* eta, double* ymma, double* zmma, double* lam, double* mu, double* zet, double* s,
                           int* counts, double* cap_epsi, void* ws, size_t ws_bytes, stt_stream_t stream) {
  STT_TRY(check_sizes(m, n, ws_bytes));
  if (!xval || !xmin || !xmax || !xold1 || !xold2 || !df0dx || !fval || !dfdx || !low || !upp || !a || !c || !d ||
      !xmma || !xsi || !eta || !ymma || !zmma || !lam || !mu || !zet || !s || !ws || dfdx_ld < n)
    return set_error(STT_ERR_INVALID, "stt_mma_sub: null pointer or bad stride");
  cudaStream_t st = (cudaStream_t)stream;
  MmaWs w;
  carve(m, n, static_cast<char*>(ws), &w);
  const int gp = (int)std::min<long long>((n + kMmaThreads - 1) / kMmaThreads, kPassBlocks);
  mma_setup_kernel<<<gp, kMmaThreads, 0, st>>>(n, iteration, xval, xmin, xmax, xold1, xold2, low, upp,
                                               {asyinit, asyinit_v}, {asyclamp_min, asyclamp_min_v},
                                               {asyclamp_max, asyclamp_max_v}, {move, move_v}, raa0, albefa, asyincr,
                                               asydecr, w.alfa, w.beta, w.rxm);
  STT_TRY(check_launch("mma_setup_kernel"));
  MmaCols cols{n, dfdx_ld, m, low, upp, w.alfa, w.beta, nullptr, nullptr, nullptr, nullptr, xval, df0dx, dfdx, w.rxm};
  std::vector<double> b(m);
  MState S;
  CapStats cap;
  if (m < n) {
    STT_TRY(check_cuda(cudaMemsetAsync(w.counters, 0, 4 * sizeof(unsigned), st), "mma: counters"));
    const Kernels k = pick_kernels<true>(m);
    k.search<<<gp, kMmaThreads, 0, st>>>(cols, xval, nullptr, nullptr, nullptr, 0.0, nullptr, MVec{}, MVec{}, 0.0,
                                         0, w.partials, w.counters + 3, w.res);
    STT_TRY(check_launch("mma_search_kernel"));
    std::vector<double> g;
    STT_TRY(d2h(g, w.res, (size_t)m, st));
    STT_TRY(check_cuda(cudaStreamSynchronize(st), "mma: b"));
    for (int i = 0; i < m; ++i) b[i] = g[i] - fval[i];
    const MData D{m, a0, a, b.data(), c, d};
    STT_TRY(device_subsolv<true>(cols, D, 1e-7, w, xmma, xsi, eta, st, S, cap));
  } else {
    const int nn = (int)n;
    std::vector<double> hl, hu, ha, hb, hr, hx, hg0, hg;
    STT_TRY(d2h(hl, low, nn, st));
    STT_TRY(d2h(hu, upp, nn, st));
    STT_TRY(d2h(ha, w.alfa, nn, st));
    STT_TRY(d2h(hb, w.beta, nn, st));
    STT_TRY(d2h(hr, w.rxm, nn, st));
    STT_TRY(d2h(hx, xval, nn, st));
    STT_TRY(d2h(hg0, df0dx, nn, st));
    STT_TRY(d2h_rows(hg, dfdx, m, n, dfdx_ld, st));
    STT_TRY(check_cuda(cudaStreamSynchronize(st), "mma: copy to host"));
    std::vector<double> p0(nn), q0(nn), P((size_t)m * nn), Q((size_t)m * nn);
    for (int j = 0; j < nn; ++j) {
      const double ux1 = hu[j] - hx[j], xl1 = hx[j] - hl[j];
      const double pp = std::max(hg0[j], 0.0), qq = std::max(-hg0[j], 0.0);
      const double pq = 0.001 * (pp + qq) + hr[j];
      p0[j] = (pp + pq) * (ux1 * ux1);
      q0[j] = (qq + pq) * (xl1 * xl1);
      for (int i = 0; i < m; ++i) {
        const double g = hg[(size_t)i * nn + j];
        const double pi = std::max(g, 0.0), qi = std::max(-g, 0.0), pqi = 0.001 * (pi + qi) + hr[j];
        P[(size_t)i * nn + j] = (pi + pqi) * (ux1 * ux1);
        Q[(size_t)i * nn + j] = (qi + pqi) * (xl1 * xl1);
      }
    }
    for (int i = 0; i < m; ++i) {
      double g1 = 0.0, g2 = 0.0;
      for (int j = 0; j < nn; ++j) {
        g1 += P[(size_t)i * nn + j] * (1.0 / (hu[j] - hx[j]));
        g2 += Q[(size_t)i * nn + j] * (1.0 / (hx[j] - hl[j]));
      }
      b[i] = g1 + g2 - fval[i];
    }
    const MData D{m, a0, a, b.data(), c, d};
    std::vector<double> x, xs, et;
    STT_TRY(host_subsolv(m, nn, 1e-7, hl, hu, ha, hb, p0, q0, P, Q, D, x, xs, et, S, cap));
    STT_TRY(h2d(xmma, x, st));
    STT_TRY(h2d(xsi, xs, st));
    STT_TRY(h2d(eta, et, st));
  }
  STT_TRY(check_cuda(cudaStreamSynchronize(st), "stt_mma_sub"));
  write_m(S, m, ymma, zmma, lam, mu, zet, s);
  if (counts) {
    counts[0] = cap.hits;
    counts[1] = cap.steps;
    counts[2] = cap.tries;
  }
  if (cap_epsi) *cap_epsi = cap.epsi;
  return STT_OK;
}

extern "C" int stt_mma_subsolv(int m, long long n, double epsimin, const double* low, const double* upp,
                               const double* alfa, const double* beta, const double* p0, const double* q0,
                               const double* P, const double* Q, long long ld, double a0, const double* a,
                               const double* b, const double* c, const double* d, double* xmma, double* xsi,
                               double* eta, double* ymma, double* zmma, double* lam, double* mu, double* zet, double* s,
                               int* counts, double* cap_epsi, void* ws, size_t ws_bytes, stt_stream_t stream) {
  STT_TRY(check_sizes(m, n, ws_bytes));
  if (!low || !upp || !alfa || !beta || !p0 || !q0 || !P || !Q || !a || !b || !c || !d || !xmma || !xsi || !eta ||
      !ymma || !zmma || !lam || !mu || !zet || !s || !ws || ld < n)
    return set_error(STT_ERR_INVALID, "stt_mma_subsolv: null pointer or bad stride");
  cudaStream_t st = (cudaStream_t)stream;
  MmaWs w;
  carve(m, n, static_cast<char*>(ws), &w);
  const MData D{m, a0, a, b, c, d};
  MState S;
  CapStats cap;
  if (m < n) {
    MmaCols cols{n, ld, m, low, upp, alfa, beta, p0, q0, P, Q, nullptr, nullptr, nullptr, nullptr};
    STT_TRY(device_subsolv<false>(cols, D, epsimin, w, xmma, xsi, eta, st, S, cap));
  } else {
    const int nn = (int)n;
    std::vector<double> hl, hu, ha, hb, hp, hq, hP, hQ, x, xs, et;
    STT_TRY(d2h(hl, low, nn, st));
    STT_TRY(d2h(hu, upp, nn, st));
    STT_TRY(d2h(ha, alfa, nn, st));
    STT_TRY(d2h(hb, beta, nn, st));
    STT_TRY(d2h(hp, p0, nn, st));
    STT_TRY(d2h(hq, q0, nn, st));
    STT_TRY(d2h_rows(hP, P, m, n, ld, st));
    STT_TRY(d2h_rows(hQ, Q, m, n, ld, st));
    STT_TRY(check_cuda(cudaStreamSynchronize(st), "mma: copy to host"));
    STT_TRY(host_subsolv(m, nn, epsimin, hl, hu, ha, hb, hp, hq, hP, hQ, D, x, xs, et, S, cap));
    STT_TRY(h2d(xmma, x, st));
    STT_TRY(h2d(xsi, xs, st));
    STT_TRY(h2d(eta, et, st));
  }
  STT_TRY(check_cuda(cudaStreamSynchronize(st), "stt_mma_subsolv"));
  write_m(S, m, ymma, zmma, lam, mu, zet, s);
  if (counts) {
    counts[0] = cap.hits;
    counts[1] = cap.steps;
    counts[2] = cap.tries;
  }
  if (cap_epsi) *cap_epsi = cap.epsi;
  return STT_OK;
}
