// Multigrid cycle kernels: damped-Jacobi sweeps and residuals on level 0 (density
// tiles) and on stencil levels, full-weighting restriction, bilinear prolongation,
// and the block-banded coarse solve.  Templated on the cycle precision T.
//
// Reference: torch_mg.VCycle._smooth/_cycle (sttopt/torch_mg.py:440-476), transfers
// _interp_axis/_restrict_axis/_on_node_grid (:75-109).
#pragma once

#include "common.cuh"
#include "q4.cuh"

namespace stt {

enum SweepMode { SW_FIRST = 0, SW_SWEEP = 1, SW_RESID = 2, SW_APPLY = 3 };

// ---- level 0: density-scaled Q4 tiles ------------------------------------------
//   SW_FIRST: out = (omega * b) / diag               (sweep from x = 0)
//   SW_SWEEP: out = x + (omega * (b - A x)) / diag
//   SW_RESID: out = b - A x
//   SW_APPLY: out = A x
// A is the projected operator P(K P .) (+ lumped reaction); x is read projected.
template <int D, typename T, int MODE>
__global__ void __launch_bounds__(kNT) l0_sweep_kernel(
    const T* __restrict__ x, long long x_rs, const T* __restrict__ b, long long b_rs,
    T* __restrict__ out, long long o_rs, const T* __restrict__ rho, long long rho_rs,
    const T* __restrict__ rdiag, long long rd_rs, const uint8_t* __restrict__ fixed,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, int nelx,
    int nely, T omega, KEq<D, T> ke) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  __shared__ Q4Smem<D, T, T> sm;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const int r0 = blockIdx.y * kTY, c0 = blockIdx.x * kTX;
  load_rho_tile<D, T, T>(sm, rho + (size_t)h * rho_rs, r0, c0, nelx, nely);
  const T* xs = x + (size_t)s * x_rs;
  if (MODE != SW_FIRST) {
    load_u_tile<D, T, T>(sm, r0, c0, nnx, nny, [&](int node, T(&v)[D]) {
      load_node<D, T>(xs, node, v);
#pragma unroll
      for (int j = 0; j < D; ++j)
        if (is_fixed(fixed, node, j)) v[j] = T(0);
    });
  }
  __syncthreads();
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int r = r0 + ty, c = c0 + tx;
  if (r >= nny || c >= nnx) return;
  const int node = r * nnx + c;
  const T* rd = rdiag + (size_t)h * rd_rs + (size_t)node * D;
  const uint8_t fl = fixed[node];
  T Ax[D], bv[D], res[D];
  if (MODE != SW_FIRST) {
    tile_Ku<D, T, T>(sm, ty, tx, ke, Ax);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      Ax[i] = fma(__ldg(rd + i), sm.u[ty + 1][tx + 1][i], Ax[i]);
      if ((fl >> i) & 1) Ax[i] = T(0);
    }
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) Ax[i] = T(0);
  }
  if (MODE != SW_APPLY) load_node<D, T>(b + (size_t)s * b_rs, node, bv);
  if (MODE == SW_FIRST || MODE == SW_SWEEP) {
    T dg[D];
    tile_diag<D, T, T>(sm, ty, tx, ke, dg);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      dg[i] += __ldg(rd + i);
      if ((fl >> i) & 1) dg[i] = T(1);
      const T xo = MODE == SW_FIRST ? T(0) : sm.u[ty + 1][tx + 1][i];
      res[i] = xo + (omega * (bv[i] - Ax[i])) / dg[i];
    }
  } else if (MODE == SW_RESID) {
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = bv[i] - Ax[i];
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = Ax[i];
  }
  store_node<D, T>(out + (size_t)s * o_rs, node, res);
}

// ---- stencil levels -------------------------------------------------------------

// (A x) at node (r, c) from the symmetric half stencil (centre, E, S, SE, SW blocks of
// this node; W, N, NW, NE couplings are the transposed E, S, SE, SW blocks of the
// neighbours).  st is this hierarchy row's [NS][nnode] array, x this row's vector.
template <int D, typename T>
STT_DEV void stencil_Ax(const T* __restrict__ st, long long nnode, int nnx, int nny, int r, int c,
                        const T* __restrict__ x, T (&acc)[D]) {
  constexpr int DD = D * D;
#pragma unroll
  for (int i = 0; i < D; ++i) acc[i] = T(0);
  const long long n = (long long)r * nnx + c;
  const int odr[5] = {0, 0, 1, 1, 1}, odc[5] = {0, 1, 0, 1, -1};
#pragma unroll
  for (int blk = 0; blk < 5; ++blk) {
    const int mr = r + odr[blk], mc = c + odc[blk];
    if (mr >= nny || mc < 0 || mc >= nnx) continue;
    const long long m = (long long)mr * nnx + mc;
    T xm[D];
    load_node<D, T>(x, (int)m, xm);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j)
        acc[i] = fma(__ldg(st + (size_t)(blk * DD + i * D + j) * nnode + n), xm[j], acc[i]);
  }
  // transposed couplings held by the neighbours: W (E block), N (S), NW (SE), NE (SW)
  const int tdr[4] = {0, -1, -1, -1}, tdc[4] = {-1, 0, -1, 1}, tblk[4] = {1, 2, 3, 4};
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int mr = r + tdr[t], mc = c + tdc[t];
    if (mr < 0 || mc < 0 || mc >= nnx) continue;
    const long long m = (long long)mr * nnx + mc;
    T xm[D];
    load_node<D, T>(x, (int)m, xm);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j)
        acc[i] = fma(__ldg(st + (size_t)(tblk[t] * DD + j * D + i) * nnode + m), xm[j], acc[i]);
  }
}

template <int D, typename T, int MODE>
__global__ void __launch_bounds__(256) st_sweep_kernel(
    const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ out, long long vec_rs,
    const T* __restrict__ st, const uint8_t* __restrict__ fixed, int nnx, int nny,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, T omega) {
  constexpr int NS = 5 * D * D;
  const int s = blockIdx.y;
  if (rst && !rst[s].active) return;
  const long long nnode = (long long)nnx * nny;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  const int h = hier_row(row_map, hrows, s);
  const T* sth = st + (size_t)h * NS * nnode;
  const int r = (int)(n / nnx), c = (int)(n - (long long)r * nnx);
  const uint8_t fl = fixed[n];
  T Ax[D], bv[D], res[D];
  if (MODE != SW_FIRST) {
    stencil_Ax<D, T>(sth, nnode, nnx, nny, r, c, x + (size_t)s * vec_rs, Ax);
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) Ax[i] = T(0);
  }
  if (MODE != SW_APPLY) load_node<D, T>(b + (size_t)s * vec_rs, (int)n, bv);
  if (MODE == SW_FIRST || MODE == SW_SWEEP) {
    T xo[D];
    if (MODE == SW_SWEEP) load_node<D, T>(x + (size_t)s * vec_rs, (int)n, xo);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T dg = __ldg(sth + (size_t)(i * D + i) * nnode + n);
      if ((fl >> i) & 1) dg = T(1);
      const T x0 = MODE == SW_FIRST ? T(0) : xo[i];
      res[i] = x0 + (omega * (bv[i] - Ax[i])) / dg;
    }
  } else if (MODE == SW_RESID) {
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = bv[i] - Ax[i];
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = Ax[i];
  }
  store_node<D, T>(out + (size_t)s * vec_rs, (int)n, res);
}

// ---- transfers -------------------------------------------------------------------

// One axis of full weighting at coarse index I (nc coarse intervals), in the
// reference's order: (block I weighted 1 - j/k) + (block I-1 weighted j/k), plus the
// last fine value on the last coarse node.
template <typename T, typename F>
STT_DEV T restrict1(F fetch, int I, int k, int nc) {
  if (k == 1) return fetch(I);
  T lo = T(0), hi = T(0);
  if (I < nc) {
    for (int j = 0; j < k; ++j) lo += fetch(k * I + j) * T(1.0 - (double)j / k);
  }
  if (I >= 1) {
    for (int j = 1; j < k; ++j) hi += fetch(k * (I - 1) + j) * T((double)j / k);
  }
  T out = lo + hi;
  if (I == nc) out += fetch(k * nc);
  return out;
}

// rc = P_c (R r_f): x pass then y pass (torch_mg._on_node_grid with _restrict_axis).
template <int D, typename T>
__global__ void restrict_kernel(const T* __restrict__ rf, long long f_rs, int fnnx, T* __restrict__ rc,
                                long long c_rs, int cnnx, int cnny, int kx, int ky,
                                const uint8_t* __restrict__ cfixed, const RowState* __restrict__ rst) {
  const int s = blockIdx.y;
  if (rst && !rst[s].active) return;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= (long long)cnnx * cnny) return;
  const int R = (int)(n / cnnx), C = (int)(n - (long long)R * cnnx);
  const T* f = rf + (size_t)s * f_rs;
  const uint8_t fl = cfixed[n];
  T out[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    auto xpass = [&](int fr) -> T {
      return restrict1<T>([&](int fc) -> T { return __ldg(f + ((size_t)fr * fnnx + fc) * D + i); },
                          C, kx, cnnx - 1);
    };
    out[i] = ((fl >> i) & 1) ? T(0) : restrict1<T>(xpass, R, ky, cnny - 1);
  }
  store_node<D, T>(rc + (size_t)s * c_rs, (int)n, out);
}

// x_f += P_f (P e_c): bilinear interpolation, x pass then y pass (_interp_axis).
template <int D, typename T>
__global__ void prolong_add_kernel(const T* __restrict__ ec, long long c_rs, int cnnx,
                                   T* __restrict__ xf, long long f_rs, int fnnx, int fnny, int kx,
                                   int ky, const uint8_t* __restrict__ ffixed,
                                   const RowState* __restrict__ rst) {
  const int s = blockIdx.y;
  if (rst && !rst[s].active) return;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= (long long)fnnx * fnny) return;
  const int r = (int)(n / fnnx), c = (int)(n - (long long)r * fnnx);
  const int R = r / ky, jy = r - R * ky, C = c / kx, jx = c - C * kx;
  const T* e = ec + (size_t)s * c_rs;
  const uint8_t fl = ffixed[n];
  T* xs = xf + (size_t)s * f_rs;
  const T wx = T((double)jx / kx), wy = T((double)jy / ky);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    auto g = [&](int RR) -> T {
      const T a = __ldg(e + ((size_t)RR * cnnx + C) * D + i);
      if (jx == 0) return a;
      const T b = __ldg(e + ((size_t)RR * cnnx + C + 1) * D + i);
      return a * (T(1) - wx) + b * wx;
    };
    T v = g(R);
    if (jy != 0) v = v * (T(1) - wy) + g(R + 1) * wy;
    if ((fl >> i) & 1) v = T(0);
    xs[(size_t)n * D + i] += v;
  }
}

// ---- coarsest level: block-banded Cholesky solve (one CTA per batch row) ----------

template <int D, typename T>
__global__ void __launch_bounds__(256) coarse_solve_kernel(
    const T* __restrict__ b, T* __restrict__ x, long long rs, const double* __restrict__ blocks,
    int B, int nb, int by_col, int nnx, int nny, const uint8_t* __restrict__ fixed,
    double* __restrict__ scratch, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst) {
  extern __shared__ double csm[];
  double* vp = csm;      // previous block's solution
  double* tv = csm + B;  // right-hand side of the current block
  const int s = blockIdx.x;
  if (rst && !rst[s].active) return;
  const int h = hier_row(row_map, hrows, s);
  const double* bh = blocks + (size_t)h * nb * 4 * B * B;
  const long long nnode = (long long)nnx * nny, n = nnode * D, np = (long long)nb * B;
  double* y = scratch + (size_t)s * np;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  auto node_of = [&](long long P, int& r, int& c, int& i) {
    const long long nd = P / D;
    i = (int)(P - nd * D);
    if (by_col) {
      c = (int)(nd / nny);
      r = (int)(nd - (long long)c * nny);
    } else {
      r = (int)(nd / nnx);
      c = (int)(nd - (long long)r * nnx);
    }
  };
  const T* bs = b + (size_t)s * rs;
  for (long long P = tid; P < np; P += blockDim.x) {
    double v = 0.0;
    if (P < n) {
      int r, c, i;
      node_of(P, r, c, i);
      v = (double)bs[((size_t)r * nnx + c) * D + i];
    }
    y[P] = v;
  }
  __syncthreads();
  auto gemv = [&](const double* M, const double* v, double* o, bool sub, const double* base) {
    // o[i] = (sub ? base[i] - (M v)[i] : (M v)[i]), M row-major B x B; warp per row
    for (int i = warp; i < B; i += nw) {
      double acc = 0.0;
      for (int l = lane; l < B; l += 32) acc = fma(M[(size_t)i * B + l], v[l], acc);
      acc = warp_sum(acc);
      if (lane == 0) o[i] = sub ? base[i] - acc : acc;
    }
  };
  // forward: y_k = Dinv_k (b_k - E_k y_{k-1})
  for (int k = 0; k < nb; ++k) {
    const double* blk = bh + (size_t)k * 4 * B * B;
    if (k == 0) {
      for (int i = tid; i < B; i += blockDim.x) tv[i] = y[i];
    } else {
      gemv(blk + 2 * (size_t)B * B, vp, tv, true, y + (size_t)k * B);
    }
    __syncthreads();
    gemv(blk, tv, vp, false, nullptr);
    __syncthreads();
    for (int i = tid; i < B; i += blockDim.x) y[(size_t)k * B + i] = vp[i];
    __syncthreads();
  }
  // backward: x_k = Dinv_k^T (y_k - E_{k+1}^T x_{k+1}); vp holds x_{k+1}
  for (int k = nb - 1; k >= 0; --k) {
    const double* blk = bh + (size_t)k * 4 * B * B;
    if (k == nb - 1) {
      for (int i = tid; i < B; i += blockDim.x) tv[i] = y[(size_t)k * B + i];
    } else {
      const double* nxt = bh + (size_t)(k + 1) * 4 * B * B;
      gemv(nxt + 3 * (size_t)B * B, vp, tv, true, y + (size_t)k * B);
    }
    __syncthreads();
    gemv(blk + (size_t)B * B, tv, vp, false, nullptr);
    __syncthreads();
    for (int i = tid; i < B; i += blockDim.x) y[(size_t)k * B + i] = vp[i];
    __syncthreads();
  }
  T* xs = x + (size_t)s * rs;
  for (long long P = tid; P < n; P += blockDim.x) {
    int r, c, i;
    node_of(P, r, c, i);
    const long long node = (long long)r * nnx + c;
    xs[node * D + i] = ((fixed[node] >> i) & 1) ? T(0) : T(y[P]);
  }
}

// ---- small vector kernels ---------------------------------------------------------

template <typename TI, typename TO>
__global__ void rows_convert_kernel(const TI* __restrict__ in, long long in_rs, TO* __restrict__ out,
                                    long long out_rs, long long n, const RowState* __restrict__ rst) {
  const int s = blockIdx.y;
  if (rst && !rst[s].active) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[(size_t)s * out_rs + i] = (TO)in[(size_t)s * in_rs + i];
}

template <typename T>
__global__ void rows_axpy_kernel(const T* __restrict__ a, T* __restrict__ y, long long rs, long long n,
                                 const RowState* __restrict__ rst) {
  const int s = blockIdx.y;
  if (rst && !rst[s].active) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[(size_t)s * rs + i] += a[(size_t)s * rs + i];
}

}  // namespace stt
