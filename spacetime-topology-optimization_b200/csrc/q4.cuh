// Level-0 (density-scaled Q4) operator: column-marching warps.
//
// K(rho) u is applied node by node with no atomics.  A warp owns a strip of 32 grid
// columns (lanes 1..30 produce output, lanes 0 and 31 are the strip's halo) and marches
// down kQRows grid rows.  Each lane streams its own node (one 64/128-bit coalesced load
// per row) and element density, takes its left/right neighbours' values with warp
// shuffles, and keeps a sliding 3-row window in registers; per output node it sums the
// four elements around it, rho_e * (KE row of the node's corner) . u_e -- the
// reference's gather / (Ue @ KE) * density / index_add (sttopt/torch_fem.py:76-82) as a
// deterministic gather.  No shared memory and no block barrier on the streaming path:
// every warp keeps its loads in flight independently.
#pragma once

#include "common.cuh"

namespace stt {

constexpr int kQCols = 30;              // output columns per warp
constexpr int kQThreads = 128;          // threads per block of the marching kernels
constexpr int kQWarps = kQThreads / 32;  // warp strips per block
constexpr int kQRows = 32;              // grid rows per warp strip
constexpr int kQAhead = 4;              // rows loaded ahead of the one being computed

template <int D, typename T>
struct KEq {
  T v[(4 * D) * (4 * D)];
};

template <int D, typename T>
STT_DEV void load_node(const T* __restrict__ p, long long node, T (&v)[D]) {
  if constexpr (D == 2 && sizeof(T) == 8) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p) + node);
    v[0] = t.x;
    v[1] = t.y;
  } else if constexpr (D == 2 && sizeof(T) == 4) {
    const float2 t = __ldg(reinterpret_cast<const float2*>(p) + node);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    v[0] = __ldg(p + node);
  }
}

template <int D, typename T>
STT_DEV void store_node(T* __restrict__ p, long long node, const T (&v)[D]) {
  if constexpr (D == 2 && sizeof(T) == 8) {
    reinterpret_cast<double2*>(p)[node] = make_double2(v[0], v[1]);
  } else if constexpr (D == 2 && sizeof(T) == 4) {
    reinterpret_cast<float2*>(p)[node] = make_float2(v[0], v[1]);
  } else {
    p[node] = v[0];
  }
}

STT_DEV bool is_fixed(const uint8_t* fixed, long long node, int i) {
  return fixed != nullptr && ((__ldg(fixed + node) >> i) & 1);
}

// Grid of the column-marching kernels: x = groups of kQWarps warp strips of kQCols
// columns, y = kQRows-row bands, z = batch rows.
inline dim3 q4_grid(int nelx, int nely, int rows) {
  const int strips = (nelx + 1 + kQCols - 1) / kQCols;
  return dim3((strips + kQWarps - 1) / kQWarps, (nely + 1 + kQRows - 1) / kQRows, rows);
}

// Marches this warp down its strip.  `loadu(r, c, v)` fills node (r, c) and
// `loadr(r, c)` returns element (r, c)'s density; both are called only in-grid (zero
// outside).  `loadx(r, c)` returns the Extra of an output node.  `emit(r, c, Ku, dg,
// uc, ex)` is called for every in-grid output node with (K u) (when KU), diag(K) (when
// DG), the node's own input value and its Extra.
// Per-node values the emit step reads besides the window (right-hand side, flags ...),
// loaded kQAhead rows ahead with the window so their latency is hidden too.
struct NoExtra {};
struct FlagX {
  uint8_t fl;
};
template <int D, typename T>
struct RhsX {  // a right-hand side value and the node's fixed flags
  T b[D];
  uint8_t fl;
};

template <int D, typename T, bool KU, bool DG, typename Extra = NoExtra, typename LoadU, typename LoadR,
          typename LoadX, typename Emit>
STT_DEV void march(const KEq<D, T>& ke, int nnx, int nny, LoadU loadu, LoadR loadr, LoadX loadx, Emit emit) {
  // FP64: the element matrix is read from shared memory per use (volatile, so it is not
  // hoisted): DFMA takes no constant-bank operand and 64 doubles in registers would cost
  // occupancy.  FP32 reads it from the constant bank.
  constexpr bool kSmemKE = sizeof(T) == 8;
  __shared__ T kes[kSmemKE ? 16 * D * D : 1];
  if constexpr (kSmemKE) {
    for (int i = threadIdx.x; i < 16 * D * D; i += blockDim.x) kes[i] = ke.v[i];
    __syncthreads();
  }
  auto KV = [&](int idx) -> T {
    if constexpr (kSmemKE) return static_cast<const volatile T*>(kes)[idx];
    else return ke.v[idx];
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kQCols - 1 + lane;  // this lane's column
  const bool out_lane = lane >= 1 && lane <= kQCols && c < nnx;
  const int r0 = blockIdx.y * kQRows;
  const int r1 = min(r0 + kQRows, nny);
  const int nelx = nnx - 1, nely = nny - 1;
  const bool col_ok = c >= 0 && c < nnx;
  const bool ecol_ok = c >= 0 && c < nelx;
  auto U = [&](int r, T(&v)[D]) {
    if (KU && col_ok && r >= 0 && r < nny) {
      loadu(r, c, v);
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) v[d] = T(0);
    }
  };
  auto Rho = [&](int r) -> T { return (ecol_ok && r >= 0 && r < nely) ? loadr(r, c) : T(0); };
  // window: rows r-1 (a) and r (b) of u at columns c-1, c, c+1; densities of element
  // row r-1 at columns c-1, c
  T ua[D], ub[D], ual[D], uar[D], ubl[D], ubr[D];
  U(r0 - 1, ua);
  U(r0, ub);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    ual[d] = __shfl_up_sync(0xffffffffu, ua[d], 1);
    uar[d] = __shfl_down_sync(0xffffffffu, ua[d], 1);
    ubl[d] = __shfl_up_sync(0xffffffffu, ub[d], 1);
    ubr[d] = __shfl_down_sync(0xffffffffu, ub[d], 1);
  }
  T ra = Rho(r0 - 1);
  T ral = __shfl_up_sync(0xffffffffu, ra, 1);
  // prefetch queue: u rows r+1 .. r+kQAhead, density and extra rows r .. r+kQAhead-1
  T qu[kQAhead][D], qr[kQAhead];
  Extra qx[kQAhead];
  auto X = [&](int r) -> Extra { return (out_lane && r < r1) ? loadx(r, c) : Extra{}; };
#pragma unroll
  for (int k = 0; k < kQAhead; ++k) {
    U(r0 + 1 + k, qu[k]);
    qr[k] = Rho(r0 + k);
    qx[k] = X(r0 + k);
  }
  for (int rb0 = r0; rb0 < r1; rb0 += kQAhead) {
#pragma unroll
    for (int k = 0; k < kQAhead; ++k) {
      const int r = rb0 + k;
      T uc[D], ucl[D], ucr[D];
#pragma unroll
      for (int d = 0; d < D; ++d) uc[d] = qu[k][d];
      const T rb = qr[k];
      const Extra ex = qx[k];
      U(r + 1 + kQAhead, qu[k]);  // refill the slot
      qr[k] = Rho(r + kQAhead);
      qx[k] = X(r + kQAhead);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        ucl[d] = __shfl_up_sync(0xffffffffu, uc[d], 1);
        ucr[d] = __shfl_down_sync(0xffffffffu, uc[d], 1);
      }
      const T rbl = __shfl_up_sync(0xffffffffu, rb, 1);
      T acc[D], dg[D];
#pragma unroll
      for (int i = 0; i < D; ++i) acc[i] = dg[i] = T(0);
      // element with density rho in which the node is corner kc; its corners' values
      auto elem = [&](const T rho, int kc, const T(&bl)[D], const T(&br)[D], const T(&tr)[D],
                      const T(&tl)[D]) {
        if (KU) {
#pragma unroll
          for (int i = 0; i < D; ++i) {
            const int kr = (kc * D + i) * (4 * D);
            T sum = T(0);
#pragma unroll
            for (int j = 0; j < D; ++j) {
              sum = fma(KV(kr + 0 * D + j), bl[j], sum);
              sum = fma(KV(kr + 1 * D + j), br[j], sum);
              sum = fma(KV(kr + 2 * D + j), tr[j], sum);
              sum = fma(KV(kr + 3 * D + j), tl[j], sum);
            }
            acc[i] = fma(rho, sum, acc[i]);
          }
        }
        if (DG) {
#pragma unroll
          for (int i = 0; i < D; ++i) dg[i] = fma(rho, KV((kc * D + i) * (4 * D) + kc * D + i), dg[i]);
        }
      };
      elem(ral, corner_of(0, 0), ubl, ub, ua, ual);  // element (r-1, c-1): node is its BR
      elem(ra, corner_of(0, 1), ub, ubr, uar, ua);   // element (r-1, c): node is its BL
      elem(rbl, corner_of(1, 0), ucl, uc, ub, ubl);  // element (r, c-1): node is its TR
      elem(rb, corner_of(1, 1), uc, ucr, ubr, ub);   // element (r, c): node is its TL
      if (out_lane && r < r1) emit(r, c, acc, dg, ub, ex);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        ua[d] = ub[d];
        ual[d] = ubl[d];
        uar[d] = ubr[d];
        ub[d] = uc[d];
        ubl[d] = ucl[d];
        ubr[d] = ucr[d];
      }
      ra = rb;
      ral = rbl;
    }
  }
}

}  // namespace stt
