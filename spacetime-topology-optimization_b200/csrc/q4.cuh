// Level-0 (density-scaled Q4) operator tiles.
//
// K(rho) u is applied node by node with no atomics: a 32 x 8 tile of output nodes
// stages its input nodes plus a one-node halo, and the densities of the elements
// touching them plus a one-element halo, in shared memory.  Each thread then sums
// the four elements around its node, rho_e * (KE row of the node's corner) . u_e,
// which is the reference's gather / (Ue @ KE) * density / index_add
// (sttopt/torch_fem.py:76-82) reorganised as a deterministic gather.
#pragma once

#include "common.cuh"

namespace stt {

template <int D, typename T>
struct KEq {
  T v[(4 * D) * (4 * D)];
};

template <int D, typename T, typename TR>
struct Q4Smem {
  T u[kTY + 2][kTX + 2][D];
  TR rho[kTY + 1][kTX + 1];
};

// Element densities of the tile (elements (r0-1 .. r0+kTY-1) x (c0-1 .. c0+kTX-1)),
// zero outside the mesh.
template <int D, typename T, typename TR>
STT_DEV void load_rho_tile(Q4Smem<D, T, TR>& s, const TR* __restrict__ rho, int r0, int c0,
                           int nelx, int nely) {
  for (int i = threadIdx.x; i < (kTY + 1) * (kTX + 1); i += kNT) {
    const int ly = i / (kTX + 1), lx = i - ly * (kTX + 1);
    const int er = r0 - 1 + ly, ec = c0 - 1 + lx;
    TR v = TR(0);
    if (er >= 0 && er < nely && ec >= 0 && ec < nelx) v = __ldg(rho + (size_t)er * nelx + ec);
    s.rho[ly][lx] = v;
  }
}

// Input-vector tile with a one-node halo; `fetch(node, v)` fills a node's D values
// (it applies the projection and any on-the-fly combination), zero off the mesh.
template <int D, typename T, typename TR, typename Fetch>
STT_DEV void load_u_tile(Q4Smem<D, T, TR>& s, int r0, int c0, int nnx, int nny, Fetch fetch) {
  for (int i = threadIdx.x; i < (kTY + 2) * (kTX + 2); i += kNT) {
    const int ly = i / (kTX + 2), lx = i - ly * (kTX + 2);
    const int r = r0 - 1 + ly, c = c0 - 1 + lx;
    T v[D];
#pragma unroll
    for (int j = 0; j < D; ++j) v[j] = T(0);
    if (r >= 0 && r < nny && c >= 0 && c < nnx) fetch(r * nnx + c, v);
#pragma unroll
    for (int j = 0; j < D; ++j) s.u[ly][lx][j] = v[j];
  }
}

// (K u) at the tile node (ty, tx), without the reaction term.
template <int D, typename T, typename TR>
STT_DEV void tile_Ku(const Q4Smem<D, T, TR>& s, int ty, int tx, const KEq<D, T>& ke,
                     T (&acc)[D]) {
#pragma unroll
  for (int i = 0; i < D; ++i) acc[i] = T(0);
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const T rho = T(s.rho[ty + a][tx + b]);
      const int k = corner_of(a, b);
      T sum[D];
#pragma unroll
      for (int i = 0; i < D; ++i) sum[i] = T(0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T* uq = s.u[ty + a + corner_dr(q)][tx + b + corner_dc(q)];
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
          for (int j = 0; j < D; ++j) sum[i] = fma(ke.v[(k * D + i) * (4 * D) + q * D + j], uq[j], sum[i]);
      }
#pragma unroll
      for (int i = 0; i < D; ++i) acc[i] = fma(rho, sum[i], acc[i]);
    }
  }
}

// diag(K) at the tile node (ty, tx), without the reaction term.
template <int D, typename T, typename TR>
STT_DEV void tile_diag(const Q4Smem<D, T, TR>& s, int ty, int tx, const KEq<D, T>& ke,
                       T (&dg)[D]) {
#pragma unroll
  for (int i = 0; i < D; ++i) dg[i] = T(0);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const T rho = T(s.rho[ty + a][tx + b]);
      const int k = corner_of(a, b);
#pragma unroll
      for (int i = 0; i < D; ++i) dg[i] = fma(rho, ke.v[(k * D + i) * (4 * D) + k * D + i], dg[i]);
    }
}

template <int D, typename T>
STT_DEV void load_node(const T* __restrict__ p, int node, T (&v)[D]) {
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
STT_DEV void store_node(T* __restrict__ p, int node, const T (&v)[D]) {
  if constexpr (D == 2 && sizeof(T) == 8) {
    reinterpret_cast<double2*>(p)[node] = make_double2(v[0], v[1]);
  } else if constexpr (D == 2 && sizeof(T) == 4) {
    reinterpret_cast<float2*>(p)[node] = make_float2(v[0], v[1]);
  } else {
    p[node] = v[0];
  }
}

STT_DEV bool is_fixed(const uint8_t* fixed, int node, int i) {
  return fixed != nullptr && ((__ldg(fixed + node) >> i) & 1);
}

}  // namespace stt
