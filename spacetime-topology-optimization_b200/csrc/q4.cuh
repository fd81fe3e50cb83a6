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

// BAND: grid rows a warp marches; 0 takes them from the launch (nny / gridDim.y, rounded
// up), for launches that choose shorter bands when they have few rows.
template <int D, typename T, bool KU, bool DG, typename Extra = NoExtra, int BAND = kQRows, typename LoadU,
          typename LoadR, typename LoadX, typename Emit>
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
  const int band = BAND > 0 ? BAND : (nny + (int)gridDim.y - 1) / (int)gridDim.y;
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, nny);
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

// ---- modal form of the element operator ----------------------------------------------
//
// On the unit-square bilinear element every element matrix of the reference (the
// plane-stress KE of sttopt/fem.py:17-30 for any nu, the diffusion KE of :98-111)
// factors exactly as KE = T^T M T.  T maps the element's corner values (per
// displacement component) to three edge modes, all with +-1 weights:
//   Gx = (u_BR - u_BL) + (u_TR - u_TL),  Gy = (u_TL + u_TR) - (u_BL + u_BR),
//   H  = (u_TR - u_TL) - (u_BR - u_BL)   (x derivative, y derivative, hourglass),
// and M is sparse: plane stress couples Gx(ux) with Gy(uy) (normal stresses), shares
// one coefficient for the shear strain Gy(ux) + Gx(uy), and keeps the two hourglass
// modes diagonal; diffusion is diagonal.  K(rho) u per element then costs ~35 flops
// instead of the 8 x 8 product's 72, and the edge sums/differences of a grid row are
// shared by the element rows above and below it.  The host recognises the form from
// the KE it is given (modal_from_ke); any other KE takes the generic march above.
template <typename T>
struct MQ {
  T m00, m01, m11, m22, m44, m55;  // D = 2: normal (00, 01, 11), shear (22), hourglass (44, 55)
                                   // D = 1: Gx (00), Gy (11), hourglass (22)
  T kd0, kd1;                      // diagonal of KE per component (equal at every corner)
};

template <typename T>
MQ<T> mq_cast(const double (&m)[8]) {
  return MQ<T>{T(m[0]), T(m[1]), T(m[2]), T(m[3]), T(m[4]), T(m[5]), T(m[6]), T(m[7])};
}

// Corner forces of one component from its mode coefficients (alpha on Gx, beta on Gy,
// gamma on H): TR = a + b + g, BL = -a - b + g, BR = a - b - g, TL = -a + b - g.
// `own` gets TL (+ the carry to this node), `send` TR (+ the carry to the right node);
// the carries become BL and BR, which land on the next grid row.
template <typename T>
STT_DEV void modal_corners(T al, T be, T ga, T& co, T& cr, T& own, T& send) {
  const T s = al + be, t = al - be;
  own = co - (t + ga);
  send = cr + (s + ga);
  co = ga - s;
  cr = t - ga;
}

// The default input record of march_modal: the node's values, used as loaded.
struct CopyIn {
  template <typename In, typename V>
  STT_DEV void operator()(int, int, uint8_t, const In& in, V& v) const {
#pragma unroll
    for (int d = 0; d < (int)(sizeof(V) / sizeof(v[0])); ++d) v[d] = in[d];
  }
};

constexpr uint8_t kInGrid = 0x80;  // march_modal's flag bit: the row was in the grid

// The level-0 operator with KE in modal form.  The warp marches element rows: lane c
// owns element (er, c) and its top-left node.  For element row er it loads the bottom
// grid row er + 1, takes the right neighbour's value by a shuffle, forms the element's
// modes, and splits its forces: TL to its own node (er, c), TR to the right lane (one
// shuffle), BL and BR carried to grid row er + 1.  Node row er is then complete and is
// emitted.
//
// Loaders (called for in-grid positions only):
//   loadf(r, c) -> uint8_t   the node's fixed flags (0 when the operator has none); read
//                            once per node and used for the input projection (PIN) and
//                            handed to emit;
//   loadu(r, c, fl, In& in)  raw loads of the node's input record (In = T[D] by default);
//                            no arithmetic on loaded values, which would wait for the
//                            load and expose its latency;
//   value(r, c, fl, in, v)   the node's input value from its record, evaluated when the
//                            row is consumed (default: the loaded values);
//   loadr(r, c) -> T         element density;
//   loadx(r, c) -> Extra     per-output-node values (right-hand side ...).
// Positions outside the grid read as zero.  emit(r, c, Ku, dg, uc, fl, ex) gets K u
// (KU), diag(K) (DG), the node's (projected) input, flags and Extra.  Every option is a
// template parameter or a loader that returns a constant: a runtime-uniform branch
// around a load in this loop cost the FP32 apply 2x on B200 (measured).  AHEAD rows of
// loads stay in flight; at ~46 registers a thread the SM holds 11 blocks, and on B200
// that beat deeper lookahead (4 rows: -20 %, 8 rows: -50 % for the FP32 apply at
// 2048x1024 x 16 rows) and two grid columns per lane (-12 %), all measured.
template <int D, typename T, bool KU, bool DG, bool PIN, typename Extra = NoExtra, typename In = T[D],
          int AHEAD = 2, int BAND = kQRows, typename LoadF, typename LoadU, typename LoadR, typename LoadX,
          typename Emit, typename Value = CopyIn>
STT_DEV void march_modal(const MQ<T>& q, int nnx, int nny, LoadF loadf, LoadU loadu, LoadR loadr, LoadX loadx,
                         Emit emit, Value value = Value{}) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kQCols - 1 + lane;  // this lane's column
  const bool out_lane = lane >= 1 && lane <= kQCols && c < nnx;
  const int band = BAND > 0 ? BAND : (nny + (int)gridDim.y - 1) / (int)gridDim.y;  // 0: from the launch
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, nny);
  const int nelx = nnx - 1, nely = nny - 1;
  const bool col_ok = c >= 0 && c < nnx;
  const bool ecol_ok = c >= 0 && c < nelx;
  auto U = [&](int r, In& in, uint8_t& fl) {
    fl = 0;
    if (col_ok && r >= 0 && r < nny) {
      fl = loadf(r, c) | kInGrid;
      if constexpr (KU) loadu(r, c, fl, in);
    }
  };
  // the consumed row's value: evaluated from its record, projected (PIN)
  auto V = [&](int r, const In& in, uint8_t fl, T(&v)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = T(0);
    if (KU && (fl & kInGrid)) {
      value(r, c, fl, in, v);
      if constexpr (PIN) {
#pragma unroll
        for (int d = 0; d < D; ++d)
          if ((fl >> d) & 1) v[d] = T(0);
      }
    }
  };
  auto Rho = [&](int r) -> T { return (ecol_ok && r >= 0 && r < nely) ? loadr(r, c) : T(0); };
  auto X = [&](int r) -> Extra { return (out_lane && r < r1) ? loadx(r, c) : Extra{}; };
  T ut[D];          // this lane's node on the top edge of the element row
  uint8_t ft;       // its flags
  T sT[D], dT[D];   // top edge: u(c) + u(c + 1), u(c + 1) - u(c)
  T co[D], cr[D];   // forces from the element row above: to this node, to the right node
  T rp = T(0);      // density of the element above (for the diagonal)
  auto edge = [&](const T(&v)[D], T(&s)[D], T(&dd)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const T vr = __shfl_down_sync(0xffffffffu, v[d], 1);
      s[d] = v[d] + vr;
      dd[d] = vr - v[d];
    }
  };
  // element row with bottom edge ub and density rho; own / send as in modal_corners
  auto step = [&](const T(&ub)[D], T rho, T(&own)[D], T(&send)[D]) {
    T sB[D], dB[D];
    edge(ub, sB, dB);
    if constexpr (KU) {
      T Gx[D], Gy[D], H[D];
#pragma unroll
      for (int d = 0; d < D; ++d) {
        Gx[d] = dB[d] + dT[d];
        Gy[d] = sT[d] - sB[d];
        H[d] = dT[d] - dB[d];
      }
      if constexpr (D == 2) {
        const T p = rho * Gx[0], pq = rho * Gy[1];
        const T a = fma(q.m01, pq, q.m00 * p);
        const T cc = fma(q.m01, p, q.m11 * pq);
        const T b = (rho * q.m22) * (Gy[0] + Gx[1]);
        modal_corners(a, b, (rho * q.m44) * H[0], co[0], cr[0], own[0], send[0]);
        modal_corners(b, cc, (rho * q.m55) * H[1], co[1], cr[1], own[1], send[1]);
      } else {
        modal_corners((rho * q.m00) * Gx[0], (rho * q.m11) * Gy[0], (rho * q.m22) * H[0], co[0], cr[0],
                      own[0], send[0]);
      }
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
      sT[d] = sB[d];
      dT[d] = dB[d];
    }
  };
  // element row r0 - 1 (zero density above the grid) fills the carries of grid row r0
  {
    In i0, i1;
    T u0[D], own[D], send[D];
    uint8_t f0;
    U(r0 - 1, i0, f0);
    U(r0, i1, ft);
    V(r0 - 1, i0, f0, u0);
    edge(u0, sT, dT);
#pragma unroll
    for (int d = 0; d < D; ++d) co[d] = cr[d] = T(0);
    V(r0, i1, ft, ut);
    const T rho = Rho(r0 - 1);
    step(ut, rho, own, send);
    rp = rho;
  }
  // prefetch queue: bottom edges (and flags) r+1 .. r+AHEAD, density and extra rows
  // r .. r+AHEAD-1
  In qu[AHEAD];
  T qr[AHEAD];
  uint8_t qf[AHEAD];
  Extra qx[AHEAD];
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) {
    U(r0 + 1 + k, qu[k], qf[k]);
    qr[k] = Rho(r0 + k);
    qx[k] = X(r0 + k);
  }
  for (int rb0 = r0; rb0 < r1; rb0 += AHEAD) {
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {
      const int r = rb0 + k;
      T ub[D];
      const uint8_t fb = qf[k];
      V(r + 1, qu[k], fb, ub);
      const T rho = qr[k];
      const Extra ex = qx[k];
      U(r + 1 + AHEAD, qu[k], qf[k]);  // refill the slot
      qr[k] = Rho(r + AHEAD);
      qx[k] = X(r + AHEAD);
      T own[D], send[D], Ku[D], dg[D];
      step(ub, rho, own, send);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        Ku[d] = KU ? own[d] + __shfl_up_sync(0xffffffffu, send[d], 1) : T(0);
        dg[d] = T(0);
      }
      if constexpr (DG) {
        const T rs = rho + rp;
        const T rsum = rs + __shfl_up_sync(0xffffffffu, rs, 1);
        dg[0] = q.kd0 * rsum;
        if constexpr (D == 2) dg[1] = q.kd1 * rsum;
      }
      rp = rho;
      if (out_lane && r < r1) emit(r, c, Ku, dg, ut, (uint8_t)(ft & ~kInGrid), ex);
#pragma unroll
      for (int d = 0; d < D; ++d) ut[d] = ub[d];
      ft = fb;
    }
  }
}

// Launch grid of the marching kernels (generic and modal share it).
template <bool MODAL, typename T>
inline dim3 march_grid(int nelx, int nely, int rows) {
  return q4_grid(nelx, nely, rows);
}

}  // namespace stt
