// Multigrid cycle kernels: damped-Jacobi sweeps and residuals on level 0 (density
// tiles) and on stencil levels, full-weighting restriction, bilinear prolongation,
// and the block-banded coarse solve.  Templated on the cycle precision T.
//
// Reference: torch_mg.VCycle._smooth/_cycle (sttopt/torch_mg.py:440-476), transfers
// _interp_axis/_restrict_axis/_on_node_grid (:75-109).
#pragma once

#include <type_traits>

#include "common.cuh"
#include "q4.cuh"

namespace stt {

enum SweepMode { SW_FIRST = 0, SW_SWEEP = 1, SW_RESID = 2, SW_APPLY = 3, SW_POST = 4 };

// Coarse-grid correction folded into a sweep's input (SW_POST): the sweep reads
// x + P_f(P e_c), bilinear interpolation x pass then y pass (torch_mg._interp_axis,
// sttopt/torch_mg.py:75-81), so the prolongation needs no pass of its own.
template <typename T>
struct ProlongSrc {
  const T* ec;  // coarse correction of this batch row (set per row in the kernel)
  long long rs;
  int cnnx, kx, ky;
};

template <int D, typename T>
STT_DEV void prolong_at(const T* __restrict__ e, int cnnx, int kx, int ky, int r, int c, T (&v)[D]) {
  const int R = div_k(r, ky), jy = r - R * ky, C = div_k(c, kx), jx = c - C * kx;
  const T wx = T((double)jx / kx), wy = T((double)jy / ky);
  const long long n0 = (long long)R * cnnx + C;
  // one vector load per coarse corner
  T e00[D], e01[D], e10[D], e11[D];
  load_node<D, T>(e, n0, e00);
  if (jx) load_node<D, T>(e, n0 + 1, e01);
  if (jy) {
    load_node<D, T>(e, n0 + cnnx, e10);
    if (jx) load_node<D, T>(e, n0 + cnnx + 1, e11);
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    T t0 = e00[i], t1 = jy ? e10[i] : T(0);
    if (jx) {
      t0 = e00[i] * (T(1) - wx) + e01[i] * wx;
      if (jy) t1 = e10[i] * (T(1) - wx) + e11[i] * wx;
    }
    v[i] = jy ? t0 * (T(1) - wy) + t1 * wy : t0;
  }
}

// ---- level 0: density-scaled Q4 tiles ------------------------------------------
//   SW_FIRST: out = (omega * b) / diag               (sweep from x = 0)
//   SW_SWEEP: out = x + (omega * (b - A x)) / diag
//   SW_RESID: out = b - A x
//   SW_APPLY: out = A x
// A is the projected operator P(K P .) (+ lumped reaction); x is read projected.

// The per-node result of a level-0 pass from A x (unprojected, without reaction), the
// diagonal of K, the node's x and b, its fixed flags and its reaction value.
// RDT: the reaction term is present (false skips its zero terms, which the compiler must
// otherwise keep: fma(0, x, y) is not y for every x and signed zero y).
template <int D, typename T, int MODE, bool RDT = true>
STT_DEV void l0_result(T (&Ax)[D], T (&dg)[D], const T (&xo)[D], const T (&bv)[D], uint8_t fl,
                       const T (&rd)[D], T omega, T (&res)[D]) {
  constexpr bool KU = MODE != SW_FIRST;
  constexpr bool DG = MODE == SW_FIRST || MODE == SW_SWEEP || MODE == SW_POST;
  if (KU) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      if constexpr (RDT) Ax[i] = fma(rd[i], xo[i], Ax[i]);
      if ((fl >> i) & 1) Ax[i] = T(0);
    }
  }
  if (DG) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      if constexpr (RDT) dg[i] += rd[i];
      if ((fl >> i) & 1) dg[i] = T(1);
      const T x0 = MODE == SW_FIRST ? T(0) : xo[i];
      res[i] = x0 + sweep_div(omega * (bv[i] - (KU ? Ax[i] : T(0))), dg[i]);
    }
  } else if (MODE == SW_RESID) {
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = bv[i] - Ax[i];
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = Ax[i];
  }
}

template <int D, typename T, int MODE>
__global__ void __launch_bounds__(kQThreads) l0_sweep_kernel(
    const T* __restrict__ x, long long x_rs, const T* __restrict__ b, long long b_rs,
    T* __restrict__ out, long long o_rs, const T* __restrict__ rho, long long rho_rs,
    const T* __restrict__ rdiag, long long rd_rs, const uint8_t* __restrict__ fixed,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, int nelx,
    int nely, T omega, KEq<D, T> ke, int proj_in, ProlongSrc<T> pro) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const T* xs = x + (size_t)s * x_rs;
  const T* es = MODE == SW_POST ? pro.ec + (size_t)s * pro.rs : nullptr;
  const T* rh = rho + (size_t)h * rho_rs;
  const T* rdh = rdiag ? rdiag + (size_t)h * rd_rs : nullptr;
  const T* bs = b + (size_t)s * b_rs;
  T* os = out + (size_t)s * o_rs;
  const uint8_t* pin = proj_in ? fixed : nullptr;
  constexpr bool KU = MODE != SW_FIRST;
  constexpr bool DG = MODE == SW_FIRST || MODE == SW_SWEEP || MODE == SW_POST;
  march<D, T, KU, DG, RhsX<D, T>>(
      ke, nnx, nny,
      [&](int r, int c, T(&v)[D]) {
        const int node = r * nnx + c;
        load_node<D, T>(xs, node, v);
        if (MODE == SW_POST) {
          T pv[D];
          prolong_at<D, T>(es, pro.cnnx, pro.kx, pro.ky, r, c, pv);
          const uint8_t fl = __ldg(fixed + node);
#pragma unroll
          for (int d = 0; d < D; ++d)
            if (!((fl >> d) & 1)) v[d] += pv[d];
        }
        if (pin) {
          const uint8_t fl = __ldg(pin + node);
#pragma unroll
          for (int d = 0; d < D; ++d)
            if ((fl >> d) & 1) v[d] = T(0);
        }
      },
      [&](int r, int c) { return __ldg(rh + (size_t)r * nelx + c); },
      [&](int r, int c) {
        RhsX<D, T> x;
        const int node = r * nnx + c;
        if (MODE != SW_APPLY) load_node<D, T>(bs, node, x.b);
        x.fl = __ldg(fixed + node);
        return x;
      },
      [&](int r, int c, T(&Ax)[D], T(&dg)[D], const T(&xo)[D], const RhsX<D, T>& ex) {
        const int node = r * nnx + c;
        T rd[D], res[D];
#pragma unroll
        for (int i = 0; i < D; ++i) rd[i] = rdh ? __ldg(rdh + node * D + i) : T(0);
        l0_result<D, T, MODE>(Ax, dg, xo, ex.b, ex.fl, rd, omega, res);
        store_node<D, T>(os, node, res);
      });
}

// Right-hand side of an output node (the modal kernels take the flags separately).
template <int D, typename T>
struct RhsB {
  T b[D];
};


// The same passes with KE in modal form (march_modal); RD adds the reaction term.  The
// input is projected in SW_APPLY only (the cycle's vectors are projected already).
template <int D, typename T, int MODE, bool RD>
__global__ void __launch_bounds__(kQThreads) l0_sweep_modal_kernel(
    const T* __restrict__ x, long long x_rs, const T* __restrict__ b, long long b_rs,
    T* __restrict__ out, long long o_rs, const T* __restrict__ rho, long long rho_rs,
    const T* __restrict__ rdiag, long long rd_rs, const uint8_t* __restrict__ fixed,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, int nelx,
    int nely, T omega, MQ<T> mq, ProlongSrc<T> pro) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const T* xs = x + (size_t)s * x_rs;
  const T* rh = rho + (size_t)h * rho_rs;
  const T* rdh = RD ? rdiag + (size_t)h * rd_rs : nullptr;
  const T* bs = b + (size_t)s * b_rs;
  T* os = out + (size_t)s * o_rs;
  constexpr bool KU = MODE != SW_FIRST;
  constexpr bool DG = MODE == SW_FIRST || MODE == SW_SWEEP;
  auto loadf = [&](int r, int c) { return __ldg(fixed + r * nnx + c); };
  auto loadr = [&](int r, int c) { return __ldg(rh + (size_t)r * nelx + c); };
  auto loadx = [&](int r, int c) {
    RhsB<D, T> e;
    if constexpr (MODE != SW_APPLY) {
      load_node<D, T>(bs, r * nnx + c, e.b);
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) e.b[d] = T(0);
    }
    return e;
  };
  auto emit = [&](int r, int c, T(&Ax)[D], T(&dg)[D], const T(&xo)[D], uint8_t fl, const RhsB<D, T>& ex) {
    const int node = r * nnx + c;
    T rd[D], res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) rd[i] = RD ? __ldg(rdh + node * D + i) : T(0);
    l0_result<D, T, MODE, RD>(Ax, dg, xo, ex.b, fl, rd, omega, res);
    store_node<D, T>(os, node, res);
  };
  static_assert(MODE != SW_POST, "the cycle prolongs with prolong_kernel");
  march_modal<D, T, KU, DG, MODE == SW_APPLY, RhsB<D, T>>(
      mq, nnx, nny, loadf, [&](int r, int c, uint8_t, T(&v)[D]) { load_node<D, T>(xs, r * nnx + c, v); },
      loadr, loadx, emit);
}

// ---- level 0: pre-smoothing in one pass (modal form, n_smooth = 2) --------------------
//
// The two pre-smoothing sweeps and the residual as one streaming pass: the passes of
// the unfused cycle (torch_mg.VCycle._smooth, sttopt/torch_mg.py:440-476) chained inside
// a warp, each one grid row behind the one before, so b and the densities cross HBM
// once instead of three times.  Per node the arithmetic is the unfused kernels' (same
// operations in the same order), so results agree with the unfused passes to rounding.
//
//   x1 = omega b / D;  x2 = x1 + omega (b - A x1) / D;  r = b - A x2.  Writes x2 and r.
//
// Each chained stage needs its input on the neighbouring lanes, so a stage's valid
// lanes shrink by one on each side (and lane 0 has no left neighbour for the diagonal):
// lanes 3..29 are output (27 columns a warp).  The front row f feeds stage A at element
// row f - 1 and stage B at f - 2; a band [r0, r1) runs f = r0 - 2 .. r1 + 1 so both
// stages are exact on the band.  (A post-smoothing twin, prolongation + two sweeps in one
// pass, measured slower on B200 than prolong_kernel + two sweeps: at 128 registers its
// 4 blocks an SM could not keep the loads in flight.)

// One modal element-row stage: the top edge, the carries and the top node's value.
template <int D, typename T>
struct ModalStage {
  T sT[D], dT[D], co[D], cr[D], ut[D];

  STT_DEV void reset() {
#pragma unroll
    for (int d = 0; d < D; ++d) sT[d] = dT[d] = co[d] = cr[d] = ut[d] = T(0);
  }
  // element row with bottom edge ub and density rho: Ku of the top node row; then the
  // bottom row becomes the top (ut = ub)
  STT_DEV void step(const MQ<T>& q, const T (&ub)[D], T rho, T (&Ku)[D]) {
    T sB[D], dB[D], own[D], send[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const T vr = __shfl_down_sync(0xffffffffu, ub[d], 1);
      sB[d] = ub[d] + vr;
      dB[d] = vr - ub[d];
    }
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
      modal_corners((rho * q.m00) * Gx[0], (rho * q.m11) * Gy[0], (rho * q.m22) * H[0], co[0], cr[0], own[0],
                    send[0]);
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
      Ku[d] = own[d] + __shfl_up_sync(0xffffffffu, send[d], 1);
      sT[d] = sB[d];
      dT[d] = dB[d];
      ut[d] = ub[d];
    }
  }
};

// The plane-stress FP32 stage with the two displacement components in float2 pairs:
// Blackwell's paired FP32 add / multiply / fma issue one instruction for both components
// (the chained level-0 passes are issue-bound).  Every operation rounds as the scalar
// stage's does (the same operations on each component, subtraction as addition of the
// negation, which is exact).
STT_DEV float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

template <>
struct ModalStage<2, float> {
  float2 sT, dT, co, cr;
  float ut[2];

  STT_DEV void reset() {
    sT = dT = co = cr = make_float2(0.f, 0.f);
    ut[0] = ut[1] = 0.f;
  }
  STT_DEV void step(const MQ<float>& q, const float (&ub)[2], float rho, float (&Ku)[2]) {
    const float2 u = make_float2(ub[0], ub[1]);
    const float2 vr = make_float2(__shfl_down_sync(0xffffffffu, ub[0], 1), __shfl_down_sync(0xffffffffu, ub[1], 1));
    const float2 sB = __fadd2_rn(u, vr);
    const float2 dB = sub2(vr, u);
    const float2 Gx = __fadd2_rn(dB, dT);
    const float2 Gy = sub2(sT, sB);
    const float2 H = sub2(dT, dB);
    const float2 rr = make_float2(rho, rho);
    const float2 P = __fmul2_rn(rr, make_float2(Gx.x, Gy.y));  // p = rho Gx(ux), pq = rho Gy(uy)
    // a = m01 pq + m00 p, cc = m01 p + m11 pq
    const float2 AC = __ffma2_rn(make_float2(q.m01, q.m01), make_float2(P.y, P.x),
                                 __fmul2_rn(make_float2(q.m00, q.m11), P));
    const float b = (rho * q.m22) * (Gy.x + Gx.y);
    const float2 GA = __fmul2_rn(__fmul2_rn(rr, make_float2(q.m44, q.m55)), H);
    // modal_corners of (a, b, GA.x) and (b, cc, GA.y)
    const float2 AL = make_float2(AC.x, b), BE = make_float2(b, AC.y);
    const float2 s = __fadd2_rn(AL, BE), t = sub2(AL, BE);
    const float2 own = sub2(co, __fadd2_rn(t, GA));
    const float2 send = __fadd2_rn(cr, __fadd2_rn(s, GA));
    co = sub2(GA, s);
    cr = sub2(t, GA);
    const float2 K = __fadd2_rn(own, make_float2(__shfl_up_sync(0xffffffffu, send.x, 1),
                                                 __shfl_up_sync(0xffffffffu, send.y, 1)));
    Ku[0] = K.x;
    Ku[1] = K.y;
    sT = sB;
    dT = dB;
    ut[0] = ub[0];
    ut[1] = ub[1];
  }
};

// Raw loads of one front row (no arithmetic, so they stay in flight).
template <int D, typename T, bool RD>
struct FrontRow {
  T b[D];
  T rd[RD ? D : 1];
  T rho;
  uint8_t fl;
};

// Per-row values a stage reads one or two rows after the front: the right-hand side,
// w = omega / diag and the free mask mf (1 on free dofs, 0 on fixed and off-grid ones;
// the diagonal is taken as 1 there, so w stays finite).
template <int D, typename T, bool RD>
struct DelayRow {
  T b[D], w[D], mf[D];
  T rd[RD ? D : 1];
  T rho;
};

// The chained level-0 stages' per-node results from A x (unprojected, without the
// reaction term):
//   SW_FIRST: mf (w b);   SW_SWEEP: mf (x + w (b - A x));   SW_RESID: mf (b - A x).
// Multiplying by the free mask makes every result the projected one, whatever the input
// holds on fixed dofs (the reference projects the cycle's input and every smoothing
// result, torch_mg.py:440-476).  The plane-stress FP32 form pairs the two components.
template <int D, typename T, int MODE, bool RDT>
STT_DEV void l0_chain_result(T (&Ax)[D], const T (&w)[D], const T (&mf)[D], const T (&xo)[D], const T (&bv)[D],
                             const T (&rd)[D], T (&res)[D]) {
  if constexpr (D == 2 && sizeof(T) == 4 && !RDT) {
    const float2 W = make_float2(w[0], w[1]), M = make_float2(mf[0], mf[1]), B = make_float2(bv[0], bv[1]);
    float2 R;
    if constexpr (MODE == SW_FIRST) {
      R = __fmul2_rn(__fmul2_rn(W, B), M);
    } else {
      const float2 Bm = __fadd2_rn(B, make_float2(-Ax[0], -Ax[1]));
      if constexpr (MODE == SW_RESID) R = __fmul2_rn(Bm, M);
      else R = __fmul2_rn(__ffma2_rn(W, Bm, make_float2(xo[0], xo[1])), M);
    }
    res[0] = R.x;
    res[1] = R.y;
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T a = Ax[i];
      if constexpr (RDT && MODE != SW_FIRST) a = fma(rd[i], xo[i], a);
      if constexpr (MODE == SW_FIRST) res[i] = (w[i] * bv[i]) * mf[i];
      else if constexpr (MODE == SW_RESID) res[i] = (bv[i] - a) * mf[i];
      else res[i] = fma(w[i], bv[i] - a, xo[i]) * mf[i];
    }
  }
}

// The front row's DelayRow from its loads: mf from the fixed flags (the loaders mark
// off-grid positions all-fixed), w = omega / diag with diag = kd * (the densities
// around the node) (+ the reaction), 1 where mf is 0.
template <int D, typename T, bool RD>
STT_DEV void l0_delay_row(const FrontRow<D, T, RD>& F, T dsum, const MQ<T>& q, T omega, DelayRow<D, T, RD>& cur) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const bool free = !((F.fl >> d) & 1);
    cur.mf[d] = free ? T(1) : T(0);
    T dg = (d == 0 ? q.kd0 : q.kd1) * dsum;
    if constexpr (RD) dg += F.rd[d];
    cur.w[d] = sweep_div(omega, free ? dg : T(1));
    cur.b[d] = F.b[d];
    if constexpr (RD) cur.rd[d] = F.rd[d];
  }
  cur.rho = F.rho;
}

// The PCG's beta from the dots of a preconditioned residual, t[0] = r.z and t[1] =
// r.z_old (flexible form): the first call of a solve only records rz; later ones set
// beta = safe_div(rz - rz_mix, rz_old) (or rz / rz_old) and rz_old = rz.
STT_DEV void pcg_rz_finish(RowState& S, const double* t, int first, int flexible) {
  if (first) {
    S.rz = t[0];
  } else {
    const double num = flexible ? t[0] - t[1] : t[0];
    S.beta = safe_div(num, S.rz);
    S.rz = t[0];
    if (!isfinite(S.beta)) S.status = STT_ERR_BREAKDOWN;
  }
}

// The PCG's dots taken by the level-0 chained passes of its preconditioner cycle z = M r,
// whose right-hand side b is the r the dots read (the FP32 copy of r in a mixed cycle):
// the pre-smoothing pass takes the flexible beta's r.z_old (into RowState::rz_mix, with
// z_old loaded beside b), the post-smoothing pass r.z as it writes z and finishes beta,
// so neither needs a pass of its own.  A node's terms are summed in the cycle's
// precision (one rounding of each FP32 product, ~1e-7 relative, the FP32 cycle's own
// level) and accumulated in FP64 per thread, reduced over the pass's blocks.
template <typename T>
struct RzFuse {
  RowState* rst;    // null: no dots
  const T* zold;    // the previous z (the flexible beta's r.z_old), else null
  long long zo_rs;
  GridRed red;      // nblk = the pass's blocks a row (set at launch)
  int first, flexible;
};

constexpr int kPreCols = 27;  // output columns per warp strip of l0_presmooth_kernel

inline dim3 presmooth_grid(int nelx, int nely, int rows) {
  const int strips = (nelx + 1 + kPreCols - 1) / kPreCols;
  return dim3((strips + kQWarps - 1) / kQWarps, (nely + 1 + kQRows - 1) / kQRows, rows);
}

// FP32: 6 blocks of 128 threads an SM (<= 80 registers), measured fastest on B200 at
// 2048x1024 x 16 rows (333 us against 351 us at the compiler's 80-95 registers with
// fewer blocks).  FP64 needs twice the registers for the same state: 3 blocks.
// MX: also r.z_old of the PCG (mx.zold), z_old loaded with the front row's b.
template <int D, typename T, bool RD, bool MX = false, int AHEAD = 2>
__global__ void __launch_bounds__(kQThreads, sizeof(T) == 4 ? 6 : 3) l0_presmooth_kernel(
    const T* __restrict__ b, long long b_rs, T* __restrict__ out_x, long long ox_rs, T* __restrict__ out_r,
    long long or_rs, const T* __restrict__ rho, long long rho_rs, const T* __restrict__ rdiag,
    long long rd_rs, const uint8_t* __restrict__ fixed, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst, int nelx, int nely, T omega, MQ<T> q, RzFuse<T> mx = RzFuse<T>{}) {
  constexpr int LO = 3, HI = 29;
  static_assert(HI - LO + 1 == kPreCols, "strip width");
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const T* rh = rho + (size_t)h * rho_rs;
  const T* rdh = RD ? rdiag + (size_t)h * rd_rs : nullptr;
  const T* bs = b + (size_t)s * b_rs;
  T* ox = out_x + (size_t)s * ox_rs;
  T* orr = out_r + (size_t)s * or_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kPreCols - LO + lane;
  const bool out_lane = lane >= LO && lane <= HI && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const bool ecol_ok = c >= 0 && c < nelx;
  const int r0 = blockIdx.y * kQRows;
  const int r1 = min(r0 + kQRows, nny);
  const T* zos = MX ? mx.zold + (size_t)s * mx.zo_rs : nullptr;
  T zq[MX ? AHEAD : 1][D];  // MX: z_old at the front rows in flight
  double mix[1] = {0.0};
  auto load_zo = [&](int f, T(&zv)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) zv[d] = T(0);
    if (col_ok && f >= 0 && f < nny) load_node<D, T>(zos, (long long)f * nnx + c, zv);
  };
  auto load_front = [&](int f, FrontRow<D, T, RD>& F) {
#pragma unroll
    for (int d = 0; d < D; ++d) F.b[d] = T(0);
    if constexpr (RD) {
#pragma unroll
      for (int d = 0; d < D; ++d) F.rd[d] = T(0);
    }
    F.fl = 0xFF;  // off the grid: every dof fixed (free mask 0)
    F.rho = (ecol_ok && f >= 0 && f < nely) ? __ldg(rh + (size_t)f * nelx + c) : T(0);
    if (!col_ok || f < 0 || f >= nny) return;
    const long long node = (long long)f * nnx + c;
    F.fl = __ldg(fixed + node);
    load_node<D, T>(bs, node, F.b);
    if constexpr (RD) {
#pragma unroll
      for (int d = 0; d < D; ++d) F.rd[d] = __ldg(rdh + node * D + d);
    }
  };
  ModalStage<D, T> A, B;
  A.reset();
  B.reset();
  DelayRow<D, T, RD> d1{}, d2{};  // rows f - 1 and f - 2
  const int f0 = r0 - 2, f1 = r1 + 1;  // front rows, inclusive
  T rho_prev = (ecol_ok && f0 - 1 >= 0 && f0 - 1 < nely) ? __ldg(rh + (size_t)(f0 - 1) * nelx + c) : T(0);
  FrontRow<D, T, RD> qf[AHEAD];
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) {
    load_front(f0 + k, qf[k]);
    if constexpr (MX) load_zo(f0 + k, zq[k]);
  }
  for (int fb = f0; fb <= f1; fb += AHEAD) {
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {
      const int f = fb + k;
      const FrontRow<D, T, RD> F = qf[k];
      load_front(f + AHEAD, qf[k]);
      if constexpr (MX) {
        // b z_old at the front row, each node once (output lanes, the block's rows)
        if (out_lane && f >= r0 && f < r1) {
          T t = F.b[0] * zq[k][0];
#pragma unroll
          for (int d = 1; d < D; ++d) t = fma(F.b[d], zq[k][d], t);
          mix[0] += (double)t;
        }
        load_zo(f + AHEAD, zq[k]);
      }
      // the row's free mask and w = omega / diag (diag: kd times the densities around the node)
      DelayRow<D, T, RD> cur;
      {
        const T rs = F.rho + rho_prev;
        const T dsum = rs + __shfl_up_sync(0xffffffffu, rs, 1);
        l0_delay_row<D, T, RD>(F, dsum, q, omega, cur);
      }
      rho_prev = F.rho;
      // x1 at row f (the first sweep from zero)
      T x1[D];
      {
        T zero[D], rdv[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          zero[d] = T(0);
          rdv[d] = RD ? cur.rd[d] : T(0);
        }
        l0_chain_result<D, T, SW_FIRST, RD>(zero, cur.w, cur.mf, zero, cur.b, rdv, x1);
      }
      // stage A: element row f - 1 -> second sweep at node row f - 1
      T KA[D], xa[D], xo_a[D];
#pragma unroll
      for (int d = 0; d < D; ++d) xo_a[d] = A.ut[d];
      A.step(q, x1, d1.rho, KA);
      {
        T rd1[D];
#pragma unroll
        for (int d = 0; d < D; ++d) rd1[d] = RD ? d1.rd[d] : T(0);
        l0_chain_result<D, T, SW_SWEEP, RD>(KA, d1.w, d1.mf, xo_a, d1.b, rd1, xa);
      }
      // stage B: element row f - 2 -> residual at node row f - 2
      T KB[D], rb[D], xo_b[D];
#pragma unroll
      for (int d = 0; d < D; ++d) xo_b[d] = B.ut[d];
      B.step(q, xa, d2.rho, KB);
      {
        T rd2[D];
#pragma unroll
        for (int d = 0; d < D; ++d) rd2[d] = RD ? d2.rd[d] : T(0);
        l0_chain_result<D, T, SW_RESID, RD>(KB, d2.w, d2.mf, xo_b, d2.b, rd2, rb);
      }
      if (out_lane) {
        if (f - 1 >= r0 && f - 1 < r1) store_node<D, T>(ox, (long long)(f - 1) * nnx + c, xa);
        if (f - 2 >= r0 && f - 2 < r1) store_node<D, T>(orr, (long long)(f - 2) * nnx + c, rb);
      }
      d2 = d1;
      d1 = cur;
    }
  }
  if constexpr (MX) {
    grid_reduce<1, kQThreads>(mx.red, s, blockIdx.y * gridDim.x + blockIdx.x, mix,
                              [&](const double* t) { mx.rst[s].rz_mix = t[0]; });
  }
}

// ---- level 0: post-smoothing in one pass (modal form, n_smooth = 2) -------------------
//
// The two post-smoothing sweeps after the prolongation, chained like l0_presmooth_kernel:
//   x1 = x0 + omega (b - A x0) / D;  x2 = x1 + omega (b - A x1) / D.  Writes x2.
// x0 (the prolonged iterate) is loaded with the front row; stage A sweeps at row f - 1,
// stage B at row f - 2.  Lanes 2..29 are output (28 columns a warp).  Per node the
// arithmetic is the unfused sweeps'.
constexpr int kPostCols = 28;

inline dim3 postsmooth_grid(int nelx, int nely, int rows) {
  const int strips = (nelx + 1 + kPostCols - 1) / kPostCols;
  return dim3((strips + kQWarps - 1) / kQWarps, (nely + 1 + kQRows - 1) / kQRows, rows);
}

template <int D, typename T, bool RD, bool RZ = false, int AHEAD = 2>
__global__ void __launch_bounds__(kQThreads, sizeof(T) == 4 ? 6 : 3) l0_postsmooth_kernel(
    const T* __restrict__ x0, long long x_rs, const T* __restrict__ b, long long b_rs, T* __restrict__ out,
    long long o_rs, const T* __restrict__ rho, long long rho_rs, const T* __restrict__ rdiag, long long rd_rs,
    const uint8_t* __restrict__ fixed, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst, int nelx, int nely, T omega, MQ<T> q, RzFuse<T> rz = RzFuse<T>{}) {
  constexpr int LO = 2, HI = 29;
  static_assert(HI - LO + 1 == kPostCols, "strip width");
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const T* rh = rho + (size_t)h * rho_rs;
  const T* rdh = RD ? rdiag + (size_t)h * rd_rs : nullptr;
  const T* xs = x0 + (size_t)s * x_rs;
  const T* bs = b + (size_t)s * b_rs;
  T* os = out + (size_t)s * o_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kPostCols - LO + lane;
  const bool out_lane = lane >= LO && lane <= HI && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const bool ecol_ok = c >= 0 && c < nelx;
  const int r0 = blockIdx.y * kQRows;
  const int r1 = min(r0 + kQRows, nny);
  struct Front {
    FrontRow<D, T, RD> F;
    T x[D];
  };
  auto load_front = [&](int f, Front& Q) {
#pragma unroll
    for (int d = 0; d < D; ++d) Q.F.b[d] = Q.x[d] = T(0);
    if constexpr (RD) {
#pragma unroll
      for (int d = 0; d < D; ++d) Q.F.rd[d] = T(0);
    }
    Q.F.fl = 0xFF;  // off the grid: every dof fixed (free mask 0)
    Q.F.rho = (ecol_ok && f >= 0 && f < nely) ? __ldg(rh + (size_t)f * nelx + c) : T(0);
    if (!col_ok || f < 0 || f >= nny) return;
    const long long node = (long long)f * nnx + c;
    Q.F.fl = __ldg(fixed + node);
    load_node<D, T>(bs, node, Q.F.b);
    load_node<D, T>(xs, node, Q.x);
    if constexpr (RD) {
#pragma unroll
      for (int d = 0; d < D; ++d) Q.F.rd[d] = __ldg(rdh + node * D + d);
    }
  };
  ModalStage<D, T> A, B;
  A.reset();
  B.reset();
  DelayRow<D, T, RD> d1{}, d2{};  // rows f - 1 and f - 2
  const int f0 = r0 - 2, f1 = r1 + 1;  // front rows, inclusive
  T rho_prev = (ecol_ok && f0 - 1 >= 0 && f0 - 1 < nely) ? __ldg(rh + (size_t)(f0 - 1) * nelx + c) : T(0);
  // RZ: the sum of b z over the nodes this thread writes
  double dots[1] = {0.0};
  Front qf[AHEAD];
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) load_front(f0 + k, qf[k]);
  for (int fb = f0; fb <= f1; fb += AHEAD) {
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {
      const int f = fb + k;
      const Front Q = qf[k];
      load_front(f + AHEAD, qf[k]);
      const bool emit = out_lane && f - 2 >= r0 && f - 2 < r1;
      DelayRow<D, T, RD> cur;
      {
        const T rs = Q.F.rho + rho_prev;
        const T dsum = rs + __shfl_up_sync(0xffffffffu, rs, 1);
        l0_delay_row<D, T, RD>(Q.F, dsum, q, omega, cur);
      }
      rho_prev = Q.F.rho;
      // stage A: element row f - 1 -> first sweep at node row f - 1
      T KA[D], xa[D], xo_a[D];
#pragma unroll
      for (int d = 0; d < D; ++d) xo_a[d] = A.ut[d];
      A.step(q, Q.x, d1.rho, KA);
      {
        T rd1[D];
#pragma unroll
        for (int d = 0; d < D; ++d) rd1[d] = RD ? d1.rd[d] : T(0);
        l0_chain_result<D, T, SW_SWEEP, RD>(KA, d1.w, d1.mf, xo_a, d1.b, rd1, xa);
      }
      // stage B: element row f - 2 -> second sweep at node row f - 2
      T KB[D], xb[D], xo_b[D];
#pragma unroll
      for (int d = 0; d < D; ++d) xo_b[d] = B.ut[d];
      B.step(q, xa, d2.rho, KB);
      {
        T rd2[D];
#pragma unroll
        for (int d = 0; d < D; ++d) rd2[d] = RD ? d2.rd[d] : T(0);
        l0_chain_result<D, T, SW_SWEEP, RD>(KB, d2.w, d2.mf, xo_b, d2.b, rd2, xb);
      }
      if (emit) {
        store_node<D, T>(os, (long long)(f - 2) * nnx + c, xb);
        if constexpr (RZ) {
          T t = d2.b[0] * xb[0];
#pragma unroll
          for (int d = 1; d < D; ++d) t = fma(d2.b[d], xb[d], t);
          dots[0] += (double)t;
        }
      }
      d2 = d1;
      d1 = cur;
    }
  }
  if constexpr (RZ) {
    if (rz.rst)
      grid_reduce<1, kQThreads>(rz.red, s, blockIdx.y * gridDim.x + blockIdx.x, dots, [&](const double* t) {
        RowState& S = rz.rst[s];
        const double t2[2] = {t[0], S.rz_mix};
        pcg_rz_finish(S, t2, rz.first, rz.flexible);
      });
  }
}

// The launch shapes a solve uses, tunable per hierarchy (stt_hier_tune) and set on the
// calling host thread for the duration of a solve entry point: pcg_band, the rows a block
// of the PCG's level-0 passes marches (8, 16 or 32; 0: the heuristic of pcg_tile_grid);
// waves, the blocks band_rows aims at in units of one block per SM (0: four).
struct LaunchTuning {
  int pcg_band = 0;
  int waves = 0;
};
inline LaunchTuning& launch_tuning() {
  static thread_local LaunchTuning t;
  return t;
}
struct ScopedTuning {
  LaunchTuning saved;
  ScopedTuning(int pcg_band, int waves) : saved(launch_tuning()) { launch_tuning() = LaunchTuning{pcg_band, waves}; }
  ~ScopedTuning() { launch_tuning() = saved; }
};

// Rows a block marches on the coarse levels: 32 where the grid then fills the GPU,
// shorter bands on small grids (the heat solve's single row, the coarse levels), whose
// launches are otherwise latency-bound by the sequential march down 32 rows.  The
// kernels derive their band from gridDim.y, so any grid.y covers the rows.
inline int band_rows(int xblocks, int nny, int rows) {
  const int waves = launch_tuning().waves > 0 ? launch_tuning().waves : 4;
  const long long target = (long long)waves * 148;  // blocks: waves of one block per B200 SM
  for (int band = 32; band > 4; band /= 2)
    if ((long long)xblocks * ((nny + band - 1) / band) * rows >= target) return band;
  return 4;
}

inline dim3 coarse_grid(int nelx, int nely, int rows) {
  const int strips = (nelx + 1 + kQCols - 1) / kQCols;
  const int xb = (strips + kQWarps - 1) / kQWarps;
  const int band = band_rows(xb, nely + 1, rows);
  return dim3(xb, (nely + 1 + band - 1) / band, rows);
}

// ---- stored stencils: layout ---------------------------------------------------------
//
// A level's half stencil holds 5 D^2 coefficients a node (centre, E, S, SE, SW blocks,
// row-major D x D each).  FP64 stencils (the coarse factorisation's input, FP64 cycles)
// are stored by coefficient planes, [rows][5 D^2][nnode].  FP32 stencils (the FP32
// cycle's) are node-major, [rows][nnode][NSP] with NSP = 5 D^2 rounded up to a multiple
// of 4, so a node's coefficients are 16-byte aligned vectors: the column-marching
// kernels load a row's coefficients with 128-bit loads from one address instead of one
// load (and one address) a coefficient.  A level swept from the level-0 densities keeps
// only its centre diagonal, compact in FP32: [rows][nnode][D] within the same extent.
template <int D, typename T>
STT_DEV const T* st_row(const T* st, int h, long long nnode) {
  return st + (size_t)h * (sizeof(T) == 4 ? st32_nsp<D>() : 5 * D * D) * nnode;
}
// coefficient k of node `node` in a row's stencil sth
template <int D, typename T>
STT_DEV T st_coef(const T* sth, long long nnode, long long node, int k) {
  if constexpr (sizeof(T) == 4) return __ldg(sth + node * st32_nsp<D>() + k);
  else return __ldg(sth + (size_t)k * nnode + node);
}
// all 5 D^2 coefficients of a node
template <int D, typename T>
STT_DEV void st_coefs(const T* sth, long long nnode, long long node, T (&co)[5 * D * D]) {
  constexpr int NS = 5 * D * D;
  if constexpr (sizeof(T) == 4) {
    const float4* v = reinterpret_cast<const float4*>(sth + node * st32_nsp<D>());
#pragma unroll
    for (int q = 0; q < (NS + 3) / 4; ++q) {
      const float4 t = __ldg(v + q);
      const float tv[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (4 * q + e < NS) co[4 * q + e] = tv[e];
    }
  } else {
#pragma unroll
    for (int k = 0; k < NS; ++k) co[k] = __ldg(sth + (size_t)k * nnode + node);
  }
}
// the centre block's diagonal of a level swept from the level-0 densities (plane stress)
template <typename T>
STT_DEV void st_diag2(const T* st, int h, long long nnode, long long node, T (&dg)[2]) {
  if constexpr (sizeof(T) == 4) {
    const float2 t = __ldg(reinterpret_cast<const float2*>(st_row<2, T>(st, h, nnode)) + node);
    dg[0] = t.x;
    dg[1] = t.y;
  } else {
    const T* sth = st_row<2, T>(st, h, nnode);
    dg[0] = __ldg(sth + node);
    dg[1] = __ldg(sth + 3 * nnode + node);
  }
}

// ---- stencil levels: column-marching sweeps -----------------------------------------
//
// The symmetric half stencil stores, per node, the centre, E, S, SE, SW blocks; the W,
// N, NW, NE couplings are the transposed E block of the left neighbour (a shuffle), S of
// the node above (this lane's previous row) and SE / SW of the nodes above-left /
// above-right (the neighbours' previous rows, shuffles).  Marching a warp down a strip
// of columns, every coefficient and every vector value is loaded once, coalesced.
//   SW_FIRST / SW_SWEEP / SW_POST / SW_RESID / SW_APPLY as on level 0; x is projected.
template <int D, typename T, int MODE>
__global__ void __launch_bounds__(kQThreads) st_sweep_kernel(
    const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ out, long long vec_rs,
    const T* __restrict__ st, const uint8_t* __restrict__ fixed, int nnx, int nny,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, T omega,
    ProlongSrc<T> pro) {
  constexpr int DD = D * D, NS = 5 * DD;
  constexpr bool KU = MODE != SW_FIRST;
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const long long nnode = (long long)nnx * nny;
  const int h = hier_row(row_map, hrows, s);
  const T* sth = st_row<D, T>(st, h, nnode);
  const T* xs = x + (size_t)s * vec_rs;
  const T* bs = b + (size_t)s * vec_rs;
  T* os = out + (size_t)s * vec_rs;
  const T* es = MODE == SW_POST ? pro.ec + (size_t)s * pro.rs : nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kQCols - 1 + lane;
  const bool out_lane = lane >= 1 && lane <= kQCols && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const int band = (nny + gridDim.y - 1) / gridDim.y;  // rows per block (any grid.y)
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, nny);
  auto X = [&](int r, T(&v)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = T(0);
    if (!KU || !col_ok || r < 0 || r >= nny) return;
    const int node = r * nnx + c;
    load_node<D, T>(xs, node, v);
    if (MODE == SW_POST) {
      T pv[D];
      prolong_at<D, T>(es, pro.cnnx, pro.kx, pro.ky, r, c, pv);
      const uint8_t fl = __ldg(fixed + node);
#pragma unroll
      for (int d = 0; d < D; ++d)
        if (!((fl >> d) & 1)) v[d] += pv[d];
    }
  };
  auto CO = [&](int r, int k) -> T {
    return (col_ok && r >= 0 && r < nny) ? st_coef<D, T>(sth, nnode, (long long)r * nnx + c, k) : T(0);
  };
  auto up = [](T v) { return __shfl_up_sync(0xffffffffu, v, 1); };
  auto dn = [](T v) { return __shfl_down_sync(0xffffffffu, v, 1); };
  T xa[D], xb[D], xal[D], xar[D], xbl[D], xbr[D];
  T pS[DD], pSE[DD], pSW[DD];  // this lane's S, SE, SW blocks of the previous row
  X(r0 - 1, xa);
  X(r0, xb);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    xal[d] = up(xa[d]);
    xar[d] = dn(xa[d]);
    xbl[d] = up(xb[d]);
    xbr[d] = dn(xb[d]);
  }
#pragma unroll
  for (int q = 0; q < DD; ++q) {
    pS[q] = KU ? CO(r0 - 1, 2 * DD + q) : T(0);
    pSE[q] = KU ? CO(r0 - 1, 3 * DD + q) : T(0);
    pSW[q] = KU ? CO(r0 - 1, 4 * DD + q) : T(0);
  }
  // one-row lookahead: coefficients, rhs and flags of row r, input of row r + 1
  auto load_row = [&](int r, T(&Cc)[DD], T(&E)[DD], T(&S)[DD], T(&SE)[DD], T(&SW)[DD], T(&xc)[D], T(&bv)[D],
                      uint8_t& fl) {
    X(r + 1, xc);
#pragma unroll
    for (int q = 0; q < DD; ++q) {
      Cc[q] = CO(r, q);
      E[q] = KU ? CO(r, DD + q) : T(0);
      S[q] = KU ? CO(r, 2 * DD + q) : T(0);
      SE[q] = KU ? CO(r, 3 * DD + q) : T(0);
      SW[q] = KU ? CO(r, 4 * DD + q) : T(0);
    }
    const bool ok = out_lane && r < r1;
    if (MODE != SW_APPLY && ok) {
      load_node<D, T>(bs, (long long)r * nnx + c, bv);
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) bv[d] = T(0);
    }
    fl = ok ? __ldg(fixed + (size_t)r * nnx + c) : (uint8_t)0;
  };
  T Cc[DD], E[DD], S[DD], SE[DD], SW[DD], xc[D], bv[D];
  uint8_t fl;
  load_row(r0, Cc, E, S, SE, SW, xc, bv, fl);
  for (int r = r0; r < r1; ++r) {
    T nC[DD], nE[DD], nS[DD], nSE[DD], nSW[DD], nxc[D], nbv[D];
    uint8_t nfl;
    load_row(r + 1, nC, nE, nS, nSE, nSW, nxc, nbv, nfl);
    T xcl[D], xcr[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      xcl[d] = up(xc[d]);
      xcr[d] = dn(xc[d]);
    }
    T Ax[D];
#pragma unroll
    for (int i = 0; i < D; ++i) Ax[i] = T(0);
    if (KU) {
#pragma unroll
      for (int q = 0; q < DD; ++q) {
        const T Ew = up(E[q]), SEnw = up(pSE[q]), SWne = dn(pSW[q]);
        const int i = q / D, j = q % D;  // block (i, j); transposed blocks contribute (j, i)
        Ax[i] = fma(Cc[q], xb[j], Ax[i]);
        Ax[i] = fma(E[q], xbr[j], Ax[i]);
        Ax[i] = fma(S[q], xc[j], Ax[i]);
        Ax[i] = fma(SE[q], xcr[j], Ax[i]);
        Ax[i] = fma(SW[q], xcl[j], Ax[i]);
        Ax[j] = fma(Ew, xbl[i], Ax[j]);
        Ax[j] = fma(pS[q], xa[i], Ax[j]);
        Ax[j] = fma(SEnw, xal[i], Ax[j]);
        Ax[j] = fma(SWne, xar[i], Ax[j]);
      }
    }
    if (out_lane) {
      const int node = r * nnx + c;
      T res[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        if (MODE == SW_FIRST || MODE == SW_SWEEP || MODE == SW_POST) {
          const T dg = ((fl >> i) & 1) ? T(1) : Cc[i * D + i];
          const T x0 = MODE == SW_FIRST ? T(0) : xb[i];
          res[i] = x0 + sweep_div(omega * (bv[i] - Ax[i]), dg);
        } else if (MODE == SW_RESID) {
          res[i] = bv[i] - Ax[i];
        } else {
          res[i] = Ax[i];
        }
      }
      store_node<D, T>(os, node, res);
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
      xa[d] = xb[d];
      xal[d] = xbl[d];
      xar[d] = xbr[d];
      xb[d] = xc[d];
      xbl[d] = xcl[d];
      xbr[d] = xcr[d];
      xc[d] = nxc[d];
      bv[d] = nbv[d];
    }
#pragma unroll
    for (int q = 0; q < DD; ++q) {
      pS[q] = S[q];
      pSE[q] = SE[q];
      pSW[q] = SW[q];
      Cc[q] = nC[q];
      E[q] = nE[q];
      S[q] = nS[q];
      SE[q] = nSE[q];
      SW[q] = nSW[q];
    }
    fl = nfl;
  }
}

// ---- stencil levels: column-marching sweeps, coupling products shuffled -------------
//
// st_sweep_kernel's operator with the four transposed couplings (W, N, NW, NE) formed by
// the lane that owns the block and shuffled as products: lane c - 1 sends E^T x (the W
// term of node c), the node above keeps S^T x for the row below, lane c - 1 sends SE^T x
// to c (NW of the row below) and lane c + 1 sends SW^T x to c (NE).  Per node that is
// 2 shuffles of x plus 3 of products per component (10 for D = 2) instead of a shuffle
// per coefficient (16), and only the coefficients of the row being emitted are held.
// AHEAD rows of raw loads (coefficients, rhs, flags, and x one row further) stay in
// flight.  Modes as st_sweep_kernel, SW_POST excepted.  dcompact: the level keeps only its
// centre diagonal (FP32, swept from the level-0 densities otherwise), which the first
// sweep from zero, the one pass that reaches such a level here, reads (st_diag2).
template <int D, typename T, int MODE, int AHEAD = 1>
__global__ void __launch_bounds__(kQThreads) st_sweep2_kernel(
    const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ out, long long vec_rs,
    const T* __restrict__ st, const uint8_t* __restrict__ fixed, int nnx, int nny,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, T omega, int dcompact = 0) {
  static_assert(MODE != SW_POST, "no folded prolongation on stencil levels");
  constexpr int DD = D * D, NS = 5 * DD;
  constexpr bool KU = MODE != SW_FIRST;
  constexpr int NC = KU ? NS : DD;  // coefficients read per node
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const long long nnode = (long long)nnx * nny;
  const int h = hier_row(row_map, hrows, s);
  const T* sth = st_row<D, T>(st, h, nnode);
  const T* xs = x + (size_t)s * vec_rs;
  const T* bs = b + (size_t)s * vec_rs;
  T* os = out + (size_t)s * vec_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kQCols - 1 + lane;
  const bool out_lane = lane >= 1 && lane <= kQCols && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const int band = (nny + gridDim.y - 1) / gridDim.y;  // rows per block (any grid.y)
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, nny);
  struct Row {
    T co[NC];   // Cc, E, S, SE, SW of node (r, c)
    T xn[D];    // x(r + 1, c)
    T b[D];
    uint8_t fl;
  };
  auto load_x = [&](int r, T(&v)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = T(0);
    if (KU && col_ok && r >= 0 && r < nny) load_node<D, T>(xs, (long long)r * nnx + c, v);
  };
  auto load_row = [&](int r, Row& R) {
#pragma unroll
    for (int k = 0; k < NC; ++k) R.co[k] = T(0);
#pragma unroll
    for (int d = 0; d < D; ++d) R.b[d] = T(0);
    R.fl = 0;
    load_x(r + 1, R.xn);
    if (!col_ok || r < 0 || r >= nny) return;
    const long long node = (long long)r * nnx + c;
    if constexpr (MODE == SW_FIRST && D == 2) {
      if (dcompact) {
        T dg[2];
        st_diag2<T>(st, h, nnode, node, dg);
        R.co[0] = dg[0];
        R.co[3] = dg[1];  // (the off-diagonal centre entries stay zero: the first sweep reads none)
      } else {
#pragma unroll
        for (int k = 0; k < NC; ++k) R.co[k] = st_coef<D, T>(sth, nnode, node, k);
      }
    } else {
#pragma unroll
      for (int k = 0; k < NC; ++k) R.co[k] = st_coef<D, T>(sth, nnode, node, k);
    }
    if (MODE != SW_APPLY) load_node<D, T>(bs, node, R.b);
    R.fl = __ldg(fixed + node);
  };
  // (B v)_i and (B^T v)_j of a D x D block stored row-major
  auto bx = [](const T* B, const T(&v)[D], T(&acc)[D]) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) acc[i] = fma(B[i * D + j], v[j], acc[i]);
  };
  auto btx = [](const T* B, const T(&v)[D], T(&acc)[D]) {
#pragma unroll
    for (int j = 0; j < D; ++j)
#pragma unroll
      for (int i = 0; i < D; ++i) acc[j] = fma(B[i * D + j], v[i], acc[j]);
  };
  // state: x(r, c), x(r, c + 1), and the N / NW / NE products from row r - 1
  T xr[D], xrr[D], nN[D], nNW[D], nNE[D];
#pragma unroll
  for (int d = 0; d < D; ++d) nN[d] = nNW[d] = nNE[d] = T(0);
  {
    // row r0 - 1 seeds the products for row r0
    T xp[D];
    load_x(r0 - 1, xp);
    load_x(r0, xr);
#pragma unroll
    for (int d = 0; d < D; ++d) xrr[d] = __shfl_down_sync(0xffffffffu, xr[d], 1);
    if constexpr (KU) {
      T Sp[DD], SEp[DD], SWp[DD];
      const bool ok = col_ok && r0 - 1 >= 0;
      const long long node = (long long)(r0 - 1) * nnx + c;
#pragma unroll
      for (int q = 0; q < DD; ++q) {
        Sp[q] = ok ? st_coef<D, T>(sth, nnode, node, 2 * DD + q) : T(0);
        SEp[q] = ok ? st_coef<D, T>(sth, nnode, node, 3 * DD + q) : T(0);
        SWp[q] = ok ? st_coef<D, T>(sth, nnode, node, 4 * DD + q) : T(0);
      }
      T pse[D], psw[D];
#pragma unroll
      for (int d = 0; d < D; ++d) pse[d] = psw[d] = T(0);
      btx(Sp, xp, nN);
      btx(SEp, xp, pse);
      btx(SWp, xp, psw);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        nNW[d] = __shfl_up_sync(0xffffffffu, pse[d], 1);
        nNE[d] = __shfl_down_sync(0xffffffffu, psw[d], 1);
      }
    }
  }
  Row q[AHEAD];
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) load_row(r0 + k, q[k]);
  for (int rb0 = r0; rb0 < r1; rb0 += AHEAD) {
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {
      const int r = rb0 + k;
      const Row R = q[k];
      load_row(r + AHEAD, q[k]);
      T Ax[D];
#pragma unroll
      for (int d = 0; d < D; ++d) Ax[d] = T(0);
      T xnl[D], xnr[D];
      if constexpr (KU) {
        const T* Cc = R.co;
        const T* E = R.co + DD;
        const T* S = R.co + 2 * DD;
        const T* SE = R.co + 3 * DD;
        const T* SW = R.co + 4 * DD;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          xnl[d] = __shfl_up_sync(0xffffffffu, R.xn[d], 1);
          xnr[d] = __shfl_down_sync(0xffffffffu, R.xn[d], 1);
        }
        T wp[D], pse[D], psw[D], pn[D];
#pragma unroll
        for (int d = 0; d < D; ++d) wp[d] = pse[d] = psw[d] = pn[d] = T(0);
        btx(E, xr, wp);    // W term of the right neighbour
        btx(S, xr, pn);    // N term of the node below
        btx(SE, xr, pse);  // NW term of the node below-right
        btx(SW, xr, psw);  // NE term of the node below-left
        bx(Cc, xr, Ax);
        bx(E, xrr, Ax);
        bx(S, R.xn, Ax);
        bx(SE, xnr, Ax);
        bx(SW, xnl, Ax);
#pragma unroll
        for (int d = 0; d < D; ++d) {
          Ax[d] += __shfl_up_sync(0xffffffffu, wp[d], 1);
          Ax[d] += nN[d] + nNW[d] + nNE[d];
          nN[d] = pn[d];
          nNW[d] = __shfl_up_sync(0xffffffffu, pse[d], 1);
          nNE[d] = __shfl_down_sync(0xffffffffu, psw[d], 1);
        }
      }
      if (out_lane && r < r1) {
        T res[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
          if (MODE == SW_FIRST || MODE == SW_SWEEP) {
            const T dg = ((R.fl >> i) & 1) ? T(1) : R.co[i * D + i];
            const T x0 = MODE == SW_FIRST ? T(0) : xr[i];
            res[i] = x0 + sweep_div(omega * (R.b[i] - Ax[i]), dg);
          } else if (MODE == SW_RESID) {
            res[i] = R.b[i] - Ax[i];
          } else {
            res[i] = Ax[i];
          }
        }
        store_node<D, T>(os, (long long)r * nnx + c, res);
      }
      if constexpr (KU) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
          xr[d] = R.xn[d];
          xrr[d] = xnr[d];
        }
      }
    }
  }
}

// ---- stencil levels: smoothing chained in one pass ---------------------------------------
//
// st_sweep2_kernel's passes chained like l0_presmooth_kernel: PRE runs the first sweep from
// zero, a sweep and the residual (writes x2 and r); POST runs two sweeps from x0 (writes
// x2).  Stage A emits node row f - 1 for the front row f, stage B node row f - 2 from stage
// A's output, so the intermediate iterate never leaves registers.  Stage B reads stage
// A's coefficient rows one step later, from cache.  Lanes 2..29 are output (28 columns a
// warp).
constexpr int kStChainCols = 28;

inline dim3 st_chain_grid(int nelx, int nely, int rows) {
  const int strips = (nelx + 1 + kStChainCols - 1) / kStChainCols;
  const int xb = (strips + kQWarps - 1) / kQWarps;
  const int band = band_rows(xb, nely + 1, rows);
  return dim3(xb, (nely + 1 + band - 1) / band, rows);
}

// One stage of the half-stencil operator (st_sweep2_kernel's march): the x of the row
// being emitted and of its right neighbour, and the N / NW / NE products carried from the
// row above.
template <int D, typename T>
struct StStage {
  T xr[D], xrr[D], nN[D], nNW[D], nNE[D];
  STT_DEV void reset() {
#pragma unroll
    for (int d = 0; d < D; ++d) xr[d] = xrr[d] = nN[d] = nNW[d] = nNE[d] = T(0);
  }
  // (A x) at the current row from its coefficients co (Cc, E, S, SE, SW) and the next
  // row's x; then the next row becomes current
  STT_DEV void step(const T* co, const T (&xn)[D], T (&Ax)[D]) {
    constexpr int DD = D * D;
    const T* Cc = co;
    const T* E = co + DD;
    const T* S = co + 2 * DD;
    const T* SE = co + 3 * DD;
    const T* SW = co + 4 * DD;
    T xnl[D], xnr[D], wp[D], pse[D], psw[D], pn[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      xnl[d] = __shfl_up_sync(0xffffffffu, xn[d], 1);
      xnr[d] = __shfl_down_sync(0xffffffffu, xn[d], 1);
      wp[d] = pse[d] = psw[d] = pn[d] = Ax[d] = T(0);
    }
#pragma unroll
    for (int j = 0; j < D; ++j)
#pragma unroll
      for (int i = 0; i < D; ++i) {
        wp[j] = fma(E[i * D + j], xr[i], wp[j]);    // W term of the right neighbour
        pn[j] = fma(S[i * D + j], xr[i], pn[j]);    // N term of the node below
        pse[j] = fma(SE[i * D + j], xr[i], pse[j]);  // NW term of the node below-right
        psw[j] = fma(SW[i * D + j], xr[i], psw[j]);  // NE term of the node below-left
      }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        Ax[i] = fma(Cc[i * D + j], xr[j], Ax[i]);
        Ax[i] = fma(E[i * D + j], xrr[j], Ax[i]);
        Ax[i] = fma(S[i * D + j], xn[j], Ax[i]);
        Ax[i] = fma(SE[i * D + j], xnr[j], Ax[i]);
        Ax[i] = fma(SW[i * D + j], xnl[j], Ax[i]);
      }
#pragma unroll
    for (int d = 0; d < D; ++d) {
      Ax[d] += __shfl_up_sync(0xffffffffu, wp[d], 1);
      Ax[d] += nN[d] + nNW[d] + nNE[d];
      nN[d] = pn[d];
      nNW[d] = __shfl_up_sync(0xffffffffu, pse[d], 1);
      nNE[d] = __shfl_down_sync(0xffffffffu, psw[d], 1);
      xr[d] = xn[d];
      xrr[d] = xnr[d];
    }
  }
};

template <int D, typename T, bool PRE>
__global__ void __launch_bounds__(kQThreads, 6) st_chain_kernel(
    const T* __restrict__ x0, const T* __restrict__ b, T* __restrict__ out_x, T* __restrict__ out_r,
    long long vec_rs, const T* __restrict__ st, const uint8_t* __restrict__ fixed, int nnx, int nny,
    const int* __restrict__ row_map, int hrows, const RowState* __restrict__ rst, T omega) {
  constexpr int DD = D * D, NS = 5 * DD, LO = 2, HI = 29;
  static_assert(HI - LO + 1 == kStChainCols, "strip width");
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const long long nnode = (long long)nnx * nny;
  const int h = hier_row(row_map, hrows, s);
  const T* sth = st_row<D, T>(st, h, nnode);
  const T* xs = PRE ? nullptr : x0 + (size_t)s * vec_rs;
  const T* bs = b + (size_t)s * vec_rs;
  T* ox = out_x + (size_t)s * vec_rs;
  T* orr = PRE ? out_r + (size_t)s * vec_rs : nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kStChainCols - LO + lane;
  const bool out_lane = lane >= LO && lane <= HI && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const int band = (nny + gridDim.y - 1) / gridDim.y;  // rows per block (any grid.y)
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, nny);
  // a node row's coefficients, right-hand side and flags (zero outside the grid)
  struct Row {
    T co[NS];
    T b[D];
    uint8_t fl;
  };
  auto load_row = [&](int r, Row& R) {
#pragma unroll
    for (int k = 0; k < NS; ++k) R.co[k] = T(0);
#pragma unroll
    for (int d = 0; d < D; ++d) R.b[d] = T(0);
    R.fl = 0;
    if (!col_ok || r < 0 || r >= nny) return;
    const long long node = (long long)r * nnx + c;
    st_coefs<D, T>(sth, nnode, node, R.co);
    load_node<D, T>(bs, node, R.b);
    R.fl = __ldg(fixed + node);
  };
  // stage A's input at the front row f: the first sweep from zero (PRE: the diagonal,
  // b, flags) or the loaded x0 (POST)
  struct Front {
    T v[D];
    T dg[PRE ? D : 1];
    uint8_t fl;
  };
  auto load_front = [&](int f, Front& F) {
#pragma unroll
    for (int d = 0; d < D; ++d) F.v[d] = T(0);
    F.fl = 0;
    if constexpr (PRE) {
#pragma unroll
      for (int d = 0; d < D; ++d) F.dg[d] = T(0);
    }
    if (!col_ok || f < 0 || f >= nny) return;
    const long long node = (long long)f * nnx + c;
    if constexpr (PRE) {
      load_node<D, T>(bs, node, F.v);
#pragma unroll
      for (int d = 0; d < D; ++d) F.dg[d] = st_coef<D, T>(sth, nnode, node, d * D + d);
      F.fl = __ldg(fixed + node);
    } else {
      load_node<D, T>(xs, node, F.v);
    }
  };
  auto sweep_at = [&](const T(&Ax)[D], const T(&xo)[D], const Row& R, T(&res)[D]) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const T dg = ((R.fl >> i) & 1) ? T(1) : R.co[i * D + i];
      res[i] = xo[i] + sweep_div(omega * (R.b[i] - Ax[i]), dg);
    }
  };
  StStage<D, T> A, B;
  A.reset();
  B.reset();
  // D = 1: stage A's coefficient row streams one step ahead; D = 2: loaded at the step
  // (its 20 coefficients a row would cost the registers of two more blocks an SM)
  constexpr bool PF = D == 1;
  const int f0 = r0 - 2, f1 = r1 + 1;  // front rows, inclusive
  Front qf;
  Row qa;
  load_front(f0, qf);
  if constexpr (PF) load_row(f0 - 1, qa);
  for (int f = f0; f <= f1; ++f) {
    const Front F = qf;
    load_front(f + 1, qf);
    Row RA;  // stage A's row (f - 1)
    if constexpr (PF) {
      RA = qa;
      load_row(f, qa);
    } else {
      load_row(f - 1, RA);
    }
    Row RB;  // stage B's row (f - 2): stage A's row of the previous step, from cache
    load_row(f - 2, RB);
    T xin[D];
    if constexpr (PRE) {
      const bool in = col_ok && f >= 0 && f < nny;  // (outside, the diagonal is zero)
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const T dg = ((F.fl >> i) & 1) ? T(1) : F.dg[i];
        xin[i] = in ? sweep_div(omega * F.v[i], dg) : T(0);
      }
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) xin[d] = F.v[d];
    }
    // stage A: a sweep at node row f - 1
    T KA[D], xa[D], xo_a[D];
#pragma unroll
    for (int d = 0; d < D; ++d) xo_a[d] = A.xr[d];
    A.step(RA.co, xin, KA);
    sweep_at(KA, xo_a, RA, xa);
    if (!(col_ok && f - 1 >= 0 && f - 1 < nny)) {
#pragma unroll
      for (int d = 0; d < D; ++d) xa[d] = T(0);
    }
    // stage B: the residual (PRE) or a second sweep (POST) at node row f - 2
    T KB[D], xbr[D], xo_b[D];
#pragma unroll
    for (int d = 0; d < D; ++d) xo_b[d] = B.xr[d];
    B.step(RB.co, xa, KB);
    if constexpr (PRE) {
#pragma unroll
      for (int d = 0; d < D; ++d) xbr[d] = RB.b[d] - KB[d];
    } else {
      sweep_at(KB, xo_b, RB, xbr);
    }
    if (out_lane) {
      if constexpr (PRE) {
        if (f - 1 >= r0 && f - 1 < r1) store_node<D, T>(ox, (long long)(f - 1) * nnx + c, xa);
        if (f - 2 >= r0 && f - 2 < r1) store_node<D, T>(orr, (long long)(f - 2) * nnx + c, xbr);
      } else {
        if (f - 2 >= r0 && f - 2 < r1) store_node<D, T>(ox, (long long)(f - 2) * nnx + c, xbr);
      }
    }
  }
}

// ---- level 1 from the level-0 densities (plane stress) --------------------------------
//
// The Galerkin element matrices of level 1 are keff[E] = sum over E's KX x KY children
// m of rho_m S_m^T KE S_m (torch_mg.build_hierarchy, sttopt/torch_mg.py:355-370, on the
// level-0 element matrices rho KE).  Each S_m^T KE S_m annihilates the coarse
// translations, so it is T^T M_m T in the element's edge modes (march_modal), with M_m a
// symmetric 6 x 6 computed on the host.  A level-1 sweep therefore reads KX*KY densities
// per element (16 B for 2 x 2, FP32) instead of 20 stencil coefficients per node (80 B):
// per element M = sum_m rho_m M_m, q = M (Gx, Gy, H modes), corner forces as
// march_modal.  The Jacobi diagonal comes from the stored stencil's centre block (the
// projected operator's diagonal).  Sweep and residual modes; the first sweep from zero
// needs only the diagonal and stays on the stencil kernel.
template <typename T, int NM>
struct L1Mat {
  T m[NM][21];  // packed upper triangle, row-major
};

// MIR (2 x 2 children whose M_m mirror M_0): M = sum_m rho_m M_m takes four signed
// density sums and one product per entry, M[e] = M_0[e] (rho_00 + sx rho_10 + sy rho_01
// + sx sy rho_11), instead of four multiply-adds per entry.
template <typename T, int MODE, int KX, int KY, int AHEAD = 2, bool MIR = false>
__global__ void __launch_bounds__(kQThreads) l1_sweep_kernel(
    const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ out, long long vec_rs,
    const T* __restrict__ rho0, long long rho_rs, int fnelx, const T* __restrict__ st,
    const uint8_t* __restrict__ fixed, int nnx, int nny, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst, T omega, L1Mat<T, MIR ? 1 : KX * KY> M) {
  static_assert(MODE == SW_SWEEP || MODE == SW_RESID, "sweep and residual only");
  constexpr int D = 2, NM = KX * KY;
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const long long nnode = (long long)nnx * nny;
  const int h = hier_row(row_map, hrows, s);
  const T* rh = rho0 + (size_t)h * rho_rs;
  const T* xs = x + (size_t)s * vec_rs;
  const T* bs = b + (size_t)s * vec_rs;
  T* os = out + (size_t)s * vec_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kQCols - 1 + lane;
  const bool out_lane = lane >= 1 && lane <= kQCols && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const int nelx = nnx - 1, nely = nny - 1;
  const bool ecol_ok = c >= 0 && c < nelx;
  const int band = (nny + gridDim.y - 1) / gridDim.y;  // rows per block (any grid.y)
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, nny);
  struct Ex {
    T b[D], dg[D];
    uint8_t fl;
  };
  auto X = [&](int r, T(&v)[D]) {
    v[0] = v[1] = T(0);
    if (col_ok && r >= 0 && r < nny) load_node<D, T>(xs, (long long)r * nnx + c, v);
  };
  auto Rho = [&](int r, T(&rm)[NM]) {
    const bool ok = ecol_ok && r >= 0 && r < nely;
#pragma unroll
    for (int my = 0; my < KY; ++my)
#pragma unroll
      for (int mx = 0; mx < KX; ++mx)
        rm[my * KX + mx] = ok ? __ldg(rh + (size_t)(KY * r + my) * fnelx + KX * c + mx) : T(0);
  };
  auto Ext = [&](int r, Ex& e) {
    e.b[0] = e.b[1] = e.dg[0] = e.dg[1] = T(0);
    e.fl = 0;
    if (!(out_lane && r < r1)) return;
    const long long node = (long long)r * nnx + c;
    load_node<D, T>(bs, node, e.b);
    st_diag2<T>(st, h, nnode, node, e.dg);
    e.fl = __ldg(fixed + node);
  };
  T ut[D], sT[D], dT[D], co[D], cr[D];
  auto edge = [&](const T(&v)[D], T(&sv)[D], T(&dv)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const T vr = __shfl_down_sync(0xffffffffu, v[d], 1);
      sv[d] = v[d] + vr;
      dv[d] = vr - v[d];
    }
  };
  auto step = [&](const T(&ub)[D], const T(&rm)[NM], T(&own)[D], T(&send)[D]) {
    T sB[D], dB[D];
    edge(ub, sB, dB);
    T md[6];
    md[0] = dB[0] + dT[0];  // Gx(ux)
    md[1] = sT[1] - sB[1];  // Gy(uy)
    md[2] = sT[0] - sB[0];  // Gy(ux)
    md[3] = dB[1] + dT[1];  // Gx(uy)
    md[4] = dT[0] - dB[0];  // H(ux)
    md[5] = dT[1] - dB[1];  // H(uy)
    T Me[21];
    if constexpr (MIR && NM == 4) {
      const T p0 = rm[0] + rm[1], p1 = rm[0] - rm[1], q0 = rm[2] + rm[3], q1 = rm[2] - rm[3];
      const T cpp = p0 + q0, cmp = p1 + q1, cpm = p0 - q0, cmm = p1 - q1;  // (sx, sy) = (+,+), (-,+), ...
      int e = 0;
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 6; ++j, ++e) {
          const bool sxn = mode_dx(i) * mode_dx(j) < 0, syn = mode_dy(i) * mode_dy(j) < 0;
          Me[e] = M.m[0][e] * (sxn ? (syn ? cmm : cmp) : (syn ? cpm : cpp));
        }
    } else {
#pragma unroll
      for (int e = 0; e < 21; ++e) {
        T a = rm[0] * M.m[0][e];
#pragma unroll
        for (int m = 1; m < NM; ++m) a = fma(rm[m], M.m[m][e], a);
        Me[e] = a;
      }
    }
    T q[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) q[i] = T(0);
    int e = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j, ++e) {
        q[i] = fma(Me[e], md[j], q[i]);
        if (j != i) q[j] = fma(Me[e], md[i], q[j]);
      }
    modal_corners(q[0], q[2], q[4], co[0], cr[0], own[0], send[0]);
    modal_corners(q[3], q[1], q[5], co[1], cr[1], own[1], send[1]);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      sT[d] = sB[d];
      dT[d] = dB[d];
    }
  };
  {
    T u0[D], own[D], send[D], rm[NM];
    X(r0 - 1, u0);
    edge(u0, sT, dT);
    co[0] = co[1] = cr[0] = cr[1] = T(0);
    X(r0, ut);
    Rho(r0 - 1, rm);
    step(ut, rm, own, send);
  }
  T qx[AHEAD][D], qr[AHEAD][NM];
  Ex qe[AHEAD];
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) {
    X(r0 + 1 + k, qx[k]);
    Rho(r0 + k, qr[k]);
    Ext(r0 + k, qe[k]);
  }
  for (int rb0 = r0; rb0 < r1; rb0 += AHEAD) {
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {
      const int r = rb0 + k;
      T ub[D], rm[NM];
#pragma unroll
      for (int d = 0; d < D; ++d) ub[d] = qx[k][d];
#pragma unroll
      for (int m = 0; m < NM; ++m) rm[m] = qr[k][m];
      const Ex ex = qe[k];
      X(r + 1 + AHEAD, qx[k]);
      Rho(r + AHEAD, qr[k]);
      Ext(r + AHEAD, qe[k]);
      T own[D], send[D], Ax[D];
      step(ub, rm, own, send);
#pragma unroll
      for (int d = 0; d < D; ++d) Ax[d] = own[d] + __shfl_up_sync(0xffffffffu, send[d], 1);
      if (out_lane && r < r1) {
        T res[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
          if ((ex.fl >> i) & 1) Ax[i] = T(0);
          if constexpr (MODE == SW_SWEEP) {
            const T dg = ((ex.fl >> i) & 1) ? T(1) : ex.dg[i];
            res[i] = ut[i] + sweep_div(omega * (ex.b[i] - Ax[i]), dg);
          } else {
            res[i] = ex.b[i] - Ax[i];
          }
        }
        store_node<D, T>(os, (long long)r * nnx + c, res);
      }
#pragma unroll
      for (int d = 0; d < D; ++d) ut[d] = ub[d];
    }
  }
}

// ---- level 1: smoothing chained in one pass (plane stress, 2 x 2 children) ---------------
//
// l1_sweep_kernel's passes chained like level 0's (l0_presmooth_kernel): PRE runs the
// first sweep from zero, a sweep and the residual (writes x2 and r); POST runs two sweeps
// from the prolonged iterate x0 (writes x2).  Stage A works on element row f - 1 for the
// front row f, stage B on element row f - 2 with the element matrices stage A assembled a
// step earlier, so each element's M = sum_m rho_m M_m is formed once per pass.  The
// Jacobi diagonal is the stored stencil's centre diagonal (as l1_sweep_kernel).  Lanes
// 2..29 are output (28 columns a warp).
constexpr int kL1ChainCols = 28;

inline dim3 l1_chain_grid(int nelx, int nely, int rows) {
  const int strips = (nelx + 1 + kL1ChainCols - 1) / kL1ChainCols;
  return dim3((strips + kQWarps - 1) / kQWarps, (nely + 1 + kQRows - 1) / kQRows, rows);
}

// One element-row stage of the level-1 modal operator (l1_sweep_kernel's step).
template <typename T>
struct L1Stage {
  T sT[2], dT[2], co[2], cr[2], ut[2];
  STT_DEV void reset() {
#pragma unroll
    for (int d = 0; d < 2; ++d) sT[d] = dT[d] = co[d] = cr[d] = ut[d] = T(0);
  }
  STT_DEV void step(const T (&Me)[21], const T (&ub)[2], T (&Ku)[2]) {
    T sB[2], dB[2];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const T vr = __shfl_down_sync(0xffffffffu, ub[d], 1);
      sB[d] = ub[d] + vr;
      dB[d] = vr - ub[d];
    }
    T md[6];
    md[0] = dB[0] + dT[0];  // Gx(ux)
    md[1] = sT[1] - sB[1];  // Gy(uy)
    md[2] = sT[0] - sB[0];  // Gy(ux)
    md[3] = dB[1] + dT[1];  // Gx(uy)
    md[4] = dT[0] - dB[0];  // H(ux)
    md[5] = dT[1] - dB[1];  // H(uy)
    T q[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) q[i] = T(0);
    int e = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j, ++e) {
        q[i] = fma(Me[e], md[j], q[i]);
        if (j != i) q[j] = fma(Me[e], md[i], q[j]);
      }
    T own[2], send[2];
    modal_corners(q[0], q[2], q[4], co[0], cr[0], own[0], send[0]);
    modal_corners(q[3], q[1], q[5], co[1], cr[1], own[1], send[1]);
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      Ku[d] = own[d] + __shfl_up_sync(0xffffffffu, send[d], 1);
      sT[d] = sB[d];
      dT[d] = dB[d];
      ut[d] = ub[d];
    }
  }
};

// M = sum over the 2 x 2 children of rho_m M_m (mirror form when MIR, as l1_sweep_kernel).
template <typename T, bool MIR>
STT_DEV void l1_assemble(const T (&rm)[4], const L1Mat<T, MIR ? 1 : 4>& M, T (&Me)[21]) {
  if constexpr (MIR) {
    const T p0 = rm[0] + rm[1], p1 = rm[0] - rm[1], q0 = rm[2] + rm[3], q1 = rm[2] - rm[3];
    const T cpp = p0 + q0, cmp = p1 + q1, cpm = p0 - q0, cmm = p1 - q1;
    int e = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j, ++e) {
        const bool sxn = mode_dx(i) * mode_dx(j) < 0, syn = mode_dy(i) * mode_dy(j) < 0;
        Me[e] = M.m[0][e] * (sxn ? (syn ? cmm : cmp) : (syn ? cpm : cpp));
      }
  } else {
#pragma unroll
    for (int e = 0; e < 21; ++e) {
      T a = rm[0] * M.m[0][e];
#pragma unroll
      for (int m = 1; m < 4; ++m) a = fma(rm[m], M.m[m][e], a);
      Me[e] = a;
    }
  }
}

template <typename T, bool PRE, bool MIR, int AHEAD = 2>
__global__ void __launch_bounds__(kQThreads, 4) l1_chain_kernel(
    const T* __restrict__ x0, const T* __restrict__ b, T* __restrict__ out_x, T* __restrict__ out_r,
    long long vec_rs, const T* __restrict__ rho0, long long rho_rs, int fnelx, const T* __restrict__ st,
    const uint8_t* __restrict__ fixed, int nnx, int nny, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst, T omega, L1Mat<T, MIR ? 1 : 4> M) {
  constexpr int D = 2, LO = 2, HI = 29;
  static_assert(HI - LO + 1 == kL1ChainCols, "strip width");
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const long long nnode = (long long)nnx * nny;
  const int h = hier_row(row_map, hrows, s);
  const T* rh = rho0 + (size_t)h * rho_rs;
  const T* xs = PRE ? nullptr : x0 + (size_t)s * vec_rs;
  const T* bs = b + (size_t)s * vec_rs;
  T* ox = out_x + (size_t)s * vec_rs;
  T* orr = PRE ? out_r + (size_t)s * vec_rs : nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int c = strip * kL1ChainCols - LO + lane;
  const bool out_lane = lane >= LO && lane <= HI && c < nnx;
  const bool col_ok = c >= 0 && c < nnx;
  const int nelx = nnx - 1, nely = nny - 1;
  const bool ecol_ok = c >= 0 && c < nelx;
  const int r0 = blockIdx.y * kQRows;
  const int r1 = min(r0 + kQRows, nny);
  struct Front {
    T b[D], dg[D], x[D], rm[4];
    uint8_t fl;
  };
  auto load_rm = [&](int f, T(&rm)[4]) {
    const bool ok = ecol_ok && f >= 0 && f < nely;
#pragma unroll
    for (int my = 0; my < 2; ++my)
#pragma unroll
      for (int mx = 0; mx < 2; ++mx)
        rm[my * 2 + mx] = ok ? __ldg(rh + (size_t)(2 * f + my) * fnelx + 2 * c + mx) : T(0);
  };
  auto load_front = [&](int f, Front& Q) {
#pragma unroll
    for (int d = 0; d < D; ++d) Q.b[d] = Q.dg[d] = Q.x[d] = T(0);
    Q.fl = 0xFF;  // off-grid positions count as fixed: their results are masked to zero
    load_rm(f, Q.rm);
    if (!col_ok || f < 0 || f >= nny) return;
    const long long node = (long long)f * nnx + c;
    Q.fl = __ldg(fixed + node);
    load_node<D, T>(bs, node, Q.b);
    st_diag2<T>(st, h, nnode, node, Q.dg);
    if constexpr (!PRE) load_node<D, T>(xs, node, Q.x);
  };
  // per node row, formed once at the front: b, w = omega / diag and the free mask mf (1 on
  // free dofs, 0 on fixed and off-grid ones, where the diagonal is taken as 1)
  struct Delay {
    T b[D], w[D], mf[D];
  };
  auto delay_of = [&](const Front& Q, Delay& e) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const bool fr = !((Q.fl >> d) & 1);
      e.mf[d] = fr ? T(1) : T(0);
      e.w[d] = sweep_div(omega, fr ? Q.dg[d] : T(1));
      e.b[d] = Q.b[d];
    }
  };
  // the first sweep from zero, a sweep or the residual at a node from K x there (masked)
  auto result = [&](auto mode, const T(&Kx)[D], const T(&xo)[D], const Delay& e, T(&res)[D]) {
    T Ax[D] = {Kx[0], Kx[1]};
    const T rd[D] = {T(0), T(0)};
    l0_chain_result<D, T, decltype(mode)::value, false>(Ax, e.w, e.mf, xo, e.b, rd, res);
  };
  using First = std::integral_constant<int, SW_FIRST>;
  using Sweep = std::integral_constant<int, SW_SWEEP>;
  using Resid = std::integral_constant<int, SW_RESID>;
  L1Stage<T> A, B;
  A.reset();
  B.reset();
  Delay d1{}, d2{};  // node rows f - 1 and f - 2 (all-zero: masked out)
  const int f0 = r0 - 2, f1 = r1 + 1;  // front rows, inclusive
  T rm_prev[4];  // children of element row f - 1
  load_rm(f0 - 1, rm_prev);
  T MeB[21];  // element row f - 2's matrix, from stage A a step earlier
#pragma unroll
  for (int e = 0; e < 21; ++e) MeB[e] = T(0);
  Front qf[AHEAD];
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) load_front(f0 + k, qf[k]);
  for (int fb = f0; fb <= f1; fb += AHEAD) {
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) {
      const int f = fb + k;
      const Front Q = qf[k];
      load_front(f + AHEAD, qf[k]);
      Delay cur;
      delay_of(Q, cur);
      // stage A's input at row f: the first sweep from zero (PRE) or the loaded x0
      T xin[D];
      if constexpr (PRE) {
        const T zero[D] = {T(0), T(0)};
        result(First{}, zero, zero, cur, xin);
      } else {
#pragma unroll
        for (int d = 0; d < D; ++d) xin[d] = Q.x[d];
      }
      // stage A: element row f - 1 -> a sweep at node row f - 1
      T MeA[21];
      l1_assemble<T, MIR>(rm_prev, M, MeA);
      T KA[D], xa[D], xo_a[D];
#pragma unroll
      for (int d = 0; d < D; ++d) xo_a[d] = A.ut[d];
      A.step(MeA, xin, KA);
      result(Sweep{}, KA, xo_a, d1, xa);
      // stage B: element row f - 2 -> the residual (PRE) or a second sweep at node row f - 2
      T KB[D], xbr[D], xo_b[D];
#pragma unroll
      for (int d = 0; d < D; ++d) xo_b[d] = B.ut[d];
      B.step(MeB, xa, KB);
      if constexpr (PRE) result(Resid{}, KB, xo_b, d2, xbr);
      else result(Sweep{}, KB, xo_b, d2, xbr);
      if (out_lane) {
        if constexpr (PRE) {
          if (f - 1 >= r0 && f - 1 < r1) store_node<D, T>(ox, (long long)(f - 1) * nnx + c, xa);
          if (f - 2 >= r0 && f - 2 < r1) store_node<D, T>(orr, (long long)(f - 2) * nnx + c, xbr);
        } else {
          if (f - 2 >= r0 && f - 2 < r1) store_node<D, T>(ox, (long long)(f - 2) * nnx + c, xbr);
        }
      }
#pragma unroll
      for (int e = 0; e < 21; ++e) MeB[e] = MeA[e];
#pragma unroll
      for (int m = 0; m < 4; ++m) rm_prev[m] = Q.rm[m];
      d2 = d1;
      d1 = cur;
    }
  }
}

// ---- restriction: column-marching full weighting ---------------------------------
//
// rc = P_c (R r_f), the x pass then the y pass of torch_mg._restrict_axis
// (sttopt/torch_mg.py:84-93): per axis, (block I weighted 1 - j/k) + (block I-1 weighted
// j/k), the last fine value landing on the last coarse node.  A warp marches down a
// strip of coarse columns; each lane loads its coarse column's own kx fine columns and
// takes the left neighbour's from the lane beside it, so every fine value is loaded
// once.  The x-pass values of the fine rows shared by consecutive coarse rows are kept.
template <int D, typename T>
__global__ void __launch_bounds__(kQThreads) restrict_kernel(
    const T* __restrict__ rf, long long f_rs, int fnnx, int fnny, T* __restrict__ rc, long long c_rs,
    int cnnx, int cnny, int kx, int ky, const uint8_t* __restrict__ cfixed,
    const RowState* __restrict__ rst) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const T* f = rf + (size_t)s * f_rs;
  T* o = rc + (size_t)s * c_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int C = strip * kQCols - 1 + lane;
  const bool out_lane = lane >= 1 && lane <= kQCols && C < cnnx;
  const bool col_ok = C >= 0 && C < cnnx;
  const int band = (cnny + gridDim.y - 1) / gridDim.y;  // coarse rows per block (any grid.y)
  const int R0 = blockIdx.y * band;
  const int R1 = min(R0 + band, cnny);
  // x pass of fine row fr at this lane's coarse column
  auto xpass = [&](int fr, T(&g)[D]) {
    T own[3][D], left[3][D];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int fc = kx * C + j;
      const bool ok = j < kx && col_ok && fr >= 0 && fr < fnny && fc < fnnx;
      T v[D];
      if (ok) {
        load_node<D, T>(f, (long long)fr * fnnx + fc, v);
      } else {
#pragma unroll
        for (int d = 0; d < D; ++d) v[d] = T(0);
      }
#pragma unroll
      for (int d = 0; d < D; ++d) {
        own[j][d] = v[d];
        left[j][d] = __shfl_up_sync(0xffffffffu, v[d], 1);
      }
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (kx == 1) {
        g[d] = own[0][d];
        continue;
      }
      T lo = T(0), hi = T(0);
#pragma unroll
      for (int j = 0; j < 3; ++j)
        if (j < kx) lo += own[j][d] * T(1.0 - (double)j / kx);
#pragma unroll
      for (int j = 1; j < 3; ++j)
        if (j < kx) hi += left[j][d] * T((double)j / kx);
      g[d] = lo + hi;
    }
  };
  T gprev[3][D];  // x-pass values of fine rows ky (R-1) + j, j = 1 .. ky-1
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    if (j >= 1 && j < ky && R0 >= 1) {
      xpass(ky * (R0 - 1) + j, gprev[j]);
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) gprev[j][d] = T(0);
    }
  }
  for (int R = R0; R < R1; ++R) {
    T gcur[3][D];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if (j < ky) {
        xpass(ky * R + j, gcur[j]);
      } else {
#pragma unroll
        for (int d = 0; d < D; ++d) gcur[j][d] = T(0);
      }
    }
    if (out_lane) {
      const uint8_t fl = cfixed ? __ldg(cfixed + (size_t)R * cnnx + C) : uint8_t(0);  // null: no projection
      T v[D];
#pragma unroll
      for (int d = 0; d < D; ++d) {
        if (ky == 1) {
          v[d] = gcur[0][d];
        } else {
          T lo = T(0), hi = T(0);
#pragma unroll
          for (int j = 0; j < 3; ++j)
            if (j < ky) lo += gcur[j][d] * T(1.0 - (double)j / ky);
#pragma unroll
          for (int j = 1; j < 3; ++j)
            if (j < ky) hi += gprev[j][d] * T((double)j / ky);
          v[d] = lo + hi;
        }
        if ((fl >> d) & 1) v[d] = T(0);
      }
      store_node<D, T>(o, (long long)R * cnnx + C, v);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int d = 0; d < D; ++d) gprev[j][d] = gcur[j][d];
  }
}

// Restriction as restrict_kernel with the coarsening factors as template parameters
// (constant weights, no divisions) and the next coarse row's fine rows loaded while the
// current one is combined.
template <int D, typename T, int KX, int KY>
__global__ void __launch_bounds__(kQThreads) restrict_t_kernel(
    const T* __restrict__ rf, long long f_rs, int fnnx, int fnny, T* __restrict__ rc, long long c_rs,
    int cnnx, int cnny, const uint8_t* __restrict__ cfixed, const RowState* __restrict__ rst) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const T* f = rf + (size_t)s * f_rs;
  T* o = rc + (size_t)s * c_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kQWarps + warp;
  const int C = strip * kQCols - 1 + lane;
  const bool out_lane = lane >= 1 && lane <= kQCols && C < cnnx;
  const bool col_ok = C >= 0 && C < cnnx;
  const int band = (cnny + gridDim.y - 1) / gridDim.y;  // coarse rows per block (any grid.y)
  const int R0 = blockIdx.y * band;
  const int R1 = min(R0 + band, cnny);
  struct FRow {
    T v[KX][D];
  };
  auto fload = [&](int fr, FRow& q) {
#pragma unroll
    for (int j = 0; j < KX; ++j) {
      const int fc = KX * C + j;
      if (col_ok && fr >= 0 && fr < fnny && fc < fnnx) {
        load_node<D, T>(f, (long long)fr * fnnx + fc, q.v[j]);
      } else {
#pragma unroll
        for (int d = 0; d < D; ++d) q.v[j][d] = T(0);
      }
    }
  };
  auto xpass = [&](const FRow& q, T(&g)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if constexpr (KX == 1) {
        g[d] = q.v[0][d];
      } else {
        T lo = T(0), hi = T(0);
#pragma unroll
        for (int j = 0; j < KX; ++j) lo += q.v[j][d] * T(1.0 - (double)j / KX);
#pragma unroll
        for (int j = 1; j < KX; ++j) hi += __shfl_up_sync(0xffffffffu, q.v[j][d], 1) * T((double)j / KX);
        g[d] = lo + hi;
      }
    }
  };
  T gprev[KY][D];  // x-pass values of fine rows KY (R - 1) + j, j = 1 .. KY - 1
#pragma unroll
  for (int j = 0; j < KY; ++j) {
    if (j >= 1 && R0 >= 1) {
      FRow q;
      fload(KY * (R0 - 1) + j, q);
      xpass(q, gprev[j]);
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) gprev[j][d] = T(0);
    }
  }
  FRow q[KY];
#pragma unroll
  for (int j = 0; j < KY; ++j) fload(KY * R0 + j, q[j]);
  for (int R = R0; R < R1; ++R) {
    FRow nq[KY];
#pragma unroll
    for (int j = 0; j < KY; ++j) {
      if (R + 1 < R1) {
        fload(KY * (R + 1) + j, nq[j]);
      } else {
#pragma unroll
        for (int jj = 0; jj < KX; ++jj)
#pragma unroll
          for (int d = 0; d < D; ++d) nq[j].v[jj][d] = T(0);
      }
    }
    T gcur[KY][D];
#pragma unroll
    for (int j = 0; j < KY; ++j) xpass(q[j], gcur[j]);
    if (out_lane) {
      const uint8_t fl = __ldg(cfixed + (size_t)R * cnnx + C);
      T v[D];
#pragma unroll
      for (int d = 0; d < D; ++d) {
        if constexpr (KY == 1) {
          v[d] = gcur[0][d];
        } else {
          T lo = T(0), hi = T(0);
#pragma unroll
          for (int j = 0; j < KY; ++j) lo += gcur[j][d] * T(1.0 - (double)j / KY);
#pragma unroll
          for (int j = 1; j < KY; ++j) hi += gprev[j][d] * T((double)j / KY);
          v[d] = lo + hi;
        }
        if ((fl >> d) & 1) v[d] = T(0);
      }
      store_node<D, T>(o, (long long)R * cnnx + C, v);
    }
#pragma unroll
    for (int j = 0; j < KY; ++j) {
#pragma unroll
      for (int d = 0; d < D; ++d) gprev[j][d] = gcur[j][d];
      q[j] = nq[j];
    }
  }
}

// ---- prolongation -----------------------------------------------------------------
//
// x_f += P_f (P e_c), the x pass then the y pass of torch_mg._interp_axis
// (sttopt/torch_mg.py:75-81).  One thread per fine node on a 2-D grid (x = columns,
// y = fine rows), so the coarse values a warp reads are contiguous and L1-resident.
constexpr int kProlongThreads = 128;

template <int D, typename T>
__global__ void __launch_bounds__(kProlongThreads) prolong_kernel(
    const T* __restrict__ ec, long long c_rs, int cnnx, int cnny, T* __restrict__ xf, long long f_rs,
    int fnnx, int fnny, int kx, int ky, const uint8_t* __restrict__ ffixed,
    const RowState* __restrict__ rst) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const int r = blockIdx.y;
  const int c = blockIdx.x * kProlongThreads + threadIdx.x;
  if (c >= fnnx) return;
  const T* e = ec + (size_t)s * c_rs;
  T* x = xf + (size_t)s * f_rs;
  const long long node = (long long)r * fnnx + c;
  T v[D], pv[D];
  load_node<D, T>(x, node, v);
  prolong_at<D, T>(e, cnnx, kx, ky, r, c, pv);
  const uint8_t fl = ffixed ? __ldg(ffixed + node) : uint8_t(0);  // null: no projection
#pragma unroll
  for (int d = 0; d < D; ++d)
    if (!((fl >> d) & 1)) v[d] += pv[d];
  store_node<D, T>(x, node, v);
}

// Column-marching prolongation: a warp owns 32 fine columns and marches down a band of
// fine rows; every lane is an output column (no halo: a fine node needs only coarse
// values).  The coarse rows R and R + 1 around the current fine row are held in
// registers for the lane's coarse columns C and C + 1 and shifted when R advances, so a
// coarse value is loaded once per coarse row (with the next coarse row in flight) instead
// of up to four times per fine node.  Arithmetic as prolong_at.
inline dim3 prolong2_grid(int fnnx, int fnny, int rows) {
  const int xb = ((fnnx + 31) / 32 + kQWarps - 1) / kQWarps;
  return dim3(xb, (fnny + band_rows(xb, fnny, rows) - 1) / band_rows(xb, fnny, rows), rows);
}

template <int D, typename T>
__global__ void __launch_bounds__(kQThreads) prolong2_kernel(
    const T* __restrict__ ec, long long c_rs, int cnnx, int cnny, T* __restrict__ xf, long long f_rs, int fnnx,
    int fnny, int kx, int ky, const uint8_t* __restrict__ ffixed, const RowState* __restrict__ rst) {
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const T* e = ec + (size_t)s * c_rs;
  T* x = xf + (size_t)s * f_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = (blockIdx.x * kQWarps + warp) * 32 + lane;
  const bool col_ok = c < fnnx;
  const int C = col_ok ? div_k(c, kx) : 0, jx = c - C * kx;
  const T wx = T((double)jx / kx);
  const bool c1 = col_ok && jx != 0;  // needs coarse column C + 1
  const int band = (fnny + gridDim.y - 1) / gridDim.y;  // fine rows per block (any grid.y)
  const int r0 = blockIdx.y * band;
  const int r1 = min(r0 + band, fnny);
  // coarse row RR at columns C (v0) and C + 1 (v1); zero outside
  auto crow = [&](int RR, T(&v0)[D], T(&v1)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) v0[d] = v1[d] = T(0);
    if (!col_ok || RR < 0 || RR >= cnny) return;
    const long long n0 = (long long)RR * cnnx + C;
    load_node<D, T>(e, n0, v0);
    if (c1) load_node<D, T>(e, n0 + 1, v1);
  };
  int R = div_k(r0, ky);
  T a0[D], a1[D], b0[D], b1[D], n0[D], n1[D];  // rows R, R + 1, and R + 2 in flight
  crow(R, a0, a1);
  crow(R + 1, b0, b1);
  crow(R + 2, n0, n1);
  // fine rows r + 1 .. r + AHEAD of x and flags in flight (raw loads)
  constexpr int AHEAD = 4;
  T qx[AHEAD][D];
  uint8_t qf[AHEAD];
  auto frow = [&](int rr, T(&v)[D], uint8_t& fl) {
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = T(0);
    fl = 0;
    if (!col_ok || rr >= r1) return;
    const long long node = (long long)rr * fnnx + c;
    load_node<D, T>(x, node, v);
    fl = __ldg(ffixed + node);
  };
#pragma unroll
  for (int k = 0; k < AHEAD; ++k) frow(r0 + k, qx[k], qf[k]);
  for (int rb = r0; rb < r1; rb += AHEAD) {
#pragma unroll
   for (int k = 0; k < AHEAD; ++k) {
    const int r = rb + k;
    if (r >= r1) break;
    const int Rr = div_k(r, ky), jy = r - Rr * ky;
    if (Rr != R) {  // advance one coarse row (the band steps rows one at a time)
#pragma unroll
      for (int d = 0; d < D; ++d) {
        a0[d] = b0[d];
        a1[d] = b1[d];
        b0[d] = n0[d];
        b1[d] = n1[d];
      }
      R = Rr;
      crow(R + 2, n0, n1);
    }
    T v[D];
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = qx[k][d];
    const uint8_t fl = qf[k];
    frow(r + AHEAD, qx[k], qf[k]);
    if (!col_ok) continue;
    const long long node = (long long)r * fnnx + c;
    const T wy = T((double)jy / ky);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      T t0 = a0[d], t1 = b0[d];
      if (jx) {
        t0 = a0[d] * (T(1) - wx) + a1[d] * wx;
        t1 = b0[d] * (T(1) - wx) + b1[d] * wx;
      }
      const T pv = jy ? t0 * (T(1) - wy) + t1 * wy : t0;
      if (!((fl >> d) & 1)) v[d] += pv;
    }
    store_node<D, T>(x, node, v);
   }
  }
}

// Prolongation as prolong2_kernel with the coarsening factors as template parameters:
// a block's band of fine rows starts on a coarse row, so the rows are walked as coarse
// rows of KY fine rows each, with the y weights constants of the unrolled inner loop
// (no per-row division), and NQ fine rows of x and flags in flight.
template <int D, typename T, int KX, int KY>
__global__ void __launch_bounds__(kQThreads) prolong_t_kernel(
    const T* __restrict__ ec, long long c_rs, int cnnx, int cnny, T* __restrict__ xf, long long f_rs, int fnnx,
    int fnny, const uint8_t* __restrict__ ffixed, const RowState* __restrict__ rst) {
  constexpr int NQ = KY == 3 ? 6 : 4;  // fine rows in flight, a multiple of KY
  constexpr int CR = NQ / KY;          // coarse rows a step
  const int s = blockIdx.z;
  if (rst && !rst[s].active) return;
  const T* e = ec + (size_t)s * c_rs;
  T* x = xf + (size_t)s * f_rs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = (blockIdx.x * kQWarps + warp) * 32 + lane;
  const bool col_ok = c < fnnx;
  const int C = col_ok ? c / KX : 0, jx = c - C * KX;
  const T wx = jx == 0 ? T(0) : (jx == 1 ? T(1.0 / KX) : T(2.0 / KX));
  const bool c1 = col_ok && jx != 0;  // needs coarse column C + 1
  int band = (fnny + gridDim.y - 1) / gridDim.y;
  band = (band + KY - 1) / KY * KY;  // bands start on coarse rows
  const int r0 = blockIdx.y * band;
  if (r0 >= fnny) return;
  const int r1 = min(r0 + band, fnny);
  auto crow = [&](int RR, T(&v0)[D], T(&v1)[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) v0[d] = v1[d] = T(0);
    if (!col_ok || RR >= cnny) return;
    const long long n0 = (long long)RR * cnnx + C;
    load_node<D, T>(e, n0, v0);
    if (c1) load_node<D, T>(e, n0 + 1, v1);
  };
  auto frow = [&](int rr, T(&v)[D], uint8_t& fl) {
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = T(0);
    fl = 0;
    if (!col_ok || rr >= r1) return;
    const long long node = (long long)rr * fnnx + c;
    load_node<D, T>(x, node, v);
    fl = __ldg(ffixed + node);
  };
  int R = r0 / KY;
  T a0[D], a1[D], b0[D], b1[D], n0[D], n1[D];  // coarse rows R, R + 1, and R + 2 in flight
  crow(R, a0, a1);
  crow(R + 1, b0, b1);
  crow(R + 2, n0, n1);
  T qx[NQ][D];
  uint8_t qf[NQ];
#pragma unroll
  for (int k = 0; k < NQ; ++k) frow(r0 + k, qx[k], qf[k]);
  for (int rb = r0; rb < r1; rb += NQ) {
#pragma unroll
    for (int cr = 0; cr < CR; ++cr) {
#pragma unroll
      for (int jy = 0; jy < KY; ++jy) {
        const int k = cr * KY + jy;
        const int r = rb + k;
        T v[D];
#pragma unroll
        for (int d = 0; d < D; ++d) v[d] = qx[k][d];
        const uint8_t fl = qf[k];
        frow(r + NQ, qx[k], qf[k]);
        if (col_ok && r < r1) {
          const T wy = jy == 0 ? T(0) : (jy == 1 ? T(1.0 / KY) : T(2.0 / KY));
#pragma unroll
          for (int d = 0; d < D; ++d) {
            T t0 = a0[d], t1 = b0[d];
            if (jx) {
              t0 = a0[d] * (T(1) - wx) + a1[d] * wx;
              t1 = b0[d] * (T(1) - wx) + b1[d] * wx;
            }
            const T pv = jy ? t0 * (T(1) - wy) + t1 * wy : t0;
            if (!((fl >> d) & 1)) v[d] += pv;
          }
          store_node<D, T>(x, (long long)r * fnnx + c, v);
        }
      }
      // advance one coarse row
#pragma unroll
      for (int d = 0; d < D; ++d) {
        a0[d] = b0[d];
        a1[d] = b1[d];
        b0[d] = n0[d];
        b1[d] = n1[d];
      }
      ++R;
      crow(R + 2, n0, n1);
    }
  }
}

// ---- coarsest level: block-banded Cholesky solve (one CTA per batch row) ----------
//
// Forward  y_k = Dinv_k (b_k - E_k y_{k-1}),  backward x_k = Dinv_k^T (y_k - E_{k+1}^T x_{k+1}):
// 2 nb sequential steps of two B x B GEMVs.  The steps are latency-bound, so each GEMV
// row is split over 4 threads (a quad: NC = B / 4 columns each, 128-bit loads, two
// shuffles), and the matrices of step j+1 are loaded into registers while step j
// computes.  blockDim = 4 B.

template <int NC>
STT_DEV void load_quad_row(const double* __restrict__ M, int B, int i, int q, double (&reg)[NC]) {
  const double2* src = reinterpret_cast<const double2*>(M + (size_t)i * B + q * NC);
#pragma unroll
  for (int c = 0; c < NC / 2; ++c) {
    const double2 t = __ldg(src + c);
    reg[2 * c] = t.x;
    reg[2 * c + 1] = t.y;
  }
}

template <int NC>
STT_DEV double quad_dot(const double (&reg)[NC], const double* __restrict__ v, int q) {
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < NC; ++c) acc = fma(reg[c], v[q * NC + c], acc);
  acc += __shfl_xor_sync(0xffffffffu, acc, 1);
  acc += __shfl_xor_sync(0xffffffffu, acc, 2);
  return acc;
}

template <int D, typename T, int NC>
__global__ void __launch_bounds__(4 * 4 * NC) coarse_solve_kernel(
    const T* __restrict__ b, T* __restrict__ x, long long rs, const double* __restrict__ blocks,
    int nb, int by_col, int nnx, int nny, const uint8_t* __restrict__ fixed,
    double* __restrict__ scratch, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst) {
  constexpr int B = 4 * NC;
  __shared__ double vp[B];  // previous step's block solution
  __shared__ double tv[B];  // current step's right-hand side
  const int s = blockIdx.x;
  if (rst && !rst[s].active) return;
  const int h = hier_row(row_map, hrows, s);
  const double* bh = blocks + (size_t)h * nb * 4 * B * B;
  const long long nnode = (long long)nnx * nny, n = nnode * D, np = (long long)nb * B;
  double* y = scratch + (size_t)s * np;
  const int tid = threadIdx.x, i = tid >> 2, q = tid & 3;
  auto node_of = [&](long long P, int& r, int& c, int& d) {
    const long long nd = P / D;
    d = (int)(P - nd * D);
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
      int r, c, d;
      node_of(P, r, c, d);
      v = (double)bs[((size_t)r * nnx + c) * D + d];
    }
    y[P] = v;
  }
  // step j < nb: forward block k = j, matrices (E_k | none, Dinv_k);
  // step j >= nb: backward block k = 2 nb - 1 - j, matrices (E_{k+1}^T | none, Dinv_k^T)
  auto mats = [&](int j, const double*& A, const double*& M) {
    if (j < nb) {
      const double* blk = bh + (size_t)j * 4 * B * B;
      A = j > 0 ? blk + 2 * (size_t)B * B : nullptr;
      M = blk;
    } else {
      const int k = 2 * nb - 1 - j;
      A = k < nb - 1 ? bh + (size_t)(k + 1) * 4 * B * B + 3 * (size_t)B * B : nullptr;
      M = bh + (size_t)k * 4 * B * B + (size_t)B * B;
    }
  };
  double ra[NC], rm[NC], na[NC], nm[NC];
  const double *A, *M;
  mats(0, A, M);
  if (A) load_quad_row<NC>(A, B, i, q, ra);
  load_quad_row<NC>(M, B, i, q, rm);
  __syncthreads();
  for (int j = 0; j < 2 * nb; ++j) {
    const int k = j < nb ? j : 2 * nb - 1 - j;
    const bool hasA = A != nullptr;
    // prefetch the next step's matrices
    const double *A2 = nullptr, *M2 = nullptr;
    if (j + 1 < 2 * nb) {
      mats(j + 1, A2, M2);
      if (A2) load_quad_row<NC>(A2, B, i, q, na);
      load_quad_row<NC>(M2, B, i, q, nm);
    }
    double rhs = y[(size_t)k * B + i];
    if (hasA) rhs -= quad_dot<NC>(ra, vp, q);
    if (q == 0) tv[i] = rhs;
    __syncthreads();
    const double v = quad_dot<NC>(rm, tv, q);
    __syncthreads();  // every quad has read vp and tv
    if (q == 0) {
      vp[i] = v;
      y[(size_t)k * B + i] = v;
    }
    __syncthreads();
    A = A2;
    M = M2;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      ra[c] = na[c];
      rm[c] = nm[c];
    }
  }
  T* xs = x + (size_t)s * rs;
  for (long long P = tid; P < n; P += blockDim.x) {
    int r, c, d;
    node_of(P, r, c, d);
    const long long node = (long long)r * nnx + c;
    xs[node * D + d] = ((fixed[node] >> d) & 1) ? T(0) : T(y[P]);
  }
}

// The coarsest level by its explicit inverse (FP32 cycles): x = A^{-1} b as one GEMV in
// the band ordering.  Grid (np / 32, rows): each CTA stages b (permuted, FP64) in shared
// memory and its 8 warps produce 4 output rows each, lanes striding a row of the
// inverse (coalesced) and a warp reduction; fixed dofs come back zero.
constexpr int kInvRowsPerCta = 32;

template <int D, typename T>
__global__ void __launch_bounds__(256) coarse_inv_solve_kernel(
    const T* __restrict__ b, T* __restrict__ x, long long rs, const double* __restrict__ inv, int np, int by_col,
    int nnx, int nny, const uint8_t* __restrict__ fixed, const int* __restrict__ row_map, int hrows,
    const RowState* __restrict__ rst) {
  extern __shared__ double yv[];  // [np]
  const int s = blockIdx.y;
  if (rst && !rst[s].active) return;
  const int h = hier_row(row_map, hrows, s);
  const long long nnode = (long long)nnx * nny, n = nnode * D;
  auto node_of = [&](long long P, int& r, int& c, int& d) {
    const long long nd = P / D;
    d = (int)(P - nd * D);
    if (by_col) {
      c = (int)(nd / nny);
      r = (int)(nd - (long long)c * nny);
    } else {
      r = (int)(nd / nnx);
      c = (int)(nd - (long long)r * nnx);
    }
  };
  const T* bs = b + (size_t)s * rs;
  for (int P = threadIdx.x; P < np; P += blockDim.x) {
    double v = 0.0;
    if (P < n) {
      int r, c, d;
      node_of(P, r, c, d);
      v = (double)bs[((size_t)r * nnx + c) * D + d];
    }
    yv[P] = v;
  }
  __syncthreads();
  const double* ih = inv + (size_t)h * np * np;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* xs = x + (size_t)s * rs;
  for (int q = 0; q < kInvRowsPerCta / 8; ++q) {
    const int P = blockIdx.x * kInvRowsPerCta + warp * (kInvRowsPerCta / 8) + q;
    if (P >= n) break;
    const double* row = ih + (size_t)P * np;
    double acc = 0.0;
    for (int Q = lane; Q < np; Q += 32) acc = fma(__ldg(row + Q), yv[Q], acc);
    acc = warp_sum(acc);
    if (lane == 0) {
      int r, c, d;
      node_of(P, r, c, d);
      const long long node = (long long)r * nnx + c;
      xs[node * D + d] = ((fixed[node] >> d) & 1) ? T(0) : T(acc);
    }
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
