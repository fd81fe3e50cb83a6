// V-cycle driver and the device-resident multigrid-preconditioned CG.
//
// The PCG recurrence is the reference's (torch_fem.pcg, sttopt/torch_fem.py:201-343):
// per-row alpha/beta with safe_div, convergence on ||r|| / ||b|| checked before the
// first iteration and after every update.  Converged rows stop (every kernel skips
// rows whose device `active` flag is clear), which is the reference's row retirement
// without the compaction copies; the host reads the row flags every few iterations
// instead of syncing on every one.  Reductions are deterministic (block partials
// summed in block order by the last block).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "errors.h"
#include "hier.h"
#include "mg.cuh"

namespace stt {

constexpr int kEwThreads = 256;

// Calls M(KX, KY) for the coarsening factors (kx, ky), each 1, 2 or 3; else runs FALLBACK.
#define STT_KXKY_DISPATCH(kx, ky, M, FALLBACK)   \
  do {                                          \
    if ((kx) == 2 && (ky) == 2) M(2, 2);         \
    else if ((kx) == 2 && (ky) == 3) M(2, 3);    \
    else if ((kx) == 3 && (ky) == 2) M(3, 2);    \
    else if ((kx) == 3 && (ky) == 3) M(3, 3);    \
    else if ((kx) == 1 && (ky) == 2) M(1, 2);    \
    else if ((kx) == 2 && (ky) == 1) M(2, 1);    \
    else if ((kx) == 1 && (ky) == 3) M(1, 3);    \
    else if ((kx) == 3 && (ky) == 1) M(3, 1);    \
    else FALLBACK;                               \
  } while (0)

static int grid1(long long n, int bs = 256) {
  long long g = (n + bs - 1) / bs;
  if (g > (1 << 30)) g = 1 << 30;
  return (int)(g < 1 ? 1 : g);
}

static int ew_blocks(long long n) {
  long long g = (n + kEwThreads * 4 - 1) / (kEwThreads * 4);
  return (int)std::min<long long>(std::max<long long>(g, 1), 2048);
}

static dim3 tile_grid(int nelx, int nely, int rows) { return q4_grid(nelx, nely, rows); }

// The PCG's level-0 passes (initial residual, p.Ap): bands of 32 grid rows, or shorter
// ones (down to 8) while the rows give fewer blocks than two waves of six 128-thread
// blocks on each of the 148 SMs (a single scalar row: the heat solves).  The kernels
// take the band from the launch (BAND = 0).
static dim3 pcg_tile_grid(int nelx, int nely, int rows, int min_band = 0) {
  const dim3 g = q4_grid(nelx, nely, rows);
  const int nny = nely + 1;
  int band = kQRows;
  if (min_band > 0) {
    band = min_band;  // the most blocks any tuning can ask for (sizes the reduction partials)
  } else if (launch_tuning().pcg_band > 0) {
    band = launch_tuning().pcg_band;
  } else {
    while (band > 8 && (long long)g.x * ((nny + band - 1) / band) * rows < 2LL * 148 * 6) band /= 2;
  }
  return dim3(g.x, (nny + band - 1) / band, rows);
}

// prolong_kernel: one thread per fine node, x = fine columns, y = fine rows.
static dim3 prolong_grid(int fnnx, int fnny, int rows) {
  return dim3((fnnx + kProlongThreads - 1) / kProlongThreads, fnny, rows);
}

// ---- workspace plan ---------------------------------------------------------------

// Row stride of the cycle's own per-level vectors: ndof rounded up to 4 words, so every
// batch row starts 16-byte aligned (the tile kernels' 128-bit staging needs it).
static long long vstride(long long ndof) { return (ndof + 3) & ~3LL; }

struct SolveWS {
  RowState* rs;
  double* partials;
  unsigned* counters;
  int* sched_last;             // rows left by the last retirement (reference schedule)
  double *r, *p, *p2, *Ap;     // FP64 [nrows][ndof0]; p and p2 alternate
  void *z, *zold, *b0;         // cycle precision [nrows][ndof0]
  void* x[kMaxLevels];         // per level [nrows][ndof_l]
  void* t[kMaxLevels];
  void* b[kMaxLevels];
  void* acc[kMaxLevels];       // gamma > 1 only
  void* rhs2[kMaxLevels];
  double* cscratch;            // [nrows][nb * B]
  int nblk_max;
  long long bytes;
};

static char* carve(char* base, long long& used, long long bytes) {
  const long long a = (bytes + 255) & ~255LL;
  char* r = base ? base + used : nullptr;
  used += a;
  return r;
}

// The solve's buffers; with pcg == false only those a lone V-cycle uses (z, the FP32
// copy of r, the per-level vectors and the coarse scratch), not the PCG's row states,
// reduction partials and r / p / Ap / z_old.
static long long plan_solve(const stt_hier* h, int nrows, int gamma, char* base, SolveWS& w, bool pcg = true) {
  std::memset(&w, 0, sizeof(w));
  long long used = 0;
  const int es = h->precision == STT_FP32 ? 4 : 8;
  const LevelDesc& l0 = h->lv[0];
  if (pcg) {
    const dim3 tg = pcg_tile_grid(h->nelx, h->nely, nrows, 8);
    // the level-0 chained passes' blocks may take the r.z reductions
    const dim3 pg = postsmooth_grid(h->nelx, h->nely, nrows), qg = presmooth_grid(h->nelx, h->nely, nrows);
    w.nblk_max = std::max<int>(std::max<int>(tg.x * tg.y, std::max(pg.x * pg.y, qg.x * qg.y)), ew_blocks(l0.ndof));
    w.rs = (RowState*)carve(base, used, sizeof(RowState) * nrows);
    w.partials = (double*)carve(base, used, 8LL * nrows * w.nblk_max * 3);
    w.counters = (unsigned*)carve(base, used, 4LL * nrows);
    w.sched_last = (int*)carve(base, used, 4);
    w.r = (double*)carve(base, used, 8LL * nrows * l0.ndof);
    w.p = (double*)carve(base, used, 8LL * nrows * l0.ndof);
    w.p2 = (double*)carve(base, used, 8LL * nrows * l0.ndof);
    w.Ap = (double*)carve(base, used, 8LL * nrows * l0.ndof);
  }
  w.z = carve(base, used, (long long)es * nrows * vstride(l0.ndof));
  if (pcg) w.zold = carve(base, used, (long long)es * nrows * vstride(l0.ndof));
  if (h->precision == STT_FP32) w.b0 = carve(base, used, 4LL * nrows * vstride(l0.ndof));
  for (int l = 0; l < h->nlevels; ++l) {
    const long long nd = vstride(h->lv[l].ndof);
    w.x[l] = carve(base, used, (long long)es * nrows * nd);
    w.t[l] = carve(base, used, (long long)es * nrows * nd);
    if (l > 0) w.b[l] = carve(base, used, (long long)es * nrows * nd);
    if (gamma > 1 && l > 0) {
      w.acc[l] = carve(base, used, (long long)es * nrows * nd);
      w.rhs2[l] = carve(base, used, (long long)es * nrows * nd);
    }
  }
  w.cscratch = (double*)carve(base, used, 8LL * nrows * h->co.nb * h->co.B);
  w.bytes = used;
  return used;
}

// ---- V-cycle ---------------------------------------------------------------------

template <int D, typename T>
struct Cycle {
  const stt_hier* h;
  SolveWS& w;
  int nrows;
  T omega;
  int n_smooth, gamma;
  const RowState* rst;
  cudaStream_t st;
  KEq<D, T> ke;
  MQ<T> mq;
  T* final_out = nullptr;  // where level 0's last sweep writes (row stride vstride(ndof0))
  bool waited_factor = false;  // the stream has waited for the coarse factorisation
  bool waited_ready = false;   // ... and for the explicit inverse
  RzFuse<T> rzf{};         // the PCG's dots for level 0's chained passes to take (rzf.rst set)
  bool mix_done = false;   // the pre-smoothing pass took r . z_old
  bool rz_done = false;    // the post-smoothing pass took r . z and set beta

  T* X(int l) const { return (T*)w.x[l]; }
  T* Tt(int l) const { return (T*)w.t[l]; }

  const T* rho0() const {
    if constexpr (sizeof(T) == 4) return (const T*)h->lv[0].rho32;
    else return (const T*)h->lv[0].rho64;
  }
  const T* rdiag0() const {
    if (!h->has_reaction) return nullptr;
    if constexpr (sizeof(T) == 4) return (const T*)h->lv[0].rdiag32;
    else return (const T*)h->lv[0].rdiag64;
  }
  const T* stl(int l) const {
    if constexpr (sizeof(T) == 4) return (const T*)h->lv[l].st32;
    else return (const T*)h->lv[l].st64;
  }

  // Level 1's sweep or residual from the level-0 densities (l1_sweep_kernel) when the
  // hierarchy allows it; false when the stencil kernel must run.
  template <int MODE>
  bool l1_pass(int l, const T* x, const T* b, T* out) {
    if constexpr (D != 2 || !(MODE == SW_SWEEP || MODE == SW_RESID)) {
      return false;
    } else {
      if (l != 1 || !h->l1) return false;
      const LevelDesc& f = h->lv[0];
      const LevelDesc& lv = h->lv[1];
      const dim3 g = coarse_grid(lv.nelx, lv.nely, nrows);
      const T* r0 = rho0();
#define STT_L1(KX, KY)                                                                               \
  do {                                                                                               \
    L1Mat<T, KX * KY> M;                                                                             \
    for (int m = 0; m < KX * KY; ++m)                                                                \
      for (int e = 0; e < 21; ++e) M.m[m][e] = T(h->l1m[m][e]);                                      \
    l1_sweep_kernel<T, MODE, KX, KY><<<g, kQThreads, 0, st>>>(x, b, out, vstride(lv.ndof), r0, f.rs_rho, \
                                                              f.nelx, stl(1), lv.fixed, lv.nnx, lv.nny,  \
                                                              h->row_map, h->hrows, rst, omega, M);      \
  } while (0)
      if (f.kx == 2 && f.ky == 2 && h->l1par) {
        L1Mat<T, 1> M;  // M_0 only
        for (int e = 0; e < 21; ++e) M.m[0][e] = T(h->l1m[0][e]);
        l1_sweep_kernel<T, MODE, 2, 2, 2, true><<<g, kQThreads, 0, st>>>(
            x, b, out, vstride(lv.ndof), r0, f.rs_rho, f.nelx, stl(1), lv.fixed, lv.nnx, lv.nny, h->row_map, h->hrows,
            rst, omega, M);
      } else if (f.kx == 2 && f.ky == 2) STT_L1(2, 2);
      else if (f.kx == 2 && f.ky == 3) STT_L1(2, 3);
      else if (f.kx == 3 && f.ky == 2) STT_L1(3, 2);
      else if (f.kx == 3 && f.ky == 3) STT_L1(3, 3);
      else return false;
#undef STT_L1
      return true;
    }
  }

  // Restriction of the fine residual rf into the coarse right-hand side, and the
  // prolongation of the coarse correction ec added into xf, with the level's coarsening
  // factors as template parameters (every combination of 1, 2 and 3).
  void transfer_down(const LevelDesc& lv, const LevelDesc& cl, const T* rf, long long nd, T* rc, long long cnd) {
    const dim3 g = coarse_grid(cl.nelx, cl.nely, nrows);
#define STT_RESTRICT(KX, KY)                                                                       \
  restrict_t_kernel<D, T, KX, KY><<<g, kQThreads, 0, st>>>(rf, nd, lv.nnx, lv.nny, rc, cnd, cl.nnx, \
                                                           cl.nny, cl.fixed, rst)
    STT_KXKY_DISPATCH(lv.kx, lv.ky, STT_RESTRICT,
                      (restrict_kernel<D, T><<<g, kQThreads, 0, st>>>(rf, nd, lv.nnx, lv.nny, rc, cnd, cl.nnx,
                                                                      cl.nny, lv.kx, lv.ky, cl.fixed, rst)));
#undef STT_RESTRICT
  }
  void transfer_up(const LevelDesc& lv, const LevelDesc& cl, const T* ec, long long cnd, T* xf, long long nd) {
    const dim3 g = prolong2_grid(lv.nnx, lv.nny, nrows);
#define STT_PROLONG(KX, KY)                                                                         \
  prolong_t_kernel<D, T, KX, KY><<<g, kQThreads, 0, st>>>(ec, cnd, cl.nnx, cl.nny, xf, nd, lv.nnx, lv.nny, \
                                                          lv.fixed, rst)
    STT_KXKY_DISPATCH(lv.kx, lv.ky, STT_PROLONG,
                      (prolong2_kernel<D, T><<<g, kQThreads, 0, st>>>(ec, cnd, cl.nnx, cl.nny, xf, nd, lv.nnx,
                                                                      lv.nny, lv.kx, lv.ky, lv.fixed, rst)));
#undef STT_PROLONG
  }

  // One smoother / residual / apply pass at level l: out = op(x, b); SW_POST reads
  // x + P(pro.ec) (the coarse correction) in place of x.
  template <int MODE>
  void pass(int l, const T* x, long long x_rs, const T* b, long long b_rs, T* out, long long o_rs,
            ProlongSrc<T> pro = ProlongSrc<T>{nullptr, 0, 1, 1, 1}) {
    const LevelDesc& lv = h->lv[l];
    if (l == 0) {
      const dim3 g = march_grid<true, T>(lv.nelx, lv.nely, nrows);
      if (h->modal && h->has_reaction)
        l0_sweep_modal_kernel<D, T, MODE, true><<<g, kQThreads, 0, st>>>(
            x, x_rs, b, b_rs, out, o_rs, rho0(), lv.rs_rho, rdiag0(), lv.ndof, lv.fixed, h->row_map,
            h->hrows, rst, lv.nelx, lv.nely, omega, mq, pro);
      else if (h->modal)
        l0_sweep_modal_kernel<D, T, MODE, false><<<g, kQThreads, 0, st>>>(
            x, x_rs, b, b_rs, out, o_rs, rho0(), lv.rs_rho, rdiag0(), lv.ndof, lv.fixed, h->row_map,
            h->hrows, rst, lv.nelx, lv.nely, omega, mq, pro);
      else
        l0_sweep_kernel<D, T, MODE><<<g, kQThreads, 0, st>>>(
            x, x_rs, b, b_rs, out, o_rs, rho0(), lv.rs_rho, rdiag0(), lv.ndof, lv.fixed, h->row_map,
            h->hrows, rst, lv.nelx, lv.nely, omega, ke, 0, pro);
    } else if (l1_pass<MODE>(l, x, b, out)) {
      // level 1 applied from the level-0 densities
    } else {
      if constexpr (MODE == SW_POST)
        st_sweep_kernel<D, T, MODE><<<tile_grid(lv.nelx, lv.nely, nrows), kQThreads, 0, st>>>(
            x, b, out, vstride(lv.ndof), stl(l), lv.fixed, lv.nnx, lv.nny, h->row_map, h->hrows, rst, omega,
            pro);
      else
        st_sweep2_kernel<D, T, MODE><<<coarse_grid(lv.nelx, lv.nely, nrows), kQThreads, 0, st>>>(
            x, b, out, vstride(lv.ndof), stl(l), lv.fixed, lv.nnx, lv.nny, h->row_map, h->hrows, rst, omega,
            (sizeof(T) == 4 && l == 1 && h->l1) ? 1 : 0);
    }
  }

  // The factorisation (and an FP32 hierarchy's explicit inverse after it) runs on the
  // hierarchy's side stream.  The first coarse solve on a fresh FP32 hierarchy takes the
  // block solves, which need only the factor, so the first cycle does not wait for the
  // inverse; every later one takes the inverse's GEMV (equal to FP64 rounding).
  void coarse(int l, const T* b, T* x) {
    const LevelDesc& lv = h->lv[l];
    const CoarseDesc& co = h->co;
    bool use_inv = sizeof(T) == 4 && co.inv;
    if (use_inv && h->sync->first_cycle.load() && h->sync->first_cycle.exchange(0) == 1) use_inv = false;
    if (use_inv && !waited_ready) {
      cudaStreamWaitEvent(st, h->sync->ready, 0);
      waited_ready = waited_factor = true;
    } else if (!use_inv && !waited_factor) {
      cudaStreamWaitEvent(st, h->sync->factored, 0);
      waited_factor = true;
    }
    if (use_inv) {
      const int np = co.nb * co.B;
      coarse_inv_solve_kernel<D, T><<<dim3((np + kInvRowsPerCta - 1) / kInvRowsPerCta, nrows), 256,
                                      sizeof(double) * np, st>>>(b, x, vstride(lv.ndof), co.inv, np, co.by_col,
                                                                 lv.nnx, lv.nny, lv.fixed, h->row_map, h->hrows,
                                                                 rst);
      return;
    }
#define STT_COARSE(NC)                                                                          \
  coarse_solve_kernel<D, T, NC><<<nrows, 16 * NC, 0, st>>>(b, x, vstride(lv.ndof), co.blocks, co.nb, co.by_col, \
                                                          lv.nnx, lv.nny, lv.fixed, w.cscratch,       \
                                                          h->row_map, h->hrows, rst)
    switch (co.B) {
      case 32: STT_COARSE(8); break;
      case 64: STT_COARSE(16); break;
      case 96: STT_COARSE(24); break;
      case 128: STT_COARSE(32); break;
      default: set_error(STT_ERR_INVALID, "coarse band block size above 128 is not supported");
    }
#undef STT_COARSE
  }

  // Level 0's pre-smoothing (n_smooth = 2) and residual in one pass (modal operator):
  // x2 into out_x, the residual into out_r.
  void presmooth(const T* b, long long b_rs, T* out_x, T* out_r) {
    const LevelDesc& lv = h->lv[0];
    const long long nd = vstride(lv.ndof);
    const dim3 g = presmooth_grid(lv.nelx, lv.nely, nrows);
    RzFuse<T> mx = rzf;
    mx.red.nblk = (int)(g.x * g.y);
#define STT_PRE(RD, MX)                                                                                  \
  l0_presmooth_kernel<D, T, RD, MX><<<g, kQThreads, 0, st>>>(b, b_rs, out_x, nd, out_r, nd, rho0(), lv.rs_rho, \
                                                           rdiag0(), lv.ndof, lv.fixed, h->row_map, h->hrows,  \
                                                           rst, lv.nelx, lv.nely, omega, mq, mx)
    if (rzf.rst && rzf.zold) {
      if (h->has_reaction) STT_PRE(true, true);
      else STT_PRE(false, true);
      mix_done = true;
    } else {
      if (h->has_reaction) STT_PRE(true, false);
      else STT_PRE(false, false);
    }
#undef STT_PRE
  }

  // Level 1's smoothing chained in one pass from the level-0 densities (FP32, 2 x 2
  // mirror-form children, two sweeps each way): PRE writes x2 to ox and the residual to
  // orr; POST sweeps twice from x0 into ox.  False when the hierarchy does not allow it
  // (the FP64 cycle keeps the unchained passes: the chained state does not fit its
  // registers).
  bool l1_chain(bool pre, const T* x0, const T* b, T* ox, T* orr) {
    if constexpr (D != 2 || sizeof(T) != 4) {
      return false;
    } else {
      const LevelDesc& f = h->lv[0];
      const LevelDesc& lv = h->lv[1];
      if (!h->l1 || !h->l1par || n_smooth != 2 || f.kx != 2 || f.ky != 2) return false;
      const dim3 g = l1_chain_grid(lv.nelx, lv.nely, nrows);
      const long long vs = vstride(lv.ndof);
#define STT_L1C(PRE, MIR, NM)                                                                                 \
  do {                                                                                                        \
    L1Mat<T, NM> M;                                                                                           \
    for (int m = 0; m < NM; ++m)                                                                              \
      for (int e = 0; e < 21; ++e) M.m[m][e] = T(h->l1m[m][e]);                                               \
    l1_chain_kernel<T, PRE, MIR><<<g, kQThreads, 0, st>>>(x0, b, ox, orr, vs, rho0(), f.rs_rho, f.nelx, stl(1), \
                                                          lv.fixed, lv.nnx, lv.nny, h->row_map, h->hrows, rst,  \
                                                          omega, M);                                            \
  } while (0)
      if (pre) STT_L1C(true, true, 1);
      else STT_L1C(false, true, 1);
#undef STT_L1C
      return true;
    }
  }

  // A stored-stencil level's smoothing chained in one pass each way (FP32, two sweeps each
  // way): PRE writes x2 to ox and the residual to orr; POST sweeps twice from x0 into ox.
  // False where it does not apply (FP64 cycles, other sweep counts, and level 1 when it
  // is swept from the densities: its FP32 stencil then holds only the diagonal).
  bool st_chain(int l, bool pre, const T* x0, const T* b, T* ox, T* orr) {
    if constexpr (sizeof(T) != 4) {
      return false;
    } else {
      if (l < 1 || n_smooth != 2 || (l == 1 && h->l1)) return false;
      const LevelDesc& lv = h->lv[l];
      const dim3 g = st_chain_grid(lv.nelx, lv.nely, nrows);
      const long long vs = vstride(lv.ndof);
      if (pre)
        st_chain_kernel<D, T, true><<<g, kQThreads, 0, st>>>(x0, b, ox, orr, vs, stl(l), lv.fixed, lv.nnx, lv.nny,
                                                             h->row_map, h->hrows, rst, omega);
      else
        st_chain_kernel<D, T, false><<<g, kQThreads, 0, st>>>(x0, b, ox, orr, vs, stl(l), lv.fixed, lv.nnx,
                                                              lv.nny, h->row_map, h->hrows, rst, omega);
      return true;
    }
  }

  // Level 0's two post-smoothing sweeps in one pass: x0 (the prolonged iterate) -> out.
  // With rzf set, the pass also takes the PCG's r.z (and r.z_old) from b and what it writes.
  void postsmooth(const T* x0, const T* b, long long b_rs, T* out) {
    const LevelDesc& lv = h->lv[0];
    const long long nd = vstride(lv.ndof);
    const dim3 g = postsmooth_grid(lv.nelx, lv.nely, nrows);
    RzFuse<T> rz = rzf;
    rz.red.nblk = (int)(g.x * g.y);
    const bool fuse = rzf.rst && (!rzf.zold || mix_done);
#define STT_POST(RD, RZ)                                                                                  \
  l0_postsmooth_kernel<D, T, RD, RZ><<<g, kQThreads, 0, st>>>(x0, nd, b, b_rs, out, nd, rho0(), lv.rs_rho,     \
                                                            rdiag0(), lv.ndof, lv.fixed, h->row_map, h->hrows, \
                                                            rst, lv.nelx, lv.nely, omega, mq, rz)
    if (fuse) {
      if (h->has_reaction) STT_POST(true, true);
      else STT_POST(false, true);
      rz_done = true;
    } else {
      if (h->has_reaction) STT_POST(true, false);
      else STT_POST(false, false);
    }
#undef STT_POST
  }

  // The correction from level l + 1 for its right-hand side bc (gamma visits).
  T* coarse_correction(int l, T* bc) {
    const LevelDesc& cl = h->lv[l + 1];
    const long long cnd = vstride(cl.ndof);
    T* ec = cycle(l + 1, bc, cnd);
    if (gamma > 1) {
      T* acc = (T*)w.acc[l + 1];
      T* rhs = (T*)w.rhs2[l + 1];
      rows_convert_kernel<T, T><<<dim3(ew_blocks(cl.ndof), nrows), kEwThreads, 0, st>>>(ec, cnd, acc, cnd, cl.ndof, rst);
      for (int g = 1; g < gamma; ++g) {
        // rhs = b_c - A_c acc
        pass<SW_RESID>(l + 1, acc, cnd, bc, cnd, rhs, cnd);
        T* e2 = cycle(l + 1, rhs, cnd);
        rows_axpy_kernel<T><<<dim3(ew_blocks(cl.ndof), nrows), kEwThreads, 0, st>>>(e2, acc, cnd, cl.ndof, rst);
      }
      ec = acc;
    }
    return ec;
  }

  // Solves level l approximately for right-hand side b (row stride b_rs); returns the
  // buffer holding the result (row stride ndof_l).
  T* cycle(int l, const T* b, long long b_rs) {
    const LevelDesc& lv = h->lv[l];
    const long long nd = vstride(lv.ndof);
    if (l == h->nlevels - 1) {
      // the coarse solve reads b with the level's own row stride
      const T* bb = b;
      if (b_rs != nd) {
        rows_convert_kernel<T, T><<<dim3(ew_blocks(lv.ndof), nrows), kEwThreads, 0, st>>>(b, b_rs, Tt(l), nd, lv.ndof, rst);
        bb = Tt(l);
      }
      coarse(l, bb, X(l));
      return X(l);
    }
    T* xa = X(l);
    T* xb = Tt(l);
    // level 0 with the modal operator: pre-smoothing + residual in one pass.  (Folding
    // the prolongation into the first post-smoothing sweep, SW_POST, measured slower on
    // B200 than the separate prolongation: 600 us against 277 + 151 us at 2048x1024 x 16.)
    const bool modal0 = l == 0 && h->modal;
    bool chained1 = false;  // level 1's smoothing chained in one pass each way
    bool chainedS = false;  // a stencil level's, likewise
    if (modal0 && n_smooth == 2) {
      presmooth(b, b_rs, xa, xb);
    } else if (l == 1 && b_rs == nd && l1_chain(true, nullptr, b, xa, xb)) {
      chained1 = true;
    } else if (b_rs == nd && st_chain(l, true, nullptr, b, xa, xb)) {
      chainedS = true;
    } else {
      pass<SW_FIRST>(l, nullptr, nd, b, b_rs, xa, nd);
      for (int k = 1; k < n_smooth; ++k) {
        pass<SW_SWEEP>(l, xa, nd, b, b_rs, xb, nd);
        std::swap(xa, xb);
      }
      // residual into xb
      pass<SW_RESID>(l, xa, nd, b, b_rs, xb, nd);
    }
    // restricted into b_{l+1}
    const LevelDesc& cl = h->lv[l + 1];
    const long long cnd = vstride(cl.ndof);
    T* bc = (T*)w.b[l + 1];
    transfer_down(lv, cl, xb, nd, bc, cnd);
    T* ec = coarse_correction(l, bc);
    transfer_up(lv, cl, ec, cnd, xa, nd);
    // post-smoothing; level 0's last sweep writes straight into final_out when given
    if (modal0 && n_smooth == 2) {
      // the fused pass reads b a few rows ahead of its writes, so it never writes over b
      // (an in-place V-cycle, z = r, goes through xb and the final copy)
      T* dst = (final_out && final_out != b) ? final_out : xb;
      postsmooth(xa, b, b_rs, dst);
      return dst;
    }
    if (chained1) {
      l1_chain(false, xa, b, xb, nullptr);
      return xb;
    }
    if (chainedS) {
      st_chain(l, false, xa, b, xb, nullptr);
      return xb;
    }
    for (int k = 0; k < n_smooth; ++k) {
      T* dst = (l == 0 && final_out && k == n_smooth - 1) ? final_out : xb;
      pass<SW_SWEEP>(l, xa, nd, b, b_rs, dst, nd);
      if (dst == xb) std::swap(xa, xb); else xa = dst;
    }
    return xa;
  }
};

// ---- PCG kernels (FP64 outer iteration) -----------------------------------------

struct PcgParams {
  double rtol;
  int it;
  int flexible;
  int sched;  // 1: a converged row iterates on until the reference's compaction retires it
};

// A row's convergence test after a residual: with the reference's schedule (sched) it
// only records the test, and pcg_retire_kernel decides when the row stops; otherwise the
// row stops at once.
STT_DEV void pcg_converged(RowState& S, const PcgParams& pp) {
  const bool c = S.rel <= pp.rtol;
  if (pp.sched) {
    S.conv = c ? 1 : 0;
  } else if (c) {
    S.active = 0;
    S.conv_iter = pp.it;
  }
}

// A row's state after the initial residual: t[0] = ||r||^2, t[1] = ||b||^2 (kept across a
// true-residual replacement, replace = 1).
STT_DEV void pcg_init_finish(RowState& S, const double* t, const PcgParams& pp, int replace) {
  if (!replace) {
    const double bn = sqrt(t[1]);
    S.bnorm_safe = bn > 0.0 ? bn : 1.0;
    S.conv_iter = -1;
    S.status = STT_OK;
    S.active = 1;
    S.conv = 0;
  }
  S.rel = sqrt(t[0]) / S.bnorm_safe;
  if (!isfinite(S.rel)) S.status = STT_ERR_BREAKDOWN;
  pcg_converged(S, pp);
}

// r = b - A x (or r = b when x is null), reductions ||r||^2 and ||b||^2.
// replace: keep bnorm and only re-test convergence (true-residual replacement).
template <int D, bool MODAL, bool RD>
__global__ void __launch_bounds__(kQThreads) pcg_init_kernel(
    const double* __restrict__ b, long long b_rs, const double* __restrict__ x, long long x_rs,
    double* __restrict__ r, long long r_rs, const double* __restrict__ rho, long long rho_rs,
    const double* __restrict__ rdiag, long long rd_rs, const uint8_t* __restrict__ fixed,
    const int* __restrict__ row_map, int hrows, RowState* __restrict__ rst, GridRed red,
    int nelx, int nely, KEq<D, double> ke, MQ<double> mq, PcgParams pp, int replace) {
  const int s = blockIdx.z;
  if (replace && !rst[s].active) return;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const double* xs = x ? x + (size_t)s * x_rs : nullptr;
  const double* rh = rho + (size_t)h * rho_rs;
  const double* rdh = RD ? rdiag + (size_t)h * rd_rs : nullptr;
  const double* bs = b + (size_t)s * b_rs;
  double* rs_ = r + (size_t)s * r_rs;
  double vals[2] = {0.0, 0.0};
  auto loadr = [&](int rr, int cc) { return __ldg(rh + (size_t)rr * nelx + cc); };
  // the residual of one node from A x (unprojected) and b
  auto finish = [&](int rr, int cc, const double(&Ax)[D], const double(&uc)[D], const double(&bv)[D],
                    uint8_t fl, bool has_x) {
    const int node = rr * nnx + cc;
    double res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      double a = 0.0;
      if (has_x) {
        a = Ax[i];
        if (RD) a = fma(__ldg(rdh + node * D + i), uc[i], a);
        if ((fl >> i) & 1) a = 0.0;
      }
      res[i] = bv[i] - a;
      vals[0] = fma(res[i], res[i], vals[0]);
      vals[1] = fma(bv[i], bv[i], vals[1]);
    }
    store_node<D, double>(rs_, node, res);
  };
  if constexpr (MODAL) {
    auto loadf = [&](int rr, int cc) { return __ldg(fixed + rr * nnx + cc); };
    auto loadu = [&](int rr, int cc, uint8_t, double(&v)[D]) { load_node<D, double>(xs, rr * nnx + cc, v); };
    auto loadx = [&](int rr, int cc) {
      RhsB<D, double> e;
      load_node<D, double>(bs, rr * nnx + cc, e.b);
      return e;
    };
    if (xs)
      march_modal<D, double, true, false, true, RhsB<D, double>, double[D], 2, 0>(
          mq, nnx, nny, loadf, loadu, loadr, loadx,
          [&](int rr, int cc, double(&Ax)[D], double(&)[D], const double(&uc)[D], uint8_t fl,
              const RhsB<D, double>& ex) { finish(rr, cc, Ax, uc, ex.b, fl, true); });
    else
      march_modal<D, double, false, false, false, RhsB<D, double>, double[D], 2, 0>(
          mq, nnx, nny, loadf, loadu, loadr, loadx,
          [&](int rr, int cc, double(&Ax)[D], double(&)[D], const double(&uc)[D], uint8_t fl,
              const RhsB<D, double>& ex) { finish(rr, cc, Ax, uc, ex.b, fl, false); });
  } else {
    auto loadu = [&](int rr, int cc, double(&v)[D]) {
      const int node = rr * nnx + cc;
      load_node<D, double>(xs, node, v);
      const uint8_t fl = __ldg(fixed + node);
#pragma unroll
      for (int d = 0; d < D; ++d)
        if ((fl >> d) & 1) v[d] = 0.0;
    };
    auto loadx = [&](int rr, int cc) {
      RhsX<D, double> e;
      const int node = rr * nnx + cc;
      load_node<D, double>(bs, node, e.b);
      e.fl = __ldg(fixed + node);
      return e;
    };
    auto emit = [&](int rr, int cc, double(&Ax)[D], double(&)[D], const double(&uc)[D],
                    const RhsX<D, double>& ex) { finish(rr, cc, Ax, uc, ex.b, ex.fl, xs != nullptr); };
    if (xs)
      march<D, double, true, false, RhsX<D, double>, 0>(ke, nnx, nny, loadu, loadr, loadx, emit);
    else
      march<D, double, false, false, RhsX<D, double>, 0>(ke, nnx, nny, loadu, loadr, loadx, emit);
  }
  const int bid = blockIdx.y * gridDim.x + blockIdx.x;
  grid_reduce<2, kQThreads>(red, s, bid, vals, [&](const double* t) { pcg_init_finish(rst[s], t, pp, replace); });
}

// r = b, its FP32 copy (r32 may be null) and ||b||^2: the initialisation from x = 0 as one
// elementwise pass (no operator apply).
__global__ void __launch_bounds__(kEwThreads) pcg_init_b_kernel(
    const double* __restrict__ b, long long b_rs, double* __restrict__ r, long long r_rs, long long n,
    float* __restrict__ r32, long long r32_rs, RowState* __restrict__ rst, GridRed red, PcgParams pp) {
  const int s = blockIdx.y;
  const double* bs = b + (size_t)s * b_rs;
  double* rs_ = r + (size_t)s * r_rs;
  float* r32s = r32 ? r32 + (size_t)s * r32_rs : nullptr;
  double vals[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)kEwThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kEwThreads) {
    const double v = bs[i];
    rs_[i] = v;
    if (r32s) r32s[i] = (float)v;
    vals[0] = fma(v, v, vals[0]);
  }
  vals[1] = vals[0];
  grid_reduce<2, kEwThreads>(red, s, blockIdx.x, vals, [&](const double* t) { pcg_init_finish(rst[s], t, pp, 0); });
}

// The search direction and its operator product in one pass:
//   PMODE 1 (first iteration): p = z;   PMODE 2: p = beta p_old + z   (p written to pout)
//   Ap = A p (projected, + lumped reaction), pAp = p . Ap, alpha = safe_div(rz, pAp).
// The reference's p update (torch_fem.py:325-331) folded into the p.Ap pass, so p and z
// cross HBM once per iteration instead of twice.  p_old and pout are different buffers:
// the halo columns and rows of a strip belong to its neighbours, which may already have
// written their p.  p is zero at fixed dofs by construction (z is projected).
template <typename TZ, int D>
struct PZIn {
  double p[D];
  TZ z[D];
};

// XP: also add the previous update's alpha p_old to x at each output node (the row's
// pending x update, RowState::xpend), so x is not streamed by the update kernel.
template <int D>
struct XPExtra {
  double x[D], p[D];
};

template <int D, bool MODAL, bool RD, typename TZ, int PMODE, bool XP>
__global__ void __launch_bounds__(kQThreads) pcg_pap_kernel(
    const double* __restrict__ pold, double* __restrict__ pout, int pout_buf, const TZ* __restrict__ z,
    long long z_rs, double* __restrict__ x, long long x_rs, double* __restrict__ Ap, long long rs,
    const double* __restrict__ rho, long long rho_rs, const double* __restrict__ rdiag, long long rd_rs,
    const uint8_t* __restrict__ fixed, const int* __restrict__ row_map, int hrows, RowState* __restrict__ rst,
    GridRed red, int nelx, int nely, KEq<D, double> ke, MQ<double> mq) {
  static_assert(PMODE == 1 || PMODE == 2, "p = z or p = beta p + z");
  static_assert(!XP || PMODE == 2, "a pending x update follows an earlier p");
  const int s = blockIdx.z;
  if (!rst[s].active) return;
  const double beta = PMODE == 2 ? rst[s].beta : 0.0;
  const bool xp = XP && rst[s].xpend;
  const double alpha_prev = XP ? rst[s].alpha : 0.0;
  double* xsr = XP ? x + (size_t)s * x_rs : nullptr;
  const int nnx = nelx + 1, nny = nely + 1;
  const int h = hier_row(row_map, hrows, s);
  const double* ps = PMODE == 2 ? pold + (size_t)s * rs : nullptr;
  double* po = pout + (size_t)s * rs;
  const TZ* zs = z + (size_t)s * z_rs;
  const double* rh = rho + (size_t)h * rho_rs;
  const double* rdh = RD ? rdiag + (size_t)h * rd_rs : nullptr;
  double* As = Ap + (size_t)s * rs;
  double vals[1] = {0.0};
  auto finish = [&](int rr, int cc, double(&Ax)[D], const double(&uc)[D], uint8_t fl, const XPExtra<D>& ex) {
    const int node = rr * nnx + cc;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      if (RD) Ax[i] = fma(__ldg(rdh + node * D + i), uc[i], Ax[i]);
      if ((fl >> i) & 1) Ax[i] = 0.0;
      vals[0] = fma(uc[i], Ax[i], vals[0]);
    }
    store_node<D, double>(As, node, Ax);
    store_node<D, double>(po, node, uc);
    if (XP && xp) {
      double xn[D];
#pragma unroll
      for (int i = 0; i < D; ++i) xn[i] = ex.x[i] + alpha_prev * ex.p[i];
      store_node<D, double>(xsr, node, xn);
    }
  };
  auto loadxp = [&](int rr, int cc) {
    XPExtra<D> e{};
    if (XP && xp) {
      const long long node = (long long)rr * nnx + cc;
      load_node<D, double>(xsr, node, e.x);
      load_node<D, double>(ps, node, e.p);
    }
    return e;
  };
  auto loadr = [&](int rr, int cc) { return __ldg(rh + (size_t)rr * nelx + cc); };
  if constexpr (MODAL) {
    march_modal<D, double, true, false, false, XPExtra<D>, PZIn<TZ, D>, 2, 0>(
        mq, nnx, nny, [&](int rr, int cc) { return __ldg(fixed + rr * nnx + cc); },
        [&](int rr, int cc, uint8_t, PZIn<TZ, D>& in) {
          const long long node = (long long)rr * nnx + cc;
          if (PMODE == 2) load_node<D, double>(ps, node, in.p);
          load_node<D, TZ>(zs, node, in.z);
        },
        loadr, loadxp,
        [&](int rr, int cc, double(&Ax)[D], double(&)[D], const double(&uc)[D], uint8_t fl,
            const XPExtra<D>& ex) { finish(rr, cc, Ax, uc, fl, ex); },
        [&](int, int, uint8_t, const PZIn<TZ, D>& in, double(&v)[D]) {
#pragma unroll
          for (int d = 0; d < D; ++d) v[d] = PMODE == 2 ? fma(in.p[d], beta, (double)in.z[d]) : (double)in.z[d];
        });
  } else {
    march<D, double, true, false, FlagX, 0>(
        ke, nnx, nny,
        [&](int rr, int cc, double(&v)[D]) {
          const long long node = (long long)rr * nnx + cc;
          TZ zv[D];
          load_node<D, TZ>(zs, node, zv);
          double pv[D];
          if (PMODE == 2) load_node<D, double>(ps, node, pv);
#pragma unroll
          for (int d = 0; d < D; ++d) v[d] = PMODE == 2 ? fma(pv[d], beta, (double)zv[d]) : (double)zv[d];
        },
        loadr, [&](int rr, int cc) { return FlagX{__ldg(fixed + rr * nnx + cc)}; },
        [&](int rr, int cc, double(&Ax)[D], double(&)[D], const double(&uc)[D], const FlagX& ex) {
          finish(rr, cc, Ax, uc, ex.fl, loadxp(rr, cc));
        });
  }
  const int bid = blockIdx.y * gridDim.x + blockIdx.x;
  grid_reduce<1, kQThreads>(red, s, bid, vals, [&](const double* t) {
    RowState& S = rst[s];
    S.pAp = t[0];
    S.alpha = safe_div(S.rz, t[0]);
    S.pbuf = pout_buf;
    if (XP) S.xpend = 0;
    if (!isfinite(S.alpha)) S.status = STT_ERR_BREAKDOWN;
  });
}

// x += alpha p, r -= alpha Ap, ||r||^2, convergence.
// r -= alpha Ap, ||r||^2, convergence.  x += alpha p is deferred: the next p.Ap pass
// (which reads this p anyway) or the final flush adds it (RowState::xpend).
__global__ void __launch_bounds__(kEwThreads) pcg_update_kernel(
    double* __restrict__ r, const double* __restrict__ Ap, long long rs, long long n,
    RowState* __restrict__ rst, GridRed red, PcgParams pp, float* __restrict__ r32, long long r32_rs) {
  const int s = blockIdx.y;
  if (!rst[s].active) return;
  const double alpha = rst[s].alpha;
  double* rsv = r + (size_t)s * rs;
  const double* as = Ap + (size_t)s * rs;
  float* r32s = r32 ? r32 + (size_t)s * r32_rs : nullptr;
  double vals[1] = {0.0};
  auto one = [&](long long i) {
    const double rv = rsv[i] - alpha * as[i];
    rsv[i] = rv;
    if (r32s) r32s[i] = (float)rv;  // the FP32 V-cycle's right-hand side
    vals[0] = fma(rv, rv, vals[0]);
  };
  if ((rs & 1) == 0) {
    // pairs of dofs (128-bit loads): with an even row stride every row starts 16-byte
    // aligned (the workspace is 256-byte aligned; the FP32 copy's stride is a multiple of 4)
    const long long n2 = n / 2;
    double2* r2 = reinterpret_cast<double2*>(rsv);
    const double2* a2 = reinterpret_cast<const double2*>(as);
    for (long long i = blockIdx.x * (long long)kEwThreads + threadIdx.x; i < n2;
         i += (long long)gridDim.x * kEwThreads) {
      const double2 rr = r2[i], aa = __ldg(a2 + i);
      const double2 rv = make_double2(rr.x - alpha * aa.x, rr.y - alpha * aa.y);
      r2[i] = rv;
      if (r32s) reinterpret_cast<float2*>(r32s)[i] = make_float2((float)rv.x, (float)rv.y);
      vals[0] = fma(rv.x, rv.x, vals[0]);
      vals[0] = fma(rv.y, rv.y, vals[0]);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) one(n - 1);  // odd-length rows
  } else {
    for (long long i = blockIdx.x * (long long)kEwThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kEwThreads)
      one(i);
  }
  grid_reduce<1, kEwThreads>(red, s, blockIdx.x, vals, [&](const double* t) {
    RowState& S = rst[s];
    S.xpend = 1;
    S.rel = sqrt(t[0]) / S.bnorm_safe;
    if (!isfinite(S.rel)) S.status = STT_ERR_BREAKDOWN;
    pcg_converged(S, pp);
  });
}

// The reference's row retirement (torch_fem.pcg, sttopt/torch_fem.py:270-331): converged
// rows keep iterating with the others until the rows still short of rtol are at most
// COMPACTION_RATIO = 3/4 of the rows left by the previous retirement (*last); then every
// converged row stops (its x stays as of this iteration), and when no row is short of
// rtol all stop.  One warp; rows in order.
__global__ void pcg_retire_kernel(RowState* __restrict__ rst, int nrows, int* __restrict__ last, int it) {
  const int lane = threadIdx.x;
  int n_left = 0;  // active rows not yet converged
  for (int s = lane; s < nrows; s += 32) n_left += (rst[s].active && !rst[s].conv) ? 1 : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n_left += __shfl_xor_sync(0xffffffffu, n_left, o);
  if (it == 0 && lane == 0) {
    int n_act = 0;
    for (int s = 0; s < nrows; ++s) n_act += rst[s].active;
    *last = n_act;
  }
  __syncwarp();
  const int prev = *last;
  // n_left <= 0.75 * last, in integers; a single row is never compacted, it just finishes
  const bool retire = n_left == 0 || (nrows > 1 && 4LL * n_left <= 3LL * prev);
  __syncwarp();
  if (!retire) return;
  for (int s = lane; s < nrows; s += 32) {
    RowState& S = rst[s];
    if (S.active && S.conv) {
      S.active = 0;
      S.conv_iter = it;
    }
  }
  if (lane == 0) *last = n_left;
}

// x += alpha p for every row whose last update is still pending (p from the buffer its
// last p.Ap pass wrote); then pcg_xclear_kernel clears the flags.
__global__ void __launch_bounds__(kEwThreads) pcg_xflush_kernel(double* __restrict__ x, long long x_rs,
                                                                const double* __restrict__ p0,
                                                                const double* __restrict__ p1, long long rs,
                                                                long long n, const RowState* __restrict__ rst) {
  const int s = blockIdx.y;
  if (!rst[s].xpend) return;
  const double alpha = rst[s].alpha;
  double* xs = x + (size_t)s * x_rs;
  const double* ps = (rst[s].pbuf ? p1 : p0) + (size_t)s * rs;
  for (long long i = blockIdx.x * (long long)kEwThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kEwThreads)
    xs[i] = xs[i] + alpha * ps[i];
}

__global__ void pcg_xclear_kernel(RowState* __restrict__ rst, int nrows) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nrows) rst[s].xpend = 0;
}

// rz = r . z (and r . z_old for the flexible beta); first: p = z, rz_old = rz;
// otherwise beta = safe_div(rz - rz_mix, rz_old), rz_old = rz.
template <typename TZ, typename TR>
__global__ void __launch_bounds__(kEwThreads) pcg_rz_kernel(
    const TR* __restrict__ r, const TZ* __restrict__ z, const TZ* __restrict__ zold,
    double* __restrict__ p, long long rs, long long z_rs, long long n, RowState* __restrict__ rst,
    GridRed red, int first, int flexible) {
  const int s = blockIdx.y;
  if (!rst[s].active) return;
  const TR* rsv = r + (size_t)s * rs;
  const TZ* zs = z + (size_t)s * z_rs;
  const TZ* zo = zold + (size_t)s * z_rs;
  double vals[2] = {0.0, 0.0};
  auto one = [&](long long i) {
    const double zv = (double)zs[i];
    const double rv = (double)rsv[i];
    vals[0] = fma(rv, zv, vals[0]);
    if (flexible && !first) vals[1] = fma(rv, (double)zo[i], vals[1]);
    if (first && p) p[(size_t)s * rs + i] = zv;
  };
  bool vec = false;
  if constexpr (sizeof(TZ) == 4 && sizeof(TR) == 4) {
    // FP32 vectors with row strides a multiple of 4 (16-byte aligned rows): 128-bit loads
    vec = !p && ((rs | z_rs) & 3) == 0 && (((uintptr_t)r | (uintptr_t)z | (uintptr_t)zold) & 15) == 0;
    if (vec) {
      const long long n4 = n / 4;
      const float4* r4 = reinterpret_cast<const float4*>(rsv);
      const float4* z4 = reinterpret_cast<const float4*>(zs);
      const float4* o4 = reinterpret_cast<const float4*>(zo);
      const bool mix = flexible && !first;
      for (long long i = blockIdx.x * (long long)kEwThreads + threadIdx.x; i < n4;
           i += (long long)gridDim.x * kEwThreads) {
        const float4 rv = __ldg(r4 + i), zv = __ldg(z4 + i);
        vals[0] = fma((double)rv.x, (double)zv.x, vals[0]);
        vals[0] = fma((double)rv.y, (double)zv.y, vals[0]);
        vals[0] = fma((double)rv.z, (double)zv.z, vals[0]);
        vals[0] = fma((double)rv.w, (double)zv.w, vals[0]);
        if (mix) {
          const float4 ov = __ldg(o4 + i);
          vals[1] = fma((double)rv.x, (double)ov.x, vals[1]);
          vals[1] = fma((double)rv.y, (double)ov.y, vals[1]);
          vals[1] = fma((double)rv.z, (double)ov.z, vals[1]);
          vals[1] = fma((double)rv.w, (double)ov.w, vals[1]);
        }
      }
      if (blockIdx.x == 0 && threadIdx.x < (n & 3)) one(n4 * 4 + threadIdx.x);  // the row's tail
    }
  }
  if (!vec)
    for (long long i = blockIdx.x * (long long)kEwThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kEwThreads)
      one(i);
  grid_reduce<2, kEwThreads>(red, s, blockIdx.x, vals,
                             [&](const double* t) { pcg_rz_finish(rst[s], t, first, flexible); });
}


__global__ void rows_zero_kernel(double* __restrict__ x, long long rs, long long n) {
  const int s = blockIdx.y;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[(size_t)s * rs + i] = 0.0;
}

// ---- drivers ----------------------------------------------------------------------

template <int D, typename T>
static KEq<D, T> ke_of(const stt_hier* h) {
  KEq<D, T> k;
  for (int i = 0; i < 16 * D * D; ++i) k.v[i] = T(h->KE[i]);
  return k;
}

// z = M r over all rows (rst may gate rows).  r FP64 with row stride r_rs; zout in the
// cycle precision with the padded stride vstride(ndof0).
template <int D, typename T>
static int run_vcycle(const stt_hier* h, SolveWS& w, int nrows, const double* r, long long r_rs,
                      T* zout, double omega, int n_smooth,
                      int gamma, const RowState* rst, cudaStream_t st, bool b0_ready = false,
                      const RzFuse<T>* rzf = nullptr, bool* rz_done = nullptr) {
  Cycle<D, T> cyc{h, w, nrows, T(omega), n_smooth, gamma, rst, st, ke_of<D, T>(h), mq_cast<T>(h->mq)};
  if (rzf) cyc.rzf = *rzf;
  const long long n = h->lv[0].ndof, vs = vstride(n);
  const T* b0;
  long long b_rs;
  if constexpr (sizeof(T) == 4) {
    // the PCG update may have written the FP32 copy of r already
    if (!b0_ready)
      rows_convert_kernel<double, float><<<dim3(ew_blocks(n), nrows), kEwThreads, 0, st>>>(
          r, r_rs, (float*)w.b0, vs, n, rst);
    b0 = (const T*)w.b0;
    b_rs = vs;
  } else {
    b0 = (const T*)r;
    b_rs = r_rs;
  }
  cyc.final_out = zout;
  T* res = cyc.cycle(0, b0, b_rs);
  if (rz_done) *rz_done = cyc.rz_done;
  if (res != zout)
    rows_convert_kernel<T, T><<<dim3(ew_blocks(n), nrows), kEwThreads, 0, st>>>(res, vs, zout, vs, n, rst);
  return check_launch("vcycle");
}

// Optional live timing of the plane-stress solves' steady-state p.Ap passes (the step's
// dominant kernel, pcg_pap_kernel<2, ..., PMODE 2, XP>): while enabled, every such launch
// is bracketed by CUDA events on its stream, and the solve adds the elapsed times at its
// end (after its final synchronisation).  Off by default; stt_pap_timing.
struct PapTiming {
  std::mutex mu;
  bool on = false;
  double total_ms = 0.0;
  long long launches = 0;
  long long rows = 0;  // summed over the launches (bytes scale with the rows)
};
static PapTiming g_pap;

struct PapEvents {
  std::vector<cudaEvent_t> ev;  // pairs (start, stop)
  std::vector<int> rows;
  size_t used = 0;
  ~PapEvents() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
  int record(cudaStream_t st, bool start, int nrows) {
    const size_t i = start ? used : used + 1;
    while (ev.size() <= i) {
      cudaEvent_t e;
      STT_TRY(check_cuda(cudaEventCreate(&e), "timing event"));
      ev.push_back(e);
    }
    STT_TRY(check_cuda(cudaEventRecord(ev[i], st), "timing record"));
    if (!start) {
      rows.push_back(nrows);
      used += 2;
    }
    return STT_OK;
  }
  // after the stream has synchronised
  void flush() {
    if (!used) return;
    double ms = 0.0;
    long long nr = 0;
    for (size_t i = 0; i + 1 < used; i += 2) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, ev[i], ev[i + 1]) == cudaSuccess) ms += t;
    }
    for (int r : rows) nr += r;
    std::lock_guard<std::mutex> lock(g_pap.mu);
    g_pap.total_ms += ms;
    g_pap.launches += (long long)(used / 2);
    g_pap.rows += nr;
    used = 0;
    rows.clear();
  }
};

template <int D, typename T>
static int run_pcg(const stt_hier* h, SolveWS& w, int nrows, const double* b, long long b_rs,
                   double* x, long long x_rs, int has_x0, double rtol, int max_iter, double omega,
                   int n_smooth, int gamma, int flexible, int replace_every, int sched, double* rel_out,
                   int* conv_out, int* n_iter_out, cudaStream_t st) {
  const LevelDesc& l0 = h->lv[0];
  const long long nd = l0.ndof;
  const dim3 tg = pcg_tile_grid(h->nelx, h->nely, nrows);
  const int ewb = ew_blocks(nd);
  GridRed red_tile{w.partials, w.counters, (int)(tg.x * tg.y)};
  GridRed red_ew{w.partials, w.counters, ewb};
  // the FP32 r.z pass: eight 128-bit loads of each vector a thread (its block partials
  // and reduction cost less than with one block per 1024 values)
  const int rzb = (int)std::max<long long>(1, std::min<long long>(ewb, (nd / 4 + 8 * kEwThreads - 1) / (8 * kEwThreads)));
  GridRed red_rz{w.partials, w.counters, rzb};
  // the r update likewise: eight 128-bit pairs of r and Ap a thread
  const int upb = (int)std::max<long long>(1, std::min<long long>(ewb, (nd / 2 + 8 * kEwThreads - 1) / (8 * kEwThreads)));
  GridRed red_up{w.partials, w.counters, upb};
  const KEq<D, double> ke = ke_of<D, double>(h);
  const double* rd0 = h->has_reaction ? l0.rdiag64 : nullptr;
  STT_TRY(check_cuda(cudaMemsetAsync(w.counters, 0, 4LL * nrows, st), "memset counters"));
  STT_TRY(check_cuda(cudaMemsetAsync(w.rs, 0, sizeof(RowState) * nrows, st), "memset rows"));
  if (!has_x0) rows_zero_kernel<<<dim3(ewb, nrows), kEwThreads, 0, st>>>(x, x_rs, nd);
  const MQ<double> mq = mq_cast<double>(h->mq);
  bool timing = false;
  if (D == 2) {
    std::lock_guard<std::mutex> lock(g_pap.mu);
    timing = g_pap.on;
  }
  PapEvents pev;
  // r = b - A x (x may be null: r = b); replace = 1 keeps ||b|| (true-residual replacement)
  // the initialisation from x = 0 also writes (FP32 cycle) r's FP32 copy, the first
  // V-cycle's right-hand side; after a warm start, which often converges at once (the
  // adjoints' alpha U), and after a true-residual replacement the cycle converts r itself
  float* r32init = sizeof(T) == 4 ? (float*)w.b0 : nullptr;
  auto init = [&](const double* xx, const PcgParams& pq, int replace) {
    if (!xx && !replace) {
      pcg_init_b_kernel<<<dim3(upb, nrows), kEwThreads, 0, st>>>(b, b_rs, w.r, nd, nd, r32init, vstride(nd), w.rs,
                                                                  red_up, pq);
      return;
    }
#define STT_INIT(MODAL, RD)                                                                              \
  pcg_init_kernel<D, MODAL, RD><<<tg, kQThreads, 0, st>>>(b, b_rs, xx, x_rs, w.r, nd, l0.rho64, l0.rs_rho, rd0, \
                                                          l0.ndof, l0.fixed, h->row_map, h->hrows, w.rs,        \
                                                          red_tile, h->nelx, h->nely, ke, mq, pq, replace)
    if (h->modal) {
      if (rd0) STT_INIT(true, true);
      else STT_INIT(true, false);
    } else {
      if (rd0) STT_INIT(false, true);
      else STT_INIT(false, false);
    }
#undef STT_INIT
  };
  PcgParams pp{rtol, 0, flexible, sched ? 1 : 0};
  init(has_x0 ? x : nullptr, pp, 0);
  if (sched) pcg_retire_kernel<<<1, 32, 0, st>>>(w.rs, nrows, w.sched_last, 0);
  STT_TRY(check_launch("pcg init"));
  std::vector<RowState> host(nrows);
  // the reads after the first V-cycle also carry the hierarchy build's status word (the
  // build does not synchronise, and the coarse factorisation runs on the hierarchy's side
  // stream, overlapping the initialisation and the first descent): a failed coarse
  // factorisation surfaces there
  int hstatus = 0;
  bool hchecked = false;
  auto pull = [&](bool with_status) -> int {
    STT_TRY(check_cuda(cudaMemcpyAsync(host.data(), w.rs, sizeof(RowState) * nrows, cudaMemcpyDeviceToHost, st), "row state"));
    with_status = with_status && !hchecked;
    if (with_status) {
      STT_TRY(check_cuda(cudaStreamWaitEvent(st, h->sync->ready, 0), "wait coarse"));
      STT_TRY(check_cuda(cudaMemcpyAsync(&hstatus, h->status, sizeof(int), cudaMemcpyDeviceToHost, st), "status copy"));
    }
    STT_TRY(check_cuda(cudaStreamSynchronize(st), "pcg sync"));
    if (with_status) {
      hchecked = true;
      STT_TRY(hier_status_code(hstatus));
    }
    return STT_OK;
  };
  auto n_active = [&]() {
    int a = 0;
    for (auto& s : host) a += s.active;
    return a;
  };
  STT_TRY(pull(false));
  int it = 0;
  if (n_active() > 0) {
    T* z = (T*)w.z;
    T* zold = (T*)w.zold;
    double* pcur = w.p;    // p of the previous iteration
    double* pnext = w.p2;  // where this iteration's p goes
    int pnext_buf = 1;     // index of pnext: 0 = w.p, 1 = w.p2
    // adds every row's pending alpha p to x (before a true-residual replacement and at
    // the end); the p.Ap pass of the next iteration does it for rows still iterating
    auto flush_x = [&]() {
      pcg_xflush_kernel<<<dim3(ewb, nrows), kEwThreads, 0, st>>>(x, x_rs, w.p, w.p2, nd, nd, w.rs);
      pcg_xclear_kernel<<<(nrows + 127) / 128, 128, 0, st>>>(w.rs, nrows);
    };
    bool pending = false;  // the rows still iterating have an x update pending
    // r . z: the mixed cycle's z carries FP32 rounding, so its dots read the FP32 copy of r
    // the cycle itself read (written by the update, or by the cycle's own conversion).
    // Level 0's chained passes take them where the cycle runs them (r . z_old beside the
    // pre-smoothing, r . z as the post-smoothing writes z); otherwise a pass of their own.
    auto fuse_of = [&](int first) {
      RzFuse<T> f{};
      f.rst = w.rs;
      f.zold = (flexible && !first) ? zold : nullptr;
      f.zo_rs = vstride(nd);
      f.red = GridRed{w.partials, w.counters, 0};
      f.first = first;
      f.flexible = flexible;
      return f;
    };
    auto rz = [&](int first) {
      if constexpr (sizeof(T) == 4)
        pcg_rz_kernel<T, float><<<dim3(rzb, nrows), kEwThreads, 0, st>>>(
            (const float*)w.b0, z, zold, nullptr, vstride(nd), vstride(nd), nd, w.rs, red_rz, first, flexible);
      else
        pcg_rz_kernel<T, double><<<dim3(ewb, nrows), kEwThreads, 0, st>>>(w.r, z, zold, nullptr, nd, vstride(nd),
                                                                           nd, w.rs, red_ew, first, flexible);
    };
    {
      const RzFuse<T> f = fuse_of(1);
      bool done = false;
      STT_TRY(run_vcycle<D, T>(h, w, nrows, w.r, nd, z, omega, n_smooth, gamma, w.rs, st,
                               r32init != nullptr && !has_x0, &f, &done));
      if (!done) rz(1);
    }
    int check_every = 1;
    for (it = 1; it <= max_iter; ++it) {
      pp.it = it;
#define STT_PAP(MODAL, RD, PM, XP)                                                                         \
  pcg_pap_kernel<D, MODAL, RD, T, PM, XP><<<tg, kQThreads, 0, st>>>(                                       \
      pcur, pnext, pnext_buf, z, vstride(nd), x, x_rs, w.Ap, nd, l0.rho64, l0.rs_rho, rd0, l0.ndof, l0.fixed, \
      h->row_map, h->hrows, w.rs, red_tile, h->nelx, h->nely, ke, mq)
#define STT_PAP2(PM, XP)                    \
  do {                                      \
    if (h->modal) {                         \
      if (rd0) STT_PAP(true, true, PM, XP);   \
      else STT_PAP(true, false, PM, XP);      \
    } else {                                \
      if (rd0) STT_PAP(false, true, PM, XP);  \
      else STT_PAP(false, false, PM, XP);     \
    }                                       \
  } while (0)
      if (it == 1) {
        STT_PAP2(1, false);
      } else if (pending) {
        if (timing) STT_TRY(pev.record(st, true, nrows));
        STT_PAP2(2, true);
        if (timing) STT_TRY(pev.record(st, false, nrows));
      } else {
        STT_PAP2(2, false);
      }
#undef STT_PAP2
#undef STT_PAP
      float* r32 = sizeof(T) == 4 ? (float*)w.b0 : nullptr;
      std::swap(pcur, pnext);
      pnext_buf ^= 1;
      pcg_update_kernel<<<dim3(upb, nrows), kEwThreads, 0, st>>>(w.r, w.Ap, nd, nd, w.rs, red_up, pp, r32,
                                                                  vstride(nd));
      if (sched) pcg_retire_kernel<<<1, 32, 0, st>>>(w.rs, nrows, w.sched_last, it);
      pending = true;
      const bool replaced = replace_every > 0 && it % replace_every == 0;
      if (replaced) {
        flush_x();
        pending = false;
        init(x, pp, 1);
      }
      if (flexible) std::swap(z, zold);
      {
        const RzFuse<T> f = fuse_of(0);
        bool done = false;
        STT_TRY(run_vcycle<D, T>(h, w, nrows, w.r, nd, z, omega, n_smooth, gamma, w.rs, st, r32 && !replaced, &f,
                                 &done));
        if (!done) rz(0);
      }
      STT_TRY(check_launch("pcg iteration"));
      if (it % check_every == 0 || it == max_iter) {
        STT_TRY(pull(true));
        if (n_active() == 0) break;
        // a wider check interval once the solve is evidently long
        if (it >= 8) check_every = 2;
        if (it >= 32) check_every = 4;
      }
    }
    flush_x();
    STT_TRY(check_launch("pcg flush"));
  }
  STT_TRY(pull(true));
  if (timing) pev.flush();
  int worst = 0, status = STT_OK;
  for (int s = 0; s < nrows; ++s) {
    rel_out[s] = host[s].rel;
    conv_out[s] = host[s].active ? -1 : host[s].conv_iter;
    worst = std::max(worst, host[s].conv_iter);
    if (host[s].active) status = STT_ERR_NOT_CONVERGED;
  }
  *n_iter_out = status == STT_OK ? worst : max_iter;
  if (status != STT_OK)
    return set_error(status, "CG did not converge within max_iter");
  return STT_OK;
}

}  // namespace stt

using namespace stt;

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

extern "C" long long stt_solve_workspace_bytes(const stt_hier* h, int nrows, int gamma) {
  if (!h || nrows <= 0) return -1;
  SolveWS w;
  return plan_solve(h, nrows, gamma, nullptr, w);
}

extern "C" long long stt_vcycle_workspace_bytes(const stt_hier* h, int nrows, int gamma) {
  if (!h || nrows <= 0) return -1;
  SolveWS w;
  return plan_solve(h, nrows, gamma, nullptr, w, false);
}

extern "C" int stt_vcycle(const stt_hier* h, int nrows, const double* r, long long r_rs, double* z,
                          long long z_rs, double omega, int n_smooth, int gamma, void* workspace,
                          long long ws_bytes, stt_stream_t stream) {
  if (!h) return set_error(STT_ERR_INVALID, "null hierarchy");
  ScopedTuning tuning(h->tune_pcg_band, h->tune_waves);
  if (!h || !r || !z || !workspace || nrows <= 0 || nrows > 65535 || n_smooth < 1 || gamma < 1)
    return set_error(STT_ERR_INVALID, "stt_vcycle: bad arguments");
  if (h->d == 2 && (!aligned16(r) || !aligned16(z) || (r_rs % 2) || (z_rs % 2)))
    return set_error(STT_ERR_INVALID, "stt_vcycle: 2-dof vectors must be 16-byte aligned with even row strides");
  SolveWS w;
  const long long need = plan_solve(h, nrows, gamma, nullptr, w, false);
  if (ws_bytes < need) return set_error(STT_ERR_WORKSPACE, "stt_vcycle: workspace too small");
  plan_solve(h, nrows, gamma, (char*)workspace, w, false);
  cudaStream_t st = (cudaStream_t)stream;
  const long long nd = h->lv[0].ndof;
  int rc;
  if (h->precision == STT_FP32) {
    rc = h->d == 2 ? run_vcycle<2, float>(h, w, nrows, r, r_rs, (float*)w.z, omega, n_smooth, gamma, nullptr, st)
                   : run_vcycle<1, float>(h, w, nrows, r, r_rs, (float*)w.z, omega, n_smooth, gamma, nullptr, st);
    if (rc == STT_OK)
      rows_convert_kernel<float, double><<<dim3(ew_blocks(nd), nrows), kEwThreads, 0, st>>>((float*)w.z, vstride(nd), z, z_rs, nd, nullptr);
  } else {
    rc = h->d == 2 ? run_vcycle<2, double>(h, w, nrows, r, r_rs, (double*)w.z, omega, n_smooth, gamma, nullptr, st)
                   : run_vcycle<1, double>(h, w, nrows, r, r_rs, (double*)w.z, omega, n_smooth, gamma, nullptr, st);
    if (rc == STT_OK)
      rows_convert_kernel<double, double><<<dim3(ew_blocks(nd), nrows), kEwThreads, 0, st>>>((double*)w.z, vstride(nd), z, z_rs, nd, nullptr);
  }
  if (rc != STT_OK) return rc;
  return check_launch("stt_vcycle");
}

extern "C" int stt_level_apply(const stt_hier* h, int level, int nrows, const double* v, long long v_rs,
                               double* out, long long out_rs, stt_stream_t stream) {
  if (!h) return set_error(STT_ERR_INVALID, "null hierarchy");
  ScopedTuning tuning(h->tune_pcg_band, h->tune_waves);
  if (!h || !v || !out || level < 0 || level >= h->nlevels || nrows <= 0 || nrows > 65535)
    return set_error(STT_ERR_INVALID, "stt_level_apply: bad arguments");
  if (h->d == 2 && (!aligned16(v) || !aligned16(out) || (v_rs % 2) || (out_rs % 2)))
    return set_error(STT_ERR_INVALID, "stt_level_apply: 2-dof vectors must be 16-byte aligned with even row strides");
  cudaStream_t st = (cudaStream_t)stream;
  const LevelDesc& lv = h->lv[level];
  if (level == 0) {
    const dim3 g = tile_grid(lv.nelx, lv.nely, nrows);
    const double* rd = h->has_reaction ? lv.rdiag64 : nullptr;
    const MQ<double> mq = mq_cast<double>(h->mq);
    const ProlongSrc<double> none{nullptr, 0, 1, 1, 1};
#define STT_L0_APPLY(D)                                                                                  \
  do {                                                                                                   \
    if (h->modal && rd)                                                                                  \
      l0_sweep_modal_kernel<D, double, SW_APPLY, true><<<g, kQThreads, 0, st>>>(                        \
          v, v_rs, nullptr, 0, out, out_rs, lv.rho64, lv.rs_rho, rd, lv.ndof, lv.fixed, h->row_map,      \
          h->hrows, nullptr, lv.nelx, lv.nely, 1.0, mq, none);                                          \
    else if (h->modal)                                                                                   \
      l0_sweep_modal_kernel<D, double, SW_APPLY, false><<<g, kQThreads, 0, st>>>(                       \
          v, v_rs, nullptr, 0, out, out_rs, lv.rho64, lv.rs_rho, rd, lv.ndof, lv.fixed, h->row_map,      \
          h->hrows, nullptr, lv.nelx, lv.nely, 1.0, mq, none);                                          \
    else                                                                                                 \
      l0_sweep_kernel<D, double, SW_APPLY><<<g, kQThreads, 0, st>>>(                                    \
          v, v_rs, nullptr, 0, out, out_rs, lv.rho64, lv.rs_rho, rd, lv.ndof, lv.fixed, h->row_map,      \
          h->hrows, nullptr, lv.nelx, lv.nely, 1.0, ke_of<D, double>(h), 1, none);                      \
  } while (0)
    if (h->d == 2) STT_L0_APPLY(2);
    else STT_L0_APPLY(1);
#undef STT_L0_APPLY
    return check_launch("level apply");
  }
  if (v_rs != out_rs)
    return set_error(STT_ERR_INVALID, "stt_level_apply: coarse levels need equal row strides");
  STT_TRY(ensure_level1_fp64(h, level, st));
  if (h->d == 2)
    st_sweep2_kernel<2, double, SW_APPLY><<<tile_grid(lv.nelx, lv.nely, nrows), kQThreads, 0, st>>>(
        v, nullptr, out, v_rs, lv.st64, lv.fixed, lv.nnx, lv.nny, h->row_map, h->hrows, nullptr, 1.0);
  else
    st_sweep2_kernel<1, double, SW_APPLY><<<tile_grid(lv.nelx, lv.nely, nrows), kQThreads, 0, st>>>(
        v, nullptr, out, v_rs, lv.st64, lv.fixed, lv.nnx, lv.nny, h->row_map, h->hrows, nullptr, 1.0);
  return check_launch("level apply");
}

extern "C" int stt_pcg_mg(const stt_hier* h, int nrows, const double* b, long long b_rs, double* x,
                          long long x_rs, int has_x0, double rtol, int max_iter, double omega,
                          int n_smooth, int gamma, int flexible, int replace_every, int retire,
                          double* rel_resid, int* conv_iter, int* n_iter, void* workspace, long long ws_bytes,
                          stt_stream_t stream) {
  if (!h) return set_error(STT_ERR_INVALID, "null hierarchy");
  ScopedTuning tuning(h->tune_pcg_band, h->tune_waves);
  if (!h || !b || !x || !workspace || !rel_resid || !conv_iter || !n_iter || nrows <= 0 ||
      nrows > 65535 || max_iter < 0 || n_smooth < 1 || gamma < 1)
    return set_error(STT_ERR_INVALID, "stt_pcg_mg: bad arguments");
  if (h->d == 2 && (!aligned16(b) || !aligned16(x) || (b_rs % 2) || (x_rs % 2)))
    return set_error(STT_ERR_INVALID, "stt_pcg_mg: 2-dof vectors must be 16-byte aligned with even row strides");
  SolveWS w;
  const long long need = plan_solve(h, nrows, gamma, nullptr, w);
  if (ws_bytes < need) return set_error(STT_ERR_WORKSPACE, "stt_pcg_mg: workspace too small");
  plan_solve(h, nrows, gamma, (char*)workspace, w);
  cudaStream_t st = (cudaStream_t)stream;
  if (h->precision == STT_FP32)
    return h->d == 2 ? run_pcg<2, float>(h, w, nrows, b, b_rs, x, x_rs, has_x0, rtol, max_iter, omega, n_smooth, gamma, flexible, replace_every, retire, rel_resid, conv_iter, n_iter, st)
                     : run_pcg<1, float>(h, w, nrows, b, b_rs, x, x_rs, has_x0, rtol, max_iter, omega, n_smooth, gamma, flexible, replace_every, retire, rel_resid, conv_iter, n_iter, st);
  return h->d == 2 ? run_pcg<2, double>(h, w, nrows, b, b_rs, x, x_rs, has_x0, rtol, max_iter, omega, n_smooth, gamma, flexible, replace_every, retire, rel_resid, conv_iter, n_iter, st)
                   : run_pcg<1, double>(h, w, nrows, b, b_rs, x, x_rs, has_x0, rtol, max_iter, omega, n_smooth, gamma, flexible, replace_every, retire, rel_resid, conv_iter, n_iter, st);
}

// ---- V-cycle without a caller workspace ---------------------------------------------
//
// Some callers cannot allocate device memory: plugins inside a host application that
// owns the device memory pool and forbids outside cudaMalloc, multi-stream pipelines
// that cannot afford cudaMalloc's implicit device synchronisation mid-run, or
// foreign-language bindings that can hand over input and output buffers but not size
// and own a scratch buffer.  stt_vcycle_noalloc serves
// them: it runs exactly stt_vcycle, with its scratch taken from a fixed-size array
// compiled into this library instead of a caller workspace.
//
// Limits and rules:
//  * the scratch is kVCycleScratchBytes (32 MiB) per device; every GPU that loads the
//    library holds it until the process exits.  A call whose V-cycle scratch
//    (stt_vcycle_workspace_bytes for the same hierarchy, rows and gamma) exceeds it is
//    rejected with STT_ERR_WORKSPACE before anything is launched;
//  * all calls on a device share the one array and it keeps the last call's
//    contents; the V-cycle writes every scratch word before reading it, so nothing has
//    to start at zero.  Calls that overlap on the GPU (different streams, or threads
//    without ordering) race on the array: order them on one stream;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current and keeps it for the life of the
//    process; make that first call before any stream capture begins.  Like the rest of
//    the library (hierarchy handles, its pooled streams), it must not be used across a
//    cudaDeviceReset or other reset of the device's primary context.

namespace {

constexpr long long kVCycleScratchBytes = 32LL << 20;

__device__ __align__(256) unsigned char g_vcycle_scratch[kVCycleScratchBytes];

std::mutex g_vcycle_scratch_mu;
void* g_vcycle_scratch_ptr[256] = {};

int vcycle_scratch_address(void** out) {
  int dev = 0;
  STT_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
  if (dev < 0 || dev >= 256) return set_error(STT_ERR_INVALID, "stt_vcycle_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_vcycle_scratch_mu);
  if (!g_vcycle_scratch_ptr[dev]) {
    void* p = nullptr;
    STT_TRY(check_cuda(cudaGetSymbolAddress(&p, g_vcycle_scratch), "cudaGetSymbolAddress(g_vcycle_scratch)"));
    g_vcycle_scratch_ptr[dev] = p;
  }
  *out = g_vcycle_scratch_ptr[dev];
  return STT_OK;
}

}  // namespace

extern "C" int stt_vcycle_noalloc(const stt_hier* h, int nrows, const double* r, long long r_rs,
                                  double* z, long long z_rs, double omega, int n_smooth, int gamma,
                                  stt_stream_t stream) {
  if (!h || nrows <= 0 || nrows > 65535 || gamma < 1)
    return set_error(STT_ERR_INVALID, "stt_vcycle_noalloc: bad arguments");
  const long long need = stt_vcycle_workspace_bytes(h, nrows, gamma);
  if (need < 0 || need > kVCycleScratchBytes)
    return set_error(STT_ERR_WORKSPACE,
                     "stt_vcycle_noalloc: this V-cycle needs more scratch than the library's fixed 32 MiB; "
                     "use stt_vcycle with a caller workspace");
  void* scratch = nullptr;
  STT_TRY(vcycle_scratch_address(&scratch));
  return stt_vcycle(h, nrows, r, r_rs, z, z_rs, omega, n_smooth, gamma, scratch, kVCycleScratchBytes, stream);
}

extern "C" int stt_hier_tune(stt_hier* h, int pcg_band, int level_waves) {
  if (!h || !(pcg_band == 0 || pcg_band == 8 || pcg_band == 16 || pcg_band == 32) || level_waves < 0 ||
      level_waves > 64)
    return set_error(STT_ERR_INVALID, "stt_hier_tune: pcg_band must be 0, 8, 16 or 32 and level_waves in [0, 64]");
  h->tune_pcg_band = pcg_band;
  h->tune_waves = level_waves;
  return STT_OK;
}

extern "C" int stt_pap_timing(int enable) {
  std::lock_guard<std::mutex> lock(g_pap.mu);
  g_pap.on = enable != 0;
  g_pap.total_ms = 0.0;
  g_pap.launches = 0;
  g_pap.rows = 0;
  return STT_OK;
}

extern "C" int stt_pap_timing_read(double* total_ms, long long* launches, long long* rows) {
  if (!total_ms || !launches || !rows) return set_error(STT_ERR_INVALID, "stt_pap_timing_read: null output");
  std::lock_guard<std::mutex> lock(g_pap.mu);
  *total_ms = g_pap.total_ms;
  *launches = g_pap.launches;
  *rows = g_pap.rows;
  return STT_OK;
}
