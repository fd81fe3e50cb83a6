// Device construction of the Galerkin multigrid hierarchy (torch_mg.build_hierarchy,
// sttopt/torch_mg.py:293-400) and the block-banded Cholesky factor of its coarsest
// level (torch_mg._dense_cholesky, :269-290).
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "errors.h"
#include "hier.h"
#include "modal.h"
#include "q4.cuh"

namespace stt {

// ---- host tables --------------------------------------------------------------

// Coarsening factor of one dimension: the smallest of 2, 3 dividing n, else 1
// (torch_mg.coarsening_factors, :53-72).
static int factor_of(int n) { return n % 2 == 0 ? 2 : (n % 3 == 0 ? 3 : 1); }

// Piecewise-linear interpolation of two coarse values at fine offset j of k, in the
// reference's operation order (torch_mg._interp_axis, :75-81).
static double interp1(double a, double b, int j, int k) {
  if (j == k) return b;
  const double w = (double)j / k;
  return a * (1 - w) + b * w;
}

// S[m][p][q]: weight of coarse local dof q on child m's local dof p
// (torch_mg.child_interpolation_matrices, :140-165), derived by interpolating the
// coarse element's unit basis vectors over its (ky+1) x (kx+1) fine nodes.
static void child_interp(int kx, int ky, int d, double* S /* [kx*ky][4d][4d] */) {
  const int nk = 4 * d;
  std::memset(S, 0, sizeof(double) * kx * ky * nk * nk);
  // coarse corners BL, BR, TR, TL at (row, col) of the 2x2 coarse node grid
  for (int qc = 0; qc < 4; ++qc) {
    const int cr = corner_dr(qc), cc = corner_dc(qc);
    for (int my = 0; my < ky; ++my)
      for (int mx = 0; mx < kx; ++mx) {
        const int m = my * kx + mx;
        for (int qf = 0; qf < 4; ++qf) {
          const int fr = my + corner_dr(qf), fc = mx + corner_dc(qf);
          // x pass on both coarse rows, then y pass
          double g[2];
          for (int R = 0; R < 2; ++R) {
            const double a = (R == cr && cc == 0) ? 1.0 : 0.0;
            const double b = (R == cr && cc == 1) ? 1.0 : 0.0;
            g[R] = interp1(a, b, fc, kx);
          }
          const double v = interp1(g[0], g[1], fr, ky);
          for (int i = 0; i < d; ++i) S[(m * nk + qf * d + i) * nk + qc * d + i] = v;
        }
      }
  }
}

// G[m] = S_m^T K S_m for a fixed (nk x nk) K.
static void galerkin_table(const double* S, const double* K, int nm, int nk, double* G) {
  for (int m = 0; m < nm; ++m) {
    const double* Sm = S + (size_t)m * nk * nk;
    for (int i = 0; i < nk; ++i)
      for (int j = 0; j < nk; ++j) {
        double acc = 0.0;
        for (int p = 0; p < nk; ++p) {
          if (Sm[p * nk + i] == 0.0) continue;
          double t = 0.0;
          for (int q = 0; q < nk; ++q) t += K[p * nk + q] * Sm[q * nk + j];
          acc += Sm[p * nk + i] * t;
        }
        G[((size_t)m * nk + i) * nk + j] = acc;
      }
  }
}

constexpr int kCoarseInvMaxRows = 48;  // hierarchy rows up to which the FP32 cycle uses the coarse inverse
constexpr int kTableStride = 9 * 64;   // doubles per table (max 9 children x 8 x 8)
constexpr int kGrandStride = 81 * 64;  // doubles per grandchild table (max 81 x 8 x 8)
constexpr int kChildStencilSize = 2 * 5 * 4 * 4 * 9;  // stencil_children_kernel tables, D = 2, 9 children

// H[g] = S1_{m1}^T G[m0] S1_{m1} for the level-0 grandchild g = (m1, m0) of a level-2
// element, with G the level-0 -> 1 child tables (S0^T K S0) and S1 the level-1 -> 2
// interpolations; g is numbered as a child of a (kx0 kx1) x (ky0 ky1) coarsening, row
// my1 ky0 + my0 and column mx1 kx0 + mx0, so keff_from_density_kernel applies it.
static void grand_table(const double* S1, const double* G, int kx0, int ky0, int kx1, int ky1, int nk,
                        double* H) {
  const int KX = kx0 * kx1;
  std::vector<double> t(nk * nk);
  for (int my1 = 0; my1 < ky1; ++my1)
    for (int mx1 = 0; mx1 < kx1; ++mx1) {
      const double* Sm = S1 + (size_t)(my1 * kx1 + mx1) * nk * nk;
      for (int my0 = 0; my0 < ky0; ++my0)
        for (int mx0 = 0; mx0 < kx0; ++mx0) {
          const double* Gm = G + (size_t)(my0 * kx0 + mx0) * nk * nk;
          const int g = (my1 * ky0 + my0) * KX + (mx1 * kx0 + mx0);
          galerkin_table(Sm, Gm, 1, nk, H + (size_t)g * nk * nk);
        }
    }
}

// For 2 x 2 children (m = my * 2 + mx): true when each M_m is the mirror image of M_0,
// M_m[i][j] = sx^mx sy^my M_0[i][j] with sx = DX_i DX_j, sy = DY_i DY_j and DX / DY the
// modes' signs under the x / y reflection of the element (l1_sweep_kernel's mirror path;
// the reference's plane-stress KE and the bilinear interpolation have this symmetry).
static bool l1_mirror_classes(const double (*m)[21]) {
  double big = 0.0;
  for (int e = 0; e < 21; ++e) big = std::max(big, std::fabs(m[0][e]));
  for (int c = 1; c < 4; ++c) {
    const int mx = c & 1, my = c >> 1;
    int e = 0;
    for (int i = 0; i < 6; ++i)
      for (int j = i; j < 6; ++j, ++e) {
        const double sx = kModeDX[i] * kModeDX[j], sy = kModeDY[i] * kModeDY[j];
        const double want = (mx ? sx : 1.0) * (my ? sy : 1.0) * m[0][e];
        if (std::fabs(m[c][e] - want) > 1e-12 * big) return false;
      }
  }
  return true;
}

// M_m = T G_m T^T / 16 for the nm plane-stress child matrices G (8 x 8 each), packed as
// the upper triangle of the symmetric 6 x 6 (row-major, i <= j); mode order Gx(ux),
// Gy(uy), Gy(ux), Gx(uy), H(ux), H(uy) as modal_from_ke.  False unless T^T M_m T
// reproduces every G_m to 1e-12 of its largest entry.
static bool l1_tables(const double* G, int nm, double (*out)[21]) {
  static const double pat[3][4] = {{-1, 1, 1, -1}, {-1, -1, 1, 1}, {1, -1, 1, -1}};
  double T[6][8] = {};
  for (int k = 0; k < 4; ++k) {
    T[0][2 * k] = pat[0][k];
    T[1][2 * k + 1] = pat[1][k];
    T[2][2 * k] = pat[1][k];
    T[3][2 * k + 1] = pat[0][k];
    T[4][2 * k] = pat[2][k];
    T[5][2 * k + 1] = pat[2][k];
  }
  for (int m = 0; m < nm; ++m) {
    const double* Gm = G + (size_t)m * 64;
    double M[6][6], gmax = 0.0;
    for (int i = 0; i < 64; ++i) gmax = std::fmax(gmax, std::fabs(Gm[i]));
    for (int a = 0; a < 6; ++a)
      for (int b = 0; b < 6; ++b) {
        double s = 0.0;
        for (int i = 0; i < 8; ++i)
          for (int j = 0; j < 8; ++j) s += T[a][i] * Gm[i * 8 + j] * T[b][j];
        M[a][b] = s / 16.0;
      }
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) {
        double s = 0.0;
        for (int a = 0; a < 6; ++a)
          for (int b = 0; b < 6; ++b) s += T[a][i] * 0.5 * (M[a][b] + M[b][a]) * T[b][j];
        if (!(std::fabs(s - Gm[i * 8 + j]) <= 1e-12 * gmax)) return false;
      }
    int e = 0;
    for (int a = 0; a < 6; ++a)
      for (int b = a; b < 6; ++b) out[m][e++] = 0.5 * (M[a][b] + M[b][a]);
  }
  return true;
}

static inline char* carve(char*& p, long long& used, long long bytes) {
  const long long a = (bytes + 255) & ~255LL;
  char* r = p ? p + used : nullptr;
  used += a;
  return r;
}

long long plan_hierarchy(stt_hier_impl& h, char* base) {
  long long used = 0;
  char* p = base;
  const int d = h.d, NS = stencil_coefs(d), NK = 4 * d;
  int nx = h.nelx, ny = h.nely, L = 0;
  while (true) {
    LevelDesc& lv = h.lv[L];
    std::memset(&lv, 0, sizeof(lv));
    lv.nelx = nx;
    lv.nely = ny;
    lv.nnx = nx + 1;
    lv.nny = ny + 1;
    lv.nnode = (long long)lv.nnx * lv.nny;
    lv.ndof = lv.nnode * d;
    lv.nel = (long long)nx * ny;
    lv.rs_rho = (lv.nel + 3) & ~3LL;
    lv.kx = lv.ky = 1;
    ++L;
    if ((long long)nx * ny <= h.mce) break;
    const int kx = factor_of(nx), ky = factor_of(ny);
    if (kx == 1 && ky == 1) break;
    if (L >= kMaxLevels) break;
    lv.kx = kx;
    lv.ky = ky;
    nx /= kx;
    ny /= ky;
  }
  h.nlevels = L;
  const bool f32 = h.precision == STT_FP32;
  for (int l = 0; l < L; ++l) {
    LevelDesc& lv = h.lv[l];
    lv.fixed = (uint8_t*)carve(p, used, lv.nnode);
    if (l == 0) {
      lv.rho64 = (double*)carve(p, used, 8LL * h.hrows * lv.rs_rho);
      if (f32) lv.rho32 = (float*)carve(p, used, 4LL * h.hrows * lv.rs_rho);
      lv.rdiag64 = (double*)carve(p, used, 8LL * h.hrows * lv.ndof);
      if (f32) lv.rdiag32 = (float*)carve(p, used, 4LL * h.hrows * lv.ndof);
    }
    if (l > 0 || L == 1) {
      lv.st64 = (double*)carve(p, used, 8LL * h.hrows * NS * lv.nnode);
      if (f32 && l > 0)
        lv.st32 = (float*)carve(p, used, 4LL * h.hrows * (d == 2 ? st32_nsp<2>() : st32_nsp<1>()) * lv.nnode);
    }
  }
  // coarse factor
  {
    const LevelDesc& c = h.lv[L - 1];
    CoarseDesc& co = h.co;
    co.n = (int)c.ndof;
    co.by_col = c.nny < c.nnx ? 1 : 0;
    const int nmin = co.by_col ? c.nny : c.nnx;
    const int bw = d * (nmin + 2) - 1;  // max |P - Q| of a nonzero
    co.B = ((bw + 31) / 32) * 32;
    if (co.B < 32) co.B = 32;
    co.nb = (co.n + co.B - 1) / co.B;
    co.blocks = (double*)carve(p, used, 8LL * h.hrows * co.nb * 4 * co.B * co.B);
    // the FP32 cycle solves the coarsest level with the explicit inverse (one GEMV) while
    // the hierarchy has few rows: the GEMV streams np^2 doubles a row per cycle, the block
    // solves ~8 B^2 nb, and from about 48 rows on (one CTA a row filling the SMs) the
    // latency-bound block solves cost less than the inverse's bytes and its build
    const long long np = (long long)co.nb * co.B;
    co.inv = (f32 && co.B <= 64 && h.hrows <= kCoarseInvMaxRows) ? (double*)carve(p, used, 8LL * h.hrows * np * np)
                                                                   : nullptr;
  }
  h.tables = (double*)carve(p, used, 8LL * kMaxLevels * 3 * kTableStride);
  h.gtables = (double*)carve(p, used, 8LL * (2 * kGrandStride + kChildStencilSize));
  // level 1 is assembled straight from the level-0 densities and level 2's element
  // matrices from its level-0 grandchildren, so the element-matrix buffers start at
  // level 2 (keffB: even levels, keffA: odd levels >= 3)
  if (L > 2) h.keffB = (double*)carve(p, used, 8LL * h.hrows * h.lv[2].nel * NK * NK);
  if (L > 3) h.keffA = (double*)carve(p, used, 8LL * h.hrows * h.lv[3].nel * NK * NK);
  carve(p, used, 256);  // status word
  h.ws_bytes = used;
  return used;
}

// ---- build kernels -----------------------------------------------------------

template <typename TI, typename TO>
__global__ void convert_kernel(const TI* __restrict__ in, TO* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (TO)in[i];
}

// Row copy of the densities, with the FP32 copy written in the same pass (out32 may be null).
__global__ void copy_rows_kernel(const double* __restrict__ in, long long in_rs,
                                 double* __restrict__ out, float* __restrict__ out32, long long out_rs,
                                 long long n) {
  const int row = blockIdx.y;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = in[(size_t)row * in_rs + i];
    out[(size_t)row * out_rs + i] = v;
    if (out32) out32[(size_t)row * out_rs + i] = (float)v;
  }
}

// Coarse fixed flags: the fine flags at the collocated nodes (torch_mg.py:376).
__global__ void coarse_fixed_kernel(const uint8_t* __restrict__ ff, int fnnx, int kx, int ky,
                                    uint8_t* __restrict__ cf, int cnnx, int cnny) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= cnnx * cnny) return;
  const int r = n / cnnx, c = n - r * cnnx;
  cf[n] = ff[(size_t)(r * ky) * fnnx + c * kx];
}

// Level-1 element matrices from the fine densities: keff[E] = sum_m rho_m G_m
// (+ sum_m reaction_m GM_m) (torch_mg.py:357-366).  One thread per (E, i).
template <int D>
__global__ void keff_from_density_kernel(const double* __restrict__ rho, long long rho_rs,
                                         const double* __restrict__ reac, long long r_rs,
                                         const double* __restrict__ G,
                                         const double* __restrict__ GM, int fnelx, int kx,
                                         int ky, int cnelx, int cnel, double* __restrict__ keff) {
  constexpr int NK = 4 * D;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  if (t >= (long long)cnel * NK) return;
  const int E = (int)(t / NK), i = (int)(t - (long long)E * NK);
  const int R = E / cnelx, C = E - R * cnelx;
  const double* rr = rho + (size_t)h * rho_rs;
  double acc[NK], acc2[NK];
#pragma unroll
  for (int j = 0; j < NK; ++j) acc[j] = acc2[j] = 0.0;
  const int nm = kx * ky;
  for (int m = 0; m < nm; ++m) {
    const int my = m / kx, mx = m - my * kx;
    const size_t e = (size_t)(R * ky + my) * fnelx + (C * kx + mx);
    const double rv = __ldg(rr + e);
    const double* g = G + ((size_t)m * NK + i) * NK;
#pragma unroll
    for (int j = 0; j < NK; ++j) acc[j] = fma(rv, __ldg(g + j), acc[j]);
    if (reac) {
      const double av = __ldg(reac + (size_t)h * r_rs + e);
      const double* gm = GM + ((size_t)m * NK + i) * NK;
#pragma unroll
      for (int j = 0; j < NK; ++j) acc2[j] = fma(av, __ldg(gm + j), acc2[j]);
    }
  }
  double* out = keff + (((size_t)h * cnel + E) * NK + i) * NK;
#pragma unroll
  for (int j = 0; j < NK; ++j) out[j] = reac ? acc[j] + acc2[j] : acc[j];
}

// keff_from_density_kernel for NM = 16 grandchildren (2 x 2 coarsening twice), a warp per
// element (D = 2: lane l holds entries l and l + 32) or per two elements (D = 1: a group of
// 16 lanes per element): the NM tables live in registers, the first NM lanes of a group
// load the child densities and shuffles broadcast them, and a warp's stores are 256
// contiguous bytes.  A warp takes U element steps at once (their density loads in flight
// together).  Grid: (blocks, hierarchy rows).
template <int D, int NM, bool RD>
__global__ void __launch_bounds__(256) keff_from_density_warp_kernel(
    const double* __restrict__ rho, long long rho_rs, const double* __restrict__ reac, long long r_rs,
    const double* __restrict__ G, const double* __restrict__ GM, int fnelx, int kx, int cnelx, int cnel,
    double* __restrict__ keff) {
  constexpr int NK = 4 * D, NE = NK * NK;       // 64 or 16 entries
  constexpr int GW = NE >= 32 ? 32 : NE;        // lanes per element
  constexpr int EPL = NE / GW;                  // entries per lane
  constexpr int EPW = 32 / GW;                  // elements per warp step
  constexpr int U = 4;                          // warp steps in flight
  static_assert(NM <= GW, "the children of an element must fit its lane group");
  const int lane = threadIdx.x & 31, sub = lane / GW, gl = lane % GW;
  const int h = blockIdx.y;
  double g[NM][EPL], gm[RD ? NM : 1][EPL];
#pragma unroll
  for (int m = 0; m < NM; ++m)
#pragma unroll
    for (int k = 0; k < EPL; ++k) {
      g[m][k] = __ldg(G + (size_t)m * NE + gl + GW * k);
      if constexpr (RD) gm[m][k] = __ldg(GM + (size_t)m * NE + gl + GW * k);
    }
  const int ky = NM / kx;
  const int my = gl / kx, mx = gl - my * kx;
  const double* rr = rho + (size_t)h * rho_rs;
  const double* ar = RD ? reac + (size_t)h * r_rs : nullptr;
  double* kh = keff + (size_t)h * cnel * NE;
  const int nw = gridDim.x * (blockDim.x / 32);
  const int w0 = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  for (int base = w0 * U * EPW; base < cnel; base += nw * U * EPW) {  // uniform per warp
    double rv[U], av[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int E = base + u * EPW + sub;
      rv[u] = av[u] = 0.0;
      if (E < cnel && gl < NM) {
        const int R = E / cnelx, C = E - R * cnelx;
        const size_t fe = (size_t)(R * ky + my) * fnelx + (C * kx + mx);
        rv[u] = __ldg(rr + fe);
        if constexpr (RD) av[u] = __ldg(ar + fe);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int E = base + u * EPW + sub;
      double acc[EPL];
#pragma unroll
      for (int k = 0; k < EPL; ++k) acc[k] = 0.0;
#pragma unroll
      for (int m = 0; m < NM; ++m) {
        const double r = __shfl_sync(0xffffffffu, rv[u], sub * GW + m);
#pragma unroll
        for (int k = 0; k < EPL; ++k) acc[k] = fma(r, g[m][k], acc[k]);
        if constexpr (RD) {
          const double a = __shfl_sync(0xffffffffu, av[u], sub * GW + m);
#pragma unroll
          for (int k = 0; k < EPL; ++k) acc[k] = fma(a, gm[m][k], acc[k]);
        }
      }
      if (E < cnel) {
#pragma unroll
        for (int k = 0; k < EPL; ++k) kh[(size_t)E * NE + gl + GW * k] = acc[k];
      }
    }
  }
}

// Galerkin product of the level above: keff_c[E] = sum_m S_m^T keff_f[child m] S_m
// (torch_mg.py:367-370).  One thread per (E, i).
template <int D>
__global__ void keff_galerkin_kernel(const double* __restrict__ kf, int fnelx, int fnel,
                                     const double* __restrict__ S, int kx, int ky, int cnelx,
                                     int cnel, double* __restrict__ kc) {
  constexpr int NK = 4 * D;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  if (t >= (long long)cnel * NK) return;
  const int E = (int)(t / NK), i = (int)(t - (long long)E * NK);
  const int R = E / cnelx, C = E - R * cnelx;
  double out[NK];
#pragma unroll
  for (int j = 0; j < NK; ++j) out[j] = 0.0;
  const int nm = kx * ky;
  for (int m = 0; m < nm; ++m) {
    const int my = m / kx, mx = m - my * kx;
    const size_t e = (size_t)(R * ky + my) * fnelx + (C * kx + mx);
    const double* K = kf + ((size_t)h * fnel + e) * NK * NK;
    const double* Sm = S + (size_t)m * NK * NK;
    double tq[NK];
#pragma unroll
    for (int q = 0; q < NK; ++q) tq[q] = 0.0;
#pragma unroll
    for (int p = 0; p < NK; ++p) {
      const double s = __ldg(Sm + p * NK + i);
      if (s != 0.0) {
#pragma unroll
        for (int q = 0; q < NK; ++q) tq[q] = fma(s, __ldg(K + p * NK + q), tq[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < NK; ++q) {
      if (tq[q] == 0.0) continue;
#pragma unroll
      for (int j = 0; j < NK; ++j) out[j] = fma(tq[q], __ldg(Sm + q * NK + j), out[j]);
    }
  }
  double* o = kc + (((size_t)h * cnel + E) * NK + i) * NK;
#pragma unroll
  for (int j = 0; j < NK; ++j) o[j] = out[j];
}

// keff_galerkin_kernel for plane stress (8 x 8 element matrices), a warp per coarse
// element: per child m the child's matrix K is staged in the warp's shared tile (two
// entries a lane, 512 coalesced bytes), T = K S_m and then S_m^T T are formed two entries
// a lane (each a dot of length 8 over shared rows), and the accumulated matrix is stored
// 256 bytes at a time.  The interpolation tables S (nm x 8 x 8) sit in shared memory.
constexpr int kGalWarps = 8;

__global__ void __launch_bounds__(32 * kGalWarps) keff_galerkin_warp_kernel(
    const double* __restrict__ kf, int fnelx, int fnel, const double* __restrict__ S, int kx, int ky, int cnelx,
    int cnel, double* __restrict__ kc) {
  constexpr int NK = 8, NE = 64;
  __shared__ double Ss[9 * NE];
  __shared__ double Ks[kGalWarps][NE], Ts[kGalWarps][NE];
  const int nm = kx * ky;
  for (int t = threadIdx.x; t < nm * NE; t += blockDim.x) Ss[t] = S[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int h = blockIdx.y;
  const double* kh = kf + (size_t)h * fnel * NE;
  double* ch = kc + (size_t)h * cnel * NE;
  // this lane's two entries (i, j): e = lane and lane + 32
  const int i0 = lane >> 3, j0 = lane & 7, i1 = i0 + 4;
  // the child matrices of the warp's elements stream through two registers a lane, the
  // next child's loads in flight while the current one is multiplied
  auto child = [&](int E, int m) {
    const int R = E / cnelx, C = E - R * cnelx, my = m / kx, mx = m - my * kx;
    return kh + ((size_t)(R * ky + my) * fnelx + (C * kx + mx)) * NE;
  };
  const int E0 = blockIdx.x * kGalWarps + w, dE = gridDim.x * kGalWarps;
  double n0 = 0.0, n1 = 0.0;
  if (E0 < cnel) {
    n0 = __ldg(child(E0, 0) + lane);
    n1 = __ldg(child(E0, 0) + lane + 32);
  }
  for (int E = E0; E < cnel; E += dE) {  // uniform per warp
    double acc0 = 0.0, acc1 = 0.0;
    for (int m = 0; m < nm; ++m) {
      Ks[w][lane] = n0;
      Ks[w][lane + 32] = n1;
      // prefetch the next child (of this element, or of the warp's next element)
      const int En = m + 1 < nm ? E : E + dE, mn = m + 1 < nm ? m + 1 : 0;
      if (En < cnel) {
        n0 = __ldg(child(En, mn) + lane);
        n1 = __ldg(child(En, mn) + lane + 32);
      }
      __syncwarp();
      const double* Sm = Ss + m * NE;
      // T[p][j] = sum_q K[p][q] S_m[q][j] for (p, j) = (i0, j0) and (i1, j0)
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int q = 0; q < NK; ++q) {
        const double sq = Sm[q * NK + j0];
        t0 = fma(Ks[w][i0 * NK + q], sq, t0);
        t1 = fma(Ks[w][i1 * NK + q], sq, t1);
      }
      Ts[w][lane] = t0;
      Ts[w][lane + 32] = t1;
      __syncwarp();
      // out[i][j] += sum_p S_m[p][i] T[p][j]
#pragma unroll
      for (int pp = 0; pp < NK; ++pp) {
        const double tp = Ts[w][pp * NK + j0];
        acc0 = fma(Sm[pp * NK + i0], tp, acc0);
        acc1 = fma(Sm[pp * NK + i1], tp, acc1);
      }
      __syncwarp();  // the tiles are rewritten for the next child
    }
    double* out = ch + (size_t)E * NE;
    out[lane] = acc0;
    out[lane + 32] = acc1;
  }
}

// Element-matrix sources for the stencil assembly.// Element-matrix sources for the stencil assembly.
template <int D>
struct KeffSource {  // explicit element matrices
  const double* keff;
  int nel;
  STT_DEV double operator()(int h, int e, int p, int q) const {
    return __ldg(keff + (((size_t)h * nel + e) * (4 * D) + p) * (4 * D) + q);
  }
};
template <int D>
struct ChildSource {  // level 1: sum over the level-0 children m of rho_m G_m (+ reaction_m GM_m)
  const double* rho;
  long long rho_rs;
  const double* reac;
  long long r_rs;
  const double* G;   // [kx ky][4D][4D]
  const double* GM;
  int fnelx, kx, ky, cnelx;
  STT_DEV double operator()(int h, int e, int p, int q) const {
    constexpr int NK = 4 * D;
    const int R = e / cnelx, C = e - R * cnelx;
    const double* rr = rho + (size_t)h * rho_rs;
    double v = 0.0;
    for (int my = 0; my < ky; ++my)
      for (int mx = 0; mx < kx; ++mx) {
        const int m = my * kx + mx;
        const size_t fe = (size_t)(R * ky + my) * fnelx + (C * kx + mx);
        v = fma(__ldg(rr + fe), __ldg(G + ((size_t)m * NK + p) * NK + q), v);
        if (reac) v = fma(__ldg(reac + (size_t)h * r_rs + fe), __ldg(GM + ((size_t)m * NK + p) * NK + q), v);
      }
    return v;
  }
};

template <int D>
struct DensitySource {  // rho_e KE (+ reaction_e I / 4), level 0 used as the coarsest
  const double* rho;
  long long rho_rs;
  const double* reac;
  long long r_rs;
  KEq<D, double> ke;
  STT_DEV double operator()(int h, int e, int p, int q) const {
    double v = __ldg(rho + (size_t)h * rho_rs + e) * ke.v[p * 4 * D + q];
    if (reac) v += __ldg(reac + (size_t)h * r_rs + e) * (p == q ? 0.25 : 0.0);
    return v;
  }
};

// The FP32 copy of stencil entry (blk, i, j) of node n in row h (st32 may be null):
// node-major records of st32_nsp<D>() coefficients, or with diag32 only the centre
// block's diagonal, [nnode][D], within the same extent.
template <int D>
__device__ __forceinline__ void st32_store(float* st32, int h, long long nnode, int n, int blk, int i, int j,
                                           int diag32, double v) {
  if (!st32) return;
  float* s32 = st32 + (size_t)h * st32_nsp<D>() * nnode;
  if (!diag32) s32[(size_t)n * st32_nsp<D>() + blk * D * D + i * D + j] = (float)v;
  else if (blk == 0 && i == j) s32[(size_t)n * D + i] = (float)v;
}

// Symmetric, projected 9-point block stencil from element matrices: block (N, M)
// sums the (corner N, corner M) blocks of the elements holding both nodes, averaged
// with the transpose of (M, N) as the reference symmetrises its dense coarse matrix
// (torch_mg.py:286), with rows and columns of fixed dofs zeroed.
// st32 (may be null) receives the FP32 copy in the same pass: every entry, or with
// diag32 only the centre block's diagonal (all a level swept from the densities reads).
template <int D, typename Src>
__global__ void stencil_kernel(Src src, const uint8_t* __restrict__ fixed, int nelx, int nely,
                               double* __restrict__ st, float* __restrict__ st32, int diag32) {
  constexpr int NS = 5 * D * D;
  const int nnx = nelx + 1, nny = nely + 1;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  if (n >= nnx * nny) return;
  const long long nnode = (long long)nnx * nny;
  const int r = n / nnx, c = n - r * nnx;
  const uint8_t fN = fixed[n];
  auto elem_ok = [&](int er, int ec) { return er >= 0 && er < nely && ec >= 0 && ec < nelx; };
  // (blk, neighbour offset, list of (element offset a,b), corner of N, corner of M)
  double* out = st + (size_t)h * NS * nnode + n;
#pragma unroll
  for (int blk = 0; blk < 5; ++blk) {
    const int dr = (blk == 0 || blk == 1) ? 0 : 1;
    const int dc = blk == 0 ? 0 : (blk == 1 ? 1 : (blk == 2 ? 0 : (blk == 3 ? 1 : -1)));
    const int mr = r + dr, mc = c + dc;
    const bool m_ok = mr >= 0 && mr < nny && mc >= 0 && mc < nnx;
    const uint8_t fM = m_ok ? fixed[mr * nnx + mc] : 0;
    double A[D][D], AT[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) A[i][j] = AT[i][j] = 0.0;
    if (m_ok) {
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const int er = r - 1 + a, ec = c - 1 + b;
          if (!elem_ok(er, ec)) continue;
          // corner of M in this element, if M belongs to it
          const int ddr = mr - er, ddc = mc - ec;
          if (ddr < 0 || ddr > 1 || ddc < 0 || ddc > 1) continue;
          const int kN = corner_of(a, b);
          const int kM = ddr == 1 ? (ddc == 0 ? 0 : 1) : (ddc == 1 ? 2 : 3);
          const int e = er * nelx + ec;
#pragma unroll
          for (int i = 0; i < D; ++i)
#pragma unroll
            for (int j = 0; j < D; ++j) {
              A[i][j] += src(h, e, kN * D + i, kM * D + j);
              AT[i][j] += src(h, e, kM * D + j, kN * D + i);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        double v = (A[i][j] + AT[i][j]) / 2;
        if (((fN >> i) & 1) || ((fM >> j) & 1)) v = 0.0;
        const size_t o = (size_t)(blk * D * D + i * D + j) * nnode;
        out[o] = v;
        st32_store<D>(st32, h, nnode, n, blk, i, j, diag32, v);
      }
  }
}

// Level-1 stencil straight from the level-0 densities.  Block b (centre, E, S, SE, SW) of
// node N, entry (i, j), is a fixed linear form in the densities of the level-0 children
// of N's (up to four) level-1 elements: W[b][i, j][element position][child] =
// Gs_m[corner of N * D + i][corner of M * D + j] when the element holds both N and the
// block's neighbour M, else 0, with Gs_m = (G_m + G_m^T) / 2 the symmetrised
// S_m^T KE S_m (the reference averages its coarse matrix with its transpose,
// torch_mg.py:286).  The table sits in shared memory; a thread per node loads the
// 4 x NM child densities once and forms its 5 D^2 coefficients, rows and columns of
// fixed dofs zeroed.  RD adds the reaction's share with its own table.  DIAG: only the
// centre block's diagonal, into st32 (a level swept from the level-0 densities reads no
// other coefficient; st is not written).
template <int D, bool RD, int NM, bool DIAG = false>
__global__ void __launch_bounds__(256) stencil_children_kernel(
    const double* __restrict__ rho, long long rho_rs, const double* __restrict__ reac, long long r_rs,
    const double* __restrict__ Wg, int fnelx, int kx, int ky, const uint8_t* __restrict__ fixed, int nelx,
    int nely, double* __restrict__ st, float* __restrict__ st32, int diag32) {
  constexpr int DD = D * D, NS = 5 * DD, NW = NS * 4 * NM;
  __shared__ double W[(RD ? 2 : 1) * NW];
  for (int i = threadIdx.x; i < (RD ? 2 : 1) * NW; i += blockDim.x) W[i] = Wg[i];
  __syncthreads();
  const int nnx = nelx + 1, nny = nely + 1;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  if (n >= nnx * nny) return;
  const long long nnode = (long long)nnx * nny;
  const int r = n / nnx, c = n - r * nnx;
  const double* rr = rho + (size_t)h * rho_rs;
  const double* ar = RD ? reac + (size_t)h * r_rs : nullptr;
  double rv[4][NM], av[RD ? 4 : 1][NM];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int er = r - 1 + p / 2, ec = c - 1 + p % 2;
    const bool ok = er >= 0 && er < nely && ec >= 0 && ec < nelx;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      const int my = m / kx, mx = m - my * kx;
      const size_t fe = ok ? (size_t)(er * ky + my) * fnelx + (ec * kx + mx) : 0;
      rv[p][m] = ok ? __ldg(rr + fe) : 0.0;
      if constexpr (RD) av[p][m] = ok ? __ldg(ar + fe) : 0.0;
    }
  }
  const uint8_t fN = fixed[n];
  double* out = st + (size_t)h * NS * nnode + n;
#pragma unroll
  for (int blk = 0; blk < 5; ++blk) {
    const int dr = (blk == 0 || blk == 1) ? 0 : 1;
    const int dc = blk == 0 ? 0 : (blk == 1 ? 1 : (blk == 2 ? 0 : (blk == 3 ? 1 : -1)));
    const int mr = r + dr, mc = c + dc;
    const bool m_ok = mr >= 0 && mr < nny && mc >= 0 && mc < nnx;
    const uint8_t fM = m_ok ? fixed[mr * nnx + mc] : 0;
#pragma unroll
    for (int q = 0; q < DD; ++q) {
      const int i = q / D, j = q % D;
      if constexpr (DIAG) {
        if (blk != 0 || i != j) continue;
      }
      const double* w = W + (size_t)(blk * DD + q) * 4 * NM;
      double v = 0.0;
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int m = 0; m < NM; ++m) {
          v = fma(rv[p][m], w[p * NM + m], v);
          if constexpr (RD) v = fma(av[p][m], w[NW + p * NM + m], v);
        }
      if (!m_ok || ((fN >> i) & 1) || ((fM >> j) & 1)) v = 0.0;
      const size_t o = (size_t)(blk * DD + q) * nnode;
      if constexpr (!DIAG) out[o] = v;
      st32_store<D>(st32, h, nnode, n, blk, i, j, diag32, v);
    }
  }
}

// The table of stencil_children_kernel from the child tables G (and GM), [5 D^2][4][nm].
static void children_stencil_table(const double* G, int nm, int d, std::vector<double>& W) {
  const int nk = 4 * d, dd = d * d;
  W.assign((size_t)5 * dd * 4 * nm, 0.0);
  for (int blk = 0; blk < 5; ++blk) {
    const int dr = (blk == 0 || blk == 1) ? 0 : 1;
    const int dc = blk == 0 ? 0 : (blk == 1 ? 1 : (blk == 2 ? 0 : (blk == 3 ? 1 : -1)));
    for (int p = 0; p < 4; ++p) {
      const int a = p / 2, b = p % 2;   // element (r - 1 + a, c - 1 + b) around node (r, c)
      const int ddr = dr + 1 - a, ddc = dc + 1 - b;  // M relative to the element's top-left node
      if (ddr < 0 || ddr > 1 || ddc < 0 || ddc > 1) continue;
      const int kN = corner_of(a, b);
      const int kM = ddr == 1 ? (ddc == 0 ? 0 : 1) : (ddc == 1 ? 2 : 3);
      for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j)
          for (int m = 0; m < nm; ++m) {
            const double* Gm = G + (size_t)m * nk * nk;
            const int P = kN * d + i, Q = kM * d + j;
            W[(((size_t)blk * dd + i * d + j) * 4 + p) * nm + m] = 0.5 * (Gm[P * nk + Q] + Gm[Q * nk + P]);
          }
    }
  }
}

// Banded coarse matrix from the coarsest stencil, written into the factor's storage:
// diagonal blocks in slot 0, sub-diagonal blocks A_{k,k-1} in slot 2.  Fixed dofs get
// a unit diagonal (torch_mg.py:287-289); padding rows are identity.
template <int D>
__global__ void band_assemble_kernel(const double* __restrict__ st, const uint8_t* __restrict__ fixed,
                                     int nnx, int nny, int by_col, int B, int nb,
                                     double* __restrict__ blocks, int* __restrict__ status) {
  constexpr int NS = 5 * D * D;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  const long long nnode = (long long)nnx * nny;
  double* bh = blocks + (size_t)h * nb * 4 * B * B;
  if (n >= nnode) {
    // padding rows (beyond n dofs) get an identity diagonal
    const long long pad = n - nnode;
    const long long I = nnode * D + pad;
    if (pad >= 0 && I < (long long)nb * B) {
      const int k = (int)(I / B), ii = (int)(I % B);
      bh[((size_t)k * 4 + 0) * B * B + (size_t)ii * B + ii] = 1.0;
    }
    return;
  }
  const int r = n / nnx, c = n - r * nnx;
  auto perm = [&](int rr, int cc, int i) -> long long {
    const long long node = by_col ? (long long)cc * nny + rr : (long long)rr * nnx + cc;
    return node * D + i;
  };
  auto put = [&](long long I, long long J, double v) {
    if (I < J) {
      const long long t = I;
      I = J;
      J = t;
    }
    const int kI = (int)(I / B), kJ = (int)(J / B);
    const int ii = (int)(I % B), jj = (int)(J % B);
    if (kI == kJ)
      bh[((size_t)kI * 4 + 0) * B * B + (size_t)ii * B + jj] = v;
    else if (kI == kJ + 1)
      bh[((size_t)kI * 4 + 2) * B * B + (size_t)ii * B + jj] = v;
    else if (v != 0.0)
      atomicOr(status, 2);
  };
  const double* sn = st + (size_t)h * NS * nnode + n;
  const uint8_t fN = fixed[n];
#pragma unroll
  for (int blk = 0; blk < 5; ++blk) {
    const int dr = (blk == 0 || blk == 1) ? 0 : 1;
    const int dc = blk == 0 ? 0 : (blk == 1 ? 1 : (blk == 2 ? 0 : (blk == 3 ? 1 : -1)));
    const int mr = r + dr, mc = c + dc;
    if (mr < 0 || mr >= nny || mc < 0 || mc >= nnx) continue;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        if (blk == 0 && j > i) continue;  // centre block: lower triangle only
        double v = sn[(size_t)(blk * D * D + i * D + j) * nnode];
        if (blk == 0 && i == j && ((fN >> i) & 1)) v = 1.0;
        put(perm(r, c, i), perm(mr, mc, j), v);
      }
  }
}

// Block-banded Cholesky of one hierarchy row's coarse matrix (one CTA):
//   D_k D_k^T = A_kk - E_k E_k^T,  E_{k+1} = A_{k+1,k} D_k^{-T}.
// Stores Dinv_k = D_k^{-1} and its transpose, and E_k and its transpose, so that the
// per-cycle triangular solves are two dense GEMVs per block.
__global__ void __launch_bounds__(256) band_factor_kernel(double* __restrict__ blocks, int B,
                                                          int nb, int* __restrict__ status) {
  extern __shared__ double sm[];
  const int ld = B + 1;
  double* A = sm;            // current diagonal block, then its Cholesky factor
  double* X = A + B * ld;    // D_k^{-1}
  double* Y = X + B * ld;    // E_k (from the previous step)
  const int tid = threadIdx.x, nt = blockDim.x;
  const int h = blockIdx.x;
  double* bh = blocks + (size_t)h * nb * 4 * B * B;
  __shared__ int bad;
  if (tid == 0) bad = 0;
  for (int k = 0; k < nb; ++k) {
    double* Dk = bh + (size_t)k * 4 * B * B;
    for (int t = tid; t < B * B; t += nt) {
      const int i = t / B, j = t % B;
      const double v = Dk[(size_t)i * B + j];
      if (j <= i) A[i * ld + j] = v;
    }
    __syncthreads();
    if (k > 0) {
      for (int t = tid; t < B * B; t += nt) {
        const int i = t / B, j = t % B;
        if (j > i) continue;
        double s = 0.0;
        for (int l = 0; l < B; ++l) s = fma(Y[i * ld + l], Y[j * ld + l], s);
        A[i * ld + j] -= s;
      }
      __syncthreads();
    }
    // unblocked right-looking Cholesky, lower triangle; two barriers per column: every
    // thread forms the pivot itself, and the diagonal entry is written back during the
    // trailing update (which does not read it)
    for (int j = 0; j < B; ++j) {
      const double p = A[j * ld + j];
      const double piv = sqrt(p > 0.0 ? p : 1.0);
      for (int i = j + 1 + tid; i < B; i += nt) A[i * ld + j] /= piv;
      __syncthreads();
      if (tid == 0) {
        if (!(p > 0.0)) bad = 1;
        A[j * ld + j] = piv;
      }
      const int m = B - j - 1;
      for (int t = tid; t < m * m; t += nt) {
        const int i = j + 1 + t / m, l = j + 1 + t % m;
        if (l <= i) A[i * ld + l] = fma(-A[i * ld + j], A[l * ld + j], A[i * ld + l]);
      }
      __syncthreads();
    }
    // X = A^{-1} by forward substitution, a quad of threads per column: the four split
    // each row's dot product and combine it by shuffles.  Loop bounds are uniform over the
    // warp (the shuffles need every lane); lanes without a column do no arithmetic.
    {
      const int q = tid & 3;
      for (int c0 = 0; c0 < B; c0 += nt / 4) {
        const int c = c0 + tid / 4;
        const bool col = c < B;
        if (col && q == 0) {
          for (int i = 0; i < c; ++i) X[i * ld + c] = 0.0;
          X[c * ld + c] = 1.0 / A[c * ld + c];
        }
        __syncwarp();
        for (int i = c0 + 1; i < B; ++i) {
          double s = 0.0;
          if (col && i > c)
            for (int l = c + q; l < i; l += 4) s = fma(A[i * ld + l], X[l * ld + c], s);
          s += __shfl_xor_sync(0xffffffffu, s, 1);
          s += __shfl_xor_sync(0xffffffffu, s, 2);
          if (col && i > c && q == 0) X[i * ld + c] = -s / A[i * ld + i];
          __syncwarp();
        }
      }
    }
    __syncthreads();
    for (int t = tid; t < B * B; t += nt) {
      const int i = t / B, j = t % B;
      Dk[(size_t)i * B + j] = X[i * ld + j];                        // Dinv
      Dk[(size_t)B * B + (size_t)i * B + j] = X[j * ld + i];        // Dinv^T
    }
    if (k + 1 < nb) {
      double* Dn = bh + (size_t)(k + 1) * 4 * B * B;
      // A_{k+1,k} into A's storage (the factor is no longer needed)
      for (int t = tid; t < B * B; t += nt) {
        const int i = t / B, j = t % B;
        A[i * ld + j] = Dn[(size_t)2 * B * B + (size_t)i * B + j];
      }
      __syncthreads();
      // E = A_{k+1,k} X^T: E[i][j] = sum_{l <= j} A[i][l] X[j][l]
      for (int t = tid; t < B * B; t += nt) {
        const int i = t / B, j = t % B;
        double s = 0.0;
        for (int l = 0; l <= j; ++l) s = fma(A[i * ld + l], X[j * ld + l], s);
        Y[i * ld + j] = s;
      }
      __syncthreads();
      for (int t = tid; t < B * B; t += nt) {
        const int i = t / B, j = t % B;
        Dn[(size_t)2 * B * B + (size_t)i * B + j] = Y[i * ld + j];  // E
        Dn[(size_t)3 * B * B + (size_t)i * B + j] = Y[j * ld + i];  // E^T
      }
    }
    __syncthreads();
  }
  if (tid == 0 && bad) atomicOr(status, 1);
}

// 16-byte asynchronous global -> shared copies (sm_80+ cp.async), for prefetching the
// next blocks while the current one factors.
STT_DEV void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
STT_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
STT_DEV void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The same factorisation for B = 16 NA (NA = 2, 4), 256 threads as a 16 x 16 grid:
//   * thread (ty, tx) owns the strided tile of entries (ty + 16 a, tx + 16 b), a, b < NA,
//     of every B x B product, so each shared-memory load feeds NA multiply-adds (a warp
//     reads 2 rows of one operand, broadcast, and 16 rows of the other at a stride of
//     B + 1 doubles, conflict-free);
//   * the Cholesky takes two columns per pair of barriers: every thread forms both
//     pivots and the two scaled columns of its rows and columns in registers (column
//     j + 1 updated by column j on the fly), then applies the rank-2 trailing update;
//   * A_{k+1,k+1} and A_{k+1,k} are copied into staging buffers with cp.async while
//     block k factors; the Schur update and E = A_{k+1,k} X^T read them from there.
// Upper triangles of the work arrays carry harmless values (only lower triangles are
// read); X = D^{-1} keeps exact zeros above its diagonal.
template <int NA>
__global__ void __launch_bounds__(256) band_factor_tiled_kernel(double* __restrict__ blocks, int nb,
                                                                int* __restrict__ status) {
  constexpr int B = 16 * NA, ld = B + 1;
  extern __shared__ __align__(16) double sm[];
  double* P0 = sm;           // staged A_{k,k} (B x B, dense rows)
  double* P1 = P0 + B * B;   // staged A_{k+1,k}
  double* A = P1 + B * B;    // current diagonal block, then its Cholesky factor (ld)
  double* X = A + B * ld;    // D_k^{-1}
  double* Y = X + B * ld;    // E_k
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  double* bh = blocks + (size_t)blockIdx.x * nb * 4 * B * B;
  __shared__ int bad;
  __shared__ double rp[B];  // reciprocals of the current block's pivots
  if (tid == 0) bad = 0;
  auto stage = [&](double* dst, const double* src) {
    for (int t = tid; t < B * B / 2; t += 256) cp_async16(dst + 2 * t, src + 2 * t);
  };
  stage(P0, bh);
  cp_async_commit();
  for (int k = 0; k < nb; ++k) {
    double* Dk = bh + (size_t)k * 4 * B * B;
    cp_async_wait_all();
    __syncthreads();
    // A = A_kk - E_k E_k^T (k > 0)
    {
      double acc[NA][NA];
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) acc[a][b] = 0.0;
      if (k > 0) {
#pragma unroll 4
        for (int m = 0; m < B; ++m) {
          double yi[NA], yl[NA];
#pragma unroll
          for (int a = 0; a < NA; ++a) yi[a] = Y[(ty + 16 * a) * ld + m];
#pragma unroll
          for (int b = 0; b < NA; ++b) yl[b] = Y[(tx + 16 * b) * ld + m];
#pragma unroll
          for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int b = 0; b < NA; ++b) acc[a][b] = fma(yi[a], yl[b], acc[a][b]);
        }
      }
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) {
          const int i = ty + 16 * a, l = tx + 16 * b;
          A[i * ld + l] = P0[i * B + l] - acc[a][b];
        }
    }
    __syncthreads();  // P0 consumed, A complete
    if (k + 1 < nb) {
      double* Dn = bh + (size_t)(k + 1) * 4 * B * B;
      stage(P0, Dn);                    // A_{k+1,k+1}
      stage(P1, Dn + (size_t)2 * B * B);  // A_{k+1,k}
      cp_async_commit();
    }
    // Cholesky, a panel of four columns per step: every thread factors the 4 x 4 pivot
    // block (one rsqrt a pivot, L_jj = t rsqrt(t), its reciprocal kept for the
    // substitution), then the panel entries of its rows and a rank-4 update
    for (int j = 0; j < B; j += 4) {
      double a[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q <= p; ++q) a[p][q] = A[(j + p) * ld + j + q];
      double l[4][4], r[4];
      bool ok = true;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double t = a[q][q];
#pragma unroll
        for (int m = 0; m < q; ++m) t = fma(-l[q][m], l[q][m], t);
        ok = ok && t > 0.0;
        const double tt = t > 0.0 ? t : 1.0;
        r[q] = rsqrt(tt);
        l[q][q] = tt * r[q];
#pragma unroll
        for (int p = q + 1; p < 4; ++p) {
          double v = a[p][q];
#pragma unroll
          for (int m = 0; m < q; ++m) v = fma(-l[p][m], l[q][m], v);
          l[p][q] = v * r[q];
        }
      }
      // the panel columns of rows i (this thread's rows) and of rows c (its columns)
      auto panel = [&](int i, double (&cv)[4]) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double v = 0.0;
          if (i > j + q) {
            v = A[i * ld + j + q];
#pragma unroll
            for (int m = 0; m < q; ++m) v = fma(-cv[m], l[q][m], v);
            v *= r[q];
          }
          cv[q] = v;
        }
      };
      double ci[NA][4], cl[NA][4];
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2) panel(ty + 16 * a2, ci[a2]);
#pragma unroll
      for (int b = 0; b < NA; ++b) panel(tx + 16 * b, cl[b]);
      __syncthreads();
      if (tx == 0) {
#pragma unroll
        for (int a2 = 0; a2 < NA; ++a2) {
          const int i = ty + 16 * a2;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (i > j + q) A[i * ld + j + q] = ci[a2][q];
        }
      }
      if (tid == 0) {
        if (!ok) bad = 1;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          A[(j + q) * ld + j + q] = l[q][q];
          rp[j + q] = r[q];
        }
      }
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
        for (int b = 0; b < NA; ++b) {
          const int i = ty + 16 * a2, c = tx + 16 * b;
          if (i > j + 3 && c > j + 3) {
            double v = A[i * ld + c];
#pragma unroll
            for (int q = 0; q < 4; ++q) v = fma(-ci[a2][q], cl[b][q], v);
            A[i * ld + c] = v;
          }
        }
      __syncthreads();
    }
    // X = A^{-1}: forward substitution with the pivots' reciprocals, a quad of threads a
    // column, each thread's share of a dot product in two independent chains
    {
      const int q = tid & 3;
      for (int c0 = 0; c0 < B; c0 += 64) {
        const int c = c0 + tid / 4;
        const bool col = c < B;
        if (col && q == 0) {
          for (int i = 0; i < c; ++i) X[i * ld + c] = 0.0;
          X[c * ld + c] = rp[c];
        }
        __syncwarp();
        for (int i = c0 + 1; i < B; ++i) {
          double s0 = 0.0, s1 = 0.0;
          if (col && i > c) {
            int l2 = c + q;
            for (; l2 + 4 < i; l2 += 8) {
              s0 = fma(A[i * ld + l2], X[l2 * ld + c], s0);
              s1 = fma(A[i * ld + l2 + 4], X[(l2 + 4) * ld + c], s1);
            }
            if (l2 < i) s0 = fma(A[i * ld + l2], X[l2 * ld + c], s0);
          }
          double sacc = s0 + s1;
          sacc += __shfl_xor_sync(0xffffffffu, sacc, 1);
          sacc += __shfl_xor_sync(0xffffffffu, sacc, 2);
          if (col && i > c && q == 0) X[i * ld + c] = -sacc * rp[i];
          __syncwarp();
        }
      }
    }
    __syncthreads();
    for (int t = tid; t < B * B; t += 256) {
      const int i = t / B, j = t % B;
      Dk[t] = X[i * ld + j];                  // Dinv
      Dk[(size_t)B * B + t] = X[j * ld + i];  // Dinv^T
    }
    if (k + 1 < nb) {
      double* Dn = bh + (size_t)(k + 1) * 4 * B * B;
      cp_async_wait_all();
      __syncthreads();  // P1 (and P0) landed for every thread
      // E = A_{k+1,k} X^T (X is zero above its diagonal)
      double acc[NA][NA];
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) acc[a][b] = 0.0;
#pragma unroll 4
      for (int l = 0; l < B; ++l) {
        double ai[NA], xj[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) ai[a] = P1[(ty + 16 * a) * B + l];
#pragma unroll
        for (int b = 0; b < NA; ++b) xj[b] = X[(tx + 16 * b) * ld + l];
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int b = 0; b < NA; ++b) acc[a][b] = fma(ai[a], xj[b], acc[a][b]);
      }
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) {
          const int i = ty + 16 * a, j = tx + 16 * b;
          Y[i * ld + j] = acc[a][b];
          Dn[(size_t)2 * B * B + i * B + j] = acc[a][b];  // E
        }
      __syncthreads();
      for (int t = tid; t < B * B; t += 256) Dn[(size_t)3 * B * B + t] = Y[(t % B) * ld + t / B];  // E^T
    }
  }
  if (tid == 0 && bad) atomicOr(status, 1);
}

}  // namespace stt

using namespace stt;

static int grid1(long long n, int bs = 256) {
  long long g = (n + bs - 1) / bs;
  if (g > 1 << 30) g = 1 << 30;
  return (int)(g < 1 ? 1 : g);
}

extern "C" long long stt_hier_workspace_bytes(int d, int nelx, int nely, int hrows,
                                              int max_coarse_elements, int precision) {
  if ((d != 1 && d != 2) || nelx <= 0 || nely <= 0 || hrows <= 0) return -1;
  stt_hier_impl h{};
  h.d = d;
  h.nelx = nelx;
  h.nely = nely;
  h.hrows = hrows;
  h.precision = precision;
  h.mce = max_coarse_elements;
  return plan_hierarchy(h, nullptr);
}

// Level 1's stencil: keff[E] = sum_m rho_m G_m (+ reaction), assembled from the level-0
// densities (level 1's flags must be built).
// Level 1's stencil from the level-0 densities.  mode 0: the FP64 stencil and the FP32 copy
// the cycle reads (all of it, or with h->l1 the centre diagonal); mode 1: only that FP32
// diagonal (an FP32 hierarchy swept from the densities: nothing in its cycle reads the
// FP64 stencil); mode 2: only the FP64 stencil (assembled on first use after mode 1).
template <int D>
static int level1_stencil(stt_hier* h, const double* reaction, long long r_rs, cudaStream_t st, int mode = 0) {
  const int H = h->hrows;
  const bool f32 = h->precision == STT_FP32;
  const LevelDesc& f = h->lv[0];
  LevelDesc& c = h->lv[1];
  const double* S = h->tables;  // the level 0 -> 1 transition's tables
  const int nm = f.kx * f.ky;
  float* s32 = (f32 && mode != 2) ? c.st32 : nullptr;
  if (mode == 1) {
    if (!(h->l1 && f32 && !reaction && (nm == 4 || nm == 6 || nm == 9)))
      return set_error(STT_ERR_INVALID, "level-1 diagonal alone: not a level swept from the densities");
#define STT_CHILD_DG(NM)                                                                                        \
  stencil_children_kernel<D, false, NM, true><<<dim3(grid1(c.nnode), H), 256, 0, st>>>(                         \
      f.rho64, f.rs_rho, nullptr, 0, h->gtables + 2 * kGrandStride, f.nelx, f.kx, f.ky, c.fixed, c.nelx, c.nely, \
      nullptr, s32, 1)
    if (nm == 4) STT_CHILD_DG(4);
    else if (nm == 6) STT_CHILD_DG(6);
    else STT_CHILD_DG(9);
#undef STT_CHILD_DG
    return check_launch("level-1 diagonal");
  }
  if (nm == 4 || nm == 6 || nm == 9) {
#define STT_CHILD_ST(RD, NM)                                                                          \
  stencil_children_kernel<D, RD, NM><<<dim3(grid1(c.nnode), H), 256, 0, st>>>(                        \
      f.rho64, f.rs_rho, reaction, r_rs, h->gtables + 2 * kGrandStride, f.nelx, f.kx, f.ky, c.fixed, \
      c.nelx, c.nely, c.st64, s32, h->l1)
    if (reaction) {
      if (nm == 4) STT_CHILD_ST(true, 4);
      else if (nm == 6) STT_CHILD_ST(true, 6);
      else STT_CHILD_ST(true, 9);
    } else {
      if (nm == 4) STT_CHILD_ST(false, 4);
      else if (nm == 6) STT_CHILD_ST(false, 6);
      else STT_CHILD_ST(false, 9);
    }
#undef STT_CHILD_ST
  } else {  // a single coarsening direction (factor 1 in the other)
    stencil_kernel<D, ChildSource<D>><<<dim3(grid1(c.nnode), H), 256, 0, st>>>(
        ChildSource<D>{f.rho64, f.rs_rho, reaction, r_rs, S + kTableStride, S + 2 * kTableStride, f.nelx,
                       f.kx, f.ky, c.nelx},
        c.fixed, c.nelx, c.nely, c.st64, s32, 0);
  }
  return check_launch("level-1 stencil");
}

template <int D>
static int build_levels(stt_hier* h, const double* rho, long long rho_rs, const double* reaction,
                        long long r_rs, const uint8_t* fixed, cudaStream_t st, bool defer_l1) {
  constexpr int NK = 4 * D, NS = 5 * D * D;
  const int H = h->hrows;
  LevelDesc& l0 = h->lv[0];
  // level 0: copies of the densities, the lumped reaction diagonal, the flags
  const bool f32 = h->precision == STT_FP32;
  copy_rows_kernel<<<dim3(grid1(l0.nel), H), 256, 0, st>>>(rho, rho_rs, l0.rho64, f32 ? l0.rho32 : nullptr,
                                                           l0.rs_rho, l0.nel);
  if (reaction)  // (without a reaction nothing reads the diagonal)
    STT_TRY(stt_lumped_reaction(D, h->nelx, h->nely, H, reaction, r_rs, l0.rdiag64, l0.ndof,
                                (stt_stream_t)st));
  if (fixed)
    STT_TRY(check_cuda(cudaMemcpyAsync(l0.fixed, fixed, l0.nnode, cudaMemcpyDeviceToDevice, st), "copy fixed"));
  else
    STT_TRY(check_cuda(cudaMemsetAsync(l0.fixed, 0, l0.nnode, st), "memset"));
  if (f32 && reaction)
    convert_kernel<double, float><<<grid1(H * l0.ndof), 256, 0, st>>>(l0.rdiag64, l0.rdiag32, H * l0.ndof);
  STT_TRY(check_launch("level0 copies"));

  // tables: per transition S, and G/GM for the first
  std::vector<double> tab((size_t)kMaxLevels * 3 * kTableStride, 0.0);
  for (int l = 0; l + 1 < h->nlevels; ++l) {
    double* S = &tab[(size_t)l * 3 * kTableStride];
    child_interp(h->lv[l].kx, h->lv[l].ky, D, S);
    if (l == 0) {
      double ME[64] = {0};
      for (int i = 0; i < NK; ++i) ME[i * NK + i] = 0.25;
      galerkin_table(S, h->KE, h->lv[0].kx * h->lv[0].ky, NK, S + kTableStride);
      galerkin_table(S, ME, h->lv[0].kx * h->lv[0].ky, NK, S + 2 * kTableStride);
    }
  }
  STT_TRY(check_cuda(cudaMemcpyAsync(h->tables, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, st), "tables"));
  // level 1 from the level-0 densities: its element matrices are sum_m rho_m G_m, and each
  // G_m = S_m^T KE S_m annihilates the coarse translations, so G_m = T^T M_m T in the
  // bilinear edge modes (q4.cuh); kept when M_m rebuilds G_m to 1e-12 (plane stress, no
  // reaction, 2 or 3 children a direction, level 1 not the coarsest)
  h->l1 = 0;
  h->l1par = 0;
  if (D == 2 && h->modal && !reaction && h->nlevels > 2 && h->lv[0].kx >= 2 && h->lv[0].ky >= 2)
    h->l1 = l1_tables(&tab[kTableStride], h->lv[0].kx * h->lv[0].ky, h->l1m) ? 1 : 0;
  if (h->l1 && h->lv[0].kx == 2 && h->lv[0].ky == 2) h->l1par = l1_mirror_classes(h->l1m) ? 1 : 0;

  // level 1's stencil tables (after the two grandchild tables)
  if (h->nlevels > 1) {
    const int nm = h->lv[0].kx * h->lv[0].ky;
    std::vector<double> W, WM;
    children_stencil_table(&tab[kTableStride], nm, D, W);
    children_stencil_table(&tab[2 * kTableStride], nm, D, WM);
    W.insert(W.end(), WM.begin(), WM.end());
    STT_TRY(check_cuda(cudaMemcpyAsync(h->gtables + 2 * kGrandStride, W.data(), W.size() * 8,
                                       cudaMemcpyHostToDevice, st), "children stencil tables"));
  }
  // level 2's element matrices from the level-0 grandchildren
  if (h->nlevels > 2) {
    const LevelDesc& f0 = h->lv[0];
    const LevelDesc& f1 = h->lv[1];
    std::vector<double> gt((size_t)2 * kGrandStride, 0.0);
    const double* S1 = &tab[(size_t)1 * 3 * kTableStride];
    grand_table(S1, &tab[kTableStride], f0.kx, f0.ky, f1.kx, f1.ky, NK, gt.data());
    grand_table(S1, &tab[2 * kTableStride], f0.kx, f0.ky, f1.kx, f1.ky, NK, gt.data() + kGrandStride);
    STT_TRY(check_cuda(cudaMemcpyAsync(h->gtables, gt.data(), gt.size() * 8, cudaMemcpyHostToDevice, st),
                       "grandchild tables"));
  }
  const double* kprev = nullptr;
  for (int l = 1; l < h->nlevels; ++l) {
    const LevelDesc& f = h->lv[l - 1];
    LevelDesc& c = h->lv[l];
    const double* S = h->tables + (size_t)(l - 1) * 3 * kTableStride;
    coarse_fixed_kernel<<<grid1(c.nnode), 256, 0, st>>>(f.fixed, f.nnx, f.kx, f.ky, c.fixed, c.nnx, c.nny);
    if (l == 1) {
      // level 1's stencil feeds no coarser level (level 2 is built from the level-0
      // densities): with more than two levels it is assembled after the coarse
      // factorisation has started (level1_stencil), so that it runs beside it
      if (!defer_l1 || h->nlevels <= 2) STT_TRY((level1_stencil<D>(h, reaction, r_rs, st)));
    } else {
      double* kc = (l % 2 == 0) ? h->keffB : h->keffA;
      const dim3 g(grid1(c.nel * NK), H);
      if (l == 2) {
        const LevelDesc& f0 = h->lv[0];
        const int KX = f0.kx * f.kx, KY = f0.ky * f.ky;
        if (KX * KY == 16) {
          // about four resident blocks' worth a row, at least one warp step per warp
          const long long per_block = 8LL * 4 * (D == 2 ? 1 : 2);  // elements a block takes per step
          const long long want = std::max<long long>(1, 148LL * 4 / H);
          const dim3 kg((unsigned)std::min<long long>(want, (c.nel + per_block - 1) / per_block), H);
          if (reaction)
            keff_from_density_warp_kernel<D, 16, true><<<kg, 256, 0, st>>>(
                l0.rho64, l0.rs_rho, reaction, r_rs, h->gtables, h->gtables + kGrandStride, f0.nelx, KX, c.nelx,
                (int)c.nel, kc);
          else
            keff_from_density_warp_kernel<D, 16, false><<<kg, 256, 0, st>>>(
                l0.rho64, l0.rs_rho, nullptr, 0, h->gtables, nullptr, f0.nelx, KX, c.nelx, (int)c.nel, kc);
        } else {
          keff_from_density_kernel<D><<<g, 256, 0, st>>>(l0.rho64, l0.rs_rho, reaction, r_rs, h->gtables,
                                                         h->gtables + kGrandStride, f0.nelx, KX, KY, c.nelx,
                                                         (int)c.nel, kc);
        }
      } else {
        if (D == 2) {
          const long long want = std::max<long long>(1, 148LL * 8 / H);
          const dim3 gw((unsigned)std::min<long long>(want, (c.nel + kGalWarps - 1) / kGalWarps), H);
          keff_galerkin_warp_kernel<<<gw, 32 * kGalWarps, 0, st>>>(kprev, f.nelx, (int)f.nel, S, f.kx, f.ky, c.nelx,
                                                                   (int)c.nel, kc);
        } else {
          keff_galerkin_kernel<D><<<g, 256, 0, st>>>(kprev, f.nelx, (int)f.nel, S, f.kx, f.ky, c.nelx,
                                                     (int)c.nel, kc);
        }
      }
      stencil_kernel<D, KeffSource<D>><<<dim3(grid1(c.nnode), H), 256, 0, st>>>(
          KeffSource<D>{kc, (int)c.nel}, c.fixed, c.nelx, c.nely, c.st64, f32 ? c.st32 : nullptr, 0);
      kprev = kc;
    }
    STT_TRY(check_launch("galerkin level"));
  }
  LevelDesc& cl = h->lv[h->nlevels - 1];
  if (h->nlevels == 1) {
    KEq<D, double> ke;
    for (int i = 0; i < NK * NK; ++i) ke.v[i] = h->KE[i];
    stencil_kernel<D, DensitySource<D>><<<dim3(grid1(cl.nnode), H), 256, 0, st>>>(
        DensitySource<D>{l0.rho64, l0.rs_rho, reaction, r_rs, ke}, cl.fixed, cl.nelx, cl.nely, cl.st64, nullptr,
        0);
  }
  return STT_OK;
}

// The explicit inverse of the coarsest matrix from its block-bidiagonal Cholesky factor
// (for the FP32 cycle, whose coarse solve is then one GEMV instead of 2 nb dependent
// block steps).  CTA (kc, h) solves A X = I for the B columns of block kc: forward
// Y_k = Dinv_k (I_k - E_k Y_{k-1}) from block kc on (Y is zero above it), then backward
// X_k = Dinv_k^T (Y_k - E_{k+1}^T X_{k+1}); Y is parked in the output rows it precedes.
// Same arithmetic as coarse_solve_kernel, so the GEMV's result matches the block solve
// to the conditioning of the coarse matrix.  B <= 64 (three B x B FP64 tiles in shared
// memory).
__global__ void __launch_bounds__(256) coarse_inverse_kernel(const double* __restrict__ blocks, int B, int nb,
                                                             double* __restrict__ inv) {
  extern __shared__ double sm[];
  double* Y = sm;              // the current block of the solution, B x B (row-major)
  double* R = Y + B * B;       // right-hand side of the step
  double* M = R + B * B;       // the step's matrix
  const int kc = blockIdx.x, h = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const long long np = (long long)nb * B;
  const double* bh = blocks + (size_t)h * nb * 4 * B * B;
  double* ih = inv + (size_t)h * np * np;
  auto load = [&](const double* src, double* dst) {
    for (int t = tid; t < B * B; t += nt) dst[t] = src[t];
  };
  // dst = A src (all B x B); A from shared memory
  auto mm = [&](const double* A, const double* src, double* dst, double sign) {
    for (int t = tid; t < B * B; t += nt) {
      const int i = t / B, j = t % B;
      double acc = 0.0;
      for (int l = 0; l < B; ++l) acc = fma(A[i * B + l], src[l * B + j], acc);
      dst[t] = sign * acc;
    }
  };
  auto park = [&](int k, const double* src) {  // rows of block k, columns of block kc
    for (int t = tid; t < B * B; t += nt) {
      const int i = t / B, j = t % B;
      ih[((size_t)k * B + i) * np + (size_t)kc * B + j] = src[t];
    }
  };
  // forward
  for (int k = kc; k < nb; ++k) {
    if (k == kc) {
      for (int t = tid; t < B * B; t += nt) R[t] = (t / B == t % B) ? 1.0 : 0.0;
    } else {
      load(bh + ((size_t)k * 4 + 2) * B * B, M);  // E_k
      __syncthreads();
      mm(M, Y, R, -1.0);
    }
    __syncthreads();
    load(bh + ((size_t)k * 4 + 0) * B * B, M);  // Dinv_k
    __syncthreads();
    mm(M, R, Y, 1.0);
    __syncthreads();
    park(k, Y);
    __syncthreads();
  }
  // backward (Y holds X_{k+1} after each step)
  for (int k = nb - 1; k >= 0; --k) {
    for (int t = tid; t < B * B; t += nt) {
      const int i = t / B, j = t % B;
      R[t] = k >= kc ? ih[((size_t)k * B + i) * np + (size_t)kc * B + j] : 0.0;
    }
    if (k < nb - 1) {
      __syncthreads();
      load(bh + ((size_t)(k + 1) * 4 + 3) * B * B, M);  // E_{k+1}^T
      __syncthreads();
      for (int t = tid; t < B * B; t += nt) {
        const int i = t / B, j = t % B;
        double acc = 0.0;
        for (int l = 0; l < B; ++l) acc = fma(M[i * B + l], Y[l * B + j], acc);
        R[t] -= acc;
      }
    }
    __syncthreads();
    load(bh + ((size_t)k * 4 + 1) * B * B, M);  // Dinv_k^T
    __syncthreads();
    mm(M, R, Y, 1.0);
    __syncthreads();
    park(k, Y);
    __syncthreads();
  }
}

// coarse_inverse_kernel for B = 16 NA (NA = 2, 4) with register-tiled products (thread
// (ty, tx) owns entries (ty + 16 a, tx + 16 b), as band_factor_tiled_kernel), computing only
// the block rows k >= kc of column block kc: A^{-1} is symmetric, so coarse_mirror_kernel
// fills the blocks above the diagonal from their transposes afterwards.
template <int NA>
__global__ void __launch_bounds__(256) coarse_inverse_tiled_kernel(const double* __restrict__ blocks, int nb,
                                                                   double* __restrict__ inv) {
  constexpr int B = 16 * NA, ld = B + 1;
  extern __shared__ double sm[];
  double* Y = sm;           // the current block of the solution (ld)
  double* R = Y + B * ld;   // right-hand side of the step
  double* M = R + B * ld;   // the step's matrix
  const int kc = blockIdx.x, h = blockIdx.y;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const long long np = (long long)nb * B;
  const double* bh = blocks + (size_t)h * nb * 4 * B * B;
  double* ih = inv + (size_t)h * np * np;
  auto load = [&](const double* src, double* dst) {
    for (int t = tid; t < B * B; t += 256) dst[(t / B) * ld + t % B] = src[t];
  };
  // acc = A src over this thread's tile
  auto mm = [&](const double* A, const double* src, double (&acc)[NA][NA]) {
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NA; ++b) acc[a][b] = 0.0;
#pragma unroll 4
    for (int l = 0; l < B; ++l) {
      double ai[NA], sj[NA];
#pragma unroll
      for (int a = 0; a < NA; ++a) ai[a] = A[(ty + 16 * a) * ld + l];
#pragma unroll
      for (int b = 0; b < NA; ++b) sj[b] = src[l * ld + tx + 16 * b];
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) acc[a][b] = fma(ai[a], sj[b], acc[a][b]);
    }
  };
  auto park_ptr = [&](int k, int i, int j) { return ih + ((size_t)k * B + i) * np + (size_t)kc * B + j; };
  double acc[NA][NA];
  // forward: Y_k = Dinv_k (I_k - E_k Y_{k-1}), k = kc .. nb - 1
  for (int k = kc; k < nb; ++k) {
    if (k == kc) {
      for (int t = tid; t < B * B; t += 256) R[(t / B) * ld + t % B] = (t / B == t % B) ? 1.0 : 0.0;
    } else {
      load(bh + ((size_t)k * 4 + 2) * B * B, M);  // E_k
      __syncthreads();
      mm(M, Y, acc);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) R[(ty + 16 * a) * ld + tx + 16 * b] = -acc[a][b];
    }
    __syncthreads();
    load(bh + ((size_t)k * 4 + 0) * B * B, M);  // Dinv_k
    __syncthreads();
    mm(M, R, acc);
    __syncthreads();  // everyone has read Y (the E_k product) and R
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NA; ++b) {
        const int i = ty + 16 * a, j = tx + 16 * b;
        Y[i * ld + j] = acc[a][b];
        *park_ptr(k, i, j) = acc[a][b];
      }
    __syncthreads();
  }
  // backward: X_k = Dinv_k^T (Y_k - E_{k+1}^T X_{k+1}), k = nb - 1 .. kc (Y holds X_{k+1})
  for (int k = nb - 1; k >= kc; --k) {
    double rv[NA][NA];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NA; ++b) rv[a][b] = *park_ptr(k, ty + 16 * a, tx + 16 * b);
    if (k < nb - 1) {
      load(bh + ((size_t)(k + 1) * 4 + 3) * B * B, M);  // E_{k+1}^T
      __syncthreads();
      mm(M, Y, acc);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NA; ++b) rv[a][b] -= acc[a][b];
    }
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NA; ++b) R[(ty + 16 * a) * ld + tx + 16 * b] = rv[a][b];
    __syncthreads();
    load(bh + ((size_t)k * 4 + 1) * B * B, M);  // Dinv_k^T
    __syncthreads();
    mm(M, R, acc);
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NA; ++b) {
        const int i = ty + 16 * a, j = tx + 16 * b;
        Y[i * ld + j] = acc[a][b];
        *park_ptr(k, i, j) = acc[a][b];
      }
    __syncthreads();
  }
}

// inv[r][c] = inv[c][r] for the block rows above the diagonal block (row block < column
// block), a 32 x 32 tile through shared memory per CTA (reads and writes coalesced).
// Grid: (np / 32, np / 32, rows); tiles wholly below the block diagonal return at once.
__global__ void __launch_bounds__(256) coarse_mirror_kernel(double* __restrict__ inv, int B, long long np) {
  __shared__ double tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;  // destination tile (rows r0.., cols c0..)
  if (r0 / B >= (c0 + 31) / B) return;                    // no destination entry above the block diagonal
  double* ih = inv + (size_t)blockIdx.z * np * np;
  for (int j = threadIdx.y; j < 32; j += 8) {  // source rows c0 + j, columns r0 + threadIdx.x
    const long long sr = c0 + j, sc = r0 + threadIdx.x;
    tile[j][threadIdx.x] = (sr < np && sc < np) ? ih[sr * np + sc] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const long long r = r0 + i, c = c0 + threadIdx.x;
    if (r < np && c < np && r / B < c / B) ih[r * np + c] = tile[threadIdx.x][i];
  }
}

// The dynamic shared-memory ceiling of the coarse kernels, raised once per device to the// The dynamic shared-memory ceiling of the coarse kernels, raised once per device to the
// device's opt-in maximum.  (Setting it per call to the call's own size raced between
// host threads building hierarchies of different block sizes: a launch could meet
// another thread's smaller ceiling and fail.)
static int allow_large_smem() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  STT_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return STT_OK;
  int max_optin = 0;
  STT_TRY(check_cuda(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                     "smem attribute"));
  // the ceiling counts the kernel's static shared memory too
  auto raise_to = [&](const void* fn) -> int {
    cudaFuncAttributes fa;
    STT_TRY(check_cuda(cudaFuncGetAttributes(&fa, fn), "function attributes"));
    return check_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           max_optin - (int)fa.sharedSizeBytes), "smem attr");
  };
  STT_TRY(raise_to((const void*)band_factor_kernel));
  STT_TRY(raise_to((const void*)band_factor_tiled_kernel<2>));
  STT_TRY(raise_to((const void*)band_factor_tiled_kernel<4>));
  STT_TRY(raise_to((const void*)coarse_inverse_kernel));
  STT_TRY(raise_to((const void*)coarse_inverse_tiled_kernel<2>));
  STT_TRY(raise_to((const void*)coarse_inverse_tiled_kernel<4>));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return STT_OK;
}

// Pool of coarse-factorisation streams and events (creating a stream per hierarchy would
// cost more than the overlap gains). The side streams have the highest priority: the
// factorisation is on the critical path of the first coarse solve, and its few CTAs
// should not wait behind the caller's wide kernels.
static std::mutex g_sync_mu;
static std::vector<CoarseSync*> g_sync_free;

static int acquire_sync(CoarseSync** out) {
  int dev = 0;
  STT_TRY(check_cuda(cudaGetDevice(&dev), "get device"));
  {
    std::lock_guard<std::mutex> lock(g_sync_mu);
    for (size_t i = 0; i < g_sync_free.size(); ++i)
      if (g_sync_free[i]->device == dev) {
        CoarseSync* s = g_sync_free[i];
        g_sync_free.erase(g_sync_free.begin() + (long)i);
        s->refs.store(1);
        s->l1_pending.store(0);
        s->first_cycle.store(0);
        *out = s;
        return STT_OK;
      }
  }
  CoarseSync* s = new CoarseSync();
  s->device = dev;
  int lo = 0, hi = 0;
  int rc = check_cuda(cudaDeviceGetStreamPriorityRange(&lo, &hi), "stream priorities");
  if (rc == STT_OK) rc = check_cuda(cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, hi), "side stream");
  if (rc == STT_OK) rc = check_cuda(cudaEventCreateWithFlags(&s->built, cudaEventDisableTiming), "event");
  if (rc == STT_OK) rc = check_cuda(cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming), "event");
  if (rc == STT_OK) rc = check_cuda(cudaEventCreateWithFlags(&s->factored, cudaEventDisableTiming), "event");
  if (rc != STT_OK) {
    if (s->factored) cudaEventDestroy(s->factored);
    if (s->ready) cudaEventDestroy(s->ready);
    if (s->built) cudaEventDestroy(s->built);
    if (s->side) cudaStreamDestroy(s->side);
    delete s;
    return rc;
  }
  *out = s;
  return STT_OK;
}

// Drops one reference; the last waits for the factorisation (it writes the workspace,
// which the caller may free or reuse after the destroy) and returns the object to the pool.
static void release_sync(CoarseSync* s) {
  if (!s || s->refs.fetch_sub(1) != 1) return;
  cudaEventSynchronize(s->ready);
  std::lock_guard<std::mutex> lock(g_sync_mu);
  g_sync_free.push_back(s);
}

template <int D>
static int build_coarse(stt_hier* h, cudaStream_t st) {
  CoarseDesc& co = h->co;
  const LevelDesc& cl = h->lv[h->nlevels - 1];
  const int H = h->hrows;
  const long long per = (long long)co.nb * 4 * co.B * co.B;
  STT_TRY(check_cuda(cudaMemsetAsync(co.blocks, 0, 8 * H * per, st), "memset coarse"));
  const long long threads = cl.nnode + ((long long)co.nb * co.B - cl.ndof);
  band_assemble_kernel<D><<<dim3(grid1(threads), H), 256, 0, st>>>(
      cl.st64, cl.fixed, cl.nnx, cl.nny, co.by_col, co.B, co.nb, co.blocks, h->status);
  STT_TRY(check_launch("band assemble"));
  const size_t smem = (size_t)3 * co.B * (co.B + 1) * sizeof(double);
  STT_TRY(allow_large_smem());
  const size_t tsmem = smem + (size_t)2 * co.B * co.B * sizeof(double);  // + two staging blocks
  if (co.B == 32)
    band_factor_tiled_kernel<2><<<H, 256, tsmem, st>>>(co.blocks, co.nb, h->status);
  else if (co.B == 64)
    band_factor_tiled_kernel<4><<<H, 256, tsmem, st>>>(co.blocks, co.nb, h->status);
  else
    band_factor_kernel<<<H, 256, smem, st>>>(co.blocks, co.B, co.nb, h->status);
  STT_TRY(check_launch("band factor"));
  STT_TRY(check_cuda(cudaEventRecord(h->sync->factored, st), "record factor"));
  if (co.inv) {
    if (co.B == 32 || co.B == 64) {
      const size_t tsm = (size_t)3 * co.B * (co.B + 1) * sizeof(double);
      if (co.B == 32)
        coarse_inverse_tiled_kernel<2><<<dim3(co.nb, H), 256, tsm, st>>>(co.blocks, co.nb, co.inv);
      else
        coarse_inverse_tiled_kernel<4><<<dim3(co.nb, H), 256, tsm, st>>>(co.blocks, co.nb, co.inv);
      const long long np = (long long)co.nb * co.B;
      const unsigned nt = (unsigned)((np + 31) / 32);
      coarse_mirror_kernel<<<dim3(nt, nt, H), dim3(32, 8), 0, st>>>(co.inv, co.B, np);
    } else {
      const size_t ism = (size_t)3 * co.B * co.B * sizeof(double);
      coarse_inverse_kernel<<<dim3(co.nb, H), 256, ism, st>>>(co.blocks, co.B, co.nb, co.inv);
    }
    STT_TRY(check_launch("coarse inverse"));
  }
  return STT_OK;
}

extern "C" int stt_hier_create(stt_hier** out, void* workspace, long long ws_bytes, int d, int nelx,
                               int nely, int hrows, const double* rho, long long rho_rs,
                               const double* reaction, long long r_rs, const uint8_t* fixed,
                               const double* KE, int max_coarse_elements, int precision,
                               stt_stream_t stream) {
  if (!out || !workspace || !rho || !KE || (d != 1 && d != 2) || nelx <= 0 || nely <= 0 ||
      hrows <= 0 || hrows > 65535 || (precision != STT_FP64 && precision != STT_FP32))
    return set_error(STT_ERR_INVALID, "stt_hier_create: bad arguments");
  if (((uintptr_t)workspace & 255) != 0)
    return set_error(STT_ERR_INVALID, "stt_hier_create: workspace must be 256-byte aligned");
  stt_hier* h = new stt_hier();
  std::memset((void*)h, 0, sizeof(stt_hier));
  h->d = d;
  h->nelx = nelx;
  h->nely = nely;
  h->hrows = hrows;
  h->precision = precision;
  h->mce = max_coarse_elements;
  h->has_reaction = reaction != nullptr;
  for (int i = 0; i < 16 * d * d; ++i) h->KE[i] = KE[i];
  h->modal = modal_from_ke(d, KE, h->mq) ? 1 : 0;
  const long long need = plan_hierarchy(*h, nullptr);
  if (ws_bytes < need) {
    delete h;
    return set_error(STT_ERR_WORKSPACE, "stt_hier_create: workspace too small");
  }
  plan_hierarchy(*h, (char*)workspace);
  h->status = (int*)((char*)workspace + need - 256);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = check_cuda(cudaMemsetAsync(h->status, 0, 256, st), "memset status");
  if (rc == STT_OK) rc = d == 2 ? build_levels<2>(h, rho, rho_rs, reaction, r_rs, fixed, st, true)
                                : build_levels<1>(h, rho, rho_rs, reaction, r_rs, fixed, st, true);
  // the coarsest level's factorisation runs on the side stream, after the levels, while
  // the caller's stream goes on (a solve's initialisation and first descent); the coarse
  // solves wait for `ready`
  if (rc == STT_OK) rc = acquire_sync(&h->sync);
  if (rc == STT_OK) rc = check_cuda(cudaEventRecord(h->sync->built, st), "record build");
  if (rc == STT_OK) rc = check_cuda(cudaStreamWaitEvent(h->sync->side, h->sync->built, 0), "side wait");
  if (rc == STT_OK) rc = d == 2 ? build_coarse<2>(h, h->sync->side) : build_coarse<1>(h, h->sync->side);
  if (rc == STT_OK) rc = check_cuda(cudaEventRecord(h->sync->ready, h->sync->side), "record coarse");
  if (rc == STT_OK) h->sync->first_cycle.store(h->co.inv ? 1 : 0);
  // level 1's stencil (deferred by build_levels) beside the factorisation; an FP32
  // hierarchy swept from the densities only its FP32 diagonal, the FP64 stencil on first use
  if (rc == STT_OK && h->nlevels > 2) {
    const int nm = h->lv[0].kx * h->lv[0].ky;
    const bool diag_only = h->l1 && precision == STT_FP32 && !reaction && (nm == 4 || nm == 6 || nm == 9);
    rc = d == 2 ? level1_stencil<2>(h, reaction, r_rs, st, diag_only ? 1 : 0)
                : level1_stencil<1>(h, reaction, r_rs, st, diag_only ? 1 : 0);
    if (rc == STT_OK && diag_only) h->sync->l1_pending.store(1);
  }
  if (rc != STT_OK) {
    if (h->sync) release_sync(h->sync);
    delete h;
    return rc;
  }
  // no synchronisation here: the build's device checks (coarse pivots, band) are read by
  // stt_hier_status, and by the first convergence check after a solve's first V-cycle
  *out = h;
  return STT_OK;
}

// Level 1's FP64 stencil of an FP32 hierarchy swept from the densities, assembled on the
// first use (on `st`) by the entry points that read it.
int stt::ensure_level1_fp64(const stt_hier* h, int level, cudaStream_t st) {
  if (level != 1 || !h->sync->l1_pending.load()) return STT_OK;
  std::lock_guard<std::mutex> lock(h->sync->l1_mu);
  if (!h->sync->l1_pending.load()) return STT_OK;
  stt_hier* hh = const_cast<stt_hier*>(h);
  STT_TRY(h->d == 2 ? level1_stencil<2>(hh, nullptr, 0, st, 2) : level1_stencil<1>(hh, nullptr, 0, st, 2));
  h->sync->l1_pending.store(0);
  return STT_OK;
}

// The build's device status word as an error code (host int s, already copied).
int stt::hier_status_code(int s) {
  if (s & 1) return set_error(STT_ERR_INVALID, "coarse operator is not positive definite (Cholesky pivot <= 0)");
  if (s & 2) return set_error(STT_ERR_INVALID, "coarse operator exceeds its planned band");
  return STT_OK;
}

extern "C" int stt_hier_status(const stt_hier* h, stt_stream_t stream) {
  if (!h) return set_error(STT_ERR_INVALID, "stt_hier_status: null hierarchy");
  cudaStream_t st = (cudaStream_t)stream;
  int s = 0;
  STT_TRY(check_cuda(cudaStreamWaitEvent(st, h->sync->ready, 0), "wait coarse"));
  STT_TRY(check_cuda(cudaMemcpyAsync(&s, h->status, sizeof(int), cudaMemcpyDeviceToHost, st), "status copy"));
  STT_TRY(check_cuda(cudaStreamSynchronize(st), "hierarchy build"));
  return hier_status_code(s);
}

extern "C" int stt_hier_select(const stt_hier* h, const int* row_map, stt_hier** out) {
  if (!h || !out) return set_error(STT_ERR_INVALID, "stt_hier_select: null");
  stt_hier* v = new stt_hier(*h);
  v->row_map = row_map;
  v->sync->refs.fetch_add(1);  // the view shares the coarse factorisation
  *out = v;
  return STT_OK;
}

extern "C" int stt_hier_destroy(stt_hier* h) {
  if (h) release_sync(h->sync);
  delete h;
  return STT_OK;
}

extern "C" int stt_hier_info(const stt_hier* h, int* nlevels, int* dims, int max_levels) {
  if (!h || !nlevels) return set_error(STT_ERR_INVALID, "stt_hier_info: null");
  *nlevels = h->nlevels;
  if (dims)
    for (int l = 0; l < h->nlevels && l < max_levels; ++l) {
      dims[4 * l + 0] = h->lv[l].nelx;
      dims[4 * l + 1] = h->lv[l].nely;
      dims[4 * l + 2] = h->lv[l].kx;
      dims[4 * l + 3] = h->lv[l].ky;
    }
  return STT_OK;
}

template <int D>
__global__ void stencil_diag_kernel(const double* __restrict__ st, const uint8_t* __restrict__ fixed,
                                    long long nnode, double* __restrict__ out) {
  constexpr int NS = 5 * D * D;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  if (n >= nnode) return;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double v = st[((size_t)h * NS + i * D + i) * nnode + n];
    if ((fixed[n] >> i) & 1) v = 1.0;
    out[((size_t)h * nnode + n) * D + i] = v;
  }
}

extern "C" int stt_hier_level_diag(const stt_hier* h, int level, double* out, stt_stream_t stream) {
  if (!h || !out || level < 0 || level >= h->nlevels) return set_error(STT_ERR_INVALID, "stt_hier_level_diag: bad level");
  const LevelDesc& lv = h->lv[level];
  cudaStream_t st = (cudaStream_t)stream;
  if (level == 0)
    return stt_q4_diag(h->d, h->nelx, h->nely, h->hrows, lv.rho64, lv.rs_rho,
                       h->has_reaction ? lv.rdiag64 : nullptr, lv.ndof,
                       lv.fixed, out, lv.ndof, h->KE, stream);
  STT_TRY(ensure_level1_fp64(h, level, st));
  if (h->d == 2)
    stencil_diag_kernel<2><<<dim3(grid1(lv.nnode), h->hrows), 256, 0, st>>>(lv.st64, lv.fixed, lv.nnode, out);
  else
    stencil_diag_kernel<1><<<dim3(grid1(lv.nnode), h->hrows), 256, 0, st>>>(lv.st64, lv.fixed, lv.nnode, out);
  return check_launch("stencil diag");
}

extern "C" int stt_hier_level_fixed(const stt_hier* h, int level, uint8_t* out, stt_stream_t stream) {
  if (!h || !out || level < 0 || level >= h->nlevels) return set_error(STT_ERR_INVALID, "stt_hier_level_fixed: bad level");
  return check_cuda(cudaMemcpyAsync(out, h->lv[level].fixed, h->lv[level].nnode, cudaMemcpyDeviceToDevice,
                                    (cudaStream_t)stream), "copy fixed");
}
