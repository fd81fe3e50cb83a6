// Cone density filter and Heaviside projection (the density field's upstream step).
//
// Reference: filters.density_filter / apply_density_filter (sttopt/filters.py:38-85):
// H[e1, e2] = max(0, rmin - dist(e1, e2)) over the square of offsets |d| <= ceil(rmin) - 1,
// xTilde = H x / Hs with Hs the row sums, and heaviside_projection /
// heaviside_projection_derivative (:109-133).  H is a stencil with zero padding outside
// the grid, so it is applied as one here: a block stages its 32 x 8 output tile plus the
// stencil's halo in shared memory (coalesced rows), and Hs is the sum of the in-grid
// weights, formed from the element's position (no matrix, no row-sum array).  H is
// symmetric, so the adjoint, H (g * P'(xTilde) / Hs), is the same stencil applied to the
// scaled field.  FP64 throughout; rows of the batch with their own strides.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "errors.h"

namespace stt {

constexpr int kFiltMaxR = 7;  // ceil(rmin) - 1 <= 7 (rmin <= 8)
constexpr int kFiltTX = 32, kFiltTY = 8;

struct FiltW {
  double w[(2 * kFiltMaxR + 1) * (2 * kFiltMaxR + 1)];  // w[(dj + R) * (2R + 1) + (di + R)]
};

// Hs of element (i, j): the sum of the weights whose offset stays in the grid.
STT_DEV double filt_hs(const FiltW& W, int R, int i, int j, int nelx, int nely) {
  const int n = 2 * R + 1;
  double s = 0.0;
  for (int dj = -R; dj <= R; ++dj) {
    if (j + dj < 0 || j + dj >= nely) continue;
    for (int di = -R; di <= R; ++di)
      if (i + di >= 0 && i + di < nelx) s += W.w[(dj + R) * n + (di + R)];
  }
  return s;
}

// P(x) and P'(x) of the Heaviside projection (beta > 0; beta = inf is the step with 1/2
// at the threshold).
STT_DEV double heaviside(double x, double beta, double eta) {
  if (isinf(beta)) return x > eta ? 1.0 : (x < eta ? 0.0 : 0.5);
  const double den = tanh(beta * eta) + tanh(beta * (1.0 - eta));
  return (tanh(beta * eta) + tanh(beta * (x - eta))) / den;
}
STT_DEV double heaviside_d(double x, double beta, double eta) {
  if (isinf(beta)) return 0.0;
  const double den = tanh(beta * eta) + tanh(beta * (1.0 - eta));
  const double t = tanh(beta * (x - eta));
  return beta * (1.0 - t * t) / den;
}

// ADJ = 0: xt = H x / Hs (and xp = P(xt) when beta > 0);
// ADJ = 1: out = H (g * s / Hs), s = P'(xt) when beta > 0 (xt given), else 1.
template <int ADJ>
__global__ void __launch_bounds__(kFiltTX * kFiltTY) cone_filter_kernel(
    const double* __restrict__ in, long long in_rs, const double* __restrict__ xt_in, long long xt_rs,
    double* __restrict__ out, double* __restrict__ xp, long long o_rs, int nelx, int nely, int R, FiltW W,
    double beta, double eta) {
  extern __shared__ double tile[];  // (kFiltTY + 2R) x (kFiltTX + 2R)
  const int s = blockIdx.z;
  const int tw = kFiltTX + 2 * R, th = kFiltTY + 2 * R;
  const int i0 = blockIdx.x * kFiltTX - R, j0 = blockIdx.y * kFiltTY - R;
  const double* xs = in + (size_t)s * in_rs;
  const double* ts = ADJ ? xt_in + (size_t)s * xt_rs : nullptr;
  const bool proj = beta > 0.0;
  for (int t = threadIdx.y * kFiltTX + threadIdx.x; t < tw * th; t += kFiltTX * kFiltTY) {
    const int ti = t % tw, tj = t / tw;
    const int i = i0 + ti, j = j0 + tj;
    double v = 0.0;
    if (i >= 0 && i < nelx && j >= 0 && j < nely) {
      const long long e = (long long)j * nelx + i;
      v = __ldg(xs + e);
      if (ADJ) {
        if (proj && ts) v *= heaviside_d(__ldg(ts + e), beta, eta);
        v /= filt_hs(W, R, i, j, nelx, nely);
      }
    }
    tile[tj * tw + ti] = v;
  }
  __syncthreads();
  const int i = blockIdx.x * kFiltTX + threadIdx.x, j = blockIdx.y * kFiltTY + threadIdx.y;
  if (i >= nelx || j >= nely) return;
  const int n = 2 * R + 1;
  double acc = 0.0;
  for (int dj = -R; dj <= R; ++dj) {
    const double* trow = tile + (threadIdx.y + R + dj) * tw + threadIdx.x + R;
    for (int di = -R; di <= R; ++di) acc = fma(W.w[(dj + R) * n + (di + R)], trow[di], acc);
  }
  const long long e = (long long)j * nelx + i;
  double* os = out + (size_t)s * o_rs;
  if (ADJ) {
    os[e] = acc;
  } else {
    const double x = acc / filt_hs(W, R, i, j, nelx, nely);
    os[e] = x;
    if (proj && xp) xp[(size_t)s * o_rs + e] = heaviside(x, beta, eta);
  }
}

// The weights max(0, rmin - hypot(di, dj)) of the reference (filters.py:52-55).
static bool filt_weights(double rmin, int& R, FiltW& W) {
  if (!(rmin > 0.0) || !std::isfinite(rmin)) return false;
  R = (int)std::ceil(rmin) - 1;
  if (R < 0 || R > kFiltMaxR) return false;
  const int n = 2 * R + 1;
  for (int dj = -R; dj <= R; ++dj)
    for (int di = -R; di <= R; ++di) W.w[(dj + R) * n + (di + R)] = std::fmax(0.0, rmin - std::hypot((double)di, (double)dj));
  return true;
}

template <int ADJ>
static int launch_filter(int nelx, int nely, int nrows, double rmin, const double* in, long long in_rs,
                         const double* xt, long long xt_rs, double* out, double* xp, long long o_rs, double beta,
                         double eta, cudaStream_t st) {
  int R;
  FiltW W;
  if (!filt_weights(rmin, R, W))
    return set_error(STT_ERR_INVALID, "cone filter: rmin must be in (0, 8]");
  const dim3 grid((nelx + kFiltTX - 1) / kFiltTX, (nely + kFiltTY - 1) / kFiltTY, nrows);
  const size_t smem = sizeof(double) * (kFiltTX + 2 * R) * (kFiltTY + 2 * R);
  cone_filter_kernel<ADJ><<<grid, dim3(kFiltTX, kFiltTY), smem, st>>>(in, in_rs, xt, xt_rs, out, xp, o_rs, nelx,
                                                                      nely, R, W, beta, eta);
  return check_launch("cone filter");
}

}  // namespace stt

using namespace stt;

extern "C" int stt_cone_filter(int nelx, int nely, int nrows, double rmin, const double* x, long long x_rs,
                               double* xt, double* xp, long long o_rs, double beta, double eta,
                               stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !x || !xt || (beta > 0.0 && !xp))
    return set_error(STT_ERR_INVALID, "stt_cone_filter: bad sizes or null pointer");
  return launch_filter<0>(nelx, nely, nrows, rmin, x, x_rs, nullptr, 0, xt, xp, o_rs, beta, eta,
                          (cudaStream_t)stream);
}

extern "C" int stt_cone_filter_adjoint(int nelx, int nely, int nrows, double rmin, const double* g,
                                       long long g_rs, const double* xt, long long xt_rs, double beta,
                                       double eta, double* out, long long o_rs, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !g || !out || (beta > 0.0 && !xt))
    return set_error(STT_ERR_INVALID, "stt_cone_filter_adjoint: bad sizes or null pointer");
  return launch_filter<1>(nelx, nely, nrows, rmin, g, g_rs, xt, xt_rs, out, nullptr, o_rs, beta, eta,
                          (cudaStream_t)stream);
}
