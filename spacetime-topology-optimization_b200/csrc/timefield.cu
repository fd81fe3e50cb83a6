// Element <-> node transfers of the stage glue and of the time fields, as node- or
// element-centric gathers (no atomics, deterministic sums):
//   * the gravity load matrix C of sttopt/gravity.py:15-36 (fe / 4 of each element to its
//     corners, fe = 1 / (nelx nely)) and its transpose;
//   * element means over the four corners (sttopt/virtual_heat.py:162-166) and their
//     transpose;
//   * the load of the Poisson distance fit, divergence_load(w, direction_field(s))
//     (sttopt/virtual_heat.py:290-320): grad s at the 2 x 2 Gauss points, normalised,
//     F_n = sum over elements of w_e / 4 sum_g X_g . grad N_n(g); and its adjoint in s
//     and w.
// Node (r, c) of the (nely + 1) x (nelx + 1) grid, row 0 at the top, is corner BR of
// element (r - 1, c - 1), BL of (r - 1, c), TR of (r, c - 1) and TL of (r, c).  FP64.
#include <cfloat>

#include "common.cuh"
#include "errors.h"

namespace stt {

static int tf_grid(long long n, int bs = 256) {
  long long g = (n + bs - 1) / bs;
  if (g > (1 << 30)) g = 1 << 30;
  return (int)(g < 1 ? 1 : g);
}

// out[n] = scale * sum of x over the elements of node n.
__global__ void node_gather_kernel(const double* __restrict__ x, long long x_rs, double* __restrict__ out,
                                   long long o_rs, int nelx, int nely, double scale) {
  const int nnx = nelx + 1;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= (long long)nnx * (nely + 1)) return;
  const int r = (int)(n / nnx), c = (int)(n - (long long)r * nnx);
  const double* xs = x + (size_t)blockIdx.y * x_rs;
  double s = 0.0;
  if (r > 0 && c > 0) s += __ldg(xs + (size_t)(r - 1) * nelx + c - 1);
  if (r > 0 && c < nelx) s += __ldg(xs + (size_t)(r - 1) * nelx + c);
  if (r < nely && c > 0) s += __ldg(xs + (size_t)r * nelx + c - 1);
  if (r < nely && c < nelx) s += __ldg(xs + (size_t)r * nelx + c);
  out[(size_t)blockIdx.y * o_rs + n] = scale * s;
}

// out[e] = scale * sum of g over the corners of element e (BL, BR, TR, TL).
__global__ void element_gather_kernel(const double* __restrict__ g, long long g_rs, double* __restrict__ out,
                                      long long o_rs, int nelx, int nely, double scale) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)nelx * nely) return;
  const int er = (int)(e / nelx), ec = (int)(e - (long long)er * nelx);
  const int nnx = nelx + 1;
  const double* gs = g + (size_t)blockIdx.y * g_rs;
  const size_t top = (size_t)er * nnx + ec, bot = top + nnx;
  const double s = __ldg(gs + bot) + __ldg(gs + bot + 1) + __ldg(gs + top + 1) + __ldg(gs + top);
  out[(size_t)blockIdx.y * o_rs + e] = scale * s;
}

// The 2 x 2 Gauss rule of a unit square: points (xi, eta) in the order
// (a, a), (b, a), (a, b), (b, b), a = 1/2 - 1/(2 sqrt 3), b = 1/2 + 1/(2 sqrt 3);
// grad N of the bilinear shape functions, x right and y up, local order BL, BR, TR, TL:
//   d/dx = (-(1 - eta), 1 - eta, eta, -eta),  d/dy = (-(1 - xi), -xi, xi, 1 - xi).
struct Gauss {
  double xi[4], eta[4];
};

STT_DEV void shape_grad(const Gauss& G, int g, double (&bx)[4], double (&by)[4]) {
  const double xi = G.xi[g], eta = G.eta[g];
  bx[0] = -(1.0 - eta);
  bx[1] = 1.0 - eta;
  bx[2] = eta;
  bx[3] = -eta;
  by[0] = -(1.0 - xi);
  by[1] = -xi;
  by[2] = xi;
  by[3] = 1.0 - xi;
}

// Element (er, ec)'s corner values of a nodal field, local order BL, BR, TR, TL.
STT_DEV void corners(const double* __restrict__ u, int er, int ec, int nnx, double (&v)[4]) {
  const size_t top = (size_t)er * nnx + ec, bot = top + nnx;
  v[0] = __ldg(u + bot);
  v[1] = __ldg(u + bot + 1);
  v[2] = __ldg(u + top + 1);
  v[3] = __ldg(u + top);
}

// Unit direction of grad s at Gauss point g (grad / sqrt(|grad|^2 + tiny)); also returns
// the gradient and the norm for the adjoint.
STT_DEV void direction(const Gauss& G, int g, const double (&s)[4], double& gx, double& gy, double& nrm) {
  double bx[4], by[4];
  shape_grad(G, g, bx, by);
  gx = 0.0;
  gy = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    gx = fma(bx[i], s[i], gx);
    gy = fma(by[i], s[i], gy);
  }
  nrm = sqrt(fma(gx, gx, gy * gy) + DBL_MIN);
}

// Element e's contribution to the load at its local corner q: w / 4 sum_g X_g . grad N_q(g).
STT_DEV double poisson_elem_load(const Gauss& G, const double (&s)[4], double w, int q) {
  double acc = 0.0;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    double gx, gy, nrm, bx[4], by[4];
    direction(G, g, s, gx, gy, nrm);
    shape_grad(G, g, bx, by);
    acc += (gx / nrm) * bx[q] + (gy / nrm) * by[q];
  }
  return w * acc * 0.25;
}

__global__ void poisson_load_kernel(const double* __restrict__ sfield, long long s_rs, const double* __restrict__ w,
                                    long long w_rs, double* __restrict__ F, long long F_rs, int nelx, int nely,
                                    Gauss G) {
  const int nnx = nelx + 1;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= (long long)nnx * (nely + 1)) return;
  const int r = (int)(n / nnx), c = (int)(n - (long long)r * nnx);
  const double* ss = sfield + (size_t)blockIdx.y * s_rs;
  const double* ws = w + (size_t)blockIdx.y * w_rs;
  double acc = 0.0;
  // (element row, element column, local corner of this node)
  const int er[4] = {r - 1, r - 1, r, r}, ec[4] = {c - 1, c, c - 1, c}, q[4] = {1, 0, 2, 3};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (er[k] < 0 || er[k] >= nely || ec[k] < 0 || ec[k] >= nelx) continue;
    double s[4];
    corners(ss, er[k], ec[k], nnx, s);
    acc += poisson_elem_load(G, s, __ldg(ws + (size_t)er[k] * nelx + ec[k]), q[k]);
  }
  F[(size_t)blockIdx.y * F_rs + n] = acc;
}

// The adjoint of F(s, w) for an output weight gF: per element, with gl the corner values
// of gF, gw_e = 1/4 sum_g X_g . (B_g gl), and the Gauss gradients' adjoint
// gG = gX / n - G (G . gX) / n^3 (gX = w/4 B_g gl) pulled back to the corners by B_g^T.
// Each node sums the corner terms of its elements (gs); the node at an element's TL
// corner also writes that element's gw.
STT_DEV void poisson_elem_adjoint(const Gauss& G, const double (&s)[4], const double (&gl)[4], double w,
                                  double (&gu)[4], double& gw) {
  gw = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) gu[i] = 0.0;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    double gx, gy, nrm, bx[4], by[4];
    direction(G, g, s, gx, gy, nrm);
    shape_grad(G, g, bx, by);
    double px = 0.0, py = 0.0;  // B_g gl
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      px = fma(bx[i], gl[i], px);
      py = fma(by[i], gl[i], py);
    }
    gw += (gx * px + gy * py) / nrm;
    const double hx = 0.25 * w * px, hy = 0.25 * w * py;  // gX
    const double dot = (gx * hx + gy * hy) / (nrm * nrm * nrm);
    const double ggx = hx / nrm - gx * dot, ggy = hy / nrm - gy * dot;
#pragma unroll
    for (int i = 0; i < 4; ++i) gu[i] += bx[i] * ggx + by[i] * ggy;
  }
  gw *= 0.25;
}

__global__ void poisson_load_adjoint_kernel(const double* __restrict__ sfield, long long s_rs,
                                            const double* __restrict__ w, long long w_rs,
                                            const double* __restrict__ gF, long long gF_rs,
                                            double* __restrict__ gs, long long gs_rs, double* __restrict__ gw,
                                            long long gw_rs, int nelx, int nely, Gauss G) {
  const int nnx = nelx + 1;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= (long long)nnx * (nely + 1)) return;
  const int r = (int)(n / nnx), c = (int)(n - (long long)r * nnx);
  const double* ss = sfield + (size_t)blockIdx.y * s_rs;
  const double* ws = w + (size_t)blockIdx.y * w_rs;
  const double* gfs = gF + (size_t)blockIdx.y * gF_rs;
  double acc = 0.0;
  const int er[4] = {r - 1, r - 1, r, r}, ec[4] = {c - 1, c, c - 1, c}, q[4] = {1, 0, 2, 3};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (er[k] < 0 || er[k] >= nely || ec[k] < 0 || ec[k] >= nelx) continue;
    double s[4], gl[4], gu[4], gwe;
    corners(ss, er[k], ec[k], nnx, s);
    corners(gfs, er[k], ec[k], nnx, gl);
    const size_t e = (size_t)er[k] * nelx + ec[k];
    poisson_elem_adjoint(G, s, gl, __ldg(ws + e), gu, gwe);
    acc += gu[q[k]];
    if (k == 3 && gw) gw[(size_t)blockIdx.y * gw_rs + e] = gwe;
  }
  if (gs) gs[(size_t)blockIdx.y * gs_rs + n] = acc;
}

static Gauss gauss_rule() {
  const double a = 0.5 - 0.5 / std::sqrt(3.0), b = 0.5 + 0.5 / std::sqrt(3.0);
  return Gauss{{a, b, a, b}, {a, a, b, b}};
}

static bool rows_ok(int nelx, int nely, int nrows) {
  return nelx > 0 && nely > 0 && nrows > 0 && nrows <= 65535;
}

}  // namespace stt

using namespace stt;

extern "C" int stt_gravity_load(int nelx, int nely, int nrows, const double* x, long long x_rs, double* out,
                                long long o_rs, int transpose, stt_stream_t stream) {
  if (!rows_ok(nelx, nely, nrows) || !x || !out)
    return set_error(STT_ERR_INVALID, "stt_gravity_load: bad sizes or null pointer");
  const double q = 0.25 / ((double)nelx * nely);
  const long long nnode = (long long)(nelx + 1) * (nely + 1), nel = (long long)nelx * nely;
  cudaStream_t st = (cudaStream_t)stream;
  if (transpose)
    element_gather_kernel<<<dim3(tf_grid(nel), nrows), 256, 0, st>>>(x, x_rs, out, o_rs, nelx, nely, q);
  else
    node_gather_kernel<<<dim3(tf_grid(nnode), nrows), 256, 0, st>>>(x, x_rs, out, o_rs, nelx, nely, q);
  return check_launch("gravity load");
}

extern "C" int stt_element_means(int nelx, int nely, int nrows, const double* u, long long u_rs, double* out,
                                 long long o_rs, int transpose, stt_stream_t stream) {
  if (!rows_ok(nelx, nely, nrows) || !u || !out)
    return set_error(STT_ERR_INVALID, "stt_element_means: bad sizes or null pointer");
  const long long nnode = (long long)(nelx + 1) * (nely + 1), nel = (long long)nelx * nely;
  cudaStream_t st = (cudaStream_t)stream;
  if (transpose)
    node_gather_kernel<<<dim3(tf_grid(nnode), nrows), 256, 0, st>>>(u, u_rs, out, o_rs, nelx, nely, 0.25);
  else
    element_gather_kernel<<<dim3(tf_grid(nel), nrows), 256, 0, st>>>(u, u_rs, out, o_rs, nelx, nely, 0.25);
  return check_launch("element means");
}

extern "C" int stt_poisson_load(int nelx, int nely, int nrows, const double* s, long long s_rs, const double* w,
                                long long w_rs, double* F, long long F_rs, stt_stream_t stream) {
  if (!rows_ok(nelx, nely, nrows) || !s || !w || !F)
    return set_error(STT_ERR_INVALID, "stt_poisson_load: bad sizes or null pointer");
  const long long nnode = (long long)(nelx + 1) * (nely + 1);
  poisson_load_kernel<<<dim3(tf_grid(nnode), nrows), 256, 0, (cudaStream_t)stream>>>(s, s_rs, w, w_rs, F, F_rs,
                                                                                      nelx, nely, gauss_rule());
  return check_launch("poisson load");
}

extern "C" int stt_poisson_load_adjoint(int nelx, int nely, int nrows, const double* s, long long s_rs,
                                        const double* w, long long w_rs, const double* gF, long long gF_rs,
                                        double* gs, long long gs_rs, double* gw, long long gw_rs,
                                        stt_stream_t stream) {
  if (!rows_ok(nelx, nely, nrows) || !s || !w || !gF || (!gs && !gw))
    return set_error(STT_ERR_INVALID, "stt_poisson_load_adjoint: bad sizes or null pointer");
  const long long nnode = (long long)(nelx + 1) * (nely + 1);
  poisson_load_adjoint_kernel<<<dim3(tf_grid(nnode), nrows), 256, 0, (cudaStream_t)stream>>>(
      s, s_rs, w, w_rs, gF, gF_rs, gs, gs_rs, gw, gw_rs, nelx, nely, gauss_rule());
  return check_launch("poisson load adjoint");
}
