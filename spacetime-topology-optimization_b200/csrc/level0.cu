// Level-0 operator entry points: K(rho) u (projected or not), diag(K), lumped reaction.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "errors.h"
#include "modal.h"
#include "q4.cuh"

namespace stt {

template <int D, typename T>
__global__ void __launch_bounds__(kQThreads) q4_apply_kernel(
    const T* __restrict__ u, long long u_rs, T* __restrict__ out, long long out_rs,
    const T* __restrict__ rho, long long rho_rs, const T* __restrict__ rdiag, long long rdiag_rs,
    const uint8_t* __restrict__ fixed, int proj_in, int proj_out, int nelx, int nely,
    KEq<D, T> ke) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int row = blockIdx.z;
  const T* ur = u + (size_t)row * u_rs;
  const T* rr = rho + (size_t)row * rho_rs;
  const T* rdr = rdiag ? rdiag + (size_t)row * rdiag_rs : nullptr;
  T* outr = out + (size_t)row * out_rs;
  const uint8_t* pin = proj_in ? fixed : nullptr;
  march<D, T, true, false, FlagX>(
      ke, nnx, nny,
      [&](int r, int c, T(&v)[D]) {
        const int node = r * nnx + c;
        load_node<D, T>(ur, node, v);
        if (pin) {
          const uint8_t fl = __ldg(pin + node);
#pragma unroll
          for (int d = 0; d < D; ++d)
            if ((fl >> d) & 1) v[d] = T(0);
        }
      },
      [&](int r, int c) { return __ldg(rr + (size_t)r * nelx + c); },
      [&](int r, int c) { return FlagX{proj_out ? __ldg(fixed + r * nnx + c) : (uint8_t)0}; },
      [&](int r, int c, T(&acc)[D], T(&)[D], const T(&uc)[D], const FlagX& ex) {
        const int node = r * nnx + c;
        if (rdr) {
#pragma unroll
          for (int i = 0; i < D; ++i) acc[i] = fma(__ldg(rdr + node * D + i), uc[i], acc[i]);
        }
#pragma unroll
        for (int i = 0; i < D; ++i)
          if ((ex.fl >> i) & 1) acc[i] = T(0);
        store_node<D, T>(outr, node, acc);
      });
}

// The same operator with KE in modal form; FL selects the options at compile time:
// bit 0 projects the input, bit 1 the output, bit 2 adds the reaction term.
template <int D, typename T, int FL>
__global__ void __launch_bounds__(kQThreads) q4_apply_modal_kernel(
    const T* __restrict__ u, long long u_rs, T* __restrict__ out, long long out_rs,
    const T* __restrict__ rho, long long rho_rs, const T* __restrict__ rdiag, long long rdiag_rs,
    const uint8_t* __restrict__ fixed, int nelx, int nely, MQ<T> mq) {
  constexpr bool PIN = FL & 1, POUT = FL & 2, RD = FL & 4;
  const int nnx = nelx + 1, nny = nely + 1;
  const int row = blockIdx.z;
  const T* ur = u + (size_t)row * u_rs;
  const T* rr = rho + (size_t)row * rho_rs;
  const T* rdr = RD ? rdiag + (size_t)row * rdiag_rs : nullptr;
  T* outr = out + (size_t)row * out_rs;
  march_modal<D, T, true, false, PIN>(
      mq, nnx, nny,
      [&](int r, int c) -> uint8_t { return (PIN || POUT) ? __ldg(fixed + r * nnx + c) : (uint8_t)0; },
      [&](int r, int c, uint8_t, T(&v)[D]) { load_node<D, T>(ur, r * nnx + c, v); },
      [&](int r, int c) { return __ldg(rr + (size_t)r * nelx + c); },
      [&](int, int) { return NoExtra{}; },
      [&](int r, int c, T(&acc)[D], T(&)[D], const T(&uc)[D], uint8_t fl, const NoExtra&) {
        const int node = r * nnx + c;
        if constexpr (RD) {
#pragma unroll
          for (int i = 0; i < D; ++i) acc[i] = fma(__ldg(rdr + node * D + i), uc[i], acc[i]);
        }
        if constexpr (POUT) {
#pragma unroll
          for (int i = 0; i < D; ++i)
            if ((fl >> i) & 1) acc[i] = T(0);
        }
        store_node<D, T>(outr, node, acc);
      });
}

// out = K(rho) u with the fixed dofs zeroed (FP64), and per row the dots u . out and
// u . f taken in the same pass (f read beside the output node), reduced over the blocks
// in a fixed order (grid_reduce): one pass over u for an adjoint load and its warm-start
// factor (torch_solve.py:121-126).  MODAL: KE in modal form, else the 8 x 8 product.
template <int D, bool MODAL>
__global__ void __launch_bounds__(kQThreads) q4_apply_dots_kernel(
    const double* __restrict__ u, long long u_rs, double* __restrict__ out, long long out_rs,
    const double* __restrict__ rho, long long rho_rs, const uint8_t* __restrict__ fixed,
    const double* __restrict__ f, long long f_rs, double* __restrict__ dots, GridRed red, int nelx, int nely,
    KEq<D, double> ke, MQ<double> mq) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int row = blockIdx.z;
  const double* ur = u + (size_t)row * u_rs;
  const double* rr = rho + (size_t)row * rho_rs;
  const double* fr = f + (size_t)row * f_rs;
  double* outr = out + (size_t)row * out_rs;
  double vals[2] = {0.0, 0.0};
  auto finish = [&](int r, int c, double(&acc)[D], const double(&uc)[D], const RhsX<D, double>& ex) {
    const int node = r * nnx + c;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      if ((ex.fl >> i) & 1) acc[i] = 0.0;
      vals[0] = fma(uc[i], acc[i], vals[0]);
      vals[1] = fma(uc[i], ex.b[i], vals[1]);
    }
    store_node<D, double>(outr, node, acc);
  };
  auto loadx = [&](int r, int c) {
    RhsX<D, double> e;
    const int node = r * nnx + c;
    load_node<D, double>(fr, node, e.b);
    e.fl = __ldg(fixed + node);
    return e;
  };
  auto loadr = [&](int r, int c) { return __ldg(rr + (size_t)r * nelx + c); };
  if constexpr (MODAL) {
    march_modal<D, double, true, false, false, RhsX<D, double>>(
        mq, nnx, nny, [&](int r, int c) -> uint8_t { return __ldg(fixed + r * nnx + c); },
        [&](int r, int c, uint8_t, double(&v)[D]) { load_node<D, double>(ur, r * nnx + c, v); }, loadr, loadx,
        [&](int r, int c, double(&acc)[D], double(&)[D], const double(&uc)[D], uint8_t,
            const RhsX<D, double>& ex) { finish(r, c, acc, uc, ex); });
  } else {
    march<D, double, true, false, RhsX<D, double>>(
        ke, nnx, nny, [&](int r, int c, double(&v)[D]) { load_node<D, double>(ur, r * nnx + c, v); }, loadr,
        loadx, [&](int r, int c, double(&acc)[D], double(&)[D], const double(&uc)[D],
                   const RhsX<D, double>& ex) { finish(r, c, acc, uc, ex); });
  }
  grid_reduce<2, kQThreads>(red, row, blockIdx.y * gridDim.x + blockIdx.x, vals, [&](const double* t) {
    dots[(size_t)row * 2] = t[0];
    dots[(size_t)row * 2 + 1] = t[1];
  });
}

// out[s] = safe_div(dots[s][0], dots[s][1]) v[s]: the adjoint's warm start alpha U with
// alpha = (U . g) / (U . F) (torch_solve.py:121-126), written where the solve starts.
__global__ void rows_warm_start_kernel(long long n, const double* __restrict__ dots, const double* __restrict__ v,
                                       long long v_rs, double* __restrict__ out, long long o_rs) {
  const int s = blockIdx.y;
  const double a = safe_div(dots[(size_t)s * 2], dots[(size_t)s * 2 + 1]);
  const double* vs = v + (size_t)s * v_rs;
  double* os = out + (size_t)s * o_rs;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    os[i] = a * vs[i];
}

template <int D>
__global__ void __launch_bounds__(kQThreads) q4_diag_kernel(
    const double* __restrict__ rho, long long rho_rs, const double* __restrict__ rdiag,
    long long rdiag_rs, const uint8_t* __restrict__ fixed, double* __restrict__ out,
    long long out_rs, int nelx, int nely, KEq<D, double> ke) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int row = blockIdx.z;
  const double* rr = rho + (size_t)row * rho_rs;
  march<D, double, false, true>(
      ke, nnx, nny, [&](int, int, double(&)[D]) {},
      [&](int r, int c) { return __ldg(rr + (size_t)r * nelx + c); },
      [&](int, int) { return NoExtra{}; },
      [&](int r, int c, double(&)[D], double(&dg)[D], const double(&)[D], const NoExtra&) {
        const int node = r * nnx + c;
#pragma unroll
        for (int i = 0; i < D; ++i) {
          if (rdiag) dg[i] += __ldg(rdiag + (size_t)row * rdiag_rs + (size_t)node * D + i);
          if (is_fixed(fixed, node, i)) dg[i] = 1.0;
        }
        store_node<D, double>(out + (size_t)row * out_rs, node, dg);
      });
}

// rdiag[node * D + i] = sum of reaction[e] / 4 over the elements around the node.
template <int D>
__global__ void lumped_reaction_kernel(const double* __restrict__ reac, long long r_rs,
                                       double* __restrict__ out, long long out_rs, int nelx,
                                       int nely) {
  const int nnx = nelx + 1, nny = nely + 1;
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (node >= nnx * nny) return;
  const int r = node / nnx, c = node - r * nnx;
  const double* rr = reac + (size_t)row * r_rs;
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int er = r - 1 + a, ec = c - 1 + b;
      if (er >= 0 && er < nely && ec >= 0 && ec < nelx) acc += __ldg(rr + (size_t)er * nelx + ec) / 4;
    }
#pragma unroll
  for (int i = 0; i < D; ++i) out[(size_t)row * out_rs + (size_t)node * D + i] = acc;
}

template <int D, typename T>
KEq<D, T> make_ke(const double* KE) {
  KEq<D, T> k;
  for (int i = 0; i < 16 * D * D; ++i) k.v[i] = T(KE[i]);
  return k;
}

template <int D, typename T>
int launch_apply(int nelx, int nely, int nrows, const void* u, long long u_rs, void* out,
                 long long out_rs, const void* rho, long long rho_rs, const void* rdiag,
                 long long rdiag_rs, const uint8_t* fixed, int flags, const double* KE,
                 cudaStream_t st) {
  double m[8];
  const int pin = (flags & STT_PROJECT_IN) ? 1 : 0, pout = (flags & STT_PROJECT_OUT) ? 1 : 0;
  const dim3 grid = q4_grid(nelx, nely, nrows);
  if (modal_from_ke(D, KE, m)) {
    const MQ<T> mq = mq_cast<T>(m);
    const int fl = pin | (pout << 1) | (rdiag ? 4 : 0);
#define STT_MODAL_APPLY(FL)                                                                          \
  q4_apply_modal_kernel<D, T, FL><<<grid, kQThreads, 0, st>>>((const T*)u, u_rs, (T*)out, out_rs,    \
                                                              (const T*)rho, rho_rs, (const T*)rdiag, \
                                                              rdiag_rs, fixed, nelx, nely, mq)
    switch (fl) {
      case 0: STT_MODAL_APPLY(0); break;
      case 1: STT_MODAL_APPLY(1); break;
      case 2: STT_MODAL_APPLY(2); break;
      case 3: STT_MODAL_APPLY(3); break;
      case 4: STT_MODAL_APPLY(4); break;
      case 5: STT_MODAL_APPLY(5); break;
      case 6: STT_MODAL_APPLY(6); break;
      default: STT_MODAL_APPLY(7); break;
    }
#undef STT_MODAL_APPLY
  } else {
    q4_apply_kernel<D, T><<<grid, kQThreads, 0, st>>>(
        (const T*)u, u_rs, (T*)out, out_rs, (const T*)rho, rho_rs, (const T*)rdiag, rdiag_rs,
        fixed, pin, pout, nelx, nely, make_ke<D, T>(KE));
  }
  return check_launch("q4_apply");
}

}  // namespace stt

using namespace stt;

extern "C" int stt_q4_apply(int precision, int d, int nelx, int nely, int nrows, const void* u,
                            long long u_rs, void* out, long long out_rs, const void* rho,
                            long long rho_rs, const void* rdiag, long long rdiag_rs,
                            const uint8_t* fixed, int flags, const double* KE,
                            stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !u || !out || !rho || !KE)
    return set_error(STT_ERR_INVALID, "stt_q4_apply: bad sizes or null pointer");
  if ((flags & STT_PROJECT_IN || flags & STT_PROJECT_OUT) && !fixed)
    return set_error(STT_ERR_INVALID, "stt_q4_apply: projection needs the fixed flags");
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == STT_FP64) {
    if (d == 2) return launch_apply<2, double>(nelx, nely, nrows, u, u_rs, out, out_rs, rho, rho_rs, rdiag, rdiag_rs, fixed, flags, KE, st);
    if (d == 1) return launch_apply<1, double>(nelx, nely, nrows, u, u_rs, out, out_rs, rho, rho_rs, rdiag, rdiag_rs, fixed, flags, KE, st);
  } else if (precision == STT_FP32) {
    if (d == 2) return launch_apply<2, float>(nelx, nely, nrows, u, u_rs, out, out_rs, rho, rho_rs, rdiag, rdiag_rs, fixed, flags, KE, st);
    if (d == 1) return launch_apply<1, float>(nelx, nely, nrows, u, u_rs, out, out_rs, rho, rho_rs, rdiag, rdiag_rs, fixed, flags, KE, st);
  }
  return set_error(STT_ERR_INVALID, "stt_q4_apply: d must be 1 or 2, precision FP64 or FP32");
}

extern "C" long long stt_q4_apply_dots_workspace_bytes(int nelx, int nely, int nrows) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0) return 0;
  const dim3 g = q4_grid(nelx, nely, nrows);
  const long long partials = 16LL * nrows * g.x * g.y;  // two doubles a block and row
  return ((partials + 255) & ~255LL) + ((4LL * nrows + 255) & ~255LL);
}

extern "C" int stt_q4_apply_dots(int d, int nelx, int nely, int nrows, const double* u, long long u_rs,
                                 double* out, long long out_rs, const double* rho, long long rho_rs,
                                 const uint8_t* fixed, const double* KE, const double* f, long long f_rs,
                                 double* dots, void* ws, long long ws_bytes, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !u || !out || !rho || !fixed || !KE || !f ||
      !dots || !ws || (d != 1 && d != 2))
    return set_error(STT_ERR_INVALID, "stt_q4_apply_dots: bad sizes or null pointer");
  if (ws_bytes < stt_q4_apply_dots_workspace_bytes(nelx, nely, nrows) || ((uintptr_t)ws & 255) != 0)
    return set_error(STT_ERR_WORKSPACE, "stt_q4_apply_dots: workspace too small or not 256-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid = q4_grid(nelx, nely, nrows);
  const long long partials = 16LL * nrows * grid.x * grid.y;
  GridRed red{(double*)ws, (unsigned*)((char*)ws + ((partials + 255) & ~255LL)), (int)(grid.x * grid.y)};
  STT_TRY(check_cuda(cudaMemsetAsync(red.counters, 0, 4LL * nrows, st), "memset counters"));
  double m[8];
  const bool modal = modal_from_ke(d, KE, m);
  const MQ<double> mq = mq_cast<double>(m);
#define STT_APD(D, MODAL)                                                                                    \
  q4_apply_dots_kernel<D, MODAL><<<grid, kQThreads, 0, st>>>(u, u_rs, out, out_rs, rho, rho_rs, fixed, f, f_rs, \
                                                             dots, red, nelx, nely, make_ke<D, double>(KE), mq)
  if (d == 2) {
    if (modal) STT_APD(2, true);
    else STT_APD(2, false);
  } else {
    if (modal) STT_APD(1, true);
    else STT_APD(1, false);
  }
#undef STT_APD
  return check_launch("q4_apply_dots");
}

extern "C" int stt_adjoint_warm_start(int nrows, long long n, const double* dots, const double* v, long long v_rs,
                                      double* out, long long o_rs, stt_stream_t stream) {
  if (nrows <= 0 || nrows > 65535 || n <= 0 || !dots || !v || !out)
    return set_error(STT_ERR_INVALID, "stt_adjoint_warm_start: bad arguments");
  const long long bx = std::min<long long>((n + 255) / 256, 4LL * 148 * 4 / nrows + 1);
  rows_warm_start_kernel<<<dim3((unsigned)bx, nrows), 256, 0, (cudaStream_t)stream>>>(n, dots, v, v_rs, out, o_rs);
  return check_launch("adjoint_warm_start");
}

extern "C" int stt_set_element_form(int form) {
  if (form != STT_FORM_MODAL && form != STT_FORM_PRODUCT) return -1;
  return element_form().exchange(form);
}

extern "C" int stt_ke_modal(int d, const double* KE, double* m) {
  if (!KE || !m || (d != 1 && d != 2)) return 0;
  double t[8];
  if (!ke_has_modal_form(d, KE, t)) return 0;
  for (int i = 0; i < 8; ++i) m[i] = t[i];
  return 1;
}

extern "C" int stt_q4_diag(int d, int nelx, int nely, int nrows, const double* rho,
                           long long rho_rs, const double* rdiag, long long rdiag_rs,
                           const uint8_t* fixed, double* out, long long out_rs,
                           const double* KE, stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !rho || !out || !KE)
    return set_error(STT_ERR_INVALID, "stt_q4_diag: bad sizes or null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid = q4_grid(nelx, nely, nrows);
  if (d == 2)
    q4_diag_kernel<2><<<grid, kQThreads, 0, st>>>(rho, rho_rs, rdiag, rdiag_rs, fixed, out, out_rs, nelx, nely, make_ke<2, double>(KE));
  else if (d == 1)
    q4_diag_kernel<1><<<grid, kQThreads, 0, st>>>(rho, rho_rs, rdiag, rdiag_rs, fixed, out, out_rs, nelx, nely, make_ke<1, double>(KE));
  else
    return set_error(STT_ERR_INVALID, "stt_q4_diag: d must be 1 or 2");
  return check_launch("q4_diag");
}

extern "C" int stt_lumped_reaction(int d, int nelx, int nely, int nrows, const double* reaction,
                                   long long r_rs, double* out, long long out_rs,
                                   stt_stream_t stream) {
  if (nelx <= 0 || nely <= 0 || nrows <= 0 || nrows > 65535 || !reaction || !out)
    return set_error(STT_ERR_INVALID, "stt_lumped_reaction: bad sizes or null pointer");
  const int nnode = (nelx + 1) * (nely + 1);
  dim3 grid((nnode + 255) / 256, nrows);
  cudaStream_t st = (cudaStream_t)stream;
  if (d == 2)
    lumped_reaction_kernel<2><<<grid, 256, 0, st>>>(reaction, r_rs, out, out_rs, nelx, nely);
  else if (d == 1)
    lumped_reaction_kernel<1><<<grid, 256, 0, st>>>(reaction, r_rs, out, out_rs, nelx, nely);
  else
    return set_error(STT_ERR_INVALID, "stt_lumped_reaction: d must be 1 or 2");
  return check_launch("lumped_reaction");
}
