/* oracle_kernels.c -- TEST INFRASTRUCTURE ONLY: C/OpenMP loops of the CPU oracle.
 *
 * The oracle (sttopt_oracle.py) restates the reference's FEM solve path in NumPy; these
 * are its three hottest loops written in C so that the oracle can run the benchmark's
 * full-size workload as the timed CPU baseline.  Same arithmetic as the NumPy forms
 * they replace (sttopt_oracle.py: matvec, keff_matvec, VCycle._smooth and the PCG's row
 * reductions and updates); only the summation order differs.  Nothing in the product
 * path links this file.
 *
 * Structured Q4 grids only (the reference's element_dof_map, sttopt/fem.py:72-95): node
 * n = row * (nelx + 1) + col with row 0 at the top, element corners BL, BR, TR, TL, d
 * interleaved dofs per node.  Vectors are batch rows with explicit row strides (in
 * doubles; stride 0 broadcasts one row).
 */
#include <stddef.h>
#include <string.h>

/* Loops over fewer values than this run on one thread (OpenMP's fork and join cost more
 * than the work on the small test grids). */
#define ORC_PAR_MIN (1LL << 17)

/* out[s] = sum over elements e of scatter(w[s][e] * (U_e[s]^T M_e[s])) -- the element
 * product of torch_fem.matvec (sttopt/torch_fem.py:62-83; M = KE shared, m_es = m_rs =
 * 0, w the SIMP densities) and torch_mg.keff_matvec (sttopt/torch_mg.py:179-193; M the
 * explicit element matrices, m_es = k * k, w NULL).  The elements are split into four
 * colours by (row parity, column parity): elements of one colour share no node, so a
 * colour's elements accumulate in parallel without atomics. */
void orc_element_apply(int nrows, int nelx, int nely, int d, const double* U, long long u_rs,
                       const double* M, long long m_es, long long m_rs, const double* w,
                       long long w_rs, double* out, long long o_rs) {
  const int k = 4 * d;
  const long long nnx = nelx + 1;
  const long long ndof = (long long)d * nnx * (nely + 1);
  const int par = (long long)nrows * ndof > ORC_PAR_MIN;
#pragma omp parallel for schedule(static) if (par)
  for (int s = 0; s < nrows; ++s) memset(out + (size_t)s * o_rs, 0, sizeof(double) * (size_t)ndof);
  for (int colour = 0; colour < 4; ++colour) {
    const int ry = colour >> 1, rx = colour & 1;
    const int nrow_c = (nely - ry + 1) / 2;
#pragma omp parallel for collapse(2) schedule(static) if (par)
    for (int s = 0; s < nrows; ++s) {
      for (int j = 0; j < nrow_c; ++j) {
        const int er = ry + 2 * j;
        const double* Us = U + (size_t)s * u_rs;
        double* Os = out + (size_t)s * o_rs;
        for (int ec = rx; ec < nelx; ec += 2) {
          const long long e = (long long)er * nelx + ec;
          const long long corner[4] = {(er + 1) * nnx + ec, (er + 1) * nnx + ec + 1, er * nnx + ec + 1,
                                       er * nnx + ec};
          long long dof[8];
          double ue[8], ve[8];
          for (int q = 0; q < 4; ++q)
            for (int i = 0; i < d; ++i) dof[q * d + i] = corner[q] * d + i;
          for (int a = 0; a < k; ++a) ue[a] = Us[dof[a]];
          const double* Me = M + (size_t)s * m_rs + (size_t)e * m_es;
          for (int b = 0; b < k; ++b) ve[b] = 0.0;
          for (int a = 0; a < k; ++a) {
            const double ua = ue[a];
            for (int b = 0; b < k; ++b) ve[b] += ua * Me[a * k + b];
          }
          const double we = w ? w[(size_t)s * w_rs + e] : 1.0;
          for (int b = 0; b < k; ++b) Os[dof[b]] += ve[b] * we;
        }
      }
    }
  }
}

/* One damped-Jacobi sweep's update (torch_mg.VCycle._smooth, sttopt/torch_mg.py:440-443):
 * x = x + omega * (b - Ax) / diag, in place, rows with their strides. */
void orc_jacobi_update(int nrows, long long n, double* x, long long x_rs, const double* b, long long b_rs,
                       const double* Ax, long long a_rs, const double* diag, long long g_rs, double omega) {
#pragma omp parallel for collapse(2) schedule(static) if ((long long)nrows * n > ORC_PAR_MIN)
  for (int s = 0; s < nrows; ++s)
    for (long long i = 0; i < n; ++i) {
      double* xs = x + (size_t)s * x_rs;
      xs[i] += omega * (b[(size_t)s * b_rs + i] - Ax[(size_t)s * a_rs + i]) / diag[(size_t)s * g_rs + i];
    }
}

/* out[s] = sum_i a[s][i] * b[s][i] (the PCG's r.z, p.Ap and norms; sttopt/torch_fem.py:253-331). */
void orc_row_dots(int nrows, long long n, const double* a, long long a_rs, const double* b, long long b_rs,
                  double* out) {
  for (int s = 0; s < nrows; ++s) {
    const double* as = a + (size_t)s * a_rs;
    const double* bs = b + (size_t)s * b_rs;
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static) if (n > ORC_PAR_MIN)
    for (long long i = 0; i < n; ++i) acc += as[i] * bs[i];
    out[s] = acc;
  }
}

/* y[s] = y[s] + alpha[s] * x[s] (the PCG's x and r updates; alpha = -alpha for r). */
void orc_row_axpy(int nrows, long long n, const double* alpha, const double* x, long long x_rs, double* y,
                  long long y_rs) {
#pragma omp parallel for collapse(2) schedule(static) if ((long long)nrows * n > ORC_PAR_MIN)
  for (int s = 0; s < nrows; ++s)
    for (long long i = 0; i < n; ++i) y[(size_t)s * y_rs + i] += alpha[s] * x[(size_t)s * x_rs + i];
}

/* p[s] = z[s] + beta[s] * p[s] (the PCG's search direction update). */
void orc_row_xpay(int nrows, long long n, const double* z, long long z_rs, const double* beta, double* p,
                  long long p_rs) {
#pragma omp parallel for collapse(2) schedule(static) if ((long long)nrows * n > ORC_PAR_MIN)
  for (int s = 0; s < nrows; ++s)
    for (long long i = 0; i < n; ++i) {
      double* ps = p + (size_t)s * p_rs;
      ps[i] = ps[i] * beta[s] + z[(size_t)s * z_rs + i];
    }
}
