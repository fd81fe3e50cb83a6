// Host-side recognition of the modal form of a Q4 element matrix (see march_modal in
// q4.cuh): KE = T^T M T with T the +-1 edge-mode map of the unit-square bilinear
// element and M of the sparsity the kernels implement.
//
// Corner order BL, BR, TR, TL and interleaved dofs (sttopt/fem.py:72-95).  Modes per
// displacement component: Gx (pattern -1, +1, +1, -1), Gy (-1, -1, +1, +1) and H
// (+1, -1, +1, -1); these rows are orthogonal with squared norm 4, so the least-squares
// M is T KE T^T / 16.  The KE is accepted only when T^T M T, rebuilt from the constants
// the kernels use, reproduces it to 1e-12 of its largest entry and its diagonal is the
// same at every corner; otherwise the caller uses the generic 8 x 8 product.
//
// stt_set_element_form(STT_FORM_PRODUCT) refuses every KE, so that the library applies
// element matrices as the reference does (the 8 x 8 product of the corner values).  The
// two forms round differently: the modal form annihilates rigid translations exactly,
// while a float64 KE gives them a stiffness of ~1e-16 per element, which shifts the
// compliance of large-displacement problems by ~1e-9 relative (measured on the 1024 x 512
// cantilever); the product form reproduces the reference's results to ~1e-12.
#pragma once

#include <atomic>
#include <cmath>

namespace stt {

inline std::atomic<int>& element_form() {
  static std::atomic<int> form{0};  // STT_FORM_MODAL
  return form;
}

inline bool generic_ke_forced() { return element_form().load(std::memory_order_relaxed) != 0; }

// m[8] = {m00, m01, m11, m22, m44, m55, kd0, kd1} in the meaning of MQ (q4.cuh).
// Recognition only; modal_from_ke below also honours the selected element form.
inline bool ke_has_modal_form(int d, const double* KE, double m[8]) {
  if (d != 1 && d != 2) return false;
  static const double pat[3][4] = {{-1, 1, 1, -1}, {-1, -1, 1, 1}, {1, -1, 1, -1}};  // Gx, Gy, H
  const int n = 4 * d, nm = 3 * d;
  // T[mode][dof]; D = 2 modes: Gx(ux), Gy(uy), Gy(ux), Gx(uy), H(ux), H(uy); D = 1: Gx, Gy, H
  double T[6][8] = {};
  for (int k = 0; k < 4; ++k) {
    if (d == 2) {
      T[0][2 * k] = pat[0][k];
      T[1][2 * k + 1] = pat[1][k];
      T[2][2 * k] = pat[1][k];
      T[3][2 * k + 1] = pat[0][k];
      T[4][2 * k] = pat[2][k];
      T[5][2 * k + 1] = pat[2][k];
    } else {
      for (int i = 0; i < 3; ++i) T[i][k] = pat[i][k];
    }
  }
  double kmax = 0.0;
  for (int i = 0; i < n * n; ++i) kmax = std::fmax(kmax, std::fabs(KE[i]));
  if (!(kmax > 0.0) || !std::isfinite(kmax)) return false;
  double M[6][6] = {};
  for (int a = 0; a < nm; ++a)
    for (int b = 0; b < nm; ++b) {
      double s = 0.0;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) s += T[a][i] * KE[i * n + j] * T[b][j];
      M[a][b] = s / 16.0;
    }
  // the M the kernels implement
  double R[6][6] = {};
  if (d == 2) {
    m[0] = M[0][0];
    m[1] = 0.5 * (M[0][1] + M[1][0]);
    m[2] = M[1][1];
    m[3] = (M[2][2] + M[3][3] + M[2][3] + M[3][2]) / 4.0;
    m[4] = M[4][4];
    m[5] = M[5][5];
    R[0][0] = m[0];
    R[0][1] = R[1][0] = m[1];
    R[1][1] = m[2];
    R[2][2] = R[2][3] = R[3][2] = R[3][3] = m[3];
    R[4][4] = m[4];
    R[5][5] = m[5];
  } else {
    m[0] = M[0][0];
    m[1] = 0.0;
    m[2] = M[1][1];
    m[3] = M[2][2];
    m[4] = m[5] = 0.0;
    R[0][0] = m[0];
    R[1][1] = m[2];
    R[2][2] = m[3];
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int a = 0; a < nm; ++a)
        for (int b = 0; b < nm; ++b) s += T[a][i] * R[a][b] * T[b][j];
      if (!(std::fabs(s - KE[i * n + j]) <= 1e-12 * kmax)) return false;
    }
  for (int i = 0; i < d; ++i) {
    const double k0 = KE[i * n + i];
    for (int k = 1; k < 4; ++k)
      if (!(std::fabs(KE[(k * d + i) * n + k * d + i] - k0) <= 1e-14 * kmax)) return false;
    m[6 + i] = k0;
  }
  if (d == 1) m[7] = 0.0;
  return true;
}

// The kernels' choice: the modal form when KE has it and the modal element form is
// selected (stt_set_element_form).
inline bool modal_from_ke(int d, const double* KE, double m[8]) {
  return !generic_ke_forced() && ke_has_modal_form(d, KE, m);
}

}  // namespace stt
