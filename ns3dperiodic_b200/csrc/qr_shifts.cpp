// Host-side implicit shifted QR on the small Hessenberg matrix of the
// implicitly restarted Arnoldi method (QR_shifts,
// Source/Arnoldi/QR_Shifts.cpp:7-72).
//
// The reference forms each orthogonal factor with LAPACK (dgeqrf, then
// dormqr applied to the identity; Source/Arnoldi/LAPACK_routines.cpp:289-345).
// This file has its own Householder QR with LAPACK's conventions: reflector
// H_i = I - tau_i v_i v_i^T with v_i(i) = 1, beta = -sign(alpha) ||(alpha, x)||,
// tau = (beta - alpha) / beta, v = x / (alpha - beta) (the dlarfg
// definition), reflectors applied left to right to the trailing columns, and
// Q = H_0 H_1 ... H_{m-1} formed by applying them in reverse order to the
// identity (dorm2r with SIDE = L, TRANS = N).  Dense products follow the
// reference's triple loop (Source/Arnoldi/Products.cpp:69-86) and its
// accumulation order.  m is small (tens), so this is microseconds of host
// work per restart.
#include <cmath>
#include <vector>

#include "ns3d.h"

namespace {

inline double& at(std::vector<double>& a, int m, int i, int j) { return a[i + (size_t)j * m]; }

// C = A B, all m x m column-major, sum over k in increasing order.
void matmul(const double* A, const double* B, double* C, int m) {
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      double s = 0.0;
      for (int k = 0; k < m; ++k) s += A[i + (size_t)k * m] * B[k + (size_t)j * m];
      C[i + (size_t)j * m] = s;
    }
}

// Householder QR of the m x m matrix A (column-major, overwritten with R and
// the reflector tails), then Q formed explicitly.
void householder_q(std::vector<double>& A, int m, std::vector<double>& Q) {
  std::vector<double> tau(m, 0.0), w(m, 0.0);
  for (int i = 0; i < m; ++i) {
    double& alpha = at(A, m, i, i);
    double xnorm2 = 0.0;
    for (int r = i + 1; r < m; ++r) xnorm2 += at(A, m, r, i) * at(A, m, r, i);
    if (xnorm2 == 0.0) {
      tau[i] = 0.0;
    } else {
      const double beta = -std::copysign(std::hypot(alpha, std::sqrt(xnorm2)), alpha);
      tau[i] = (beta - alpha) / beta;
      const double scal = 1.0 / (alpha - beta);
      for (int r = i + 1; r < m; ++r) at(A, m, r, i) *= scal;
      alpha = beta;
    }
    if (tau[i] == 0.0 || i == m - 1) continue;
    // apply H_i to A(i:m, i+1:m): w = A^T v, A -= tau v w^T
    for (int j = i + 1; j < m; ++j) {
      double s = at(A, m, i, j);
      for (int r = i + 1; r < m; ++r) s += at(A, m, r, i) * at(A, m, r, j);
      w[j] = s;
    }
    for (int j = i + 1; j < m; ++j) {
      const double tw = tau[i] * w[j];
      at(A, m, i, j) -= tw;
      for (int r = i + 1; r < m; ++r) at(A, m, r, j) -= at(A, m, r, i) * tw;
    }
  }
  Q.assign((size_t)m * m, 0.0);
  for (int i = 0; i < m; ++i) at(Q, m, i, i) = 1.0;
  for (int i = m - 1; i >= 0; --i) {
    if (tau[i] == 0.0) continue;
    // Q(i:m, :) = H_i Q(i:m, :)
    for (int j = 0; j < m; ++j) {
      double s = at(Q, m, i, j);
      for (int r = i + 1; r < m; ++r) s += at(A, m, r, i) * at(Q, m, r, j);
      const double tw = tau[i] * s;
      at(Q, m, i, j) -= tw;
      for (int r = i + 1; r < m; ++r) at(Q, m, r, j) -= at(A, m, r, i) * tw;
    }
  }
}

// One QR step of QR_step (QR_Shifts.cpp:7-40): Qacc <- Qacc Q, H <- Q^T H Q.
void qr_step(double* Qacc, double* H, double er, double ei, int m) {
  std::vector<double> H1((size_t)m * m), H2((size_t)m * m), Q, QT((size_t)m * m);
  for (size_t e = 0; e < H1.size(); ++e) H1[e] = H[e];
  for (int i = 0; i < m; ++i) at(H1, m, i, i) -= er;
  if (std::fabs(ei) > 1.0e-15) {
    matmul(H1.data(), H1.data(), H2.data(), m);
    for (int i = 0; i < m; ++i) at(H2, m, i, i) += ei * ei;
    H1.swap(H2);
  }
  householder_q(H1, m, Q);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) at(QT, m, i, j) = at(Q, m, j, i);
  matmul(QT.data(), H, H2.data(), m);  // Q^T H
  matmul(H2.data(), Q.data(), H, m);   // (Q^T H) Q
  for (int j = 0; j < m - 1; ++j)
    for (int i = m - 1; i > j + 1; --i) H[i + (size_t)j * m] = 0.0;
  matmul(Qacc, Q.data(), H2.data(), m);
  for (size_t e = 0; e < H2.size(); ++e) Qacc[e] = H2[e];
}

}  // namespace

extern "C" ns3d_status ns3d_qr_shifts(int k, int m, double* Q, double* H, const double* eig_re,
                                      const double* eig_im, int* ko) {
  if (!Q || !H || !eig_re || !eig_im || !ko || m < 1 || k < 0 || k > m) return NS3D_ERR_BAD_ARG;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) Q[i + (size_t)j * m] = (i == j) ? 1.0 : 0.0;
  int j = m;
  while (j > k) {
    const double er = eig_re[j - 1], ei = eig_im[j - 1];
    qr_step(Q, H, er, ei, m);
    // the reference tests the step width in single precision (fabsf)
    j -= (std::fabs(static_cast<float>(ei)) > 1.0e-15) ? 2 : 1;
  }
  *ko = j;
  return NS3D_OK;
}
