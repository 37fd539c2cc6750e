// Dense complex FP64 linear algebra for the operator precompute (host only).
//
// The reference builds its operators offline with MATLAB's svd, qr (LAPACK)
// and pinv (matlab/aug3d_lowdata.m:57, aug3d_hghdata.m:194-239).  This file
// holds the project's own versions of those factorizations:
//   * Householder QR (economic, explicit Q) and column-pivoted Householder QR
//     stopped at the first pivot below a relative threshold;
//   * one-sided (Hestenes) Jacobi SVD, after a QR of the input;
//   * the Moore-Penrose pseudo-inverse and the inverse of a triangular factor;
//   * a cache-blocked complex GEMM with optional conjugate transposes.
// Matrices are CMat (ops.hpp): column-major std::complex<double>.
#pragma once
#include <vector>

#include "ops.hpp"

namespace ddfmm {
namespace dense {

CMat zeros(int m, int n);
CMat conj_transpose(const CMat& A);
// Rows `rows` of A, in that order.
CMat take_rows(const CMat& A, const std::vector<int>& rows);
double frob(const CMat& A);

// C = op(A) op(B); op(X) = X, or X^H when the flag is set.
CMat gemm(const CMat& A, bool ah, const CMat& B, bool bh);
// C += A B (no transposes), shapes must agree.
void gemm_acc(const CMat& A, const CMat& B, CMat& C);

// Economic Householder QR of A (m x n, m >= n): A = Q R with Q m x n
// (orthonormal columns) and R n x n upper triangular.  R's diagonal is real
// (the reflector convention of LAPACK's zgeqrf: beta = -sign(Re a) |x|).
void qr(const CMat& A, CMat& Q, CMat& R);

// Column-pivoted Householder QR of A (m x n), pivot = column of largest
// remaining norm (norms downdated, recomputed on cancellation as LAPACK's
// zlaqp2 does), stopped at the first step whose |R_kk| <= reltol |R_00|.
// Returns the chosen columns in pivot order (the skeleton); rdiag, if given,
// receives |R_kk| of the accepted steps.
std::vector<int> qr_pivoted(CMat A, double reltol, std::vector<double>* rdiag = nullptr);

// Thin SVD of A (m x n, m >= n): A = U diag(s) V^H with U m x n, V n x n and
// s descending.  A QR of A first, then one-sided Jacobi rotations on R until
// every column pair is orthogonal to machine precision.
void svd(const CMat& A, CMat& U, std::vector<double>& s, CMat& V);

// Moore-Penrose pseudo-inverse (n x m) of A (m x n, any shape); singular
// values at or below max(m, n) * eps * s_max are dropped (MATLAB's pinv
// default tolerance).
CMat pinv(const CMat& A);

// Inverse of the upper triangular R (n x n); lower = true for a lower
// triangular input.
CMat inv_triangular(const CMat& R, bool lower = false);

}  // namespace dense
}  // namespace ddfmm
