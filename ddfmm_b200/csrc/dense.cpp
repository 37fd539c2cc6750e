// Dense complex FP64 linear algebra for the operator precompute (dense.hpp).
//
// Hot loops work on the interleaved (re, im) doubles directly: std::complex
// products follow C99 Annex G (inf/nan recovery), which keeps them out of
// vector registers.  The factorizations and the GEMM are compiled twice, for
// x86-64-v3 (AVX2, FMA) and for the baseline, and the loader picks the one
// the host supports.
#include "dense.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>

#if defined(__x86_64__) && defined(__GNUC__)
#define TUNED __attribute__((target_clones("arch=x86-64-v3", "default")))
#else
#define TUNED
#endif

namespace ddfmm {
namespace dense {

namespace {
constexpr double kEps = 2.220446049250313e-16;

inline double* dp(cpx* p) { return reinterpret_cast<double*>(p); }
inline const double* dp(const cpx* p) { return reinterpret_cast<const double*>(p); }

// sum_i conj(v_i) y_i over n entries (four partial sums, so the additions
// of consecutive entries do not wait on one another)
inline cpx dotc(const cpx* v, const cpx* y, int n) {
    const double* a = dp(v);
    const double* b = dp(y);
    double re[4] = {0, 0, 0, 0}, im[4] = {0, 0, 0, 0};
    int i = 0;
    for (; i + 4 <= n; i += 4)
        for (int u = 0; u < 4; ++u) {
            const double ar = a[2 * (i + u)], ai = a[2 * (i + u) + 1], br = b[2 * (i + u)], bi = b[2 * (i + u) + 1];
            re[u] += ar * br + ai * bi;
            im[u] += ar * bi - ai * br;
        }
    for (; i < n; ++i) {
        re[0] += a[2 * i] * b[2 * i] + a[2 * i + 1] * b[2 * i + 1];
        im[0] += a[2 * i] * b[2 * i + 1] - a[2 * i + 1] * b[2 * i];
    }
    return cpx((re[0] + re[1]) + (re[2] + re[3]), (im[0] + im[1]) + (im[2] + im[3]));
}

// y += alpha x over n entries
inline void axpy(cpx alpha, const cpx* x, cpx* y, int n) {
    const double ar = alpha.real(), ai = alpha.imag();
    const double* a = dp(x);
    double* b = dp(y);
    for (int i = 0; i < n; ++i) {
        const double xr = a[2 * i], xi = a[2 * i + 1];
        b[2 * i] += ar * xr - ai * xi;
        b[2 * i + 1] += ar * xi + ai * xr;
    }
}

inline double nrm2sq(const cpx* x, int n) {
    const double* a = dp(x);
    double s[4] = {0, 0, 0, 0};
    int i = 0;
    for (; i + 4 <= 2 * n; i += 4)
        for (int u = 0; u < 4; ++u) s[u] += a[i + u] * a[i + u];
    for (; i < 2 * n; ++i) s[0] += a[i] * a[i];
    return (s[0] + s[1]) + (s[2] + s[3]);
}

// Elementary reflector H = I - tau v v^H with H^H (alpha; x) = (beta; 0), beta
// real, v = (1; x / (alpha - beta)) (LAPACK's zlarfg convention).  x[0] holds
// alpha on entry and beta on return; x[1..len) the tail of v.
cpx reflector(cpx* x, int len) {
    const double xn2 = len > 1 ? nrm2sq(x + 1, len - 1) : 0.0;
    const cpx alpha = x[0];
    if (xn2 == 0.0 && alpha.imag() == 0.0) return cpx(0, 0);
    const double beta = -std::copysign(std::sqrt(std::norm(alpha) + xn2), alpha.real());
    const cpx tau((beta - alpha.real()) / beta, -alpha.imag() / beta);
    const cpx scal = 1.0 / (alpha - beta);
    double* t = dp(x + 1);
    for (int i = 0; i < len - 1; ++i) {
        const double xr = t[2 * i], xi = t[2 * i + 1];
        t[2 * i] = xr * scal.real() - xi * scal.imag();
        t[2 * i + 1] = xr * scal.imag() + xi * scal.real();
    }
    x[0] = cpx(beta, 0);
    return tau;
}

// y -= ctau (v^H y) v with v = (1; vt), over len entries
inline void apply_reflector(const cpx* vt, cpx ctau, cpx* y, int len) {
    cpx w = y[0] + (len > 1 ? dotc(vt, y + 1, len - 1) : cpx(0, 0));
    w *= ctau;
    y[0] -= w;
    if (len > 1) axpy(-w, vt, y + 1, len - 1);
}

// C(m x n) += A(m x k) B(k x n), all column-major with leading dimensions
TUNED void gemm_nn(const cpx* A, int lda, const cpx* B, int ldb, cpx* C, int ldc, int m, int n, int k) {
    constexpr int MB = 192;
    int j0 = 0;
    for (; j0 + 4 <= n; j0 += 4) {
        for (int i0 = 0; i0 < m; i0 += MB) {
            const int i1 = std::min(m, i0 + MB);
            double* c0 = dp(C + (size_t)(j0 + 0) * ldc);
            double* c1 = dp(C + (size_t)(j0 + 1) * ldc);
            double* c2 = dp(C + (size_t)(j0 + 2) * ldc);
            double* c3 = dp(C + (size_t)(j0 + 3) * ldc);
            for (int p = 0; p < k; ++p) {
                const double* a = dp(A + (size_t)p * lda);
                const cpx b0 = B[(size_t)(j0 + 0) * ldb + p], b1 = B[(size_t)(j0 + 1) * ldb + p];
                const cpx b2 = B[(size_t)(j0 + 2) * ldb + p], b3 = B[(size_t)(j0 + 3) * ldb + p];
                const double b0r = b0.real(), b0i = b0.imag(), b1r = b1.real(), b1i = b1.imag();
                const double b2r = b2.real(), b2i = b2.imag(), b3r = b3.real(), b3i = b3.imag();
                for (int i = i0; i < i1; ++i) {
                    const double xr = a[2 * i], xi = a[2 * i + 1];
                    c0[2 * i] += xr * b0r - xi * b0i;
                    c0[2 * i + 1] += xr * b0i + xi * b0r;
                    c1[2 * i] += xr * b1r - xi * b1i;
                    c1[2 * i + 1] += xr * b1i + xi * b1r;
                    c2[2 * i] += xr * b2r - xi * b2i;
                    c2[2 * i + 1] += xr * b2i + xi * b2r;
                    c3[2 * i] += xr * b3r - xi * b3i;
                    c3[2 * i + 1] += xr * b3i + xi * b3r;
                }
            }
        }
    }
    for (; j0 < n; ++j0)
        for (int p = 0; p < k; ++p) axpy(B[(size_t)j0 * ldb + p], A + (size_t)p * lda, C + (size_t)j0 * ldc, m);
}
}  // namespace

CMat zeros(int m, int n) {
    CMat c;
    c.m = m;
    c.n = n;
    c.a.assign((size_t)m * n, cpx(0, 0));
    return c;
}

CMat conj_transpose(const CMat& A) {
    CMat c = zeros(A.n, A.m);
    for (int j = 0; j < A.n; ++j)
        for (int i = 0; i < A.m; ++i) c(j, i) = std::conj(A(i, j));
    return c;
}

CMat take_rows(const CMat& A, const std::vector<int>& rows) {
    CMat c = zeros((int)rows.size(), A.n);
    for (int j = 0; j < A.n; ++j)
        for (size_t i = 0; i < rows.size(); ++i) c((int)i, j) = A(rows[i], j);
    return c;
}

double frob(const CMat& A) { return std::sqrt(nrm2sq(A.a.data(), (int)A.a.size())); }

void gemm_acc(const CMat& A, const CMat& B, CMat& C) {
    if (A.n != B.m || C.m != A.m || C.n != B.n) throw std::invalid_argument("gemm: shapes do not agree");
    if (A.m == 0 || B.n == 0 || A.n == 0) return;
    gemm_nn(A.a.data(), A.m, B.a.data(), B.m, C.a.data(), C.m, A.m, B.n, A.n);
}

CMat gemm(const CMat& A, bool ah, const CMat& B, bool bh) {
    CMat At, Bt;
    const CMat& a = ah ? (At = conj_transpose(A)) : A;
    const CMat& b = bh ? (Bt = conj_transpose(B)) : B;
    CMat C = zeros(a.m, b.n);
    gemm_acc(a, b, C);
    return C;
}

TUNED void qr(const CMat& A0, CMat& Q, CMat& R) {
    const int m = A0.m, n = A0.n;
    if (m < n) throw std::invalid_argument("qr: needs m >= n");
    CMat A = A0;
    std::vector<cpx> tau(n);
    for (int k = 0; k < n; ++k) {
        cpx* col = &A(k, k);
        tau[k] = reflector(col, m - k);
        const cpx ct = std::conj(tau[k]);
        if (ct != cpx(0, 0))
            for (int j = k + 1; j < n; ++j) apply_reflector(col + 1, ct, &A(k, j), m - k);
    }
    R = zeros(n, n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) R(i, j) = A(i, j);
    // Q = H_0 H_1 ... H_{n-1} [I; 0]
    Q = zeros(m, n);
    for (int j = 0; j < n; ++j) Q(j, j) = 1.0;
    for (int k = n - 1; k >= 0; --k) {
        if (tau[k] == cpx(0, 0)) continue;
        const cpx* vt = &A(k, k) + 1;
        for (int j = k; j < n; ++j) apply_reflector(vt, tau[k], &Q(k, j), m - k);
    }
}

// Blocked form (the BLAS-3 pivoted QR of Quintana-Orti, Sun and Bischof, as in
// LAPACK's zlaqps): within a block of up to NB steps the trailing columns are
// not updated; each step updates only its pivot column and pivot row from
// F = tau A^H v (one read-only pass over the trailing matrix), and the block
// ends with one update A -= V F^H.  A block also ends early after a step whose
// norm downdate lost accuracy; those norms are recomputed after the update.
TUNED std::vector<int> qr_pivoted(CMat A, double reltol, std::vector<double>* rdiag) {
    constexpr int NB = 32;
    const int m = A.m, n = A.n, kmax = std::min(m, n);
    std::vector<int> perm(n), piv;
    std::iota(perm.begin(), perm.end(), 0);
    std::vector<double> vn1(n), vn2(n);
    for (int j = 0; j < n; ++j) vn1[j] = vn2[j] = std::sqrt(nrm2sq(&A(0, j), m));
    const double tol3z = std::sqrt(kEps);
    double r00 = 0;
    if (rdiag) rdiag->clear();
    CMat F = zeros(n, NB);  // row c: column c of the matrix; column i: step i of the block
    std::vector<cpx> aux(NB);
    std::vector<int> recompute;
    int k = 0;
    while (k < kmax) {
        const int nb = std::min(NB, kmax - k);
        for (int i = 0; i < nb; ++i) std::fill(&F(0, i), &F(0, i) + n, cpx(0, 0));
        recompute.clear();
        int jb = 0;
        for (int j = 0; j < nb; ++j) {
            const int kk = k + j;
            const int p = kk + (int)(std::max_element(vn1.begin() + kk, vn1.end()) - (vn1.begin() + kk));
            if (p != kk) {
                std::swap_ranges(&A(0, p), &A(0, p) + m, &A(0, kk));
                std::swap(perm[p], perm[kk]);
                vn1[p] = vn1[kk];
                vn2[p] = vn2[kk];
                for (int i = 0; i < j; ++i) std::swap(F(p, i), F(kk, i));
            }
            // pivot column: apply this block's earlier reflectors, A(kk:, kk) -= V(kk:, 0:j) F(kk, 0:j)^H
            for (int i = 0; i < j; ++i) {
                const cpx f = std::conj(F(kk, i));
                if (f != cpx(0, 0)) axpy(-f, &A(kk, k + i), &A(kk, kk), m - kk);
            }
            cpx* col = &A(kk, kk);
            const cpx tau = reflector(col, m - kk);
            const double rkk = std::abs(col[0]);
            if (kk == 0) {
                r00 = rkk;
                if (r00 == 0) return piv;
            }
            if (rkk <= reltol * r00) return piv;
            piv.push_back(perm[kk]);
            if (rdiag) rdiag->push_back(rkk);
            jb = j + 1;
            if (kk + 1 >= kmax) break;
            // F(c, j) = tau (A(kk:, c)^H v) for the trailing columns, v = (1; col[1..])
            const cpx beta = col[0];
            col[0] = 1.0;
            for (int c = kk + 1; c < n; ++c) F(c, j) = tau * std::conj(dotc(col, &A(kk, c), m - kk));
            // F(:, j) -= tau F(:, 0:j) (V(kk:, 0:j)^H v)
            if (j > 0) {
                for (int i = 0; i < j; ++i) aux[i] = -tau * dotc(&A(kk, k + i), col, m - kk);
                for (int i = 0; i < j; ++i)
                    if (aux[i] != cpx(0, 0))
                        for (int c = kk + 1; c < n; ++c) F(c, j) += F(c, i) * aux[i];
            }
            // pivot row: A(kk, c) -= sum_{i <= j} V(kk, i) conj(F(c, i)), V(kk, j) = 1
            for (int c = kk + 1; c < n; ++c) {
                cpx s(0, 0);
                for (int i = 0; i <= j; ++i) s += A(kk, k + i) * std::conj(F(c, i));
                A(kk, c) -= s;
            }
            col[0] = beta;
            // norm downdate from the updated pivot row
            bool lost = false;
            for (int c = kk + 1; c < n; ++c) {
                if (vn1[c] == 0) continue;
                double t = std::abs(A(kk, c)) / vn1[c];
                t = std::max(0.0, (1.0 + t) * (1.0 - t));
                const double r = vn1[c] / vn2[c];
                if (t * r * r <= tol3z) {
                    recompute.push_back(c);
                    vn1[c] = 0;  // not a pivot candidate until recomputed
                    lost = true;
                } else {
                    vn1[c] *= std::sqrt(t);
                }
            }
            if (lost) break;
        }
        const int kend = k + jb;
        if (kend >= kmax) break;
        // trailing update A(kend:, kend:) -= V(kend:, 0:jb) F(kend:, 0:jb)^H
        if (m > kend && n > kend) {
            CMat Fh = zeros(jb, n - kend);
            for (int c = kend; c < n; ++c)
                for (int i = 0; i < jb; ++i) Fh(i, c - kend) = -std::conj(F(c, i));
            gemm_nn(&A(kend, k), m, Fh.a.data(), jb, &A(kend, kend), m, m - kend, n - kend, jb);
        }
        for (int c : recompute) {
            vn1[c] = kend < m ? std::sqrt(nrm2sq(&A(kend, c), m - kend)) : 0.0;
            vn2[c] = vn1[c];
        }
        k = kend;
    }
    return piv;
}

TUNED void svd(const CMat& A, CMat& U, std::vector<double>& s, CMat& V) {
    const int m = A.m, n = A.n;
    if (m < n) throw std::invalid_argument("svd: needs m >= n");
    CMat Q, X;
    qr(A, Q, X);  // A = Q X, X n x n
    V = zeros(n, n);
    for (int j = 0; j < n; ++j) V(j, j) = 1.0;
    std::vector<double> nrm(n);
    for (int j = 0; j < n; ++j) nrm[j] = nrm2sq(&X(0, j), n);
    const double tol = kEps;
    for (int sweep = 0; sweep < 60; ++sweep) {
        bool rotated = false;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double alpha = nrm[p], beta = nrm[q];
                if (alpha == 0 || beta == 0) continue;
                const cpx gamma = dotc(&X(0, p), &X(0, q), n);
                const double g = std::abs(gamma);
                if (g <= tol * std::sqrt(alpha * beta)) continue;
                rotated = true;
                const cpx e = gamma / g;
                const double zeta = (beta - alpha) / (2 * g);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::abs(zeta) + std::sqrt(1 + zeta * zeta));
                const double c = 1 / std::sqrt(1 + t * t), sn = c * t;
                const cpx ce = std::conj(e);
                // [x_p, x_q] <- [c x_p - s conj(e) x_q, s x_p + c conj(e) x_q]; the same for V
                auto rot = [&](cpx* xp, cpx* xq, int len) {
                    double* a = dp(xp);
                    double* b = dp(xq);
                    const double er = ce.real(), ei = ce.imag();
                    for (int i = 0; i < len; ++i) {
                        const double pr = a[2 * i], pi = a[2 * i + 1];
                        const double qr_ = b[2 * i] * er - b[2 * i + 1] * ei, qi = b[2 * i] * ei + b[2 * i + 1] * er;
                        a[2 * i] = c * pr - sn * qr_;
                        a[2 * i + 1] = c * pi - sn * qi;
                        b[2 * i] = sn * pr + c * qr_;
                        b[2 * i + 1] = sn * pi + c * qi;
                    }
                };
                rot(&X(0, p), &X(0, q), n);
                rot(&V(0, p), &V(0, q), n);
                nrm[p] = nrm2sq(&X(0, p), n);
                nrm[q] = nrm2sq(&X(0, q), n);
            }
        if (!rotated) break;
    }
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::vector<double> sv(n);
    for (int j = 0; j < n; ++j) sv[j] = std::sqrt(nrm2sq(&X(0, j), n));
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return sv[a] > sv[b]; });
    CMat UR = zeros(n, n), Vs = zeros(n, n);
    s.assign(n, 0.0);
    for (int jj = 0; jj < n; ++jj) {
        const int j = ord[jj];
        s[jj] = sv[j];
        for (int i = 0; i < n; ++i) {
            UR(i, jj) = sv[j] > 0 ? X(i, j) / sv[j] : cpx(0, 0);
            Vs(i, jj) = V(i, j);
        }
    }
    V = std::move(Vs);
    U = gemm(Q, false, UR, false);
}

CMat pinv(const CMat& A) {
    if (A.m < A.n) return conj_transpose(pinv(conj_transpose(A)));
    CMat U, V;
    std::vector<double> s;
    svd(A, U, s, V);
    const double cut = std::max(A.m, A.n) * kEps * (s.empty() ? 0.0 : s[0]);
    int r = 0;
    while (r < (int)s.size() && s[r] > cut) ++r;
    // V(:, :r) diag(1/s) U(:, :r)^H
    CMat Vs = zeros(A.n, r), Ur = zeros(A.m, r);
    for (int j = 0; j < r; ++j) {
        for (int i = 0; i < A.n; ++i) Vs(i, j) = V(i, j) / s[j];
        for (int i = 0; i < A.m; ++i) Ur(i, j) = U(i, j);
    }
    return gemm(Vs, false, Ur, true);
}

CMat inv_triangular(const CMat& R, bool lower) {
    const int n = R.n;
    if (R.m != n) throw std::invalid_argument("inv_triangular: not square");
    CMat X = zeros(n, n);
    for (int j = 0; j < n; ++j) {
        if (!lower) {
            for (int i = j; i >= 0; --i) {  // rows j..0 of column j
                cpx acc = (i == j) ? cpx(1, 0) : cpx(0, 0);
                for (int k = i + 1; k <= j; ++k) acc -= R(i, k) * X(k, j);
                X(i, j) = acc / R(i, i);
            }
        } else {
            for (int i = j; i < n; ++i) {
                cpx acc = (i == j) ? cpx(1, 0) : cpx(0, 0);
                for (int k = j; k < i; ++k) acc -= R(i, k) * X(k, j);
                X(i, j) = acc / R(i, i);
            }
        }
    }
    return X;
}

}  // namespace dense
}  // namespace ddfmm
