// Separable 3-D DFT standing in for FFTW3 in the oracle build (test
// infrastructure only).  Each axis is transformed with an O(n^2) DFT whose
// twiddles exp(sign*2*pi*i*(jk mod n)/n) are tabulated once per plan in long
// double; n <= 16 for every accuracy level of the reference, so the cost is
// negligible next to the rest of an eval.  Row-major layout, as FFTW's:
// element (i0,i1,i2) sits at (i0*n1 + i1)*n2 + i2.
#include "fftw3.h"
#include <complex>
#include <vector>

struct ddfmm_fftw_plan_s {
    int n[3];
    int sign;
    std::complex<double>* in;
    std::complex<double>* out;
    std::vector<std::complex<double> > tw[3];  // tw[d][j*n+k]
};

extern "C" fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out,
                                      int sign, unsigned) {
    ddfmm_fftw_plan_s* p = new ddfmm_fftw_plan_s;
    p->n[0] = n0; p->n[1] = n1; p->n[2] = n2;
    p->sign = sign;
    p->in = reinterpret_cast<std::complex<double>*>(in);
    p->out = reinterpret_cast<std::complex<double>*>(out);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int d = 0; d < 3; ++d) {
        int n = p->n[d];
        p->tw[d].resize((size_t)n * n);
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                long double a = twopi * (long double)((j * k) % n) / (long double)n;
                p->tw[d][(size_t)j * n + k] =
                    std::complex<double>((double)cosl(a), (double)(sign * sinl(a)));
            }
    }
    return p;
}

extern "C" void fftw_execute(const fftw_plan p) {
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const size_t tot = (size_t)n0 * n1 * n2;
    std::vector<std::complex<double> > a(p->in, p->in + tot), line(16 > n0 ? 16 : n0);
    const int ns[3] = {n0, n1, n2};
    const size_t strides[3] = {(size_t)n1 * n2, (size_t)n2, 1};
    for (int d = 0; d < 3; ++d) {
        const int n = ns[d];
        if ((int)line.size() < n) line.resize(n);
        const size_t st = strides[d];
        for (size_t base = 0; base < tot; ++base) {
            // visit each line once: base has coordinate 0 along axis d
            if ((base / st) % n != 0) continue;
            for (int k = 0; k < n; ++k) {
                std::complex<double> s(0, 0);
                const std::complex<double>* w = &p->tw[d][(size_t)k * n];
                for (int j = 0; j < n; ++j) s += a[base + j * st] * w[j];
                line[k] = s;
            }
            for (int k = 0; k < n; ++k) a[base + k * st] = line[k];
        }
    }
    for (size_t i = 0; i < tot; ++i) p->out[i] = a[i];
}

extern "C" void fftw_destroy_plan(fftw_plan p) { delete p; }
