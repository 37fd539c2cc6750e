// Shim self-test (oracle infrastructure): reads a (2P)^3 complex grid and a
// small complex matrix/vector from stdin as text, prints the forward and
// backward 3-D DFT and zgemv results so a test can compare them with numpy.
#include "fftw3.h"
#include <complex>
#include <cstdio>
#include <vector>
typedef std::complex<double> zc;
extern "C" void zgemv_(char*, int*, int*, zc*, zc*, int*, zc*, int*, zc*, zc*, int*);
int main() {
    int n;
    if (scanf("%d", &n) != 1) return 1;
    std::vector<zc> g((size_t)n * n * n), h;
    for (auto& v : g) { double re, im; if (scanf("%lf %lf", &re, &im) != 2) return 1; v = zc(re, im); }
    h = g;
    fftw_plan f = fftw_plan_dft_3d(n, n, n, (fftw_complex*)g.data(), (fftw_complex*)g.data(), FFTW_FORWARD, FFTW_MEASURE);
    fftw_plan b = fftw_plan_dft_3d(n, n, n, (fftw_complex*)h.data(), (fftw_complex*)h.data(), FFTW_BACKWARD, FFTW_ESTIMATE);
    fftw_execute(f); fftw_execute(b);
    for (auto& v : g) printf("%.17e %.17e\n", v.real(), v.imag());
    for (auto& v : h) printf("%.17e %.17e\n", v.real(), v.imag());
    int m, k;
    if (scanf("%d %d", &m, &k) != 2) return 1;
    std::vector<zc> A((size_t)m * k), x(k), y(m);
    for (auto& v : A) { double re, im; if (scanf("%lf %lf", &re, &im) != 2) return 1; v = zc(re, im); }
    for (auto& v : x) { double re, im; if (scanf("%lf %lf", &re, &im) != 2) return 1; v = zc(re, im); }
    for (auto& v : y) { double re, im; if (scanf("%lf %lf", &re, &im) != 2) return 1; v = zc(re, im); }
    char t = 'N'; int one = 1; zc al(1.0, 0.0), be(1.0, 0.0);
    zgemv_(&t, &m, &k, &al, A.data(), &m, x.data(), &one, &be, y.data(), &one);
    for (auto& v : y) printf("%.17e %.17e\n", v.real(), v.imag());
    fftw_destroy_plan(f); fftw_destroy_plan(b);
    return 0;
}
