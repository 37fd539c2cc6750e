// FP64 translation-operator precompute (host C++), writing the reference's
// ld / hd operator files.
//
// The reference builds these offline in MATLAB (matlab/aug3d_script.m,
// aug3d_lowdata.m, aug3d_hghdata.m) and ships none.  This is the project's
// restatement in C++ on its own linear algebra (dense.hpp) and hull
// (hull.hpp):
//   * low frequency, widths 2^-7 .. 2^-1 (aug3d_script.m:25): equivalent and
//     check surfaces of a P^3 grid, the SVD pseudo-inverse of K(ucp, uep)
//     split as {V, 1/sigma, U^H} (aug3d_lowdata.m:35-61), and the 316 FFT'd
//     M2L tensors on the (2P)^3 wrap-around grid (aug3d_lowdata.m:81-105);
//   * high frequency, widths 1, 2, 4, ... (aug3d_script.m:58-68): per
//     canonical wedge (a, b, C), a <= b odd, randomised pivoted-QR skeletons
//     of the far-field interaction plus the middle factor G
//     (aug3d_hghdata.m:18-284), the wedges of one width in parallel.
// MATLAB draws with an unseeded rand; here each wedge has its own xoshiro256**
// stream seeded from (kernel, ACCU, W, wedge), so a file is reproducible and
// independent of the thread count.  Both kernels (exp(2 pi i r)/r and
// exp(2 pi i r), include/kernel3d.hpp:24-27) are supported; the MATLAB only
// wrote helm files (matlab/kernel3d.m:31).
#pragma once
#include <cstdint>
#include <functional>
#include <map>
#include <string>

#include "ops.hpp"

namespace ddfmm {
namespace precompute {

int accu_to_p(int accu);  // 4 / 6 / 8 (aug3d_lowdata.m:23-29)

// Dense kernel matrix K(trg, src) (matlab/kernel3d.m); kind 0: exp(2 pi i r)/r,
// 1: exp(2 pi i r).  The precompute never evaluates coincident pairs.
CMat kernel_matrix(const PMat& trg, const PMat& src, int kind);

// Surface nodes of a P^3 grid on [-L/2, L/2]^3 in ndgrid order, x fastest
// (aug3d_lowdata.m:35-50).
PMat surface_grid(double L, int P);

LowFreqOp low_entry(int accu, double W, int kind);

// One canonical wedge n = (a, b, C) at width W from the child sets pspre /
// ptpre (width W/2: the previous level's uep and -uep, or the low-frequency
// surface of width W/2 at W = 1).
HighFreqOp high_wedge(int accu, double W, int kind, const Idx3& n, const PMat& pspre, const PMat& ptpre,
                      uint64_t seed);

// Seed of a wedge's random stream.
uint64_t wedge_seed(int kind, int accu, double W, const Idx3& n);

// Parent wedge at W/2 of a canonical wedge (aug3d_hghdata_predir.m).
Idx3 predir(const Idx3& n);

std::map<double, LowFreqOp> low_levels(int accu, int kind, int threads);
// Widths 1, 2, 4, ... <= wmax; progress(W, wedges done, wedges of W) after each wedge.
std::map<double, std::map<Idx3, HighFreqOp> > high_levels(
    int accu, int kind, int wmax, int threads, const std::function<void(double, int, int)>& progress = nullptr);

void write_ld(const std::string& path, const std::map<double, LowFreqOp>& ld);
void write_hd(const std::string& path, const std::map<double, std::map<Idx3, HighFreqOp> >& hd);

}  // namespace precompute
}  // namespace ddfmm
