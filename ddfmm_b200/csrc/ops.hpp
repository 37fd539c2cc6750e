// Translation operators read from the reference's ld/hd operator files.
//
// File layouts (Mlib3d::setup, src/mlib3d.cpp:70-103; element formats
// include/serialize.hpp):
//   ld: map<double W, {DblNumMat uep, DblNumMat ucp, NumVec<CpxNumMat> uc2ue,
//                      NumTns<CpxNumTns> ue2dc (7x7x7)}>   (mlib3d.cpp:361-379)
//   hd: map<double W, map<Index3 wedge, {DblNumMat uep, DblNumMat ucp,
//                      NumVec<CpxNumMat> uc2ue}>>          (mlib3d.cpp:382-405)
// Matrices are column-major; points are 3 x n (coordinate fastest).
#pragma once
#include <complex>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "tree.hpp"

namespace ddfmm {

typedef std::complex<double> cpx;

struct CMat {
    int m = 0, n = 0;
    std::vector<cpx> a;  // column-major
    cpx& operator()(int i, int j) { return a[(size_t)j * m + i]; }
    const cpx& operator()(int i, int j) const { return a[(size_t)j * m + i]; }
};

struct PMat {  // 3 x n points
    int n = 0;
    std::vector<double> x;  // x[3*k + d]
};

struct LowFreqOp {
    double W = 0;
    PMat uep, ucp;
    CMat v, is, up;                   // uc2ue = {v, 1/sigma, U^H}
    std::vector<std::vector<cpx> > ue2dc;  // 343 tensors (2P)^3, empty when near
    int tdim = 0;                     // 2P
};

struct HighFreqOp {
    PMat uep, ucp;   // skeleton source (r1) / target (r2) points
    CMat E1, E2, E3; // uc2ue = {E1, E2, E3}
};

struct OperatorLib {
    std::map<double, LowFreqOp> ld;
    std::map<double, std::map<Idx3, HighFreqOp> > hd;
    void load(const std::string& ld_path, const std::string& hd_path);
    // The files as loaded once per process: sessions of the same files share one
    // read-only copy while any of them holds it (keyed by path, size and
    // modification time of both files, so a rewritten file is read again).
    static std::shared_ptr<const OperatorLib> shared(const std::string& ld_path, const std::string& hd_path);
    // Shapes every entry must have for accuracy level `accu` (P = 4/6/8): LF
    // surfaces of P^3 - (P-2)^3 points, uc2ue factors v (n x r), 1/sigma (r x 1),
    // U^H (r x n), ue2dc tensors of edge 2P (or empty); HF factors E1 (r1 x r1),
    // E2 (r1 x r2), E3 (r2 x r2) for r1 / r2 skeleton points, r1, r2 <= 400
    // (DVMAX, src/wave3d_eval.cpp:25).  Throws with the first violation.
    void validate(int accu) const;
    const LowFreqOp& low(double W) const;
    const HighFreqOp& high(double W, const Idx3& canon) const;
};

}  // namespace ddfmm
