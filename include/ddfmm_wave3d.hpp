// Header-only C++ drop-in for the reference's Wave3d evaluation path, on the
// C ABI of libddfmm_b200 (include/ddfmm.h).
//
// Mirrors the member API the reference's driver uses (include/wave3d.hpp:
// 219-265, src/tt.cpp:103-185):
//
//   ddfmm_b200::Mlib3d mlib("mlib3d_");   mlib.kernel() = k;   mlib.setup(opts);
//   ddfmm_b200::Wave3d wave("wave3d_");
//   wave.posptr() = &pos.lclmap();   // std::map<int, Point3> (ParVec's local map)
//   wave.kernel() = k;  wave.mlibptr() = &mlib;  wave.geomprtn() = geomprtn.m();
//   wave.setup(opts);                // -wave3d_ACCU / NPQ / K / ctr / ptsmax / maxlevel
//   wave.eval(den.lclmap(), val.lclmap());
//   wave.check(den.lclmap(), val.lclmap(), chkkeys, relerr);
//
// Point ids must be 0..N-1 (one rank holds every point, as the reference's
// single-rank runs do).  Failures throw `new std::exception()` exactly like
// the reference's SAFE_FUNC_EVAL / CHECK_TRUE (include/commoninc.hpp:52-53);
// ddfmm_last_error() holds the reason.  Unlike the reference, eval() may be
// called repeatedly on one object: values do not accumulate.
#ifndef DDFMM_B200_WAVE3D_HPP
#define DDFMM_B200_WAVE3D_HPP

#include <cmath>
#include <complex>
#include <exception>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ddfmm.h"

namespace ddfmm_b200 {

typedef std::complex<double> cpx;

inline void raise_if(int rc) {
    if (rc != DDFMM_OK) throw new std::exception();
}

template <class T>
inline void read_opt(std::map<std::string, std::string>& opts, const std::string& key, T& v) {
    std::map<std::string, std::string>::iterator it = opts.find(key);
    if (it != opts.end()) {
        std::istringstream ss(it->second);
        ss >> v;
    }
}

// Operator library: names the ld/hd operator files (src/mlib3d.cpp:70-103).
class Mlib3d {
public:
    explicit Mlib3d(const std::string& prefix = "mlib3d_") : prefix_(prefix), kernel_(0), NPQ_(4) {}
    int& kernel() { return kernel_; }
    int& NPQ() { return NPQ_; }
    std::string& ldname() { return ld_; }
    std::string& hdname() { return hd_; }
    int setup(std::map<std::string, std::string>& opts) {
        read_opt(opts, "-" + prefix_ + "NPQ", NPQ_);
        read_opt(opts, "-" + prefix_ + "ldname", ld_);
        read_opt(opts, "-" + prefix_ + "hdname", hd_);
        if (ld_.empty() || hd_.empty()) throw new std::exception();
        return 0;
    }

private:
    std::string prefix_;
    int kernel_, NPQ_;
    std::string ld_, hd_;
};

// PosMap: std::map<int, P> with P indexable as p[0..2] (the reference's Point3).
template <class PosMap>
class Wave3dT {
public:
    explicit Wave3dT(const std::string& prefix = "wave3d_", int device = 0)
        : prefix_(prefix), device_(device), pos_(0), kernel_(0), mlib_(0), ncell_(0), ACCU_(1), NPQ_(4),
          K_(64), ptsmax_(100), maxlevel_(-1), s_(0), n_(0) {
        ctr_[0] = ctr_[1] = ctr_[2] = 0;
    }
    ~Wave3dT() { ddfmm_session_destroy(s_); }

    const PosMap*& posptr() { return pos_; }
    int& kernel() { return kernel_; }
    Mlib3d*& mlibptr() { return mlib_; }
    int& geomprtn() { return ncell_; }  // cells per edge of the partition tensor
    int& ACCU() { return ACCU_; }
    int& NPQ() { return NPQ_; }
    double& K() { return K_; }
    int& ptsmax() { return ptsmax_; }
    int& maxlevel() { return maxlevel_; }

    // Wave3d::setup (src/wave3d_setup.cpp:21-97)
    int setup(std::map<std::string, std::string>& opts) {
        const std::string p = "-" + prefix_;
        read_opt(opts, p + "ACCU", ACCU_);
        read_opt(opts, p + "NPQ", NPQ_);
        read_opt(opts, p + "K", K_);
        read_opt(opts, p + "ptsmax", ptsmax_);
        read_opt(opts, p + "maxlevel", maxlevel_);
        std::map<std::string, std::string>::iterator it = opts.find(p + "ctr");
        if (it != opts.end()) {
            std::istringstream ss(it->second);
            ss >> ctr_[0] >> ctr_[1] >> ctr_[2];
        }
        if (!pos_ || !mlib_ || ncell_ <= 0 || maxlevel_ < 1) throw new std::exception();
        std::vector<double> xyz;
        xyz.reserve(3 * pos_->size());
        int expect = 0;
        for (typename PosMap::const_iterator mi = pos_->begin(); mi != pos_->end(); ++mi, ++expect) {
            if (mi->first != expect) throw new std::exception();  // ids must be 0..N-1
            for (int d = 0; d < 3; ++d) xyz.push_back(mi->second[d]);
        }
        ddfmm_session_destroy(s_);
        s_ = 0;
        n_ = expect;
        raise_if(ddfmm_session_create(xyz.data(), n_, kernel_, ACCU_, NPQ_, K_, ctr_, ptsmax_, maxlevel_, ncell_,
                                      mlib_->ldname().c_str(), mlib_->hdname().c_str(), device_, &s_));
        return 0;
    }

    // Wave3d::eval (src/wave3d_eval.cpp:299-415): val[id] = FMM matvec of den.
    template <class ValMap>
    int eval(const ValMap& den, ValMap& val) {
        std::vector<cpx> d(n_), v(n_);
        gather(den, d);
        raise_if(ddfmm_eval(s_, reinterpret_cast<const double*>(d.data()), reinterpret_cast<double*>(v.data())));
        for (int i = 0; i < n_; ++i) val[i] = v[i];
        return 0;
    }

    // Wave3d::check (src/wave3d_check.cpp:22-100): relerr = |direct - fmm| / |fmm|
    template <class ValMap>
    int check(const ValMap& den, const ValMap& val, const std::vector<int>& chk, double& relerr) {
        std::vector<cpx> d(n_), truth(chk.size());
        gather(den, d);
        raise_if(ddfmm_direct(s_, reinterpret_cast<const double*>(d.data()), chk.data(), (int)chk.size(),
                              reinterpret_cast<double*>(truth.data())));
        double en = 0, tn = 0;
        for (size_t i = 0; i < chk.size(); ++i) {
            typename ValMap::const_iterator it = val.find(chk[i]);
            if (it == val.end()) throw new std::exception();
            en += std::norm(truth[i] - it->second);
            tn += std::norm(it->second);
        }
        relerr = std::sqrt(en) / std::sqrt(tn);
        return 0;
    }

private:
    template <class ValMap>
    void gather(const ValMap& den, std::vector<cpx>& d) const {
        if ((int)den.size() != n_ || !s_) throw new std::exception();
        int i = 0;
        for (typename ValMap::const_iterator mi = den.begin(); mi != den.end(); ++mi, ++i) {
            if (mi->first != i) throw new std::exception();
            d[i] = mi->second;
        }
    }
    std::string prefix_;
    int device_;
    const PosMap* pos_;
    int kernel_;
    Mlib3d* mlib_;
    int ncell_, ACCU_, NPQ_;
    double K_;
    int ptsmax_, maxlevel_;
    double ctr_[3];
    ddfmm_session* s_;
    int n_;
};

}  // namespace ddfmm_b200

#endif
