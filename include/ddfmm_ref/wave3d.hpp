// Drop-in replacement for the reference's include/wave3d.hpp (arbenson/ddfmm)
// that runs Wave3d::eval on the B200 through the C ABI of libddfmm_b200
// (include/ddfmm.h).
//
// A program written against the reference -- its driver src/tt.cpp
// unchanged -- builds against this header by putting this directory ahead of
// the reference's include directory on the include path and linking
// libddfmm_b200.so instead of the reference's wave3d*.cpp objects.  Everything
// else stays the reference's: ParVec<int, cpx, PtPrtn> (include/parvec.hpp),
// Point3 / Index3 (include/vec3t.hpp), IntNumTns / IntNumVec, Kernel3d and
// Mlib3d (whose setup still reads the ld / hd operator files; this class
// hands the same file names to the GPU session).
//
// The class keeps the reference's public interface (include/wave3d.hpp:
// 219-265): posptr() / kernel() / mlibptr() / geomprtn() and the option
// accessors, setup(opts) with the reference's -<prefix>ACCU / NPQ / K / ctr /
// ptsmax / maxlevel options (src/wave3d_setup.cpp:21-97, defaults of
// src/wave3d.cpp:24-26), eval(den, val) (src/wave3d_eval.cpp:299-415) and
// check(den, val, chkkeys, relerr) (src/wave3d_check.cpp:22-100).  Two
// options the reference does not read are accepted: -<prefix>device (CUDA
// ordinal, default 0) and -<prefix>precision (0 plain FP64, the default; 1
// mixed).  Failures print the library's reason and throw
// `new std::exception()` as the reference's CHECK_TRUE / SAFE_FUNC_EVAL do
// (include/commoninc.hpp:52-53).
//
// Single rank: the process must own every point (PtPrtn with one owner), as
// in the reference's one-rank runs.  Unlike the reference, eval may be
// called any number of times on one object; values do not accumulate.
#ifndef _WAVE3D_HPP_
#define _WAVE3D_HPP_

#include <algorithm>
#include <cmath>
#include <complex>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "comobject.hpp"
#include "kernel3d.hpp"
#include "mlib3d.hpp"
#include "numtns.hpp"
#include "parvec.hpp"
#include "vec3t.hpp"

#include "../ddfmm.h"

// Owner of a point id: _ownerinfo holds the prefix offsets of the ids per
// rank (the reference's PtPrtn, include/wave3d.hpp:40-57; the same layout
// is read and written by deserialize / serialize below).
class PtPrtn {
public:
    std::vector<int> _ownerinfo;
    std::vector<int>& ownerinfo() { return _ownerinfo; }
    int owner(int key) {
        std::vector<int>::iterator it = std::upper_bound(_ownerinfo.begin(), _ownerinfo.end(), key);
        return int(it - _ownerinfo.begin()) - 1;
    }
};

inline int serialize(const PtPrtn& p, std::ostream& os, const std::vector<int>& mask) {
    return serialize(p._ownerinfo, os, mask);
}
inline int deserialize(PtPrtn& p, std::istream& is, const std::vector<int>& mask) {
    return deserialize(p._ownerinfo, is, mask);
}

class Wave3d : public ComObject {
public:
    ParVec<int, Point3, PtPrtn>* _posptr;
    Kernel3d _kernel;
    int _ACCU;
    int _NPQ;
    Mlib3d* _mlibptr;
    IntNumTns _geomprtn;
    double _K;
    Point3 _ctr;
    int _ptsmax;
    int _maxlevel;

    explicit Wave3d(const std::string& p)
        : ComObject(p), _posptr(NULL), _ACCU(1), _NPQ(4), _mlibptr(NULL), _K(64), _ctr(Point3(0, 0, 0)),
          _ptsmax(100), _maxlevel(-1), _device(0), _precision(DDFMM_PLAIN_FP64), _s(NULL) {}
    ~Wave3d() { ddfmm_session_destroy(_s); }

    ParVec<int, Point3, PtPrtn>*& posptr() { return _posptr; }
    Kernel3d& kernel() { return _kernel; }
    int& ACCU() { return _ACCU; }
    int& NPQ() { return _NPQ; }
    Mlib3d*& mlibptr() { return _mlibptr; }
    IntNumTns& geomprtn() { return _geomprtn; }
    double& K() { return _K; }
    Point3& ctr() { return _ctr; }
    int& ptsmax() { return _ptsmax; }
    int& maxlevel() { return _maxlevel; }

    // Wave3d::setup: read the options, build the octree, lists and operators
    // on the GPU (one ddfmm session).
    int setup(std::map<std::string, std::string>& opts) {
        const std::string p = "-" + prefix();
        opt(opts, p + "ACCU", _ACCU);
        opt(opts, p + "NPQ", _NPQ);
        opt(opts, p + "K", _K);
        std::map<std::string, std::string>::iterator mi = opts.find(p + "ctr");
        if (mi != opts.end()) {
            std::istringstream ss(mi->second);
            double x, y, z;
            ss >> x >> y >> z;
            _ctr = Point3(x, y, z);
        }
        opt(opts, p + "ptsmax", _ptsmax);
        opt(opts, p + "maxlevel", _maxlevel);
        opt(opts, p + "device", _device);
        opt(opts, p + "precision", _precision);
        if (!_posptr || !_mlibptr) raise("posptr and mlibptr must be set before setup");
        if (_geomprtn.m() < 1 || _geomprtn.m() != _geomprtn.n() || _geomprtn.m() != _geomprtn.p())
            raise("geomprtn must be a cubic cell partition");
        std::map<int, Point3>& pos = _posptr->lclmap();
        _ids.clear();
        _ids.reserve(pos.size());
        std::vector<double> xyz;
        xyz.reserve(3 * pos.size());
        for (std::map<int, Point3>::iterator it = pos.begin(); it != pos.end(); ++it) {
            _ids.push_back(it->first);
            for (int d = 0; d < 3; ++d) xyz.push_back(it->second(d));
        }
        std::vector<int>& own = _posptr->prtn().ownerinfo();
        if (!own.empty() && own.back() != (int)pos.size())
            raise("this drop-in runs on one rank: the process must own every point");
        const double c[3] = {_ctr(0), _ctr(1), _ctr(2)};
        // the files Mlib3d::setup read: SharedRead opens data/<name> (src/parallel.cpp:67-71)
        const std::string ld = "data/" + _mlibptr->ldname(), hd = "data/" + _mlibptr->hdname();
        ddfmm_session_destroy(_s);
        _s = NULL;
        status(ddfmm_session_create_ex(xyz.empty() ? NULL : &xyz[0], (int)_ids.size(), _kernel.type(), _ACCU, _NPQ,
                                       _K, c, _ptsmax, _maxlevel, _geomprtn.m(), ld.c_str(), hd.c_str(), _device,
                                       _precision, &_s));
        return 0;
    }

    // Wave3d::eval: val(id) = sum_j G(x_id, x_j) den(j) for every point id.
    int eval(ParVec<int, cpx, PtPrtn>& den, ParVec<int, cpx, PtPrtn>& val) {
        std::vector<cpx> d, v(_ids.size());
        gather(den, d);
        status(ddfmm_eval(session(), reinterpret_cast<const double*>(&d[0]), reinterpret_cast<double*>(&v[0])));
        std::map<int, cpx>& out = val.lclmap();
        for (size_t i = 0; i < _ids.size(); ++i) out[_ids[i]] = v[i];
        return 0;
    }

    // Wave3d::check: relerr = |direct - val| / |val| over the ids in chkkeys,
    // the direct sum taken in FP64 over every point.
    int check(ParVec<int, cpx, PtPrtn>& den, ParVec<int, cpx, PtPrtn>& val, IntNumVec& chkkeys, double& relerr) {
        std::vector<cpx> d;
        gather(den, d);
        std::map<int, size_t> dense;
        for (size_t i = 0; i < _ids.size(); ++i) dense[_ids[i]] = i;
        std::vector<int> idx(chkkeys.m());
        for (int k = 0; k < chkkeys.m(); ++k) {
            std::map<int, size_t>::iterator it = dense.find(chkkeys(k));
            if (it == dense.end()) raise("check id is not a point id");
            idx[k] = (int)it->second;
        }
        std::vector<cpx> truth(idx.size());
        status(ddfmm_direct(session(), reinterpret_cast<const double*>(&d[0]), idx.empty() ? NULL : &idx[0],
                            (int)idx.size(), truth.empty() ? NULL : reinterpret_cast<double*>(&truth[0])));
        double en = 0, tn = 0;
        std::map<int, cpx>& vm = val.lclmap();
        for (size_t k = 0; k < idx.size(); ++k) {
            std::map<int, cpx>::iterator it = vm.find(chkkeys((int)k));
            if (it == vm.end()) raise("val has no entry for a check id");
            en += std::norm(truth[k] - it->second);
            tn += std::norm(it->second);
        }
        relerr = std::sqrt(en) / std::sqrt(tn);
        return 0;
    }

private:
    int _device, _precision;
    ddfmm_session* _s;
    std::vector<int> _ids;  // point ids in key order: the session's dense order

    template <class T>
    static void opt(std::map<std::string, std::string>& opts, const std::string& key, T& v) {
        std::map<std::string, std::string>::iterator it = opts.find(key);
        if (it != opts.end()) {
            std::istringstream ss(it->second);
            ss >> v;
        }
    }
    static void raise(const char* why) {
        std::cerr << "Wave3d: " << why << std::endl;
        throw new std::exception();
    }
    static void status(int rc) {
        if (rc != DDFMM_OK) {
            std::cerr << "Wave3d: " << ddfmm_last_error() << std::endl;
            throw new std::exception();
        }
    }
    ddfmm_session* session() {
        if (!_s) raise("setup has not been called");
        return _s;
    }
    void gather(ParVec<int, cpx, PtPrtn>& den, std::vector<cpx>& d) {
        session();
        std::map<int, cpx>& m = den.lclmap();
        d.resize(_ids.size());
        for (size_t i = 0; i < _ids.size(); ++i) {
            std::map<int, cpx>::iterator it = m.find(_ids[i]);
            if (it == m.end()) raise("den has no entry for a point id");
            d[i] = it->second;
        }
        if (d.empty()) raise("no points");
    }
};

#endif  // _WAVE3D_HPP_
