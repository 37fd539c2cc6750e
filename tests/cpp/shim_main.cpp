// Drives the header-only Wave3d drop-in (include/ddfmm_wave3d.hpp) the way
// the reference's tt driver drives Wave3d (src/tt.cpp:103-185).
//   shim_main <case-dir>     reads case-dir/{pos,den}.bin (raw doubles),
//                            case-dir/opts.txt ("key value" lines), writes
//                            case-dir/val.bin and prints "relerr <e>".
//   shim_main --no-gpu       expects setup to throw (no device)
#include <array>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>

#include "ddfmm_wave3d.hpp"

typedef std::array<double, 3> Point3;
typedef ddfmm_b200::Wave3dT<std::map<int, Point3> > Wave3d;

static std::vector<double> slurp(const std::string& p) {
    std::ifstream f(p.c_str(), std::ios::binary);
    std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<double> v(b.size() / 8);
    if (!v.empty()) std::memcpy(v.data(), b.data(), v.size() * 8);
    return v;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::string arg = argv[1];
    std::map<std::string, std::string> opts;
    std::map<int, Point3> pos;
    std::map<int, ddfmm_b200::cpx> den, val;
    std::vector<int> chk;
    if (arg == "--no-gpu") {
        for (int i = 0; i < 8; ++i) pos[i] = Point3{{0.1 * i, 0.0, 0.0}};
        opts["-mlib3d_ldname"] = "missing.ld";
        opts["-mlib3d_hdname"] = "missing.hd";
        opts["-wave3d_maxlevel"] = "6";
        opts["-wave3d_K"] = "4";
    } else {
        std::ifstream of((arg + "/opts.txt").c_str());
        std::string k, v;
        while (of >> k >> v) opts[k] = v;
        std::vector<double> p = slurp(arg + "/pos.bin"), d = slurp(arg + "/den.bin"), c = slurp(arg + "/chk.bin");
        for (size_t i = 0; i < p.size() / 3; ++i) pos[(int)i] = Point3{{p[3 * i], p[3 * i + 1], p[3 * i + 2]}};
        for (size_t i = 0; i < d.size() / 2; ++i) den[(int)i] = ddfmm_b200::cpx(d[2 * i], d[2 * i + 1]);
        for (double x : c) chk.push_back((int)x);
    }
    ddfmm_b200::Mlib3d mlib("mlib3d_");
    int kernel = 0;
    ddfmm_b200::read_opt(opts, "-kernel", kernel);
    mlib.kernel() = kernel;
    Wave3d wave("wave3d_");
    try {
        mlib.setup(opts);
        wave.posptr() = &pos;
        wave.kernel() = kernel;
        wave.mlibptr() = &mlib;
        int nc = 4;
        ddfmm_b200::read_opt(opts, "-geomprtn", nc);
        wave.geomprtn() = nc;
        wave.setup(opts);
    } catch (std::exception* e) {
        std::cout << "setup threw: " << ddfmm_last_error() << std::endl;
        delete e;
        return arg == "--no-gpu" ? 0 : 1;
    }
    if (arg == "--no-gpu") return 1;
    val = den;  // tt presets val = den (src/tt.cpp:97-98)
    try {
        wave.eval(den, val);
        wave.eval(den, val);  // repeated evals must not accumulate
        double relerr;
        wave.check(den, val, chk, relerr);
        std::ofstream o((arg + "/val.bin").c_str(), std::ios::binary);
        for (auto& kv : val) o.write(reinterpret_cast<const char*>(&kv.second), 16);
        printf("relerr %.9e\n", relerr);
    } catch (std::exception* e) {
        std::cout << "eval threw: " << ddfmm_last_error() << std::endl;
        delete e;
        return 1;
    }
    return 0;
}
