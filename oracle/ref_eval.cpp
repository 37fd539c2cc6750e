// Timing driver around the reference library (oracle/CPU baseline only).
// Makes the same calls as the reference's src/tt.cpp:43-198 -- read pos/den,
// Mlib3d::setup, Wave3d::setup, Wave3d::eval, serialize val, optional
// Wave3d::check -- but times setup and eval with a steady clock (tt uses
// time(0), 1 s resolution) and prints one machine-readable line:
//   REF_EVAL setup_s=<s> eval_s=<s> n=<N> relerr=<e|nan>
// Files are read from data/ under the working directory, as tt does
// (src/parallel.cpp:33,81).  One eval per process: Wave3d::eval accumulates
// into extval on a second call (src/wave3d_eval.cpp:518-521).
#include "wave3d.hpp"
#include "parallel.hpp"
#include <chrono>
#include <cstdio>

static std::string opt(std::map<std::string, std::string>& o, const char* k) {
    std::map<std::string, std::string>::iterator it = o.find(k);
    return it == o.end() ? std::string() : it->second;
}

int main(int argc, char** argv) {
    MPI_Init(&argc, &argv);
    std::map<std::string, std::string> opts;
    for (int k = 1; k + 1 < argc; k += 2) opts[argv[k]] = argv[k + 1];
    std::vector<int> all(1, 1);
    try {
        ParVec<int, Point3, PtPrtn> pos;
        std::istringstream piss;
        SAFE_FUNC_EVAL(SeparateRead(opt(opts, "-posfile"), piss));
        SAFE_FUNC_EVAL(deserialize(pos, piss, all));
        ParVec<int, cpx, PtPrtn> den;
        std::istringstream diss;
        SAFE_FUNC_EVAL(SeparateRead(opt(opts, "-denfile"), diss));
        SAFE_FUNC_EVAL(deserialize(den, diss, all));
        ParVec<int, cpx, PtPrtn> val;
        val = den;
        Kernel3d kernel(KERNEL_HELM);
        if (!opt(opts, "-kernel").empty()) kernel.type() = atoi(opt(opts, "-kernel").c_str());
        Mlib3d mlib("mlib3d_");
        mlib.kernel() = kernel;
        mlib.NPQ() = 4;
        SAFE_FUNC_EVAL(mlib.setup(opts));
        IntNumTns geomprtn;
        std::istringstream giss;
        SAFE_FUNC_EVAL(SharedRead(opt(opts, "-geomprtn"), giss));
        SAFE_FUNC_EVAL(deserialize(geomprtn, giss, all));
        Wave3d wave("wave3d_");
        wave.posptr() = &pos;
        wave.kernel() = kernel;
        wave.mlibptr() = &mlib;
        wave.geomprtn() = geomprtn;
        typedef std::chrono::steady_clock clk;
        clk::time_point t0 = clk::now();
        SAFE_FUNC_EVAL(wave.setup(opts));
        clk::time_point t1 = clk::now();
        SAFE_FUNC_EVAL(wave.eval(den, val));
        clk::time_point t2 = clk::now();
        std::ostringstream oss;
        SAFE_FUNC_EVAL(serialize(val, oss, all));
        SAFE_FUNC_EVAL(SeparateWrite(opt(opts, "-valfile"), oss));
        double relerr = NAN;
        if (!opt(opts, "-chkfile").empty()) {
            IntNumVec chk;
            std::istringstream iss;
            SAFE_FUNC_EVAL(SharedRead(opt(opts, "-chkfile"), iss));
            SAFE_FUNC_EVAL(deserialize(chk, iss, all));
            SAFE_FUNC_EVAL(wave.check(den, val, chk, relerr));
        }
        std::vector<int>& info = pos.prtn().ownerinfo();
        printf("REF_EVAL setup_s=%.6f eval_s=%.6f n=%d relerr=%.6e\n",
               std::chrono::duration<double>(t1 - t0).count(),
               std::chrono::duration<double>(t2 - t1).count(), info.back(), relerr);
    } catch (...) {
        fprintf(stderr, "REF_EVAL failed: the reference threw\n");
        return 1;
    }
    MPI_Finalize();
    return 0;
}
