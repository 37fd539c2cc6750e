// Reader for the reference's operator files (see ops.hpp).
#include "ops.hpp"

#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <stdexcept>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace ddfmm {

namespace {
// A whole operator file mapped read-only; the matrices are copied out of the
// mapping (no intermediate copy of the file).
struct In {
    const char* buf = nullptr;
    size_t size = 0;
    size_t o = 0;
    std::string name;
    In() = default;
    In(const In&) = delete;
    In& operator=(const In&) = delete;
    ~In() {
        if (buf && size) munmap(const_cast<char*>(buf), size);
    }
    void need(size_t n) {
        if (o + n > size)
            throw std::runtime_error("operator file " + name + " is truncated");
    }
    int i32() {
        need(4);
        int v;
        std::memcpy(&v, &buf[o], 4);
        o += 4;
        return v;
    }
    double f64() {
        need(8);
        double v;
        std::memcpy(&v, &buf[o], 8);
        o += 8;
        return v;
    }
    int dim() {
        int v = i32();
        if (v < 0 || v > (1 << 26)) throw std::runtime_error("operator file " + name + ": bad dimension");
        return v;
    }
    void dbl(double* dst, size_t n) {
        need(8 * n);
        std::memcpy(dst, &buf[o], 8 * n);
        o += 8 * n;
    }
    PMat pmat() {
        int m = dim(), n = dim();
        if (m != 3 && !(m == 0 && n == 0)) throw std::runtime_error("operator file " + name + ": points are not 3 x n");
        PMat p;
        p.n = n;
        p.x.resize((size_t)3 * n);
        dbl(p.x.data(), p.x.size());
        return p;
    }
    CMat cmat() {
        CMat c;
        c.m = dim();
        c.n = dim();
        c.a.resize((size_t)c.m * c.n);
        dbl(reinterpret_cast<double*>(c.a.data()), 2 * c.a.size());
        return c;
    }
    std::vector<cpx> ctns(int& edge) {
        int m = dim(), n = dim(), p = dim();
        std::vector<cpx> t((size_t)m * n * p);
        dbl(reinterpret_cast<double*>(t.data()), 2 * t.size());
        if (!t.empty()) {
            if (m != n || n != p) throw std::runtime_error("operator file " + name + ": ue2dc tensor not cubic");
            edge = m;
        }
        return t;
    }
};

void slurp(const std::string& path, In& in) {
    const int fd = open(path.c_str(), O_RDONLY);
    if (fd < 0) throw std::runtime_error("cannot open operator file " + path);
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        throw std::runtime_error("cannot size operator file " + path);
    }
    in.name = path;
    in.size = (size_t)st.st_size;
    if (in.size > 0) {
        void* p = mmap(nullptr, in.size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, fd, 0);
        if (p == MAP_FAILED) {
            close(fd);
            in.size = 0;
            throw std::runtime_error("cannot map operator file " + path);
        }
        in.buf = static_cast<const char*>(p);
    }
    close(fd);
}
}  // namespace

void OperatorLib::load(const std::string& ld_path, const std::string& hd_path) {
    ld.clear();
    hd.clear();
    In a;
    slurp(ld_path, a);
    int nw = a.dim();
    for (int w = 0; w < nw; ++w) {
        LowFreqOp op;
        op.W = a.f64();
        op.uep = a.pmat();
        op.ucp = a.pmat();
        int nv = a.dim();
        if (nv != 3) throw std::runtime_error("ld file: uc2ue must hold 3 matrices");
        op.v = a.cmat();
        op.is = a.cmat();
        op.up = a.cmat();
        int t0 = a.dim(), t1 = a.dim(), t2 = a.dim();
        if (t0 != 7 || t1 != 7 || t2 != 7) throw std::runtime_error("ld file: ue2dc must be 7x7x7");
        op.ue2dc.resize(343);
        for (int i = 0; i < 343; ++i) op.ue2dc[i] = a.ctns(op.tdim);
        ld[op.W] = std::move(op);
    }
    if (a.o != a.size) throw std::runtime_error("ld file has trailing bytes");
    In b;
    slurp(hd_path, b);
    nw = b.dim();
    for (int w = 0; w < nw; ++w) {
        double W = b.f64();
        int nd = b.dim();
        auto& lvl = hd[W];
        for (int k = 0; k < nd; ++k) {
            Idx3 key{{b.i32(), b.i32(), b.i32()}};
            HighFreqOp op;
            op.uep = b.pmat();
            op.ucp = b.pmat();
            int nv = b.dim();
            if (nv != 3) throw std::runtime_error("hd file: uc2ue must hold 3 matrices");
            op.E1 = b.cmat();
            op.E2 = b.cmat();
            op.E3 = b.cmat();
            lvl[key] = std::move(op);
        }
    }
    if (b.o != b.size) throw std::runtime_error("hd file has trailing bytes");
}

std::shared_ptr<const OperatorLib> OperatorLib::shared(const std::string& ld_path, const std::string& hd_path) {
    auto stamp = [](const std::string& path) {
        struct stat st;
        if (stat(path.c_str(), &st) != 0) throw std::runtime_error("cannot open operator file " + path);
        return std::to_string((long long)st.st_size) + ":" + std::to_string((long long)st.st_mtim.tv_sec) + "." +
               std::to_string((long long)st.st_mtim.tv_nsec);
    };
    const std::string key = ld_path + "|" + stamp(ld_path) + "|" + hd_path + "|" + stamp(hd_path);
    static std::mutex mu;
    static std::map<std::string, std::weak_ptr<const OperatorLib> > cache;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end())
            if (auto p = it->second.lock()) return p;
    }
    auto lib = std::make_shared<OperatorLib>();
    lib->load(ld_path, hd_path);  // outside the lock: seconds for large files
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = cache.begin(); it != cache.end();)
        it = it->second.expired() ? cache.erase(it) : std::next(it);
    auto& slot = cache[key];
    if (auto p = slot.lock()) return p;  // another thread loaded the same files meanwhile
    slot = lib;
    return lib;
}

void OperatorLib::validate(int accu) const {
    if (accu < 1 || accu > 3) throw std::invalid_argument("ACCU must be 1, 2 or 3");
    const int P = accu == 1 ? 4 : (accu == 2 ? 6 : 8);
    const int nE = P * P * P - (P - 2) * (P - 2) * (P - 2);
    auto bad = [](const std::string& what, double W) {
        std::ostringstream s;
        s << what << " (width " << W << ")";
        throw std::runtime_error(s.str());
    };
    for (const auto& kv : ld) {
        const LowFreqOp& o = kv.second;
        if (o.uep.n != nE || o.ucp.n != nE) bad("ld file: surfaces do not have P^3-(P-2)^3 points for this ACCU", kv.first);
        const int r = o.v.n;
        if (o.v.m != nE || o.is.m != r || o.is.n != 1 || o.up.m != r || o.up.n != nE)
            bad("ld file: uc2ue factors have inconsistent shapes", kv.first);
        if (o.tdim != 0 && o.tdim != 2 * P) bad("ld file: ue2dc tensors are not (2P)^3 for this ACCU", kv.first);
    }
    for (const auto& kv : hd)
        for (const auto& dk : kv.second) {
            const HighFreqOp& o = dk.second;
            const int r1 = o.uep.n, r2 = o.ucp.n;
            if (o.E1.m != r1 || o.E1.n != r1 || o.E2.m != r1 || o.E2.n != r2 || o.E3.m != r2 || o.E3.n != r2)
                bad("hd file: E1/E2/E3 shapes do not match the skeleton point counts", kv.first);
            if (r1 > 400 || r2 > 400) bad("hd file: skeleton rank exceeds DVMAX=400", kv.first);
        }
}

const LowFreqOp& OperatorLib::low(double W) const {
    auto it = ld.find(W);
    if (it == ld.end()) {
        std::ostringstream s;
        s << "no low-frequency operators for width " << W;
        throw std::runtime_error(s.str());
    }
    return it->second;
}

const HighFreqOp& OperatorLib::high(double W, const Idx3& canon) const {
    auto it = hd.find(W);
    if (it != hd.end()) {
        auto jt = it->second.find(canon);
        if (jt != it->second.end()) return jt->second;
    }
    std::ostringstream s;
    s << "no high-frequency operators for width " << W << " wedge (" << canon[0] << "," << canon[1] << ","
      << canon[2] << ")";
    throw std::runtime_error(s.str());
}

}  // namespace ddfmm
