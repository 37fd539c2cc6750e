// Plan flattening and the eval launch sequence (see session.hpp).
//
// Pass structure and data flow follow Wave3d::eval (src/wave3d_eval.cpp:299-415):
//   1. low-frequency upward, widths ascending        (EvalUpwardLow :418-490)
//   2. high-frequency upward, widths ascending       (EvalUpwardHigh :773-854)
//   3. high-frequency downward, widths descending    (EvalDownwardHigh :996-1040,
//      HighFrequencyM2L :876-928, HighFrequencyL2L :931-993)
//   4. low-frequency downward, widths descending     (EvalDownwardLow :493-583 with
//      U/V/W/X lists :585-718)
// The reference walks directions recursively (pre-order up, post-order down,
// :721-751); every (box, wedge) only depends on its children (up) or its
// parent (down), so processing whole widths at a time gives the same sums.
// Operators are the reference's: Mlib3d::*Fetch (src/mlib3d.cpp:106-280).
#include "session.hpp"

#include "plan.hpp"

#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <exception>
#include <set>
#include <stdexcept>
#include <thread>
#include <unordered_map>
#include <unordered_set>

namespace ddfmm {

#define CK(x)                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" + \
                                     #x + ")");                                                    \
    } while (0)

static int accu_to_p(int accu) {
    if (accu < 1 || accu > 3) throw std::runtime_error("ACCU must be 1, 2 or 3");  // src/wave3d.cpp:149
    return accu == 1 ? 4 : (accu == 2 ? 6 : 8);
}

template <class T>
T* Session::dalloc(size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaMalloc(&p, count * sizeof(T)));
    t_malloc_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ++n_malloc_;
    allocs_.push_back(p);
    alloc_bytes_[p] = count * sizeof(T);
    stats_.device_bytes += count * sizeof(T);
    return static_cast<T*>(p);
}

void Session::dfree(const void* p) {
    auto it = alloc_bytes_.find(p);
    if (it == alloc_bytes_.end()) return;  // not an allocation of this session (or an interior pointer)
    CK(cudaFree(const_cast<void*>(p)));
    stats_.device_bytes -= it->second;
    alloc_bytes_.erase(it);
    allocs_.erase(std::remove(allocs_.begin(), allocs_.end(), p), allocs_.end());
}

template <class T>
T* Session::upload_n(const T* src, size_t count) {
    const size_t bytes = count * sizeof(T);
    if (bytes > kArenaMax) {
        const auto t0 = std::chrono::steady_clock::now();
        T* d = nullptr;
        if (bytes <= kMidMax) {
            const size_t need = (bytes + 255) & ~(size_t)255;
            if (mid_used_ + need > mid_cap_) {  // chunks of 4 MiB doubling to 64 MiB: small sessions stay small
                const size_t cap = std::max(need, std::min(kMidChunk, std::max((size_t)kMidMax, 2 * mid_cap_)));
                void* chunk = nullptr;
                CK(cudaMalloc(&chunk, cap));
                allocs_.push_back(chunk);
                stats_.device_bytes += cap;
                mid_dev_ = static_cast<char*>(chunk);
                mid_used_ = 0;
                mid_cap_ = cap;
            }
            d = reinterpret_cast<T*>(mid_dev_ + mid_used_);
            mid_used_ += need;
        } else {
            d = dalloc<T>(count);
        }
        stage_copy(d, src, bytes);  // the caller's array may die right after: the data is staged
        t_big_uploads_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return d;
    }
    const size_t need = (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;  // 256-byte aligned slots
    if (arena_.used + need > arena_.cap) {
        flush_uploads();
        // the copy out of the old host image may still be running: keep the
        // image until the end of the plan (released after a stream sync)
        if (!arena_.host.empty()) arena_.retired.push_back(std::move(arena_.host));
        // chunks of 1 MiB doubling to 64 MiB: small sessions stay small
        arena_.cap = std::max(need, std::min((size_t)64 << 20, std::max((size_t)1 << 20, 2 * arena_.cap)));
        // not through dalloc: a chunk must never be released by dfree(), which
        // would take an array that happens to start the chunk for its base
        void* chunk = nullptr;
        CK(cudaMalloc(&chunk, arena_.cap));
        allocs_.push_back(chunk);
        stats_.device_bytes += arena_.cap;
        arena_.dev = static_cast<char*>(chunk);
        arena_.host.assign(arena_.cap, 0);
        arena_.used = arena_.sent = 0;
    }
    char* d = arena_.dev + arena_.used;
    if (bytes) std::memcpy(arena_.host.data() + arena_.used, src, bytes);
    arena_.used += need;
    return reinterpret_cast<T*>(d);
}

void Session::flush_uploads() {
    if (arena_.used > arena_.sent)
        stage_copy(arena_.dev + arena_.sent, arena_.host.data() + arena_.sent, arena_.used - arena_.sent);
    arena_.sent = arena_.used;
}

void Session::stage_copy(void* dst, const void* src, size_t bytes) {
    if (!stage_[0])
        for (int k = 0; k < 2; ++k) {
            CK(cudaHostAlloc((void**)&stage_[k], kStage, cudaHostAllocDefault));
            CK(cudaEventCreateWithFlags(&stage_ev_[k], cudaEventDisableTiming));
            CK(cudaEventRecord(stage_ev_[k], stream_));
        }
    for (size_t off = 0; off < bytes;) {
        const size_t n = std::min(kStage, bytes - off);
        const int k = stage_next_;
        stage_next_ ^= 1;
        const auto t0 = std::chrono::steady_clock::now();
        CK(cudaEventSynchronize(stage_ev_[k]));  // the device has read this buffer's previous contents
        const auto t1 = std::chrono::steady_clock::now();
        std::memcpy(stage_[k], static_cast<const char*>(src) + off, n);
        t_stage_wait_ += std::chrono::duration<double>(t1 - t0).count();
        t_stage_copy_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        ++n_stage_;
        CK(cudaMemcpyAsync(static_cast<char*>(dst) + off, stage_[k], n, cudaMemcpyHostToDevice, stream_));
        CK(cudaEventRecord(stage_ev_[k], stream_));
        off += n;
    }
}

void Session::stage_release() {
    for (int k = 0; k < 2; ++k) {
        if (stage_ev_[k]) cudaEventDestroy(stage_ev_[k]);
        if (stage_[k]) cudaFreeHost(stage_[k]);
        stage_ev_[k] = nullptr;
        stage_[k] = nullptr;
    }
}

Session::Session(const double* pos3n, int n, const SessionParams& p, const std::string& ld_path,
                 const std::string& hd_path)
    : prm_(p), npts_(n) {
    if (n <= 0) throw std::runtime_error("no points");
    auto t0 = std::chrono::steady_clock::now();
    // operator files first (Mlib3d::setup): a bad file is reported before any device work
    ld_path_ = ld_path;
    hd_path_ = hd_path;
    auto since = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
    };
    ops_ = OperatorLib::shared(ld_path, hd_path);
    ops_->validate(p.accu);
    stats_.ops_seconds = since(t0);
    CK(cudaSetDevice(p.device));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    pos_.assign(pos3n, pos3n + 3 * (size_t)n);
    auto t1 = std::chrono::steady_clock::now();
    tree_.build(pos_.data(), n, p.tree);
    stats_.tree_seconds = since(t1);
    t1 = std::chrono::steady_clock::now();
    build();
    CK(cudaStreamSynchronize(stream_));
    stats_.plan_seconds = since(t1);
    t1 = std::chrono::steady_clock::now();
    autotune();
    CK(cudaStreamSynchronize(stream_));
    stats_.tune_seconds = since(t1);
    stats_.setup_seconds = since(t0);
}

Session::~Session() {
    if (stream_) cudaStreamSynchronize(stream_);
    stage_release();
    for (cudaEvent_t e : ev_) cudaEventDestroy(e);
    for (void* p : allocs_) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
}

void Session::add_gemm(std::vector<GemmProblem>& probs, std::vector<std::vector<long long> >& xo,
                       std::vector<std::vector<long long> >& yo, const double2* X, double2* Y, int mode,
                       const char* label) {
    struct Clock {
        double& acc;
        std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
        ~Clock() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
    } clock{t_emit_gemm_};
    double flops = 0, bytes = 0;
    std::vector<GemmProblem> P;
    std::vector<size_t> from;  // the caller's problem of each P
    std::vector<GemmTile> tiles;
    size_t ncols = 0;
    for (size_t i = 0; i < probs.size(); ++i) {
        if (xo[i].empty() || probs[i].m == 0 || probs[i].k == 0) continue;
        GemmProblem q = probs[i];
        q.col0 = (int)ncols;
        q.ncol = (int)xo[i].size();
        if (yo[i].size() != xo[i].size()) throw std::logic_error("GEMM problem with unequal column lists");
        int pid = (int)P.size();
        P.push_back(q);
        from.push_back(i);
        ncols += (size_t)q.ncol;
        for (int r0 = 0; r0 < q.m; r0 += GEMM_TILE_M)
            for (int c0 = 0; c0 < q.ncol; c0 += GEMM_TILE_N) tiles.push_back(GemmTile{pid, r0, c0, 0});
        flops += 8.0 * q.m * q.k * (double)q.ncol;
        // operator once, each input and output column once (read-modify-write for += modes)
        bytes += 16.0 * ((double)q.m * q.k + (double)q.k * q.ncol + (mode == GEMM_SET ? 1.0 : 2.0) * q.m * q.ncol);
    }
    if (ncols > (size_t)INT_MAX) throw std::runtime_error("too many GEMM columns in one launch");
    // the launch's column offsets, concatenated in problem order on all host cores
    // (pieces of at most 64k columns); the arrays are not zeroed first
    std::unique_ptr<long long[]> xs(new long long[std::max<size_t>(ncols, 1)]);
    std::unique_ptr<long long[]> ys(new long long[std::max<size_t>(ncols, 1)]);
    {
        std::vector<std::array<size_t, 3> > pieces;  // (P index, first column, end column)
        for (size_t j = 0; j < P.size(); ++j)
            for (size_t c = 0; c < (size_t)P[j].ncol; c += 65536)
                pieces.push_back({{j, c, std::min((size_t)P[j].ncol, c + 65536)}});
        host_parallel_for(pieces.size(), [&](size_t e) {
            const size_t j = pieces[e][0], c0 = pieces[e][1], n = pieces[e][2] - c0;
            std::memcpy(xs.get() + P[j].col0 + c0, xo[from[j]].data() + c0, n * sizeof(long long));
            std::memcpy(ys.get() + P[j].col0 + c0, yo[from[j]].data() + c0, n * sizeof(long long));
        });
    }
    stats_.flops_gemm += flops;
    if (tiles.empty()) return;
    Step st{};
    st.kind = 0;
    st.label = label;
    st.flops = flops;
    st.bytes = bytes;
    if (umma()) {
        add_umma(P, xs.get(), ys.get(), ncols, X, Y, mode, st);
        push_step(st);
        stats_.gemm_launches++;
        return;
    }
    st.g.probs = upload(P);
    st.g.tiles = upload(tiles);
    st.g.xoff = upload_n(xs.get(), ncols);
    st.g.yoff = upload_n(ys.get(), ncols);
    st.g.ntiles = (int)tiles.size();
    st.g.X = X;
    st.g.Y = Y;
    st.g.mode = mode;
    push_step(st);
    stats_.gemm_launches++;
}

const float* Session::cached_op(const std::string& key) {
    if (opctx_.empty()) return nullptr;
    std::shared_ptr<PackedOp> e = OpCache::find(opctx_ + "|" + key);
    if (!e) return nullptr;
    held_.push_back(e);
    return e->p;
}

const float* Session::packed_operator(const GemmProblem& q) {
    if (q.packed) return q.packed;  // shared copy from the cache
    struct Clock {
        double& acc;
        std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
        ~Clock() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
    } clock{t_pack_};
    const auto key = std::make_pair((const void*)q.A, ((long long)q.m << 32) | (long long)q.k);
    auto it = packed_.find(key);
    if (it != packed_.end()) return it->second;
    // packed operators are sub-allocated from device chunks (256-byte aligned; cp.async.bulk
    // needs 16), the unit the operator cache frees; one larger than a chunk gets its own
    const size_t nf = (umma_packed_floats(q.m, q.k) + 63) & ~(size_t)63;
    if (nf > chunk_left_) {
        Clock ca{t_pack_alloc_};
        // chunks of 16 MiB doubling to 128 MiB: small sessions stay small, large
        // ones make few allocations
        const size_t last = chunk_ ? chunk_->bytes() / sizeof(float) : 0;
        const size_t floats = std::max(nf, std::min((size_t)32 << 20, std::max((size_t)4 << 20, 2 * last)));
        chunk_ = std::make_shared<DevChunk>(prm_.device, floats * sizeof(float));
        chunk_pos_ = chunk_->data();
        chunk_left_ = floats;
        chunk_bytes_ += floats * sizeof(float);
        stats_.device_bytes += floats * sizeof(float);
    }
    float* d = chunk_pos_;
    chunk_pos_ += nf;
    chunk_left_ -= nf;
    std::shared_ptr<PackedOp> op = std::make_shared<PackedOp>(PackedOp{chunk_, d});
    held_.push_back(op);
    auto k = opkey_.find((const void*)q.A);
    if (k != opkey_.end()) to_publish_.push_back(std::make_pair(opctx_ + "|" + k->second, op));
    pack_jobs_.push_back(UmmaPackJob{(const float2*)q.A, d, umma_tile_stride(q.k), q.m, q.k, q.lda, umma_nkb(q.k)});
    return packed_[key] = d;
}

// tcgen05 form of one grouped GEMM launch: tiles of 128 gathered columns x
// 128 complex operator rows, the tiles of one problem adjacent so that blocks
// in flight share its packed operator in L2.
void Session::add_umma(const std::vector<GemmProblem>& P, const long long* xs, const long long* ys, size_t ncols,
                       const double2* X, double2* Y, int mode, Step& st) {
    std::vector<UmmaProblem> U;
    std::vector<UmmaTile> tiles;
    for (size_t i = 0; i < P.size(); ++i) {
        const GemmProblem& q = P[i];
        U.push_back(UmmaProblem{packed_operator(q), umma_tile_stride(q.k), q.m, q.k, umma_nkb(q.k), q.col0, q.ncol});
        for (int rt = 0; rt * 128 < q.m; ++rt)
            for (int c0 = 0; c0 < q.ncol; c0 += 128) {
                tiles.push_back(UmmaTile{(int)i, rt, rt * 128, std::min(128, q.m - rt * 128), c0, 0});
                st.uop.push_back(U.back().B + (size_t)rt * U.back().tile_stride);
            }
    }
    st.kind = 5;
    st.hu = UmmaSub{upload(U), upload(tiles), upload_n(xs, ncols), upload_n(ys, ncols), reinterpret_cast<const float2*>(X),
                    reinterpret_cast<float2*>(Y), (int)tiles.size(), mode, 0, 0};
    set_multi(st, st.hu, (int)tiles.size());
}

template <class Sub>
void Session::set_multi(Step& st, const Sub& sub, int total) {
    st.msubs = upload(std::vector<Sub>(1, sub));
    st.mpre = upload(std::vector<int>{0, total});
    st.mtotal = total;
}

// Steps are emitted in blocks (phase, width): LF upward and HF upward by
// ascending width, HF downward and LF downward by descending width.
void Session::begin_block(int phase, double W) {
    cur_phase_ = phase;
    const long long w = std::lround(std::log2(W));
    cur_wkey_ = phase < 2 ? 1000 + w : 1000 - w;
    block_counts_.clear();
}

void Session::push_step(Step st) {
    // step types in the order the blocks emit them
    static const char* const order[] = {"lf_s2m",   "lf_m2m",       "lf_uc2ue",     "memset",   "hf_m2m",
                                        "hf_uc2ue", "hf_m2l",       "hf_dc2de",     "hf_l2l",   "lf_vlist_fft",
                                        "lf_vlist_m2l", "lf_vlist_inv", "lf_xlist", "lf_ulist", "lf_wlist",
                                        "lf_dc2de", "lf_l2t",       "lf_l2l"};
    std::string base(st.label);
    const size_t u = base.rfind("_w");
    if (u != std::string::npos && u + 2 < base.size() && std::isdigit((unsigned char)base[u + 2]))
        base = base.substr(0, u);  // per-width label "pass_w<W>"

    long long rank = 63;
    for (size_t i = 0; i < sizeof(order) / sizeof(order[0]); ++i)
        if (base == order[i]) rank = (long long)i;
    const long long occ = block_counts_[base]++;
    st.key = ((long long)cur_phase_ << 48) | (cur_wkey_ << 32) | (rank << 16) | occ;
    steps_.push_back(st);
}

void Session::flush_packs() {
    flush_uploads();
    if (pack_jobs_.empty()) return;
    UmmaPackJob* d = nullptr;
    CK(cudaMalloc(&d, sizeof(UmmaPackJob) * pack_jobs_.size()));
    CK(cudaMemcpyAsync(d, pack_jobs_.data(), sizeof(UmmaPackJob) * pack_jobs_.size(), cudaMemcpyHostToDevice,
                       stream_));
    launch_umma_pack(d, (int)pack_jobs_.size(), stream_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    CK(cudaFree(d));
    pack_jobs_.clear();
    // packed and complete: other sessions may use them from now on
    for (auto& kp : to_publish_) OpCache::publish(kp.first, kp.second);
    to_publish_.clear();
}

void Session::check_device_error() {
    if (!d_err_) return;
    int h = 0;
    CK(cudaMemcpyAsync(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    if (h) {
        CK(cudaMemsetAsync(d_err_, 0, sizeof(int), stream_));
        CK(cudaStreamSynchronize(stream_));
        throw std::runtime_error("CUDA error: a tensor-core GEMM block timed out waiting on its pipeline");
    }
}

void Session::arm_gemm_stall(double wait_s) {
    if (!umma()) throw std::invalid_argument("the GEMM stall hook needs a DDFMM_MIXED (tcgen05) session");
    if (!(wait_s > 0 && wait_s <= 1.0)) throw std::invalid_argument("stall wait must be in (0, 1] seconds");
    stall_wait_ns_ = (unsigned long long)(wait_s * 1e9);
}

const char* Session::width_label(const char* pass, double W) {
    char buf[64];
    snprintf(buf, sizeof buf, "%s_w%g", pass, W);
    for (const std::string& l : label_store_)
        if (l == buf) return l.c_str();
    label_store_.reserve(256);  // pointers into the store must stay valid
    if (label_store_.size() >= 256) return pass;
    label_store_.push_back(buf);
    return label_store_.back().c_str();
}

void Session::add_pt(const std::vector<PtItem>& items, const std::vector<PtSrc>& srcs, const char* label) {
    if (items.empty()) return;
    Step st{};
    st.kind = 1;
    st.label = label;
    for (const PtItem& it : items) {
        long long ns = 0;
        for (int k = it.src_begin; k < it.src_end; ++k) ns += srcs[k].src.n;
        // one kernel evaluation (sqrt, reciprocal, sincospi) + one complex MAC per pair
        st.flops += 20.0 * it.trg.n * (double)ns;
        st.bytes += 40.0 * ns + 56.0 * it.trg.n;
    }
    st.pt.items = upload(items);
    st.pt.srcs = upload(srcs);
    st.pt.nitems = (int)items.size();
    if (mixed()) {
        st.hp = PtSub{st.pt.items, st.pt.srcs, st.pt.nitems, prm_.kernel, 0, 0};
        set_multi(st, st.hp, st.pt.nitems);
    }
    push_step(st);
}

namespace {
// Setup-time matrix products C = A * B for many small operators in one
// launch: each product is one grouped-GEMM problem whose "columns" are the
// columns of B (read from pool X) and of C (written to pool Y).
struct GemmBatch {
    std::vector<GemmProblem> probs;
    std::vector<long long> xs, ys;
    // A (m x k, lda m, device pointer), B = X[bx ..] (k x n), C = Y[cy ..] (m x n)
    void product(const double2* A, int m, int k, size_t bx, int n, size_t cy) {
        GemmProblem p{A, m, k, m, (int)xs.size(), n};
        for (int j = 0; j < n; ++j) {
            xs.push_back((long long)(bx + (size_t)j * k));
            ys.push_back((long long)(cy + (size_t)j * m));
        }
        probs.push_back(p);
    }
    void run(const double2* X, double2* Y, cudaStream_t s) {
        if (probs.empty()) return;
        std::vector<GemmTile> tiles;
        for (size_t i = 0; i < probs.size(); ++i)
            for (int r0 = 0; r0 < probs[i].m; r0 += GEMM_TILE_M)
                for (int c0 = 0; c0 < probs[i].ncol; c0 += GEMM_TILE_N) tiles.push_back(GemmTile{(int)i, r0, c0, 0});
        GemmProblem* dp;
        GemmTile* dt;
        long long *dx, *dy;
        CK(cudaMalloc(&dp, sizeof(GemmProblem) * probs.size()));
        CK(cudaMalloc(&dt, sizeof(GemmTile) * tiles.size()));
        CK(cudaMalloc(&dx, sizeof(long long) * xs.size()));
        CK(cudaMalloc(&dy, sizeof(long long) * ys.size()));
        CK(cudaMemcpyAsync(dp, probs.data(), sizeof(GemmProblem) * probs.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dt, tiles.data(), sizeof(GemmTile) * tiles.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dx, xs.data(), sizeof(long long) * xs.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dy, ys.data(), sizeof(long long) * ys.size(), cudaMemcpyHostToDevice, s));
        launch_gemm(dp, dt, (int)tiles.size(), dx, dy, X, Y, GEMM_SET, s);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        cudaFree(dp);
        cudaFree(dt);
        cudaFree(dx);
        cudaFree(dy);
    }
};

Pt3 shifted_point(int ind, double W) {  // ShiftedPoint, src/mlib3d.cpp:21-30
    int a = (ind & 4) >> 2, b = (ind & 2) >> 1, c = ind & 1;
    return Pt3{{(a - 0.5) * W / 2, (b - 0.5) * W / 2, (c - 0.5) * W / 2}};
}
// HighFetchShuffle, src/mlib3d.cpp:308-325: res(prm(d)) = tmp(d), then res(d) *= sgn(d)
std::vector<double> shuffle(const PMat& p, const Idx3& prm, const Idx3& sgn, double extra_sign) {
    std::vector<double> r((size_t)3 * p.n);
    for (int k = 0; k < p.n; ++k) {
        double t[3];
        for (int d = 0; d < 3; ++d) t[prm[d]] = p.x[3 * k + d];
        for (int d = 0; d < 3; ++d) r[3 * k + d] = extra_sign * (sgn[d] * t[d]);
    }
    return r;
}
std::vector<double2> to_d2(const CMat& m) {
    std::vector<double2> r(m.a.size());
    for (size_t i = 0; i < m.a.size(); ++i) r[i] = make_double2(m.a[i].real(), m.a[i].imag());
    return r;
}
std::vector<double2> to_d2_transpose(const CMat& m) {  // Transpose, src/mlib3d.cpp:32-42
    std::vector<double2> r(m.a.size());
    for (int i = 0; i < m.m; ++i)
        for (int j = 0; j < m.n; ++j) r[(size_t)i * m.n + j] = make_double2(m(i, j).real(), m(i, j).imag());
    return r;
}
}  // namespace

void Session::build() {
    // DDFMM_SETUP_TRACE=1: time each part of the plan (with the stream drained
    // at each mark, so device work is charged to the part that enqueued it)
    // and print the times to stderr
    const bool trace = std::getenv("DDFMM_SETUP_TRACE") != nullptr;
    auto tmark = std::chrono::steady_clock::now();
    auto phase = [&](const char* what) {
        if (!trace) return;
        CK(cudaStreamSynchronize(stream_));
        const auto t = std::chrono::steady_clock::now();
        std::fprintf(stderr, "ddfmm setup %-16s %8.3f s\n", what, std::chrono::duration<double>(t - tmark).count());
        tmark = t;
    };
    const double eps = 1e-12;
    const int P = accu_to_p(prm_.accu), G = 2 * P, G3 = G * G * G;
    const int nE = P * P * P - (P - 2) * (P - 2) * (P - 2);
    const int kern = prm_.kernel;
    if (kern != KERNEL_HELM && kern != KERNEL_EXPR) throw std::runtime_error("unknown kernel type");
    // complex state: double2 (plain FP64 form) or float2 (mixed form); plan
    // offsets are in elements, so both forms share one plan
    const bool mixed = this->mixed();
    if (umma()) opctx_ = OpCache::context(prm_.device, kern, prm_.accu, prm_.tree.npq, ld_path_, hd_path_);
    const size_t es = mixed ? sizeof(float2) : sizeof(double2);
    auto E = [&](double2* base, size_t elems) { return (double2*)((char*)base + elems * es); };
    auto salloc = [&](size_t elems) { return (double2*)dalloc<char>(elems * es); };
    // operators are built in FP64; the mixed form multiplies with FP32 copies
    std::map<const double2*, const double2*> op32;
    auto opm = [&](const double2* a, size_t n) -> const double2* {
        if (!mixed) return a;
        auto it = op32.find(a);
        if (it != op32.end()) return it->second;
        float2* b = dalloc<float2>(n);
        flush_uploads();
        launch_to_c64(a, b, (long long)n, stream_);
        CK(cudaGetLastError());
        return op32[a] = (const double2*)b;
    };
    Tree& T = tree_;
    const int nb = (int)T.boxes.size();
    stats_.n_points = npts_;
    stats_.n_boxes = nb;

    // ---------------------------------------------------------------- LF boxes, leaves, points
    std::vector<int> lfbox, lfidx(nb, -1);
    for (int b : T.order)
        if (T.boxes[b].has_pts() && T.width(T.boxes[b].level) < 1 - eps) {
            lfidx[b] = (int)lfbox.size();
            lfbox.push_back(b);
        }
    const int nLF = (int)lfbox.size();
    stats_.n_lf_boxes = nLF;
    std::vector<int> perm, leaf_off(nLF, -1), leaf_cnt(nLF, 0);
    std::vector<double> pos_sorted;
    perm.reserve(npts_);
    pos_sorted.reserve(3 * (size_t)npts_);
    for (int l = 0; l < nLF; ++l) {
        const Box& B = T.boxes[lfbox[l]];
        if (!B.terminal()) continue;
        leaf_off[l] = (int)perm.size();
        leaf_cnt[l] = (int)B.pts.size();
        for (int id : B.pts) {
            perm.push_back(id);
            for (int d = 0; d < 3; ++d) pos_sorted.push_back(pos_[3 * (size_t)id + d]);
        }
        stats_.n_leaves++;
    }
    if ((int)perm.size() != npts_) throw std::runtime_error("tree leaves do not hold every point exactly once");
    d_perm_ = upload(perm);
    d_pos_ids_ = upload(pos_);
    d_pos_sorted_ = upload(pos_sorted);
    d_den_sorted_ = salloc(npts_);
    d_val_sorted_ = salloc(npts_);
    d_den_io_ = dalloc<double2>(npts_);
    d_val_io_ = dalloc<double2>(npts_);
    zero_at_start_.push_back(Memset{d_val_sorted_, es * npts_});

    phase("points");
    std::map<int, std::vector<int> > lflevels;  // level -> lf ids (key order)
    for (int l = 0; l < nLF; ++l) lflevels[T.boxes[lfbox[l]].level].push_back(l);

    double2* lf_upeq = salloc((size_t)nLF * nE);
    double2* lf_upchk = salloc((size_t)nLF * nE);
    double2* lf_mid = salloc((size_t)nLF * nE);
    double2* lf_dnchk = salloc((size_t)nLF * nE);
    double2* lf_dneq = salloc((size_t)nLF * nE);
    double2* lf_spec = salloc((size_t)nLF * G3);
    spectra_elems_ = (size_t)nLF * G3;
    stats_.fft_spectra_bytes = (long long)nLF * G3 * 16;
    zero_at_start_.push_back(Memset{lf_upchk, es * (size_t)nLF * nE});
    zero_at_start_.push_back(Memset{lf_dnchk, es * (size_t)nLF * nE});

    // per-LF-level device operators
    struct LfLevelOps {
        double W;
        const double *uep, *ucp;
        double2 *up_s, *v, *vT_s, *upT, *tns;
        int* cube_idx;
        int r;
        double2* ue2uc[8];
        double2* de2dc[8];
        bool has_children;
    };
    std::map<int, LfLevelOps> lfops;
    std::vector<KmatJob> jobs;  // kernel-matrix generation, run once below
    long long job_elems = 0;
    auto add_job = [&](const double* trg, Pt3 ts, const double* src, Pt3 ss, int m, int k, double2* out) {
        KmatJob j;
        j.trg = trg;
        j.src = src;
        j.out = out;
        for (int d = 0; d < 3; ++d) {
            j.ts[d] = ts[d];
            j.ss[d] = ss[d];
        }
        j.m = m;
        j.k = k;
        j.elem0 = job_elems;
        job_elems += (long long)m * k;
        jobs.push_back(j);
    };
    const Pt3 zero3{{0, 0, 0}};
    std::vector<double2> twf(G), twb(G);
    {
        const long double twopi = 6.283185307179586476925286766559005768L;
        for (int m = 0; m < G; ++m) {
            long double a = twopi * (long double)m / (long double)G;
            twf[m] = make_double2((double)cosl(a), -(double)sinl(a));
            twb[m] = make_double2((double)cosl(a), (double)sinl(a));
        }
    }
    const double2* d_twf = opm(upload(twf), G);
    const double2* d_twb = opm(upload(twb), G);
    vlist_init(G);
    gemm_init();
    vlist32_init(G);
    cgemm_init();
    if (umma()) {
        umma_init();
        d_err_ = dalloc<int>(1);
        CK(cudaMemsetAsync(d_err_, 0, sizeof(int), stream_));
    }

    for (auto& kv : lflevels) {
        int level = kv.first;
        double W = T.width(level);
        const LowFreqOp& op = ops_->low(W);
        if (op.uep.n != nE || op.ucp.n != nE)
            throw std::runtime_error("low-frequency operator size does not match ACCU");
        LfLevelOps L{};
        L.W = W;
        L.r = op.up.m;
        L.uep = upload(op.uep.x);
        L.ucp = upload(op.ucp.x);
        // fold the 1/sigma scaling into the rows of U^H (up) and of v^T.  The mixed
        // form truncates the pseudo-inverse further, at sigma < 1e-7 sigma_max: FP32
        // check values carry ~1e-7 relative noise, which the directions below that
        // would amplify into equivalent densities whose norm swamps every later FP32
        // translation (at P = 8 sigma spans 12 decades)
        double smax = 0;
        for (int i = 0; i < L.r; ++i) smax = std::max(smax, 1.0 / std::abs(op.is(i, 0)));
        std::vector<double2> up_s((size_t)L.r * nE), vT_s((size_t)L.r * nE);
        for (int i = 0; i < L.r; ++i)
            for (int j = 0; j < nE; ++j) {
                cpx s = op.is(i, 0);
                if (mixed && 1.0 / std::abs(s) < 1e-7 * smax) s = 0;
                cpx a = s * op.up(i, j), b = s * op.v(j, i);
                up_s[(size_t)j * L.r + i] = make_double2(a.real(), a.imag());
                vT_s[(size_t)j * L.r + i] = make_double2(b.real(), b.imag());
            }
        L.up_s = upload(up_s);
        L.vT_s = upload(vT_s);
        L.v = upload(to_d2(op.v));
        L.upT = upload(to_d2_transpose(op.up));
        // V-list tensors and grid positions of the uep / dcp nodes (src/wave3d_eval.cpp:607-659)
        if (op.tdim != 0 && op.tdim != G) throw std::runtime_error("ue2dc tensor size does not match ACCU");
        std::vector<double2> tns((size_t)343 * G3, make_double2(0, 0));
        for (int o = 0; o < 343; ++o) {
            const auto& t = op.ue2dc[o];
            if (t.empty()) continue;
            for (int e = 0; e < G3; ++e) tns[(size_t)o * G3 + e] = make_double2(t[e].real(), t[e].imag());
        }
        L.tns = (double2*)opm(upload(tns), tns.size());
        // (src/wave3d_eval.cpp:626-628,655-657): a = round((x + W/2)/step) + P in [P, 2P)
        std::vector<int> cidx(nE);
        double step = W / (P - 1);
        for (int k = 0; k < nE; ++k) {
            int a[3];
            for (int d = 0; d < 3; ++d) a[d] = (int)std::round((op.uep.x[3 * k + d] + W / 2) / step) + P;
            for (int d = 0; d < 3; ++d)
                if (a[d] < P || a[d] >= 2 * P) throw std::runtime_error("V-list grid index outside the corner cube");
            cidx[k] = (a[0] - P) + P * ((a[1] - P) + P * (a[2] - P));
        }
        L.cube_idx = upload(cidx);
        L.has_children = false;
        for (int l : kv.second)
            if (!T.boxes[lfbox[l]].terminal()) L.has_children = true;
        if (L.has_children) {
            const LowFreqOp& ch = ops_->low(W / 2);  // UpwardLowFetch / DownwardLowFetch
            const double* chuep = upload(ch.uep.x);
            for (int ind = 0; ind < 8; ++ind) {
                L.ue2uc[ind] = dalloc<double2>((size_t)nE * nE);
                L.de2dc[ind] = dalloc<double2>((size_t)nE * nE);
                add_job(L.ucp, zero3, chuep, shifted_point(ind, W), nE, nE, L.ue2uc[ind]);
                add_job(chuep, shifted_point(ind, W), L.ucp, zero3, nE, nE, L.de2dc[ind]);
            }
        }
        lfops[level] = L;
    }

    phase("lf_operators");
    // ---------------------------------------------------------------- HF nodes
    struct Canon {
        double W;
        Idx3 srt;
        const HighFreqOp* op;
        int r1, r2;
        double2 *E1, *E2, *E3, *E1t, *E2t, *E3t;
        double *uep, *neg_uep;
    };
    std::vector<Canon> hfcanon;
    std::map<std::pair<double, Idx3>, int> canon_id;
    auto get_canon = [&](double W, const Idx3& dir, Idx3& sgn, Idx3& prmv) -> int {
        Idx3 srt;
        index3_sort(dir, srt, sgn, prmv);
        auto key = std::make_pair(W, srt);
        auto it = canon_id.find(key);
        if (it != canon_id.end()) return it->second;
        Canon c{};
        c.W = W;
        c.srt = srt;
        c.op = &ops_->high(W, srt);
        c.r1 = c.op->uep.n;
        c.r2 = c.op->ucp.n;
        if (c.op->E1.m != c.r1 || c.op->E1.n != c.r1 || c.op->E2.m != c.r1 || c.op->E2.n != c.r2 ||
            c.op->E3.m != c.r2 || c.op->E3.n != c.r2)
            throw std::runtime_error("high-frequency operator shapes are inconsistent");
        if (c.r1 > 400 || c.r2 > 400)  // DVMAX, src/wave3d_eval.cpp:25,842-844
            throw std::runtime_error("high-frequency rank exceeds DVMAX=400");
        c.E1 = upload(to_d2(c.op->E1));
        c.E2 = upload(to_d2(c.op->E2));
        c.E3 = upload(to_d2(c.op->E3));
        c.E1t = upload(to_d2_transpose(c.op->E1));
        c.E2t = upload(to_d2_transpose(c.op->E2));
        c.E3t = upload(to_d2_transpose(c.op->E3));
        c.uep = upload(c.op->uep.x);
        std::vector<double> neg(c.op->uep.x);
        for (double& v : neg) v = -v;
        c.neg_uep = upload(neg);
        int id = (int)hfcanon.size();
        hfcanon.push_back(c);
        canon_id[key] = id;
        return id;
    };
    // per (W, dir) shuffled point sets
    struct DirPts {
        double *ucp, *dep, *uep, *dcp;  // S*ucp, -S*ucp, S*uep, -S*uep
        int r1, r2, canon;
        int did;  // dense id, in order of first use
    };
    std::map<std::pair<double, Idx3>, DirPts> dirpts;
    // dense index into dirpts (node addresses are stable): per width, the wedge's
    // components (each in [-C, C], C = npq W) address a (2C+1)^3 table
    struct DirTable {
        double W;
        int C;
        std::vector<const DirPts*> t;
    };
    std::deque<DirTable> dirtabs;
    DirTable* last_tab = nullptr;
    auto dir_slot = [&](double W, const Idx3& d) -> const DirPts** {
        if (!last_tab || last_tab->W != W) {
            last_tab = nullptr;
            for (DirTable& x : dirtabs)
                if (x.W == W) last_tab = &x;
            if (!last_tab) {
                const int C = prm_.tree.npq * (int)std::round(W);
                if (C <= 0 || C > 128) return nullptr;
                dirtabs.push_back(DirTable{W, C, std::vector<const DirPts*>((size_t)(2 * C + 1) * (2 * C + 1) * (2 * C + 1), nullptr)});
                last_tab = &dirtabs.back();
            }
        }
        const int C = last_tab->C, E = 2 * C + 1;
        for (int k = 0; k < 3; ++k)
            if (d[k] < -C || d[k] > C) return nullptr;
        return &last_tab->t[((size_t)(d[0] + C) * E + (d[1] + C)) * E + (d[2] + C)];
    };
    auto get_dir = [&](double W, const Idx3& dir) -> const DirPts& {
        const DirPts** slot = dir_slot(W, dir);
        if (slot && *slot) return **slot;
        auto key = std::make_pair(W, dir);
        auto it = dirpts.find(key);
        if (it != dirpts.end()) {
            if (slot) *slot = &it->second;
            return it->second;
        }
        Idx3 sgn, pv;
        int c = get_canon(W, dir, sgn, pv);
        const HighFreqOp& op = *hfcanon[c].op;
        DirPts d{};
        d.did = (int)dirpts.size();
        d.canon = c;
        d.r1 = hfcanon[c].r1;
        d.r2 = hfcanon[c].r2;
        d.ucp = upload(shuffle(op.ucp, pv, sgn, 1.0));
        d.dep = upload(shuffle(op.ucp, pv, sgn, -1.0));
        d.uep = upload(shuffle(op.uep, pv, sgn, 1.0));
        d.dcp = upload(shuffle(op.uep, pv, sgn, -1.0));
        DirPts& stored = dirpts[key] = d;
        if (slot) *slot = &stored;
        return stored;
    };

    std::map<int, std::vector<int> > hflevels;  // level -> tree boxes with points, width >= 1
    for (int b : T.order)
        if (T.boxes[b].has_pts() && T.width(T.boxes[b].level) > 1 - eps) hflevels[T.boxes[b].level].push_back(b);

    // nodes of a box are contiguous and in its (sorted) wedge order, so a
    // (box, wedge) node is found by binary search in the box's range (HfNodes::find)
    HfNodes up, dn;
    up.first.assign(nb, 0);
    up.cnt.assign(nb, 0);
    dn.first.assign(nb, 0);
    dn.cnt.assign(nb, 0);
    {
        size_t nu = 0, nd = 0;
        for (auto& kv : hflevels)
            for (int b : kv.second) {
                nu += T.boxes[b].outdirs.size();
                nd += T.boxes[b].incdirs.size();
            }
        up.v.reserve(nu);
        dn.v.reserve(nd);
    }
    std::map<int, long long> tmp_up_level;  // level -> temporary elements of its M2M sums
    long long upeq_total = 0, dnchk_total = 0, tmp_max = 0;
    for (auto& kv : hflevels) {
        const double W = T.width(kv.first);
        const std::vector<int>& bx = kv.second;
        const size_t nbx = bx.size();
        // the level's wedges, created in first-use order (their dense ids follow it):
        // a box's outgoing wedges, then its incoming ones, box by box
        for (int b : bx) {
            for (const Idx3& d : T.boxes[b].outdirs) get_dir(W, d);
            for (const Idx3& d : T.boxes[b].incdirs) get_dir(W, d);
        }
        // every wedge of the level now has its point sets: the nodes are filled on
        // all host cores from per-box prefix sums (a box's nodes are contiguous, in
        // its sorted wedge order), read-only lookups through the level's table
        const DirPts** tab = dir_slot(W, Idx3{{0, 0, 0}}) ? last_tab->t.data() : nullptr;
        const int C = last_tab ? last_tab->C : 0, E = 2 * C + 1;
        auto lookup = [&](const Idx3& d) -> const DirPts& {
            if (tab && d[0] >= -C && d[0] <= C && d[1] >= -C && d[1] <= C && d[2] >= -C && d[2] <= C) {
                const DirPts* q = tab[((size_t)(d[0] + C) * E + (d[1] + C)) * E + (d[2] + C)];
                if (q) return *q;
            }
            return dirpts.at(std::make_pair(W, d));
        };
        std::vector<long long> uo(nbx + 1, 0), ut(nbx + 1, 0), dof(nbx + 1, 0), dt(nbx + 1, 0);
        std::vector<int> un(nbx + 1, 0), dnn(nbx + 1, 0);
        host_parallel_for(nbx, [&](size_t i) {
            const Box& B = T.boxes[bx[i]];
            long long a = 0, at = 0, c = 0, ct = 0;
            for (const Idx3& d : B.outdirs) {
                const DirPts& dp = lookup(d);
                a += dp.r1;
                at += std::max(dp.r1, dp.r2);
            }
            for (const Idx3& d : B.incdirs) {
                const DirPts& dp = lookup(d);
                c += dp.r1;
                ct += std::max(dp.r1, dp.r2);
            }
            uo[i + 1] = a;
            ut[i + 1] = at;
            dof[i + 1] = c;
            dt[i + 1] = ct;
            un[i + 1] = (int)B.outdirs.size();
            dnn[i + 1] = (int)B.incdirs.size();
        });
        const int u0 = (int)up.v.size(), d0 = (int)dn.v.size();
        uo[0] = upeq_total;
        dof[0] = dnchk_total;
        un[0] = u0;
        dnn[0] = d0;
        for (size_t i = 0; i < nbx; ++i) {
            uo[i + 1] += uo[i];
            ut[i + 1] += ut[i];
            dof[i + 1] += dof[i];
            dt[i + 1] += dt[i];
            un[i + 1] += un[i];
            dnn[i + 1] += dnn[i];
        }
        up.v.resize((size_t)un[nbx]);
        dn.v.resize((size_t)dnn[nbx]);
        host_parallel_for(nbx, [&](size_t i) {
            const int b = bx[i];
            const Box& B = T.boxes[b];
            up.first[b] = un[i];
            up.cnt[b] = un[i + 1] - un[i];
            long long o = uo[i], t = ut[i];
            int k = un[i];
            for (const Idx3& d : B.outdirs) {
                const DirPts& dp = lookup(d);
                up.v[k++] = HfNode{b, d, dp.canon, o, t, dp.did};
                o += dp.r1;
                t += std::max(dp.r1, dp.r2);
            }
            dn.first[b] = dnn[i];
            dn.cnt[b] = dnn[i + 1] - dnn[i];
            o = dof[i];
            t = dt[i];
            k = dnn[i];
            for (const Idx3& d : B.incdirs) {
                const DirPts& dp = lookup(d);
                dn.v[k++] = HfNode{b, d, dp.canon, o, t, dp.did};
                o += dp.r1;
                t += std::max(dp.r1, dp.r2);
            }
        });
        upeq_total = uo[nbx];
        dnchk_total = dof[nbx];
        const long long tmp_up = ut[nbx], tmp_dn = dt[nbx];
        up.range[kv.first] = std::make_pair(u0, (int)up.v.size());
        tmp_up_level[kv.first] = tmp_up;
        dn.range[kv.first] = std::make_pair(d0, (int)dn.v.size());
        tmp_max = std::max(tmp_max, std::max(tmp_up, tmp_dn));
    }
    phase("hf_nodes");
    stats_.hf_up_nodes = (long long)up.v.size();
    stats_.hf_down_nodes = (long long)dn.v.size();
    double2* hf_upeq = salloc((size_t)upeq_total);
    double2* hf_dnchk = salloc((size_t)dnchk_total);
    double2* T0 = salloc((size_t)tmp_max);
    double2* T1 = salloc((size_t)tmp_max);
    zero_at_start_.push_back(Memset{hf_dnchk, es * (size_t)dnchk_total});

    // ---------------------------------------------------------------- HF operators
    // Raw kernel matrices -- M2M ue2uc and L2L de2dc per (W, wedge, child), M2L per
    // (W, canonical wedge, canonical offset) -- are generated once, then folded
    // with the skeleton factors of uc2ue = {E1, E2, E3} (src/mlib3d.cpp:204-207,
    // :246-250) so that the eval applies one dense operator per translation plus
    // E2 / E2^T per (box, wedge):
    //   upward   w    = E2 * sum_c [E3 * ue2uc_c * E1(child)] w_c        (upeqnden = E1 w)
    //   M2L      u_t += [E1^T * M(o) * E1] w_s                          (u = E1^T dnchkval)
    //   downward u_c += [E1(child)^T * de2dc_c * E3^T] (E2^T u)          (dneqnden = E3^T E2^T u)
    // At W = 1 the children are low-frequency boxes and carry no E1 factor.
    // E1 = inv(R1) and E3 = inv(R2^H) are ill-conditioned (~1e7), so they are
    // only ever multiplied into the smooth kernel matrices, never into each other.
    auto take = [](size_t& pool, size_t n) {
        size_t o = pool;
        pool += (n + 15) & ~(size_t)15;
        return o;
    };
    size_t scr = 0, keep = 0;
    // cache keys of the shared operators: (kind, width, wedge, child or offset)
    auto opk = [](const char* kind, double W, const Idx3& d, int a, int b = 0, int c = 0) {
        char buf[128];
        snprintf(buf, sizeof buf, "%s|%.17g|%d,%d,%d|%d,%d,%d", kind, W, d[0], d[1], d[2], a, b, c);
        return std::string(buf);
    };
    struct DirMats {
        size_t raw[8], tmp[8], fin[8];
        int mrows, mcols, canon, ccanon;
        bool cached;            // all eight come from the shared cache
        const float* pk[8];     // their packed copies
    };
    std::map<std::pair<double, Idx3>, DirMats> m2m_mats, l2l_mats;
    const double* lf_half_uep = nullptr;
    if (!hflevels.empty()) {
        const LowFreqOp& lf_half = ops_->low(0.5);
        if (lf_half.uep.n != nE) throw std::runtime_error("width-1/2 operators do not match ACCU");
        lf_half_uep = upload(lf_half.uep.x);
    }
    auto child_pts = [&](double W, const Idx3& dir, bool upward, int& rc, int& ccanon) -> const double* {
        if (W == 1.0) {
            rc = nE;
            ccanon = -1;
            return lf_half_uep;  // LF uep at W/2 for both directions (src/mlib3d.cpp:199-202,254-257)
        }
        const DirPts& cp = get_dir(W / 2, predir(dir));
        rc = cp.r1;
        ccanon = cp.canon;
        return upward ? cp.uep : cp.dcp;
    };
    std::vector<char> m2m_seen(dirpts.size(), 0), l2l_seen(dirpts.size(), 0);  // by dense wedge id: already planned
    for (auto& kv : hflevels) {
        double W = T.width(kv.first);
        auto ur = up.range[kv.first], dr = dn.range[kv.first];
        for (int i = ur.first; i < ur.second; ++i) {
            if (m2m_seen[up.v[i].did]) continue;
            m2m_seen[up.v[i].did] = 1;
            auto key = std::make_pair(W, up.v[i].dir);
            const DirPts& dp = get_dir(W, up.v[i].dir);
            DirMats M{};
            child_pts(W, up.v[i].dir, true, M.mcols, M.ccanon);
            M.mrows = dp.r2;
            M.canon = dp.canon;
            M.cached = !opctx_.empty();
            for (int ind = 0; ind < 8 && M.cached; ++ind)
                M.cached = (M.pk[ind] = cached_op(opk("m2m", W, up.v[i].dir, ind))) != nullptr;
            for (int ind = 0; ind < 8 && !M.cached; ++ind) {
                size_t n = (size_t)M.mrows * M.mcols;
                M.raw[ind] = take(scr, n);
                if (M.ccanon >= 0) M.tmp[ind] = take(scr, n);
                M.fin[ind] = take(keep, n);
            }
            m2m_mats[key] = M;
        }
        for (int i = dr.first; i < dr.second; ++i) {
            if (l2l_seen[dn.v[i].did]) continue;
            l2l_seen[dn.v[i].did] = 1;
            auto key = std::make_pair(W, dn.v[i].dir);
            const DirPts& dp = get_dir(W, dn.v[i].dir);
            DirMats M{};
            child_pts(W, dn.v[i].dir, false, M.mrows, M.ccanon);
            M.mcols = dp.r2;
            M.canon = dp.canon;
            M.cached = !opctx_.empty();
            for (int ind = 0; ind < 8 && M.cached; ++ind)
                M.cached = (M.pk[ind] = cached_op(opk("l2l", W, dn.v[i].dir, ind))) != nullptr;
            for (int ind = 0; ind < 8 && !M.cached; ++ind) {
                size_t n = (size_t)M.mrows * M.mcols;
                M.raw[ind] = take(scr, n);
                M.fin[ind] = take(keep, n);
                M.tmp[ind] = M.ccanon >= 0 ? take(scr, n) : M.fin[ind];
            }
            l2l_mats[key] = M;
        }
    }
    phase("m2m_l2l_plan");
    // M2L: canonical offset o_c = S^-1 (c_t - c_s), so M(dir, o) = M(canon, o_c)
    std::unordered_map<uint64_t, int> m2l_id;  // (canon, ox, oy, oz) packed -> matrix
    struct M2LMat {
        size_t raw, tmp, fin;
        int canon, r1;
        Pt3 shift;
        const float* pk;  // packed copy from the shared cache, or null
        std::string key;
    };
    std::vector<M2LMat> m2l_mats;
    std::map<int, std::vector<std::vector<long long> > > m2l_x, m2l_y;  // level -> per problem columns
    std::map<int, std::vector<int> > m2l_probs;                         // level -> matrix ids
    {
        // far pairs listed on all host cores (plan.cpp), merged here in chunk order:
        // matrix ids, problem order and column order as one pass in node order
        std::vector<M2LChunk> chunks = m2l_pairs(T, up, dn);
        std::vector<int> local;  // matrix id -> problem index within its level (-1: none yet)
        int cur_level = INT_MIN;
        for (M2LChunk& C : chunks) {
            if (C.level != cur_level) {
                cur_level = C.level;
                local.assign(m2l_mats.size(), -1);
            }
            const double W = T.width(C.level);
            auto& X = m2l_x[C.level];
            auto& Y = m2l_y[C.level];
            auto& Pids = m2l_probs[C.level];
            for (size_t k = 0; k < C.keys.size(); ++k) {
                auto mit = m2l_id.find(C.keys[k]);
                int gid;
                if (mit == m2l_id.end()) {
                    const Canon& c = hfcanon[C.kcanon[k]];
                    const std::array<int, 3>& oc = C.koc[k];
                    gid = (int)m2l_mats.size();
                    size_t n = (size_t)c.r1 * c.r1;
                    const std::string key = opk("m2l", W, c.srt, oc[0], oc[1], oc[2]);
                    const float* pk = cached_op(key);
                    M2LMat M{0, 0, 0, C.kcanon[k], c.r1, Pt3{{oc[0] * W, oc[1] * W, oc[2] * W}}, pk, key};
                    if (!pk) {
                        M.raw = take(scr, n);
                        M.tmp = take(scr, n);
                        M.fin = take(keep, n);
                    }
                    m2l_mats.push_back(M);
                    m2l_id[C.keys[k]] = gid;
                } else {
                    gid = mit->second;
                }
                if ((size_t)gid >= local.size()) local.resize(m2l_mats.size(), -1);
                int li = local[gid];
                if (li < 0) {
                    li = (int)Pids.size();
                    local[gid] = li;
                    Pids.push_back(gid);
                    X.emplace_back();
                    Y.emplace_back();
                }
                X[li].insert(X[li].end(), C.X[k].begin(), C.X[k].end());
                Y[li].insert(Y[li].end(), C.Y[k].begin(), C.Y[k].end());
            }
            stats_.hf_far_pairs += C.pairs;
            std::vector<std::vector<long long> >().swap(C.X);
            std::vector<std::vector<long long> >().swap(C.Y);
        }
    }
    phase("m2l_plan");
    stats_.m2l_matrices = (long long)m2l_mats.size();
    // right factors E1 and E3^T as gatherable columns in the scratch pool
    std::vector<size_t> scr_E1(hfcanon.size()), scr_E3t(hfcanon.size());
    for (size_t c = 0; c < hfcanon.size(); ++c) {
        scr_E1[c] = take(scr, (size_t)hfcanon[c].r1 * hfcanon[c].r1);
        scr_E3t[c] = take(scr, (size_t)hfcanon[c].r2 * hfcanon[c].r2);
    }
    double2* dkeep = dalloc<double2>(keep);
    double2* dscr = nullptr;
    if (scr) CK(cudaMalloc(&dscr, sizeof(double2) * scr));
    flush_uploads();
    for (size_t c = 0; c < hfcanon.size(); ++c) {
        CK(cudaMemcpyAsync(dscr + scr_E1[c], hfcanon[c].E1, sizeof(double2) * hfcanon[c].r1 * hfcanon[c].r1,
                           cudaMemcpyDeviceToDevice, stream_));
        CK(cudaMemcpyAsync(dscr + scr_E3t[c], hfcanon[c].E3t, sizeof(double2) * hfcanon[c].r2 * hfcanon[c].r2,
                           cudaMemcpyDeviceToDevice, stream_));
    }
    for (auto& kv : m2m_mats) {
        if (kv.second.cached) continue;
        double W = kv.first.first;
        const DirPts& dp = get_dir(W, kv.first.second);
        int rc, cc;
        const double* cp = child_pts(W, kv.first.second, true, rc, cc);
        for (int ind = 0; ind < 8; ++ind)
            add_job(dp.ucp, zero3, cp, shifted_point(ind, W), dp.r2, rc, dscr + kv.second.raw[ind]);
    }
    for (auto& kv : l2l_mats) {
        if (kv.second.cached) continue;
        double W = kv.first.first;
        const DirPts& dp = get_dir(W, kv.first.second);
        int rc, cc;
        const double* cp = child_pts(W, kv.first.second, false, rc, cc);
        for (int ind = 0; ind < 8; ++ind)
            add_job(cp, shifted_point(ind, W), dp.dep, zero3, rc, dp.r2, dscr + kv.second.raw[ind]);
    }
    for (const M2LMat& M : m2l_mats)
        if (!M.pk) add_job(hfcanon[M.canon].neg_uep, M.shift, hfcanon[M.canon].uep, zero3, M.r1, M.r1, dscr + M.raw);

    phase("job_list");
    // generate every kernel matrix now
    if (!jobs.empty()) {
        KmatJob* d_jobs = upload(jobs);
        flush_uploads();
        launch_kmat(d_jobs, (int)jobs.size(), job_elems, kern, stream_);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(stream_));
    }

    phase("kmat");
    // fold: right products (raw * E1 or raw * E3^T), then left products (E3 * . or E1^T * .)
    if (scr) {
        GemmBatch right_s, right_k, left;
        for (auto& kv : m2m_mats) {
            const DirMats& M = kv.second;
            for (int ind = 0; ind < 8 && !M.cached; ++ind) {
                if (M.ccanon >= 0) {  // tmp = ue2uc * E1(child)
                    right_s.product(dscr + M.raw[ind], M.mrows, M.mcols, scr_E1[M.ccanon], M.mcols, M.tmp[ind]);
                    left.product(hfcanon[M.canon].E3, M.mrows, M.mrows, M.tmp[ind], M.mcols, M.fin[ind]);
                } else {
                    left.product(hfcanon[M.canon].E3, M.mrows, M.mrows, M.raw[ind], M.mcols, M.fin[ind]);
                }
            }
        }
        for (auto& kv : l2l_mats) {
            const DirMats& M = kv.second;
            for (int ind = 0; ind < 8 && !M.cached; ++ind) {
                if (M.ccanon >= 0) {  // tmp = de2dc * E3^T ; fin = E1(child)^T * tmp
                    right_s.product(dscr + M.raw[ind], M.mrows, M.mcols, scr_E3t[M.canon], M.mcols, M.tmp[ind]);
                    left.product(hfcanon[M.ccanon].E1t, M.mrows, M.mrows, M.tmp[ind], M.mcols, M.fin[ind]);
                } else {  // children are low-frequency boxes: fin = de2dc * E3^T
                    right_k.product(dscr + M.raw[ind], M.mrows, M.mcols, scr_E3t[M.canon], M.mcols, M.fin[ind]);
                }
            }
        }
        for (const M2LMat& M : m2l_mats) {
            if (M.pk) continue;
            right_s.product(dscr + M.raw, M.r1, M.r1, scr_E1[M.canon], M.r1, M.tmp);
            left.product(hfcanon[M.canon].E1t, M.r1, M.r1, M.tmp, M.r1, M.fin);
        }
        right_s.run(dscr, dscr, stream_);
        right_k.run(dscr, dkeep, stream_);
        left.run(dscr, dkeep, stream_);
        CK(cudaStreamSynchronize(stream_));
        CK(cudaFree(dscr));
    }
    phase("fold");
    const double2* dkeepm = opm(dkeep, keep);
    auto KP = [&](size_t off) { return E((double2*)dkeepm, off); };

    // ---------------------------------------------------------------- steps: LF upward
    auto lf_set = [&](const double* x, int n, Pt3 shift, double scale) {
        PtSet s;
        s.x = x;
        s.n = n;
        for (int d = 0; d < 3; ++d) s.shift[d] = shift[d];
        s.scale = scale;
        return s;
    };
    auto leaf_set = [&](int l) { return lf_set(d_pos_sorted_ + 3 * (size_t)leaf_off[l], leaf_cnt[l], zero3, 1.0); };
    auto single = [&](const GemmProblem& p, const std::vector<long long>& x, const std::vector<long long>& y,
                      const double2* X, double2* Y, int mode, const char* label) {
        std::vector<GemmProblem> ps(1, p);
        std::vector<std::vector<long long> > xo(1, x), yo(1, y);
        add_gemm(ps, xo, yo, X, Y, mode, label);
    };
    for (auto it = lflevels.rbegin(); it != lflevels.rend(); ++it) {
        const LfLevelOps& L = lfops[it->first];
        const auto& ids = it->second;
        begin_block(0, L.W);
        // S2M at leaves (src/wave3d_eval.cpp:441-451)
        std::vector<PtItem> items;
        std::vector<PtSrc> srcs;
        for (int l : ids) {
            const Box& B = T.boxes[lfbox[l]];
            if (!B.terminal()) continue;
            PtItem itm;
            itm.trg = lf_set(L.ucp, nE, T.center(B), 1.0);
            itm.out = E(lf_upchk, (size_t)l * nE);
            itm.src_begin = (int)srcs.size();
            srcs.push_back(PtSrc{leaf_set(l), E(d_den_sorted_, leaf_off[l])});
            itm.src_end = (int)srcs.size();
            items.push_back(itm);
        }
        add_pt(items, srcs, "lf_s2m");
        // M2M from children (src/wave3d_eval.cpp:452-463)
        if (L.has_children)
            for (int ind = 0; ind < 8; ++ind) {
                std::vector<long long> x, y;
                for (int l : ids) {
                    int b = lfbox[l];
                    if (T.boxes[b].terminal()) continue;
                    int c = T.child(b, ind);
                    if (c < 0 || !T.boxes[c].has_pts()) continue;
                    x.push_back((long long)lfidx[c] * nE);
                    y.push_back((long long)l * nE);
                }
                single(GemmProblem{opm(L.ue2uc[ind], (size_t)nE * nE), nE, nE, nE, 0, 0}, x, y, lf_upeq, lf_upchk, GEMM_ADD,
                       "lf_m2m");
            }
        // upeqnden = v * (1/sigma .* (U^H * upchk))   (src/wave3d_eval.cpp:466-478)
        std::vector<long long> a, b2;
        for (int l : ids) {
            a.push_back((long long)l * nE);
            b2.push_back((long long)l * nE);
        }
        single(GemmProblem{opm(L.up_s, (size_t)L.r * nE), L.r, nE, L.r, 0, 0}, a, b2, lf_upchk, lf_mid, GEMM_SET,
               "lf_uc2ue");
        single(GemmProblem{opm(L.v, (size_t)L.r * nE), nE, L.r, nE, 0, 0}, a, b2, lf_mid, lf_upeq, GEMM_SET,
               "lf_uc2ue");
    }

    phase("steps_lf_up");
    // children with points of every high-frequency box (-1: none)
    std::vector<int> kids((size_t)nb * 8, -1);
    for (auto& kv : hflevels)
        for (int b : kv.second)
            for (int ind = 0; ind < 8; ++ind) {
                const int c = T.child(b, ind);
                if (c >= 0 && T.boxes[c].has_pts()) kids[(size_t)b * 8 + ind] = c;
            }
    // the column lists of every level's M2M, E2, E2^T and L2L launches, built on
    // all host cores (plan.cpp)
    std::vector<std::pair<double, Idx3> > did_wedge(dirpts.size());
    for (auto& kv : dirpts) did_wedge[kv.second.did] = kv.first;
    std::vector<long long> lf_off(nb, -1);
    for (int l = 0; l < nLF; ++l) lf_off[lfbox[l]] = (long long)l * nE;
    HfColumns cols = hf_columns(T, up, dn, kids, lf_off, dirpts.size(), hfcanon.size());
    phase("hf_columns");
    // ---------------------------------------------------------------- steps: HF upward
    // widths ascending = levels descending; hf_upeq holds w (upeqnden = E1 w)
    for (auto hit = hflevels.rbegin(); hit != hflevels.rend(); ++hit) {
        int level = hit->first;
        double W = T.width(level);
        auto ur = up.range[level];
        if (ur.first == ur.second) continue;
        begin_block(1, W);
        Step ms{};
        ms.kind = 4;
        ms.label = "memset";
        ms.ms = Memset{T0, es * (size_t)tmp_up_level[level]};  // this level's sums only
        push_step(ms);
        // M2M: E3 upchkval = sum_children [E3 ue2uc E1(child)] w_child (src/wave3d_eval.cpp:796-834),
        // one launch for the 8 child positions: a problem per (wedge, child), all adding into
        // the parents' sums
        {
            ColLists& L = cols.m2m.at(level);
            std::vector<GemmProblem> probs;
            for (int k : L.key) {
                const Idx3& dir = did_wedge[k / 8].second;
                const int ind = k % 8;
                const DirMats& M = m2m_mats.at(std::make_pair(W, dir));
                if (M.cached) {
                    probs.push_back(GemmProblem{nullptr, M.mrows, M.mcols, M.mrows, 0, 0, M.pk[ind]});
                } else {
                    probs.push_back(GemmProblem{KP(M.fin[ind]), M.mrows, M.mcols, M.mrows, 0, 0});
                    if (!opctx_.empty()) opkey_[KP(M.fin[ind])] = opk("m2m", W, dir, ind);
                }
            }
            add_gemm(probs, L.x, L.y, W == 1.0 ? lf_upeq : hf_upeq, T0, GEMM_ATOMIC, width_label("hf_m2m", W));
        }
        // w = E2 * (E3 upchkval)   (src/wave3d_eval.cpp:837-849)
        {
            ColLists& L = cols.e2.at(level);
            std::vector<GemmProblem> p2;
            for (int k : L.key) {
                const Canon& c = hfcanon[k];
                const std::string key = opk("e2", c.W, c.srt, 0);
                if (const float* pk = cached_op(key)) {
                    p2.push_back(GemmProblem{nullptr, c.r1, c.r2, c.r1, 0, 0, pk});
                } else {
                    const double2* a = opm(c.E2, (size_t)c.r1 * c.r2);
                    p2.push_back(GemmProblem{a, c.r1, c.r2, c.r1, 0, 0});
                    if (!opctx_.empty()) opkey_[a] = key;
                }
            }
            add_gemm(p2, L.x, L.y, T0, hf_upeq, GEMM_SET, width_label("hf_uc2ue", W));
        }
    }

    phase("steps_hf_up");
    // ---------------------------------------------------------------- steps: HF downward
    // widths descending = levels ascending; hf_dnchk holds u = E1^T dnchkval
    for (auto it = hflevels.begin(); it != hflevels.end(); ++it) {
        int level = it->first;
        double W = T.width(level);
        auto dr = dn.range[level];
        if (dr.first == dr.second) continue;
        begin_block(2, W);
        // M2L (src/wave3d_eval.cpp:876-928)
        {
            std::vector<GemmProblem> probs;
            for (int gid : m2l_probs[level]) {
                const M2LMat& M = m2l_mats[gid];
                if (M.pk) {
                    probs.push_back(GemmProblem{nullptr, M.r1, M.r1, M.r1, 0, 0, M.pk});
                } else {
                    probs.push_back(GemmProblem{KP(M.fin), M.r1, M.r1, M.r1, 0, 0});
                    if (!opctx_.empty()) opkey_[KP(M.fin)] = M.key;
                }
            }
            add_gemm(probs, m2l_x[level], m2l_y[level], hf_upeq, hf_dnchk, GEMM_ATOMIC, width_label("hf_m2l", W));
        }
        // t = E2^T u   (dneqnden = E3^T t, src/wave3d_eval.cpp:938-948, src/mlib3d.cpp:246-250)
        {
            ColLists& L = cols.e2t.at(level);
            std::vector<GemmProblem> p2;
            for (int k : L.key) {
                const Canon& c = hfcanon[k];
                const std::string key = opk("e2t", c.W, c.srt, 0);
                if (const float* pk = cached_op(key)) {
                    p2.push_back(GemmProblem{nullptr, c.r2, c.r1, c.r2, 0, 0, pk});
                } else {
                    const double2* a = opm(c.E2t, (size_t)c.r1 * c.r2);
                    p2.push_back(GemmProblem{a, c.r2, c.r1, c.r2, 0, 0});
                    if (!opctx_.empty()) opkey_[a] = key;
                }
            }
            add_gemm(p2, L.x, L.y, hf_dnchk, T1, GEMM_SET, width_label("hf_dc2de", W));
        }
        // L2L into the children's (pdir) u, or LF dnchkval at W=1 (src/wave3d_eval.cpp:950-991),
        // one launch for the 8 child positions: a problem per (wedge, child)
        {
            ColLists& L = cols.l2l.at(level);
            std::vector<GemmProblem> probs;
            for (int k : L.key) {
                const Idx3& dir = did_wedge[k / 8].second;
                const int ind = k % 8;
                const DirMats& M = l2l_mats.at(std::make_pair(W, dir));
                if (M.cached) {
                    probs.push_back(GemmProblem{nullptr, M.mrows, M.mcols, M.mrows, 0, 0, M.pk[ind]});
                } else {
                    probs.push_back(GemmProblem{KP(M.fin[ind]), M.mrows, M.mcols, M.mrows, 0, 0});
                    if (!opctx_.empty()) opkey_[KP(M.fin[ind])] = opk("l2l", W, dir, ind);
                }
            }
            add_gemm(probs, L.x, L.y, T1, W == 1.0 ? lf_dnchk : hf_dnchk, GEMM_ATOMIC, width_label("hf_l2l", W));
        }
    }

    phase("steps_hf_down");
    // ---------------------------------------------------------------- steps: LF downward
    for (auto& kv : lflevels) {  // levels ascending = widths descending
        int level = kv.first;
        const LfLevelOps& L = lfops[level];
        const auto& ids = kv.second;
        double W = L.W;
        begin_block(3, W);
        // V list: FFT M2L (src/wave3d_eval.cpp:602-661).  The pointwise sums run by
        // target parent (kernels.cuh, VlistGroups): the targets of a parent share one
        // pass over the union of their V-list sources; then one inverse transform
        // per target.
        {
            const auto tv = std::chrono::steady_clock::now();
            VlistGroupPlan vg = vlist_groups(T, lfbox, lfidx, ids);
            t_emit_vgroups_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - tv).count();
            stats_.v_pairs += vg.pairs;
            const std::vector<int>& trg = vg.trg;
            if (!trg.empty()) {
                const std::vector<int>& srcb = vg.src;
                VlistLevel VL{G, P, nE, L.cube_idx, L.tns, d_twf, d_twb};  // FP32 data in the mixed form
                Step f{};
                f.kind = 2;
                f.label = "lf_vlist_fft";
                f.flops = 8.0 * 3 * (double)G3 * G * srcb.size();
                f.bytes = 16.0 * ((double)nE + G3) * srcb.size();
                f.v.L = VL;
                f.v.src_boxes = upload(srcb);
                f.v.nsrc = (int)srcb.size();
                f.v.upeq = lf_upeq;
                f.v.spec = lf_spec;
                if (mixed) {
                    f.hvf = VfSub{VL, f.v.src_boxes, reinterpret_cast<const float2*>(lf_upeq),
                                  reinterpret_cast<float2*>(lf_spec), f.v.nsrc, 0};
                    set_multi(f, f.hvf, f.v.nsrc);
                }
                push_step(f);
                // summed target spectra: a high-frequency buffer when one is large enough
                // (every high-frequency pass has run before this low-frequency downward
                // step, so the outgoing densities, the incoming check values and both
                // temporaries are all free by then), else a buffer of their own
                const size_t tsp_elems = trg.size() * (size_t)G3;
                double2* tsp = tsp_elems <= (size_t)upeq_total    ? hf_upeq
                               : tsp_elems <= (size_t)dnchk_total ? hf_dnchk
                               : tsp_elems <= (size_t)tmp_max     ? T0
                                                                  : salloc(tsp_elems);
                const int ngroups = (int)vg.gptr.size() - 1;
                const long long npairs = vg.pairs;
                Step a{};
                a.kind = 3;
                a.label = "lf_vlist_m2l";
                a.flops = 8.0 * (double)G3 * npairs;
                // compulsory: each source spectrum, the 316 tensors, each target's summed spectrum
                a.bytes = 16.0 * ((double)G3 * srcb.size() + 316.0 * G3 + (double)G3 * trg.size());
                a.v.L = VL;
                a.v.grp = VlistGroups{upload(vg.gptr), reinterpret_cast<const int2*>(upload(vg.gsrc)), upload(vg.gtrg),
                                      ngroups};
                a.v.spec = lf_spec;
                a.v.tsp = tsp;
                if (mixed) {
                    a.hva = VaSub{VL, a.v.grp.gptr, a.v.grp.gsrc, a.v.grp.gtrg, reinterpret_cast<const float2*>(lf_spec),
                                  reinterpret_cast<float2*>(tsp), ngroups, 0};
                    set_multi(a, a.hva, ngroups);
                }
                push_step(a);
                Step iv{};
                iv.kind = 6;
                iv.label = "lf_vlist_inv";
                iv.flops = 8.0 * (double)G * ((double)G * G * P + G * P * P + P * P * P) * trg.size();
                iv.bytes = 16.0 * ((double)G3 + 2.0 * nE) * trg.size();
                iv.v.L = VL;
                iv.v.trg = upload(trg);
                iv.v.ntrg = (int)trg.size();
                iv.v.tsp = tsp;
                iv.v.dnchk = lf_dnchk;
                if (mixed) {
                    iv.hvi = ViSub{VL, iv.v.trg, reinterpret_cast<const float2*>(tsp), reinterpret_cast<float2*>(lf_dnchk),
                                   iv.v.ntrg, 0};
                    set_multi(iv, iv.hvi, iv.v.ntrg);
                }
                push_step(iv);
            }
        }
        // X list (src/wave3d_eval.cpp:663-686), into dnchk or, for small leaves, into extval
        {
            std::vector<PtItem> itemsA, itemsB;
            std::vector<PtSrc> srcsA, srcsB;
            for (int l : ids) {
                const Box& B = T.boxes[lfbox[l]];
                if (B.xlist.empty()) continue;
                bool direct = B.terminal() && leaf_cnt[l] < nE;
                PtItem itm;
                itm.trg = direct ? leaf_set(l) : lf_set(L.uep, nE, T.center(B), 1.0);
                itm.out = direct ? E(d_val_sorted_, leaf_off[l]) : E(lf_dnchk, (size_t)l * nE);
                auto& S = direct ? srcsA : srcsB;
                itm.src_begin = (int)S.size();
                for (int s : B.xlist) {
                    int ls = lfidx[s];
                    S.push_back(PtSrc{leaf_set(ls), E(d_den_sorted_, leaf_off[ls])});
                    stats_.x_pairs++;
                }
                itm.src_end = (int)S.size();
                (direct ? itemsA : itemsB).push_back(itm);
            }
            add_pt(itemsA, srcsA, "lf_xlist");
            add_pt(itemsB, srcsB, "lf_xlist");
        }
        // U list (src/wave3d_eval.cpp:585-600) and W list (:688-718) into extval
        {
            std::vector<PtItem> items, witems;
            std::vector<PtSrc> srcs, wsrcs;
            for (int l : ids) {
                const Box& B = T.boxes[lfbox[l]];
                if (!B.ulist.empty()) {
                    PtItem itm;
                    itm.trg = leaf_set(l);
                    itm.out = E(d_val_sorted_, leaf_off[l]);
                    itm.src_begin = (int)srcs.size();
                    for (int s : B.ulist) {
                        int ls = lfidx[s];
                        srcs.push_back(PtSrc{leaf_set(ls), E(d_den_sorted_, leaf_off[ls])});
                        stats_.u_pairs++;
                        stats_.u_interactions += (long long)leaf_cnt[l] * leaf_cnt[ls];
                    }
                    itm.src_end = (int)srcs.size();
                    items.push_back(itm);
                }
                if (!B.wlist.empty()) {
                    PtItem itm;
                    itm.trg = leaf_set(l);
                    itm.out = E(d_val_sorted_, leaf_off[l]);
                    itm.src_begin = (int)wsrcs.size();
                    for (int s : B.wlist) {
                        int ls = lfidx[s];
                        const Box& SB = T.boxes[s];
                        if (SB.terminal() && leaf_cnt[ls] < nE) {
                            wsrcs.push_back(PtSrc{leaf_set(ls), E(d_den_sorted_, leaf_off[ls])});
                        } else {
                            double coef = T.width(SB.level) / W;
                            wsrcs.push_back(PtSrc{lf_set(L.uep, nE, T.center(SB), coef), E(lf_upeq, (size_t)ls * nE)});
                        }
                        stats_.w_pairs++;
                    }
                    itm.src_end = (int)wsrcs.size();
                    witems.push_back(itm);
                }
            }
            add_pt(items, srcs, "lf_ulist");
            add_pt(witems, wsrcs, "lf_wlist");
        }
        // dneqnden = up^T (1/sigma .* (v^T dnchk))   (src/wave3d_eval.cpp:536-547, src/mlib3d.cpp:147-152)
        std::vector<long long> a;
        for (int l : ids) a.push_back((long long)l * nE);
        single(GemmProblem{opm(L.vT_s, (size_t)L.r * nE), L.r, nE, L.r, 0, 0}, a, a, lf_dnchk, lf_mid, GEMM_SET,
               "lf_dc2de");
        single(GemmProblem{opm(L.upT, (size_t)L.r * nE), nE, L.r, nE, 0, 0}, a, a, lf_mid, lf_dneq, GEMM_SET,
               "lf_dc2de");
        // L2T at leaves (src/wave3d_eval.cpp:550-560)
        {
            std::vector<PtItem> items;
            std::vector<PtSrc> srcs;
            for (int l : ids) {
                const Box& B = T.boxes[lfbox[l]];
                if (!B.terminal()) continue;
                PtItem itm;
                itm.trg = leaf_set(l);
                itm.out = E(d_val_sorted_, leaf_off[l]);
                itm.src_begin = (int)srcs.size();
                srcs.push_back(PtSrc{lf_set(L.ucp, nE, T.center(B), 1.0), E(lf_dneq, (size_t)l * nE)});
                itm.src_end = (int)srcs.size();
                items.push_back(itm);
            }
            add_pt(items, srcs, "lf_l2t");
        }
        // L2L to the children (src/wave3d_eval.cpp:562-579)
        if (L.has_children)
            for (int ind = 0; ind < 8; ++ind) {
                std::vector<long long> x, y;
                for (int l : ids) {
                    int b = lfbox[l];
                    if (T.boxes[b].terminal()) continue;
                    int c = T.child(b, ind);
                    if (c < 0 || !T.boxes[c].has_pts()) continue;
                    x.push_back((long long)l * nE);
                    y.push_back((long long)lfidx[c] * nE);
                }
                single(GemmProblem{opm(L.de2dc[ind], (size_t)nE * nE), nE, nE, nE, 0, 0}, x, y, lf_dneq, lf_dnchk, GEMM_ADD,
                       "lf_l2l");
            }
    }
    phase("steps_lf_down");
    if (trace)
        std::fprintf(stderr,
                     "ddfmm setup   (host seconds in GEMM step emission %.3f, V-list grouping %.3f, uploads above "
                     "64 KB %.3f, operator packing %.3f of which chunk allocation %.3f; %lld device allocations "
                     "%.3f, %lld staged copies: waits %.3f, host copies %.3f)\n",
                     t_emit_gemm_, t_emit_vgroups_, t_big_uploads_, t_pack_, t_pack_alloc_, n_malloc_, t_malloc_,
                     n_stage_, t_stage_wait_, t_stage_copy_);
    flush_packs();
    if (mixed) {
        // the mixed eval reads only the FP32 copies (and, on tcgen05, only the packed
        // GEMM operators): release the FP64 operators and the unpacked GEMM copies
        CK(cudaStreamSynchronize(stream_));
        std::set<const void*> vlist32{d_twf, d_twb};
        for (auto& kv : lfops) vlist32.insert(kv.second.tns);
        for (auto& kv : op32) {
            dfree(kv.first);
            if (umma() && !vlist32.count(kv.second)) dfree(kv.second);
        }
    }
    flush_uploads();
    CK(cudaStreamSynchronize(stream_));
    stage_release();
    std::vector<char>().swap(arena_.host);  // every chunk is on the device now
    arena_.retired.clear();
    arena_.used = arena_.sent = arena_.cap;
    phase("packs_release");
    stats_.kernel_launches = (long long)steps_.size() + 2;
}

static const char* kernel_name(int kind, int tpi) {
    switch (kind) {
        case 0: return "zgemm_kernel";
        case 1:
            switch (tpi) {  // the launch shape the autotuner chose
                case 4: return "pt_kernel<4>";
                case 8: return "pt_kernel<8>";
                case 16: return "pt_kernel<16>";
                case PT_WARP_TARGETS: return "ptw_kernel<targets,4>";
                case PT_WARP_TARGETS2: return "ptw_kernel<targets,2>";
                case PT_WARP_SOURCES: return "ptw_kernel<sources,8>";
                case PT_WARP_SOURCES4: return "ptw_kernel<sources,4>";
                default: return "pt_kernel<32>";
            }
        case 2: return "vlist_forward_kernel";
        case 3: return "vlist_group_kernel";
        case 6: return "vlist_inverse_kernel";
        case 5: return "umma_cgemm_kernel";
        default: return "memset";
    }
}

void Session::launch_step(const Step& st, cudaStream_t s, double2* spec) {
    const bool m = mixed();
    switch (st.kind) {
        case 0:
            if (m)
                launch_cgemm(st.g.probs, st.g.tiles, st.g.ntiles, st.g.xoff, st.g.yoff, st.g.X, st.g.Y, st.g.mode, s);
            else
                launch_gemm(st.g.probs, st.g.tiles, st.g.ntiles, st.g.xoff, st.g.yoff, st.g.X, st.g.Y, st.g.mode, s);
            break;
        case 1:
            if (m)
                launch_pt32(static_cast<const PtSub*>(st.msubs), st.mpre, 1, st.mtotal, nullptr, s, st.tpi ? st.tpi : 32);
            else
                launch_pt(st.pt.items, st.pt.nitems, st.pt.srcs, prm_.kernel, s, st.tpi ? st.tpi : 32);
            break;
        case 2:
            if (m)
                launch_vlist_forward32(static_cast<const VfSub*>(st.msubs), st.mpre, 1, st.mtotal, st.v.L.G, nullptr,
                                       spec != st.v.spec ? spec : nullptr, s, &st.hvf);
            else
                launch_vlist_forward(st.v.L, st.v.src_boxes, st.v.nsrc, st.v.upeq, spec, s);
            break;
        case 3:
            if (m)
                launch_vlist_group32(static_cast<const VaSub*>(st.msubs), st.mpre, 1, st.mtotal, st.v.L.G, nullptr,
                                     spec != st.v.spec ? spec : nullptr, s, &st.hva);
            else
                launch_vlist_group(st.v.L, st.v.grp, spec, st.v.tsp, s);
            break;
        case 6:
            if (m)
                launch_vlist_inverse32(static_cast<const ViSub*>(st.msubs), st.mpre, 1, st.mtotal, st.v.L.G, nullptr, s,
                                       &st.hvi);
            else
                launch_vlist_inverse(st.v.L, st.v.trg, st.v.ntrg, st.v.tsp, st.v.dnchk, s);
            break;
        case 4:
            CK(cudaMemsetAsync(st.ms.p, 0, st.ms.bytes, s));
            break;
        case 5: {
            const unsigned long long wait_ns = stall_wait_ns_;
            stall_wait_ns_ = 0;  // one launch only
            launch_umma_cgemm(static_cast<const UmmaSub*>(st.msubs), st.mpre, 1, st.mtotal, nullptr, d_err_, s, &st.hu,
                              wait_ns, wait_ns ? 1 : 0);
            break;
        }
    }
}

// The accumulators a point-interaction step writes are zeroed at the start of
// every eval, so running it here on setup-time contents is harmless.
void Session::autotune() {
    cudaEvent_t a = nullptr, b = nullptr;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (Step& st : steps_) {
        if (st.kind != 1) continue;
        static const std::vector<int> shapes{32, 16, 8, 4, PT_WARP_TARGETS, PT_WARP_TARGETS2, PT_WARP_SOURCES,
                                             PT_WARP_SOURCES4};
        float best = 0.f;
        int best_tpi = shapes[0];
        // per-launch time of one shape over `reps` launches after a warm-up
        auto time_shape = [&](int reps) {
            launch_step(st, stream_, st.v.spec);
            CK(cudaEventRecord(a, stream_));
            for (int r = 0; r < reps; ++r) launch_step(st, stream_, st.v.spec);
            CK(cudaEventRecord(b, stream_));
            CK(cudaEventSynchronize(b));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, a, b));
            return ms / reps;
        };
        for (int tpi : shapes) {
            st.tpi = tpi;
            float ms = time_shape(3);
            // short steps: time over ~0.5 ms of launches, or three launches read mostly noise
            if (ms * 3 < 0.5f) ms = time_shape(std::min(50, (int)(0.5f / std::max(ms, 1e-3f)) + 1));
            if (tpi == shapes[0] || ms < best) {
                best = ms;
                best_tpi = tpi;
            }
        }
        st.tpi = best_tpi;
        stats_.tuned_steps++;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
}

void Session::run_steps(cudaStream_t s) {
    for (const Memset& m : zero_at_start_) CK(cudaMemsetAsync(m.p, 0, m.bytes, s));
    if (profiling_ && ev_.size() < 2 * steps_.size()) {
        size_t have = ev_.size();
        ev_.resize(2 * steps_.size());
        for (size_t i = have; i < ev_.size(); ++i) CK(cudaEventCreate(&ev_[i]));
    }
    if (profiling_ && !ev_pending_.empty()) profile_read();  // keep one eval of events in flight at most
    for (size_t i = 0; i < steps_.size(); ++i) {
        const Step& st = steps_[i];
        if (profiling_) CK(cudaEventRecord(ev_[2 * i], s));
        launch_step(st, s, st.v.spec);
        if (profiling_) {
            CK(cudaEventRecord(ev_[2 * i + 1], s));
            ev_pending_.push_back(std::make_pair((int)i, (int)(2 * i)));
        }
    }
}

void Session::profile_enable(bool on) {
    if (!on && !ev_pending_.empty()) profile_read();
    profiling_ = on;
}

std::vector<Session::ProfileEntry> Session::profile_read() {
    for (auto& pe : ev_pending_) {
        CK(cudaEventSynchronize(ev_[pe.second + 1]));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev_[pe.second], ev_[pe.second + 1]));
        const Step& st = steps_[pe.first];
        ProfileEntry& e = prof_[st.label];
        e.label = st.label;
        e.kernel = kernel_name(st.kind, st.tpi);
        e.launches += 1;
        e.ms += ms;
        e.flops += st.flops;
        e.bytes += st.bytes;
    }
    ev_pending_.clear();
    // in launch order: by the first step of each label
    std::vector<ProfileEntry> out;
    std::set<std::string> seen;
    for (const Step& st : steps_) {
        auto it = prof_.find(st.label);
        if (it != prof_.end() && seen.insert(st.label).second) out.push_back(it->second);
    }
    return out;
}

void Session::eval_device(const double2* den, double2* val, cudaStream_t s) {
    if (mixed())
        launch_gather32(den, d_perm_, d_den_sorted_, npts_, 0, s);
    else
        launch_gather_den(den, d_perm_, d_den_sorted_, npts_, s);
    run_steps(s);
    if (mixed())
        launch_scatter32(d_val_sorted_, d_perm_, val, npts_, 0, s);
    else
        launch_scatter_val(d_val_sorted_, d_perm_, val, npts_, s);
    CK(cudaGetLastError());
}

void Session::eval_device_c64(const float2* den, float2* val, cudaStream_t s) {
    if (!mixed()) throw std::invalid_argument("complex64 evaluation needs a mixed-precision session");
    launch_gather32(den, d_perm_, d_den_sorted_, npts_, 1, s);
    run_steps(s);
    launch_scatter32(d_val_sorted_, d_perm_, val, npts_, 1, s);
    CK(cudaGetLastError());
}

void Session::eval_host_c64(const std::complex<float>* den, std::complex<float>* val) {
    if (!mixed()) throw std::invalid_argument("complex64 evaluation needs a mixed-precision session");
    CK(cudaMemcpyAsync(d_den_io_, den, sizeof(float2) * npts_, cudaMemcpyHostToDevice, stream_));
    eval_device_c64((const float2*)d_den_io_, (float2*)d_val_io_, stream_);
    CK(cudaMemcpyAsync(val, d_val_io_, sizeof(float2) * npts_, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    check_device_error();
}

// run_steps with the V-list launches on `spec` for the spectra, no profiling.
void Session::run_steps_spec(cudaStream_t s, double2* spec) {
    for (const Memset& m : zero_at_start_) CK(cudaMemsetAsync(m.p, 0, m.bytes, s));
    for (const Step& st : steps_) launch_step(st, s, spec);
}

void Session::eval_device_scratch(const double2* den, double2* val, cudaStream_t s, double2* spec, size_t capacity) {
    const size_t es = mixed() ? sizeof(float2) : sizeof(double2);
    if (spectra_elems_ * es > capacity * sizeof(double2)) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "the session's V-list spectra need %.1f MiB, more than the %.1f MiB of fixed scratch",
                 spectra_elems_ * es / 1048576.0, capacity * sizeof(double2) / 1048576.0);
        throw std::invalid_argument(msg);
    }
    if (mixed())
        launch_gather32(den, d_perm_, d_den_sorted_, npts_, 0, s);
    else
        launch_gather_den(den, d_perm_, d_den_sorted_, npts_, s);
    run_steps_spec(s, spec);
    if (mixed())
        launch_scatter32(d_val_sorted_, d_perm_, val, npts_, 0, s);
    else
        launch_scatter_val(d_val_sorted_, d_perm_, val, npts_, s);
    CK(cudaGetLastError());
}

void Session::eval_host(const std::complex<double>* den, std::complex<double>* val) {
    CK(cudaMemcpyAsync(d_den_io_, den, sizeof(double2) * npts_, cudaMemcpyHostToDevice, stream_));
    eval_device(d_den_io_, d_val_io_, stream_);
    CK(cudaMemcpyAsync(val, d_val_io_, sizeof(double2) * npts_, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    check_device_error();
}

void Session::direct_host(const std::complex<double>* den, const int* ids, int nids, std::complex<double>* out) {
    if (nids <= 0) return;
    for (int i = 0; i < nids; ++i)
        if (ids[i] < 0 || ids[i] >= npts_) throw std::runtime_error("check id out of range");
    int* d_ids = nullptr;
    double2* d_out = nullptr;
    CK(cudaMalloc(&d_ids, sizeof(int) * nids));
    CK(cudaMalloc(&d_out, sizeof(double2) * nids));
    CK(cudaMemcpyAsync(d_den_io_, den, sizeof(double2) * npts_, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(d_ids, ids, sizeof(int) * nids, cudaMemcpyHostToDevice, stream_));
    launch_direct(d_pos_ids_, d_den_io_, npts_, d_ids, nids, d_out, prm_.kernel, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d_out, sizeof(double2) * nids, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    cudaFree(d_ids);
    cudaFree(d_out);
}

}  // namespace ddfmm
