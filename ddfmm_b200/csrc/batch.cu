// Merged multi-instance launch sequence (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>

namespace ddfmm {

#define BCK(x)                                                                                     \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" + \
                                     #x + ")");                                                    \
    } while (0)

void* Batch::upload_bytes(const void* p, size_t bytes) {
    void* d = nullptr;
    BCK(cudaMalloc(&d, bytes ? bytes : 16));
    allocs_.push_back(d);
    if (bytes) BCK(cudaMemcpy(d, p, bytes, cudaMemcpyHostToDevice));
    return d;
}

// counts[j] = work items of sub-launch j; the device gets their prefix sums
template <class Sub, class Pre>
void Batch::add(Kind kind, const std::vector<Sub>& subs, const std::vector<Pre>& counts, int G) {
    if (subs.empty()) return;
    std::vector<Pre> prefix(1, 0);
    for (Pre c : counts) prefix.push_back(prefix.back() + c);
    Launch L;
    L.kind = kind;
    L.subs = upload_bytes(subs.data(), sizeof(Sub) * subs.size());
    L.prefix = upload_bytes(prefix.data(), sizeof(Pre) * prefix.size());
    L.nsub = (int)subs.size();
    L.total = (long long)prefix.back();
    L.G = G;
    static_assert(sizeof(Sub) <= sizeof(L.one), "sub-launch larger than its host copy");
    std::memcpy(L.one, subs.data(), sizeof(Sub));
    if (L.total > 0) launches_.push_back(L);
}

Batch::Batch(const std::vector<Session*>& sessions) : sessions_(sessions) {
    if (sessions_.empty()) throw std::invalid_argument("a batch needs at least one session");
    device_ = sessions_[0]->device();
    for (Session* s : sessions_) {
        if (!s->umma()) throw std::invalid_argument("batched sessions must use the mixed (tcgen05) form");
        if (s->device() != device_) throw std::invalid_argument("batched sessions must share one device");
    }
    int prev = -1;
    BCK(cudaGetDevice(&prev));
    BCK(cudaSetDevice(device_));
    BCK(cudaMalloc(&d_err_, sizeof(int)));
    BCK(cudaMemset(d_err_, 0, sizeof(int)));
    allocs_.push_back(d_err_);

    // eval prologue: zero the accumulators, densities into leaf order
    {
        std::vector<ZeroSub> z;
        std::vector<long long> n;
        std::vector<MoveSub> g;
        std::vector<int> gn;
        for (int i = 0; i < size(); ++i) {
            Session* S = sessions_[i];
            for (const Session::Memset& m : S->zero_at_start_) {
                if (m.bytes % 8) throw std::logic_error("accumulator size is not a multiple of 8 bytes");
                z.push_back(ZeroSub{m.p, (long long)(m.bytes / 8), i, 0});
                n.push_back((long long)(m.bytes / 8));
            }
            g.push_back(MoveSub{S->d_den_io_, S->d_perm_, S->d_den_sorted_, S->npts_, i});
            gn.push_back(S->npts_);
        }
        add(ZERO, z, n);
        add(GATHER, g, gn);
    }
    // the passes: steps with equal keys run as one launch, keys in ascending order
    std::map<long long, std::vector<std::pair<int, const Session::Step*> > > by_key;
    for (int i = 0; i < size(); ++i)
        for (const Session::Step& st : sessions_[i]->steps_) by_key[st.key].push_back(std::make_pair(i, &st));
    for (auto& kv : by_key) {
        // one launch per step kind present under the key (normally one kind)
        std::map<int, std::vector<std::pair<int, const Session::Step*> > > by_kind;
        for (auto& e : kv.second) by_kind[e.second->kind].push_back(e);
        for (auto& kk : by_kind) {
            const int kind = kk.first;
            if (kind == 5) {
                std::vector<UmmaSub> subs;
                std::vector<int> n;
                long long tiles = 0;
                for (auto& e : kk.second) {
                    UmmaSub u = e.second->hu;
                    u.inst = e.first;
                    subs.push_back(u);
                    n.push_back(u.ntiles);
                    tiles += u.ntiles;
                }
                add(GEMM, subs, n);
                // Instances share packed operators (the process-wide cache): tiles that
                // read one operator block run next to each other across instances, so
                // the block comes from DRAM once while the blocks in flight share it in
                // L2, instead of once per instance.  Within an operator, instance order
                // and each instance's tile order are kept.
                if (subs.size() > 1 && tiles > 0 && subs.size() < 256) {  // add() appended this launch
                    std::vector<std::pair<const float*, int> > key;
                    bool fits = true;
                    for (size_t j = 0; j < kk.second.size(); ++j) {
                        const std::vector<const float*>& op = kk.second[j].second->uop;
                        if ((int)op.size() != n[j] || op.size() >= (1u << 24)) fits = false;
                        for (size_t t = 0; fits && t < op.size(); ++t)
                            key.push_back(std::make_pair(op[t], (int)((j << 24) | t)));
                    }
                    if (fits) {
                        std::stable_sort(key.begin(), key.end(),
                                         [](const std::pair<const float*, int>& a, const std::pair<const float*, int>& b) {
                                             return a.first < b.first;
                                         });
                        std::vector<int> order(key.size());
                        for (size_t i = 0; i < key.size(); ++i) order[i] = key[i].second;
                        launches_.back().order = upload_bytes(order.data(), sizeof(int) * order.size());
                    }
                }
            } else if (kind == 1) {
                std::vector<PtSub> subs;
                std::vector<int> n;
                for (auto& e : kk.second) {
                    PtSub u = e.second->hp;
                    u.inst = e.first;
                    subs.push_back(u);
                    n.push_back(u.nitems);
                }
                add(PT, subs, n);
                if (!launches_.empty() && launches_.back().kind == PT) {
                    // the shape the session with the most items of the merged steps was tuned to
                    int tpi = 32, most = -1;
                    for (auto& e : kk.second)
                        if (e.second->hp.nitems > most) {
                            most = e.second->hp.nitems;
                            tpi = e.second->tpi ? e.second->tpi : 32;
                        }
                    launches_.back().tpi = tpi;
                }
            } else if (kind == 2 || kind == 3 || kind == 6) {
                // V-list launches are templated on the grid size: one launch per G
                std::map<int, std::vector<std::pair<int, const Session::Step*> > > by_g;
                for (auto& e : kk.second) by_g[e.second->v.L.G].push_back(e);
                for (auto& gg : by_g) {
                    if (kind == 2) {
                        std::vector<VfSub> subs;
                        std::vector<int> n;
                        for (auto& e : gg.second) {
                            VfSub u = e.second->hvf;
                            u.inst = e.first;
                            subs.push_back(u);
                            n.push_back(u.nbox);
                        }
                        add(VFWD, subs, n, gg.first);
                    } else if (kind == 3) {
                        std::vector<VaSub> subs;
                        std::vector<int> n;
                        for (auto& e : gg.second) {
                            VaSub u = e.second->hva;
                            u.inst = e.first;
                            subs.push_back(u);
                            n.push_back(u.ngroups);
                        }
                        add(VACC, subs, n, gg.first);
                    } else {
                        std::vector<ViSub> subs;
                        std::vector<int> n;
                        for (auto& e : gg.second) {
                            ViSub u = e.second->hvi;
                            u.inst = e.first;
                            subs.push_back(u);
                            n.push_back(u.ntrg);
                        }
                        add(VINV, subs, n, gg.first);
                    }
                }
            } else if (kind == 4) {
                std::vector<ZeroSub> subs;
                std::vector<long long> n;
                for (auto& e : kk.second) {
                    const Session::Memset& m = e.second->ms;
                    if (m.bytes % 8) throw std::logic_error("temporary size is not a multiple of 8 bytes");
                    subs.push_back(ZeroSub{m.p, (long long)(m.bytes / 8), e.first, 0});
                    n.push_back((long long)(m.bytes / 8));
                }
                add(ZERO, subs, n);
            } else {
                throw std::logic_error("step kind not supported in a batch");
            }
        }
    }
    // epilogue: values back to point-id order
    {
        std::vector<MoveSub> g;
        std::vector<int> gn;
        for (int i = 0; i < size(); ++i) {
            Session* S = sessions_[i];
            g.push_back(MoveSub{S->d_val_sorted_, S->d_perm_, S->d_val_io_, S->npts_, i});
            gn.push_back(S->npts_);
        }
        add(SCATTER, g, gn);
    }
    BCK(cudaSetDevice(prev));
}

Batch::~Batch() {
    for (Graph& g : graphs_) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    for (void* p : allocs_) cudaFree(p);
}

float2* Batch::den(int i) const { return reinterpret_cast<float2*>(sessions_.at(i)->d_den_io_); }
float2* Batch::val(int i) const { return reinterpret_cast<float2*>(sessions_.at(i)->d_val_io_); }

void Batch::run(const int* active, cudaStream_t s) {
    for (const Launch& L : launches_) {
        switch (L.kind) {
            case ZERO:
                launch_zero(static_cast<const ZeroSub*>(L.subs), static_cast<const long long*>(L.prefix), L.nsub,
                            L.total, active, s);
                break;
            case GATHER:
            case SCATTER:
                launch_move32(static_cast<const MoveSub*>(L.subs), static_cast<const int*>(L.prefix), L.nsub,
                              (int)L.total, active, L.kind == SCATTER, s);
                break;
            case GEMM:
                launch_umma_cgemm(static_cast<const UmmaSub*>(L.subs), static_cast<const int*>(L.prefix), L.nsub,
                                  (int)L.total, active, d_err_, s,
                                  L.nsub == 1 ? reinterpret_cast<const UmmaSub*>(L.one) : nullptr, 0, 0,
                                  static_cast<const int*>(L.order));
                break;
            case PT:
                launch_pt32(static_cast<const PtSub*>(L.subs), static_cast<const int*>(L.prefix), L.nsub, (int)L.total,
                            active, s, L.tpi);
                break;
            case VFWD:
                launch_vlist_forward32(static_cast<const VfSub*>(L.subs), static_cast<const int*>(L.prefix), L.nsub,
                                       (int)L.total, L.G, active, nullptr, s, L.nsub == 1 ? reinterpret_cast<const VfSub*>(L.one) : nullptr);
                break;
            case VACC:
                launch_vlist_group32(static_cast<const VaSub*>(L.subs), static_cast<const int*>(L.prefix), L.nsub,
                                     (int)L.total, L.G, active, nullptr, s, L.nsub == 1 ? reinterpret_cast<const VaSub*>(L.one) : nullptr);
                break;
            case VINV:
                launch_vlist_inverse32(static_cast<const ViSub*>(L.subs), static_cast<const int*>(L.prefix), L.nsub,
                                       (int)L.total, L.G, active, s, L.nsub == 1 ? reinterpret_cast<const ViSub*>(L.one) : nullptr);
                break;
        }
    }
    BCK(cudaGetLastError());
}

void Batch::run_graph(const int* active, cudaStream_t s) {
    for (const Graph& g : graphs_)
        if (g.active == active) {
            BCK(cudaGraphLaunch(g.exec, s));
            return;
        }
    if (graphs_.size() >= 4) {  // keep a few: the caller's mask arrays
        cudaGraphExecDestroy(graphs_.front().exec);
        cudaGraphDestroy(graphs_.front().graph);
        graphs_.erase(graphs_.begin());
    }
    Graph g{active, nullptr, nullptr};
    BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        run(active, s);
    } catch (...) {
        cudaGraph_t part = nullptr;
        cudaStreamEndCapture(s, &part);
        if (part) cudaGraphDestroy(part);
        throw;
    }
    BCK(cudaStreamEndCapture(s, &g.graph));
    const cudaError_t e = cudaGraphInstantiate(&g.exec, g.graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g.graph);
        BCK(e);
    }
    graphs_.push_back(g);
    BCK(cudaGraphLaunch(g.exec, s));
}

void Batch::check_error(cudaStream_t s) {
    int h = 0;
    BCK(cudaMemcpyAsync(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    if (h) {
        BCK(cudaMemsetAsync(d_err_, 0, sizeof(int), s));
        BCK(cudaStreamSynchronize(s));
        throw std::runtime_error("CUDA error: a tensor-core GEMM block timed out waiting on its pipeline");
    }
}

}  // namespace ddfmm
