// Many independent FMM instances (sessions) evaluated together: the launch
// sequences of the sessions are merged step by step (Session::Step::key:
// same pass, width and step type) into multi-instance launches, so one
// matvec of every instance costs as many launches as the deepest single
// instance, and the whole sequence can be replayed as one CUDA graph.  A
// device mask selects which instances a run computes; the others are skipped
// inside the kernels, so one captured graph serves every subset.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "session.hpp"

namespace ddfmm {

class Batch {
public:
    // sessions: mixed-form (tcgen05) sessions of one device with the same
    // accuracy level; they must outlive the batch.
    explicit Batch(const std::vector<Session*>& sessions);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    int size() const { return (int)sessions_.size(); }
    Session* session(int i) const { return sessions_[i]; }
    // Device I/O arrays of instance i: complex64 densities and values in
    // point-id order (session(i)->npts() entries each).
    float2* den(int i) const;
    float2* val(int i) const;
    // One matvec of every instance i with active[i] != 0 (device array of
    // size() ints; nullptr = all), enqueued on s.
    void run(const int* active, cudaStream_t s);
    // The same through a CUDA graph, captured on first use for each `active`
    // array (a few are kept: one per mask array of the caller).  Graphs of
    // different mask arrays may run at once on different streams when their
    // active instances are disjoint.
    void run_graph(const int* active, cudaStream_t s);
    int launches() const { return (int)launches_.size(); }
    // Throws if a tensor-core GEMM block gave up waiting (the flag is reset);
    // synchronises s.
    void check_error(cudaStream_t s);

private:
    enum Kind { ZERO, GATHER, SCATTER, GEMM, PT, VFWD, VACC, VINV };
    struct Launch {
        Kind kind;
        void* subs;
        void* prefix;
        int nsub;
        long long total;
        int G;
        int tpi = 32;  // point interactions: threads per item
        void* order = nullptr;  // tcgen05 GEMM: tiles by operator across the sub-launches (launch_umma_cgemm)
        alignas(16) unsigned char one[256];  // host copy of the first sub-launch
    };
    template <class Sub, class Pre>
    void add(Kind kind, const std::vector<Sub>& subs, const std::vector<Pre>& counts, int G = 0);
    void* upload_bytes(const void* p, size_t bytes);

    std::vector<Session*> sessions_;
    std::vector<Launch> launches_;
    std::vector<void*> allocs_;
    int device_ = 0;
    int* d_err_ = nullptr;
    struct Graph {
        const int* active;
        cudaGraph_t graph;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs_;  // captured sequences by mask array
};

}  // namespace ddfmm
