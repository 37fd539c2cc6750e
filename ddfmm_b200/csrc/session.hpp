// One FMM instance resident on one GPU: tree, lists, operators and buffers
// built once (Wave3d::setup, src/wave3d_setup.cpp:21-97), then any number of
// matvecs (Wave3d::eval, src/wave3d_eval.cpp:299-415) with fresh densities.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <map>
#include <string>
#include <vector>

#include <memory>

#include "kernels.cuh"
#include "opcache.hpp"
#include "ops.hpp"
#include "tree.hpp"

namespace ddfmm {

struct SessionParams {
    TreeParams tree;
    int accu = 1;    // -wave3d_ACCU: P = 4/6/8 (src/wave3d.cpp:145-158)
    int kernel = 0;  // KERNEL_HELM / KERNEL_EXPR
    int device = 0;
    int precision = 0;  // PRECISION_FP64 (plain) / PRECISION_MIXED / PRECISION_MIXED_MMA_SYNC
};

struct SessionStats {
    int n_points = 0, n_boxes = 0, n_leaves = 0, n_lf_boxes = 0;
    long long u_pairs = 0, u_interactions = 0, v_pairs = 0, w_pairs = 0, x_pairs = 0;
    long long hf_up_nodes = 0, hf_down_nodes = 0, hf_far_pairs = 0;
    long long m2l_matrices = 0, gemm_launches = 0, kernel_launches = 0;
    double flops_gemm = 0;        // 8 real flops per complex multiply-add
    long long fft_spectra_bytes = 0;
    double setup_seconds = 0;
    size_t device_bytes = 0;
    double ops_seconds = 0, tree_seconds = 0, plan_seconds = 0, tune_seconds = 0;  // parts of setup_seconds
    int tuned_steps = 0;  // steps whose launch shape the autotuner chose
};

class Session {
public:
    Session(const double* pos3n, int n, const SessionParams& p, const std::string& ld_path,
            const std::string& hd_path);
    ~Session();
    Session(const Session&) = delete;
    Session& operator=(const Session&) = delete;

    // val = G * den at every point; arrays in point-id order, complex128.
    void eval_host(const std::complex<double>* den, std::complex<double>* val);
    void eval_device(const double2* den, double2* val, cudaStream_t s);
    // complex64 densities / values (mixed form only)
    void eval_device_c64(const float2* den, float2* val, cudaStream_t s);
    void eval_host_c64(const std::complex<float>* den, std::complex<float>* val);
    bool mixed() const {
        return prm_.precision == PRECISION_MIXED || prm_.precision == PRECISION_MIXED_MMA_SYNC;
    }
    bool umma() const { return prm_.precision == PRECISION_MIXED; }
    // Throws if a tensor-core GEMM gave up waiting on its pipeline since the last
    // check (the flag is reset); synchronises the session's stream.
    void check_device_error();
    // Failure-path test hook (tcgen05 sessions): the next eval's first
    // tensor-core GEMM launch runs with its pipeline waits bounded by wait_s and
    // withholds the operator copies of its block 0, so that block's wait runs
    // out and the session reports the timeout at its next synchronous call.
    void arm_gemm_stall(double wait_s);
    // Same matvec with the V-list spectra in caller-provided scratch of
    // `capacity` double2 (must hold spectra_elems()); nothing is allocated.
    void eval_device_scratch(const double2* den, double2* val, cudaStream_t s, double2* spec, size_t capacity);
    size_t spectra_elems() const { return spectra_elems_; }
    // FP64 direct sum at the given point ids (Wave3d::check, src/wave3d_check.cpp:22-100)
    void direct_host(const std::complex<double>* den, const int* ids, int nids, std::complex<double>* out);

    const SessionStats& stats() const { return stats_; }

    struct ProfileEntry {
        std::string label, kernel;
        int launches = 0;
        double ms = 0, flops = 0, bytes = 0;
    };
    // Event-timed per-step profile of subsequent evals (on their stream).
    void profile_enable(bool on);
    std::vector<ProfileEntry> profile_read();
    void profile_reset() { prof_.clear(); }
    int npts() const { return npts_; }
    int device() const { return prm_.device; }
    // device bytes of the packed-operator chunks this session created (part of
    // stats().device_bytes; other sessions may share them)
    size_t chunk_bytes() const { return chunk_bytes_; }
    cudaStream_t stream() const { return stream_; }

private:
    struct GemmLaunch {
        GemmProblem* probs = nullptr;
        GemmTile* tiles = nullptr;
        long long* xoff = nullptr;
        long long* yoff = nullptr;
        int ntiles = 0;
        const double2* X = nullptr;
        double2* Y = nullptr;
        int mode = 0;
    };
    struct PtLaunch {
        PtItem* items = nullptr;
        PtSrc* srcs = nullptr;
        int nitems = 0;
    };
    struct VLaunch {
        VlistLevel L;
        int* src_boxes = nullptr;  // forward transforms: the source boxes
        int nsrc = 0;
        VlistGroups grp{};         // sums by target parent
        int* trg = nullptr;        // inverse transforms: the target boxes (rows of tsp)
        int ntrg = 0;
        const double2* upeq = nullptr;
        double2* spec = nullptr;
        double2* tsp = nullptr;    // summed target spectra
        double2* dnchk = nullptr;
    };
    struct Memset {
        void* p;
        size_t bytes;
    };
    // one step of the eval: exactly one of these is used
    struct Step {
        int kind;  // 0 gemm, 1 pt, 2 vfwd, 3 V-list sums, 4 memset, 5 tcgen05 gemm, 6 V-list inverse
        const char* label;  // pass name for profiling
        double flops;       // algorithmic flops of the launch
        double bytes;       // algorithmic DRAM bytes of the launch
        GemmLaunch g;
        PtLaunch pt;
        VLaunch v;
        Memset ms;
        // Position of the step in the pass structure, equal across sessions for steps
        // that play the same part (phase, width, step type, occurrence): a Batch
        // merges the steps of its sessions that share a key into one launch.
        long long key;
        int tpi;  // point interactions: launch shape (launch_pt; 0 = 32 threads per item), set by autotune()
        // mixed form: the step as a one-instance launch (device sub-launch array and
        // prefix sums) and the host copy of its sub-launch
        void* msubs;
        int* mpre;
        int mtotal;
        UmmaSub hu;
        std::vector<const float*> uop;  // tcgen05 GEMM: each tile's packed operator block (batch tile order)
        PtSub hp;
        VfSub hvf;
        VaSub hva;
        ViSub hvi;
    };
    friend class Batch;

    template <class T>
    T* dalloc(size_t count);
    // Copies a host array to the device and returns its device address.
    // Arrays above kArenaMax bytes get their own allocation and a completed
    // copy (the caller's vector may die right after).  Arrays up to kArenaMax
    // bytes -- most of the plan's many small tables -- are copied into the
    // host image of a device chunk (1 MiB doubling to 64 MiB); flush_uploads()
    // sends what is new in the image with one copy, and must run before any
    // device work reads those arrays.  Images stay alive until the plan's
    // last stream sync, as an asynchronous copy may still be reading them.
    template <class T>
    T* upload_n(const T* p, size_t n);
    template <class T, class A>
    T* upload(const std::vector<T, A>& v) {
        return upload_n(v.data(), v.size());
    }
    void flush_uploads();
    void dfree(const void* p);  // release one allocation made by dalloc / a large upload
    void add_gemm(std::vector<GemmProblem>& probs, std::vector<std::vector<long long> >& xo,
                  std::vector<std::vector<long long> >& yo, const double2* X, double2* Y, int mode,
                  const char* label);
    const float* packed_operator(const GemmProblem& q);
    void add_umma(const std::vector<GemmProblem>& P, const long long* xs, const long long* ys, size_t ncols,
                  const double2* X, double2* Y, int mode, Step& st);
    void flush_packs();
    void add_pt(const std::vector<PtItem>& items, const std::vector<PtSrc>& srcs, const char* label);
    template <class Sub>
    void set_multi(Step& st, const Sub& sub, int total);
    void begin_block(int phase, double W);
    void push_step(Step st);
    void build();
    // Times the launch-shape variants of each step on this session's own data
    // and keeps the fastest (point interactions: threads per item).
    void autotune();
    void run_steps(cudaStream_t s);
    void run_steps_spec(cudaStream_t s, double2* spec);
    void launch_step(const Step& st, cudaStream_t s, double2* spec);

    SessionParams prm_;
    int npts_ = 0;
    std::vector<double> pos_;
    Tree tree_;
    std::shared_ptr<const OperatorLib> ops_;  // shared with sessions of the same files
    std::vector<void*> allocs_;
    std::map<const void*, size_t> alloc_bytes_;
    static constexpr size_t kArenaMax = 64 << 10;
    struct UploadArena {
        char* dev = nullptr;     // current device chunk
        std::vector<char> host;  // its host image
        std::vector<std::vector<char> > retired;  // images of earlier chunks, kept until the plan's last sync
        size_t cap = 0, used = 0, sent = 0;
    } arena_;
    // Host-to-device copies of the plan go through two pinned staging buffers
    // (a pageable copy's speed varies several-fold between hosts): the source is
    // copied into a free buffer, which the device then reads asynchronously, so
    // the source may be released as soon as stage_copy returns.
    static constexpr size_t kStage = 8 << 20;
    // Arrays above kArenaMax and up to kMidMax bytes (most of them operators of a
    // wedge) are placed in device chunks of 4 MiB doubling to 64 MiB, staged
    // straight to the device: a few allocations instead of one cudaMalloc each.  Like the small arena's
    // chunks they are released with the session, never by dfree().
    static constexpr size_t kMidMax = 4 << 20, kMidChunk = 64 << 20;
    char* mid_dev_ = nullptr;
    size_t mid_used_ = 0, mid_cap_ = 0;
    char* stage_[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev_[2] = {nullptr, nullptr};
    int stage_next_ = 0;
    void stage_copy(void* dst, const void* src, size_t bytes);
    void stage_release();  // after a stream sync
    std::vector<Step> steps_;
    cudaStream_t stream_ = nullptr;
    SessionStats stats_;

    // device state
    int* d_perm_ = nullptr;
    double* d_pos_ids_ = nullptr;
    double* d_pos_sorted_ = nullptr;
    double2* d_den_sorted_ = nullptr;
    double2* d_val_sorted_ = nullptr;
    double2* d_den_io_ = nullptr;
    double2* d_val_io_ = nullptr;
    std::vector<Memset> zero_at_start_;
    int* d_err_ = nullptr;  // set by a tensor-core GEMM that timed out
    unsigned long long stall_wait_ns_ = 0;  // armed failure-path hook (0: none)
    std::map<std::pair<const void*, long long>, const float*> packed_;  // (operator, m k) -> packed copy
    std::vector<UmmaPackJob> pack_jobs_;
    // setup trace: host seconds in add_gemm, vlist_groups, uploads above kArenaMax,
    // packed_operator, and of that in packed-operator chunk allocations
    double t_emit_gemm_ = 0, t_emit_vgroups_ = 0, t_big_uploads_ = 0, t_pack_ = 0, t_pack_alloc_ = 0;
    // and in device allocations, staging-buffer waits and copies into the staging buffers
    double t_malloc_ = 0, t_stage_wait_ = 0, t_stage_copy_ = 0;
    long long n_malloc_ = 0, n_stage_ = 0;                                 // packing still to launch
    // packed operators (tcgen05 form): the chunk being filled, the operators this
    // session uses (its own and shared ones), and those it created but has not yet
    // published to the process-wide cache (they are, once their packing completed)
    std::string ld_path_, hd_path_, opctx_;
    std::shared_ptr<DevChunk> chunk_;
    float* chunk_pos_ = nullptr;
    size_t chunk_left_ = 0;   // floats
    size_t chunk_bytes_ = 0;  // bytes of the chunks this session created
    std::vector<std::shared_ptr<PackedOp> > held_;
    std::map<const void*, std::string> opkey_;  // operator (FP32 copy) -> cache key
    std::vector<std::pair<std::string, std::shared_ptr<PackedOp> > > to_publish_;
    const float* cached_op(const std::string& key);
    size_t spectra_elems_ = 0;
    bool profiling_ = false;
    std::vector<cudaEvent_t> ev_;
    std::vector<std::pair<int, int> > ev_pending_;  // (step, event index) recorded, not yet read
    std::map<std::string, ProfileEntry> prof_;
    std::vector<std::string> label_store_;  // per-width pass labels (Step::label points here)
    int cur_phase_ = 0;
    long long cur_wkey_ = 0;
    std::map<std::string, int> block_counts_;  // occurrences of each step type in the current block
    const char* width_label(const char* pass, double W);
};

}  // namespace ddfmm
