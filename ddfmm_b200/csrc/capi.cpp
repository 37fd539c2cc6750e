// extern "C" entry points (include/ddfmm.h).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/ddfmm.h"
#include "batch.hpp"
#include "precompute.hpp"
#include "server.hpp"
#include "session.hpp"

struct ddfmm_session {
    ddfmm::Session* impl;
};

struct ddfmm_server {
    ddfmm::Server* impl;
};

struct ddfmm_batch {
    ddfmm::Batch* impl = nullptr;
    int* d_active = nullptr;  // device mask of the sessions a call computes
    int* h_active = nullptr;  // pinned host copy
    cudaEvent_t copied = nullptr;  // the last mask copy has left h_active
    cudaStream_t stream = nullptr;
    int device = 0;
};

namespace ddfmm {
double2* noalloc_scratch(size_t* capacity);  // noalloc.cu
}

namespace {
thread_local std::string g_err;

#define CKA(x)                                                                                     \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" + \
                                     #x + ")");                                                    \
    } while (0)

// makes `device` current for a scope and restores the caller's device after
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        CKA(cudaSetDevice(device));
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return DDFMM_OK;
    } catch (const std::bad_alloc&) {
        return fail(DDFMM_ENOMEM, "host out of memory");
    } catch (const std::invalid_argument& e) {
        return fail(DDFMM_EINVAL, e.what());
    } catch (const std::runtime_error& e) {
        std::string m = e.what();
        if (m.rfind("CUDA error", 0) == 0) {
            if (m.find("out of memory") != std::string::npos) return fail(DDFMM_ENOMEM, m);
            return fail(DDFMM_ECUDA, m);
        }
        return fail(DDFMM_ESETUP, m);
    } catch (const std::exception& e) {
        return fail(DDFMM_ESETUP, e.what());
    }
}
}  // namespace

extern "C" {

const char* ddfmm_last_error(void) { return g_err.c_str(); }

int ddfmm_session_create(const double* pos3n, int n, int kernel, int accu, int npq, double K, const double* ctr3,
                         int ptsmax, int maxlevel, int ncell, const char* ld_path, const char* hd_path, int device,
                         ddfmm_session** out) {
    return ddfmm_session_create_ex(pos3n, n, kernel, accu, npq, K, ctr3, ptsmax, maxlevel, ncell, ld_path, hd_path,
                                   device, DDFMM_PLAIN_FP64, out);
}

}  // extern "C"

// Validation shared by session creation and server admission (the reference's
// option checks, src/wave3d.cpp:145-158 and src/wave3d_setup.cpp:21-97).
static int make_params(const double* pos3n, int n, int kernel, int accu, int npq, double K, const double* ctr3,
                       int ptsmax, int maxlevel, int ncell, const char* ld_path, const char* hd_path, int device,
                       int precision, ddfmm::SessionParams* out) {
    if (!pos3n || n <= 0) return fail(DDFMM_EINVAL, "need n > 0 points");
    if (kernel != DDFMM_KERNEL_HELM && kernel != DDFMM_KERNEL_EXPR) return fail(DDFMM_EINVAL, "unknown kernel type");
    if (accu < 1 || accu > 3) return fail(DDFMM_EINVAL, "ACCU must be 1, 2 or 3");
    if (npq <= 0 || npq % 2) return fail(DDFMM_EINVAL, "NPQ must be a positive even number");
    if (!(K >= 1) || !std::isfinite(K)) return fail(DDFMM_EINVAL, "K must be >= 1");
    if (ncell < 1 || (ncell & (ncell - 1)) || K / ncell < 1 - 1e-12)
        return fail(DDFMM_EINVAL, "ncell must be a power of two with K/ncell >= 1");
    if (ptsmax < 1 || maxlevel < 1) return fail(DDFMM_EINVAL, "ptsmax and maxlevel must be positive");
    if (precision != DDFMM_PLAIN_FP64 && precision != DDFMM_MIXED && precision != DDFMM_MIXED_MMA_SYNC)
        return fail(DDFMM_EINVAL, "precision must be DDFMM_PLAIN_FP64, DDFMM_MIXED or DDFMM_MIXED_MMA_SYNC");
    if (!ld_path || !hd_path) return fail(DDFMM_EINVAL, "operator file paths are required");
    for (long long i = 0; i < 3LL * n; ++i)
        if (!std::isfinite(pos3n[i])) return fail(DDFMM_EINVAL, "non-finite point coordinate");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(DDFMM_ECUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(DDFMM_EINVAL, "device ordinal out of range");
    ddfmm::SessionParams& p = *out;
    p.tree.K = K;
    p.tree.ctr = {{ctr3 ? ctr3[0] : 0.0, ctr3 ? ctr3[1] : 0.0, ctr3 ? ctr3[2] : 0.0}};
    p.tree.ptsmax = ptsmax;
    p.tree.maxlevel = maxlevel;
    p.tree.npq = npq;
    p.tree.ncell = ncell;
    p.accu = accu;
    p.kernel = kernel;
    p.device = device;
    p.precision = precision;
    return DDFMM_OK;
}

extern "C" {

int ddfmm_session_create_ex(const double* pos3n, int n, int kernel, int accu, int npq, double K, const double* ctr3,
                            int ptsmax, int maxlevel, int ncell, const char* ld_path, const char* hd_path, int device,
                            int precision, ddfmm_session** out) {
    if (!out) return fail(DDFMM_EINVAL, "out is NULL");
    *out = nullptr;
    ddfmm::SessionParams p;
    int rc = make_params(pos3n, n, kernel, accu, npq, K, ctr3, ptsmax, maxlevel, ncell, ld_path, hd_path, device,
                         precision, &p);
    if (rc != DDFMM_OK) return rc;
    ddfmm::Session* impl = nullptr;
    rc = guarded([&] { impl = new ddfmm::Session(pos3n, n, p, ld_path, hd_path); });
    if (rc != DDFMM_OK) return rc;
    *out = new ddfmm_session{impl};
    return DDFMM_OK;
}

int ddfmm_eval(ddfmm_session* s, const double* den, double* val) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    if (!den || !val) return fail(DDFMM_EINVAL, "NULL density or value array");
    return guarded([&] {
        s->impl->eval_host(reinterpret_cast<const std::complex<double>*>(den),
                           reinterpret_cast<std::complex<double>*>(val));
    });
}

int ddfmm_eval_device(ddfmm_session* s, const void* den_dev, void* val_dev, void* stream) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    if (!den_dev || !val_dev) return fail(DDFMM_EINVAL, "NULL device array");
    return guarded([&] {
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->impl->stream();
        s->impl->eval_device(static_cast<const double2*>(den_dev), static_cast<double2*>(val_dev), st);
    });
}

int ddfmm_eval_c64(ddfmm_session* s, const float* den, float* val) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    if (!den || !val) return fail(DDFMM_EINVAL, "NULL density or value array");
    return guarded([&] {
        s->impl->eval_host_c64(reinterpret_cast<const std::complex<float>*>(den),
                               reinterpret_cast<std::complex<float>*>(val));
    });
}

int ddfmm_eval_device_c64(ddfmm_session* s, const void* den_dev, void* val_dev, void* stream) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    if (!den_dev || !val_dev) return fail(DDFMM_EINVAL, "NULL device array");
    return guarded([&] {
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->impl->stream();
        s->impl->eval_device_c64(static_cast<const float2*>(den_dev), static_cast<float2*>(val_dev), st);
    });
}

int ddfmm_eval_device_noalloc(ddfmm_session* s, const void* den_dev, void* val_dev, void* stream) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    if (!den_dev || !val_dev) return fail(DDFMM_EINVAL, "NULL device array");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return fail(DDFMM_ECUDA, "cudaGetDevice failed");
    int rc = guarded([&] {
        // the scratch address is per device: resolve it on the session's GPU
        if (cudaSetDevice(s->impl->device()) != cudaSuccess) throw std::runtime_error("CUDA error: cudaSetDevice");
        size_t cap = 0;
        double2* spec = ddfmm::noalloc_scratch(&cap);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->impl->stream();
        s->impl->eval_device_scratch(static_cast<const double2*>(den_dev), static_cast<double2*>(val_dev), st, spec,
                                     cap);
    });
    cudaSetDevice(prev);
    return rc;
}

int ddfmm_direct(ddfmm_session* s, const double* den, const int* ids, int nids, double* out) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    if (!den || (nids > 0 && (!ids || !out)) || nids < 0) return fail(DDFMM_EINVAL, "bad direct-sum arguments");
    return guarded([&] {
        s->impl->direct_host(reinterpret_cast<const std::complex<double>*>(den), ids, nids,
                             reinterpret_cast<std::complex<double>*>(out));
    });
}

int ddfmm_session_stats(const ddfmm_session* s, ddfmm_stats* out) {
    if (!s || !s->impl || !out) return fail(DDFMM_EINVAL, "NULL argument");
    const ddfmm::SessionStats& t = s->impl->stats();
    out->n_points = t.n_points;
    out->n_boxes = t.n_boxes;
    out->n_leaves = t.n_leaves;
    out->n_lf_boxes = t.n_lf_boxes;
    out->u_pairs = t.u_pairs;
    out->u_interactions = t.u_interactions;
    out->v_pairs = t.v_pairs;
    out->w_pairs = t.w_pairs;
    out->x_pairs = t.x_pairs;
    out->hf_up_nodes = t.hf_up_nodes;
    out->hf_down_nodes = t.hf_down_nodes;
    out->hf_far_pairs = t.hf_far_pairs;
    out->m2l_matrices = t.m2l_matrices;
    out->gemm_launches = t.gemm_launches;
    out->kernel_launches = t.kernel_launches;
    out->flops_gemm = t.flops_gemm;
    out->fft_spectra_bytes = t.fft_spectra_bytes;
    out->setup_seconds = t.setup_seconds;
    out->ops_seconds = t.ops_seconds;
    out->tree_seconds = t.tree_seconds;
    out->plan_seconds = t.plan_seconds;
    out->tune_seconds = t.tune_seconds;
    out->device_bytes = (long long)t.device_bytes;
    return DDFMM_OK;
}

int ddfmm_operators_check(const char* ld_path, const char* hd_path, int accu, int* n_ld_widths, int* n_hd_wedges) {
    if (!ld_path || !hd_path) return fail(DDFMM_EINVAL, "operator file paths are required");
    if (accu < 1 || accu > 3) return fail(DDFMM_EINVAL, "ACCU must be 1, 2 or 3");
    return guarded([&] {
        ddfmm::OperatorLib ops;
        ops.load(ld_path, hd_path);
        ops.validate(accu);
        if (n_ld_widths) *n_ld_widths = (int)ops.ld.size();
        if (n_hd_wedges) {
            long long n = 0;
            for (const auto& kv : ops.hd) n += (long long)kv.second.size();
            *n_hd_wedges = (int)n;
        }
    });
}

int ddfmm_precompute_operators(int kernel, int accu, int wmax, int threads, const char* ld_path, const char* hd_path,
                               int verbose) {
    if (kernel != 0 && kernel != 1) return fail(DDFMM_EINVAL, "kernel must be 0 (exp(ir)/r) or 1 (exp(ir))");
    if (accu < 1 || accu > 3) return fail(DDFMM_EINVAL, "ACCU must be 1, 2 or 3");
    if (wmax < 1 || wmax > 1024 || (wmax & (wmax - 1))) return fail(DDFMM_EINVAL, "wmax must be a power of two >= 1");
    if (!ld_path && !hd_path) return fail(DDFMM_EINVAL, "no output file given");
    // arguments are checked above: every failure below is a precompute failure
    return guarded([&] {
        try {
            if (ld_path) {
                auto t0 = std::chrono::steady_clock::now();
                ddfmm::precompute::write_ld(ld_path, ddfmm::precompute::low_levels(accu, kernel, threads));
                if (verbose)
                    std::fprintf(stderr, "precompute: low frequency written in %.1f s\n",
                                 std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
            }
            if (hd_path) {
                auto t0 = std::chrono::steady_clock::now();
                auto progress = [&](double W, int done, int total) {
                    if (verbose && done == total)
                        std::fprintf(stderr, "precompute: width %g, %d wedges, %.1f s\n", W, total,
                                     std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
                };
                ddfmm::precompute::write_hd(hd_path,
                                            ddfmm::precompute::high_levels(accu, kernel, wmax, threads, progress));
            }
        } catch (const std::bad_alloc&) {
            throw;
        } catch (const std::exception& e) {
            throw std::runtime_error(std::string("operator precompute failed: ") + e.what());
        }
    });
}

int ddfmm_session_test_gemm_stall(ddfmm_session* s, double wait_s) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    return guarded([&] { s->impl->arm_gemm_stall(wait_s); });
}

int ddfmm_tree_stats(const double* pos3n, int n, double K, const double* ctr3, int ptsmax, int maxlevel, int ncell,
                     int npq, int* total_boxes, int* empty_boxes, int* nlevels, ddfmm_tree_level* levels) {
    if (!pos3n || n <= 0 || !total_boxes || !empty_boxes || !nlevels || !levels)
        return fail(DDFMM_EINVAL, "bad tree-stats arguments");
    if (ncell < 1 || (ncell & (ncell - 1)) || K / ncell < 1 - 1e-12)
        return fail(DDFMM_EINVAL, "ncell must be a power of two with K/ncell >= 1");
    return guarded([&] {
        ddfmm::TreeParams p;
        p.K = K;
        p.ctr = {{ctr3 ? ctr3[0] : 0.0, ctr3 ? ctr3[1] : 0.0, ctr3 ? ctr3[2] : 0.0}};
        p.ptsmax = ptsmax;
        p.maxlevel = maxlevel;
        p.ncell = ncell;
        p.npq = npq;
        ddfmm::Tree t;
        t.build(pos3n, n, p);
        std::map<int, ddfmm_tree_level> lv;
        int empty = 0;
        for (const ddfmm::Box& b : t.boxes) {
            if (!b.has_pts()) {
                ++empty;
                continue;
            }
            ddfmm_tree_level& L = lv[b.level];
            L.level = b.level;
            L.width = t.width(b.level);
            L.boxes++;
            if (b.terminal()) L.leaves++;
            for (auto& kv : b.far) L.far_pairs += (long long)kv.second.size();
            L.out_dirs += (long long)b.outdirs.size();
            L.inc_dirs += (long long)b.incdirs.size();
            L.u_pairs += (long long)b.ulist.size();
            L.v_pairs += (long long)b.vlist.size();
            L.w_pairs += (long long)b.wlist.size();
            L.x_pairs += (long long)b.xlist.size();
        }
        if (lv.size() > 64) throw std::runtime_error("more than 64 levels");
        int i = 0;
        for (auto& kv : lv) levels[i++] = kv.second;
        *nlevels = i;
        *total_boxes = (int)t.boxes.size();
        *empty_boxes = empty;
    });
}

int ddfmm_profile_enable(ddfmm_session* s, int on) {
    if (!s || !s->impl) return fail(DDFMM_EINVAL, "NULL session");
    return guarded([&] { s->impl->profile_enable(on != 0); });
}

int ddfmm_profile_read(ddfmm_session* s, ddfmm_profile_entry* out, int max_entries, int* n_entries, int reset) {
    if (!s || !s->impl || !n_entries || (max_entries > 0 && !out)) return fail(DDFMM_EINVAL, "bad profile arguments");
    return guarded([&] {
        auto v = s->impl->profile_read();
        int n = 0;
        for (auto& e : v) {
            if (n >= max_entries) break;
            ddfmm_profile_entry& o = out[n++];
            std::memset(&o, 0, sizeof(o));
            std::strncpy(o.label, e.label.c_str(), sizeof(o.label) - 1);
            std::strncpy(o.kernel, e.kernel.c_str(), sizeof(o.kernel) - 1);
            o.launches = e.launches;
            o.ms = e.ms;
            o.flops = e.flops;
            o.bytes = e.bytes;
        }
        *n_entries = n;
        if (reset) s->impl->profile_reset();
    });
}

int ddfmm_session_destroy(ddfmm_session* s) {
    if (!s) return DDFMM_OK;
    int rc = guarded([&] { delete s->impl; });
    delete s;
    return rc;
}

static void batch_free(ddfmm_batch* b) {
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b->impl;
    if (b->d_active) cudaFree(b->d_active);
    if (b->h_active) cudaFreeHost(b->h_active);
    if (b->copied) cudaEventDestroy(b->copied);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int ddfmm_batch_create(ddfmm_session* const* sessions, int n, ddfmm_batch** out) {
    if (!out) return fail(DDFMM_EINVAL, "out is NULL");
    *out = nullptr;
    if (!sessions || n <= 0) return fail(DDFMM_EINVAL, "need at least one session");
    std::vector<ddfmm::Session*> v;
    for (int i = 0; i < n; ++i) {
        if (!sessions[i]) return fail(DDFMM_EINVAL, "session is NULL");
        v.push_back(sessions[i]->impl);
    }
    ddfmm_batch* b = new (std::nothrow) ddfmm_batch();
    if (!b) return fail(DDFMM_ENOMEM, "host out of memory");
    int rc = guarded([&] {
        b->device = v[0]->device();
        DeviceGuard dg(b->device);
        b->impl = new ddfmm::Batch(v);
        CKA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        CKA(cudaMalloc(&b->d_active, sizeof(int) * n));
        CKA(cudaMallocHost(&b->h_active, sizeof(int) * n));
        CKA(cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming));
        CKA(cudaEventRecord(b->copied, b->stream));
    });
    if (rc != DDFMM_OK) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return DDFMM_OK;
}

// mask from the non-NULL inputs, copied to the device on st; then the graph
static void batch_launch(ddfmm_batch* b, const void* const* den, cudaStream_t st) {
    const int n = b->impl->size();
    CKA(cudaEventSynchronize(b->copied));
    for (int i = 0; i < n; ++i) b->h_active[i] = den[i] != nullptr;
    CKA(cudaMemcpyAsync(b->d_active, b->h_active, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    CKA(cudaEventRecord(b->copied, st));
    b->impl->run_graph(b->d_active, st);
}

int ddfmm_batch_eval_c64(ddfmm_batch* b, const float* const* den, float* const* val) {
    if (!b || !den || !val) return fail(DDFMM_EINVAL, "NULL argument");
    return guarded([&] {
        DeviceGuard dg(b->device);
        const int n = b->impl->size();
        for (int i = 0; i < n; ++i) {
            if (den[i] && !val[i]) throw std::invalid_argument("val[i] is NULL for a computed session");
            if (den[i])
                CKA(cudaMemcpyAsync(b->impl->den(i), den[i], sizeof(float2) * b->impl->session(i)->npts(),
                                    cudaMemcpyHostToDevice, b->stream));
        }
        batch_launch(b, reinterpret_cast<const void* const*>(den), b->stream);
        for (int i = 0; i < n; ++i)
            if (den[i])
                CKA(cudaMemcpyAsync(val[i], b->impl->val(i), sizeof(float2) * b->impl->session(i)->npts(),
                                    cudaMemcpyDeviceToHost, b->stream));
        b->impl->check_error(b->stream);
    });
}

int ddfmm_batch_eval_device_c64(ddfmm_batch* b, const void* const* den_dev, void* const* val_dev, void* stream) {
    if (!b || !den_dev || !val_dev) return fail(DDFMM_EINVAL, "NULL argument");
    return guarded([&] {
        DeviceGuard dg(b->device);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
        const int n = b->impl->size();
        for (int i = 0; i < n; ++i) {
            if (den_dev[i] && !val_dev[i]) throw std::invalid_argument("val_dev[i] is NULL for a computed session");
            if (den_dev[i])
                CKA(cudaMemcpyAsync(b->impl->den(i), den_dev[i], sizeof(float2) * b->impl->session(i)->npts(),
                                    cudaMemcpyDeviceToDevice, st));
        }
        batch_launch(b, den_dev, st);
        for (int i = 0; i < n; ++i)
            if (den_dev[i])
                CKA(cudaMemcpyAsync(val_dev[i], b->impl->val(i), sizeof(float2) * b->impl->session(i)->npts(),
                                    cudaMemcpyDeviceToDevice, st));
        CKA(cudaGetLastError());
    });
}

int ddfmm_batch_launches(ddfmm_batch* b, int* launches) {
    if (!b || !launches) return fail(DDFMM_EINVAL, "NULL argument");
    *launches = b->impl->launches();
    return DDFMM_OK;
}

int ddfmm_batch_destroy(ddfmm_batch* b) {
    if (!b) return DDFMM_OK;
    return guarded([&] { batch_free(b); });
}

int ddfmm_server_create(int device, double budget_bytes, ddfmm_server** out) {
    if (!out) return fail(DDFMM_EINVAL, "out is NULL");
    *out = nullptr;
    if (!(budget_bytes > 0)) return fail(DDFMM_EINVAL, "the device-memory budget must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(DDFMM_ECUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(DDFMM_EINVAL, "device ordinal out of range");
    ddfmm::Server* impl = nullptr;
    int rc = guarded([&] {
        DeviceGuard dg(device);
        impl = new ddfmm::Server(device, (size_t)budget_bytes);
    });
    if (rc != DDFMM_OK) return rc;
    *out = new ddfmm_server{impl};
    return DDFMM_OK;
}

int ddfmm_server_add_session(ddfmm_server* sv, const double* pos3n, int n, int kernel, int accu, int npq, double K,
                             const double* ctr3, int ptsmax, int maxlevel, int ncell, const char* ld_path,
                             const char* hd_path, int* sid) {
    if (!sv || !sid) return fail(DDFMM_EINVAL, "NULL argument");
    ddfmm::SessionParams p;
    int dev = 0;
    cudaGetDevice(&dev);
    int rc = make_params(pos3n, n, kernel, accu, npq, K, ctr3, ptsmax, maxlevel, ncell, ld_path, hd_path, dev,
                         DDFMM_MIXED, &p);
    if (rc != DDFMM_OK) return rc;
    return guarded([&] {
        ddfmm::SessionSpec spec;
        spec.pos.assign(pos3n, pos3n + 3 * (size_t)n);
        spec.n = n;
        spec.params = p;
        spec.ld = ld_path;
        spec.hd = hd_path;
        *sid = sv->impl->add_session(std::move(spec));
    });
}

int ddfmm_server_session_state(ddfmm_server* sv, int sid, int* state) {
    if (!sv || !state) return fail(DDFMM_EINVAL, "NULL argument");
    std::string why;
    const int st = sv->impl->state(sid, &why);
    if (st < 0) return fail(DDFMM_EINVAL, "unknown session");
    *state = st;
    if (!why.empty()) g_err = why;
    return DDFMM_OK;
}

int ddfmm_server_remove_session(ddfmm_server* sv, int sid) {
    if (!sv) return fail(DDFMM_EINVAL, "NULL server");
    return guarded([&] { sv->impl->remove_session(sid); });
}

int ddfmm_server_submit(ddfmm_server* sv, int sid, const float* den, float* val, long long* ticket) {
    if (!sv || !den || !val || !ticket) return fail(DDFMM_EINVAL, "NULL argument");
    return guarded([&] {
        *ticket = sv->impl->submit(sid, reinterpret_cast<const std::complex<float>*>(den),
                                   reinterpret_cast<std::complex<float>*>(val));
    });
}

int ddfmm_server_wait(ddfmm_server* sv, long long ticket, double timeout_s, int* done) {
    if (!sv || !done) return fail(DDFMM_EINVAL, "NULL argument");
    return guarded([&] { *done = sv->impl->wait(ticket, timeout_s) == 0; });
}

int ddfmm_server_poll(ddfmm_server* sv, long long ticket, int* done) {
    if (!sv || !done) return fail(DDFMM_EINVAL, "NULL argument");
    const int r = sv->impl->poll(ticket);
    if (r < 0) return fail(DDFMM_ECUDA, "request failed (ddfmm_server_wait gives the reason)");
    *done = r == 0;
    return DDFMM_OK;
}

int ddfmm_server_get_stats(ddfmm_server* sv, ddfmm_server_stats* out, int reset) {
    if (!sv || !out) return fail(DDFMM_EINVAL, "NULL argument");
    return guarded([&] {
        const ddfmm::ServerStats s = sv->impl->stats(reset != 0);
        out->requests = s.requests;
        out->ticks = s.ticks;
        out->mean_batch = s.mean_batch;
        out->p50_ms = s.p50_ms;
        out->p99_ms = s.p99_ms;
        out->max_ms = s.max_ms;
        out->busy_s = s.busy_s;
        out->used_bytes = (long long)s.used_bytes;
        out->admitted = s.admitted;
        out->waiting = s.waiting;
    });
}

int ddfmm_server_destroy(ddfmm_server* sv) {
    if (!sv) return DDFMM_OK;
    int rc = guarded([&] { delete sv->impl; });
    delete sv;
    return rc;
}

}  // extern "C"
