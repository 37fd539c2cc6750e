/* C ABI of the B200 directional FMM matvec (drop-in for Wave3d::eval).
 *
 * The reference's interface for this path is the C++ class Wave3d
 * (include/wave3d.hpp:219-265 of arbenson/ddfmm):
 *   wave.posptr() = &pos; wave.kernel() = k; wave.mlibptr() = &mlib;
 *   wave.geomprtn() = geomprtn;            (src/tt.cpp:134-138)
 *   wave.setup(opts);                      (src/wave3d_setup.cpp:21-97)
 *   wave.eval(den, val);                   (src/wave3d_eval.cpp:299-415)
 *   wave.check(den, val, chk, relerr);     (src/wave3d_check.cpp:22-100)
 * with Mlib3d::setup reading the ld/hd operator files
 * (src/mlib3d.cpp:70-103).  Each entry point below replaces one of those
 * calls; the reference's ParVec<int,...> maps become dense arrays indexed by
 * point id 0..n-1 (the map's key order).  Complex values are interleaved
 * (re, im) doubles, i.e. std::complex<double> / cpx.
 *
 * All functions return DDFMM_OK (0) or a nonzero status; the reference
 * throws `new std::exception()` in the same situations
 * (include/commoninc.hpp:52-53).  ddfmm_last_error() describes the last
 * failure of the calling thread.  The library owns all device memory; the
 * caller owns every host array.  A session is used by one host thread at a
 * time (the reference keeps one active Wave3d per process,
 * src/wave3d.cpp:21). */
#ifndef DDFMM_B200_H
#define DDFMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    DDFMM_OK = 0,
    DDFMM_EINVAL = 1,   /* bad argument (reference: CHECK_TRUE failure) */
    DDFMM_ECUDA = 2,    /* CUDA runtime error or no usable GPU */
    DDFMM_ESETUP = 3,   /* tree / operator inconsistency, unreadable operator file */
    DDFMM_ENOMEM = 4
};

enum { DDFMM_KERNEL_HELM = 0, DDFMM_KERNEL_EXPR = 1 }; /* include/kernel3d.hpp:24-27 */

/* Arithmetic of a session.  PLAIN_FP64: every pass in FP64 (the form that
 * matches the reference to 1e-10).  MIXED: operators still built in FP64,
 * then stored and applied in complex FP32 -- translations as 3xTF32 products
 * on the tensor cores (tcgen05, accumulators in tensor memory) with FP32
 * accumulation, the near field in FP32 on FP64 coordinate differences.  Error
 * vs the FP64 direct sum is then set by FP32 rounding (about 1e-6) on top of
 * the method's own (1e-4 / 1e-6 / 1e-8).  MIXED_MMA_SYNC: the same form with
 * the translations on the warp-level mma.sync path instead (for comparison). */
enum { DDFMM_PLAIN_FP64 = 0, DDFMM_MIXED = 1, DDFMM_MIXED_MMA_SYNC = 2 };

typedef struct ddfmm_session ddfmm_session;

typedef struct ddfmm_stats {
    int n_points, n_boxes, n_leaves, n_lf_boxes;
    long long u_pairs, u_interactions, v_pairs, w_pairs, x_pairs;
    long long hf_up_nodes, hf_down_nodes, hf_far_pairs, m2l_matrices;
    long long gemm_launches, kernel_launches;
    double flops_gemm;          /* 8 real flops per complex multiply-add */
    long long fft_spectra_bytes;
    double setup_seconds;
    long long device_bytes;
    /* setup_seconds split: operator files, octree and lists, plan and
     * operators on the device, launch-shape tuning */
    double ops_seconds, tree_seconds, plan_seconds, tune_seconds;
} ddfmm_stats;

/* Wave3d::setup + Mlib3d::setup.  pos3n: n points, x/y/z interleaved, in
 * wavelengths.  kernel: DDFMM_KERNEL_HELM (exp(ir)/r) or DDFMM_KERNEL_EXPR.
 * accu, npq, K, ctr, ptsmax, maxlevel: the -wave3d_* options.  ncell:
 * geomprtn.m(), the cells per edge of the partition tensor (power of two,
 * K/ncell >= 1).  ld_path / hd_path: operator files in the reference format
 * (-mlib3d_ldname / -mlib3d_hdname).  device: CUDA ordinal. */
int ddfmm_session_create(const double* pos3n, int n, int kernel, int accu, int npq, double K,
                         const double* ctr3, int ptsmax, int maxlevel, int ncell,
                         const char* ld_path, const char* hd_path, int device,
                         ddfmm_session** out);

/* ddfmm_session_create with the arithmetic chosen by `precision`
 * (DDFMM_PLAIN_FP64, DDFMM_MIXED or DDFMM_MIXED_MMA_SYNC). */
int ddfmm_session_create_ex(const double* pos3n, int n, int kernel, int accu, int npq, double K,
                            const double* ctr3, int ptsmax, int maxlevel, int ncell,
                            const char* ld_path, const char* hd_path, int device, int precision,
                            ddfmm_session** out);

/* Wave3d::eval: val[i] = sum_j G(p_i, p_j) den[j] via the directional FMM.
 * den, val: host arrays of n complex128 in point-id order.  Unlike the
 * reference, repeated calls do not accumulate (src/wave3d_eval.cpp:518-521). */
int ddfmm_eval(ddfmm_session* s, const double* den, double* val);

/* Mixed sessions only: complex64 densities and values (interleaved floats),
 * host arrays / device arrays of the session's GPU.  ddfmm_eval and
 * ddfmm_eval_device also work on mixed sessions (complex128 in and out). */
int ddfmm_eval_c64(ddfmm_session* s, const float* den, float* val);
int ddfmm_eval_device_c64(ddfmm_session* s, const void* den_dev, void* val_dev, void* stream);

/* Same, with den / val already in device memory of the session's GPU
 * (n complex128 each); stream is a cudaStream_t or NULL for the session's
 * own stream.  Returns after enqueueing; the caller synchronises. */
int ddfmm_eval_device(ddfmm_session* s, const void* den_dev, void* val_dev, void* stream);

/* No counterpart in the reference.  ddfmm_eval_device for callers that
 * cannot allocate device memory while they run: a solver embedded in a host
 * application whose own allocator owns all of the GPU's memory (cudaMalloc
 * there fails or is forbidden once the application has started), or a
 * real-time loop with a device-memory budget fixed up front, where an
 * allocation at the call would break the budget or stall on the driver.
 * The session's per-eval V-list spectra (one (2P)^3 complex FFT per
 * low-frequency box) go to one fixed, statically sized device array of
 * 16 MiB that every GPU loading this library holds until the process exits,
 * instead of session memory; nothing else changes and the call allocates
 * nothing.  Limits and rules:
 *  - sessions whose spectra exceed 16 MiB (about 2000 low-frequency boxes at
 *    ACCU 1, 600 at ACCU 2, 250 at ACCU 3) get DDFMM_EINVAL and a message;
 *  - every call resolves the array's device address (cudaGetSymbolAddress,
 *    which allocates nothing) on the current device, so the address is
 *    right after a cudaDeviceReset too;
 *  - every call and every session on a device share the one array: calls
 *    whose work overlaps on the GPU race.  stream == NULL means the session's
 *    own private stream, so two sessions both called with NULL overlap: with
 *    several sessions, pass one explicit shared stream, or synchronise between
 *    calls;
 *  - each call writes every spectrum it reads, so no zeroing is needed and a
 *    previous call's leftovers are never used.
 * den_dev / val_dev / stream as in ddfmm_eval_device. */
int ddfmm_eval_device_noalloc(ddfmm_session* s, const void* den_dev, void* val_dev, void* stream);

/* Wave3d::check's direct sum: out[k] = sum_j G(p_ids[k], p_j) den[j] in
 * FP64 over all points (self pair included, r:=1 when r < 1e-8). */
int ddfmm_direct(ddfmm_session* s, const double* den, const int* ids, int nids, double* out);

int ddfmm_session_stats(const ddfmm_session* s, ddfmm_stats* out);

/* Host-only (no GPU): Mlib3d::setup (src/mlib3d.cpp:70-103) without a
 * session -- read the ld / hd operator files and check every entry's shapes
 * against accuracy level accu (surfaces of P^3-(P-2)^3 points, uc2ue factor
 * shapes, ue2dc tensors of edge 2P, E1/E2/E3 against the skeleton counts,
 * ranks <= 400).  DDFMM_ESETUP for an unreadable, truncated, trailing-byte
 * or inconsistent file (the reference throws from deserialize or a CHECK
 * there); DDFMM_EINVAL for bad arguments.  Optional outputs: the number of
 * low-frequency widths and of (width, canonical wedge) entries. */
int ddfmm_operators_check(const char* ld_path, const char* hd_path, int accu, int* n_ld_widths, int* n_hd_wedges);

/* Host-only (no GPU): write the translation-operator files that
 * Mlib3d::setup reads (src/mlib3d.cpp:70-103) for kernel (0: exp(ir)/r,
 * 1: exp(ir)), accuracy level accu and high-frequency widths 1, 2, 4, ...
 * up to wmax -- the FP64 precompute the reference runs offline in MATLAB
 * (matlab/aug3d_script.m, aug3d_lowdata.m, aug3d_hghdata.m).  ld_path gets
 * the 7 low-frequency widths 2^-7..2^-1, hd_path the high-frequency wedges;
 * either may be NULL to skip that file.  threads <= 0 uses every host core;
 * verbose != 0 prints one progress line per width on stderr.  The output
 * does not depend on the thread count.  DDFMM_EINVAL for bad arguments,
 * DDFMM_ESETUP when a factorization fails (e.g. a rank above DVMAX=400) or a
 * file cannot be written. */
int ddfmm_precompute_operators(int kernel, int accu, int wmax, int threads, const char* ld_path, const char* hd_path,
                               int verbose);

/* Failure-path test hook, no counterpart in the reference.  On a DDFMM_MIXED
 * session: the next eval's first tensor-core GEMM launch bounds its pipeline
 * waits by wait_s (0 < wait_s <= 1) and its first block withholds the copies
 * that block waits on, so that wait runs out; the block then drains its work,
 * frees its tensor memory and flags the session, whose next synchronous call
 * (ddfmm_eval and the like) returns DDFMM_ECUDA.  Nothing faults and the
 * context stays usable.  DDFMM_EINVAL on other sessions. */
int ddfmm_session_test_gemm_stall(ddfmm_session* s, double wait_s);

/* Host-only (no GPU): build the octree and interaction lists of
 * Wave3d::setup (src/wave3d_setup.cpp:100-299) and report, per level, what
 * Wave3d::eval prints about them (src/wave3d_eval.cpp:345-372): boxes with
 * points, and the summed directional far-list sizes; plus the total number
 * of boxes created and how many are empty.  levels must hold 64 entries;
 * *nlevels receives the count used. */
typedef struct ddfmm_tree_level {
    int level;
    double width;
    int boxes;          /* boxes with points */
    int leaves;         /* terminal boxes with points */
    long long far_pairs;
    long long out_dirs; /* (box, outgoing wedge) pairs */
    long long inc_dirs; /* (box, incoming wedge) pairs */
    long long u_pairs, v_pairs, w_pairs, x_pairs;
} ddfmm_tree_level;
int ddfmm_tree_stats(const double* pos3n, int n, double K, const double* ctr3, int ptsmax, int maxlevel,
                     int ncell, int npq, int* total_boxes, int* empty_boxes, int* nlevels,
                     ddfmm_tree_level* levels);
/* Per-pass profile: while enabled, every launch of ddfmm_eval* is bracketed
 * by CUDA events on its stream.  ddfmm_profile_read returns the totals
 * accumulated since the last reset (one entry per pass label, in the order
 * the eval first launches each label), with the algorithmic flops and DRAM
 * bytes of those launches.  The reference's
 * counterpart is the per-pass wall time it prints (src/wave3d_eval.cpp:59-66). */
typedef struct ddfmm_profile_entry {
    char label[32];
    char kernel[32];
    int launches;
    double ms;
    double flops;
    double bytes;
} ddfmm_profile_entry;
int ddfmm_profile_enable(ddfmm_session* s, int on);
int ddfmm_profile_read(ddfmm_session* s, ddfmm_profile_entry* out, int max_entries, int* n_entries,
                       int reset);

int ddfmm_session_destroy(ddfmm_session* s);
const char* ddfmm_last_error(void);

/* ---------------------------------------------------------------- batches
 * No counterpart in the reference (one Wave3d per process there).  A batch
 * evaluates many independent sessions together: their launch sequences are
 * merged pass by pass (same pass, width and step type) into multi-instance
 * launches and replayed as one CUDA graph, so one matvec of every session
 * costs as many launches as the deepest single session.  Sessions must be
 * DDFMM_MIXED sessions of one device and one ACCU, must outlive the batch,
 * and must not be evaluated on their own while a batch call on them is in
 * flight (the batch uses their device buffers). */
typedef struct ddfmm_batch ddfmm_batch;
int ddfmm_batch_create(ddfmm_session* const* sessions, int n, ddfmm_batch** out);
/* One matvec of every session i with den[i] != NULL (complex64 host arrays of
 * that session's n points, interleaved floats); val[i] receives it.  Entries
 * with den[i] == NULL are not computed and val[i] is not touched.  Returns
 * when every val[i] is filled. */
int ddfmm_batch_eval_c64(ddfmm_batch* b, const float* const* den, float* const* val);
/* The same with device arrays, enqueued on `stream` (a cudaStream_t, or NULL
 * for the batch's own stream); returns after enqueueing. */
int ddfmm_batch_eval_device_c64(ddfmm_batch* b, const void* const* den_dev, void* const* val_dev, void* stream);
/* Launches per batch matvec (the merged sequence). */
int ddfmm_batch_launches(ddfmm_batch* b, int* launches);
int ddfmm_batch_destroy(ddfmm_batch* b);

/* ---------------------------------------------------------------- server
 * No counterpart in the reference.  A matvec server for callers that issue
 * matvecs on many geometries at once (iterative boundary-integral solvers):
 * sessions (DDFMM_MIXED) are admitted against a device-memory budget and a
 * serving thread batches pending requests across sessions.  Each tick takes
 * the oldest pending request of every admitted session and evaluates them
 * together (one masked batch matvec); requests arriving meanwhile go to the
 * next tick.  Sessions are created by an admission thread; one that does not
 * fit the budget waits, in order, until a removal frees memory, and one
 * larger than the whole budget is rejected. */
typedef struct ddfmm_server ddfmm_server;
enum {
    DDFMM_SESSION_WAITING = 0,
    DDFMM_SESSION_ADMITTED = 1,
    DDFMM_SESSION_REJECTED = 2,
    DDFMM_SESSION_REMOVED = 3,
    DDFMM_SESSION_FAILED = 4
};
typedef struct ddfmm_server_stats {
    long long requests;       /* completed since the last reset */
    long long ticks;
    double mean_batch;        /* requests per tick */
    double p50_ms, p99_ms, max_ms;  /* submit -> completion */
    double busy_s;            /* time spent in ticks */
    long long used_bytes;     /* device bytes of the admitted sessions */
    int admitted, waiting;
} ddfmm_server_stats;
int ddfmm_server_create(int device, double budget_bytes, ddfmm_server** out);
/* Arguments as ddfmm_session_create; the session is queued for admission on
 * the server's device.  *sid identifies it. */
int ddfmm_server_add_session(ddfmm_server* sv, const double* pos3n, int n, int kernel, int accu, int npq, double K,
                             const double* ctr3, int ptsmax, int maxlevel, int ncell, const char* ld_path,
                             const char* hd_path, int* sid);
/* *state = DDFMM_SESSION_*; for REJECTED / FAILED ddfmm_last_error gives why. */
int ddfmm_server_session_state(ddfmm_server* sv, int sid, int* state);
/* Queued requests of a removed session fail; its memory is released between ticks. */
int ddfmm_server_remove_session(ddfmm_server* sv, int sid);
/* Queue one matvec: den / val are complex64 host arrays of the session's n
 * points (interleaved floats) that must stay valid until it completes. */
int ddfmm_server_submit(ddfmm_server* sv, int sid, const float* den, float* val, long long* ticket);
/* *done = 1 when the request completed (val filled), 0 after timeout_s;
 * a failed request returns an error status with the reason. */
int ddfmm_server_wait(ddfmm_server* sv, long long ticket, double timeout_s, int* done);
int ddfmm_server_poll(ddfmm_server* sv, long long ticket, int* done);
int ddfmm_server_get_stats(ddfmm_server* sv, ddfmm_server_stats* out, int reset);
int ddfmm_server_destroy(ddfmm_server* sv);

#ifdef __cplusplus
}
#endif
#endif
