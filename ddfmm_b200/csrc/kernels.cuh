// Device kernels of the directional FMM eval and their launch descriptors.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace ddfmm {

enum KernelType { KERNEL_HELM = 0, KERNEL_EXPR = 1 };  // include/kernel3d.hpp:24-27
enum GemmMode { GEMM_SET = 0, GEMM_ADD = 1, GEMM_ATOMIC = 2 };

// One shared operator A (m x k, column-major, leading dimension lda) applied
// to ncol gathered columns: y[yoff[c]..] (op)= A * x[xoff[c]..].
struct GemmProblem {
    const double2* A;
    int m, k, lda;
    int col0;  // first entry in the column arrays
    int ncol;
    const float* packed;  // tcgen05 form: an already packed copy of A (A may then be null)
};
// A launch is a list of output tiles of up to GEMM_TILE_M rows x GEMM_TILE_N columns.
constexpr int GEMM_TILE_M = 64, GEMM_TILE_N = 64;
void gemm_init();
struct GemmTile {
    int prob;
    int row0;
    int col0;  // relative to the problem's first column
    int pad;
};

// Kernel-matrix generation job: out(i,j) = G(trg_i + ts, src_j + ss),
// trg/src are 3 x n point arrays (coordinate fastest), out column-major.
struct KmatJob {
    const double* trg;
    const double* src;
    double2* out;
    double ts[3];
    double ss[3];
    int m, k;
    long long elem0;  // prefix offset of this job's elements in the launch
};

// A set of points: p_k = scale * x[3k..3k+2] + shift.
struct PtSet {
    const double* x;
    double shift[3];
    double scale;
    int n;
};
// Point-interaction work item: out[t] += sum_s G(trg_t, src_s) den[s] over
// the source segments src_begin..src_end of the item.
struct PtItem {
    PtSet trg;
    double2* out;
    int src_begin, src_end;
};
struct PtSrc {
    PtSet src;
    const double2* den;
};

void launch_kmat(const KmatJob* jobs_dev, int njobs, long long total, int kernel, cudaStream_t s);
void launch_gemm(const GemmProblem* probs_dev, const GemmTile* tiles_dev, int ntiles,
                 const long long* xoff, const long long* yoff, const double2* X, double2* Y, int mode,
                 cudaStream_t s);
// tpi: the launch shape, chosen per step by the session's autotuner: 4, 8, 16 or
// 32 threads per item, each thread taking targets and walking the sources in
// global memory; or one warp per item with the item's sources staged in
// shared memory, lanes over targets (PT_WARP_TARGETS: 4 targets a lane;
// PT_WARP_TARGETS2: 2, fewer registers) or over sources with a warp-shuffle
// reduction per target (PT_WARP_SOURCES: 8 targets a pass; PT_WARP_SOURCES4: 4)
constexpr int PT_WARP_TARGETS = 1001, PT_WARP_SOURCES = 1002, PT_WARP_TARGETS2 = 1003, PT_WARP_SOURCES4 = 1004;
__host__ __device__ constexpr bool pt_warp_shape(int tpi) { return tpi >= PT_WARP_TARGETS && tpi <= PT_WARP_SOURCES4; }
void launch_pt(const PtItem* items_dev, int nitems, const PtSrc* srcs_dev, int kernel, cudaStream_t s, int tpi = 32);

// FFT-based low-frequency M2L on a G^3 grid (G = 2P), see kernels.cu.
struct VlistLevel {
    int G, P;
    int nE;                 // equivalent / check points per box
    const int* cube_idx;    // nE indices of the uep (== dcp) nodes in the P^3 corner cube [P, 2P)^3
    const double2* tns;     // 343 x G^3 FFT'd translation tensors (zero when near)
    const double2* twf;     // G forward twiddles exp(-2 pi i m / G)
    const double2* twb;     // G backward twiddles exp(+2 pi i m / G)
};
void vlist_init(int G);
// The forward and inverse transforms take one box per block and one thread per
// (ka, kb) line of the grid; their shared memory holds the twiddles (G P) and
// the three partial transforms (P^3, P^2 G, P G^2 elements of es bytes).
__host__ __device__ constexpr int vt_threads(int G) { return ((G * G + 31) / 32) * 32; }
size_t vt_smem(int G, size_t es);
void launch_vlist_forward(const VlistLevel& L, const int* boxes, int nbox, const double2* upeq,
                          double2* spec, cudaStream_t s);
// The V-list sums in Fourier space, by target parent: the target boxes of a
// level are grouped by their parent (the groups in Morton order of the
// parents); a group lists the union of its targets' V-list sources, each as
//   {spectrum row of the source, (tbase << 8) | mask}
// where bit c of mask says that the child at position c = 4a + 2b + c' of
// the parent (offset (a, b, c') from twice the parent's index) has the
// source in its V list, and tbase is the translation-tensor index of that
// pair for child position 0; child position c adds a + 7b + 49c'.
// tsp[t] (G^3 per target, rows in group order) receives the summed spectrum
// of target t, overwritten each eval.
constexpr int VGROUP_WARPS = 8;  // target parents per block of the sums
struct VlistGroups {
    const int* gptr;   // ngroups + 1: the source entries of each group
    const int2* gsrc;  // the source entries
    const int* gtrg;   // ngroups x 8: row of tsp of each child position, -1 where none
    int ngroups;
};
void launch_vlist_group(const VlistLevel& L, const VlistGroups& V, const double2* spec, double2* tsp,
                        cudaStream_t s);
// dnchk[trg[t]] += pruned inverse DFT of tsp[t] / G^3 at the corner-cube nodes
void launch_vlist_inverse(const VlistLevel& L, const int* trg, int ntrg, const double2* tsp, double2* dnchk,
                          cudaStream_t s);

// mixed-precision form (kernels_mixed.cu): complex FP32 data behind the same
// descriptors; GemmProblem::A, PtItem::out, PtSrc::den and VlistLevel::tns /
// twf / twb then point to float2 data.
// PRECISION_MIXED multiplies on tcgen05 (kernels_umma.cu); PRECISION_MIXED_MMA_SYNC
// is the same form with the warp-level mma.sync GEMM (cgemm_kernel), kept for comparison.
enum Precision { PRECISION_FP64 = 0, PRECISION_MIXED = 1, PRECISION_MIXED_MMA_SYNC = 2 };
void cgemm_init();
void launch_cgemm(const GemmProblem* probs_dev, const GemmTile* tiles_dev, int ntiles, const long long* xoff,
                  const long long* yoff, const void* X, void* Y, int mode, cudaStream_t s);

// Multi-instance launches of the mixed form.  A launch is a device array of
// per-instance sub-launches plus the prefix sums of their work items (nsub + 1
// entries); a sub-launch is skipped when `active` (indexed by `inst`) is given
// and holds 0.  A single session is a launch with one sub-launch.
struct PtSub {
    const PtItem* items;
    const PtSrc* srcs;
    int nitems;
    int kernel;  // KERNEL_HELM / KERNEL_EXPR
    int inst;
    int pad;
};
struct VfSub {  // V-list source spectra, one work item per source box
    VlistLevel L;
    const int* boxes;
    const float2* upeq;
    float2* spec;
    int nbox;
    int inst;
};
struct VaSub {  // V-list sums by target parent (VlistGroups), one work item per group
    VlistLevel L;
    const int* gptr;
    const int2* gsrc;
    const int* gtrg;
    const float2* spec;
    float2* tsp;
    int ngroups;
    int inst;
};
struct ViSub {  // V-list inverse transforms, one work item per target box
    VlistLevel L;
    const int* trg;
    const float2* tsp;
    float2* dnchk;
    int ntrg;
    int inst;
};
struct MoveSub {  // complex64 point data between point-id and leaf order
    const void* in;
    const int* perm;
    void* out;
    int n;
    int inst;
};
struct ZeroSub {
    void* p;
    long long n8;  // 8-byte words
    int inst;
    int pad;
};
void launch_pt32(const PtSub* subs, const int* prefix, int nsub, int nitems, const int* active, cudaStream_t s,
                 int tpi = 32);
void vlist32_init(int G);
// A launch with nsub == 1 passes its sub-launch as `one` (host copy, sent as
// a kernel parameter); `subs` / `prefix` are then not read.
void launch_vlist_forward32(const VfSub* subs, const int* prefix, int nsub, int nbox, int G, const int* active,
                            void* spec_override, cudaStream_t s, const VfSub* one);
// work items: groups (launch_vlist_group32) or targets (launch_vlist_inverse32)
void launch_vlist_group32(const VaSub* subs, const int* prefix, int nsub, int ngroups, int G, const int* active,
                          const void* spec_override, cudaStream_t s, const VaSub* one);
void launch_vlist_inverse32(const ViSub* subs, const int* prefix, int nsub, int ntrg, int G, const int* active,
                            cudaStream_t s, const ViSub* one);
void launch_move32(const MoveSub* subs, const int* prefix, int nsub, int n, const int* active, int scatter,
                   cudaStream_t s);
void launch_zero(const ZeroSub* subs, const long long* prefix, int nsub, long long n8, const int* active,
                 cudaStream_t s);
void launch_gather32(const void* den, const int* perm, void* out, int n, int c64, cudaStream_t s);
void launch_scatter32(const void* in, const int* perm, void* val, int n, int c64, cudaStream_t s);
void launch_to_c64(const double2* a, float2* b, long long n, cudaStream_t s);

// mixed-form GEMM on tcgen05 (kernels_umma.cu): 128 gathered columns x up to
// 128 complex operator rows per tile, operator packed at setup as split TF32.
struct UmmaProblem {
    const float* B;      // packed operator (umma_pack_kernel layout)
    size_t tile_stride;  // floats between 128-row tiles of the packed operator
    int m, k, nkb;       // complex rows, complex columns, 16-wide real K blocks
    int col0, ncol;      // gathered columns, as in GemmProblem
};
struct UmmaTile {
    int prob;
    int rtile;  // 128-row tile of the operator
    int row0;   // = 128 * rtile
    int rows;   // complex rows of this tile (<= 128)
    int col0;   // relative to the problem's first column
    int pad;
};
struct UmmaSub {  // one instance's part of a multi-instance GEMM launch
    const UmmaProblem* probs;
    const UmmaTile* tiles;
    const long long* xoff;
    const long long* yoff;
    const float2* X;
    float2* Y;
    int ntiles;
    int mode;
    int inst;
    int pad;
};
struct UmmaPackJob {
    const float2* A;  // complex FP32 operator, column-major
    float* dst;
    size_t tile_stride;
    int m, k, lda, nkb;
};
void umma_init();
int umma_nkb(int k);
size_t umma_tile_stride(int k);
size_t umma_packed_floats(int m, int k);
void launch_umma_pack(const UmmaPackJob* jobs_dev, int njobs, cudaStream_t s);
// nsub == 1: `one` is that sub-launch (host copy, sent as a kernel parameter).
// wait_ns bounds every pipeline wait (0: 1 s); withhold != 0 is the failure-path
// test hook: block 0 issues no operator copies, so its first wait runs out, the
// block drains, frees its tensor memory and sets *err.  order (nsub > 1,
// optional): the launch's tiles in the order the blocks take them, entry
// j << 24 | t for tile t of sub-launch j (j < 256, t < 2^24).
void launch_umma_cgemm(const UmmaSub* subs, const int* prefix, int nsub, int ntiles, const int* active, int* err,
                       cudaStream_t s, const UmmaSub* one, unsigned long long wait_ns = 0, int withhold = 0,
                       const int* order = nullptr);

// gather/scatter helpers
void launch_gather_den(const double2* den, const int* perm, double2* out, int n, cudaStream_t s);
void launch_scatter_val(const double2* in, const int* perm, double2* val, int n, cudaStream_t s);
void launch_direct(const double* pos, const double2* den, int n, const int* chk, int nchk,
                   double2* out, int kernel, cudaStream_t s);

}  // namespace ddfmm
