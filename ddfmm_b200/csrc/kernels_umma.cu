// Mixed-form complex GEMM on the 5th-generation tensor cores (tcgen05, TMEM).
//
// Problem (as in cgemm_kernel): Y[:, c] (op)= A * X[:, c] for gathered
// columns c, A an m x k complex operator.  One tile is posed as the real GEMM
//     D (128 x N) = Xt (128 x K) * Bt (K x N)
// with M = 128 gathered columns, K = 2k (each complex x_j as the pair re, im)
// and N = 2 * rows: operator row i becomes the two real rows
//     [Ar(i,:), -Ai(i,:)] (real part)  and  [Ai(i,:), Ar(i,:)] (imaginary part)
// interleaved per j, so row c of D is output column c as interleaved complex.
// 3xTF32: B = Bhi + Blo and X = Xhi + Xlo in TF32, D = Xhi Bhi + Xlo Bhi +
// Xhi Blo accumulated in FP32 in tensor memory (TMEM lane = gathered column,
// TMEM column = real output row).
//
// Operands sit in shared memory K-major.  The operator uses the no-swizzle
// core-matrix layout: a core matrix is 8 rows x 16 bytes (4 TF32 along K); the
// two core matrices of an 8-wide K block are 128 B apart (descriptor LBO) and
// 8-row groups UBK * 32 B apart (SBO); it is packed into exactly this layout,
// already split, at session setup (umma_pack_kernel), and copied in linearly.
// The gathered columns use the 64-byte swizzled layout (core_off_a): a
// column's K block is one 64-byte row, so the producers' stores of whole
// column blocks hit every shared-memory bank once per half-warp.
//
// Persistent: one block per SM walks the tile list (tiles of one
// problem adjacent, so the blocks in flight share its packed operator in L2)
// with two TMEM accumulators of 256 columns, so the epilogue of one tile
// overlaps the main loop of the next.  Warp roles, over a USTAGES-deep ring of
// K blocks that runs on across tiles:
//   producers  UPSETS sets of 4 warps, set j taking every UPSETS-th K block from
//              j on; 32 gathered columns per warp: load the 8 complex of a K block
//              of each column (8-lane groups, 64 contiguous bytes; zero past k
//              or ncol), UPREF blocks ahead in registers; when a ring slot is
//              free, split (hi = the top 19 bits, lo = TF32(x - hi)) into it,
//              fence to the async proxy, arrive on full[s] (every lane, or one
//              elected lane per warp after __syncwarp).
//   W_LOAD_B   one thread: operator hi/lo blocks by cp.async.bulk onto full[s].
//   W_MMA      one thread: per tile waits until its accumulator is drained
//              (tmem_empty), then per block waits full[s], issues the three
//              MMAs, commits to empty[s]; after the tile commits tmem_full.
//   W_EPI..    epilogue, UEPI groups of 4 warps: warp w on TMEM lanes 32 (w % 4) ..,
//              its group on every UEPI-th 64-column chunk: TMEM -> a parking
//              area -> global, two columns at a time in 256-byte coalesced
//              rows of 16-byte stores (vector atomics where outputs collide);
//              then arrive on tmem_empty.
// Every mbarrier wait is bounded (1 s, or sooner once another role failed):
// a block that gives up stops issuing work, lets its MMAs and copies drain
// (bounded), frees its TMEM and sets *err.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace ddfmm {

constexpr int UM = 128;      // gathered columns per tile (MMA M)
#ifndef DDFMM_UMMA_BK
#define DDFMM_UMMA_BK 16
#endif
constexpr int UBK = DDFMM_UMMA_BK;  // real K per block: UBK / 8 MMA K-steps
constexpr int CPB = UBK / 2;        // complex per gathered column per block
static_assert(UBK == 8 || UBK == 16, "K block of 8 or 16");
constexpr int UNMAX = 256;   // max real rows per tile (MMA N)
#ifndef DDFMM_UMMA_STAGES
#define DDFMM_UMMA_STAGES (UBK == 16 ? 3 : 6)
#endif
#ifndef DDFMM_UMMA_PREF
#define DDFMM_UMMA_PREF (UBK == 16 ? 4 : 8)
#endif
#ifndef DDFMM_UMMA_PCH
#define DDFMM_UMMA_PCH 32
#endif
constexpr int USTAGES = DDFMM_UMMA_STAGES;  // ring depth
constexpr int UPREF = DDFMM_UMMA_PREF;      // gathered-column blocks prefetched into registers
#ifndef DDFMM_UMMA_PSETS
#define DDFMM_UMMA_PSETS 2
#endif
#ifndef DDFMM_UMMA_ELECT
#define DDFMM_UMMA_ELECT 0
#endif
constexpr int UPSETS = DDFMM_UMMA_PSETS;     // producer sets (4 warps each), alternating K blocks
constexpr bool UELECT = DDFMM_UMMA_ELECT;    // one mbarrier arrival per warp instead of per thread
#ifndef DDFMM_UMMA_EPI
#define DDFMM_UMMA_EPI 1
#endif
constexpr int UEPI = DDFMM_UMMA_EPI;  // epilogue groups of 4 warps (split an accumulator's columns)
constexpr int W_LOAD_B = 4 * UPSETS, W_MMA = W_LOAD_B + 1, W_EPI = W_LOAD_B + 2;  // warp roles
constexpr int UTHREADS = 32 * (W_EPI + 4 * UEPI);
constexpr int U_FULL_COUNT = (UELECT ? 4 : UM) + 1;  // producer arrivals + the operator loader's
constexpr int U_EMPTY_ACC_COUNT = (UELECT ? 4 : UM) * UEPI;  // epilogue arrivals
constexpr int U_A_BYTES = UM * UBK * 4;
constexpr int U_B_BYTES = UNMAX * UBK * 4;
constexpr int U_STAGE_BYTES = 2 * U_A_BYTES + 2 * U_B_BYTES;
constexpr int PCH = DDFMM_UMMA_PCH;  // epilogue chunk: complex rows parked per column
static_assert(PCH == 32, "epilogue chunk of 32 rows");
constexpr int UPS = PCH + 2;  // parking-area row stride (complex): 16-byte rows, conflict-free 16-byte accesses
constexpr int U_PARK_BYTES = 4 * UEPI * 32 * UPS * 8;  // 32 columns x PCH complex (+2 pad) per warp
// ring + parking area + alignment slack: one block per SM (also what the 512
// TMEM columns need)
constexpr int UGEMM_SMEM = USTAGES * U_STAGE_BYTES + U_PARK_BYTES + 1024;
static_assert(UGEMM_SMEM + 4096 <= 232448, "shared memory per block");
constexpr unsigned long long U_WAIT_NS = 1000000000ull;  // 1 s
constexpr uint32_t U_WAIT_ITERS = 1u << 26;

// byte offset of element (r, kk), kk < UBK, of a K block in the core-matrix layout
__host__ __device__ __forceinline__ int core_off(int r, int kk) {
    return (r >> 3) * (UBK * 32) + (kk >> 2) * 128 + (r & 7) * 16 + (kk & 3) * 4;
}

constexpr int U_ARB = UBK * 4;         // bytes of one gathered column per K block
// byte offset of element (r, kk) of a gathered-column K block in the K-major
// swizzled layout (64-byte swizzle for UBK = 16, 32-byte for UBK = 8): row r
// is U_ARB contiguous bytes at (r>>3) 8 U_ARB + (r&7) U_ARB, its 16-byte chunk
// j stored at chunk j ^ (address bits 7.. of the row), so rows r and r+1 of a
// half-warp store cover the 32 banks once
__host__ __device__ __forceinline__ int core_off_a(int r, int kk) {
    const int row = (r >> 3) * (8 * U_ARB) + (r & 7) * U_ARB;
    return row + ((((kk >> 2) ^ ((((r & 7) * U_ARB) >> 7) & (U_ARB / 16 - 1)))) << 4) + (kk & 3) * 4;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// descriptor of a gathered-column block in the swizzled layout: 8-row groups
// 8 U_ARB bytes apart (SBO), leading offset unused (one swizzle row spans the
// block's K), layout type 64-byte (4) or 32-byte (6) swizzle in bits 61-63;
// the K step of 8 TF32 moves the start address by 32 bytes
__device__ __forceinline__ uint64_t sdesc_a(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(((8 * U_ARB) >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)(U_ARB == 64 ? 4 : 6) << 61;
    return d;
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;         // LBO: K-adjacent core matrices
    d |= (uint64_t)(((UBK * 32) >> 4) & 0x3FFF) << 32;  // SBO: 8-row groups
    d |= (uint64_t)1 << 46;                        // descriptor version 1; layout type 0 (no swizzle)
    return d;
}

__device__ __forceinline__ uint32_t idesc_tf32(int n) {
    // D f32 (bits 4-5 = 1), A tf32 (7-9 = 2), B tf32 (10-12 = 2), K-major A and B
    // (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(UM >> 4) << 24);
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Wait for the phase of parity `parity`; false after limit_ns, 2^26 polls, or
// once *failed is set by another role.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* failed,
                                          unsigned long long limit_ns) {
    const uint32_t addr = smem_u32(bar);
    unsigned long long t0 = 0;
    for (uint32_t it = 0; it < U_WAIT_ITERS; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255) {
            if (failed && *failed) return false;
            const unsigned long long t = gtimer();
            if (t0 == 0)
                t0 = t;
            else if (t - t0 > limit_ns)
                return false;
        }
    }
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;\n" ::"r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void umma_tf32(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(dtmem),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

// operator split: hi = TF32 rounding of x, lo = TF32 rounding of the rest
__device__ __forceinline__ void split2(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_bits(x);
    lo = tf32_bits(x - __uint_as_float(hi));
}

// gathered-column split in place: hi = x with the 13 low mantissa bits cleared
// (exact), lo = x - hi rounded to TF32 (nearest, ties away from zero) on its
// bit pattern: add half of the dropped range, clear it (a carry moves into the
// exponent as it should).  Two integer operations instead of a conversion,
// which runs on the SM's narrow conversion pipe.
__device__ __forceinline__ void split_mask(uint32_t& w, uint32_t& lo) {
    const uint32_t hi = w & 0xFFFFE000u;
    lo = (__float_as_uint(__uint_as_float(w) - __uint_as_float(hi)) + 0x1000u) & 0xFFFFE000u;
    w = hi;
}

// ---------------------------------------------------------------- packing
// Real, interleaved, split, blocked copy of a complex operator (setup only).
// Row tile t (complex rows 128t .. 128t+rows_t, N_t = round_up(2 rows_t, 16)
// real rows) starts at dst + t * tile_stride floats and holds, per K block b,
// the hi block (N_t x 8 TF32 in core-matrix order) then the lo block.
__global__ void umma_pack_kernel(const UmmaPackJob* __restrict__ jobs, int njobs) {
    for (int j = blockIdx.y; j < njobs; j += gridDim.y) {
        const UmmaPackJob J = jobs[j];
        for (int t = 0; t * 128 < J.m; ++t) {
            const int rows = min(128, J.m - t * 128);
            const int N = ((2 * rows + 15) / 16) * 16;
            char* base = reinterpret_cast<char*>(J.dst + (size_t)t * J.tile_stride);
            const long long total = (long long)J.nkb * N * UBK;
            for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
                 e += (long long)gridDim.x * blockDim.x) {
                const int kk = (int)(e % UBK);
                const int n = (int)((e / UBK) % N);
                const int b = (int)(e / ((long long)UBK * N));
                const int kr = b * UBK + kk;  // real k
                const int i = n >> 1, kc = kr >> 1;
                float v = 0.f;
                if (i < rows && kc < J.k) {
                    const float2 a = J.A[(size_t)kc * J.lda + t * 128 + i];
                    if ((n & 1) == 0)
                        v = (kr & 1) ? -a.y : a.x;  // real-part row: [Ar, -Ai]
                    else
                        v = (kr & 1) ? a.x : a.y;   // imaginary-part row: [Ai, Ar]
                }
                uint32_t hi, lo;
                split2(v, hi, lo);
                char* blk = base + (size_t)b * 2 * N * UBK * 4;
                *reinterpret_cast<uint32_t*>(blk + core_off(n, kk)) = hi;
                *reinterpret_cast<uint32_t*>(blk + (size_t)N * UBK * 4 + core_off(n, kk)) = lo;
            }
        }
    }
}

void launch_umma_pack(const UmmaPackJob* jobs_dev, int njobs, cudaStream_t s) {
    if (njobs == 0) return;
    dim3 grid(16, njobs < 4096 ? njobs : 4096);
    umma_pack_kernel<<<grid, 256, 0, s>>>(jobs_dev, njobs);
}

int umma_nkb(int k) { return (2 * k + UBK - 1) / UBK; }

size_t umma_tile_stride(int k) { return (size_t)umma_nkb(k) * 2 * UNMAX * UBK; }

size_t umma_packed_floats(int m, int k) {
    const int nt = (m + 127) / 128;
    const int last = m - (nt - 1) * 128;
    return (size_t)(nt - 1) * umma_tile_stride(k) + (size_t)umma_nkb(k) * 2 * (((2 * last + 15) / 16) * 16) * UBK;
}

// ---------------------------------------------------------------- GEMM
// Epilogue stores of one parked chunk (PCH complex rows from row0 on, 32 columns):
// two columns per instruction, each lane two consecutive rows of one column, as
// one 16-byte store or vector atomic where the output is 16-byte aligned (two
// 8-byte ones otherwise, or one at an odd last row).  Column c of the warp's 32
// writes at Y + (c's yoff) + row.
template <int MODE>
__device__ __forceinline__ void store_one(float2* y, float2 v) {
    if (MODE == GEMM_SET) {
        *y = v;
    } else if (MODE == GEMM_ADD) {
        const float2 o = *y;
        *y = make_float2(o.x + v.x, o.y + v.y);
    } else {
        atomicAdd(y, v);
    }
}
template <int MODE>
__device__ __forceinline__ void store_chunk(const float2* park, float2* Y, long long my_yo, int col_base, int ncol,
                                            int row0, int rows, int lane) {
    const int sub = lane >> 4, r2 = 2 * (lane & 15), i = row0 + r2;
    for (int cc = 0; cc < 32; cc += 2) {
        const int col = cc + sub;
        const long long yb = __shfl_sync(0xffffffffu, my_yo, col);
        if (col_base + cc >= ncol) break;
        if (i >= rows || col_base + col >= ncol) continue;
        const float4 v = *reinterpret_cast<const float4*>(park + col * UPS + r2);
        float2* y = Y + yb + i;
        const bool two = i + 1 < rows;
        if (two && (reinterpret_cast<uintptr_t>(y) & 15) == 0) {
            float4* y4 = reinterpret_cast<float4*>(y);
            if (MODE == GEMM_SET) {
                *y4 = v;
            } else if (MODE == GEMM_ADD) {
                const float4 o = *y4;
                *y4 = make_float4(o.x + v.x, o.y + v.y, o.z + v.z, o.w + v.w);
            } else {
                atomicAdd(y4, v);
            }
        } else {
            store_one<MODE>(y, make_float2(v.x, v.y));
            if (two) store_one<MODE>(y + 1, make_float2(v.z, v.w));
        }
    }
}

// Tile ti of a launch: its sub-launch (prefix[j] <= ti < prefix[j+1], or
// order[ti] = j << 24 | tile of sub-launch j where the launch gives an order),
// tile and problem; `on` is false when the sub-launch's instance is inactive.
struct TileInfo {
    UmmaTile t;
    UmmaProblem p;
    const float2* X;
    float2* Y;
    const long long* xoff;
    const long long* yoff;
    int mode;
    bool on;
};
// MULTI = false: the launch's only sub-launch `one` (kernel parameter space);
// else subs / prefix: the block's shared-memory copies (U_SUBS_SMEM entries at
// most) or the global arrays
template <bool MULTI>
__device__ __forceinline__ TileInfo tile_info(const UmmaSub& one, const UmmaSub* subs, const int* prefix, int nsub,
                                              const int* __restrict__ order, const int* __restrict__ active, int ti) {
    int lo = 0, t = ti;
    if (MULTI) {
        if (order) {
            const unsigned e = (unsigned)__ldg(order + ti);
            lo = (int)(e >> 24);
            t = (int)(e & 0xFFFFFFu);
        } else {
            int hi = nsub - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (prefix[mid] <= ti)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            t = ti - prefix[lo];
        }
    }
    const UmmaSub& S = MULTI ? subs[lo] : one;
    TileInfo r;
    r.on = !active || active[S.inst];
    r.t = S.tiles[t];
    r.p = S.probs[r.t.prob];
    r.X = S.X;
    r.Y = S.Y;
    r.xoff = S.xoff;
    r.yoff = S.yoff;
    r.mode = S.mode;
    return r;
}
__device__ __forceinline__ int tile_n(int rows) { return ((2 * rows + 15) / 16) * 16; }

constexpr int U_SUBS_SMEM = 64;  // sub-launches cached in shared memory

template <bool MULTI>
__global__ void __launch_bounds__(UTHREADS, 1) umma_cgemm_kernel(const UmmaSub one,
                                                                 const UmmaSub* __restrict__ gsubs,
                                                                 const int* __restrict__ gprefix, int nsub,
                                                                 int ntiles, const int* __restrict__ order,
                                                                 const int* __restrict__ active, int* err,
                                                                 unsigned long long wait_ns, int withhold) {
    extern __shared__ __align__(1024) unsigned char usm_raw[];
    __shared__ UmmaSub ssubs[MULTI ? U_SUBS_SMEM : 1];
    __shared__ int sprefix[MULTI ? U_SUBS_SMEM + 1 : 1];
    const bool cached = MULTI && nsub <= U_SUBS_SMEM;
    if (cached) {
        for (int i = threadIdx.x; i < nsub; i += blockDim.x) ssubs[i] = gsubs[i];
        for (int i = threadIdx.x; i <= nsub; i += blockDim.x) sprefix[i] = gprefix[i];
    }
    const UmmaSub* subs = cached ? ssubs : gsubs;
    const int* prefix = cached ? sprefix : gprefix;
    __shared__ __align__(8) uint64_t full[USTAGES], empty[USTAGES], tmem_full[2], tmem_empty[2];
    __shared__ uint32_t tmem_base;
    __shared__ int failed_s;
    volatile int* failed = &failed_s;
    unsigned char* usm = (unsigned char*)(((uintptr_t)usm_raw + 1023) & ~(uintptr_t)1023);
    float2* park_all = reinterpret_cast<float2*>(usm + USTAGES * U_STAGE_BYTES);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        failed_s = 0;
        for (int s = 0; s < USTAGES; ++s) {
            mbar_init(&full[s], U_FULL_COUNT);
            mbar_init(&empty[s], 1);      // tcgen05.commit
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tmem_full[a], 1);    // tcgen05.commit
            mbar_init(&tmem_empty[a], U_EMPTY_ACC_COUNT);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {  // 512 TMEM columns: two accumulators of 128 lanes x 256 FP32
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;

    if (warp < W_LOAD_B) {
        // ------------------------------------------------ gathered columns
        // producer set `set` takes the blocks g = set, set + UPSETS, ... of the block
        // sequence of this block's tiles; within a set, warp cw covers columns 32cw ..
        // 32cw + 31: load i reads columns 32cw + i (32/CPB) .., CPB lanes per column
        // (lane = column, complex q), so each column's block is one contiguous load
        // and a half-warp store fills two swizzled rows (all 32 banks once).  Blocks
        // are prefetched UPREF deep into registers and split into a ring slot once
        // free.
        const int set = warp >> 2, cw = warp & 3;
        const int colw = cw * 32 + lane / CPB, q = lane % CPB;
        int coff[CPB];  // core_off_a(column, 2q) of load i
#pragma unroll
        for (int i = 0; i < CPB; ++i) coff[i] = core_off_a(colw + i * (32 / CPB), 2 * q);
        // load cursor: tile ti_i, block kb_i of nkb_i, its columns' offsets xr[]
        int ti_i = blockIdx.x, kb_i = 0, nkb_i = 0, k_i = 0;
        long long xr[CPB];
        const float2* X = nullptr;
        auto load_tile = [&]() {  // the first active tile from ti_i on
            for (; ti_i < ntiles; ti_i += gridDim.x) {
                const TileInfo T = tile_info<MULTI>(one, subs, prefix, nsub, order, active, ti_i);
                if (!T.on) continue;
                nkb_i = T.p.nkb;
                k_i = T.p.k;
                X = T.X;
                const int ncol = min(UM, T.p.ncol - T.t.col0);
#pragma unroll
                for (int i = 0; i < CPB; ++i) {
                    const int c = colw + i * (32 / CPB);
                    xr[i] = c < ncol ? __ldg(T.xoff + T.p.col0 + T.t.col0 + c) : -1;
                }
                return;
            }
        };
        auto advance = [&]() {
            if (++kb_i == nkb_i) {
                kb_i = 0;
                ti_i += gridDim.x;
                load_tile();
            }
        };
        auto fetch = [&](float2(&dst)[CPB]) {  // the block at the cursor, then advance it
#pragma unroll
            for (int i = 0; i < CPB; ++i) {
                const int kc = kb_i * CPB + q;
                const long long x = xr[i];
                dst[i] = (x >= 0 && kc < k_i) ? __ldg(X + x + kc) : make_float2(0.f, 0.f);
            }
            for (int a = 0; a < UPSETS && ti_i < ntiles; ++a) advance();
        };
        load_tile();
        for (int a = 0; a < set && ti_i < ntiles; ++a) advance();
        float2 pre[UPREF][CPB];
        int loaded = 0;
#pragma unroll
        for (int d = 0; d < UPREF; ++d)
            if (ti_i < ntiles) {
                fetch(pre[d]);
                ++loaded;
            }
        int n = 0;  // this set's blocks done; block n sits in pre[n % UPREF]
        while (n < loaded && !*failed) {
#pragma unroll
            for (int d = 0; d < UPREF; ++d) {
                if (n >= loaded || *failed) break;
                const int g = n * UPSETS + set;
                const int s = g % USTAGES;
                if (g >= USTAGES && !mbar_wait(&empty[s], ((g / USTAGES) - 1) & 1, failed, wait_ns)) {
                    *failed = 1;
                    break;
                }
                unsigned char* ahi = usm + s * U_STAGE_BYTES;
                unsigned char* alo = ahi + U_A_BYTES;
#pragma unroll
                for (int i = 0; i < CPB; ++i) {
                    uint2 w = make_uint2(__float_as_uint(pre[d][i].x), __float_as_uint(pre[d][i].y));
                    uint2 l;
                    split_mask(w.x, l.x);
                    split_mask(w.y, l.y);
                    *reinterpret_cast<uint2*>(ahi + coff[i]) = w;
                    *reinterpret_cast<uint2*>(alo + coff[i]) = l;
                }
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                if (UELECT) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&full[s]);
                } else {
                    mbar_arrive(&full[s]);
                }
                if (ti_i < ntiles) {
                    fetch(pre[d]);
                    ++loaded;
                }
                ++n;
            }
        }
    } else if (warp == W_LOAD_B) {
        // ------------------------------------------------ operator blocks
        // withhold (failure-path test hook): block 0 issues no operator copy and no
        // arrival at all, so its MMA issuer's bounded wait on full[0] runs out
        if (lane == 0 && !(withhold && blockIdx.x == 0)) {
            int g = 0;
            for (int ti = blockIdx.x; ti < ntiles && !*failed; ti += gridDim.x) {
                const TileInfo T = tile_info<MULTI>(one, subs, prefix, nsub, order, active, ti);
                if (!T.on) continue;
                const char* Bt = reinterpret_cast<const char*>(T.p.B + (size_t)T.t.rtile * T.p.tile_stride);
                const uint32_t blk = (uint32_t)tile_n(T.t.rows) * UBK * 4;
                for (int kb = 0; kb < T.p.nkb; ++kb, ++g) {
                    const int s = g % USTAGES;
                    if (g >= USTAGES && !mbar_wait(&empty[s], ((g / USTAGES) - 1) & 1, failed, wait_ns)) {
                        *failed = 1;
                        break;
                    }
                    unsigned char* bhi = usm + s * U_STAGE_BYTES + 2 * U_A_BYTES;
                    const char* src = Bt + (size_t)kb * 2 * blk;
                    mbar_expect_tx(&full[s], 2 * blk);
                    bulk_g2s(bhi, src, blk, &full[s]);
                    bulk_g2s(bhi + U_B_BYTES, src + blk, blk, &full[s]);
                }
            }
        }
    } else if (warp == W_MMA) {
        // ------------------------------------------------ MMA issue
        if (lane == 0) {
            int g = 0, it = 0, last = -1;
            for (int ti = blockIdx.x; ti < ntiles && !*failed; ti += gridDim.x) {
                const TileInfo T = tile_info<MULTI>(one, subs, prefix, nsub, order, active, ti);
                if (!T.on) continue;
                const uint32_t idesc = idesc_tf32(tile_n(T.t.rows));
                const int acc = it & 1;
                if (it >= 2 && !mbar_wait(&tmem_empty[acc], ((it >> 1) - 1) & 1, failed, wait_ns)) {
                    *failed = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(acc * 256);
                for (int kb = 0; kb < T.p.nkb; ++kb, ++g) {
                    const int s = g % USTAGES;
                    if (!mbar_wait(&full[s], (g / USTAGES) & 1, failed, wait_ns)) {
                        *failed = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t ahi = smem_u32(usm + s * U_STAGE_BYTES), alo = ahi + U_A_BYTES;
                    const uint32_t bhi = ahi + 2 * U_A_BYTES, blo = bhi + U_B_BYTES;
                    const int KS = min(UBK / 8, (2 * T.p.k - kb * UBK + 7) >> 3);  // K steps holding k (zeros past it)
#pragma unroll
                    for (int ks = 0; ks < UBK / 8; ++ks) {  // K = 8 per MMA
                        if (ks >= KS) break;
                        const uint32_t o = ks * 256, oa = ks * 32;  // operator: two core matrices; columns: 32 B
                        const uint64_t dah = sdesc_a(ahi + oa), dal = sdesc_a(alo + oa);
                        umma_tf32(d, dah, sdesc(bhi + o), idesc, (kb > 0 || ks > 0) ? 1u : 0u);
                        umma_tf32(d, dal, sdesc(bhi + o), idesc, 1u);
                        umma_tf32(d, dah, sdesc(blo + o), idesc, 1u);
                    }
                    umma_commit(&empty[s]);
                    last = g;
                }
                if (*failed) break;
                umma_commit(&tmem_full[acc]);
                ++it;
            }
            if (*failed && last >= 0)  // let the MMAs already issued finish before TMEM is freed
                mbar_wait(&empty[last % USTAGES], (last / USTAGES) & 1, nullptr, wait_ns);
        }
    } else {
        // ------------------------------------------------ epilogue
        const int ew = warp - W_EPI;  // group ew / 4 takes every UEPI-th chunk of accumulator columns
        const int qw = warp & 3;      // TMEM lanes 32 qw .. 32 qw + 31 = tile columns
        const int first = (ew >> 2) * 2 * PCH;
        float2* park = park_all + ew * (32 * UPS);
        auto release = [&](int acc) {  // this warp is done reading the accumulator
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            if (UELECT) {
                __syncwarp();
                if (lane == 0) mbar_arrive(&tmem_empty[acc]);
            } else {
                mbar_arrive(&tmem_empty[acc]);
            }
        };
        int it = 0;
        for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
            const TileInfo T = tile_info<MULTI>(one, subs, prefix, nsub, order, active, ti);
            if (!T.on) continue;
            const int ncol = min(UM, T.p.ncol - T.t.col0);
            const int rows = T.t.rows, N = tile_n(rows);
            const int acc = it & 1;
            const int mycol = qw * 32 + lane;
            const long long my_yo = mycol < ncol ? __ldg(T.yoff + T.p.col0 + T.t.col0 + mycol) + T.t.row0 : 0;
            float2* const Y = T.Y;
            const int mode = T.mode;
            bool ok = !*failed && mbar_wait(&tmem_full[acc], (it >> 1) & 1, failed, wait_ns);
            ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
            if (!ok) {
                *failed = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t src = tmem + ((uint32_t)(qw * 32) << 16) + (uint32_t)(acc * 256);
            if (first >= N) release(acc);
            for (int c0 = first; c0 < N; c0 += UEPI * 2 * PCH) {
#pragma unroll
                for (int h = 0; h < 2 * PCH; h += 16) {
                    if (c0 + h < N) {  // N is a multiple of 16
                        uint32_t v[16];
                        asm volatile(
                            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                            "%15}, [%16];\n"
                            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                              "=r"(v[14]), "=r"(v[15])
                            : "r"(src + (uint32_t)(c0 + h))
                            : "memory");
                        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                        for (int e = 0; e < 8; e += 2)  // 16-byte stores: 8 lanes cover the 32 banks once
                            *reinterpret_cast<float4*>(park + lane * UPS + (h >> 1) + e) =
                                make_float4(__uint_as_float(v[2 * e]), __uint_as_float(v[2 * e + 1]),
                                            __uint_as_float(v[2 * e + 2]), __uint_as_float(v[2 * e + 3]));
                    }
                }
                if (c0 + UEPI * 2 * PCH >= N) release(acc);  // last chunk read: accumulator back to the MMA issuer
                __syncwarp();
                const int row0 = c0 >> 1;  // first complex row of the chunk
                if (mode == GEMM_SET)
                    store_chunk<GEMM_SET>(park, Y, my_yo, qw * 32, ncol, row0, rows, lane);
                else if (mode == GEMM_ADD)
                    store_chunk<GEMM_ADD>(park, Y, my_yo, qw * 32, ncol, row0, rows, lane);
                else
                    store_chunk<GEMM_ATOMIC>(park, Y, my_yo, qw * 32, ncol, row0, rows, lane);
                __syncwarp();
            }
            ++it;
        }
    }
    __syncthreads();
    if (*failed && tid == 0) {
        // bounded drain of operator copies still in flight, then report
        const unsigned long long t0 = gtimer();
        while (gtimer() - t0 < 200000ull) __nanosleep(1000);
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512) : "memory");
}

static int g_umma_sms = 0;

void umma_init() {
    cudaFuncSetAttribute(umma_cgemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, UGEMM_SMEM);
    cudaFuncSetAttribute(umma_cgemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, UGEMM_SMEM);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_umma_sms, cudaDevAttrMultiProcessorCount, dev);
}

void launch_umma_cgemm(const UmmaSub* subs, const int* prefix, int nsub, int ntiles, const int* active, int* err,
                       cudaStream_t s, const UmmaSub* one, unsigned long long wait_ns, int withhold, const int* order) {
    if (ntiles == 0) return;
    const int sms = g_umma_sms > 0 ? g_umma_sms : 148;
    const int grid = ntiles < sms ? ntiles : sms;
    if (wait_ns == 0) wait_ns = U_WAIT_NS;
    if (nsub == 1) {
        if (!one) return;  // a single sub-launch is passed by value
        umma_cgemm_kernel<false><<<grid, UTHREADS, UGEMM_SMEM, s>>>(*one, subs, prefix, nsub, ntiles, nullptr, active,
                                                                     err, wait_ns, withhold);
    } else {
        umma_cgemm_kernel<true><<<grid, UTHREADS, UGEMM_SMEM, s>>>(UmmaSub{}, subs, prefix, nsub, ntiles, order, active,
                                                                    err, wait_ns, withhold);
    }
}

}  // namespace ddfmm
