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
// Operands sit in shared memory in the no-swizzle K-major core-matrix layout:
// a core matrix is 8 rows x 16 bytes (4 TF32 along K), K-adjacent core
// matrices are 128 B apart (descriptor LBO) and 8-row groups 512 B apart
// (SBO) within a 16-element K block.  The operator is packed into exactly
// this layout, already split, at session setup (umma_pack_kernel) and copied
// per K block with cp.async.bulk; the gathered columns are split and stored
// by the block's threads.  One thread issues the MMAs of block kb while all
// threads prefetch block kb+1; tcgen05.commit arrives on an mbarrier when
// the MMAs are done reading a stage.  Every mbarrier wait is bounded in time
// and iterations: on timeout the block drains what it has in flight (again
// bounded), records an error in *err, skips its output and frees its TMEM.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace ddfmm {

constexpr int UM = 128;      // gathered columns per tile (MMA M)
constexpr int UBK = 16;      // real K elements per block (two K=8 MMAs)
constexpr int UNMAX = 256;   // max real rows per tile (MMA N)
constexpr int UTHREADS = 128;
// per stage: A hi + lo (128 x 16 TF32 each), B hi + lo (up to 256 x 16 each)
constexpr int U_A_BYTES = UM * UBK * 4;
constexpr int U_B_BYTES = UNMAX * UBK * 4;
constexpr int U_STAGE_BYTES = 2 * U_A_BYTES + 2 * U_B_BYTES;
// two stages + alignment slack: ~101 KB per block with the static part, so at
// most two blocks share an SM and their 2 x 256 TMEM columns always fit
constexpr int UGEMM_SMEM = 2 * U_STAGE_BYTES + 1024;
constexpr unsigned long long U_WAIT_NS = 1000000000ull;  // 1 s
constexpr uint32_t U_WAIT_ITERS = 1u << 26;

// byte offset of element (r, kk) of a K block in the core-matrix layout
__host__ __device__ __forceinline__ int core_off(int r, int kk) {
    return (r >> 3) * 512 + (kk >> 2) * 128 + (r & 7) * 16 + (kk & 3) * 4;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;    // LBO: K-adjacent core matrices
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;    // SBO: 8-row groups
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

// wait for the phase of parity `parity` to complete; false after 1 s or 2^26 polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
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
            unsigned long long t = gtimer();
            if (t0 == 0)
                t0 = t;
            else if (t - t0 > U_WAIT_NS)
                return false;
        }
    }
    return false;
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

__device__ __forceinline__ void split2(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_bits(x);
    lo = tf32_bits(x - __uint_as_float(hi));
}

// ---------------------------------------------------------------- packing
// Real, interleaved, split, blocked copy of a complex operator (setup only).
// Row tile t (complex rows 128t .. 128t+rows_t, N_t = round_up(2 rows_t, 16)
// real rows) starts at dst + t * tile_stride floats and holds, per K block b,
// the hi block (N_t x 16 TF32 in core-matrix order) then the lo block.
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

size_t umma_tile_stride(int k) { return (size_t)((2 * k + UBK - 1) / UBK) * 2 * UNMAX * UBK; }

size_t umma_packed_floats(int m, int k) {
    const int nkb = (2 * k + UBK - 1) / UBK;
    const int nt = (m + 127) / 128;
    const int last = m - (nt - 1) * 128;
    return (size_t)(nt - 1) * umma_tile_stride(k) + (size_t)nkb * 2 * (((2 * last + 15) / 16) * 16) * UBK;
}

int umma_nkb(int k) { return (2 * k + UBK - 1) / UBK; }

// ---------------------------------------------------------------- GEMM
__global__ void __launch_bounds__(UTHREADS) umma_cgemm_kernel(const UmmaProblem* __restrict__ probs,
                                                              const UmmaTile* __restrict__ tiles,
                                                              const long long* __restrict__ xoff,
                                                              const long long* __restrict__ yoff,
                                                              const float2* __restrict__ X, float2* Y, int mode,
                                                              int* err) {
    extern __shared__ __align__(1024) unsigned char usm_raw[];
    __shared__ __align__(8) uint64_t bar_b[2], bar_mma[2];
    __shared__ uint32_t tmem_base;
    __shared__ long long xo[UM], yo[UM];
    __shared__ int failed;
    unsigned char* usm = (unsigned char*)(((uintptr_t)usm_raw + 1023) & ~(uintptr_t)1023);

    const UmmaTile t = tiles[blockIdx.x];
    const UmmaProblem p = probs[t.prob];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncol = min(UM, p.ncol - t.col0);
    const int rows = t.rows;                     // complex rows of this tile
    const int N = ((2 * rows + 15) / 16) * 16;   // real rows (MMA N)
    const int nkb = p.nkb;
    const char* Bt = reinterpret_cast<const char*>(p.B + (size_t)t.rtile * p.tile_stride);
    const uint32_t blk_bytes = (uint32_t)N * UBK * 4;

    xo[tid] = tid < ncol ? xoff[p.col0 + t.col0 + tid] : -1;
    yo[tid] = tid < ncol ? yoff[p.col0 + t.col0 + tid] : -1;
    if (tid == 0) {
        failed = 0;
        for (int s = 0; s < 2; ++s) {
            mbar_init(&bar_b[s], 1);
            mbar_init(&bar_mma[s], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {  // 256 TMEM columns: 128 lanes x 256 FP32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;

    // gathered columns: per K block each thread handles 4 (column, 2 complex) pieces;
    // a warp instruction covers 8 columns x 4 pieces -> 16-byte conflict-free stores
    const int q4 = lane & 3;
    float2 pre[4][2];
    auto fetch_a = [&](int kb) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int r = warp * 32 + c * 8 + (lane >> 2);
            const int kc = kb * (UBK / 2) + 2 * q4;
            const long long o = xo[r];
            pre[c][0] = (o >= 0 && kc < p.k) ? X[o + kc] : make_float2(0.f, 0.f);
            pre[c][1] = (o >= 0 && kc + 1 < p.k) ? X[o + kc + 1] : make_float2(0.f, 0.f);
        }
    };
    auto store_a = [&](int s) {
        unsigned char* ahi = usm + s * U_STAGE_BYTES;
        unsigned char* alo = ahi + U_A_BYTES;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int r = warp * 32 + c * 8 + (lane >> 2);
            uint4 h, l;
            split2(pre[c][0].x, h.x, l.x);
            split2(pre[c][0].y, h.y, l.y);
            split2(pre[c][1].x, h.z, l.z);
            split2(pre[c][1].y, h.w, l.w);
            const int off = core_off(r, 4 * q4);
            *reinterpret_cast<uint4*>(ahi + off) = h;
            *reinterpret_cast<uint4*>(alo + off) = l;
        }
    };
    // operator K block (hi and lo) into stage s: one thread, two bulk copies
    auto load_b = [&](int s, int kb) {
        unsigned char* bhi = usm + s * U_STAGE_BYTES + 2 * U_A_BYTES;
        const char* src = Bt + (size_t)kb * 2 * blk_bytes;
        mbar_expect_tx(&bar_b[s], 2 * blk_bytes);
        bulk_g2s(bhi, src, blk_bytes, &bar_b[s]);
        bulk_g2s(bhi + U_B_BYTES, src + blk_bytes, blk_bytes, &bar_b[s]);
    };

    int last_load = -1, last_commit = -1;  // tracked by thread 0
    if (tid == 0) {
        load_b(0, 0);
        last_load = 0;
    }
    fetch_a(0);
    store_a(0);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    const uint32_t idesc = idesc_tf32(N);
    for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb & 1;
        if (kb + 1 < nkb) fetch_a(kb + 1);  // global loads in flight during the MMA issue
        if (tid == 0 && !failed) {
            if (!mbar_wait(&bar_b[s], (kb >> 1) & 1)) {
                failed = 1;
            } else {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t ahi = smem_u32(usm + s * U_STAGE_BYTES), alo = ahi + U_A_BYTES;
                const uint32_t bhi = ahi + 2 * U_A_BYTES, blo = bhi + U_B_BYTES;
#pragma unroll
                for (int ks = 0; ks < UBK / 8; ++ks) {  // K = 8 per MMA: two core-matrix columns, 256 B
                    const uint32_t o = ks * 256;
                    umma_tf32(tmem, sdesc(ahi + o), sdesc(bhi + o), idesc, (kb > 0 || ks > 0) ? 1u : 0u);
                    umma_tf32(tmem, sdesc(alo + o), sdesc(bhi + o), idesc, 1u);
                    umma_tf32(tmem, sdesc(ahi + o), sdesc(blo + o), idesc, 1u);
                }
                umma_commit(&bar_mma[s]);
                last_commit = kb;
            }
        }
        if (kb + 1 < nkb) {
            const int ns = s ^ 1;
            if (kb >= 1) {  // the MMAs of block kb-1 must be done reading stage ns
                if (tid == 0 && !failed && !mbar_wait(&bar_mma[ns], ((kb - 1) >> 1) & 1)) failed = 1;
                __syncthreads();
            }
            if (tid == 0 && !failed) {
                load_b(ns, kb + 1);
                last_load = kb + 1;
            }
            store_a(ns);
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        }
        __syncthreads();
    }
    // the last commit tracks completion of every MMA issued before it
    if (tid == 0 && !failed && !mbar_wait(&bar_mma[(nkb - 1) & 1], ((nkb - 1) >> 1) & 1)) failed = 1;
    if (tid == 0 && failed) {  // drain what is still in flight, bounded
        if (last_commit >= 0) mbar_wait(&bar_mma[last_commit & 1], (last_commit >> 1) & 1);
        if (last_load >= 0) mbar_wait(&bar_b[last_load & 1], (last_load >> 1) & 1);
        atomicExch(err, 1);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!failed) {
        // warp w reads TMEM lanes 32w..32w+31: each thread one gathered column, N FP32 values
        const int col = warp * 32 + lane;
        float2* y = (col < ncol) ? Y + yo[col] + t.row0 : nullptr;
        for (int c0 = 0; c0 < N; c0 += 8) {
            uint32_t v[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (!y) continue;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int i = (c0 >> 1) + e;  // complex row within the tile
                if (i >= rows) break;
                const float2 val = make_float2(__uint_as_float(v[2 * e]), __uint_as_float(v[2 * e + 1]));
                if (mode == GEMM_SET) {
                    y[i] = val;
                } else if (mode == GEMM_ADD) {
                    const float2 o = y[i];
                    y[i] = make_float2(o.x + val.x, o.y + val.y);
                } else {
                    atomicAdd(&y[i].x, val.x);
                    atomicAdd(&y[i].y, val.y);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(256) : "memory");
}

void umma_init() {
    cudaFuncSetAttribute(umma_cgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, UGEMM_SMEM);
}

void launch_umma_cgemm(const UmmaProblem* probs, const UmmaTile* tiles, int ntiles, const long long* xoff,
                       const long long* yoff, const void* X, void* Y, int mode, int* err, cudaStream_t s) {
    if (ntiles == 0) return;
    umma_cgemm_kernel<<<ntiles, UTHREADS, UGEMM_SMEM, s>>>(probs, tiles, xoff, yoff, static_cast<const float2*>(X),
                                                          static_cast<float2*>(Y), mode, err);
}

}  // namespace ddfmm
