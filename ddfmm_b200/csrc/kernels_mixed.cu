// Device kernels of the mixed-precision form: complex FP32 storage, FP32
// accumulation, translations on the tensor cores as 3xTF32 products.
//
// 3xTF32: a float x = hi + lo with hi = tf32(x), lo = tf32(x - hi); a product
// is hi*hi' + hi*lo' + lo*hi' (the lo*lo' term is below FP32 rounding), so
// three TF32 MMAs reproduce an FP32 product to about FP32 accuracy.
// Point interactions evaluate the reference kernel (src/kernel3d.cpp:26-107)
// in FP32 on coordinate differences formed in FP64 (|p_t - p_s| is then
// exact to FP32 and the phase 2 pi r stays accurate however far from the
// origin the leaf sits).
#include "kernels.cuh"

namespace ddfmm {

__device__ __forceinline__ float2 kfun32(double dx, double dy, double dz, int kernel) {
    float x = (float)dx, y = (float)dy, z = (float)dz;
    float r2 = x * x + y * y + z * z;
    if (r2 < 1e-16f) r2 = 1.0f;
    float r = sqrtf(r2);
    float s, c;
    sincospif(2.0f * r, &s, &c);
    if (kernel == KERNEL_HELM) {
        float ir = 1.0f / r;
        return make_float2(c * ir, s * ir);
    }
    return make_float2(c, s);
}

__device__ __forceinline__ void cfma32(float2& acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
}

// ---------------------------------------------------------------- 3xTF32 complex GEMM
// Same problem/tile/column conventions as zgemm_kernel (kernels.cuh), data in
// float2.  Block: 64 rows x 64 columns; warp (wm, wn) owns rows wm*32..+32 (two
// m16 blocks) and columns wn*16..+16 (two n8 blocks).  K slices of 32 through a
// 3-stage cp.async pipeline (8-byte copies: operator columns of odd length are
// only 8-byte aligned).  Operator slice stored [k][row ^ 4*(k & 3)], column
// slice [col][k] with a 36-element stride: both fragment loads are free of
// bank conflicts.
constexpr int CBM = 64, CBN = 64, CBK = 32, CBKP = 36, CSTAGES = 3;
constexpr int CSTAGE = CBK * CBM + CBN * CBKP;  // float2 per stage
constexpr int CGEMM_SMEM = CSTAGES * CSTAGE * (int)sizeof(float2);

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit32() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait32() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ unsigned tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split(float x, unsigned& hi, unsigned& lo) {
    hi = tf32(x);
    lo = tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(256, 2) cgemm_kernel(const GemmProblem* __restrict__ probs,
                                                       const GemmTile* __restrict__ tiles,
                                                       const long long* __restrict__ xoff,
                                                       const long long* __restrict__ yoff,
                                                       const float2* __restrict__ X, float2* Y, int mode) {
    extern __shared__ float2 csm[];
    __shared__ long long xo[CBN], yo[CBN];
    const GemmTile t = tiles[blockIdx.x];
    const GemmProblem p = probs[t.prob];
    const float2* A = reinterpret_cast<const float2*>(p.A);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3, wm = warp >> 2, wn = warp & 3;
    const int ncol = min(CBN, p.ncol - t.col0);
    const int rows = min(CBM, p.m - t.row0);
    const bool active = wm * 32 < rows && wn * 16 < ncol;
    if (tid < CBN) {
        xo[tid] = tid < ncol ? xoff[p.col0 + t.col0 + tid] : 0;
        yo[tid] = tid < ncol ? yoff[p.col0 + t.col0 + tid] : 0;
    }
    __syncthreads();
    auto load = [&](int stage, int k0) {
        float2* As = csm + stage * CSTAGE;
        float2* Xs = As + CBK * CBM;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            int e = tid + 256 * q, row = e & 63, kk = e >> 6;
            int gk = k0 + kk;
            bool ok = row < rows && gk < p.k;
            cp_async8(&As[kk * CBM + (row ^ ((kk & 3) << 2))],
                      ok ? (const void*)(A + (size_t)gk * p.lda + t.row0 + row) : (const void*)A, ok ? 8 : 0);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            int e = tid + 256 * q, kk = e & 31, col = e >> 5;
            int gk = k0 + kk;
            bool ok = col < ncol && gk < p.k;
            cp_async8(&Xs[col * CBKP + kk], ok ? (const void*)(X + xo[col] + gk) : (const void*)X, ok ? 8 : 0);
        }
    };
    float cr[2][2][4], ci[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) cr[i][j][e] = ci[i][j][e] = 0.f;
    const int nk = (p.k + CBK - 1) / CBK;
#pragma unroll
    for (int s = 0; s < CSTAGES - 1; ++s) {
        if (s < nk) load(s, s * CBK);
        cp_async_commit32();
    }
    for (int it = 0; it < nk; ++it) {
        cp_async_wait32<CSTAGES - 2>();
        __syncthreads();
        {
            int nx = it + CSTAGES - 1;
            if (nx < nk) load(nx % CSTAGES, nx * CBK);
            cp_async_commit32();
        }
        if (active) {
            const float2* As = csm + (it % CSTAGES) * CSTAGE;
            const float2* Xs = As + CBK * CBM;
#pragma unroll
            for (int ks = 0; ks < CBK / 8; ++ks) {
                // B fragments (8 x 8, col): b0 = X[col g][k tg], b1 = X[col g][k tg+4]
                unsigned brh[2][2], brl[2][2], bih[2][2], bil[2][2];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const float2* xp = Xs + (wn * 16 + j * 8 + g) * CBKP + ks * 8 + tg;
                    float2 b0 = xp[0], b1 = xp[4];
                    split(b0.x, brh[j][0], brl[j][0]);
                    split(b1.x, brh[j][1], brl[j][1]);
                    split(b0.y, bih[j][0], bil[j][0]);
                    split(b1.y, bih[j][1], bil[j][1]);
                }
                // A fragments (16 x 8, row): rows g, g+8; k tg, tg+4; split re / im / -im into hi, lo
                unsigned arh[2][4], arl[2][4], aih[2][4], ail[2][4], anh[2][4], anl[2][4];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int r = wm * 32 + i * 16 + g;
                    const int k = ks * 8 + tg;
                    const int sw = (k & 3) << 2;
                    float2 a[4] = {As[k * CBM + (r ^ sw)], As[k * CBM + ((r + 8) ^ sw)],
                                   As[(k + 4) * CBM + (r ^ sw)], As[(k + 4) * CBM + ((r + 8) ^ sw)]};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        split(a[e].x, arh[i][e], arl[i][e]);
                        split(a[e].y, aih[i][e], ail[i][e]);
                        anh[i][e] = aih[i][e] ^ 0x80000000u;  // -Ai
                        anl[i][e] = ail[i][e] ^ 0x80000000u;
                    }
                }
                // Cr += Ar Br - Ai Bi ; Ci += Ar Bi + Ai Br, each product as hi*hi + hi*lo + lo*hi;
                // every term runs over the four output blocks before the next one
#define DDFMM_TERM(ACC, AF, BF)                                                    \
    _Pragma("unroll") for (int i = 0; i < 2; ++i) _Pragma("unroll") for (int j = 0; j < 2; ++j) { \
        const unsigned bb[2] = {BF[j][0], BF[j][1]};                               \
        mma_tf32(ACC[i][j], AF[i], bb);                                            \
    }
                DDFMM_TERM(cr, arh, brh)
                DDFMM_TERM(ci, arh, bih)
                DDFMM_TERM(cr, anh, bih)
                DDFMM_TERM(ci, aih, brh)
                DDFMM_TERM(cr, arh, brl)
                DDFMM_TERM(ci, arh, bil)
                DDFMM_TERM(cr, anh, bil)
                DDFMM_TERM(ci, aih, brl)
                DDFMM_TERM(cr, arl, brh)
                DDFMM_TERM(ci, arl, bih)
                DDFMM_TERM(cr, anl, bih)
                DDFMM_TERM(ci, ail, brh)
#undef DDFMM_TERM
            }
        }
    }
    cp_async_wait32<0>();
    if (!active) return;
    // C fragment (16 x 8): c0 = C[g][2tg], c1 = C[g][2tg+1], c2 = C[g+8][2tg], c3 = C[g+8][2tg+1]
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                int row = wm * 32 + i * 16 + g + (e >> 1) * 8;
                int col = wn * 16 + j * 8 + 2 * tg + (e & 1);
                if (row >= rows || col >= ncol) continue;
                float2* y = Y + yo[col] + t.row0 + row;
                float2 v = make_float2(cr[i][j][e], ci[i][j][e]);
                if (mode == GEMM_SET) {
                    *y = v;
                } else if (mode == GEMM_ADD) {
                    float2 o = *y;
                    *y = make_float2(o.x + v.x, o.y + v.y);
                } else {
                    atomicAdd(&y->x, v.x);
                    atomicAdd(&y->y, v.y);
                }
            }
}

void cgemm_init() { cudaFuncSetAttribute(cgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CGEMM_SMEM); }

void launch_cgemm(const GemmProblem* probs, const GemmTile* tiles, int ntiles, const long long* xoff,
                  const long long* yoff, const void* X, void* Y, int mode, cudaStream_t s) {
    if (ntiles == 0) return;
    cgemm_kernel<<<ntiles, 256, CGEMM_SMEM, s>>>(probs, tiles, xoff, yoff, static_cast<const float2*>(X),
                                                  static_cast<float2*>(Y), mode);
}

// ---------------------------------------------------------------- points (FP32)
// ---------------------------------------------------------------- multi-instance launches
// Every mixed-form launch below walks a list of per-instance sub-launches
// (one entry for a single session, one per session for a batch): work item i
// of the launch belongs to sub-launch j with prefix[j] <= i < prefix[j+1], and
// is skipped when active != nullptr and active[sub.inst] == 0.
template <class T>
__device__ __forceinline__ int find_sub(const T* __restrict__ prefix, int nsub, T i) {
    int lo = 0, hi = nsub - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One warp per item as pt_kernel; densities / outputs are float2 (the
// descriptors' double2 pointers are reinterpreted).  Differences of the FP64
// coordinates are taken in FP64, the kernel is evaluated in FP32.
template <int TPI>
__global__ void pt32_kernel(const PtSub* __restrict__ subs, const int* __restrict__ prefix, int nsub, int nitems,
                            const int* __restrict__ active) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / TPI, lane = threadIdx.x % TPI;
    if (w >= nitems) return;
    const int j = find_sub(prefix, nsub, w);
    const PtSub S = subs[j];
    if (active && !active[S.inst]) return;
    const PtItem it = S.items[w - prefix[j]];
    float2* out = reinterpret_cast<float2*>(it.out);
    for (int t = lane; t < it.trg.n; t += TPI) {
        const double* tp = it.trg.x + 3 * t;
        double tx = it.trg.scale * tp[0] + it.trg.shift[0];
        double ty = it.trg.scale * tp[1] + it.trg.shift[1];
        double tz = it.trg.scale * tp[2] + it.trg.shift[2];
        float2 acc = make_float2(0.f, 0.f);
        for (int s = it.src_begin; s < it.src_end; ++s) {
            const PtSrc Q = S.srcs[s];
            const float2* den = reinterpret_cast<const float2*>(Q.den);
            for (int q = 0; q < Q.src.n; ++q) {
                const double* sp = Q.src.x + 3 * q;
                double sx = Q.src.scale * sp[0] + Q.src.shift[0];
                double sy = Q.src.scale * sp[1] + Q.src.shift[1];
                double sz = Q.src.scale * sp[2] + Q.src.shift[2];
                cfma32(acc, kfun32(tx - sx, ty - sy, tz - sz, S.kernel), den[q]);
            }
        }
        float2 o = out[t];
        out[t] = make_float2(o.x + acc.x, o.y + acc.y);
    }
}

// Warp-tiled point interactions: one warp per item.  The item's source points
// are staged in shared memory, PTW_TILE at a time, scaled and shifted once (in
// FP64, not once per target); every difference is taken in FP64 and rounded
// to FP32 before the kernel is evaluated, as in pt32_kernel, so |p_t - p_s|
// is accurate to FP32 however close the pair (a coincident pair gives exactly
// zero).  MODE 0: each lane owns up to NT targets (lane + 32 i) and walks
// the staged sources (broadcast reads); MODE 1: the targets go NT at a
// time, each lane takes every 32nd staged source and the per-target sums are
// reduced across the warp with shuffles.  Segment descriptors are read 32 at
// a time into shared memory; their point counts, prefix-summed across the
// warp, map a staged point to its segment.
constexpr int PTW_WARPS = 8, PTW_TILE = 64;

template <int MODE, int NT>
__global__ void __launch_bounds__(32 * PTW_WARPS) pt32w_kernel(const PtSub* __restrict__ subs,
                                                               const int* __restrict__ prefix, int nsub, int nitems,
                                                               const int* __restrict__ active) {
    __shared__ double sx[PTW_WARPS][PTW_TILE], sy[PTW_WARPS][PTW_TILE], sz[PTW_WARPS][PTW_TILE];
    __shared__ float2 sd[PTW_WARPS][PTW_TILE];
    __shared__ PtSrc seg[PTW_WARPS][32];
    __shared__ int soff[PTW_WARPS][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * PTW_WARPS + warp;
    if (w >= nitems) return;  // whole warps only: the kernel syncs nothing wider than a warp
    const int j = find_sub(prefix, nsub, w);
    const PtSub S = subs[j];
    if (active && !active[S.inst]) return;
    const PtItem it = S.items[w - prefix[j]];
    float2* out = reinterpret_cast<float2*>(it.out);
    const PtSet& T = it.trg;
    constexpr int TCH = MODE == 0 ? 32 * NT : NT;  // targets per pass
    for (int t0 = 0; t0 < T.n; t0 += TCH) {
        double tx[NT], ty[NT], tz[NT];
        float2 acc[NT];
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            const int t = MODE == 0 ? t0 + lane + 32 * i : t0 + i;
            tx[i] = ty[i] = tz[i] = 0.0;
            if (t < T.n) {
                const double* tp = T.x + 3 * t;
                tx[i] = T.scale * tp[0] + T.shift[0];
                ty[i] = T.scale * tp[1] + T.shift[1];
                tz[i] = T.scale * tp[2] + T.shift[2];
            }
            acc[i] = make_float2(0.f, 0.f);
        }
        for (int sb = it.src_begin; sb < it.src_end; sb += 32) {
            const int nseg = min(32, it.src_end - sb);
            int n_i = 0;
            if (lane < nseg) {
                seg[warp][lane] = S.srcs[sb + lane];
                n_i = seg[warp][lane].src.n;
            }
            int incl = n_i;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += y;
            }
            soff[warp][lane + 1] = incl;
            if (lane == 0) soff[warp][0] = 0;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            __syncwarp();
            for (int p0 = 0; p0 < total; p0 += PTW_TILE) {
                const int cnt = min(PTW_TILE, total - p0);
                for (int p = lane; p < cnt; p += 32) {
                    const int gp = p0 + p;
                    int lo = 0, hi = nseg - 1;  // the segment holding staged point gp
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (soff[warp][mid] <= gp)
                            lo = mid;
                        else
                            hi = mid - 1;
                    }
                    const PtSrc& Q = seg[warp][lo];
                    const int q = gp - soff[warp][lo];
                    const double* xp = Q.src.x + 3 * q;
                    sx[warp][p] = Q.src.scale * xp[0] + Q.src.shift[0];
                    sy[warp][p] = Q.src.scale * xp[1] + Q.src.shift[1];
                    sz[warp][p] = Q.src.scale * xp[2] + Q.src.shift[2];
                    sd[warp][p] = reinterpret_cast<const float2*>(Q.den)[q];
                }
                __syncwarp();
                if (MODE == 0) {
                    for (int p = 0; p < cnt; ++p) {
                        const double px = sx[warp][p], py = sy[warp][p], pz = sz[warp][p];
                        const float2 dv = sd[warp][p];
#pragma unroll
                        for (int i = 0; i < NT; ++i)
                            cfma32(acc[i], kfun32(tx[i] - px, ty[i] - py, tz[i] - pz, S.kernel), dv);
                    }
                } else {
                    for (int p = lane; p < cnt; p += 32) {
                        const double px = sx[warp][p], py = sy[warp][p], pz = sz[warp][p];
                        const float2 dv = sd[warp][p];
#pragma unroll
                        for (int i = 0; i < NT; ++i)
                            if (t0 + i < T.n) cfma32(acc[i], kfun32(tx[i] - px, ty[i] - py, tz[i] - pz, S.kernel), dv);
                    }
                }
                __syncwarp();
            }
        }
        if (MODE == 0) {
#pragma unroll
            for (int i = 0; i < NT; ++i) {
                const int t = t0 + lane + 32 * i;
                if (t < T.n) {
                    const float2 o = out[t];
                    out[t] = make_float2(o.x + acc[i].x, o.y + acc[i].y);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < NT; ++i) {
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) {
                    acc[i].x += __shfl_xor_sync(0xffffffffu, acc[i].x, d);
                    acc[i].y += __shfl_xor_sync(0xffffffffu, acc[i].y, d);
                }
            }
#pragma unroll
            for (int i = 0; i < NT; ++i)
                if (lane == i && t0 + i < T.n) {
                    const float2 o = out[t0 + i];
                    out[t0 + i] = make_float2(o.x + acc[i].x, o.y + acc[i].y);
                }
        }
    }
}

void launch_pt32(const PtSub* subs, const int* prefix, int nsub, int nitems, const int* active, cudaStream_t s,
                 int tpi) {
    if (nitems == 0) return;
    if (pt_warp_shape(tpi)) {
        const int blocks = (nitems + PTW_WARPS - 1) / PTW_WARPS;
        switch (tpi) {
            case PT_WARP_TARGETS: pt32w_kernel<0, 4><<<blocks, 32 * PTW_WARPS, 0, s>>>(subs, prefix, nsub, nitems, active); break;
            case PT_WARP_TARGETS2: pt32w_kernel<0, 2><<<blocks, 32 * PTW_WARPS, 0, s>>>(subs, prefix, nsub, nitems, active); break;
            case PT_WARP_SOURCES: pt32w_kernel<1, 8><<<blocks, 32 * PTW_WARPS, 0, s>>>(subs, prefix, nsub, nitems, active); break;
            default: pt32w_kernel<1, 4><<<blocks, 32 * PTW_WARPS, 0, s>>>(subs, prefix, nsub, nitems, active); break;
        }
        return;
    }
    const int blocks = (int)(((long long)nitems * tpi + 255) / 256);
    switch (tpi) {
        case 4: pt32_kernel<4><<<blocks, 256, 0, s>>>(subs, prefix, nsub, nitems, active); break;
        case 8: pt32_kernel<8><<<blocks, 256, 0, s>>>(subs, prefix, nsub, nitems, active); break;
        case 16: pt32_kernel<16><<<blocks, 256, 0, s>>>(subs, prefix, nsub, nitems, active); break;
        default: pt32_kernel<32><<<blocks, 256, 0, s>>>(subs, prefix, nsub, nitems, active); break;
    }
}

// ---------------------------------------------------------------- V list (FP32)
// The pruned corner-cube transforms of kernels.cu in complex FP32; one block
// per source box (forward) or target box (accumulate).  All sub-launches of a
// launch share G = 2P; spec_override, when set, replaces every sub-launch's
// spectra array (fixed-scratch entry point, single instance).
// MULTI = false: the single sub-launch `one` (kernel parameter space, as a
// one-instance launch); MULTI = true: the block's sub-launch from `subs`.
template <int G>
__device__ __forceinline__ void vlist_forward32_body(const VfSub& S, int local, float2* spec_override);

template <int G, bool MULTI>
__global__ void __launch_bounds__(vt_threads(G)) vlist_forward32_kernel(const VfSub one, const VfSub* __restrict__ subs,
                                                                        const int* __restrict__ prefix, int nsub,
                                                                        const int* __restrict__ active,
                                                                        float2* spec_override) {
    if (!MULTI) {
        if (active && !active[one.inst]) return;
        vlist_forward32_body<G>(one, blockIdx.x, spec_override);
        return;
    }
    __shared__ VfSub Sm;
    __shared__ int lm;
    if (threadIdx.x == 0) {
        const int j = find_sub(prefix, nsub, (int)blockIdx.x);
        Sm = subs[j];
        lm = blockIdx.x - prefix[j];
    }
    __syncthreads();
    if (active && !active[Sm.inst]) return;
    vlist_forward32_body<G>(Sm, lm, spec_override);
}

// The forward transform of kernels.cu (vlist_forward_kernel) in complex FP32.
template <int G>
__device__ __forceinline__ void vlist_forward32_body(const VfSub& S, int local, float2* spec_override) {
    constexpr int P = G / 2, PP = P * P, G2 = G * G;
    extern __shared__ float2 sm32[];
    float2* W = sm32;               // W[k * P + a]
    float2* cube = W + G * P;       // [c'][b'][a']
    float2* b1 = cube + PP * P;     // [c'][b'][ka]
    float2* b2 = b1 + PP * G;       // [c'][kb][ka]
    const VlistLevel& L = S.L;
    const float2* twf = reinterpret_cast<const float2*>(L.twf);
    const float2* upeq = S.upeq;
    float2* spec = spec_override ? spec_override : S.spec;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int b = S.boxes[local];
    for (int e = tid; e < G * P; e += nt) W[e] = twf[((P + e % P) * (e / P)) % G];
    for (int e = tid; e < PP * P; e += nt) cube[e] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int k = tid; k < L.nE; k += nt) cube[L.cube_idx[k]] = upeq[(size_t)b * L.nE + k];
    __syncthreads();
    if (const int line = tid; line < PP) {  // one line per thread: nt >= G^2
        float2 x[P];
#pragma unroll
        for (int a = 0; a < P; ++a) x[a] = cube[line * P + a];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int a = 0; a < P; ++a) cfma32(acc, x[a], W[k * P + a]);
            b1[line * G + k] = acc;
        }
    }
    __syncthreads();
    if (const int e = tid; e < P * G) {
        const int c = e / G, ka = e % G;
        float2 x[P];
#pragma unroll
        for (int bb = 0; bb < P; ++bb) x[bb] = b1[(c * P + bb) * G + ka];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int bb = 0; bb < P; ++bb) cfma32(acc, x[bb], W[k * P + bb]);
            b2[(c * G + k) * G + ka] = acc;
        }
    }
    __syncthreads();
    float2* o = spec + (size_t)b * G2 * G;
    if (const int kab = tid; kab < G2) {
        float2 x[P];
#pragma unroll
        for (int c = 0; c < P; ++c) x[c] = b2[c * G2 + kab];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < P; ++c) cfma32(acc, x[c], W[k * P + c]);
            o[k * G2 + kab] = acc;
        }
    }
}

// V-list sums by target parent (see vlist_group_kernel in kernels.cu): warp =
// one group (target parent), lane = one frequency of a 32-frequency chunk
// (blockIdx.y).  MULTI: each warp finds its own sub-launch from the prefix
// sums of the groups; spec_override replaces the source spectra (single
// instance).
__host__ __device__ constexpr int child_voff32(int c) { return ((c >> 2) & 1) + 7 * ((c >> 1) & 1) + 49 * (c & 1); }

template <int G, bool MULTI>
__global__ void __launch_bounds__(256) vlist_group32_kernel(const VaSub one, const VaSub* __restrict__ subs,
                                                            const int* __restrict__ prefix, int nsub, int ngroups,
                                                            const int* __restrict__ active,
                                                            const float2* spec_override) {
    constexpr int G3 = G * G * G;
    const int g = blockIdx.x * VGROUP_WARPS + (threadIdx.x >> 5);
    if (g >= ngroups) return;
    int j = 0, grp = g;
    if (MULTI) {
        j = find_sub(prefix, nsub, g);
        grp = g - __ldg(prefix + j);
    }
    const VaSub& S = MULTI ? subs[j] : one;
    if (active && !active[S.inst]) return;
    const float2* __restrict__ spec = spec_override ? spec_override : S.spec;
    const float2* __restrict__ tns = reinterpret_cast<const float2*>(S.L.tns);
    const int f = blockIdx.y * 32 + (threadIdx.x & 31);
    float2 acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = make_float2(0.f, 0.f);
    const int e1 = __ldg(S.gptr + grp + 1);
    for (int e = __ldg(S.gptr + grp); e < e1; ++e) {
        const int2 ent = __ldg(S.gsrc + e);
        const float2 sv = __ldg(spec + (size_t)ent.x * G3 + f);
        const int mask = ent.y & 255;
        const float2* tb = tns + (size_t)(ent.y >> 8) * G3 + f;
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (mask & (1 << c)) cfma32(acc[c], __ldg(tb + (size_t)child_voff32(c) * G3), sv);
    }
    float2* tsp = S.tsp;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int t = __ldg(S.gtrg + 8 * grp + c);
        if (t >= 0) tsp[(size_t)t * G3 + f] = acc[c];
    }
}

// The inverse transform of kernels.cu (vlist_inverse_kernel) in complex FP32,
// one block per target.
template <int G>
__device__ __forceinline__ void vlist_inverse32_body(const ViSub& S, int ti) {
    constexpr int P = G / 2, PP = P * P, G2 = G * G, G3 = G2 * G;
    extern __shared__ float2 sm32[];
    float2* W = sm32;               // W[a * G + k]
    float2* c1 = W + P * G;         // [c'][kb][ka]
    float2* c2 = c1 + P * G2;       // [c'][b'][ka]
    float2* c3 = c2 + PP * G;       // [c'][b'][a']
    const VlistLevel& L = S.L;
    const float2* twb = reinterpret_cast<const float2*>(L.twb);
    float2* dnchk = S.dnchk;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int t = S.trg[ti];
    for (int e = tid; e < P * G; e += nt) W[e] = twb[((P + e / G) * (e % G)) % G];
    __syncthreads();
    const float2* src = S.tsp + (size_t)ti * G3;
    if (const int kab = tid; kab < G2) {
        float2 x[G];
#pragma unroll
        for (int k = 0; k < G; ++k) x[k] = __ldg(src + k * G2 + kab);
#pragma unroll
        for (int c = 0; c < P; ++c) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < G; ++k) cfma32(acc, x[k], W[c * G + k]);
            c1[c * G2 + kab] = acc;
        }
    }
    __syncthreads();
    if (const int e = tid; e < P * G) {
        const int c = e / G, ka = e % G;
        float2 x[G];
#pragma unroll
        for (int k = 0; k < G; ++k) x[k] = c1[(c * G + k) * G + ka];
#pragma unroll
        for (int bb = 0; bb < P; ++bb) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < G; ++k) cfma32(acc, x[k], W[bb * G + k]);
            c2[(c * P + bb) * G + ka] = acc;
        }
    }
    __syncthreads();
    if (const int line = tid; line < PP) {  // one line per thread: nt >= G^2
        float2 x[G];
#pragma unroll
        for (int k = 0; k < G; ++k) x[k] = c2[line * G + k];
#pragma unroll
        for (int a = 0; a < P; ++a) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < G; ++k) cfma32(acc, x[k], W[a * G + k]);
            c3[line * P + a] = acc;
        }
    }
    __syncthreads();
    const float coef = 1.0f / (float)G3;
    for (int k = tid; k < L.nE; k += nt) {
        float2 v = c3[L.cube_idx[k]];
        float2 o = dnchk[(size_t)t * L.nE + k];
        dnchk[(size_t)t * L.nE + k] = make_float2(o.x + v.x * coef, o.y + v.y * coef);
    }
}

template <int G, bool MULTI>
__global__ void __launch_bounds__(vt_threads(G)) vlist_inverse32_kernel(const ViSub one, const ViSub* __restrict__ subs,
                                                              const int* __restrict__ prefix, int nsub,
                                                              const int* __restrict__ active) {
    if (!MULTI) {
        if (active && !active[one.inst]) return;
        vlist_inverse32_body<G>(one, blockIdx.x);
        return;
    }
    __shared__ ViSub Sm;
    __shared__ int lm;
    if (threadIdx.x == 0) {
        const int j = find_sub(prefix, nsub, (int)blockIdx.x);
        Sm = subs[j];
        lm = blockIdx.x - prefix[j];
    }
    __syncthreads();
    if (active && !active[Sm.inst]) return;
    vlist_inverse32_body<G>(Sm, lm);
}

void vlist32_init(int) {
#define DDFMM_VT_ATTR(k, g)                                                                      \
    cudaFuncSetAttribute(k<g, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(g, 8)); \
    cudaFuncSetAttribute(k<g, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(g, 8));
    DDFMM_VT_ATTR(vlist_forward32_kernel, 8)
    DDFMM_VT_ATTR(vlist_forward32_kernel, 12)
    DDFMM_VT_ATTR(vlist_forward32_kernel, 16)
    DDFMM_VT_ATTR(vlist_inverse32_kernel, 8)
    DDFMM_VT_ATTR(vlist_inverse32_kernel, 12)
    DDFMM_VT_ATTR(vlist_inverse32_kernel, 16)
#undef DDFMM_VT_ATTR
}

// L.tns, L.twf, L.twb hold float2 data in this form.
void launch_vlist_forward32(const VfSub* subs, const int* prefix, int nsub, int nbox, int G, const int* active,
                            void* spec_override, cudaStream_t s, const VfSub* one) {
    if (nbox == 0) return;
    VfSub o{};
    if (nsub == 1) {
        if (!one) return;  // a single sub-launch is passed by value
        o = *one;
    }
    const size_t sm = vt_smem(G, sizeof(float2));
    float2* so = static_cast<float2*>(spec_override);
#define DDFMM_VFWD(g)                                                                                   \
    if (nsub == 1)                                                                                      \
        vlist_forward32_kernel<g, false><<<nbox, vt_threads(g), sm, s>>>(o, subs, prefix, nsub, active, so); \
    else                                                                                                \
        vlist_forward32_kernel<g, true><<<nbox, vt_threads(g), sm, s>>>(o, subs, prefix, nsub, active, so);
    switch (G) {
        case 8: DDFMM_VFWD(8) break;
        case 12: DDFMM_VFWD(12) break;
        case 16: DDFMM_VFWD(16) break;
        default: break;
    }
#undef DDFMM_VFWD
}

void launch_vlist_group32(const VaSub* subs, const int* prefix, int nsub, int ngroups, int G, const int* active,
                          const void* spec_override, cudaStream_t s, const VaSub* one) {
    if (ngroups == 0) return;
    VaSub o{};
    if (nsub == 1) {
        if (!one) return;  // a single sub-launch is passed by value
        o = *one;
    }
    const float2* so = static_cast<const float2*>(spec_override);
    const dim3 grid((ngroups + VGROUP_WARPS - 1) / VGROUP_WARPS, G * G * G / 32);
#define DDFMM_VGRP(g)                                                                                             \
    if (nsub == 1)                                                                                                \
        vlist_group32_kernel<g, false><<<grid, 32 * VGROUP_WARPS, 0, s>>>(o, subs, prefix, nsub, ngroups, active, so); \
    else                                                                                                          \
        vlist_group32_kernel<g, true><<<grid, 32 * VGROUP_WARPS, 0, s>>>(o, subs, prefix, nsub, ngroups, active, so);
    switch (G) {
        case 8: DDFMM_VGRP(8) break;
        case 12: DDFMM_VGRP(12) break;
        case 16: DDFMM_VGRP(16) break;
        default: break;
    }
#undef DDFMM_VGRP
}

void launch_vlist_inverse32(const ViSub* subs, const int* prefix, int nsub, int ntrg, int G, const int* active,
                            cudaStream_t s, const ViSub* one) {
    if (ntrg == 0) return;
    ViSub o{};
    if (nsub == 1) {
        if (!one) return;  // a single sub-launch is passed by value
        o = *one;
    }
    const size_t sm = vt_smem(G, sizeof(float2));
#define DDFMM_VINV(g)                                                                                   \
    if (nsub == 1)                                                                                      \
        vlist_inverse32_kernel<g, false><<<ntrg, vt_threads(g), sm, s>>>(o, subs, prefix, nsub, active); \
    else                                                                                                \
        vlist_inverse32_kernel<g, true><<<ntrg, vt_threads(g), sm, s>>>(o, subs, prefix, nsub, active);
    switch (G) {
        case 8: DDFMM_VINV(8) break;
        case 12: DDFMM_VINV(12) break;
        case 16: DDFMM_VINV(16) break;
        default: break;
    }
#undef DDFMM_VINV
}

// Batch I/O: complex64 densities in point-id order into leaf order (gather),
// leaf-order values back to point-id order (scatter); one thread per point.
__global__ void move32_kernel(const MoveSub* __restrict__ subs, const int* __restrict__ prefix, int nsub, int n,
                              const int* __restrict__ active, int scatter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = find_sub(prefix, nsub, i);
    const MoveSub S = subs[j];
    if (active && !active[S.inst]) return;
    const int l = i - prefix[j];
    const float2* in = static_cast<const float2*>(S.in);
    float2* out = static_cast<float2*>(S.out);
    if (scatter)
        out[S.perm[l]] = in[l];
    else
        out[l] = in[S.perm[l]];
}
void launch_move32(const MoveSub* subs, const int* prefix, int nsub, int n, const int* active, int scatter,
                   cudaStream_t s) {
    if (n > 0) move32_kernel<<<(n + 255) / 256, 256, 0, s>>>(subs, prefix, nsub, n, active, scatter);
}

// Zeroing of several instances' arrays, 8-byte words.
__global__ void zero_kernel(const ZeroSub* __restrict__ subs, const long long* __restrict__ prefix, int nsub,
                            long long n, const int* __restrict__ active) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int j = find_sub(prefix, nsub, i);
        const ZeroSub S = subs[j];
        if (active && !active[S.inst]) continue;
        static_cast<unsigned long long*>(S.p)[i - prefix[j]] = 0ull;
    }
}
void launch_zero(const ZeroSub* subs, const long long* prefix, int nsub, long long n8, const int* active,
                 cudaStream_t s) {
    if (n8 <= 0) return;
    long long blocks = (n8 + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    zero_kernel<<<(unsigned)blocks, 256, 0, s>>>(subs, prefix, nsub, n8, active);
}

// ---------------------------------------------------------------- conversions
__global__ void gather32_kernel(const double2* __restrict__ den, const int* __restrict__ perm,
                                float2* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double2 v = den[perm[i]];
        out[i] = make_float2((float)v.x, (float)v.y);
    }
}
__global__ void gather32c_kernel(const float2* __restrict__ den, const int* __restrict__ perm,
                                 float2* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = den[perm[i]];
}
__global__ void scatter32_kernel(const float2* __restrict__ in, const int* __restrict__ perm,
                                 double2* __restrict__ val, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        float2 v = in[i];
        val[perm[i]] = make_double2(v.x, v.y);
    }
}
__global__ void scatter32c_kernel(const float2* __restrict__ in, const int* __restrict__ perm,
                                  float2* __restrict__ val, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) val[perm[i]] = in[i];
}
// den / val are complex128 (c64 = 0) or complex64 (c64 = 1) arrays in point-id order
void launch_gather32(const void* den, const int* perm, void* out, int n, int c64, cudaStream_t s) {
    if (n <= 0) return;
    if (c64)
        gather32c_kernel<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const float2*>(den), perm,
                                                         static_cast<float2*>(out), n);
    else
        gather32_kernel<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const double2*>(den), perm,
                                                        static_cast<float2*>(out), n);
}
void launch_scatter32(const void* in, const int* perm, void* val, int n, int c64, cudaStream_t s) {
    if (n <= 0) return;
    if (c64)
        scatter32c_kernel<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const float2*>(in), perm,
                                                          static_cast<float2*>(val), n);
    else
        scatter32_kernel<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const float2*>(in), perm,
                                                         static_cast<double2*>(val), n);
}

__global__ void to_c64_kernel(const double2* __restrict__ a, float2* __restrict__ b, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
void launch_to_c64(const double2* a, float2* b, long long n, cudaStream_t s) {
    if (n > 0) to_c64_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
}

}  // namespace ddfmm
