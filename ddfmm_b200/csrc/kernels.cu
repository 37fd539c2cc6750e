// Device kernels of the directional FMM eval (plain FP64 form).
//
// Every interaction evaluates the reference kernel (src/kernel3d.cpp:26-107):
//   G(r) = exp(2 pi i r) / r   (KERNEL_HELM)   or   exp(2 pi i r)  (KERNEL_EXPR)
// with r taken as 1 when r^2 < (1e-8)^2, which makes a coincident pair
// contribute exp(2 pi i) = 1 times the density (src/kernel3d.cpp:21,47-49).
// The phase is evaluated with sincospi(2r), i.e. without rounding 2*pi*r.
#include "kernels.cuh"

#include <cstdio>

namespace ddfmm {

__device__ __forceinline__ double2 kfun(double x, double y, double z, int kernel) {
    const double mindif2 = 1e-8 * 1e-8;
    double r2 = x * x + y * y + z * z;
    if (r2 < mindif2) r2 = 1.0;
    double r = sqrt(r2);
    double s, c;
    sincospi(2.0 * r, &s, &c);
    if (kernel == KERNEL_HELM) {
        double ir = 1.0 / r;
        return make_double2(c * ir, s * ir);
    }
    return make_double2(c, s);
}

__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

// ---------------------------------------------------------------- kmat
__global__ void kmat_kernel(const KmatJob* __restrict__ jobs, int njobs, long long total, int kernel) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {  // last job with elem0 <= e
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].elem0 <= e) lo = mid; else hi = mid - 1;
    }
    const KmatJob& J = jobs[lo];
    long long l = e - J.elem0;
    int i = (int)(l % J.m), j = (int)(l / J.m);
    double tx = J.trg[3 * i + 0] + J.ts[0], ty = J.trg[3 * i + 1] + J.ts[1], tz = J.trg[3 * i + 2] + J.ts[2];
    double sx = J.src[3 * j + 0] + J.ss[0], sy = J.src[3 * j + 1] + J.ss[1], sz = J.src[3 * j + 2] + J.ss[2];
    J.out[(size_t)j * J.m + i] = kfun(tx - sx, ty - sy, tz - sz, kernel);
}

void launch_kmat(const KmatJob* jobs, int njobs, long long total, int kernel, cudaStream_t s) {
    if (njobs == 0 || total == 0) return;
    long long blocks = (total + 255) / 256;
    kmat_kernel<<<(unsigned)blocks, 256, 0, s>>>(jobs, njobs, total, kernel);
}

// ---------------------------------------------------------------- gemm
// Grouped complex FP64 GEMM with gathered input columns and scattered output
// columns, on the FP64 tensor path (mma.sync m16n8k8 f64; the m8n8k4 and
// m16n8k16 shapes reach the same 37 TF/s on B200).  A 256-thread block
// computes up to 64 rows x 64 columns; warp (wm, wn) owns the 16-row slab wm
// (one 16-row MMA block) and columns wn*32 .. +32 (four 8-column blocks).  A
// complex block product takes three real MMAs (the three-multiplication form
// of a complex product, Gauss's trick):
//   P1 += Ar Br,  P2 += Ai Bi,  P3 += (Ar + Ai)(Br + Bi);
//   Cr = P1 - P2,  Ci = P3 - P1 - P2,
// the sums formed from the fragments in registers; 25% fewer MMAs than the
// four-product form at the same FP64 accuracy (outputs agree to ~3e-15).
// Slabs beyond the operator's rows are skipped (a tile carries
// ceil(rows / 16) active slabs), so an 80-150-row translation operator
// wastes at most 15 rows; so are 8-column blocks past the tile's columns and
// 8-wide K steps past k (warp-uniform), which the last, partial column tile of
// a problem and a k of 77-111 rounded up to the 16-wide K slice would
// otherwise spend on zeros.  K is consumed in slices of BK (16) through a
// GSTAGES-deep (3) cp.async pipeline; rows, columns and k beyond the problem are zero-filled
// by the copy (src-size 0).  128-bit shared loads are served in 8-lane
// phases (lanes with g in {2p, 2p+1}, tig 0..3); both fragment layouts put
// those 8 granules in 8 different bank groups: the operator slice is stored
// [k][row ^ 2*(k & 3)] and the column slice [col][k] with a BK + 4 granule stride
// (k = tig and tig + 4 of a fragment share k & 3, hence the same swizzle).
// Build-time variants (measured against each other): K slice DDFMM_ZGEMM_BK
// (16 or 32), ring depth DDFMM_ZGEMM_STAGES, blocks per SM DDFMM_ZGEMM_MINB.
#ifndef DDFMM_ZGEMM_BK
#define DDFMM_ZGEMM_BK 16
#endif
#ifndef DDFMM_ZGEMM_STAGES
#define DDFMM_ZGEMM_STAGES 3
#endif
#ifndef DDFMM_ZGEMM_MINB
#define DDFMM_ZGEMM_MINB 2
#endif
constexpr int BM = GEMM_TILE_M, BN = GEMM_TILE_N, BK = DDFMM_ZGEMM_BK, BKP = BK + 4, GSTAGES = DDFMM_ZGEMM_STAGES;
static_assert(BN * BK % 256 == 0, "whole column loads per thread");
static_assert(BK == 8 || BK == 16 || BK == 32, "K slice of 8, 16 or 32");
constexpr int GSTAGE = BK * BM + BN * BKP;  // double2 per stage
constexpr int GEMM_SMEM = GSTAGES * GSTAGE * (int)sizeof(double2);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// D (16 x 8) += A (16 x 8, rows g and g + 8 at k = tig and tig + 4) * B (8 x 8,
// k = tig and tig + 4 at column g); D element q: row g + 8 (q >> 1), column 2 tig + (q & 1)
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// D (8 x 8) += A (8 x 4, row g at k = tig) * B (4 x 8, k = tig at column g);
// D elements 0, 1: row g, columns 2 tig, 2 tig + 1 -- the first two elements
// of dmma16's D, at the same rows and columns
__device__ __forceinline__ void dmma8(double (&c)[4], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// One K slice of a warp's 16 x 8NJ block (NJ 8-column blocks), its first KS
// 8-wide K steps: the three real products cr = Ar Xr, ci = Ai Xi,
// cs = (Ar + Ai)(Xr + Xi) into the accumulators of blocks 0 .. NJ-1.  HALF:
// the slab holds at most 8 of the operator's rows, so each 16-row product is
// two 8-row m8n8k4 products over k = tig and tig + 4 (the same fragments'
// first rows), half the tensor work of the m16n8k8 form, rows g + 8 left zero.
template <int NJ, bool HALF>
__device__ __forceinline__ void zgemm_slice(const double2* As, const double2* Xs, int KS, double (&cr)[4][4],
                                            double (&ci)[4][4], double (&cs)[4][4]) {
#pragma unroll
    for (int ks = 0; ks < BK / 8; ++ks) {
        if (ks >= KS) break;
        // m16n8k8 fragments: A rows g, g+8 at k = tig, tig + 4; B k = tig, tig + 4 at column g
        double2 a[4], b[NJ][2];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (!HALF || (q & 1) == 0) a[q] = As[(ks * 8 + 4 * (q >> 1)) * BM + 8 * (q & 1)];
#pragma unroll
        for (int j = 0; j < NJ; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) b[j][h] = Xs[j * 8 * BKP + ks * 8 + 4 * h];
        if (HALF) {
            const double ar0 = a[0].x, ar2 = a[2].x, ai0 = a[0].y, ai2 = a[2].y;
            const double as0 = a[0].x + a[0].y, as2 = a[2].x + a[2].y;
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                dmma8(cr[j], ar0, b[j][0].x);
                dmma8(cr[j], ar2, b[j][1].x);
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                dmma8(ci[j], ai0, b[j][0].y);
                dmma8(ci[j], ai2, b[j][1].y);
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                dmma8(cs[j], as0, b[j][0].x + b[j][0].y);
                dmma8(cs[j], as2, b[j][1].x + b[j][1].y);
            }
        } else {
            double ar[4], ai[4], as[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ar[q] = a[q].x;
                ai[q] = a[q].y;
                as[q] = a[q].x + a[q].y;
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const double br[2] = {b[j][0].x, b[j][1].x};
                dmma16(cr[j], ar, br);
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const double bi[2] = {b[j][0].y, b[j][1].y};
                dmma16(ci[j], ai, bi);
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const double bs[2] = {b[j][0].x + b[j][0].y, b[j][1].x + b[j][1].y};
                dmma16(cs[j], as, bs);
            }
        }
    }
}

__global__ void __launch_bounds__(256, DDFMM_ZGEMM_MINB) zgemm_kernel(const GemmProblem* __restrict__ probs,
                                                       const GemmTile* __restrict__ tiles,
                                                       const long long* __restrict__ xoff,
                                                       const long long* __restrict__ yoff,
                                                       const double2* __restrict__ X, double2* Y, int mode) {
    extern __shared__ double2 gsm[];
    __shared__ long long xo[BN], yo[BN];
    const GemmTile t = tiles[blockIdx.x];
    const GemmProblem p = probs[t.prob];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int ncol = min(BN, p.ncol - t.col0);
    const int rows = min(BM, p.m - t.row0);
    const int nrow = ((rows + 15) >> 4) << 4;  // rows of the active slabs
    // warps over (slab, column group): 4 slabs x 2 groups of up to 32 columns; a
    // tile of 1 or 2 slabs (an operator's last rows) splits the columns into 8 or
    // 4 groups instead, and the groups share the tile's columns evenly (in
    // multiples of 8), so all 8 warps share its work when it has few columns too
    const int nslab = nrow >> 4;
    const int ngrp = min(BN / 8, nslab == 1 ? 8 : nslab == 2 ? 4 : 2);
    const int cpg = min(BN / ngrp, max(8, ((ncol + ngrp - 1) / ngrp + 7) / 8 * 8));  // columns per group
    const int wm = warp / ngrp, wn = warp % ngrp;
    const bool active = wm < nslab && wn * cpg < ncol;
    const int njb = min(cpg / 8, (ncol - wn * cpg + 7) >> 3);  // 8-column blocks of this warp holding columns
    const bool half = rows - wm * 16 <= 8;               // this warp's slab holds at most 8 operator rows
    if (tid < BN) {
        xo[tid] = tid < ncol ? xoff[p.col0 + t.col0 + tid] : 0;
        yo[tid] = tid < ncol ? yoff[p.col0 + t.col0 + tid] : 0;
    }
    __syncthreads();
    auto load = [&](int stage, int k0) {
        double2* As = gsm + stage * GSTAGE;
        double2* Xs = As + BK * BM;
        for (int e = tid; e < BK * nrow; e += 256) {
            int kk = e / nrow, row = e - kk * nrow;
            int gk = k0 + kk;
            bool ok = row < rows && gk < p.k;
            cp_async16(&As[kk * BM + (row ^ ((kk & 3) << 1))],
                       ok ? (const void*)(p.A + (size_t)gk * p.lda + t.row0 + row) : (const void*)p.A, ok ? 16 : 0);
        }
#pragma unroll
        for (int q = 0; q < BN * BK / 256; ++q) {
            int e = tid + 256 * q, kk = e % BK, col = e / BK;
            int gk = k0 + kk;
            bool ok = col < ncol && gk < p.k;
            cp_async16(&Xs[col * BKP + kk], ok ? (const void*)(X + xo[col] + gk) : (const void*)X, ok ? 16 : 0);
        }
    };
    // accumulators of the four 16x8 output blocks j: element q = 2h + e is row g + 8h, column 2 tig + e
    double cr[4][4], ci[4][4], cs[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) cr[j][q] = ci[j][q] = cs[j][q] = 0.0;
    const int nk = (p.k + BK - 1) / BK;
#pragma unroll
    for (int s = 0; s < GSTAGES - 1; ++s) {
        if (s < nk) load(s, s * BK);
        cp_async_commit();
    }
    for (int it = 0; it < nk; ++it) {
        cp_async_wait<GSTAGES - 2>();
        __syncthreads();
        {
            int nx = it + GSTAGES - 1;
            if (nx < nk) load(nx % GSTAGES, nx * BK);
            cp_async_commit();
        }
        if (active) {
            const double2* As = gsm + (it % GSTAGES) * GSTAGE + tig * BM + ((wm * 16 + g) ^ (tig << 1));
            const double2* Xs = gsm + (it % GSTAGES) * GSTAGE + BK * BM + (wn * cpg + g) * BKP + tig;
            const int KS = min(BK / 8, (p.k - it * BK + 7) >> 3);  // 8-wide K steps holding k
            if (half) {
                switch (njb) {
                    case 4: zgemm_slice<4, true>(As, Xs, KS, cr, ci, cs); break;
                    case 3: zgemm_slice<3, true>(As, Xs, KS, cr, ci, cs); break;
                    case 2: zgemm_slice<2, true>(As, Xs, KS, cr, ci, cs); break;
                    default: zgemm_slice<1, true>(As, Xs, KS, cr, ci, cs); break;
                }
            } else {
                switch (njb) {
                    case 4: zgemm_slice<4, false>(As, Xs, KS, cr, ci, cs); break;
                    case 3: zgemm_slice<3, false>(As, Xs, KS, cr, ci, cs); break;
                    case 2: zgemm_slice<2, false>(As, Xs, KS, cr, ci, cs); break;
                    default: zgemm_slice<1, false>(As, Xs, KS, cr, ci, cs); break;
                }
            }
        }
    }
    cp_async_wait<0>();
    if (!active) return;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            if (j * 8 >= cpg) break;  // the group's own 8-column blocks only
            int col = wn * cpg + j * 8 + 2 * tig + e;
            if (col >= ncol) continue;
            double2* y = Y + yo[col] + t.row0;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                int row = wm * 16 + i * 8 + g;
                if (row >= rows) continue;
                const int q = 2 * i + e;
                double2 v = make_double2(cr[j][q] - ci[j][q], cs[j][q] - cr[j][q] - ci[j][q]);
                if (mode == GEMM_SET) {
                    y[row] = v;
                } else if (mode == GEMM_ADD) {
                    double2 o = y[row];
                    o.x += v.x;
                    o.y += v.y;
                    y[row] = o;
                } else {
                    atomicAdd(&y[row].x, v.x);
                    atomicAdd(&y[row].y, v.y);
                }
            }
        }
}

void gemm_init() {
    cudaFuncSetAttribute(zgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM);
}

void launch_gemm(const GemmProblem* probs, const GemmTile* tiles, int ntiles, const long long* xoff,
                 const long long* yoff, const double2* X, double2* Y, int mode, cudaStream_t s) {
    if (ntiles == 0) return;
    zgemm_kernel<<<ntiles, 256, GEMM_SMEM, s>>>(probs, tiles, xoff, yoff, X, Y, mode);
}

// ---------------------------------------------------------------- points
// One warp per item; lanes over the item's target points.
// TPI consecutive threads per item, striding over its targets (TPI = 32: a
// warp per item, for items with many targets; 4 or 8 for leaf-sized ones).
template <int TPI>
__global__ void pt_kernel(const PtItem* __restrict__ items, int nitems, const PtSrc* __restrict__ srcs,
                          int kernel) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / TPI, lane = threadIdx.x % TPI;
    if (w >= nitems) return;
    const PtItem it = items[w];
    for (int t = lane; t < it.trg.n; t += TPI) {
        const double* tp = it.trg.x + 3 * t;
        double tx = it.trg.scale * tp[0] + it.trg.shift[0];
        double ty = it.trg.scale * tp[1] + it.trg.shift[1];
        double tz = it.trg.scale * tp[2] + it.trg.shift[2];
        double2 acc = make_double2(0.0, 0.0);
        for (int s = it.src_begin; s < it.src_end; ++s) {
            const PtSrc S = srcs[s];
            for (int q = 0; q < S.src.n; ++q) {
                const double* sp = S.src.x + 3 * q;
                double sx = S.src.scale * sp[0] + S.src.shift[0];
                double sy = S.src.scale * sp[1] + S.src.shift[1];
                double sz = S.src.scale * sp[2] + S.src.shift[2];
                cfma(acc, kfun(tx - sx, ty - sy, tz - sz, kernel), S.den[q]);
            }
        }
        double2 o = it.out[t];
        o.x += acc.x;
        o.y += acc.y;
        it.out[t] = o;
    }
}

// Warp-tiled point interactions (launch shapes PT_WARP_TARGETS / _SOURCES):
// one warp per item, its source points staged PTW_TILE at a time in shared
// memory (scaled and shifted once, not once per target), segment descriptors
// 32 at a time with their point counts prefix-summed across the warp.  MODE 0:
// lane = target (up to NT per lane), sources read by broadcast; MODE 1:
// NT targets per pass, lane = every 32nd source, per-target sums reduced
// with warp shuffles.
constexpr int PTW_WARPS = 8, PTW_TILE = 64;

template <int MODE, int NT>
__global__ void __launch_bounds__(32 * PTW_WARPS) ptw_kernel(const PtItem* __restrict__ items, int nitems,
                                                             const PtSrc* __restrict__ srcs, int kernel) {
    __shared__ double sx[PTW_WARPS][PTW_TILE], sy[PTW_WARPS][PTW_TILE], sz[PTW_WARPS][PTW_TILE];
    __shared__ double2 sd[PTW_WARPS][PTW_TILE];
    __shared__ PtSrc seg[PTW_WARPS][32];
    __shared__ int soff[PTW_WARPS][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * PTW_WARPS + warp;
    if (w >= nitems) return;  // whole warps only: the kernel syncs nothing wider than a warp
    const PtItem it = items[w];
    const PtSet& T = it.trg;
    constexpr int TCH = MODE == 0 ? 32 * NT : NT;  // targets per pass
    for (int t0 = 0; t0 < T.n; t0 += TCH) {
        double tx[NT], ty[NT], tz[NT];
        double2 acc[NT];
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
            acc[i] = make_double2(0.0, 0.0);
        }
        for (int sb = it.src_begin; sb < it.src_end; sb += 32) {
            const int nseg = min(32, it.src_end - sb);
            int n_i = 0;
            if (lane < nseg) {
                seg[warp][lane] = srcs[sb + lane];
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
                    sd[warp][p] = Q.den[q];
                }
                __syncwarp();
                if (MODE == 0) {
                    for (int p = 0; p < cnt; ++p) {
                        const double px = sx[warp][p], py = sy[warp][p], pz = sz[warp][p];
                        const double2 dv = sd[warp][p];
#pragma unroll
                        for (int i = 0; i < NT; ++i) cfma(acc[i], kfun(tx[i] - px, ty[i] - py, tz[i] - pz, kernel), dv);
                    }
                } else {
                    for (int p = lane; p < cnt; p += 32) {
                        const double px = sx[warp][p], py = sy[warp][p], pz = sz[warp][p];
                        const double2 dv = sd[warp][p];
#pragma unroll
                        for (int i = 0; i < NT; ++i)
                            if (t0 + i < T.n) cfma(acc[i], kfun(tx[i] - px, ty[i] - py, tz[i] - pz, kernel), dv);
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
                    double2 o = it.out[t];
                    o.x += acc[i].x;
                    o.y += acc[i].y;
                    it.out[t] = o;
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
                    double2 o = it.out[t0 + i];
                    o.x += acc[i].x;
                    o.y += acc[i].y;
                    it.out[t0 + i] = o;
                }
        }
    }
}

void launch_pt(const PtItem* items, int nitems, const PtSrc* srcs, int kernel, cudaStream_t s, int tpi) {
    if (nitems == 0) return;
    if (pt_warp_shape(tpi)) {
        const int blocks = (nitems + PTW_WARPS - 1) / PTW_WARPS;
        switch (tpi) {
            case PT_WARP_TARGETS: ptw_kernel<0, 4><<<blocks, 32 * PTW_WARPS, 0, s>>>(items, nitems, srcs, kernel); break;
            case PT_WARP_TARGETS2: ptw_kernel<0, 2><<<blocks, 32 * PTW_WARPS, 0, s>>>(items, nitems, srcs, kernel); break;
            case PT_WARP_SOURCES: ptw_kernel<1, 8><<<blocks, 32 * PTW_WARPS, 0, s>>>(items, nitems, srcs, kernel); break;
            default: ptw_kernel<1, 4><<<blocks, 32 * PTW_WARPS, 0, s>>>(items, nitems, srcs, kernel); break;
        }
        return;
    }
    const int blocks = (int)(((long long)nitems * tpi + 255) / 256);
    switch (tpi) {
        case 4: pt_kernel<4><<<blocks, 256, 0, s>>>(items, nitems, srcs, kernel); break;
        case 8: pt_kernel<8><<<blocks, 256, 0, s>>>(items, nitems, srcs, kernel); break;
        case 16: pt_kernel<16><<<blocks, 256, 0, s>>>(items, nitems, srcs, kernel); break;
        default: pt_kernel<32><<<blocks, 256, 0, s>>>(items, nitems, srcs, kernel); break;
    }
}

// ---------------------------------------------------------------- V list
// FFT-based M2L of the low-frequency V list (src/wave3d_eval.cpp:602-661).
// The reference scatters a box's equivalent density onto a G^3 grid (G = 2P)
// at the surface nodes of the P^3 corner cube [P, 2P)^3, FFTs it, multiplies
// by the FFT'd translation tensor of the box offset, inverse-FFTs and reads
// the check values back at the same corner-cube nodes.  Grid element
// (a, b, c) sits at a + G*(b + G*c) (CpxNumTns layout, include/numtns.hpp).
// Both transforms are pruned to the corner cube: the forward DFT only reads
// the P^3 cube (3 passes of G*P^2, G^2*P and G^3 outputs with P-term sums)
// and the inverse only produces it (G^2*P, G*P^2 and P^3 outputs with G-term
// sums), about a third of the work of full G^3 transforms.  Signs follow
// FFTW: forward exp(-2 pi i jk/G), backward exp(+2 pi i jk/G), unnormalised.

// Forward transform of one source box per block, in three passes of P-term
// sums (x, then y, then z), each thread taking whole lines: it loads the P
// inputs of its line once and produces the line's G outputs, the twiddle
// factors W[k][a] = exp(-2 pi i (P + a) k / G) read from shared memory.
template <int G>
__global__ void __launch_bounds__(vt_threads(G)) vlist_forward_kernel(VlistLevel L, const int* __restrict__ boxes,
                                                                      const double2* __restrict__ upeq,
                                                                      double2* __restrict__ spec,
                                                                      const double2* __restrict__ twf) {
    constexpr int P = G / 2, PP = P * P, G2 = G * G;
    extern __shared__ double2 vsm[];
    double2* W = vsm;               // W[k * P + a]
    double2* cube = W + G * P;      // [c'][b'][a']
    double2* b1 = cube + PP * P;    // [c'][b'][ka]
    double2* b2 = b1 + PP * G;      // [c'][kb][ka]
    const int tid = threadIdx.x, nt = blockDim.x;
    const int b = boxes[blockIdx.x];
    for (int e = tid; e < G * P; e += nt) W[e] = twf[((P + e % P) * (e / P)) % G];
    for (int e = tid; e < PP * P; e += nt) cube[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int k = tid; k < L.nE; k += nt) cube[L.cube_idx[k]] = upeq[(size_t)b * L.nE + k];
    __syncthreads();
    if (const int line = tid; line < PP) {  // x: line (c', b'); one line per thread, nt >= G^2
        double2 x[P];
#pragma unroll
        for (int a = 0; a < P; ++a) x[a] = cube[line * P + a];
#pragma unroll 1
        for (int k = 0; k < G; ++k) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int a = 0; a < P; ++a) cfma(acc, x[a], W[k * P + a]);
            b1[line * G + k] = acc;
        }
    }
    __syncthreads();
    if (const int e = tid; e < P * G) {  // y: line (c', ka)
        const int c = e / G, ka = e % G;
        double2 x[P];
#pragma unroll
        for (int bb = 0; bb < P; ++bb) x[bb] = b1[(c * P + bb) * G + ka];
#pragma unroll 1
        for (int k = 0; k < G; ++k) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int bb = 0; bb < P; ++bb) cfma(acc, x[bb], W[k * P + bb]);
            b2[(c * G + k) * G + ka] = acc;
        }
    }
    __syncthreads();
    double2* o = spec + (size_t)b * G2 * G;
    if (const int kab = tid; kab < G2) {  // z: line (ka, kb), the box's spectrum
        double2 x[P];
#pragma unroll
        for (int c = 0; c < P; ++c) x[c] = b2[c * G2 + kab];
#pragma unroll 1
        for (int k = 0; k < G; ++k) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < P; ++c) cfma(acc, x[c], W[k * P + c]);
            o[k * G2 + kab] = acc;
        }
    }
}

// The pointwise products of the V list, by target parent: warp w of a block
// takes target parent blockIdx.x * VGROUP_WARPS + w and lane l frequency
// 32 blockIdx.y + l of the G^3 grid, with one accumulator per child position.
// The loop over the parent's source entries is the same for the 32 lanes, so
// the child mask branches are warp-uniform; a source's spectrum value is
// loaded once and used by every child that has it in its V list.  Blocks of
// one frequency chunk run together (blockIdx.x varies fastest), so the
// translation tensors' 32-frequency slices of that chunk (316 x 512 bytes)
// stay in the SM's L1 while the chunk lasts, and the source spectra's slices
// (32 MB over all boxes at the bench workload) in L2.
__host__ __device__ constexpr int child_voff(int c) { return ((c >> 2) & 1) + 7 * ((c >> 1) & 1) + 49 * (c & 1); }

template <int G>
__global__ void __launch_bounds__(256) vlist_group_kernel(const int* __restrict__ gptr, const int2* __restrict__ gsrc,
                                                          const int* __restrict__ gtrg, int ngroups,
                                                          const double2* __restrict__ spec,
                                                          const double2* __restrict__ tns, double2* __restrict__ tsp) {
    constexpr int G3 = G * G * G;
    const int grp = blockIdx.x * VGROUP_WARPS + (threadIdx.x >> 5);
    if (grp >= ngroups) return;
    const int f = blockIdx.y * 32 + (threadIdx.x & 31);
    double2 acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = make_double2(0.0, 0.0);
    const int e1 = __ldg(gptr + grp + 1);
    for (int e = __ldg(gptr + grp); e < e1; ++e) {
        const int2 ent = __ldg(gsrc + e);
        const double2 S = __ldg(spec + (size_t)ent.x * G3 + f);
        const int mask = ent.y & 255;
        const double2* tb = tns + (size_t)(ent.y >> 8) * G3 + f;
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (mask & (1 << c)) cfma(acc[c], __ldg(tb + (size_t)child_voff(c) * G3), S);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int t = __ldg(gtrg + 8 * grp + c);
        if (t >= 0) tsp[(size_t)t * G3 + f] = acc[c];
    }
}

// Pruned inverse DFT of one target's summed spectrum per block: P outputs
// of G-term sums along z (each thread one (ka, kb) line, its G inputs read
// straight from the summed spectrum), then y, then x; the corner-cube nodes
// scaled by 1/G^3 are added into the target's check values.  Twiddles
// W[a][k] = exp(+2 pi i (P + a) k / G) from shared memory.
template <int G>
__global__ void __launch_bounds__(vt_threads(G)) vlist_inverse_kernel(VlistLevel L, const int* __restrict__ trg,
                                                                      const double2* __restrict__ tsp,
                                                                      double2* __restrict__ dnchk,
                                                                      const double2* __restrict__ twb) {
    constexpr int P = G / 2, PP = P * P, G2 = G * G, G3 = G2 * G;
    extern __shared__ double2 vsm[];
    double2* W = vsm;               // W[a * G + k]
    double2* c1 = W + P * G;        // [c'][kb][ka]
    double2* c2 = c1 + P * G2;      // [c'][b'][ka]
    double2* c3 = c2 + PP * G;      // [c'][b'][a']
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ti = blockIdx.x, t = trg[ti];
    for (int e = tid; e < P * G; e += nt) W[e] = twb[((P + e / G) * (e % G)) % G];
    __syncthreads();
    const double2* src = tsp + (size_t)ti * G3;
    if (const int kab = tid; kab < G2) {  // z
        double2 x[G];
#pragma unroll
        for (int k = 0; k < G; ++k) x[k] = __ldg(src + k * G2 + kab);
#pragma unroll 1
        for (int c = 0; c < P; ++c) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < G; ++k) cfma(acc, x[k], W[c * G + k]);
            c1[c * G2 + kab] = acc;
        }
    }
    __syncthreads();
    if (const int e = tid; e < P * G) {  // y: line (c', ka)
        const int c = e / G, ka = e % G;
        double2 x[G];
#pragma unroll
        for (int k = 0; k < G; ++k) x[k] = c1[(c * G + k) * G + ka];
#pragma unroll 1
        for (int bb = 0; bb < P; ++bb) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < G; ++k) cfma(acc, x[k], W[bb * G + k]);
            c2[(c * P + bb) * G + ka] = acc;
        }
    }
    __syncthreads();
    if (const int line = tid; line < PP) {  // x: line (c', b'); one line per thread, nt >= G^2
        double2 x[G];
#pragma unroll
        for (int k = 0; k < G; ++k) x[k] = c2[line * G + k];
#pragma unroll 1
        for (int a = 0; a < P; ++a) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < G; ++k) cfma(acc, x[k], W[a * G + k]);
            c3[line * P + a] = acc;
        }
    }
    __syncthreads();
    const double coef = 1.0 / (double)G3;
    for (int k = tid; k < L.nE; k += nt) {
        double2 v = c3[L.cube_idx[k]];
        double2 o = dnchk[(size_t)t * L.nE + k];
        o.x += v.x * coef;
        o.y += v.y * coef;
        dnchk[(size_t)t * L.nE + k] = o;
    }
}

size_t vt_smem(int G, size_t es) {
    const size_t P = G / 2;
    return es * (G * P + P * P * P + P * P * G + P * G * G);
}

void vlist_init(int) {
    cudaFuncSetAttribute(vlist_forward_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(8, 16));
    cudaFuncSetAttribute(vlist_forward_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(12, 16));
    cudaFuncSetAttribute(vlist_forward_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(16, 16));
    cudaFuncSetAttribute(vlist_inverse_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(8, 16));
    cudaFuncSetAttribute(vlist_inverse_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(12, 16));
    cudaFuncSetAttribute(vlist_inverse_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vt_smem(16, 16));
}

void launch_vlist_forward(const VlistLevel& L, const int* boxes, int nbox, const double2* upeq, double2* spec,
                          cudaStream_t s) {
    if (nbox == 0) return;
    const size_t sm = vt_smem(L.G, sizeof(double2));
    switch (L.G) {
        case 8: vlist_forward_kernel<8><<<nbox, vt_threads(8), sm, s>>>(L, boxes, upeq, spec, L.twf); break;
        case 12: vlist_forward_kernel<12><<<nbox, vt_threads(12), sm, s>>>(L, boxes, upeq, spec, L.twf); break;
        case 16: vlist_forward_kernel<16><<<nbox, vt_threads(16), sm, s>>>(L, boxes, upeq, spec, L.twf); break;
        default: break;
    }
}

void launch_vlist_group(const VlistLevel& L, const VlistGroups& V, const double2* spec, double2* tsp,
                        cudaStream_t s) {
    if (V.ngroups == 0) return;
    const dim3 grid((V.ngroups + VGROUP_WARPS - 1) / VGROUP_WARPS, L.G * L.G * L.G / 32);
    switch (L.G) {
        case 8: vlist_group_kernel<8><<<grid, 32 * VGROUP_WARPS, 0, s>>>(V.gptr, V.gsrc, V.gtrg, V.ngroups, spec, L.tns, tsp); break;
        case 12: vlist_group_kernel<12><<<grid, 32 * VGROUP_WARPS, 0, s>>>(V.gptr, V.gsrc, V.gtrg, V.ngroups, spec, L.tns, tsp); break;
        case 16: vlist_group_kernel<16><<<grid, 32 * VGROUP_WARPS, 0, s>>>(V.gptr, V.gsrc, V.gtrg, V.ngroups, spec, L.tns, tsp); break;
        default: break;
    }
}

void launch_vlist_inverse(const VlistLevel& L, const int* trg, int ntrg, const double2* tsp, double2* dnchk,
                          cudaStream_t s) {
    if (ntrg == 0) return;
    const size_t sm = vt_smem(L.G, sizeof(double2));
    switch (L.G) {
        case 8: vlist_inverse_kernel<8><<<ntrg, vt_threads(8), sm, s>>>(L, trg, tsp, dnchk, L.twb); break;
        case 12: vlist_inverse_kernel<12><<<ntrg, vt_threads(12), sm, s>>>(L, trg, tsp, dnchk, L.twb); break;
        case 16: vlist_inverse_kernel<16><<<ntrg, vt_threads(16), sm, s>>>(L, trg, tsp, dnchk, L.twb); break;
        default: break;
    }
}

// ---------------------------------------------------------------- misc
__global__ void gather_kernel(const double2* __restrict__ den, const int* __restrict__ perm,
                              double2* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = den[perm[i]];
}
__global__ void scatter_kernel(const double2* __restrict__ in, const int* __restrict__ perm,
                               double2* __restrict__ val, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) val[perm[i]] = in[i];
}
void launch_gather_den(const double2* den, const int* perm, double2* out, int n, cudaStream_t s) {
    if (n > 0) gather_kernel<<<(n + 255) / 256, 256, 0, s>>>(den, perm, out, n);
}
void launch_scatter_val(const double2* in, const int* perm, double2* val, int n, cudaStream_t s) {
    if (n > 0) scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(in, perm, val, n);
}

// Direct FP64 sum at check targets (the reference's Wave3d::check,
// src/wave3d_check.cpp:61-71): one block per target, all points as sources.
__global__ void direct_kernel(const double* __restrict__ pos, const double2* __restrict__ den, int n,
                              const int* __restrict__ chk, double2* __restrict__ out, int kernel) {
    __shared__ double2 red[256];
    const int t = chk[blockIdx.x];
    double tx = pos[3 * t], ty = pos[3 * t + 1], tz = pos[3 * t + 2];
    double2 acc = make_double2(0.0, 0.0);
    for (int s = threadIdx.x; s < n; s += blockDim.x)
        cfma(acc, kfun(tx - pos[3 * s], ty - pos[3 * s + 1], tz - pos[3 * s + 2], kernel), den[s]);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[threadIdx.x].x += red[threadIdx.x + w].x;
            red[threadIdx.x].y += red[threadIdx.x + w].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}
void launch_direct(const double* pos, const double2* den, int n, const int* chk, int nchk, double2* out,
                   int kernel, cudaStream_t s) {
    if (nchk > 0) direct_kernel<<<nchk, 256, 0, s>>>(pos, den, n, chk, out, kernel);
}

}  // namespace ddfmm
