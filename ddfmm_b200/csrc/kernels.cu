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
// columns.  A 256-thread block computes up to 64 rows x 64 columns: thread
// (tx, ty) owns rows tx + 16*i (i < MT) and columns ty + 16*j (j < 4), so
// consecutive lanes write consecutive rows of one output vector.  MT =
// ceil(tile rows / 16) is a compile-time specialisation chosen per tile, so
// an 80-150-row translation operator wastes at most 15 rows and the inner
// loop carries no guards.  K is consumed in slices of 16 through a 3-stage
// cp.async pipeline; rows, columns and k beyond the problem are zero-filled
// by the copy (src-size 0).
constexpr int BM = 64, BN = 64, BK = 16, GSTAGES = 3;
constexpr int GEMM_SMEM = GSTAGES * (BK * BM + BK * BN) * (int)sizeof(double2);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int MT>
__device__ __forceinline__ void zgemm_tile(const GemmProblem& p, const GemmTile& t, int ncol, int rows,
                                           const long long* xo, const long long* yo, const double2* __restrict__ X,
                                           double2* Y, int mode, double2* gsm) {
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    auto load = [&](int stage, int k0) {
        double2* As = gsm + stage * (BK * (BM + BN));
        double2* Xs = As + BK * BM;
#pragma unroll
        for (int q = 0; q < MT; ++q) {  // BK x (16*MT) elements of A, MT per thread
            int e = tid + 256 * q, row = e % (16 * MT), kk = e / (16 * MT);
            int gk = k0 + kk;
            bool ok = row < rows && gk < p.k;
            cp_async16(&As[kk * BM + row], ok ? (const void*)(p.A + (size_t)gk * p.lda + t.row0 + row) : (const void*)p.A,
                       ok ? 16 : 0);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int e = tid + 256 * q, kk = e & 15, col = e >> 4;
            int gk = k0 + kk;
            bool ok = col < ncol && gk < p.k;
            cp_async16(&Xs[col * BK + kk], ok ? (const void*)(X + xo[col] + gk) : (const void*)X, ok ? 16 : 0);
        }
    };
    double2 acc[MT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
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
        const double2* As = gsm + (it % GSTAGES) * (BK * (BM + BN));
        const double2* Xs = As + BK * BM;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double2 a[MT], x[4];
#pragma unroll
            for (int i = 0; i < MT; ++i) a[i] = As[kk * BM + tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) x[j] = Xs[(ty + 16 * j) * BK + kk];
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) cfma(acc[i][j], a[i], x[j]);
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int col = ty + 16 * j;
        if (col >= ncol) continue;
        double2* y = Y + yo[col] + t.row0;
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            int row = tx + 16 * i;
            if (row >= rows) continue;
            if (mode == GEMM_SET) {
                y[row] = acc[i][j];
            } else if (mode == GEMM_ADD) {
                double2 v = y[row];
                v.x += acc[i][j].x;
                v.y += acc[i][j].y;
                y[row] = v;
            } else {
                atomicAdd(&y[row].x, acc[i][j].x);
                atomicAdd(&y[row].y, acc[i][j].y);
            }
        }
    }
}

__global__ void __launch_bounds__(256, 2) zgemm_kernel(const GemmProblem* __restrict__ probs,
                                                       const GemmTile* __restrict__ tiles,
                                                       const long long* __restrict__ xoff,
                                                       const long long* __restrict__ yoff,
                                                       const double2* __restrict__ X, double2* Y, int mode) {
    extern __shared__ double2 gsm[];
    __shared__ long long xo[BN], yo[BN];
    const GemmTile t = tiles[blockIdx.x];
    const GemmProblem p = probs[t.prob];
    const int tid = threadIdx.x;
    const int ncol = min(BN, p.ncol - t.col0);
    const int rows = min(BM, p.m - t.row0);
    if (tid < BN) {
        xo[tid] = tid < ncol ? xoff[p.col0 + t.col0 + tid] : 0;
        yo[tid] = tid < ncol ? yoff[p.col0 + t.col0 + tid] : 0;
    }
    __syncthreads();
    switch ((rows + 15) >> 4) {
        case 1: zgemm_tile<1>(p, t, ncol, rows, xo, yo, X, Y, mode, gsm); break;
        case 2: zgemm_tile<2>(p, t, ncol, rows, xo, yo, X, Y, mode, gsm); break;
        case 3: zgemm_tile<3>(p, t, ncol, rows, xo, yo, X, Y, mode, gsm); break;
        default: zgemm_tile<4>(p, t, ncol, rows, xo, yo, X, Y, mode, gsm); break;
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
__global__ void pt_kernel(const PtItem* __restrict__ items, int nitems, const PtSrc* __restrict__ srcs,
                          int kernel) {
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nitems) return;
    const PtItem it = items[w];
    for (int t = lane; t < it.trg.n; t += 32) {
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

void launch_pt(const PtItem* items, int nitems, const PtSrc* srcs, int kernel, cudaStream_t s) {
    if (nitems == 0) return;
    int blocks = (nitems * 32 + 255) / 256;
    pt_kernel<<<blocks, 256, 0, s>>>(items, nitems, srcs, kernel);
}

// ---------------------------------------------------------------- V list
// Separable DFT of a G^3 grid held in shared memory, element (a,b,c) at
// a + G*(b + G*c) as in the reference's CpxNumTns (include/numtns.hpp:104-117).
// sign -1 is FFTW_FORWARD, +1 FFTW_BACKWARD (unnormalised).
__device__ void dft3_smem(double2* g, int G, const double2* __restrict__ tw, int nthreads) {
    const int tot = G * G * G;
    const int stride[3] = {1, G, G * G};
    for (int ax = 0; ax < 3; ++ax) {
        const int st = stride[ax];
        double2 out[16];
        int cnt = 0;
        for (int e = threadIdx.x; e < tot; e += nthreads, ++cnt) {
            int k = (e / st) % G;
            int base = e - k * st;
            double2 acc = make_double2(0.0, 0.0);
            for (int j = 0; j < G; ++j) cfma(acc, g[base + j * st], tw[(j * k) % G]);
            out[cnt] = acc;
        }
        __syncthreads();
        cnt = 0;
        for (int e = threadIdx.x; e < tot; e += nthreads, ++cnt) g[e] = out[cnt];
        __syncthreads();
    }
}

__global__ void vlist_forward_kernel(VlistLevel L, const int* __restrict__ boxes,
                                     const double2* __restrict__ upeq, double2* __restrict__ spec,
                                     const double2* __restrict__ twf) {
    extern __shared__ double2 grid[];
    const int G = L.G, tot = G * G * G;
    const int b = boxes[blockIdx.x];
    for (int e = threadIdx.x; e < tot; e += blockDim.x) grid[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int k = threadIdx.x; k < L.nE; k += blockDim.x) grid[L.grid_idx[k]] = upeq[(size_t)b * L.nE + k];
    __syncthreads();
    dft3_smem(grid, G, twf, blockDim.x);
    double2* o = spec + (size_t)b * tot;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) o[e] = grid[e];
}

__global__ void vlist_accum_kernel(VlistLevel L, const int* __restrict__ trg, const int* __restrict__ vptr,
                                   const int* __restrict__ vsrc, const int* __restrict__ voff,
                                   const double2* __restrict__ spec, double2* __restrict__ dnchk,
                                   const double2* __restrict__ twb) {
    extern __shared__ double2 grid[];
    const int G = L.G, tot = G * G * G;
    const int ti = blockIdx.x, t = trg[ti];
    double2 acc[16];
    int cnt = 0;
    for (int e = threadIdx.x; e < tot; e += blockDim.x, ++cnt) acc[cnt] = make_double2(0.0, 0.0);
    for (int v = vptr[ti]; v < vptr[ti + 1]; ++v) {
        const double2* sp = spec + (size_t)vsrc[v] * tot;
        const double2* tn = L.tns + (size_t)voff[v] * tot;
        cnt = 0;
        for (int e = threadIdx.x; e < tot; e += blockDim.x, ++cnt) cfma(acc[cnt], sp[e], tn[e]);
    }
    cnt = 0;
    for (int e = threadIdx.x; e < tot; e += blockDim.x, ++cnt) grid[e] = acc[cnt];
    __syncthreads();
    dft3_smem(grid, G, twb, blockDim.x);
    const double coef = 1.0 / (double)(G * G * G);
    for (int k = threadIdx.x; k < L.nE; k += blockDim.x) {
        double2 v = grid[L.grid_idx[k]];
        double2 o = dnchk[(size_t)t * L.nE + k];
        o.x += v.x * coef;
        o.y += v.y * coef;
        dnchk[(size_t)t * L.nE + k] = o;
    }
}

void vlist_init(int G) {
    int sm = (int)(sizeof(double2) * G * G * G);
    cudaFuncSetAttribute(vlist_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(vlist_accum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

static int vlist_threads(int G) { return G * G * G / 16 > 256 ? G * G * G / 16 : 256; }

void launch_vlist_forward(const VlistLevel& L, const int* boxes, int nbox, const double2* upeq, double2* spec,
                          cudaStream_t s) {
    if (nbox == 0) return;
    size_t sm = sizeof(double2) * L.G * L.G * L.G;
    vlist_forward_kernel<<<nbox, vlist_threads(L.G), sm, s>>>(L, boxes, upeq, spec, L.twf);
}

void launch_vlist_accum(const VlistLevel& L, const int* trg, int ntrg, const int* vptr, const int* vsrc,
                        const int* voff, const double2* spec, double2* dnchk, cudaStream_t s) {
    if (ntrg == 0) return;
    size_t sm = sizeof(double2) * L.G * L.G * L.G;
    vlist_accum_kernel<<<ntrg, vlist_threads(L.G), sm, s>>>(L, trg, vptr, vsrc, voff, spec, dnchk, L.twb);
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
