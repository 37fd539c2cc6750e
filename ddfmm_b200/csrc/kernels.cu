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
// columns, on the FP64 tensor path (mma.sync m8n8k4 f64).  A 256-thread block
// computes up to 64 rows x 64 columns; warp (wm, wn) owns the 16-row slab wm
// (two 8-row MMA blocks) and columns wn*32 .. +32 (four 8-column blocks).  A
// complex block product takes three real MMAs (the three-multiplication form
// of a complex product, Gauss's trick):
//   P1 += Ar Br,  P2 += Ai Bi,  P3 += (Ar + Ai)(Br + Bi);
//   Cr = P1 - P2,  Ci = P3 - P1 - P2,
// the sums formed from the fragments in registers; 25% fewer MMAs than the
// four-product form at the same FP64 accuracy (outputs agree to ~3e-15).
// Slabs beyond the operator's rows are skipped (a tile carries
// ceil(rows / 16) active slabs), so an 80-150-row translation operator
// wastes at most 15 rows.  K is consumed in slices of 16 through a 3-stage
// cp.async pipeline; rows, columns and k beyond the problem are zero-filled
// by the copy (src-size 0).  128-bit shared loads are served in 8-lane
// phases (lanes with g in {2p, 2p+1}, tig 0..3); both fragment layouts put
// those 8 granules in 8 different bank groups: the operator slice is stored
// [k][row ^ 2*(k & 3)] and the column slice [col][k] with a 20-granule stride.
constexpr int BM = 64, BN = 64, BK = 16, BKP = 20, GSTAGES = 3;
constexpr int GSTAGE = BK * BM + BN * BKP;  // double2 per stage
constexpr int GEMM_SMEM = GSTAGES * GSTAGE * (int)sizeof(double2);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
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
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3, wm = warp >> 1, wn = warp & 1;
    const int ncol = min(BN, p.ncol - t.col0);
    const int rows = min(BM, p.m - t.row0);
    const int nrow = ((rows + 15) >> 4) << 4;  // rows of the active slabs
    const bool active = wm * 16 < rows;
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
        for (int q = 0; q < 4; ++q) {
            int e = tid + 256 * q, kk = e & 15, col = e >> 4;
            int gk = k0 + kk;
            bool ok = col < ncol && gk < p.k;
            cp_async16(&Xs[col * BKP + kk], ok ? (const void*)(X + xo[col] + gk) : (const void*)X, ok ? 16 : 0);
        }
    };
    double cr[2][4][2], ci[2][4][2], cs[2][4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = cs[i][j][0] = cs[i][j][1] = 0.0;
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
            const double2* Xs = gsm + (it % GSTAGES) * GSTAGE + BK * BM + (wn * 32 + g) * BKP + tig;
#pragma unroll
            for (int ks = 0; ks < BK / 4; ++ks) {
                double2 a[2], b[4];
#pragma unroll
                for (int i = 0; i < 2; ++i) a[i] = As[ks * 4 * BM + i * 8];
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = Xs[j * 8 * BKP + ks * 4];
                // three real products: cr = ArXr, ci = AiXi, cs = (Ar+Ai)(Xr+Xi)
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma(cr[i][j], a[i].x, b[j].x);
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma(ci[i][j], a[i].y, b[j].y);
                double as[2], bs[4];
#pragma unroll
                for (int i = 0; i < 2; ++i) as[i] = a[i].x + a[i].y;
#pragma unroll
                for (int j = 0; j < 4; ++j) bs[j] = b[j].x + b[j].y;
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma(cs[i][j], as[i], bs[j]);
            }
        }
    }
    cp_async_wait<0>();
    if (!active) return;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            int col = wn * 32 + j * 8 + 2 * tig + e;
            if (col >= ncol) continue;
            double2* y = Y + yo[col] + t.row0;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                int row = wm * 16 + i * 8 + g;
                if (row >= rows) continue;
                double2 v = make_double2(cr[i][j][e] - ci[i][j][e], cs[i][j][e] - cr[i][j][e] - ci[i][j][e]);
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

void launch_pt(const PtItem* items, int nitems, const PtSrc* srcs, int kernel, cudaStream_t s, int tpi) {
    if (nitems == 0) return;
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

__global__ void vlist_forward_kernel(VlistLevel L, const int* __restrict__ boxes,
                                     const double2* __restrict__ upeq, double2* __restrict__ spec,
                                     const double2* __restrict__ twf) {
    extern __shared__ double2 sm[];
    const int G = L.G, P = L.P, PP = P * P;
    double2* cube = sm;             // [c'][b'][a'], a', b', c' < P
    double2* b1 = cube + PP * P;    // [c'][b'][ka]
    double2* b2 = b1 + G * PP;      // [c'][kb][ka]
    const int b = boxes[blockIdx.x];
    for (int e = threadIdx.x; e < PP * P; e += blockDim.x) cube[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int k = threadIdx.x; k < L.nE; k += blockDim.x) cube[L.cube_idx[k]] = upeq[(size_t)b * L.nE + k];
    __syncthreads();
    for (int e = threadIdx.x; e < G * PP; e += blockDim.x) {
        int ka = e % G, line = e / G;
        double2 acc = make_double2(0.0, 0.0);
        for (int a = 0; a < P; ++a) cfma(acc, cube[line * P + a], twf[((P + a) * ka) % G]);
        b1[e] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < G * G * P; e += blockDim.x) {
        int ka = e % G, kb = (e / G) % G, c = e / (G * G);
        double2 acc = make_double2(0.0, 0.0);
        for (int bb = 0; bb < P; ++bb) cfma(acc, b1[(c * P + bb) * G + ka], twf[((P + bb) * kb) % G]);
        b2[e] = acc;
    }
    __syncthreads();
    double2* o = spec + (size_t)b * G * G * G;
    for (int e = threadIdx.x; e < G * G * G; e += blockDim.x) {
        int kab = e % (G * G), kc = e / (G * G);
        double2 acc = make_double2(0.0, 0.0);
        for (int c = 0; c < P; ++c) cfma(acc, b2[c * G * G + kab], twf[((P + c) * kc) % G]);
        o[e] = acc;
    }
}

template <int G>
__global__ void __launch_bounds__(256) vlist_accum_kernel(VlistLevel L, const int* __restrict__ trg,
                                                          const int* __restrict__ vptr, const int* __restrict__ vsrc,
                                                          const int* __restrict__ voff,
                                                          const double2* __restrict__ spec,
                                                          double2* __restrict__ dnchk, const double2* __restrict__ twb) {
    extern __shared__ double2 sm[];
    constexpr int P = G / 2, PP = P * P, G3 = G * G * G, NE = (G3 + 255) / 256;
    double2* grid = sm;          // G^3 accumulated spectrum, later [c'][b'][ka]
    double2* c1 = sm + G3;       // [c'][kb][ka], later the P^3 cube
    const int ti = blockIdx.x, t = trg[ti];
    double2 acc[NE];
#pragma unroll
    for (int q = 0; q < NE; ++q) acc[q] = make_double2(0.0, 0.0);
    for (int v = vptr[ti]; v < vptr[ti + 1]; ++v) {
        const double2* sp = spec + (size_t)vsrc[v] * G3;
        const double2* tn = L.tns + (size_t)voff[v] * G3;
#pragma unroll
        for (int q = 0; q < NE; ++q) {
            int e = threadIdx.x + 256 * q;
            if (e < G3) cfma(acc[q], __ldg(sp + e), __ldg(tn + e));
        }
    }
#pragma unroll
    for (int q = 0; q < NE; ++q) {
        int e = threadIdx.x + 256 * q;
        if (e < G3) grid[e] = acc[q];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < G * G * P; e += blockDim.x) {  // z: outputs c' < P
        int kab = e % (G * G), c = e / (G * G);
        double2 s = make_double2(0.0, 0.0);
        for (int kc = 0; kc < G; ++kc) cfma(s, grid[kc * G * G + kab], twb[((P + c) * kc) % G]);
        c1[e] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < G * PP; e += blockDim.x) {  // y: outputs b' < P
        int ka = e % G, bb = (e / G) % P, c = e / (G * P);
        double2 s = make_double2(0.0, 0.0);
        for (int kb = 0; kb < G; ++kb) cfma(s, c1[(c * G + kb) * G + ka], twb[((P + bb) * kb) % G]);
        grid[e] = s;  // [c'][b'][ka]
    }
    __syncthreads();
    for (int e = threadIdx.x; e < PP * P; e += blockDim.x) {  // x: outputs a' < P
        int a = e % P, line = e / P;
        double2 s = make_double2(0.0, 0.0);
        for (int ka = 0; ka < G; ++ka) cfma(s, grid[line * G + ka], twb[((P + a) * ka) % G]);
        c1[e] = s;  // [c'][b'][a']
    }
    __syncthreads();
    const double coef = 1.0 / (double)G3;
    for (int k = threadIdx.x; k < L.nE; k += blockDim.x) {
        double2 v = c1[L.cube_idx[k]];
        double2 o = dnchk[(size_t)t * L.nE + k];
        o.x += v.x * coef;
        o.y += v.y * coef;
        dnchk[(size_t)t * L.nE + k] = o;
    }
}

static size_t vfwd_smem(int G, int P) { return sizeof(double2) * (P * P * P + G * P * P + G * G * P); }
static size_t vacc_smem(int G, int P) { return sizeof(double2) * (G * G * G + G * G * P); }

void vlist_init(int G) {
    int P = G / 2;
    cudaFuncSetAttribute(vlist_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vfwd_smem(G, P));
    cudaFuncSetAttribute(vlist_accum_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vacc_smem(8, 4));
    cudaFuncSetAttribute(vlist_accum_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vacc_smem(12, 6));
    cudaFuncSetAttribute(vlist_accum_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vacc_smem(16, 8));
}

void launch_vlist_forward(const VlistLevel& L, const int* boxes, int nbox, const double2* upeq, double2* spec,
                          cudaStream_t s) {
    if (nbox == 0) return;
    vlist_forward_kernel<<<nbox, 256, vfwd_smem(L.G, L.P), s>>>(L, boxes, upeq, spec, L.twf);
}

void launch_vlist_accum(const VlistLevel& L, const int* trg, int ntrg, const int* vptr, const int* vsrc,
                        const int* voff, const double2* spec, double2* dnchk, cudaStream_t s) {
    if (ntrg == 0) return;
    size_t sm = vacc_smem(L.G, L.P);
    switch (L.G) {
        case 8: vlist_accum_kernel<8><<<ntrg, 256, sm, s>>>(L, trg, vptr, vsrc, voff, spec, dnchk, L.twb); break;
        case 12: vlist_accum_kernel<12><<<ntrg, 256, sm, s>>>(L, trg, vptr, vsrc, voff, spec, dnchk, L.twb); break;
        case 16: vlist_accum_kernel<16><<<ntrg, 256, sm, s>>>(L, trg, vptr, vsrc, voff, spec, dnchk, L.twb); break;
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
