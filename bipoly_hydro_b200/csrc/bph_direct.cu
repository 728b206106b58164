// bph_direct.cu -- direct FP32 solve of the defect equation, the inner
// solver of the mixed-precision converged forms (refinement kind
// BPH_MIXED_DIRECT).
//
// A refinement cycle forms the FP64 residual r = R - A phi of the current
// potential (R = -4 pi rho_hat; the Dirichlet columns of phi enter through
// the stencil), solves A delta = r in FP32 with homogeneous boundary values
// and adds delta to phi in FP64.  The ADI kinds solve for delta with a
// cycle of ADI steps; this kind solves it exactly (to FP32 rounding) by
// the eigen-decomposition of the vertical operator (bph_direct.h):
//
//   Y = E X              (X = r of the slot as a [k][j] matrix; E: nz x nz)
//   (A_r + gamma lambda_q) y_q = Y_q     one radial tridiagonal per mode q
//   delta = E^T y
//
// One kernel per cycle, one CTA per (block row, slot), two per SM: it
// forms the residual of its slot, solves, and adds delta to phi with the
// slot's norms, everything between in shared memory: the residual as X^T
// ([j][k], FP32, transformed in place), the transform matrix (E, then E^T),
// the radial coefficients of the slot and the elimination ratios.
// The transforms run on the tensor cores (TF32 mma.sync, split in hi and
// lo parts for FP32 accuracy), the tridiagonals two threads per mode
// (twisted factorization in FP32 with factors formed on the way: the radial
// operator is diagonally dominant and every shift gamma lambda_q is
// positive).  Each cycle shrinks the error by about the FP32 forward error
// of the solve, so a converged solve takes three cycles instead of four of
// ten ADI steps.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "bph_direct.h"
#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kDThreads = direct::kThreads;

struct DirectArgs {
    double *P;                 // slot arrays [inst][N][numr*numz], updated in place
    const double *R;           // [inst][N][nr*nz]
    const float *E, *Et;       // [nzp][lda] row-major and transposed, zero-padded
    const double *sig;         // [nz] vertical shifts gamma lambda_q (FP64)
    const double *brb;         // [N][numr] radial diagonal
    const double *alphar, *betar, *bzb;
    double *norms;             // per (instance, slot) |delta|^2, |phi|^2
    const int *inst_map;       // instance of each block row (nullptr: row)
    int N, numr, numz, nr, nz, nrp, nzp, ldk, lda, cpb, isym;  // cpb: column pairs per transform block
    int off_bd, off_ms, off_lo, off_up;                        // shared-memory regions (floats)
    double gamma;
};

// TF32 tensor-core product with an FP32-accurate split (three products:
// hi*hi + hi*lo + lo*hi of x = hi + lo, each part rounded to TF32).
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// X <- A X in place on the transposed layout: X^T is [nrp][ldk] in shared
// memory (row j of X^T is column j of X; ldk = nzp + 4) and A (nzp x nzp)
// is row-major [nzp][lda] (lda = nzp + 4).  Warp tiles of 32 rows x 16
// columns (2 x 2 m16n8k8 tiles, three split-TF32 products each per k-step,
// every split fragment used twice).  The column pairs are taken in blocks of
// cpb, at most kTilesPerWarp warp tiles per warp: all products of a block
// are formed in registers, then, after a barrier, written over it.  With both
// strides 4 modulo 32 words the fragment loads (A row g, column t; X^T row g,
// column t) and the accumulator stores (X^T row 2t, column g) touch 32
// different banks.  Fragments of m16n8k8:
//   a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4);
//   b0 (k = t, n = g), b1 (k = t + 4, n = g);
//   d0 (g, 2t), d1 (g, 2t + 1), d2 (g + 8, 2t), d3 (g + 8, 2t + 1).
constexpr int kWarpsD = direct::kWarps;
constexpr int kRows = 8;  // rows (radii) whose loads a thread issues together in the residual and radial loops
constexpr int kTilesPerWarp = direct::kTilesPerWarp;

__device__ __forceinline__ void tc_transform(const float *A, int lda, float *Xt, int ldk, int nzp, int nrp, int cpb) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int cp = nrp / 16;
    for (int cp0 = 0; cp0 < cp; cp0 += cpb) {
        const int ncp = min(cpb, cp - cp0), tiles = (nzp / 32) * ncp;
        float acc[kTilesPerWarp][2][2][4];
#pragma unroll
        for (int r = 0; r < kTilesPerWarp; ++r) {
#pragma unroll
            for (int m = 0; m < 2; ++m)
#pragma unroll
                for (int n = 0; n < 2; ++n)
#pragma unroll
                    for (int v = 0; v < 4; ++v) acc[r][m][n][v] = 0.f;
            const int tile = warp + kWarpsD * r;
            if (tile >= tiles) continue;
            int i0, c0;
            direct::warp_tile(tile, cp0, ncp, i0, c0);
            for (int k0 = 0; k0 < nzp; k0 += 8) {
                uint32_t ah[2][4], al[2][4], bh[2][2], bl[2][2];
#pragma unroll
                for (int m = 0; m < 2; ++m)
#pragma unroll
                    for (int v = 0; v < 4; ++v)
                        split_tf32(A[direct::a_offset(i0, m, k0, g, t, lda, v)], ah[m][v], al[m][v]);
#pragma unroll
                for (int n = 0; n < 2; ++n)
#pragma unroll
                    for (int v = 0; v < 2; ++v)
                        split_tf32(Xt[direct::b_offset(c0, n, k0, g, t, ldk, v)], bh[n][v], bl[n][v]);
#pragma unroll
                for (int m = 0; m < 2; ++m)
#pragma unroll
                    for (int n = 0; n < 2; ++n) {
                        mma_tf32(acc[r][m][n], al[m], bh[n][0], bh[n][1]);
                        mma_tf32(acc[r][m][n], ah[m], bl[n][0], bl[n][1]);
                        mma_tf32(acc[r][m][n], ah[m], bh[n][0], bh[n][1]);
                    }
            }
        }
        __syncthreads();  // every product of this block has read its columns
#pragma unroll
        for (int r = 0; r < kTilesPerWarp; ++r) {
            const int tile = warp + kWarpsD * r;
            if (tile >= tiles) continue;
            int i0, c0;
            direct::warp_tile(tile, cp0, ncp, i0, c0);
#pragma unroll
            for (int m = 0; m < 2; ++m)
#pragma unroll
                for (int n = 0; n < 2; ++n)
#pragma unroll
                    for (int v = 0; v < 4; ++v) Xt[direct::d_offset(i0, m, c0, n, g, t, ldk, v)] = acc[r][m][n][v];
        }
        __syncthreads();
    }
}

// The nzp x lda matrix M (global, padded rows) into shared memory: every
// 16-byte copy issued at once (cp.async, through L2), completed by
// wait_copies() before the barrier that precedes the first reader.
__device__ __forceinline__ void load_matrix(float *dst, const float *__restrict__ M, int nzp, int lda) {
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(dst);
    for (int e = threadIdx.x; e < nzp * lda / 4; e += kDThreads)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(base + 16u * (uint32_t)e), "l"(M + 4 * e)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void wait_copies() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One refinement cycle of a slot: one CTA per (block row, slot), two per SM.
//  1. r = R - A phi in FP64, rounded into X^T.  A warp takes 32 columns and
//     a band of rows and sweeps up the band with the rows below and at hand
//     in registers (east and west neighbours by shuffle), so every potential
//     value is read once; the Dirichlet columns enter through the stencil.
//  2. X <- E X.  3. (A_r + gamma lambda_q) y_q = (E r)_q for every mode q:
//     twisted factorization, two threads per mode, from the slot's radial
//     coefficients in shared memory.  4. X <- E^T X.
//  5. phi += delta in FP64, with the slot's |delta|^2 and |phi|^2.
__global__ void __launch_bounds__(kDThreads, 2) k_defect_direct(DirectArgs a) {
    extern __shared__ __align__(16) float dsm[];
    __shared__ double red[2][kWarpsD];
    const int nzp = a.nzp, ldk = a.ldk, nr = a.nr, nz = a.nz, numr = a.numr;
    float *Xt = dsm;                                              // [nrp][ldk]: r, E r, y, delta
    double *bd = reinterpret_cast<double *>(dsm + a.off_bd);      // radial diagonal of the slot
    float *Ms = dsm + a.off_ms;                                   // E; the ratios c' [nr][nz]; E^T
    float *cl = dsm + a.off_lo, *cu = dsm + a.off_up;             // radial coefficients of j - 1, j + 1
    const int s = blockIdx.x % a.N, row = blockIdx.x / a.N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    load_matrix(Ms, a.E, nzp, a.lda);
    for (int j = threadIdx.x; j < nr; j += kDThreads) {
        bd[j] = a.brb[(long long)s * numr + j + 1];
        cl[j] = (float)a.betar[j + 1];
        cu[j] = (float)a.alphar[j + 1];
    }
    for (int e = threadIdx.x; e < a.nrp * nzp; e += kDThreads) {  // padding: columns j >= nr, rows k >= nz
        const int j = e / nzp, k = e - j * nzp;
        if (j >= nr || k >= nz) Xt[j * ldk + k] = 0.f;
    }
    pdl_wait();
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    double *Pg = a.P + blk * (long long)numr * a.numz;
    const double *Rg = a.R + blk * (long long)nr * nz;
    {
        for (int it = warp; it < direct::sweep_items(nr); it += kWarpsD) {
            int jc, k0, k1;
            direct::sweep_item(it, nr, nz, jc, k0, k1);
            if (k0 >= k1) continue;  // warp-uniform
            const int j = jc + lane;
            const bool on = j < nr;
            const double *col = Pg + min(j, nr) + 1;  // interior column, or the outer Dirichlet column
            const double br = on ? a.brb[(long long)s * numr + j + 1] : 0.0;
            const double al = on ? a.alphar[j + 1] : 0.0;
            const double be = on ? a.betar[j + 1] : 0.0;
            double so = (k0 > 0 || a.isym == 1) ? col[(long long)numr * k0] : 0.0;
            double c = col[(long long)numr * (k0 + 1)];
            for (int kb = k0; kb < k1; kb += kRows) {  // the loads of kRows rows in flight at once
                // edge: the east neighbour of lane 31, the west neighbour of lane 0
                double no[kRows], rr[kRows], edge[kRows], bz[kRows];
#pragma unroll
                for (int u = 0; u < kRows; ++u) {
                    const int k = kb + u;
                    if (k >= k1) break;  // warp-uniform
                    no[u] = col[(long long)numr * (k + 2)];
                    rr[u] = on ? Rg[(long long)k * nr + j] : 0.0;
                    edge[u] = (lane == 31 && on)  ? col[(long long)numr * (k + 1) + 1]
                              : (lane == 0 && j > 0) ? col[(long long)numr * (k + 1) - 1]
                                                     : 0.0;
                    bz[u] = a.bzb[k + 1];
                }
#pragma unroll
                for (int u = 0; u < kRows; ++u) {
                    const int k = kb + u;
                    if (k >= k1) break;
                    const double e_ = __shfl_down_sync(0xffffffffu, c, 1);
                    const double w_ = __shfl_up_sync(0xffffffffu, c, 1);
                    const double east = (lane == 31) ? edge[u] : e_;
                    const double west = (lane == 0) ? edge[u] : w_;
                    const double ar = br * c + al * east + be * west;
                    const double az = bz[u] * c - a.gamma * no[u] - a.gamma * so;
                    if (on) Xt[j * ldk + k] = (float)(rr[u] - ar - az);
                    so = c;
                    c = no[u];
                }
            }
        }
    }
    wait_copies();  // E, issued before the residual
    __syncthreads();
    tc_transform(Ms, a.lda, Xt, ldk, nzp, a.nrp, a.cpb);  // 2. X <- E X
    // 3. (A_r + gamma lambda_q) y_q = (E r)_q for every mode q: the twisted
    //    factorization, two threads per mode (rows 0 .. nr/2 - 1 downwards,
    //    the rest upwards), factors formed on the way from the slot's radial
    //    coefficients, the ratios kept in the transform's region.
    float *cr = Ms;  // [nr][nz]; E has no reader left
    direct::Radial tr;
    tr.b = bd;
    tr.lo = cl;
    tr.up = cu;
    tr.n = nr;
    for (int t = threadIdx.x; t < 2 * nz; t += kDThreads) {
        const int q = t % nz;
        tr.sigma = a.sig[q];
        direct::twisted_eliminate<kRows>(tr, t / nz, Xt + q, ldk, cr + q, nz);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * nz; t += kDThreads) {
        const int q = t % nz, side = t / nz;
        float x0, x1;
        direct::twisted_meet(tr, Xt + q, ldk, cr + q, nz, x0, x1);
        direct::twisted_substitute<kRows>(tr, side, side ? x1 : x0, Xt + q, ldk, cr + q, nz);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nz; q += kDThreads) {  // the meeting rows, once both sides have read them
        float x0, x1;
        direct::twisted_meet(tr, Xt + q, ldk, cr + q, nz, x0, x1);
        if (nr / 2 > 0) Xt[(nr / 2 - 1) * ldk + q] = x0;
        Xt[(nr / 2) * ldk + q] = x1;
    }
    __syncthreads();
    load_matrix(Ms, a.Et, nzp, a.lda);  // the ratios have no reader left
    wait_copies();
    __syncthreads();
    tc_transform(Ms, a.lda, Xt, ldk, nzp, a.nrp, a.cpb);  // 4. delta = E^T y
    double sd = 0.0, sp = 0.0;                              // 5. phi += delta
#pragma unroll 4
    for (int e = threadIdx.x; e < nr * nz; e += kDThreads) {
        const int k = e / nr, j = e - k * nr;
        const double d = (double)Xt[j * ldk + k];
        double *pp = Pg + (long long)numr * (k + 1) + 1 + j;
        const double ph = *pp + d;
        *pp = ph;
        sd += d * d;
        sp += ph * ph;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sd += __shfl_down_sync(0xffffffffu, sd, off);
        sp += __shfl_down_sync(0xffffffffu, sp, off);
    }
    if (lane == 0) {
        red[0][warp] = sd;
        red[1][warp] = sp;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int w = 0; w < kWarpsD; ++w) t += red[threadIdx.x][w];
        const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
        a.norms[2 * blk + threadIdx.x] = wgt * t;
    }
    pdl_trigger();
}

}  // namespace

int direct_configure(bph_ctx *c) {
    c->mixed_smem_kind[BPH_MIXED_DIRECT] = 0;
    const direct::Shape d = direct::shape(c->nr, c->nz);
    int dev_max = 0;
    cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    const size_t smem = sizeof(float) * d.floats;
    if (d.cpb == 0 || smem > (size_t)dev_max) return BPH_OK;  // slot beyond one CTA: kind not offered
    std::vector<long double> E, lam;
    direct::vertical_eigen(c->nz, c->g.isym, E, lam);
    std::vector<float> hE((size_t)d.nzp * d.lda, 0.f), hEt((size_t)d.nzp * d.lda, 0.f);
    for (int q = 0; q < c->nz; ++q) {
        for (int k = 0; k < c->nz; ++k) {
            const float v = (float)E[(size_t)q * c->nz + k];
            hE[(size_t)q * d.lda + k] = v;
            hEt[(size_t)k * d.lda + q] = v;
        }
    }
    const size_t ne = hE.size();
    e = cudaMalloc((void **)&c->d_dir32, sizeof(float) * 2 * ne);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(direct solve tables)");
    c->bytes += sizeof(float) * 2 * ne;
    e = cudaMemcpy(c->d_dir32, hE.data(), sizeof(float) * ne, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_dir32 + ne, hEt.data(), sizeof(float) * ne, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = raise_smem_limit((const void *)k_defect_direct, (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_defect_direct, kDThreads, smem);
    if (e != cudaSuccess) return cuda_fail(e, "direct solve set-up");
    {
        // the shifts gamma lambda_q of the radial systems, in FP64
        std::vector<double> hs((size_t)c->nz);
        for (int q = 0; q < c->nz; ++q) hs[q] = (double)((long double)c->gamma * lam[q]);
        e = cudaMalloc((void **)&c->d_dirS, sizeof(double) * (size_t)c->nz);
        if (e == cudaSuccess) e = cudaMemcpy(c->d_dirS, hs.data(), sizeof(double) * (size_t)c->nz, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "direct solve shifts");
        c->bytes += sizeof(double) * (size_t)c->nz;
    }
    c->mixed_smem_kind[BPH_MIXED_DIRECT] = (int)smem;
    c->mixed_per_sm_kind[BPH_MIXED_DIRECT] = per_sm;
    return BPH_OK;
}

cudaError_t launch_defect_direct(bph_ctx *c, double *P, const double *R, int nrows, const int *inst_map,
                                 double *norms) {
    if (!c->mixed_smem_kind[BPH_MIXED_DIRECT] || !c->d_dir32 || !c->d_dirS || !norms) return cudaErrorNotSupported;
    const direct::Shape d = direct::shape(c->nr, c->nz);
    const size_t ne = (size_t)d.nzp * d.lda;
    DirectArgs a;
    a.P = P;
    a.R = R;
    a.E = c->d_dir32;
    a.Et = c->d_dir32 + ne;
    a.sig = c->d_dirS;
    a.brb = c->d_brb;
    a.alphar = c->d_alphar;
    a.betar = c->d_betar;
    a.bzb = c->d_bzb;
    a.norms = norms;
    a.inst_map = inst_map;
    a.N = c->N;
    a.numr = c->g.numr;
    a.numz = c->g.numz;
    a.nr = c->nr;
    a.nz = c->nz;
    a.nrp = d.nrp;
    a.nzp = d.nzp;
    a.ldk = d.ldk;
    a.lda = d.lda;
    a.cpb = d.cpb;
    a.off_bd = (int)d.off_bd;
    a.off_ms = (int)d.off_ms;
    a.off_lo = (int)d.off_lo;
    a.off_up = (int)d.off_up;
    a.isym = c->g.isym;
    a.gamma = c->gamma;
    c->launches += 1;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, dim3((unsigned)(c->N * nrows)), dim3(kDThreads), sizeof(float) * d.floats, attr);
    return cudaLaunchKernelEx(&cfg, k_defect_direct, a);
}

}  // namespace bph
