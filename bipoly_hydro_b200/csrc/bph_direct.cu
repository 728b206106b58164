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
// Three kernels per cycle: the FP64 residual rounded to float (one thread
// per zone), the solve, and phi += delta with the per-slot norms (one CTA
// per slot and block row, many resident per SM).  The solve takes one CTA
// per (block row, slot), everything in shared memory: the residual
// and the transformed matrix (FP32, [k][j] rows padded to 16 bytes), the
// transform matrix (E, then E^T) and the radial sub-diagonal.
// The transforms run on the tensor cores (TF32 mma.sync, split in hi and
// lo parts for FP32 accuracy), the tridiagonals one thread per mode
// (Thomas with factors computed at set-up in FP64: the radial operator is
// diagonally dominant and every shift gamma lambda_q is positive).  Each
// cycle shrinks the error by about the FP32 forward error of the solve, so
// a converged solve takes three cycles instead of four of ten ADI steps.
#include <cstdlib>
#include <vector>

#include "bph_direct.h"
#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kDThreads = 384;

struct DirectArgs {
    double *P;                 // slot arrays [inst][N][numr*numz], updated in place
    const double *R;           // [inst][N][nr*nz]
    const float *E, *Et;       // [nzp][lda] row-major and transposed, zero-padded
    const float *lam;          // [nz]
    const float2 *F;           // radial Thomas factors (1/m_j, c'_j) [N][nr][nz]
    const double *brb;         // [N][numr] radial diagonal
    const double *alphar, *betar, *bzb;
    double *norms;             // per (instance, slot) |delta|^2, |phi|^2
    const int *inst_map;       // instance of each block row (nullptr: row)
    int N, numr, numz, nr, nz, nrp, nzp, ldx, lda, isym;
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

// out (nzp x nrp) = A in, A in shared memory row-major with row length
// lda (= nzp + 4: the 8 fragment rows of a load fall on different banks),
// in and out shared [nzp][ldx].  Warp tiles of 16 rows x 32 columns
// (four m16n8k8 tiles), three split-TF32 products per k-step:
//   a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4);
//   b0 (k = t, n = g), b1 (k = t + 4, n = g);
//   d0 (g, 2t), d1 (g, 2t + 1), d2 (g + 8, 2t), d3 (g + 8, 2t + 1).
__device__ __forceinline__ void tc_product(const float *A, int lda, const float *in, float *out, int nzp, int nrp,
                                           int ldx) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int nti = nzp / 16, ntj = nrp / 32;
    for (int wt = warp; wt < nti * ntj; wt += kDThreads / 32) {
        const int i0 = 16 * (wt / ntj), j0 = 32 * (wt % ntj);
        float acc[4][4];
#pragma unroll
        for (int n = 0; n < 4; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
        for (int k0 = 0; k0 < nzp; k0 += 8) {
            uint32_t ah[4], al[4];
            split_tf32(A[(i0 + g) * lda + k0 + t], ah[0], al[0]);
            split_tf32(A[(i0 + g + 8) * lda + k0 + t], ah[1], al[1]);
            split_tf32(A[(i0 + g) * lda + k0 + t + 4], ah[2], al[2]);
            split_tf32(A[(i0 + g + 8) * lda + k0 + t + 4], ah[3], al[3]);
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                uint32_t bh0, bl0, bh1, bl1;
                split_tf32(in[(k0 + t) * ldx + j0 + 8 * n + g], bh0, bl0);
                split_tf32(in[(k0 + t + 4) * ldx + j0 + 8 * n + g], bh1, bl1);
                mma_tf32(acc[n], al, bh0, bh1);
                mma_tf32(acc[n], ah, bl0, bl1);
                mma_tf32(acc[n], ah, bh0, bh1);
            }
        }
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            *reinterpret_cast<float2 *>(out + (i0 + g) * ldx + j0 + 8 * n + 2 * t) = make_float2(acc[n][0], acc[n][1]);
            *reinterpret_cast<float2 *>(out + (i0 + g + 8) * ldx + j0 + 8 * n + 2 * t) =
                make_float2(acc[n][2], acc[n][3]);
        }
    }
}

// The nzp x lda matrix M (global, padded rows) into shared memory.
__device__ __forceinline__ void load_matrix(float *dst, const float *__restrict__ M, int nzp, int lda) {
    for (int e = threadIdx.x; e < nzp * lda / 4; e += kDThreads)
        reinterpret_cast<float4 *>(dst)[e] = __ldg(reinterpret_cast<const float4 *>(M) + e);
}

// FP64 residual r = R - A phi of the current potential, rounded to float:
// one thread per zone, `bps` CTAs per (block row, slot), consecutive threads
// on consecutive zones of a row; written [row][slot][k][j].
__global__ void __launch_bounds__(256) k_direct_residual(DirectArgs a, float *r32, int bps) {
    const int qq = blockIdx.x / bps;
    const int s = qq % a.N, row = qq / a.N;
    const int nr = a.nr, tot = nr * a.nz;
    const int e = (blockIdx.x - qq * bps) * 256 + threadIdx.x;
    pdl_wait();
    if (e >= tot) return;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int numr = a.numr;
    const int k = e / nr, j = e - k * nr;
    const double *pc = a.P + blk * (long long)numr * a.numz + numr * (k + 1) + 1 + j;
    const double c = pc[0], ea = pc[1], no = pc[numr];
    const double we = (j > 0) ? pc[-1] : 0.0;
    const double so = (k > 0 || a.isym == 1) ? pc[-numr] : 0.0;
    const double ar = a.brb[(long long)s * numr + j + 1] * c + a.alphar[j + 1] * ea + a.betar[j + 1] * we;
    const double az = a.bzb[k + 1] * c - a.gamma * no - a.gamma * so;
    r32[((long long)row * a.N + s) * tot + e] = (float)(a.R[blk * tot + e] - ar - az);
}

// phi += delta (delta rounded to float, [row][slot][k][j]) in FP64, with the
// per-slot |delta|^2 and |phi|^2: one CTA per (block row, slot).
__global__ void __launch_bounds__(256) k_direct_update(DirectArgs a, const float *d32) {
    const int s = blockIdx.x % a.N, row = blockIdx.x / a.N;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int nr = a.nr, tot = nr * a.nz, numr = a.numr;
    double *Pg = a.P + blk * (long long)numr * a.numz;
    const float *dg = d32 + ((long long)row * a.N + s) * tot;
    pdl_wait();
    double sd = 0.0, sp = 0.0;
#pragma unroll 4
    for (int e = threadIdx.x; e < tot; e += 256) {
        const int k = e / nr, j = e - k * nr;
        const double d = (double)dg[e];
        double *pp = Pg + numr * (k + 1) + 1 + j;
        const double ph = *pp + d;
        *pp = ph;
        sd += d * d;
        sp += ph * ph;
    }
    __shared__ double red[2][8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sd += __shfl_down_sync(0xffffffffu, sd, off);
        sp += __shfl_down_sync(0xffffffffu, sp, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sd;
        red[1][threadIdx.x >> 5] = sp;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[threadIdx.x][w];
        const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
        a.norms[2 * blk + threadIdx.x] = wgt * t;
    }
}

__device__ __forceinline__ void cp4(float *dst, const float *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}

__global__ void __launch_bounds__(kDThreads, 1) k_defect_direct(DirectArgs a, float *r32) {
    extern __shared__ __align__(16) float dsm[];
    const int nzp = a.nzp, ldx = a.ldx, nr = a.nr, nz = a.nz, numr = a.numr;
    float *X = dsm;                   // residual, then the Thomas carries, then delta
    float *Y = dsm + nzp * ldx;       // E X, then the radial solutions
    float *Ms = Y + nzp * ldx;        // E, then E^T ([nzp][lda])
    float *cl = Ms + nzp * a.lda;     // radial coefficient of j - 1
    const int s = blockIdx.x % a.N, row = blockIdx.x / a.N;
    float *rg = r32 + ((long long)row * a.N + s) * (long long)nr * nz;  // residual in, delta out
    for (int j = threadIdx.x; j < nr; j += kDThreads) cl[j] = (float)a.betar[j + 1];
    load_matrix(Ms, a.E, nzp, a.lda);
    // zero padding of X (rows k >= nz, columns j >= nr), then the residual by cp.async
    for (int e = threadIdx.x; e < nzp * ldx; e += kDThreads) {
        const int k = e / ldx, j = e - k * ldx;
        if (k >= nz || j >= nr) X[e] = 0.f;
    }
    pdl_wait();
    for (int e = threadIdx.x; e < nz * nr; e += kDThreads) {
        const int k = e / nr, j = e - k * nr;
        cp4(X + k * ldx + j, rg + e);
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;" ::: "memory");
    __syncthreads();
    // 2. Y = E X
    tc_product(Ms, a.lda, X, Y, nzp, a.nrp, ldx);
    __syncthreads();
    load_matrix(Ms, a.Et, nzp, a.lda);  // for step 4; no reader of E is left
    // 3. (A_r + gamma lambda_q) y_q = Y_q for every mode q: Thomas sweeps with the
    //    slot's factors (1/m_j, c'_j) from set-up, read coalesced over q
    const float2 *fs = a.F + (long long)s * nr * nz;
    for (int q = threadIdx.x; q < nz; q += kDThreads) {
        float *yq = Y + q * ldx;
        float dp = 0.f;
#pragma unroll 8
        for (int j = 0; j < nr; ++j) {
            const float lo = (j > 0) ? cl[j] : 0.f;
            const float2 f = __ldg(fs + (long long)j * nz + q);
            dp = (yq[j] - lo * dp) * f.x;
            yq[j] = dp;
        }
        float y = dp;
#pragma unroll 8
        for (int j = nr - 2; j >= 0; --j) {
            const float2 f = __ldg(fs + (long long)j * nz + q);
            y = yq[j] - f.y * y;
            yq[j] = y;
        }
    }
    __syncthreads();
    // 4. delta = E^T y (into X)
    tc_product(Ms, a.lda, Y, X, nzp, a.nrp, ldx);
    __syncthreads();
    // 5. delta (float) over the residual, for k_direct_update
    for (int e = threadIdx.x; e < nz * nr; e += kDThreads) {
        const int k = e / nr, j = e - k * nr;
        rg[e] = X[k * ldx + j];
    }
    pdl_trigger();
}

// Thomas factors of (A_r(s) + gamma lambda_q) for every slot s and mode q,
// in FP64, stored as float (1/m_j, c'_j) at [s][j][q]: one thread per (s, q).
__global__ void k_direct_factors(const double *__restrict__ brb, const double *__restrict__ alphar,
                                 const double *__restrict__ betar, const double *__restrict__ lam, float2 *F, int N,
                                 int numr, int nr, int nz, double gamma) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * nz) return;
    const int s = t / nz, q = t % nz;
    const double shift = gamma * lam[q];
    double cp = 0.0;
    for (int j = 0; j < nr; ++j) {
        const double lo = (j > 0) ? betar[j + 1] : 0.0;
        const double m = brb[(long long)s * numr + j + 1] + shift - lo * cp;
        cp = alphar[j + 1] / m;
        F[((long long)s * nr + j) * nz + q] = make_float2((float)(1.0 / m), (float)cp);
    }
}

struct DirectShape {
    int nrp, nzp, ldx, lda;
    size_t smem;
};

DirectShape direct_shape(int nr, int nz) {
    DirectShape d;
    d.nrp = (nr + 31) / 32 * 32;  // warp tiles of 32 columns
    d.nzp = (nz + 15) / 16 * 16;  // and 16 rows
    d.ldx = d.nrp + 4;            // rows stay 16-byte aligned; the Thomas threads spread over 8 banks
    d.lda = d.nzp + 4;            // fragment rows of E on different banks
    d.smem = sizeof(float) * ((size_t)2 * d.nzp * d.ldx + (size_t)d.nzp * d.lda + (size_t)nr);
    return d;
}

}  // namespace

int direct_configure(bph_ctx *c) {
    c->mixed_smem_kind[BPH_MIXED_DIRECT] = 0;
    const DirectShape d = direct_shape(c->nr, c->nz);
    int dev_max = 0;
    cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    if (d.smem + 2 * sizeof(double) * (kDThreads / 32) > (size_t)dev_max) return BPH_OK;  // slot beyond shared memory
    std::vector<long double> E, lam;
    direct::vertical_eigen(c->nz, c->g.isym, E, lam);
    std::vector<float> hE((size_t)d.nzp * d.lda, 0.f), hEt((size_t)d.nzp * d.lda, 0.f), hl((size_t)c->nz);
    for (int q = 0; q < c->nz; ++q) {
        hl[q] = (float)lam[q];
        for (int k = 0; k < c->nz; ++k) {
            const float v = (float)E[(size_t)q * c->nz + k];
            hE[(size_t)q * d.lda + k] = v;
            hEt[(size_t)k * d.lda + q] = v;
        }
    }
    const size_t ne = hE.size();
    e = cudaMalloc((void **)&c->d_dir32, sizeof(float) * (2 * ne + (size_t)c->nz));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(direct solve tables)");
    c->bytes += sizeof(float) * (2 * ne + (size_t)c->nz);
    e = cudaMemcpy(c->d_dir32, hE.data(), sizeof(float) * ne, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_dir32 + ne, hEt.data(), sizeof(float) * ne, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(c->d_dir32 + 2 * ne, hl.data(), sizeof(float) * (size_t)c->nz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = raise_smem_limit((const void *)k_defect_direct, (int)d.smem);
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_defect_direct, kDThreads, d.smem);
    if (e != cudaSuccess) return cuda_fail(e, "direct solve set-up");
    {
        // radial factors for every (slot, mode), from the eigenvalues in FP64
        std::vector<double> hl64((size_t)c->nz);
        for (int q = 0; q < c->nz; ++q) hl64[q] = (double)lam[q];
        double *d_l64 = nullptr;
        const size_t nf = (size_t)c->N * c->nr * c->nz;
        e = cudaMalloc((void **)&c->d_dirF, sizeof(float2) * nf);
        if (e == cudaSuccess) e = cudaMalloc((void **)&d_l64, sizeof(double) * (size_t)c->nz);
        if (e == cudaSuccess) e = cudaMemcpy(d_l64, hl64.data(), sizeof(double) * (size_t)c->nz, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            const int n = c->N * c->nz;
            k_direct_factors<<<(n + 127) / 128, 128, 0, c->stream>>>(c->d_brb, c->d_alphar, c->d_betar, d_l64,
                                                                      reinterpret_cast<float2 *>(c->d_dirF), c->N,
                                                                      c->g.numr, c->nr, c->nz, c->gamma);
            ++c->launches;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (d_l64) cudaFree(d_l64);
        if (e != cudaSuccess) return cuda_fail(e, "direct solve factors");
        c->bytes += sizeof(float2) * nf;
    }
    if (!c->d_r32) {
        const size_t n32 = (size_t)c->N * c->np;
        e = cudaMalloc((void **)&c->d_r32, sizeof(float) * n32);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(rounded residual)");
        c->bytes += sizeof(float) * n32;
    }
    c->mixed_smem_kind[BPH_MIXED_DIRECT] = (int)d.smem;
    c->mixed_per_sm_kind[BPH_MIXED_DIRECT] = per_sm;
    return BPH_OK;
}

cudaError_t launch_defect_direct(bph_ctx *c, double *P, const double *R, int nrows, const int *inst_map,
                                 double *norms, float *r32) {
    if (!c->mixed_smem_kind[BPH_MIXED_DIRECT] || !c->d_dir32 || !c->d_dirF || !norms || !r32)
        return cudaErrorNotSupported;
    const DirectShape d = direct_shape(c->nr, c->nz);
    const size_t ne = (size_t)d.nzp * d.lda;
    DirectArgs a;
    a.P = P;
    a.R = R;
    a.E = c->d_dir32;
    a.Et = c->d_dir32 + ne;
    a.lam = c->d_dir32 + 2 * ne;
    a.F = reinterpret_cast<const float2 *>(c->d_dirF);
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
    a.ldx = d.ldx;
    a.lda = d.lda;
    a.isym = c->g.isym;
    a.gamma = c->gamma;
    c->launches += 3;
    const int bps = (c->nr * c->nz + 255) / 256;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, dim3((unsigned)((long long)bps * c->N * nrows)), dim3(256), 0, attr);
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_direct_residual, a, r32, bps);
    if (e != cudaSuccess) return e;
    cfg = launch_config(c, dim3((unsigned)(c->N * nrows)), dim3(kDThreads), d.smem, attr);
    e = cudaLaunchKernelEx(&cfg, k_defect_direct, a, r32);
    if (e != cudaSuccess) return e;
    cfg = launch_config(c, dim3((unsigned)(c->N * nrows)), dim3(256), 0, attr);
    return cudaLaunchKernelEx(&cfg, k_direct_update, a, (const float *)r32);
}

}  // namespace bph
