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
// One CTA per (block row, slot), everything in shared memory: the residual
// and the transformed matrix (FP32, [k][j] rows padded to 16 bytes), the
// radial coefficients of the slot.  The transforms are register-tiled
// products (4 x 4 outputs per thread, E and E^T from L1), the tridiagonals
// one thread per mode (Thomas: the radial operator is diagonally dominant
// and every shift gamma lambda_q is positive).  Each cycle shrinks the
// error by about the FP32 forward error of the solve, so a converged solve
// takes two or three cycles instead of four cycles of ten ADI steps.
#include <cstdlib>
#include <vector>

#include "bph_direct.h"
#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kDThreads = 256;

struct DirectArgs {
    double *P;                 // slot arrays [inst][N][numr*numz], updated in place
    const double *R;           // [inst][N][nr*nz]
    const float *E, *Et;       // [nzp][nzp] row-major and transposed, zero-padded
    const float *lam;          // [nz]
    const double *brb;         // [N][numr] radial diagonal
    const double *alphar, *betar, *bzb;
    double *norms;             // per (instance, slot) |delta|^2, |phi|^2
    const int *inst_map;       // instance of each block row (nullptr: row)
    int N, numr, numz, nr, nz, nrp, nzp, ldx, isym;
    double gamma;
};

__device__ __forceinline__ void fma4x4(float (&acc)[4][4], const float4 a, const float4 b) {
    const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fmaf(av[i], bv[jj], acc[i][jj]);
}

// out[i][:] (rows i0.., 4 x 4 tiles) = sum_l A[i][l] in[l][:], with A given
// transposed (At[l][i], row length nzp) so that 4 consecutive rows load as
// one float4; in and out are shared [nzp][ldx].
__device__ __forceinline__ void tiled_product(const float *__restrict__ At, const float *in, float *out, int nzp,
                                              int nrp, int ldx) {
    const int nti = nzp / 4, ntj = nrp / 4;
    for (int t = threadIdx.x; t < nti * ntj; t += kDThreads) {
        const int i0 = 4 * (t / ntj), j0 = 4 * (t % ntj);
        float acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) acc[i][jj] = 0.f;
#pragma unroll 4
        for (int l = 0; l < nzp; ++l) {
            const float4 a = __ldg(reinterpret_cast<const float4 *>(At + (size_t)l * nzp + i0));
            const float4 b = *reinterpret_cast<const float4 *>(in + l * ldx + j0);
            fma4x4(acc, a, b);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            *reinterpret_cast<float4 *>(out + (i0 + i) * ldx + j0) = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
    }
}

__global__ void __launch_bounds__(kDThreads) k_defect_direct(DirectArgs a) {
    extern __shared__ __align__(16) float dsm[];
    const int nzp = a.nzp, ldx = a.ldx, nr = a.nr, nz = a.nz, numr = a.numr;
    float *X = dsm;                   // residual, then the Thomas carries, then delta
    float *Y = dsm + nzp * ldx;       // E X, then the radial solutions
    float *cb = Y + nzp * ldx;        // radial diagonal of the slot
    float *ca = cb + nr;              // coefficient of j + 1
    float *cl = ca + nr;              // coefficient of j - 1
    const int s = blockIdx.x % a.N, row = blockIdx.x / a.N;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    double *Pg = a.P + blk * (long long)numr * a.numz;
    const double *Rg = a.R + blk * (long long)nr * nz;
    const double gamma = a.gamma;
    for (int j = threadIdx.x; j < nr; j += kDThreads) {
        cb[j] = (float)a.brb[(long long)s * numr + j + 1];
        ca[j] = (float)a.alphar[j + 1];
        cl[j] = (float)a.betar[j + 1];
    }
    pdl_wait();
    // 1. FP64 residual r = R - A phi, rounded into X (zero in the padding)
    for (int e = threadIdx.x; e < nzp * ldx; e += kDThreads) {
        const int k = e / ldx, j = e - k * ldx;
        float r = 0.f;
        if (k < nz && j < nr) {
            const double *pc = Pg + (long long)numr * (k + 1) + 1 + j;
            const double c = pc[0], ea = pc[1], no = pc[numr];
            const double we = (j > 0) ? pc[-1] : 0.0;
            const double so = (k > 0 || a.isym == 1) ? pc[-numr] : 0.0;
            const double ar = a.brb[(long long)s * numr + j + 1] * c + a.alphar[j + 1] * ea + a.betar[j + 1] * we;
            const double az = a.bzb[k + 1] * c - gamma * no - gamma * so;
            r = (float)(Rg[(long long)k * nr + j] - ar - az);
        }
        X[e] = r;
    }
    __syncthreads();
    // 2. Y = E X
    tiled_product(a.Et, X, Y, nzp, a.nrp, ldx);
    __syncthreads();
    // 3. (A_r + gamma lambda_q) y_q = Y_q for every mode q (Thomas; carries kept in X)
    const float gf = (float)gamma;
    for (int q = threadIdx.x; q < nz; q += kDThreads) {
        const float shift = gf * a.lam[q];
        float *yq = Y + q * ldx, *cq = X + q * ldx;
        float cp = 0.f, dp = 0.f;
        for (int j = 0; j < nr; ++j) {
            const float lo = (j > 0) ? cl[j] : 0.f;
            const float m = (cb[j] + shift) - lo * cp;
            cp = ca[j] / m;
            dp = (yq[j] - lo * dp) / m;
            cq[j] = cp;
            yq[j] = dp;
        }
        float y = dp;
        for (int j = nr - 2; j >= 0; --j) {
            y = yq[j] - cq[j] * y;
            yq[j] = y;
        }
    }
    __syncthreads();
    // 4. delta = E^T y (into X)
    tiled_product(a.E, Y, X, nzp, a.nrp, ldx);
    __syncthreads();
    pdl_trigger();
    // 5. phi += delta in FP64; per-slot update and potential norms
    double sd = 0.0, sp = 0.0;
    for (int e = threadIdx.x; e < nz * nr; e += kDThreads) {
        const int k = e / nr, j = e - k * nr;
        const double d = (double)X[k * ldx + j];
        double *pp = Pg + (long long)numr * (k + 1) + 1 + j;
        const double ph = *pp + d;
        *pp = ph;
        sd += d * d;
        sp += ph * ph;
    }
    __shared__ double red[2][kDThreads / 32];
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
        for (int w = 0; w < kDThreads / 32; ++w) t += red[threadIdx.x][w];
        const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
        a.norms[2 * blk + threadIdx.x] = wgt * t;
    }
}

struct DirectShape {
    int nrp, nzp, ldx;
    size_t smem;
};

DirectShape direct_shape(int nr, int nz) {
    DirectShape d;
    d.nrp = (nr + 3) / 4 * 4;
    d.nzp = (nz + 3) / 4 * 4;
    d.ldx = d.nrp + 4;  // rows stay 16-byte aligned; the Thomas threads spread over 8 banks
    d.smem = sizeof(float) * ((size_t)2 * d.nzp * d.ldx + 3 * (size_t)nr);
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
    std::vector<float> hE((size_t)d.nzp * d.nzp, 0.f), hEt((size_t)d.nzp * d.nzp, 0.f), hl((size_t)c->nz);
    for (int q = 0; q < c->nz; ++q) {
        hl[q] = (float)lam[q];
        for (int k = 0; k < c->nz; ++k) {
            const float v = (float)E[(size_t)q * c->nz + k];
            hE[(size_t)q * d.nzp + k] = v;
            hEt[(size_t)k * d.nzp + q] = v;
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
    c->mixed_smem_kind[BPH_MIXED_DIRECT] = (int)d.smem;
    c->mixed_per_sm_kind[BPH_MIXED_DIRECT] = per_sm;
    return BPH_OK;
}

cudaError_t launch_defect_direct(bph_ctx *c, double *P, const double *R, int nrows, const int *inst_map,
                                 double *norms) {
    if (!c->mixed_smem_kind[BPH_MIXED_DIRECT] || !c->d_dir32 || !norms) return cudaErrorNotSupported;
    const DirectShape d = direct_shape(c->nr, c->nz);
    const size_t ne = (size_t)d.nzp * d.nzp;
    DirectArgs a;
    a.P = P;
    a.R = R;
    a.E = c->d_dir32;
    a.Et = c->d_dir32 + ne;
    a.lam = c->d_dir32 + 2 * ne;
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
    a.isym = c->g.isym;
    a.gamma = c->gamma;
    ++c->launches;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, dim3((unsigned)(c->N * nrows)), dim3(kDThreads), d.smem, attr);
    return cudaLaunchKernelEx(&cfg, k_defect_direct, a);
}

}  // namespace bph
