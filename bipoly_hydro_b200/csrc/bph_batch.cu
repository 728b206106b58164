// bph_batch.cu -- many independent solves on one grid.
//
// A batch owns the per-instance state of n solves that share a context's
// Green tables, trig data and ADI factors: the slot arrays P (each
// instance's warm state, contiguous as [n][numphi][plane] so that the ADI
// runs as one launch over n*numphi slots), -4 pi rho_hat and the moments.
//
// Per call (all instances at the same tstep):
//   k_fft_fwd<rho>      per instance; moments in the layout mom[m][i][cos|sin][p]
//   DGEMM, per mode m   C_m (nb x 2n) = G_m^T (nb x np) * M_m (np x 2n): every
//                       instance's boundary moments from ONE pass over the
//                       tables (the single-solve contraction is a GEMV that
//                       reads the whole table per solve).  A plain strided-
//                       batched library GEMM over the modes.
//   k_boundary_slots_batch   Dirichlet slots of every instance from C
//   k_adi_seg           one launch over n*numphi slots (no wave-quantisation
//                       tail of a single 256-slot launch)
//   k_fft_inv           per instance

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "bph_internal.cuh"
#include "bph_slices.h"

struct bph_batch {
    bph_ctx *c = nullptr;
    int cap = 0;
    double *d_P = nullptr;     // [cap][N][nplane]
    double *d_R = nullptr;     // [cap][N][np]
    double *d_mom = nullptr;   // [mmax][cap][2][np]
    double *d_C = nullptr;     // [mmax][2cap][nb] column-major per mode
    double *d_rho_stage = nullptr, *d_pot_stage = nullptr;  // [cap][ntot] for host arrays
    // Per-call position tables, double-buffered (call k uses set k % 2, and
    // waits for the event of the call two before it): caller input and output
    // array of each position, then the instance of each position.
    void *d_tab[2] = {nullptr, nullptr};
    void *h_tab[2] = {nullptr, nullptr};  // pinned
    cudaEvent_t tab_ev[2] = {nullptr, nullptr};
    int tab_k = 0;
    int *d_stat = nullptr;     // [cap] non-finite flag of each batch position (host-array calls)
    int *h_stat = nullptr;     // [cap] pinned host copy
    int stage_cap = 0;         // positions of the host-array staging buffers
    double *d_LW = nullptr, *d_LQ = nullptr;  // grid-wide ADI scratch [cap][N][np] (large slots)
    double *d_prev = nullptr;         // converged FP64 solves: slot arrays of the previous cycle (on first use)
    double *d_work32 = nullptr;       // FP32 work arrays of the mixed converged forms (kind-dependent size)
    size_t work32_doubles = 0;        // its size in doubles
    double *d_cnorm = nullptr;        // converged solves: per (instance, slot) norm pairs [cap][N][2]
    double *h_cnorm = nullptr;        // its pinned host copy
    double *d_cpart = nullptr;        // split-K partial sums of the batched contraction
    unsigned int *d_ccnt = nullptr;   // its arrival counters [mmax][row groups]
    bool own_contract = false;        // the CUDA-core k_contract_batch for up to kBatchOwnMax positions
    size_t bytes = 0;
};

namespace bph {
namespace {

// ---------------------------------------------------------------------------
// k_contract_batch: C_m = G_m^T M_m for a small batch (NC = 2n columns,
// n <= 4), the multi-right-hand-side form of k_green_contract.  The tables
// are streamed once from HBM (16-byte evict-first loads); the moment
// columns of the CTA's slice of zones are read by every warp of the CTA and
// stay in L1.  Each warp owns kRowsPerWarp table rows, its lanes stride over
// the zones; split-K slices write partial sums and the last CTA of each
// (mode, row group) adds them in slice order (deterministic).  The library
// GEMM stays for larger batches, where the contraction becomes FP64
// compute-bound.
constexpr int kBatchOwnMax = 4;        // batch positions handled by k_contract_batch
constexpr int kBatchSplitMax = 16;
constexpr int kBatchContractThreads = 256;

template <int NC>
struct BcShape {
    static constexpr int kRowsPerWarp = (NC <= 4) ? 4 : 2;
    static constexpr int kRows = (kBatchContractThreads / 32) * kRowsPerWarp;
};

template <int NC>
__global__ void __launch_bounds__(kBatchContractThreads, 2)
k_contract_batch(const double *__restrict__ G, const double *__restrict__ mom, long long mstride, long long np,
                 int nb, double *__restrict__ C, long long cstride, unsigned int *__restrict__ counters,
                 double *__restrict__ partials) {
    constexpr int RW = BcShape<NC>::kRowsPerWarp, RC = BcShape<NC>::kRows;
    const int m = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int bc = blockIdx.x * RC, bw = bc + warp * RW;
    const int nrows = max(0, min(RW, nb - bw));
    const long long nu = np / 2;
    const long long chunk = (nu + nsplit - 1) / nsplit;
    const long long u0 = split * chunk, u1 = min(nu, u0 + chunk);
    const double2 *g2[RW];
#pragma unroll
    for (int r = 0; r < RW; ++r)
        g2[r] = reinterpret_cast<const double2 *>(G + ((long long)m * nb + (r < nrows ? bw + r : bc)) * np);
    const double2 *m2 = reinterpret_cast<const double2 *>(mom + m * mstride);
    double acc[RW][NC];
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[r][c] = 0.0;
    pdl_wait();
#pragma unroll 2
    for (long long i = u0 + lane; i < u1; i += 32) {
        double2 g[RW];
#pragma unroll
        for (int r = 0; r < RW; ++r) g[r] = (r < nrows) ? __ldcs(g2[r] + i) : make_double2(0.0, 0.0);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const double2 v = __ldg(m2 + c * nu + i);
#pragma unroll
            for (int r = 0; r < RW; ++r) {
                acc[r][c] = fma(g[r].x, v.x, acc[r][c]);
                acc[r][c] = fma(g[r].y, v.y, acc[r][c]);
            }
        }
    }
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[r][c] += __shfl_down_sync(0xffffffffu, acc[r][c], off);
    const int mmax = gridDim.y;
    if (nsplit == 1) {
        if (lane == 0)
            for (int r = 0; r < nrows; ++r)
#pragma unroll
                for (int c = 0; c < NC; ++c) C[m * cstride + (long long)c * nb + bw + r] = acc[r][c];
        return;
    }
    // partial sums [split][m][b][c]
    const long long pstride = (long long)mmax * nb * NC;
    if (lane == 0)
        for (int r = 0; r < nrows; ++r)
#pragma unroll
            for (int c = 0; c < NC; ++c) partials[split * pstride + ((long long)m * nb + bw + r) * NC + c] = acc[r][c];
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    const int tile = m * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) last = (atomicAdd(counters + tile, 1u) == (unsigned)(nsplit - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int nrc = min(RC, nb - bc);
    for (int t = threadIdx.x; t < nrc * NC; t += kBatchContractThreads) {
        const int r = t / NC, c = t % NC;
        double sum = 0.0;
        for (int k = 0; k < nsplit; ++k) sum += __ldcg(partials + k * pstride + ((long long)m * nb + bc + r) * NC + c);
        C[m * cstride + (long long)c * nb + bc + r] = sum;
    }
    if (threadIdx.x == 0) counters[tile] = 0u;
}

template <int NC>
cudaError_t contract_batch_launch(bph_ctx *c, bph_batch *b, long long mstride) {
    const int groups = (c->nb + BcShape<NC>::kRows - 1) / BcShape<NC>::kRows;
    const long long base = (long long)groups * c->g.mmax;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    // enough CTAs for two waves at two per SM, slices of at least 1024 zone pairs
    int nsplit = 1;
    while (nsplit < kBatchSplitMax && base * nsplit < 4LL * sms && (c->np / 2) / (nsplit + 1) >= 1024) ++nsplit;
    dim3 grid((unsigned)groups, (unsigned)c->g.mmax, (unsigned)nsplit);
    ++c->launches;
    k_contract_batch<NC><<<grid, kBatchContractThreads, 0, c->stream>>>(
        c->d_green, b->d_mom, mstride, c->np, c->nb, b->d_C, 2LL * b->cap * c->nb, b->d_ccnt, b->d_cpart);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// k_contract_dmma: C_m = G_m^T M_m on the FP64 tensor cores (DMMA,
// mma.sync m16n8k8 .f64), the batched boundary contraction for every batch
// size.  Warp w of a CTA owns a 16-row tile of boundary rows b and all
// 8 NT columns c of the launch's column block; the CTA's 8 warps share one
// (mode, slice of zones).  Per 8-zone step a warp streams its 16 x 8 table
// tile (four 8-byte evict-first loads per thread, prefetched kDmmaStages
// steps ahead so that ~64 KB of table bytes per SM are in flight) and reads
// the moment fragments (L1: every warp of the CTA reads the same ones).
// Slices write partial sums; the last CTA of each (mode, row group) to
// arrive adds them in slice order (deterministic) and writes C.
//   A (16 x 8, row major) = G[m][b0 + r][k0 + q]      (table rows)
//   B (8 x 8, column major) = M[m][c0 + n][k0 + q]     (moment columns)
//   fragment layout of m16n8k8 .f64 (lane = 4 group + t):
//     a0 (group, t), a1 (group + 8, t), a2 (group, t + 4), a3 (group + 8, t + 4)
//     b0 (k = t, n = group), b1 (k = t + 4, n = group)
//     d0 (group, 2t), d1 (group, 2t + 1), d2 (group + 8, 2t), d3 (group + 8, 2t + 1)
constexpr int kDmmaWarps = 8;
constexpr int kDmmaStages = 4;  // 8-zone steps per staged chunk
constexpr int kDmmaPipe = 3;    // chunks in flight (cp.async stages)

constexpr int kDmmaMaxTiles = 8;  // column tiles of 8 per launch (64 columns)

__device__ __forceinline__ void dmma16x8x8(double (&d)[4], const double (&a)[4], double b0, double b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}

template <int NT>
struct DmmaSmem {
    static constexpr int KC = 8 * kDmmaStages;   // zones per chunk
    static constexpr int KS = KC + 4;            // padded row (doubles): a half-warp's fragment reads hit 16 banks
    static constexpr int NCP = 8 * NT;           // moment columns of the launch's block
    static constexpr int ROWS = kDmmaWarps * 16;  // table rows of a CTA
    static constexpr int A = ROWS * KS, B = NCP * KS;  // doubles per stage
    static constexpr size_t bytes = sizeof(double) * (size_t)kDmmaPipe * (A + B);
};

template <int NT>
__global__ void __launch_bounds__(kDmmaWarps * 32, 1)
k_contract_dmma(const double *__restrict__ G, const double *__restrict__ mom, long long mstride, long long np, int nb,
                int c0, int ncol, double *__restrict__ C, long long cstride, unsigned int *__restrict__ counters,
                double *__restrict__ partials) {
    using L = DmmaSmem<NT>;
    constexpr int KC = L::KC, KS = L::KS, NCP = L::NCP, ROWS = L::ROWS;
    extern __shared__ __align__(16) double dsm[];
    double *As = dsm;                       // [kDmmaPipe][ROWS][KS]
    double *Bs = dsm + kDmmaPipe * L::A;    // [kDmmaPipe][NCP][KS]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane >> 2, t = lane & 3;
    const int m = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
    const int rows_base = blockIdx.x * ROWS;
    const int b0 = rows_base + warp * 16;
    const bool live = b0 < nb;
    // slices of whole chunks; a chunk never reads past its slice's last zone
    const ZoneSlice sl = zone_slice(np, nsplit, split, kDmmaStages);
    const long long k_begin = sl.k_begin, k_end = sl.k_end, zend = sl.z_end;
    double acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
    // Chunk ch = zones [8 (k_begin + 4 ch), +32): the CTA's 128 table rows and the NCP
    // moment columns, copied by cp.async into stage ch % kDmmaPipe; rows beyond nb,
    // columns beyond ncol and zones beyond the slice (or np) are zero-filled.
    const double *gbase = G + (long long)m * nb * np;
    const double *mbase = mom + m * mstride;
    const long long nchunk = (k_end - k_begin + kDmmaStages - 1) / kDmmaStages;
    const bool even_np = (np & 1) == 0;
    // L2 policy of the table stream: evict first (each element is read once per call)
    unsigned long long evict_first;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(evict_first));
    auto issue_chunk = [&](long long ch, int st) {
        const long long zc = 8 * (k_begin + ch * kDmmaStages);
        double *as = As + st * L::A, *bs = Bs + st * L::B;
        if (even_np) {
            for (int q = threadIdx.x; q < (ROWS + NCP) * (KC / 2); q += kDmmaWarps * 32) {
                const int rr = q / (KC / 2), zz = 2 * (q % (KC / 2));
                const long long z = zc + zz;
                const bool tab = rr < ROWS;
                const int idx = tab ? rows_base + rr : c0 + rr - ROWS;
                const bool ok = (tab ? idx < nb : idx < ncol) && z < zend;
                const double *src = ok ? (tab ? gbase : mbase) + (long long)idx * np + z : gbase;
                double *dst = tab ? as + rr * KS + zz : bs + (rr - ROWS) * KS + zz;
                if (tab)
                    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2, %3;" ::"r"(
                                     (uint32_t)__cvta_generic_to_shared(dst)),
                                 "l"(src), "r"(ok ? 16 : 0), "l"(evict_first)
                                 : "memory");
                else
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                                     (uint32_t)__cvta_generic_to_shared(dst)),
                                 "l"(src), "r"(ok ? 16 : 0)
                                 : "memory");
            }
        } else {
            for (int q = threadIdx.x; q < (ROWS + NCP) * KC; q += kDmmaWarps * 32) {
                const int rr = q / KC, zz = q % KC;
                const long long z = zc + zz;
                const bool tab = rr < ROWS;
                const int idx = tab ? rows_base + rr : c0 + rr - ROWS;
                const bool ok = (tab ? idx < nb : idx < ncol) && z < zend;
                const double *src = ok ? (tab ? gbase : mbase) + (long long)idx * np + z : gbase;
                double *dst = tab ? as + rr * KS + zz : bs + (rr - ROWS) * KS + zz;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                                 (uint32_t)__cvta_generic_to_shared(dst)),
                             "l"(src), "r"(ok ? 8 : 0)
                             : "memory");
            }
        }
    };
    pdl_wait();
#pragma unroll
    for (int st = 0; st < kDmmaPipe - 1; ++st) {
        if (st < nchunk) issue_chunk(st, st);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (long long ch = 0; ch < nchunk; ++ch) {
        asm volatile("cp.async.wait_group %0;" ::"n"(kDmmaPipe - 2) : "memory");
        __syncthreads();  // chunk ch has landed; every warp is done with chunk ch - 1
        const long long nxt = ch + kDmmaPipe - 1;
        if (nxt < nchunk) issue_chunk(nxt, (int)(nxt % kDmmaPipe));
        asm volatile("cp.async.commit_group;" ::: "memory");
        const int st_buf = (int)(ch % kDmmaPipe);
        const double *as = As + st_buf * L::A + (warp * 16 + grp) * KS + t;
        const double *bs = Bs + st_buf * L::B + grp * KS + t;
        if (live) {
#pragma unroll
            for (int st = 0; st < kDmmaStages; ++st) {
                const double a[4] = {as[8 * st], as[8 * KS + 8 * st], as[8 * st + 4], as[8 * KS + 8 * st + 4]};
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    const double *bj = bs + 8 * j * KS + 8 * st;
                    dmma16x8x8(acc[j], a, bj[0], bj[4]);
                }
            }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    pdl_trigger();
    const int rows0 = blockIdx.x * kDmmaWarps * 16;
    const int nrows = min(kDmmaWarps * 16, nb - rows0);
    auto put = [&](double *dst, long long rstride, long long cstr) {
        // d0 (grp, 2t), d1 (grp, 2t+1), d2 (grp+8, 2t), d3 (grp+8, 2t+1) of every column tile
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = b0 + grp + ((e & 2) ? 8 : 0);
                const int cc = 8 * j + 2 * t + (e & 1);
                if (live && r < nb) dst[(long long)r * rstride + (long long)cc * cstr] = acc[j][e];
            }
    };
    if (nsplit == 1) {
        // C[m][c0 + cc][r], columns within ncol only
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = b0 + grp + ((e & 2) ? 8 : 0);
                const int col = c0 + 8 * j + 2 * t + (e & 1);
                if (live && r < nb && col < ncol) C[m * cstride + (long long)col * nb + r] = acc[j][e];
            }
        return;
    }
    // partials [split][m][b][NCP]
    const long long pstride = (long long)gridDim.y * nb * NCP;
    put(partials + split * pstride + (long long)m * nb * NCP, NCP, 1);
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    const int tile = m * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) last = (atomicAdd(counters + tile, 1u) == (unsigned)(nsplit - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int q = threadIdx.x; q < nrows * NCP; q += kDmmaWarps * 32) {
        const int r = rows0 + q / NCP, cc = q % NCP;
        const int col = c0 + cc;
        if (col >= ncol) continue;
        double sum = 0.0;
        for (int sp = 0; sp < nsplit; ++sp) sum += __ldcg(partials + sp * pstride + ((long long)m * nb + r) * NCP + cc);
        C[m * cstride + (long long)col * nb + r] = sum;
    }
    if (threadIdx.x == 0) counters[tile] = 0u;
}

template <int NT>
cudaError_t contract_dmma_launch_nt(bph_ctx *c, bph_batch *b, long long mstride, int c0, int ncol, int nsplit) {
    const int groups = (c->nb + kDmmaWarps * 16 - 1) / (kDmmaWarps * 16);
    dim3 grid((unsigned)groups, (unsigned)c->g.mmax, (unsigned)nsplit);
    ++c->launches;
    cudaLaunchAttribute attr[1];
    const size_t smem = DmmaSmem<NT>::bytes;
    cudaError_t e = raise_smem_limit((const void *)k_contract_dmma<NT>, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = launch_config(c, grid, dim3(kDmmaWarps * 32), smem, attr);
    const double *G = c->d_green;
    const double *mom = b->d_mom;
    long long np = c->np, cstride = 2LL * b->cap * c->nb;
    int nb = c->nb;
    double *C = b->d_C;
    unsigned int *cnt = b->d_ccnt;
    double *part = b->d_cpart;
    void *args[] = {(void *)&G, (void *)&mom, (void *)&mstride, (void *)&np, (void *)&nb, (void *)&c0,
                    (void *)&ncol, (void *)&C, (void *)&cstride, (void *)&cnt, (void *)&part};
    return cudaLaunchKernelExC(&cfg, (const void *)k_contract_dmma<NT>, args);
}

// Slices of the zone range (one CTA per SM): the count, up to kBatchSplitMax
// with at least 64 steps of 8 zones per slice and at least two waves, whose
// last wave is the fullest.
int dmma_splits(const bph_ctx *c) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const long long groups = (c->nb + kDmmaWarps * 16 - 1) / (kDmmaWarps * 16);
    const long long base = groups * c->g.mmax;
    const long long nk = (c->np + 7) / 8;
    int best = 1;
    double best_eff = -1.0;
    for (int ns = 1; ns <= kBatchSplitMax; ++ns) {
        if (ns > 1 && nk / ns < 64) break;
        const long long ctas = base * ns;
        const long long waves = (ctas + sms - 1) / sms;
        const double eff = (double)ctas / (double)(waves * sms) + (waves >= 2 ? 0.25 : 0.0);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = ns;
        }
    }
    return best;
}

// C for the 2n columns of n batch positions: one launch per block of 64 columns.
cudaError_t contract_dmma_launch(bph_ctx *c, bph_batch *b, long long mstride, int n) {
    const int ncol = 2 * n;
    const int nsplit = dmma_splits(c);
    for (int c0 = 0; c0 < ncol; c0 += 8 * kDmmaMaxTiles) {
        const int tiles = min(kDmmaMaxTiles, (ncol - c0 + 7) / 8);
        cudaError_t e;
        switch (tiles) {
            case 1: e = contract_dmma_launch_nt<1>(c, b, mstride, c0, ncol, nsplit); break;
            case 2: e = contract_dmma_launch_nt<2>(c, b, mstride, c0, ncol, nsplit); break;
            case 3: e = contract_dmma_launch_nt<3>(c, b, mstride, c0, ncol, nsplit); break;
            case 4: e = contract_dmma_launch_nt<4>(c, b, mstride, c0, ncol, nsplit); break;
            case 5: e = contract_dmma_launch_nt<5>(c, b, mstride, c0, ncol, nsplit); break;
            case 6: e = contract_dmma_launch_nt<6>(c, b, mstride, c0, ncol, nsplit); break;
            case 7: e = contract_dmma_launch_nt<7>(c, b, mstride, c0, ncol, nsplit); break;
            default: e = contract_dmma_launch_nt<8>(c, b, mstride, c0, ncol, nsplit); break;
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// One thread per (instance, boundary row or corner, slot), as k_boundary_slots.
__global__ void k_boundary_slots_batch(const double *__restrict__ C, const double2 *__restrict__ ph,
                                       double *__restrict__ P, int numr, int numz, int nr, int nz, int nb, int N,
                                       int mmax, int fm, int isym, double nfactor, int n, int cap,
                                       const int *__restrict__ map) {
    const int M = N / 2;
    const int ncorner = (isym == 1) ? 2 : 1;
    const long long per = (long long)(nb + ncorner) * N;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per * n) return;
    const int inst = (int)(t / per);  // batch position
    t -= inst * per;
    const int s = (int)(t % N), b = (int)(t / N);
    const long long nplane = (long long)numr * numz;
    double *Pi = P + (long long)(map ? map[inst] : inst) * N * nplane;
    int jz, kz;
    if (b < nr) {
        jz = b + 1;
        kz = numz - 1;
    } else if (b < nr + nz) {
        jz = numr - 1;
        kz = b - nr + 1;
    } else if (b < nb) {
        jz = b - nr - nz + 1;
        kz = 0;
    } else {
        jz = numr - 1;
        kz = (b == nb) ? numz - 1 : 0;
        Pi[(long long)s * nplane + jz + (long long)numr * kz] = 0.0;
        return;
    }
    const bool imag = s > M;
    const int k = imag ? s - M : s;
    double v = 0.0;
    if (k < M && k % fm == 0 && k / fm < mmax) {
        const int m = k / fm;
        const double *Cm = C + (long long)m * (2LL * cap) * nb;
        const double sc = Cm[(2LL * inst) * nb + b];
        const double ss = (m == 0) ? 0.0 : Cm[(2LL * inst + 1) * nb + b];
        const double2 w = ph[m];
        v = imag ? nfactor * (w.y * sc - w.x * ss) : nfactor * (w.x * sc + w.y * ss);
    }
    Pi[(long long)s * nplane + jz + (long long)numr * kz] = v;
}

int batch_alloc(bph_batch *b, double **p, size_t count) {
    cudaError_t e = cudaMalloc((void **)p, sizeof(double) * (count ? count : 1));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        set_error("batch allocation of %zu bytes failed: %s", sizeof(double) * count, cudaGetErrorString(e));
        return BPH_ERR_NOMEM;
    }
    b->bytes += sizeof(double) * count;
    return BPH_OK;
}

}  // namespace

// Schedules are shared with the single-solve path (bph_api.cu).
int batch_schedule(bph_ctx *c, int nsteps, Schedule **out);
int batch_enqueue(bph_batch *b, int n, const double *const *d_in, double *const *d_out, const int *d_map,
                  Schedule &sch, bool warm, bool per_pos);

int batch_converged_run(bph_batch *b, int n, const int *inst, const int *d_map, const double *const *d_in,
                        double *const *d_out, BatchConv &cv, bool per_pos);

}  // namespace bph

using namespace bph;

extern "C" {

int bph_batch_create(bph_ctx_t *c, int capacity, bph_batch_t **out) {
    if (!out) {
        set_error("out-pointer is NULL");
        return BPH_ERR_INVALID;
    }
    *out = nullptr;
    if (!c || capacity < 1 || capacity > 4096) {
        set_error("invalid context or capacity (1..4096)");
        return BPH_ERR_INVALID;
    }
    const bool large = !c->adi_seg;  // slots beyond shared memory: the grid-wide kernels
    if (large && c->adi_smem) {
        set_error("batched solves need the segmented or the grid-wide ADI kernels for this grid");
        return BPH_ERR_INVALID;
    }
    if (large && (long long)capacity * c->N > 65535) {
        set_error("batch capacity %d too large for the grid-wide ADI kernels (capacity * numphi <= 65535)", capacity);
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    cudaError_t e;
    size_t need = sizeof(double) * (size_t)capacity *
                  ((size_t)c->N * c->nplane + (size_t)c->N * c->np * (large ? 3 : 1) + 2ull * c->g.mmax * c->np +
                   2ull * c->g.mmax * c->nb);
    size_t free_b = 0, total_b = 0;
    e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
    if (need + (64ull << 20) > free_b) {
        set_error("batch of %d needs %zu bytes of device memory, %zu free", capacity, need, free_b);
        return BPH_ERR_NOMEM;
    }
    bph_batch *b = new bph_batch();
    b->c = c;
    ctx_retain(c);  // the context's device state stays until this batch is destroyed
    b->cap = capacity;
    int rc = BPH_OK;
    if (!rc) rc = batch_alloc(b, &b->d_P, (size_t)capacity * c->N * c->nplane);
    if (!rc) rc = batch_alloc(b, &b->d_R, (size_t)capacity * c->N * c->np);
    if (!rc) rc = batch_alloc(b, &b->d_mom, (size_t)c->g.mmax * capacity * 2 * c->np);
    if (!rc) rc = batch_alloc(b, &b->d_C, (size_t)c->g.mmax * 2 * capacity * c->nb);
    if (!rc && large) rc = batch_alloc(b, &b->d_LW, (size_t)capacity * c->N * c->np);
    if (!rc && large) rc = batch_alloc(b, &b->d_LQ, (size_t)capacity * c->N * c->np);
    if (!rc) {
        // split-K scratch of the contraction: partial sums for the widest
        // column block (8 per CUDA-core launch, up to 64 per tensor-core
        // launch) and arrival counters for the narrowest row groups (16 rows)
        const size_t cols = std::max<size_t>(8, std::min<size_t>(8 * kDmmaMaxTiles, 8 * ((2 * (size_t)capacity + 7) / 8)));
        rc = batch_alloc(b, &b->d_cpart, (size_t)kBatchSplitMax * c->g.mmax * c->nb * cols);
        if (!rc) {
            const size_t ncnt = (size_t)c->g.mmax * ((c->nb + 15) / 16);
            e = cudaMalloc((void **)&b->d_ccnt, sizeof(unsigned int) * ncnt);
            if (e == cudaSuccess) e = cudaMemsetAsync(b->d_ccnt, 0, sizeof(unsigned int) * ncnt, c->stream);
            if (e != cudaSuccess) {
                cudaGetLastError();
                set_error("batch counter allocation failed: %s", cudaGetErrorString(e));
                rc = BPH_ERR_NOMEM;
            }
        }
    }
    if (!rc) {
        // BPH_BATCH_CONTRACT=simt: the CUDA-core kernel for up to kBatchOwnMax
        // positions (comparison only; the tensor-core kernel is the default)
        const char *g = std::getenv("BPH_BATCH_CONTRACT");
        b->own_contract = (c->np % 2 == 0) && g && g[0] == 's';
    }
    if (!rc) {
        const size_t tab_bytes = (2 * sizeof(void *) + sizeof(int)) * (size_t)capacity;
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
            e = cudaMalloc(&b->d_tab[k], tab_bytes);
            if (e == cudaSuccess) e = cudaMallocHost(&b->h_tab[k], tab_bytes);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->tab_ev[k], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_stat, sizeof(int) * capacity);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_stat, sizeof(int) * capacity);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("batch map allocation failed: %s", cudaGetErrorString(e));
            rc = BPH_ERR_NOMEM;
        }
    }
    if (!rc) {
        e = cudaMemsetAsync(b->d_P, 0, sizeof(double) * (size_t)capacity * c->N * c->nplane, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_mom, 0, sizeof(double) * (size_t)c->g.mmax * capacity * 2 * c->np,
                                                  c->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemsetAsync");
    }
    if (rc) {
        bph_batch_destroy(b);
        return rc;
    }
    *out = b;
    return BPH_OK;
}

int bph_batch_destroy(bph_batch_t *b) {
    if (!b) return BPH_OK;
    ::bph::DeviceScope scope_(b->c ? b->c->device : 0);
    if (b->c && b->c->stream) cudaStreamSynchronize(b->c->stream);
    double *bufs[] = {b->d_P,     b->d_R,     b->d_mom, b->d_C,    b->d_rho_stage, b->d_pot_stage,
                      b->d_cpart, b->d_LW,    b->d_LQ,  b->d_prev, b->d_cnorm, b->d_work32};
    for (double *p : bufs)
        if (p) cudaFree(p);
    if (b->d_ccnt) cudaFree(b->d_ccnt);
    for (int k = 0; k < 2; ++k) {
        if (b->d_tab[k]) cudaFree(b->d_tab[k]);
        if (b->h_tab[k]) cudaFreeHost(b->h_tab[k]);
        if (b->tab_ev[k]) cudaEventDestroy(b->tab_ev[k]);
    }
    if (b->d_stat) cudaFree(b->d_stat);
    if (b->h_stat) cudaFreeHost(b->h_stat);
    if (b->h_cnorm) cudaFreeHost(b->h_cnorm);
    if (b->c) ctx_release(b->c);
    delete b;
    return BPH_OK;
}

int bph_batch_solve(bph_batch_t *b, int n, const double *const *rho, double *const *pot, int tstep, int on_device) {
    return bph_batch_solve_instances(b, n, nullptr, rho, pot, tstep, on_device);
}

int bph_batch_solve_instances(bph_batch_t *b, int n, const int *instances, const double *const *rho,
                              double *const *pot, int tstep, int on_device) {
    return bph::batch_solve_core(b, n, instances, rho, pot, tstep > 1, on_device != 0, nullptr);
}

int bph_batch_solve_converged(bph_batch_t *b, int n, const double *const *rho, double *const *pot, int nsteps,
                              int cold, double tol, int max_cycles, int mixed, int on_device, int *cycles_out,
                              double *resid_out) {
    if (!b || nsteps < 1 || nsteps > 10000 || max_cycles < 1 || !(tol >= 0.0)) {
        set_error("invalid arguments");
        return BPH_ERR_INVALID;
    }
    bph_ctx *c = b->c;
    if (mixed && !c->adi_mixed_smem) {
        set_error("no mixed-precision ADI kernel is configured for this grid");
        return BPH_ERR_INVALID;
    }
    BatchConv cv;
    cv.nsteps = nsteps;
    cv.max_cycles = max_cycles;
    cv.cold = cold != 0;
    cv.mixed = mixed != 0;
    cv.tol = tol;
    cv.want_resid = resid_out != nullptr;
    const int rc = bph::batch_solve_core(b, n, nullptr, rho, pot, !cold, on_device != 0, nullptr, &cv);
    if (cycles_out) *cycles_out = cv.cycles;
    if (resid_out) *resid_out = cv.resid;
    return rc;
}

}  // extern "C"

namespace bph {

// pos_status (host arrays only): per-position BPH_OK / BPH_ERR_NONFINITE
// instead of one aggregated status.
int batch_solve_core(bph_batch *b, int n, const int *instances, const double *const *rho, double *const *pot,
                     bool warm, bool on_device, int *pos_status, BatchConv *conv) {
    if (!b || !rho || !pot || n < 1 || n > b->cap) {
        set_error("invalid batch arguments (n must be in 1..capacity)");
        return BPH_ERR_INVALID;
    }
    for (int i = 0; i < n; ++i)
        if (!rho[i] || !pot[i]) {
            set_error("batch position %d has a NULL array", i);
            return BPH_ERR_INVALID;
        }
    if (instances) {
        // distinct instances in range
        std::vector<char> seen((size_t)b->cap, 0);
        for (int i = 0; i < n; ++i) {
            const int v = instances[i];
            if (v < 0 || v >= b->cap || seen[(size_t)v]) {
                set_error("instance %d at position %d is out of range or repeated", v, i);
                return BPH_ERR_INVALID;
            }
            seen[(size_t)v] = 1;
        }
    }
    bph_ctx *c = b->c;
    BPH_DEVICE_SCOPE(c);
    Schedule *s;  // warm: 5 steps, cold: 20 (potential_solver.F90:80-94); converged: its cycle length
    int rc = batch_schedule(c, conv ? conv->nsteps : (warm ? 5 : 20), &s);
    if (rc) return rc;
    const size_t bytes = sizeof(double) * (size_t)c->ntot;
    std::vector<int> inst(n);
    for (int i = 0; i < n; ++i) inst[i] = instances ? instances[i] : i;

    std::vector<const double *> d_rho(n);
    std::vector<double *> d_pot(n);
    if (on_device) {
        for (int i = 0; i < n; ++i) {
            d_rho[i] = rho[i];
            d_pot[i] = pot[i];
        }
    } else {
        if (b->stage_cap < n) {
            // staging grows to the largest batch seen
            BPH_CUDA(cudaStreamSynchronize(c->stream));
            if (b->d_rho_stage) {
                cudaFree(b->d_rho_stage);
                b->bytes -= sizeof(double) * (size_t)b->stage_cap * c->ntot;
                b->d_rho_stage = nullptr;
            }
            if (b->d_pot_stage) {
                cudaFree(b->d_pot_stage);
                b->bytes -= sizeof(double) * (size_t)b->stage_cap * c->ntot;
                b->d_pot_stage = nullptr;
            }
            b->stage_cap = 0;
            if ((rc = batch_alloc(b, &b->d_rho_stage, (size_t)n * c->ntot))) return rc;
            if ((rc = batch_alloc(b, &b->d_pot_stage, (size_t)n * c->ntot))) return rc;
            b->stage_cap = n;
        }
        for (int i = 0; i < n; ++i) {
            d_rho[i] = b->d_rho_stage + (size_t)i * c->ntot;
            d_pot[i] = b->d_pot_stage + (size_t)i * c->ntot;
            BPH_CUDA(cudaMemcpyAsync((void *)d_rho[i], rho[i], bytes, cudaMemcpyHostToDevice, c->stream));
        }
    }
    // position tables of this call (set tab_k, free once the call two before has consumed it)
    const int tk = b->tab_k;
    b->tab_k ^= 1;
    BPH_CUDA(cudaEventSynchronize(b->tab_ev[tk]));
    char *hb = static_cast<char *>(b->h_tab[tk]);
    const double **h_in = reinterpret_cast<const double **>(hb);
    double **h_out = reinterpret_cast<double **>(hb + sizeof(void *) * b->cap);
    int *h_inst = reinterpret_cast<int *>(hb + 2 * sizeof(void *) * b->cap);
    for (int i = 0; i < n; ++i) {
        h_in[i] = d_rho[i];
        h_out[i] = d_pot[i];
        h_inst[i] = inst[i];
    }
    BPH_CUDA(cudaMemcpyAsync(b->d_tab[tk], b->h_tab[tk], (2 * sizeof(void *) + sizeof(int)) * (size_t)b->cap,
                             cudaMemcpyHostToDevice, c->stream));
    char *db = static_cast<char *>(b->d_tab[tk]);
    const double *const *d_in = reinterpret_cast<const double *const *>(db);
    double *const *d_out = reinterpret_cast<double *const *>(db + sizeof(void *) * b->cap);
    const int *d_map = instances ? reinterpret_cast<const int *>(db + 2 * sizeof(void *) * b->cap) : nullptr;
    // per-position non-finite flags: host-array calls and callers that want per-position status
    const bool per_pos = !on_device || pos_status;
    if (conv) {
        conv->report_divergence = (pos_status == nullptr);
        rc = batch_converged_run(b, n, inst.data(), d_map, d_in, d_out, *conv, per_pos);
    }
    else
        rc = batch_enqueue(b, n, d_in, d_out, d_map, *s, warm, per_pos);
    if (rc) return rc;
    BPH_CUDA(cudaEventRecord(b->tab_ev[tk], c->stream));
    if (per_pos) {
        if (!on_device)
            for (int i = 0; i < n; ++i)
                BPH_CUDA(cudaMemcpyAsync(pot[i], d_pot[i], bytes, cudaMemcpyDeviceToHost, c->stream));
        BPH_CUDA(cudaMemcpyAsync(b->h_stat, b->d_stat, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
        BPH_CUDA(cudaStreamSynchronize(c->stream));
        int bad = -1;
        for (int i = 0; i < n; ++i) {
            const bool nf = (b->h_stat[i] & kStatusNonFinite) != 0;
            if (pos_status) pos_status[i] = nf ? BPH_ERR_NONFINITE : BPH_OK;
            if (nf && bad < 0) bad = i;
        }
        if (bad >= 0 && !pos_status) {
            set_error("density of batch position %d contains NaN or Inf", bad);
            return BPH_ERR_NONFINITE;
        }
        return BPH_OK;
    }
    return BPH_OK;
}

// The device work of one batched call on c->stream: n positions whose input
// and output arrays (and instances, d_map; nullptr: position = instance) are
// read from device tables.  per_pos: non-finite flags per position in d_stat
// (else the context's aggregated status).  Host-synchronisation free, so that
// it can be captured into a graph.
// Forward transforms, boundary contraction and Dirichlet slots of a
// batched call (the part before the ADI).
static int batch_prologue(bph_batch *b, int n, const double *const *d_in, const int *d_map, bool per_pos) {
    bph_ctx *c = b->c;
    if (per_pos) BPH_CUDA(cudaMemsetAsync(b->d_stat, 0, sizeof(int) * n, c->stream));
    const long long np = c->np;
    const long long mstride = 2LL * b->cap * np;
    BPH_CUDA(launch_fft_fwd_rho_batch(c, n, d_in, d_map, b->d_R, (long long)c->N * np, b->d_mom, mstride, 2LL * np,
                                      per_pos ? b->d_stat : c->d_status, per_pos));
    // C_m = G_m^T M_m for every mode: FP64 tensor-core contraction (or, on
    // request, the CUDA-core kernel for up to kBatchOwnMax positions)
    if (!b->own_contract || n > kBatchOwnMax) {
        BPH_CUDA(contract_dmma_launch(c, b, mstride, n));
    } else {
        cudaError_t ce = cudaSuccess;
        switch (n) {
            case 1: ce = contract_batch_launch<2>(c, b, mstride); break;
            case 2: ce = contract_batch_launch<4>(c, b, mstride); break;
            case 3: ce = contract_batch_launch<6>(c, b, mstride); break;
            default: ce = contract_batch_launch<8>(c, b, mstride); break;
        }
        BPH_CUDA(ce);
    }
    {
        const int ncorner = (c->g.isym == 1) ? 2 : 1;
        const long long total = (long long)(c->nb + ncorner) * c->N * n;
        ++c->launches;
        k_boundary_slots_batch<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(
            b->d_C, c->d_ph, b->d_P, c->g.numr, c->g.numz, c->nr, c->nz, c->nb, c->N, c->g.mmax, c->fm, c->g.isym,
            (double)c->N * c->factor, n, b->cap, d_map);
        BPH_CUDA(cudaGetLastError());
    }
    return BPH_OK;
}

int batch_enqueue(bph_batch *b, int n, const double *const *d_in, double *const *d_out, const int *d_map,
                  Schedule &sch, bool warm, bool per_pos) {
    bph_ctx *c = b->c;
    Schedule *s = &sch;
    int rc = batch_prologue(b, n, d_in, d_map, per_pos);
    if (rc) return rc;
    if (c->adi_seg)
        BPH_CUDA(launch_adi(c, *s, 0, s->nsteps, !warm, b->d_P, b->d_R, n, d_map));
    else
        BPH_CUDA(launch_adi_large(c, *s, 0, s->nsteps, !warm, b->d_P, b->d_R, n, d_map, b->d_LW, b->d_LQ));
    BPH_CUDA(launch_fft_inv_batch(c, n, d_out, d_map, b->d_P, (long long)c->N * c->nplane));
    return BPH_OK;
}

int batch_reserve_converged(bph_batch *b, bool mixed) {
    bph_ctx *c = b->c;
    int rc;
    if (!b->d_cnorm && (rc = batch_alloc(b, &b->d_cnorm, 2ull * b->cap * c->N))) return rc;
    if (!b->h_cnorm) BPH_CUDA(cudaMallocHost((void **)&b->h_cnorm, sizeof(double) * 2 * (size_t)b->cap * c->N));
    // FP64 on the grid-wide kernels: the previous cycle's slot arrays (the segmented kernel
    // forms the update while writing back)
    if (!mixed && !c->adi_seg && !b->d_prev &&
        (rc = batch_alloc(b, &b->d_prev, (size_t)b->cap * c->N * c->nplane)))
        return rc;
    // FP32 work arrays of the refinement: the grid-wide cycle keeps r, delta and two right-hand
    // sides per position; the warp-cooperative one the rounded residual per position
    size_t need = 0;
    if (mixed && c->mixed_kind == BPH_MIXED_ADI_GLOBAL) need = 2ull * b->cap * c->N * c->np;
    if (mixed && c->mixed_kind == BPH_MIXED_ADI_WARP)
        need = ((size_t)b->cap * c->N * c->np + 1) / 2;
    if (need > b->work32_doubles) {
        if (b->d_work32) {
            cudaStreamSynchronize(c->stream);
            cudaFree(b->d_work32);
            b->bytes -= sizeof(double) * b->work32_doubles;
            b->d_work32 = nullptr;
            b->work32_doubles = 0;
        }
        if ((rc = batch_alloc(b, &b->d_work32, need))) return rc;
        b->work32_doubles = need;
    }
    return BPH_OK;
}

// Sums the per-slot norm pairs of instance i: sqrt(sum |a|^2 / sum |b|^2).
static double instance_ratio(const double *h, int N, int i) {
    double num = 0.0, den = 0.0;
    for (int sl = 0; sl < N; ++sl) {
        num += h[2 * ((size_t)i * N + sl)];
        den += h[2 * ((size_t)i * N + sl) + 1];
    }
    return den > 0.0 ? std::sqrt(num / den) : std::sqrt(num);
}

// Converged solves of n batch positions (instance inst[i] on the host,
// d_map on the device; d_map nullptr: position = instance): the transforms
// and boundary once, then cycles of nsteps ADI steps (FP64: update measured
// against the previous cycle's slot arrays) or FP32 refinement cycles on
// the FP64 defect (the update is the cycle's own correction), until every
// instance's relative update is at most tol (mixed: or no longer halves)
// or max_cycles.  Norms are indexed by instance.  One host synchronisation
// per cycle.
int batch_converged_run(bph_batch *b, int n, const int *inst, const int *d_map, const double *const *d_in,
                        double *const *d_out, BatchConv &cv, bool per_pos) {
    bph_ctx *c = b->c;
    Schedule *s;
    int rc = batch_schedule(c, cv.nsteps, &s);
    if (rc) return rc;
    const size_t ibytes = sizeof(double) * (size_t)c->N * c->nplane;  // one instance's slot arrays
    int top = 0;  // instances 0..top-1 hold every position's norms
    for (int i = 0; i < n; ++i) top = std::max(top, inst[i] + 1);
    if ((rc = batch_reserve_converged(b, cv.mixed))) return rc;
    if (cv.cold)  // before the Dirichlet slots
        for (int i = 0; i < n; ++i)
            BPH_CUDA(cudaMemsetAsync(b->d_P + (size_t)inst[i] * c->N * c->nplane, 0, ibytes, c->stream));
    if ((rc = batch_prologue(b, n, d_in, d_map, per_pos))) return rc;
    std::vector<double> prev_upd((size_t)n, INFINITY);
    std::vector<char> done((size_t)n, 0);
    const size_t hbytes = sizeof(double) * 2 * (size_t)top * c->N;
    int cyc = 0;
    bool diverged = false;
    for (;;) {
        if (cv.mixed) {
            if (c->mixed_kind == BPH_MIXED_ADI_GLOBAL)
                BPH_CUDA(launch_adi_defect_large_batch(c, *s, b->d_P, b->d_R, n, d_map,
                                                       reinterpret_cast<float *>(b->d_work32), b->d_cnorm));
            else if (c->mixed_kind == BPH_MIXED_ADI_WARP)
                BPH_CUDA(launch_defect_warp(c, *s, b->d_P, b->d_R, n, d_map, b->d_cnorm,
                                            reinterpret_cast<float *>(b->d_work32)));
            else if (c->mixed_kind == BPH_MIXED_DIRECT)
                BPH_CUDA(launch_defect_direct(c, b->d_P, b->d_R, n, d_map, b->d_cnorm));
            else
                BPH_CUDA(launch_defect_batch(c, *s, b->d_P, b->d_R, n, d_map, b->d_cnorm));
        } else if (c->adi_seg) {  // update norms from the sweep's write-back
            BPH_CUDA(launch_adi(c, *s, 0, s->nsteps, false, b->d_P, b->d_R, n, d_map, b->d_cnorm));
        } else {
            if (d_map) {
                for (int i = 0; i < n; ++i) {
                    const size_t off = (size_t)inst[i] * c->N * c->nplane;
                    BPH_CUDA(cudaMemcpyAsync(b->d_prev + off, b->d_P + off, ibytes, cudaMemcpyDeviceToDevice,
                                             c->stream));
                }
            } else {
                BPH_CUDA(cudaMemcpyAsync(b->d_prev, b->d_P, ibytes * n, cudaMemcpyDeviceToDevice, c->stream));
            }
            BPH_CUDA(launch_adi_large(c, *s, 0, s->nsteps, false, b->d_P, b->d_R, n, d_map, b->d_LW, b->d_LQ));
            BPH_CUDA(launch_norms_batch(c, false, b->d_P, b->d_prev, nullptr, n, d_map, b->d_cnorm));
        }
        ++cyc;
        BPH_CUDA(cudaMemcpyAsync(b->h_cnorm, b->d_cnorm, hbytes, cudaMemcpyDeviceToHost, c->stream));
        BPH_CUDA(cudaStreamSynchronize(c->stream));
        bool all = true;
        for (int i = 0; i < n; ++i) {
            if (done[(size_t)i]) continue;  // converged instances keep cycling with the rest (harmless)
            const double upd = instance_ratio(b->h_cnorm, c->N, inst[i]);
            // a non-finite update ends the instance (a non-finite density is
            // also flagged per position by the forward transform)
            bool stop = upd <= cv.tol || !(upd == upd);
            if (!(upd == upd) && cv.mixed) diverged = true;
            if (cv.mixed) stop = stop || upd > 0.5 * prev_upd[(size_t)i];
            prev_upd[(size_t)i] = upd;
            done[(size_t)i] = stop;
            all = all && stop;
        }
        if (all || diverged || cyc >= cv.max_cycles) break;
    }
    cv.cycles = cyc;
    if (cv.want_resid) {
        BPH_CUDA(launch_norms_batch(c, true, b->d_P, nullptr, b->d_R, n, d_map, b->d_cnorm));
        BPH_CUDA(cudaMemcpyAsync(b->h_cnorm, b->d_cnorm, hbytes, cudaMemcpyDeviceToHost, c->stream));
        BPH_CUDA(cudaStreamSynchronize(c->stream));
        cv.resid = 0.0;
        for (int i = 0; i < n; ++i) cv.resid = std::max(cv.resid, instance_ratio(b->h_cnorm, c->N, inst[i]));
    }
    BPH_CUDA(launch_fft_inv_batch(c, n, d_out, d_map, b->d_P, (long long)c->N * c->nplane));
    if (diverged && cv.report_divergence) {
        set_error("mixed-precision refinement diverged (or a density is non-finite) in a batch instance");
        return BPH_ERR_NONFINITE;
    }
    return BPH_OK;
}

}  // namespace bph

extern "C" {

size_t bph_batch_device_bytes(const bph_batch_t *b) { return b ? b->bytes : 0; }

int bph_batch_copy_moments(bph_batch_t *b, int n, double *out, size_t count) {
    if (!b || !out || n < 1 || n > b->cap) {
        set_error("invalid batch, position count or output");
        return BPH_ERR_INVALID;
    }
    bph_ctx *c = b->c;
    const size_t per = (size_t)c->g.mmax * c->nb * 2;
    if (count < per * (size_t)n) {
        set_error("output holds %zu doubles, %zu needed", count, per * (size_t)n);
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    // C[m][2 pos + cs][b] -> out[pos][m][b][cs]
    const size_t cn = (size_t)c->g.mmax * 2 * b->cap * c->nb;
    std::vector<double> h(cn);
    BPH_CUDA(cudaMemcpyAsync(h.data(), b->d_C, sizeof(double) * cn, cudaMemcpyDeviceToHost, c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    for (int pos = 0; pos < n; ++pos)
        for (int m = 0; m < c->g.mmax; ++m)
            for (int r = 0; r < c->nb; ++r)
                for (int cs = 0; cs < 2; ++cs) {
                    const double v = h[((size_t)m * 2 * b->cap + 2 * pos + cs) * c->nb + r];
                    out[(((size_t)pos * c->g.mmax + m) * c->nb + r) * 2 + cs] = (m == 0 && cs == 1) ? 0.0 : v;
                }
    return BPH_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Plans: the device work of several batches (one per grid shape) recorded as
// one CUDA graph.  Capture forks from a private stream into one stream per
// part (each part's work is batch_enqueue on its context, unchanged), joins
// back, and instantiates; a launch replays the graph on the caller's stream.
// The position tables are written once at creation (the arrays are fixed).
struct bph_plan {
    int device = 0;
    std::vector<bph_batch *> parts;
    std::vector<int> counts;
    std::vector<void *> d_tab;          // per part: [in counts[p]][out counts[p]] device pointers
    std::vector<cudaStream_t> streams;  // per part (capture only)
    std::vector<cudaEvent_t> joins;     // per part
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // cold, warm
    std::vector<long long> build_id[2];            // schedules captured, per kind and part
    std::vector<long long> launches_part;          // kernel launches of each part per replay
    int launches = 0;
};

namespace bph {

static int plan_record(bph_plan *pl, bool warm) {
    const int np_ = (int)pl->parts.size();
    // schedules first: building one synchronises, which capture forbids
    std::vector<Schedule *> sch((size_t)np_);
    for (int p = 0; p < np_; ++p) {
        int rc = batch_schedule(pl->parts[(size_t)p]->c, warm ? 5 : 20, &sch[(size_t)p]);
        if (rc) return rc;
    }
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate(plan capture)");
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(pl->fork, cs);
    int rc = BPH_OK;
    std::vector<long long> counted((size_t)np_, 0);
    for (int p = 0; p < np_ && e == cudaSuccess && rc == BPH_OK; ++p) {
        bph_batch *b = pl->parts[(size_t)p];
        bph_ctx *c = b->c;
        cudaStream_t sp = pl->streams[(size_t)p];
        e = cudaStreamWaitEvent(sp, pl->fork, 0);
        if (e != cudaSuccess) break;
        cudaStream_t keep = c->stream;
        const bool keep_pdl = c->pdl;
        const long long before = c->launches;
        c->stream = sp;
        c->pdl = false;  // plain edges: each branch starts after an event node
        const char *db = static_cast<const char *>(pl->d_tab[(size_t)p]);
        const int n = pl->counts[(size_t)p];
        rc = batch_enqueue(b, n, reinterpret_cast<const double *const *>(db),
                           reinterpret_cast<double *const *>(db + sizeof(void *) * (size_t)n), nullptr,
                           *sch[(size_t)p], warm, false);
        counted[(size_t)p] = c->launches - before;
        c->launches = before;
        c->stream = keep;
        c->pdl = keep_pdl;
        if (rc == BPH_OK) e = cudaEventRecord(pl->joins[(size_t)p], sp);
        if (e == cudaSuccess && rc == BPH_OK) e = cudaStreamWaitEvent(cs, pl->joins[(size_t)p], 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t ee = cudaStreamEndCapture(cs, &g);
    if (e == cudaSuccess) e = ee;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess && rc == BPH_OK) e = cudaGraphInstantiate(&exec, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    if (rc != BPH_OK) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return rc;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return cuda_fail(e, "plan graph capture");
    }
    const int k = warm ? 1 : 0;
    if (pl->exec[k]) cudaGraphExecDestroy(pl->exec[k]);
    pl->exec[k] = exec;
    pl->build_id[k].clear();
    for (Schedule *x : sch) pl->build_id[k].push_back(x->build_id);
    pl->launches_part = counted;
    long long tot = 0;
    for (long long v : counted) tot += v;
    pl->launches = (int)tot;
    return BPH_OK;
}

}  // namespace bph

extern "C" {

int bph_plan_destroy(bph_plan_t *pl) {
    if (!pl) return BPH_OK;
    ::bph::DeviceScope scope_(pl->device);
    for (cudaGraphExec_t &x : pl->exec)
        if (x) cudaGraphExecDestroy(x);
    for (void *t : pl->d_tab)
        if (t) cudaFree(t);
    for (cudaStream_t s : pl->streams)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t ev : pl->joins)
        if (ev) cudaEventDestroy(ev);
    if (pl->fork) cudaEventDestroy(pl->fork);
    delete pl;
    return BPH_OK;
}

int bph_plan_create(int nparts, bph_batch_t *const *batches, const int *counts, const double *const *const *rho,
                    double *const *const *pot, bph_plan_t **out) {
    if (!out) {
        set_error("out-pointer is NULL");
        return BPH_ERR_INVALID;
    }
    *out = nullptr;
    if (nparts < 1 || nparts > 256 || !batches || !counts || !rho || !pot) {
        set_error("invalid plan arguments (1..256 parts, non-NULL arrays)");
        return BPH_ERR_INVALID;
    }
    for (int p = 0; p < nparts; ++p) {
        const bph_batch *b = batches[p];
        if (!b || counts[p] < 1 || counts[p] > b->cap || !rho[p] || !pot[p]) {
            set_error("plan part %d: NULL batch or arrays, or count outside 1..capacity", p);
            return BPH_ERR_INVALID;
        }
        if (b->c->device != batches[0]->c->device) {
            set_error("plan part %d lives on device %d, part 0 on %d", p, b->c->device, batches[0]->c->device);
            return BPH_ERR_INVALID;
        }
        for (int q = 0; q < p; ++q)
            if (batches[q] == b || batches[q]->c == b->c) {
                set_error("plan parts %d and %d share a batch or a context", q, p);
                return BPH_ERR_INVALID;
            }
        for (int i = 0; i < counts[p]; ++i)
            if (!rho[p][i] || !pot[p][i]) {
                set_error("plan part %d position %d has a NULL array", p, i);
                return BPH_ERR_INVALID;
            }
    }
    bph_plan *pl = new bph_plan();
    pl->device = batches[0]->c->device;
    ::bph::DeviceScope scope_(pl->device);
    cudaError_t e = scope_.status();
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->fork, cudaEventDisableTiming);
    for (int p = 0; p < nparts && e == cudaSuccess; ++p) {
        pl->parts.push_back(batches[p]);
        pl->counts.push_back(counts[p]);
        const int n = counts[p];
        std::vector<const void *> h((size_t)2 * n);
        for (int i = 0; i < n; ++i) {
            h[(size_t)i] = rho[p][i];
            h[(size_t)(n + i)] = pot[p][i];
        }
        void *d = nullptr;
        e = cudaMalloc(&d, sizeof(void *) * h.size());
        pl->d_tab.push_back(d);
        if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), sizeof(void *) * h.size(), cudaMemcpyHostToDevice);
        cudaStream_t s = nullptr;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        pl->streams.push_back(s);
        cudaEvent_t ev = nullptr;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        pl->joins.push_back(ev);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        bph_plan_destroy(pl);
        return cuda_fail(e, "plan creation");
    }
    *out = pl;
    return BPH_OK;
}

int bph_plan_launch(bph_plan_t *pl, int tstep, void *stream) {
    if (!pl) {
        set_error("plan is NULL");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(pl);
    const bool warm = tstep > 1;
    const int k = warm ? 1 : 0;
    // a schedule rebuilt since the recording invalidates the graph
    bool stale = !pl->exec[k];
    for (size_t p = 0; p < pl->parts.size() && !stale; ++p) {
        Schedule *x = nullptr;
        const int rc = batch_schedule(pl->parts[p]->c, warm ? 5 : 20, &x);
        if (rc) return rc;
        stale = x->build_id != pl->build_id[k][p];
    }
    int rc;
    if (stale && (rc = plan_record(pl, warm))) return rc;
    BPH_CUDA(cudaGraphLaunch(pl->exec[k], (cudaStream_t)stream));
    for (size_t p = 0; p < pl->parts.size(); ++p) pl->parts[p]->c->launches += pl->launches_part[p];
    return BPH_OK;
}

int bph_plan_synchronize(bph_plan_t *pl, void *stream) {
    if (!pl) {
        set_error("plan is NULL");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(pl);
    BPH_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    int worst = BPH_OK;
    for (bph_batch *b : pl->parts) {
        const int rc = context_status(b->c);
        if (rc && !worst) worst = rc;
    }
    return worst;
}

int bph_plan_launches(const bph_plan_t *pl) { return pl ? pl->launches : 0; }

}  // extern "C"
