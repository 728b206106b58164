// bph_boundary.cu -- the boundary potential (bessel.F90:170-488).
//
// k_green_contract: S[m][b] = sum_p G[m][b][p] * (cos, sin moment)[m][p],
// the per-mode contraction of the Green tables with the interior density
// moments (bessel.F90:186-296).  The tables (8 bytes per element, read once
// per solve) dominate the compulsory bytes of a solve, so the kernel is a
// streaming GEMV with two right-hand sides: 16-byte evict-first loads of the
// table rows, the moment vectors (small, L2-resident) read once per CTA
// for BR rows, and a fixed-order CTA reduction (deterministic results).
//
// k_boundary_slots: the Dirichlet data of the ADI sweeps in Fourier-slot
// space.  The reference synthesises the physical boundary potential
//   Phi_B(l) = factor [S_C0 + 2 sum_{m>=1} (S_Cm cos k th_l + S_Sm sin k th_l)],
// th_l = (l - 1/2) dphi, k = fm*m (bessel.F90:399-488), writes it into potp
// and transforms it with the rest of potp (helmadi.F90:159).  For k < N/2
// that transform is exact in closed form:
//   F_0 = N factor S_C0,  F_k = e^{-i pi k/N} N factor (S_Cm + i S_Sm),
// and zero at every other frequency, so the slots are written directly.
#include <cmath>

#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kContractRows = 8;
constexpr int kContractThreads = 256;

// Grid (row groups, mmax, nsplit).  CTA (g, m, k) reduces table rows
// b0..b0+7 of mode m over the k-th slice of the interior zones; the number
// of slices is chosen at setup so that the launch fills whole waves of the
// GPU.  Slices write partial sums, and the last CTA of each (m, group) to
// arrive adds them in slice order (deterministic) and writes S; it also
// resets its arrival counter for the next launch.
// Dirichlet slots of one boundary row, written by the CTA that finishes the
// row's moments (the closed form of k_boundary_slots below, fused so that
// the solve needs no separate launch).  Slots of modes without boundary
// data and the corner columns are zero from set-up and never written.
struct SlotOut {
    double *P;          // slot array [N][nplane], or nullptr: S only
    const double2 *ph;  // (cos, sin) of pi fm m / N
    int numr, numz, nr, nz, M, fm;
    double nfactor;     // N * factor
};

template <bool kVec>
__global__ void __launch_bounds__(kContractThreads, 2)
k_green_contract(const double *__restrict__ G, const double *__restrict__ mom, double *__restrict__ S,
                 long long np, int nb, unsigned int *__restrict__ counters, double *__restrict__ partials,
                 SlotOut so) {
    const int m = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
    const int b0 = blockIdx.x * kContractRows;
    const int nrows = min(kContractRows, nb - b0);
    // slice bounds in units of 2 doubles (16-byte loads) when vectorised
    const long long unit = kVec ? 2 : 1, nu = np / unit;
    const long long chunk = (nu + nsplit - 1) / nsplit;
    const long long u0 = split * chunk, u1 = min(nu, u0 + chunk);
    const double *mc = mom + (2LL * m) * np;
    const double *ms = mom + (2LL * m + 1) * np;
    const double *g0 = G + ((long long)m * nb + b0) * np;
    double ac[kContractRows], as[kContractRows];
#pragma unroll
    for (int r = 0; r < kContractRows; ++r) ac[r] = as[r] = 0.0;
    pdl_wait();
    if (kVec) {
        const double2 *mc2 = reinterpret_cast<const double2 *>(mc);
        const double2 *ms2 = reinterpret_cast<const double2 *>(ms);
        for (long long i = u0 + threadIdx.x; i < u1; i += kContractThreads) {
            double2 g[kContractRows];
#pragma unroll
            for (int r = 0; r < kContractRows; ++r)
                g[r] = (r < nrows) ? __ldcs(reinterpret_cast<const double2 *>(g0 + r * np) + i) : make_double2(0.0, 0.0);
            const double2 vc = __ldg(mc2 + i), vs = __ldg(ms2 + i);
#pragma unroll
            for (int r = 0; r < kContractRows; ++r) {
                ac[r] = fma(g[r].x, vc.x, ac[r]);
                ac[r] = fma(g[r].y, vc.y, ac[r]);
                as[r] = fma(g[r].x, vs.x, as[r]);
                as[r] = fma(g[r].y, vs.y, as[r]);
            }
        }
    } else {
        for (long long i = u0 + threadIdx.x; i < u1; i += kContractThreads) {
            const double vc = __ldg(mc + i), vs = __ldg(ms + i);
#pragma unroll
            for (int r = 0; r < kContractRows; ++r) {
                if (r < nrows) {
                    const double g = __ldcs(g0 + r * np + i);
                    ac[r] = fma(g, vc, ac[r]);
                    as[r] = fma(g, vs, as[r]);
                }
            }
        }
    }
    pdl_trigger();
    __shared__ double red[kContractThreads / 32][2 * kContractRows];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < kContractRows; ++r) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            ac[r] += __shfl_down_sync(0xffffffffu, ac[r], off);
            as[r] += __shfl_down_sync(0xffffffffu, as[r], off);
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < kContractRows; ++r) {
            red[warp][2 * r] = ac[r];
            red[warp][2 * r + 1] = as[r];
        }
    }
    __syncthreads();
    const long long slice_stride = (long long)gridDim.y * nb * 2;
    double v = 0.0;
    if (threadIdx.x < 2 * nrows) {
#pragma unroll
        for (int w = 0; w < kContractThreads / 32; ++w) v += red[w][threadIdx.x];
    }
    // Threads 2r, 2r+1 of warp 0 hold (S_C, S_S) of row b0 + r.
    auto finish = [&](double val) {
        const double other = __shfl_xor_sync(0xffffffffu, val, 1);
        if (threadIdx.x >= 2 * nrows) return;
        const int r = threadIdx.x >> 1, cs = threadIdx.x & 1;
        const double mine = (m == 0 && cs == 1) ? 0.0 : val;
        S[((long long)m * nb + b0 + r) * 2 + cs] = mine;
        if (!so.P) return;
        const double sc = cs ? other : mine;
        const double ss = (m == 0) ? 0.0 : (cs ? mine : other);
        const int b = b0 + r;
        int jz, kz;
        if (b < so.nr) {
            jz = b + 1;
            kz = so.numz - 1;
        } else if (b < so.nr + so.nz) {
            jz = so.numr - 1;
            kz = b - so.nr + 1;
        } else {
            jz = b - so.nr - so.nz + 1;
            kz = 0;
        }
        const long long nplane = (long long)so.numr * so.numz;
        const long long pos = jz + (long long)so.numr * kz;
        const int k = so.fm * m;
        const double2 w = so.ph[m];
        if (cs == 0)
            so.P[(long long)k * nplane + pos] = so.nfactor * (w.x * sc + w.y * ss);
        else if (m > 0)
            so.P[(long long)(so.M + k) * nplane + pos] = so.nfactor * (w.y * sc - w.x * ss);
    };
    if (nsplit == 1) {
        if (threadIdx.x < 32) finish(v);
        return;
    }
    if (threadIdx.x < 2 * nrows) partials[split * slice_stride + ((long long)m * nb + b0) * 2 + threadIdx.x] = v;
    __threadfence();
    __syncthreads();
    const int tile = m * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) last = (atomicAdd(counters + tile, 1u) == (unsigned)(nsplit - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 32) {
        double t = 0.0;
        if (threadIdx.x < 2 * nrows)
            for (int k = 0; k < nsplit; ++k)
                t += __ldcg(partials + k * slice_stride + ((long long)m * nb + b0) * 2 + threadIdx.x);
        finish(t);
    }
    if (threadIdx.x == 0) counters[tile] = 0u;
}

// One thread per (boundary row b, slot s); rows nb.. write the corner
// columns, which stay zero (bessel.F90:417,452: pott(numr)=pots(numz)=0).
__global__ void k_boundary_slots(const double *__restrict__ S, const double2 *__restrict__ ph,
                                 double *__restrict__ P, int numr, int numz, int nr, int nz, int nb, int N,
                                 int mmax, int fm, int isym, double nfactor) {
    const int M = N / 2;
    const int ncorner = (isym == 1) ? 2 : 1;
    pdl_wait();
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)(nb + ncorner) * N) return;
    const int s = (int)(t % N), b = (int)(t / N);
    const long long nplane = (long long)numr * numz;
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
        P[(long long)s * nplane + jz + (long long)numr * kz] = 0.0;
        return;
    }
    const bool imag = s > M;
    const int k = imag ? s - M : s;
    double v = 0.0;
    if (k < M && k % fm == 0 && k / fm < mmax) {
        const int m = k / fm;
        const double sc = S[((long long)m * nb + b) * 2], ss = S[((long long)m * nb + b) * 2 + 1];
        const double2 w = ph[m];  // (cos, sin) of pi k / N
        v = imag ? nfactor * (w.y * sc - w.x * ss) : nfactor * (w.x * sc + w.y * ss);
    }
    P[(long long)s * nplane + jz + (long long)numr * kz] = v;
}

}  // namespace

int contract_configure(bph_ctx *c) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_green_contract<true>, kContractThreads, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const long long slots = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const long long tiles = (long long)c->g.mmax * ((c->nb + kContractRows - 1) / kContractRows);
    // smallest slice count whose last wave is >= 90% full, at least 2048 zones per slice
    int best = 1;
    double best_eff = 0.0;
    for (int k = 1; k <= 16; ++k) {
        if (k > 1 && c->np / k < 2048) break;
        double waves = (double)(tiles * k) / (double)slots;
        double eff = waves / std::ceil(waves);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = k;
        }
        if (eff >= 0.9) break;
    }
    c->contract_split = best;
    return BPH_OK;
}

cudaError_t launch_green_contract(bph_ctx *c, bool write_slots) {
    dim3 grid((unsigned)((c->nb + kContractRows - 1) / kContractRows), (unsigned)c->g.mmax,
              (unsigned)c->contract_split);
    SlotOut so;
    so.P = write_slots ? c->d_P : nullptr;
    so.ph = c->d_ph;
    so.numr = c->g.numr;
    so.numz = c->g.numz;
    so.nr = c->nr;
    so.nz = c->nz;
    so.M = c->M;
    so.fm = c->fm;
    so.nfactor = (double)c->N * c->factor;
    ++c->launches;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, grid, dim3(kContractThreads), 0, attr);
    const double *G = c->d_green, *mom = c->d_mom;
    if (c->np % 2 == 0)
        return cudaLaunchKernelEx(&cfg, k_green_contract<true>, G, mom, c->d_S, c->np, c->nb, c->d_ccnt, c->d_cpart,
                                  so);
    return cudaLaunchKernelEx(&cfg, k_green_contract<false>, G, mom, c->d_S, c->np, c->nb, c->d_ccnt, c->d_cpart, so);
}

cudaError_t launch_boundary_slots(bph_ctx *c) {
    int ncorner = (c->g.isym == 1) ? 2 : 1;
    long long n = (long long)(c->nb + ncorner) * c->N;
    int threads = 256;
    ++c->launches;
    k_boundary_slots<<<(unsigned)((n + threads - 1) / threads), threads, 0, c->stream>>>(
        c->d_S, c->d_ph, c->d_P, c->g.numr, c->g.numz, c->nr, c->nz, c->nb, c->N, c->g.mmax, c->fm, c->g.isym,
        (double)c->N * c->factor);
    return cudaGetLastError();
}

}  // namespace bph
