// bph_noalloc.cu -- boundary contraction that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need the
// boundary moments: code that runs inside a region where the allocator is
// off limits (an application-owned memory pool that must not grow, a
// real-time loop in which cudaMalloc's implicit device synchronisation is
// not acceptable, or host code that only holds pointers handed to it by
// its caller).  bph_green_contract_noalloc serves them: the caller passes
// the inputs (a context whose tables were built earlier, and the density
// moments) and the output array, and the kernel's scratch -- split-K
// partial sums and per-tile arrival counters -- lives in the file-scope
// array below, which every GPU that loads this library holds until the
// process exits.
//
// The scratch is shared by all calls on a device and keeps the last call's
// contents; the counters are cleared on the stream before every launch.
// Calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on the scratch and must be serialised by
// the caller.
//
// In host code the name bph_noalloc_scratch is a host-side stand-in, not a
// device address: bph_setup resolves the array's device address once for
// its context (noalloc_setup, with the context's device current) and the
// entry point passes that address to the kernel, so the call path itself
// makes no runtime lookup.
#include "bph_internal.cuh"
#include "bph_noalloc_plan.h"

namespace bph {
namespace {

using noalloc::kCounterBytes;
using noalloc::kRows;
constexpr int kThreads = 256;

static __device__ __align__(256) unsigned char bph_noalloc_scratch[noalloc::kScratchBytes];

// Grid (row groups, mmax, splits).  Each CTA reduces its p-range for kRows
// boundary rows of one mode into partials[split][m][b][2]; the last CTA of a
// (m, row group) to arrive sums the partials in split order (deterministic)
// and writes S.
__global__ void __launch_bounds__(kThreads)
k_green_contract_splitk(const double *__restrict__ G, const double *__restrict__ mom, double *__restrict__ S,
                        long long np, int nb, int nsplit, unsigned int *__restrict__ counters,
                        double *__restrict__ partials) {
    const int m = blockIdx.y, split = blockIdx.z, mmax = gridDim.y;
    const int b0 = blockIdx.x * kRows;
    const int nrows = min(kRows, nb - b0);
    const long long chunk = (np + nsplit - 1) / nsplit;
    const long long p_begin = split * chunk, p_end = min(np, p_begin + chunk);
    const double *mc = mom + (2LL * m) * np, *ms = mom + (2LL * m + 1) * np;
    const double *g0 = G + ((long long)m * nb + b0) * np;
    double ac[kRows], as[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) ac[r] = as[r] = 0.0;
    for (long long i = p_begin + threadIdx.x; i < p_end; i += kThreads) {
        double vc = __ldg(mc + i), vs = __ldg(ms + i);
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            if (r < nrows) {
                double g = __ldcs(g0 + r * np + i);
                ac[r] = fma(g, vc, ac[r]);
                as[r] = fma(g, vs, as[r]);
            }
        }
    }
    __shared__ double red[kThreads / 32][2 * kRows];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            ac[r] += __shfl_down_sync(0xffffffffu, ac[r], off);
            as[r] += __shfl_down_sync(0xffffffffu, as[r], off);
        }
    if (lane == 0)
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            red[warp][2 * r] = ac[r];
            red[warp][2 * r + 1] = as[r];
        }
    __syncthreads();
    const long long tile_stride = (long long)mmax * nb * 2;
    if (threadIdx.x < 2 * nrows) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) v += red[w][threadIdx.x];
        partials[split * tile_stride + ((long long)m * nb + b0) * 2 + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    const int tile = m * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) last = (atomicAdd(counters + tile, 1u) == (unsigned)(nsplit - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 2 * nrows) {
        double v = 0.0;
        for (int s = 0; s < nsplit; ++s)
            v += __ldcg(partials + s * tile_stride + ((long long)m * nb + b0) * 2 + threadIdx.x);
        int r = threadIdx.x >> 1, cs = threadIdx.x & 1;
        S[((long long)m * nb + b0 + r) * 2 + cs] = (m == 0 && cs == 1) ? 0.0 : v;
    }
    if (threadIdx.x == 0) counters[tile] = 0u;
}

}  // namespace

// Resolves the device address of the scratch array for a context being set
// up (its device is current).  Every context holds its own copy, so a
// context created after a device reset sees the array where the reloaded
// module put it.
int noalloc_setup(bph_ctx *c) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, bph_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(bph_noalloc_scratch)");
    c->noalloc_scratch = p;
    return BPH_OK;
}

}  // namespace bph

extern "C" int bph_green_contract_noalloc(bph_ctx_t *c, const double *d_mom, double *d_S) {
    using namespace bph;
    if (!c) {
        set_error("context is NULL");
        return BPH_ERR_INVALID;
    }
    if (!d_mom || !d_S) {
        set_error("d_mom and d_S must be device arrays");
        return BPH_ERR_INVALID;
    }
    const int mmax = c->g.mmax, nb = c->nb;
    noalloc::Plan plan;
    if (!noalloc::plan(mmax, nb, c->np, &plan)) {
        set_error("grid too large for the %zu-byte no-allocation scratch (mmax*nb = %d; limit %zu tiles, "
                  "%zu partial doubles per split)",
                  noalloc::kScratchBytes, mmax * nb, kCounterBytes / sizeof(unsigned int),
                  noalloc::partial_capacity());
        return BPH_ERR_INVALID;
    }
    if (!c->noalloc_scratch) {
        set_error("the context has no scratch address (bph_setup did not complete)");
        return BPH_ERR_STATE;
    }
    BPH_DEVICE_SCOPE(c);
    unsigned int *counters = reinterpret_cast<unsigned int *>(c->noalloc_scratch);
    double *partials = reinterpret_cast<double *>(static_cast<unsigned char *>(c->noalloc_scratch) + kCounterBytes);
    cudaError_t e = cudaMemsetAsync(counters, 0, plan.tiles * sizeof(unsigned int), c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(counters)");
    dim3 grid((unsigned)plan.groups, (unsigned)mmax, (unsigned)plan.nsplit);
    k_green_contract_splitk<<<grid, kThreads, 0, c->stream>>>(c->d_green, d_mom, d_S, c->np, nb, plan.nsplit,
                                                             counters, partials);
    ++c->launches;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_green_contract_splitk");
    return BPH_OK;
}
