// bph_green.cu -- SM partitions for the overlapped solve.
//
// The boundary contraction streams 660 MB of Green tables (HBM-bound) and
// the ADI of the slots that carry no boundary data needs only SMs and
// shared memory; both depend only on the forward FFT.  On one stream, or
// on two ordinary streams, the contraction's CTAs take every SM and the
// ADI waits for them to drain (an ADI CTA fills a whole SM).  Green
// contexts split the GPU's SMs into two disjoint partitions: the
// contraction runs on one, the free-slot ADI on the other, at the same
// time.  The slots with boundary data follow on the whole GPU.
//
// The driver entry points come through cudaGetDriverEntryPointByVersion,
// so the library needs no link against the driver library (and loads on
// machines without a GPU).  Anything that fails leaves the partitions off
// and the solve takes its ordinary path.
#include <cuda.h>

#include <cstdlib>

#include "bph_internal.cuh"

namespace bph {
namespace {

using PFN_getDevResource = CUresult(CUDAAPI *)(CUdevice, CUdevResource *, CUdevResourceType);
using PFN_split = CUresult(CUDAAPI *)(CUdevResource *, unsigned int *, const CUdevResource *, CUdevResource *,
                                      unsigned int, unsigned int);
using PFN_genDesc = CUresult(CUDAAPI *)(CUdevResourceDesc *, CUdevResource *, unsigned int);
using PFN_greenCreate = CUresult(CUDAAPI *)(CUgreenCtx *, CUdevResourceDesc, CUdevice, unsigned int);
using PFN_greenDestroy = CUresult(CUDAAPI *)(CUgreenCtx);
using PFN_greenStream = CUresult(CUDAAPI *)(CUstream *, CUgreenCtx, unsigned int, int);
using PFN_streamDestroy = CUresult(CUDAAPI *)(CUstream);

template <typename F>
bool entry(const char *name, F *out) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion(name, &fn, 12080, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        (void)cudaGetLastError();
        return false;
    }
    *out = reinterpret_cast<F>(fn);
    return true;
}

}  // namespace

// Two partitions: `contract_sms` SMs (rounded up by the driver to its
// granularity, a multiple of 8 on this architecture) for the contraction,
// the rest for the free-slot ADI.  0 on success or when partitions are not
// available (c->green stays false); an error only for CUDA failures after
// partial creation.
int green_setup(bph_ctx *c, int contract_sms) {
    c->green = false;
    c->green_fail = 1;  // driver entry points
    PFN_getDevResource getRes;
    PFN_split split;
    PFN_genDesc gen;
    PFN_greenCreate create;
    PFN_greenStream mkstream;
    if (!entry("cuDeviceGetDevResource", &getRes) || !entry("cuDevSmResourceSplitByCount", &split) ||
        !entry("cuDevResourceGenerateDesc", &gen) || !entry("cuGreenCtxCreate", &create) ||
        !entry("cuGreenCtxStreamCreate", &mkstream))
        return BPH_OK;
    CUdevResource all, part[1], rest;
    c->green_fail = 2;  // device SM resource
    if (getRes((CUdevice)c->device, &all, CU_DEV_RESOURCE_TYPE_SM) != CUDA_SUCCESS) return BPH_OK;
    c->green_fail = 3;  // split
    unsigned int ngroups = 1;
    if (split(part, &ngroups, &all, &rest, 0, (unsigned)contract_sms) != CUDA_SUCCESS || ngroups != 1) return BPH_OK;
    if (rest.sm.smCount < 8) return BPH_OK;
    CUdevResourceDesc da, db;
    c->green_fail = 4;  // descriptors
    if (gen(&da, &part[0], 1) != CUDA_SUCCESS || gen(&db, &rest, 1) != CUDA_SUCCESS) return BPH_OK;
    CUgreenCtx ga = nullptr, gb = nullptr;
    c->green_fail = 5;  // green contexts
    if (create(&ga, da, (CUdevice)c->device, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS) return BPH_OK;
    if (create(&gb, db, (CUdevice)c->device, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS) {
        PFN_greenDestroy destroy;
        if (entry("cuGreenCtxDestroy", &destroy)) destroy(ga);
        return BPH_OK;
    }
    CUstream sa = nullptr, sb = nullptr;
    c->green_fail = 6;  // streams
    if (mkstream(&sa, ga, CU_STREAM_NON_BLOCKING, 0) != CUDA_SUCCESS ||
        mkstream(&sb, gb, CU_STREAM_NON_BLOCKING, 0) != CUDA_SUCCESS) {
        c->green_ctx[0] = ga;
        c->green_ctx[1] = gb;
        c->green_stream[0] = (cudaStream_t)sa;
        c->green_stream[1] = (cudaStream_t)sb;
        green_free(c);
        return BPH_OK;
    }
    c->green_ctx[0] = ga;
    c->green_ctx[1] = gb;
    c->green_stream[0] = (cudaStream_t)sa;
    c->green_stream[1] = (cudaStream_t)sb;
    c->green_sms[0] = (int)part[0].sm.smCount;
    c->green_sms[1] = (int)rest.sm.smCount;
    c->green = true;
    c->green_fail = 0;
    return BPH_OK;
}

void green_free(bph_ctx *c) {
    PFN_streamDestroy sdestroy;
    PFN_greenDestroy gdestroy;
    const bool hs = entry("cuStreamDestroy_v2", &sdestroy) || entry("cuStreamDestroy", &sdestroy);
    const bool hg = entry("cuGreenCtxDestroy", &gdestroy);
    for (int i = 0; i < 2; ++i) {
        if (c->green_stream[i]) {
            cudaStreamSynchronize(c->green_stream[i]);
            if (hs) sdestroy((CUstream)c->green_stream[i]);
            c->green_stream[i] = nullptr;
        }
        if (c->green_ctx[i] && hg) gdestroy((CUgreenCtx)c->green_ctx[i]);
        c->green_ctx[i] = nullptr;
    }
    c->green = false;
}

}  // namespace bph
