// bph_converge.cu -- the cycle loop of the converged solves on the device.
//
// A converged solve repeats an ADI cycle until the potential stops
// changing: FP64 (bph_solve_converged) copies the slot array, runs nsteps
// ADI steps and measures ||phi - phi_prev|| / ||phi||; the mixed form
// (bph_solve_converged_mixed) runs one FP32 refinement cycle that reports
// ||delta|| / ||phi|| itself.  Instead of a host round trip per cycle, the
// cycle is the body of a CUDA graph `while` node: after each cycle
// k_conv_check reduces the per-slot norms, applies the stopping rule and sets
// the node's condition, so the whole loop is one graph launch and the host
// reads the cycle count once at the end.  The graph is built by stream
// capture of the same launchers the host loop uses, once per context,
// schedule and kernel choice.
#include <cmath>

#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kCheckThreads = 256;

__global__ void k_conv_init(ConvState *st, double tol, int max_cycles, int mixed) {
    st->tol = tol;
    st->prev = INFINITY;
    st->upd = INFINITY;
    st->max_cycles = max_cycles;
    st->cycles = 0;
    st->mixed = mixed;
}

// red[2 i] = sum over slot i of |update|^2, red[2 i + 1] = |phi|^2 (Parseval
// weights included).  Fixed-order reduction (deterministic).
__global__ void __launch_bounds__(kCheckThreads) k_conv_check(const double *__restrict__ red, int N, ConvState *st,
                                                              cudaGraphConditionalHandle cond) {
    __shared__ double sn[kCheckThreads], sd[kCheckThreads];
    double num = 0.0, den = 0.0;
    for (int i = threadIdx.x; i < N; i += kCheckThreads) {
        num += red[2 * i];
        den += red[2 * i + 1];
    }
    sn[threadIdx.x] = num;
    sd[threadIdx.x] = den;
    __syncthreads();
    for (int w = kCheckThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sn[threadIdx.x] += sn[threadIdx.x + w];
            sd[threadIdx.x] += sd[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double upd = sd[0] > 0.0 ? sqrt(sn[0] / sd[0]) : sqrt(sn[0]);
        const int cyc = st->cycles + 1;
        // Stop at the tolerance or the cycle limit; the mixed form also when a
        // cycle no longer halves the update (its FP32 solves are then at
        // their accuracy) or the update is not finite.
        bool stop = (upd <= st->tol) || (cyc >= st->max_cycles);
        if (st->mixed) stop = stop || !(upd == upd) || (upd > 0.5 * st->prev);
        st->cycles = cyc;
        st->upd = upd;
        st->prev = upd;
        cudaGraphSetConditional(cond, stop ? 0u : 1u);
    }
}

}  // namespace

// Builds the while-graph of one converged form on the context's current
// arrays and schedule s (the cycle body captured from the launchers).
static int build_conv_graph(bph_ctx *c, Schedule &s, bool mixed, cudaGraphExec_t *out) {
    *out = nullptr;
    cudaGraph_t g = nullptr;
    cudaStream_t cs = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    cudaGraphConditionalHandle cond = 0;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams p = {};
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) {
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = cond;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(cs, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaStream_t keep = c->stream;
        const bool keep_pdl = c->pdl;
        c->stream = cs;
        c->pdl = false;  // plain serial edges inside the loop body
        cudaError_t ce = cudaSuccess;
        if (mixed) {
            ce = launch_adi_defect(c, s);
        } else if (c->adi_seg) {  // the update norms come from the sweep's write-back
            ce = launch_adi(c, s, 0, s.nsteps, false, nullptr, nullptr, 1, nullptr, c->d_red);
        } else {
            ce = cudaMemcpyAsync(c->d_prev, c->d_P, sizeof(double) * (size_t)c->N * c->nplane,
                                 cudaMemcpyDeviceToDevice, cs);
            if (ce == cudaSuccess) ce = launch_adi(c, s, 0, s.nsteps, false);
            if (ce == cudaSuccess) ce = launch_update_norm(c, c->d_red);
        }
        if (ce == cudaSuccess) {
            k_conv_check<<<1, kCheckThreads, 0, cs>>>(c->d_red, c->N, c->d_conv, cond);
            ce = cudaGetLastError();
        }
        ++c->launches;
        c->stream = keep;
        c->pdl = keep_pdl;
        cudaGraph_t body = nullptr;
        e = cudaStreamEndCapture(cs, &body);
        if (e == cudaSuccess) e = ce;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
    if (cs) cudaStreamDestroy(cs);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return cuda_fail(e, "converged-loop graph");
    }
    *out = exec;
    return BPH_OK;
}

int conv_loop_device(bph_ctx *c, Schedule &s, bool mixed, double tol, int max_cycles) {
    int rc;
    if (!c->d_conv) {
        cudaError_t e = cudaMalloc((void **)&c->d_conv, sizeof(ConvState));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cuda_fail(e, "cudaMalloc(converged-loop state)");
        }
        c->bytes += sizeof(ConvState);
    }
    ConvGraph &cg = c->conv[mixed ? 1 : 0];
    const int kind = mixed ? (c->mixed_kind * 2 + (c->mixed_pf ? 1 : 0)) : 0;
    if (!cg.exec || cg.build_id != s.build_id || cg.kind != kind) {
        if (cg.exec) cudaGraphExecDestroy(cg.exec);
        cg.exec = nullptr;
        if ((rc = build_conv_graph(c, s, mixed, &cg.exec))) return rc;
        cg.build_id = s.build_id;
        cg.kind = kind;
    }
    ++c->launches;
    k_conv_init<<<1, 1, 0, c->stream>>>(c->d_conv, tol, max_cycles, mixed ? 1 : 0);
    BPH_CUDA(cudaGetLastError());
    BPH_CUDA(cudaGraphLaunch(cg.exec, c->stream));
    return BPH_OK;
}

void conv_graphs_free(bph_ctx *c) {
    for (ConvGraph &cg : c->conv) {
        if (cg.exec) cudaGraphExecDestroy(cg.exec);
        cg = ConvGraph();
    }
    if (c->d_conv) cudaFree(c->d_conv);
    c->d_conv = nullptr;
}

}  // namespace bph
