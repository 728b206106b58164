// bph_internal.cuh -- shared definitions of the B200 Poisson solver.
//
// HBM layout of one solve (numr x numz x numphi grid, N = numphi, M = N/2):
//   rho, pot   Fortran column-major (J fastest, then K, then L), the
//              reference's COMMON /poisson/ layout.
//   P          Fourier-slot potential, slot-major P[s][K][J] (same plane
//              layout per slot): interior from the forward FFT / ADI,
//              boundary columns (J=numr, K=numz, K=1 for isym 1) from the
//              Green-function boundary solve.  Slot s holds F_s (s = 0, M)
//              or Re F_s (0 < s < M) or -Im F_{s-M} (s > M), the order
//              helmadi.F90:133-156 gives its slots.  It also carries the
//              warm-start state between calls.
//   R          -4 pi rho_hat on the interior only, R[s][k][j] packed
//              (j = J-2, k = K-2), zero on the zeroed rows of rhop.
//   mom        interior density moments mom[m][cos|sin][p], p = j + nr*k.
//   green      boundary Green tables G[m][b][p].
//   S          boundary moments S[m][b][cos|sin].
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>

#include "bph.h"

namespace bph {

constexpr int kHyprUprBnd = 110;       // pot.h:7
constexpr double kHyprCutoff = 1.025;  // pot.h:5
constexpr int kMaxMmax = 64;
constexpr int kNumSchedules = 3;       // 5 steps (warm), 20 steps (cold), one custom

// Deferred device status bits (d_status).
constexpr int kStatusNonFinite = 1;
constexpr int kStatusTimeout = 2;  // a bounded device wait (bulk-copy barrier) expired

// Segment length of the partitioned line solves in the on-chip ADI kernel.
constexpr int kAdiSeg = 32;
// Factor arrays per line system: 1/bet, a/bet, gam, forward carry, backward carry.
constexpr int kAdiFactors = 5;

// Programmatic dependent launch.  Kernels of a solve are launched with the
// programmatic-serialisation attribute, so a kernel's CTAs may become
// resident while the previous kernel in the stream drains.  Every kernel
// calls pdl_wait() before its first access to memory that an earlier kernel
// of the stream writes (it returns once those kernels have completed and
// their writes are visible; at once when the launch had no such attribute).
// Only read-only set-up data (twiddles, ADI factors, coefficient tables) is
// touched before it.  pdl_trigger() marks the point after a CTA's main work
// (before its final stores) from which the next kernel may launch; a kernel
// without it triggers when it exits.  Triggering at the start instead made
// the 130x98x256 solve 11% slower on B200 (early CTAs of the next kernel
// held SM resources while they waited); triggering late is 1.6% faster than
// no programmatic launch at all.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Packed factor block of one line system of length n in type T, the
// shared-memory layout the segmented ADI kernels read: [1/bet n][a/bet n]
// [(G_j, gam_{j+1}) pairs 2n][K n], padded to 16 bytes so that one bulk copy
// moves it.
template <typename T>
__host__ __device__ inline int packed_block(int n) {
    const int al = 16 / (int)sizeof(T);
    return ((5 * n + al - 1) / al) * al;
}

struct Schedule {
    int nsteps = 0;
    double *d_dt = nullptr;   // [nsteps]
    double *d_rad = nullptr;  // [nsteps][N][kAdiFactors][nr] radial Thomas factors
    double *d_ver = nullptr;  // [nsteps][kAdiFactors][nz]    vertical Thomas factors
    double *h_dt = nullptr;   // host copy of the dt schedule
    // packed blocks ([0]: double, [1]: float): radial [nsteps][N][packed_block(nr)],
    // vertical [nsteps][packed_block(nz)]
    void *d_rad_pk[2] = {nullptr, nullptr};
    void *d_ver_pk[2] = {nullptr, nullptr};
    long long build_id = 0;  // distinct for every schedule built (graphs that captured it)
    // warp-cooperative ADI (bph_adi_warp.cu): segment-interleaved FP64 blocks,
    // radial [nsteps][N][40 nr/8 + 48], vertical [nsteps][40 nz/8 + 48]
    double *d_warp_rad = nullptr;
    double *d_warp_ver = nullptr;
    float *d_warp_rad32 = nullptr;  // the same blocks in float (warp-cooperative refinement kernel)
    float *d_warp_ver32 = nullptr;
};

// Converged-loop state on the device (bph_converge.cu).
struct ConvState {
    double tol, prev, upd;
    int max_cycles, cycles, mixed;
};

// Instantiated while-graph of a converged form and what it captured.
struct ConvGraph {
    cudaGraphExec_t exec = nullptr;
    long long build_id = -1;
    int kind = -1;
};

}  // namespace bph

struct bph_ctx {
    bph_grid_t g;
    int nr = 0, nz = 0, nb = 0, N = 0, M = 0;
    int fm = 1;  // azimuthal frequency of boundary mode m is fm*m (2 for isym 3)
    long long np = 0, nplane = 0, ntot = 0;
    double pi = 0, dz = 0, dphi = 0, drinv = 0, dzinv = 0, dphiinv = 0;
    double gamma = 0, four_pi = 0, factor = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int device = 0;

    // Setup-time constants.
    double *d_green = nullptr;   // [mmax][nb][np]
    double *d_brb = nullptr;     // [N][numr]  radial diagonal without dt
    double *d_elz = nullptr;     // [N][numr]  elambdazb
    double *d_alphar = nullptr;  // [numr]
    double *d_betar = nullptr;   // [numr]
    double *d_bzb = nullptr;     // [numz]
    double *d_qcoef = nullptr;   // [mmax] coefh, [mmax] nu, [mmax][111] dcoefh
    double *d_grid = nullptr;    // rhf_g[numr], rhfinv_g[numr], zhf_g[numz]
    double2 *d_tw = nullptr;     // e^{+2 pi i k / M}, k = 0..M-1
    double2 *d_tw2 = nullptr;    // e^{+2 pi i k / N}, k = 0..M
    double2 *d_ph = nullptr;     // e^{+i pi fm m / N}, m = 0..mmax-1
    bph::Schedule sched[bph::kNumSchedules];

    // Per-solve buffers.
    double *d_R = nullptr;       // [N][np]
    double *d_P = nullptr;       // [N][nplane]
    double *d_prev = nullptr;    // [N][nplane] (converged form only)
    double *d_mom = nullptr;     // [mmax][2][np]
    double *d_S = nullptr;       // [mmax][nb][2]
    double *d_W = nullptr;       // ADI work slabs when they do not fit on chip
    double *d_W2 = nullptr;      // tiled large-grid ADI: the radial half-sweep result [N][np], transposed
    double *d_P2 = nullptr;      // ADI potential slabs when they do not fit on chip
    double *d_red = nullptr;     // reduction scratch
    double *d_rho_stage = nullptr;
    double *d_pot_stage = nullptr;
    double *d_phieff_stage = nullptr;
    int *d_status = nullptr;
    unsigned int *d_ccnt = nullptr;  // contraction arrival counters [mmax][row groups]
    double *d_cpart = nullptr;       // contraction partial sums [split][mmax][nb][2]
    int contract_split = 1;
    // compact Green tables (bph_compact.h) and the contraction that reads them
    int compact = 0;                 // 1: the single-solve contraction streams the compact tables
    double *d_gtile = nullptr;       // symmetric tiles of the top (and bottom) rows [m][set][k][tile][64]
    double *d_gside = nullptr;       // side-row vectors [m][j][U | V][stride]
    double *d_kpart = nullptr;       // partial sums [m][tile parts | side parts]
    unsigned int *d_kcnt = nullptr;  // arrival counters [mmax] + [mmax][tile sets + side groups]

    int adi_smem = 0;            // dynamic shared bytes of the on-chip ADI kernel (0: global variant)
    int adi_seg = 0;             // threads of the segmented on-chip ADI kernel (0: not used)
    int large_kb[2] = {0, 0};    // rows of a grid-wide radial ADI panel, FP64 / FP32 (0: does not fit)
    bool adi_full = false;       // both line lengths are multiples of the segment length
    bool adi_pf = false;         // FP64 segmented ADI with bulk-copy factor prefetch
    bool mixed_pf = false;       // the same for the FP32 forwarding-form refinement kernel
    int adi_mixed_threads = 0;   // threads of the FP32 defect-correction ADI kernels
    int adi_mixed_smem = 0;      // dynamic shared bytes of the one in use (0: mixed form unavailable)
    int adi_mixed_per_sm = 0;    // its resident CTAs per SM
    int mixed_kind = 0;          // refinement ADI in use: BPH_MIXED_ADI_FORWARD or _INCREMENT
    int mixed_smem_kind[6] = {0, 0, 0, 0, 0, 0};    // per kind: dynamic shared bytes (0: does not fit)
    int mixed_per_sm_kind[6] = {0, 0, 0, 0, 0, 0};  // per kind: resident CTAs per SM
    float mixed_tuned_us[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // per kind: setup-time measurement (0: not timed)
    float *d_dir32 = nullptr;  // direct defect solve: E, E^T, zero-padded [nzp][lda] (bph_direct.cu)
    double *d_dirS = nullptr;  // its radial shifts gamma lambda_q per vertical mode (FP64)
    // set-up autotuning (autotune_setup): timings of the candidates, us (0: not timed)
    float tuned_contract_us[2] = {0.f, 0.f};  // full tables, compact tables
    float tuned_fft_us[2] = {0.f, 0.f};       // forward + inverse FFT: regular tiles, dense tiles
    float tuned_adi_us[2] = {0.f, 0.f};       // 5 ADI steps of every slot: segmented, warp-cooperative
    float *d_work32 = nullptr;                // global-memory refinement kernels: [4][N][np] (lazy)
    int adi_threads = 256;
    int fft_smem_fwd = 0, fft_smem_inv = 0;
    bool fft_dense = false;      // FFT tiles compiled for eight CTAs per SM (BPH_FFT_DENSE=1)
    bool have_warm = false;
    bool pdl = true;             // launch solve kernels with programmatic dependent launch
    // Overlapped solve: slots whose mode carries no boundary data (k not a
    // boundary mode fm*m, m < mmax) run their ADI on a low-priority side
    // stream from the end of the forward FFT, beside the contraction.
    bph::ConvState *d_conv = nullptr;  // converged-loop state
    bph::ConvGraph conv[2];            // [0] FP64, [1] mixed converged loop graphs
    bool conv_graph = true;            // run converged loops as device-side while graphs
    bool overlap = false;
    int nfree = 0;                     // slots without boundary data
    int *d_slot_map = nullptr;         // [N]: the nfree free slots, then the dependent ones
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fft = nullptr, ev_free = nullptr, ev_contract = nullptr;
    // SM partitions (green contexts, bph_green.cu): [0] the contraction's,
    // [1] the free-slot ADI's; used by the overlapped solve when set
    bool green = false;
    void *green_ctx[2] = {nullptr, nullptr};
    cudaStream_t green_stream[2] = {nullptr, nullptr};
    int green_sms[2] = {0, 0};
    int green_fail = 0;  // set-up step that failed (0: none or not requested)
    int adi_warp = 0;                  // warp-cooperative FP64 ADI shape (0: not used; bph_adi_warp.cu)
    int adi_warp_smem = 0;             // its dynamic shared bytes
    double *d_warp_coef = nullptr;     // its per-slot (elambdazb, alphaz, betaz) blocks
    int mixed_warp = 0;                // FP32 warp-cooperative refinement kernel available
    float *d_warp_coef32 = nullptr;    // its coefficient blocks
    float *d_r32 = nullptr;            // rounded residual of one solve [N][np] (FP32 warp refinement)
    double *d_scf = nullptr;           // SCF-step mass partials and scale (bph_scf.cu)
    void *noalloc_scratch = nullptr;   // device address of the allocation-free contraction's scratch array
    long long launches = 0;
    size_t bytes = 0;
    // Holders of the device state: the caller's handle (until bph_destroy)
    // and each batch on the context (until bph_batch_destroy); the state is
    // freed when the last one lets go, in whichever order they do.
    std::atomic<int> refs{1};
};

namespace bph {

// Error helpers (bph_api.cu).
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

#define BPH_CUDA(call)                                          \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return ::bph::cuda_fail(_e, #call); \
    } while (0)

}  // namespace bph

#include "bph_device_scope.h"

namespace bph {

// Launch configuration with the programmatic-serialisation attribute when
// the context uses it (attrs must outlive the launch call).
inline cudaLaunchConfig_t launch_config(const bph_ctx *c, dim3 grid, dim3 block, size_t smem,
                                        cudaLaunchAttribute *attrs) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    attrs[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attrs[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attrs;
    cfg.numAttrs = c->pdl ? 1 : 0;
    return cfg;
}

// Launch wrappers (one per kernel family); each returns a cudaError_t of
// the launch and counts it in ctx->launches.
cudaError_t launch_qcoef(bph_ctx *c);
cudaError_t launch_green_tables(bph_ctx *c);
cudaError_t launch_adi_factors(bph_ctx *c, Schedule &s);
// Packed double and float factor blocks of a schedule (after launch_adi_factors).
cudaError_t launch_pack_factors(bph_ctx *c, Schedule &s);
// Optional arguments select batch buffers (R, moments with m-stride, P, instance count).
// status: where a non-finite density is flagged (nullptr: the context's status word).
cudaError_t launch_fft_fwd_rho(bph_ctx *c, const double *rho, double *R = nullptr, double *mom = nullptr,
                               long long mstride = 0, int *status = nullptr);
cudaError_t launch_fft_fwd_pot(bph_ctx *c, const double *pot);
// One launch over npos batch positions: position j reads d_in[j] (device
// table) and writes instance d_inst[j]'s R (at inst * inst_stride from R),
// its moments at mom + j * pos_stride and its non-finite flag at status[j]
// (status_per_pos) or at *status.
cudaError_t launch_fft_fwd_rho_batch(bph_ctx *c, int npos, const double *const *d_in, const int *d_inst, double *R,
                                     long long inst_stride, double *mom, long long mstride, long long pos_stride,
                                     int *status, bool status_per_pos);
// One launch over npos positions: instance d_inst[j]'s slots -> d_out[j].
cudaError_t launch_fft_inv_batch(bph_ctx *c, int npos, double *const *d_out, const int *d_inst, const double *P,
                                 long long inst_stride);
cudaError_t launch_fft_inv(bph_ctx *c, double *pot, double *phieff = nullptr, double omega = 0.0,
                           const double *P = nullptr);
// write_slots: the contraction also writes the Dirichlet slots of P (the
// fused form of launch_boundary_slots, which stays for phase timing).
cudaError_t launch_green_contract(bph_ctx *c, bool write_slots = true);
cudaError_t launch_boundary_slots(bph_ctx *c);
// ninst instances of slot arrays P/R; block row i solves instance d_inst_map[i]
// (nullptr: instance i).
// norms (segmented kernel only): per (instance, slot) |P_new - P_old|^2 and
// |P_new|^2, formed while the result is written back.
cudaError_t launch_adi(bph_ctx *c, const Schedule &s, int step0, int nsteps_run, bool cold, double *P = nullptr,
                       const double *R = nullptr, int ninst = 1, const int *d_inst_map = nullptr,
                       double *norms = nullptr);
// The slots d_slots[0..nslots) of the context's own arrays, on stream st
// (pdl: with programmatic dependent launch on that stream).
cudaError_t launch_adi_slots(bph_ctx *c, const Schedule &s, bool cold, const int *d_slots, int nslots,
                             cudaStream_t st, bool pdl);
cudaError_t launch_adi_defect(bph_ctx *c, const Schedule &s);
// Slots too large for shared memory (bph_adi_large.cu): the drop-in ADI on
// the slot array P with source R, and one FP32 refinement cycle (work area
// c->d_work32: r, delta and two [N][np] buffers).
// ninst instances (row i -> instance d_inst_map[i]); W, Q: scratch of
// ninst * N * np doubles each (nullptr: the context's, one instance).
cudaError_t launch_adi_large(bph_ctx *c, const Schedule &s, int step0, int nsteps_run, bool cold, double *P,
                             const double *R, int ninst = 1, const int *d_inst_map = nullptr, double *W = nullptr,
                             double *Q = nullptr);
cudaError_t launch_adi_defect_large(bph_ctx *c, const Schedule &s);
// The same FP32 refinement cycle for npos batch positions (instance
// d_map[i], nullptr: position = instance) of batch arrays P/R; work: 4 *
// npos * N * np floats; norms by instance * N + slot.
cudaError_t launch_adi_defect_large_batch(bph_ctx *c, const Schedule &s, double *P, const double *R, int npos,
                                         const int *d_map, float *work, double *norms);
// Panel sizes and shared-memory limits of the grid-wide ADI kernels.
int large_configure(bph_ctx *c);
cudaError_t launch_update_norm(bph_ctx *c, double *d_out);
cudaError_t launch_residual_norm(bph_ctx *c, double *d_out);

int adi_configure(bph_ctx *c);
// Converged-solve cycle loop as a CUDA graph while node (bph_converge.cu):
// enqueues the loop on c->stream; the state (cycles, last update) is in
// c->d_conv.  conv_graphs_free releases the graphs and the state.
int conv_loop_device(bph_ctx *c, Schedule &s, bool mixed, double tol, int max_cycles);
void conv_graphs_free(bph_ctx *c);
// Batched solve of batch positions 0..n-1 (bph_batch.cu); instances may be
// nullptr (position i = instance i).  With pos_status (per-position
// BPH_OK / BPH_ERR_NONFINITE) or host arrays the call is synchronous.
// A converged batched call (bph_batch_solve_converged; servers in
// converged mode).
struct BatchConv {
    int nsteps = 0, max_cycles = 0;
    bool cold = false, mixed = false;
    double tol = 0.0;
    int cycles = 0;           // out: cycles run
    double resid = 0.0;       // out: largest relative FP64 residual over the instances
    bool want_resid = false;
    bool report_divergence = true;  // false: per-position status reports bad densities
};
// Norm buffers (FP64: the previous-cycle slot arrays; mixed on grid-wide
// kernels: the FP32 work arrays) of converged batched calls, allocated ahead
// of the first one.
int batch_reserve_converged(bph_batch *b, bool mixed);
int batch_solve_core(bph_batch *b, int n, const int *instances, const double *const *rho, double *const *pot,
                     bool warm, bool on_device, int *pos_status, BatchConv *conv = nullptr);
// Raises the dynamic shared memory limit of kernel fn on the current device
// to at least bytes.  The limit is a process-wide property of the kernel
// while contexts of different grids share kernels, so it only ever grows
// (a context set up later with a smaller need must not lower it).
cudaError_t raise_smem_limit(const void *fn, int bytes);
// FP32 refinement cycle (on-chip kinds) over n batch positions of the
// batch arrays P/R (d_map: instance of each position, nullptr: position =
// instance); per (instance, slot) norms into norms[2 (i N + s) + 0/1].
cudaError_t launch_defect_batch(bph_ctx *c, const Schedule &sch, double *P, const double *R, int n, const int *d_map,
                                double *norms);
// Per (instance, slot) update (|P - prev|^2, |P|^2) or residual (|R - A P|^2,
// |R|^2) norms of n batch positions, indexed as above.
cudaError_t launch_norms_batch(bph_ctx *c, bool residual, const double *P, const double *prev, const double *R, int n,
                               const int *d_map, double *d_out);
// Reads and clears the context's device status word (synchronises its stream).
int context_status(bph_ctx *c);
// Makes kind (BPH_MIXED_ADI_FORWARD / _INCREMENT) the refinement ADI kernel.
int select_mixed_kind(bph_ctx *c, int kind);
// Work area of the global-memory refinement kernel (allocated on first use).
int ensure_mixed_work(bph_ctx *c);
int contract_configure(bph_ctx *c);
// Compact tables: allocation and build at set-up (BPH_COMPACT=0 leaves them
// off), bph_setup.cu builds them.
int compact_configure(bph_ctx *c);
// Direct FP32 defect solve (bph_direct.cu): set-up of its tables, and one
// refinement cycle for nrows block rows (instance of a row: inst_map), in
// one launch with no scratch in global memory.
int direct_configure(bph_ctx *c);
cudaError_t launch_defect_direct(bph_ctx *c, double *P, const double *R, int nrows, const int *inst_map,
                                 double *norms);
cudaError_t launch_green_compact(bph_ctx *c);
// Warp-cooperative FP64 ADI (bph_adi_warp.cu).  warp_configure selects it
// for the grids it covers (c->adi_warp != 0) and packs the per-slot
// coefficients; launch_pack_warp fills a schedule's factor blocks;
// launch_adi_warp runs nsteps_run steps of nslots * nrows slots (block row
// r solves instance inst_map[r], slot slot_map[b] of the row).
int warp_configure(bph_ctx *c);
// SM partitions for the overlapped solve (bph_green.cu): contract_sms SMs
// for the contraction, the rest for the free-slot ADI; leaves c->green
// false when the driver offers no partitions.
int green_setup(bph_ctx *c, int contract_sms);
void green_free(bph_ctx *c);
// SCF-like density update and renormalisation in place (bph_scf.cu);
// d_part: scf_scratch_doubles() of scratch (partials, then scale and mass).
cudaError_t launch_scf_update(bph_ctx *c, double *d_rho, double eps, double mass, unsigned long long seed,
                              int iteration, double *d_part);
size_t scf_scratch_doubles();
size_t warp_block_doubles(int n);
cudaError_t launch_pack_warp(bph_ctx *c, Schedule &s);
// One FP32 refinement cycle of the warp-cooperative kind on nrows instance
// rows of the slot arrays P/R (row r: instance inst_map[r]); per (instance,
// slot) norms into norms[2 (i N + s) + 0/1]; r32: nrows * N * np floats of
// scratch for the rounded residual.
cudaError_t launch_defect_warp(bph_ctx *c, const Schedule &s, double *P, const double *R, int nrows,
                               const int *inst_map, double *norms, float *r32);
cudaError_t launch_adi_warp(bph_ctx *c, const Schedule &s, int step0, int nsteps_run, bool cold, double *P,
                            const double *R, int nrows, const int *inst_map, const int *slot_map, int nslots,
                            double *norms, cudaStream_t st, bool pdl);
// Device address of the allocation-free contraction's file-scope scratch
// array for a context being set up (bph_noalloc.cu).
int noalloc_setup(bph_ctx *c);
int fft_configure(bph_ctx *c);
// Context references (bph_api.cu): a batch takes one at creation and gives
// it back at its destruction; the last release frees the device state.
void ctx_retain(bph_ctx *c);
void ctx_release(bph_ctx *c);

}  // namespace bph
