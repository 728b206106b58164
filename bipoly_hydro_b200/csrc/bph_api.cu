// bph_api.cu -- the C ABI (include/bph.h): context setup (potsetup.F90),
// the solve driver (potential_solver.F90) and its host/device entry points.
//
// One solve is five kernels on the context's stream:
//   k_fft_fwd<rho>     rho -> R = -4 pi rho_hat (slot-major) + moments
//   k_green_contract   moments x Green tables -> S
//   k_boundary_slots   S -> Dirichlet slots of P (top, side, bottom)
//   k_adi              nsteps ADI steps per slot on P
//   k_fft_inv          P -> pot, with the axis and equator conditions
// A warm start reuses the Fourier-space potential P of the previous solve,
// which is what the reference's forward transform of its kept potp gives
// (helmadi.F90:159) up to rounding, so no forward transform of the old
// potential is needed.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bph_compact.h"
#include "bph_internal.cuh"

namespace bph {

static thread_local char g_err[512];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error("CUDA error in %s: %s (%d)", what, cudaGetErrorString(e), (int)e);
    return (e == cudaErrorMemoryAllocation) ? BPH_ERR_NOMEM : BPH_ERR_CUDA;
}

namespace {

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

template <typename T>
int dev_alloc(bph_ctx *c, T **p, size_t count) {
    size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return BPH_ERR_NOMEM;
    }
    c->bytes += bytes;
    return BPH_OK;
}

void dev_free(void *p) {
    if (p) cudaFree(p);
}

// Grid coordinates (setup_frac.F90:374-463, one rank) and the ADI
// coefficient arrays (potsetup.F90:151-252), evaluated on the host in the
// reference's expression order: they are O(numr*numphi) setup constants.
struct HostCoef {
    std::vector<double> r_g, rhf_g, rinv_g, rhfinv_g, zhf_g;
    std::vector<double> alphar, betar, brb, elz, bzb;
};

void host_coefficients(bph_ctx *c, HostCoef &h) {
    const bph_grid_t &g = c->g;
    const int numr = g.numr, numz = g.numz, N = g.numphi;
    h.r_g.assign(numr, 0.0);
    h.rhf_g.assign(numr, 0.0);
    h.rinv_g.assign(numr, 0.0);
    h.rhfinv_g.assign(numr, 0.0);
    h.zhf_g.assign(numz, 0.0);
    double x = 1.0;
    for (int J = 1; J <= numr; ++J) {
        h.r_g[J - 1] = (x - 2.0) * g.dr;
        x = x + 1.0;
    }
    for (int J = 1; J <= numr; ++J) {
        h.rhf_g[J - 1] = h.r_g[J - 1] + 0.5 * g.dr;
        h.rinv_g[J - 1] = (h.r_g[J - 1] != 0.0) ? 1.0 / h.r_g[J - 1] : 0.0;
        h.rhfinv_g[J - 1] = 1.0 / h.rhf_g[J - 1];
    }
    x = 1.0;
    double offset = (g.isym != 1) ? 0.0 : -(double)(numz / 2) * c->dz;
    for (int K = 1; K <= numz; ++K) {
        h.zhf_g[K - 1] = (g.isym != 1) ? (x - 1.5) * c->dz : offset + (x - 0.5) * c->dz;
        x = x + 1.0;
    }
    const double drinv2 = c->drinv * c->drinv, dphiinv2 = c->dphiinv * c->dphiinv;
    h.alphar.assign(numr, 0.0);
    h.betar.assign(numr, 0.0);
    for (int J = 2; J <= numr - 1; ++J) {
        h.alphar[J - 1] = -h.r_g[J] * h.rhfinv_g[J - 1] * drinv2;
        h.betar[J - 1] = -h.r_g[J - 1] * h.rhfinv_g[J - 1] * drinv2;
    }
    h.brb.assign((size_t)N * numr, 0.0);
    h.elz.assign((size_t)N * numr, 0.0);
    const int lstop = N / 2 + 1;
    for (int L = 1; L <= N; ++L) {
        int mode;
        if (g.isym == 3)
            mode = (L <= lstop) ? (L - 1) * (L - 1) : (L - lstop) * (L - lstop);
        else
            mode = (L <= lstop) ? L - 1 : L - lstop;
        double m1mode = (mode % 2 == 0) ? 1.0 : -1.0;
        double em1 = std::cos((double)mode * c->dphi) - 1.0;
        double *brb = h.brb.data() + (size_t)(L - 1) * numr;
        double *elz = h.elz.data() + (size_t)(L - 1) * numr;
        for (int J = 3; J <= numr - 1; ++J)
            brb[J - 1] = 2.0 * drinv2 - 2.0 * em1 * dphiinv2 * h.rhfinv_g[J - 1] * h.rhfinv_g[J - 1];
        double az2 = 2.0 * em1 * dphiinv2 * h.rhfinv_g[1] * h.rhfinv_g[1];
        if (g.isym == 3)
            brb[1] = -h.alphar[1] - 2.0 * h.betar[1] - az2;
        else
            brb[1] = -h.alphar[1] + (m1mode - 1.0) * h.betar[1] - az2;
        for (int J = 2; J <= numr - 1; ++J)
            elz[J - 1] = -2.0 * drinv2 + 2.0 * em1 * dphiinv2 * h.rhfinv_g[J - 1] * h.rhfinv_g[J - 1];
        if (g.isym == 3)
            elz[1] = h.alphar[1] + 2.0 * h.betar[1] + az2;
        else
            elz[1] = h.alphar[1] - (m1mode - 1.0) * h.betar[1] + az2;
    }
    h.bzb.assign(numz, 0.0);
    for (int K = 2; K <= numz - 1; ++K) h.bzb[K - 1] = 2.0 * c->gamma;
    if (g.isym != 1) h.bzb[1] = c->gamma;
}

// dt schedule of helmadi.F90:124-129.
void dt_schedule(const HostCoef &h, int numr, int nsteps, double *dt) {
    dt[nsteps - 1] = 4.0 * (h.rinv_g[numr - 1] * h.rinv_g[numr - 1]);
    double alph = std::pow(h.r_g[numr - 1] * h.rinv_g[2], 2.0 / ((double)nsteps - 1.0));
    for (int I = 2; I <= nsteps; ++I) {
        int idx = nsteps + 1 - I;
        dt[idx - 1] = alph * dt[idx];
    }
}

void free_schedule(bph_ctx *c, Schedule &s) {
    dev_free(s.d_dt);
    dev_free(s.d_rad);
    dev_free(s.d_ver);
    for (int k = 0; k < 2; ++k) {
        dev_free(s.d_rad_pk[k]);
        dev_free(s.d_ver_pk[k]);
    }
    dev_free(s.d_warp_rad);
    dev_free(s.d_warp_ver);
    dev_free(s.d_warp_rad32);
    dev_free(s.d_warp_ver32);
    free(s.h_dt);
    s = Schedule();
    (void)c;
}

// Builds (or returns the cached) schedule for nsteps ADI steps.
int get_schedule(bph_ctx *c, int nsteps, Schedule **out) {
    for (auto &s : c->sched)
        if (s.nsteps == nsteps) {
            *out = &s;
            return BPH_OK;
        }
    Schedule &s = (nsteps == 5) ? c->sched[0] : (nsteps == 20) ? c->sched[1] : c->sched[2];
    if (s.nsteps) free_schedule(c, s);
    HostCoef h;
    host_coefficients(c, h);
    s.h_dt = (double *)malloc(sizeof(double) * nsteps);
    dt_schedule(h, c->g.numr, nsteps, s.h_dt);
    int rc;
    if ((rc = dev_alloc(c, &s.d_dt, nsteps))) return rc;
    if ((rc = dev_alloc(c, &s.d_rad, (size_t)nsteps * c->N * kAdiFactors * c->nr))) return rc;
    if ((rc = dev_alloc(c, &s.d_ver, (size_t)nsteps * kAdiFactors * c->nz))) return rc;
    BPH_CUDA(cudaMemcpyAsync(s.d_dt, s.h_dt, sizeof(double) * nsteps, cudaMemcpyHostToDevice, c->stream));
    s.nsteps = nsteps;
    static long long next_build_id = 1;
    s.build_id = next_build_id++;
    BPH_CUDA(launch_adi_factors(c, s));
    {
        double *r64, *v64;
        float *r32, *v32;
        if ((rc = dev_alloc(c, &r64, (size_t)nsteps * c->N * packed_block<double>(c->nr)))) return rc;
        s.d_rad_pk[0] = r64;
        if ((rc = dev_alloc(c, &v64, (size_t)nsteps * packed_block<double>(c->nz)))) return rc;
        s.d_ver_pk[0] = v64;
        if ((rc = dev_alloc(c, &r32, (size_t)nsteps * c->N * packed_block<float>(c->nr)))) return rc;
        s.d_rad_pk[1] = r32;
        if ((rc = dev_alloc(c, &v32, (size_t)nsteps * packed_block<float>(c->nz)))) return rc;
        s.d_ver_pk[1] = v32;
    }
    BPH_CUDA(launch_pack_factors(c, s));
    if (c->adi_warp) {
        if ((rc = dev_alloc(c, &s.d_warp_rad, (size_t)nsteps * c->N * warp_block_doubles(c->nr)))) return rc;
        if ((rc = dev_alloc(c, &s.d_warp_ver, (size_t)nsteps * warp_block_doubles(c->nz)))) return rc;
        if (c->mixed_warp) {
            if ((rc = dev_alloc(c, &s.d_warp_rad32, (size_t)nsteps * c->N * warp_block_doubles(c->nr)))) return rc;
            if ((rc = dev_alloc(c, &s.d_warp_ver32, (size_t)nsteps * warp_block_doubles(c->nz)))) return rc;
        }
        BPH_CUDA(launch_pack_warp(c, s));
    }
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    *out = &s;
    return BPH_OK;
}

int validate(const bph_grid_t *g) {
    if (!g) {
        set_error("grid is NULL");
        return BPH_ERR_INVALID;
    }
    if (g->numr < 5 || g->numz < 5) {
        set_error("numr and numz must be >= 5 (got %d, %d)", g->numr, g->numz);
        return BPH_ERR_INVALID;
    }
    if (!is_pow2(g->numphi) || g->numphi < 16 || g->numphi > 512) {
        set_error("numphi must be a power of two in [16, 512] (got %d)", g->numphi);
        return BPH_ERR_INVALID;
    }
    if (g->isym < 1 || g->isym > 3) {
        set_error("isym must be 1, 2 or 3 (got %d)", g->isym);
        return BPH_ERR_INVALID;
    }
    if (g->mmax < 2 || g->mmax > kMaxMmax) {
        set_error("mmax must be in [2, %d] (got %d)", kMaxMmax, g->mmax);
        return BPH_ERR_INVALID;
    }
    int fm = (g->isym == 3) ? 2 : 1;
    if (fm * (g->mmax - 1) >= g->numphi / 2) {
        set_error("numphi=%d too small for mmax=%d (need numphi/2 > %d*(mmax-1))", g->numphi, g->mmax, fm);
        return BPH_ERR_INVALID;
    }
    if (!(g->dr > 0.0) || !std::isfinite(g->dr)) {
        set_error("dr must be positive and finite");
        return BPH_ERR_INVALID;
    }
    return BPH_OK;
}

int upload(bph_ctx *c, void *dst, const void *src, size_t bytes) {
    BPH_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return BPH_OK;
}
// Times each fitting refinement ADI kernel (one 5-step cycle over the
// zeroed slot array: r = 0, so the state stays zero) and keeps the faster.
// Set-up autotuning of the per-grid kernel choices: the boundary contraction
// (compact or full tables), the FFT tiles (regular or dense) and the FP64
// ADI kernel (warp-cooperative or segmented, where both apply).  Each
// candidate runs once untimed and three times timed on zero data, and the
// faster stays; BPH_COMPACT, BPH_FFT_DENSE and BPH_ADI_WARP in the
// environment force their choice, BPH_AUTOTUNE=0 skips all of it.
int autotune_setup(bph_ctx *c) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    auto timed = [&](auto &&launch, float *us) {
        if (e == cudaSuccess) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        *us = 1e3f * ms / 3.f;
    };
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_P, 0, sizeof(double) * (size_t)c->N * c->nplane, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_mom, 0, sizeof(double) * 2 * (size_t)c->g.mmax * c->np, c->stream);
    // boundary contraction
    if (e == cudaSuccess && c->compact && !std::getenv("BPH_COMPACT")) {
        c->compact = 0;
        timed([&] { return launch_green_contract(c); }, &c->tuned_contract_us[0]);
        c->compact = 1;
        timed([&] { return launch_green_contract(c); }, &c->tuned_contract_us[1]);
        c->compact = (c->tuned_contract_us[1] <= c->tuned_contract_us[0]) ? 1 : 0;
    }
    // FFT tiles: the forward transform of a zero field, the inverse into scratch
    if (e == cudaSuccess && !std::getenv("BPH_FFT_DENSE")) {
        double *scratch = nullptr;
        e = cudaMalloc((void **)&scratch, sizeof(double) * (size_t)c->ntot);
        for (int dense = 0; dense < 2 && e == cudaSuccess; ++dense) {
            c->fft_dense = dense != 0;
            timed(
                [&] {
                    cudaError_t f = launch_fft_fwd_rho(c, c->d_P);
                    return f == cudaSuccess ? launch_fft_inv(c, scratch) : f;
                },
                &c->tuned_fft_us[dense]);
        }
        c->fft_dense = c->tuned_fft_us[1] < c->tuned_fft_us[0];
        if (scratch) {
            cudaStreamSynchronize(c->stream);
            cudaFree(scratch);
        }
    }
    // FP64 ADI kernel
    if (e == cudaSuccess && c->adi_warp && c->adi_seg && !std::getenv("BPH_ADI_WARP")) {
        Schedule *s;
        int rc = get_schedule(c, 5, &s);
        if (rc) return rc;
        const int shape = c->adi_warp;
        c->adi_warp = 0;
        timed([&] { return launch_adi(c, *s, 0, 5, false); }, &c->tuned_adi_us[0]);
        c->adi_warp = shape;
        timed([&] { return launch_adi(c, *s, 0, 5, false); }, &c->tuned_adi_us[1]);
        if (c->tuned_adi_us[0] < c->tuned_adi_us[1]) c->adi_warp = 0;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "set-up autotune");
    BPH_CUDA(cudaMemsetAsync(c->d_P, 0, sizeof(double) * (size_t)c->N * c->nplane, c->stream));
    BPH_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    return BPH_OK;
}

int autotune_mixed(bph_ctx *c) {
    const int kinds[4] = {BPH_MIXED_ADI_FORWARD, BPH_MIXED_ADI_INCREMENT, BPH_MIXED_ADI_WARP, BPH_MIXED_DIRECT};
    int avail = 0;
    for (int k : kinds) avail += c->mixed_smem_kind[k] ? 1 : 0;
    if (avail < 2) return BPH_OK;
    // one refinement cycle of the converged forms' usual length (10 steps): the kinds
    // differ in per-launch work (the warp kind adds its residual kernel), so a short
    // schedule would favour the others
    Schedule *s;
    int rc;
    if ((rc = get_schedule(c, 10, &s))) return rc;
    BPH_CUDA(cudaMemsetAsync(c->d_R, 0, sizeof(double) * (size_t)c->N * c->np, c->stream));
    BPH_CUDA(cudaMemsetAsync(c->d_P, 0, sizeof(double) * (size_t)c->N * c->nplane, c->stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int best = c->mixed_kind;
    float best_ms = 0.f;
    bool first = true;
    for (int k : kinds) {
        if (e != cudaSuccess) break;
        if (!c->mixed_smem_kind[k]) continue;
        select_mixed_kind(c, k);
        e = launch_adi_defect(c, *s);
        if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch_adi_defect(c, *s);
        if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) break;
        c->mixed_tuned_us[k] = 1e3f * ms / 3.f;
        if (first || ms < best_ms) {
            best = k;
            best_ms = ms;
            first = false;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "refinement ADI autotune");
    BPH_CUDA(cudaMemsetAsync(c->d_P, 0, sizeof(double) * (size_t)c->N * c->nplane, c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    return select_mixed_kind(c, best);
}


int setup_impl(bph_ctx *c) {
    const bph_grid_t &g = c->g;
    int rc;
    BPH_CUDA(cudaGetDevice(&c->device));
    BPH_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    c->nr = g.numr - 2;
    c->nz = g.numz - 2;
    c->nb = (g.isym == 1) ? 2 * c->nr + c->nz : c->nr + c->nz;
    c->N = g.numphi;
    c->M = g.numphi / 2;
    c->fm = (g.isym == 3) ? 2 : 1;
    c->np = (long long)c->nr * c->nz;
    c->nplane = (long long)g.numr * g.numz;
    c->ntot = c->nplane * g.numphi;
    c->pi = std::acos(-1.0);
    c->dz = g.dr;
    c->dphi = 2.0 * c->pi * (1.0 / (double)g.numphi);
    c->drinv = 1.0 / g.dr;
    c->dzinv = 1.0 / c->dz;
    c->dphiinv = 1.0 / c->dphi;
    c->gamma = c->dzinv * c->dzinv;
    c->four_pi = 4.0 * c->pi;
    c->factor = (g.isym == 3) ? -(2.0 * g.dr * c->dz * c->dphi) : -(g.dr * c->dz * c->dphi);

    // Admission: refuse a context that cannot fit in free device memory.
    size_t need = sizeof(double) * ((size_t)g.mmax * c->nb * c->np + (size_t)c->N * c->np +
                                    (size_t)c->N * c->nplane + 2ull * g.mmax * c->np);
    size_t free_b = 0, total_b = 0;
    BPH_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (need + (64ull << 20) > free_b) {
        set_error("context needs %zu bytes of device memory, %zu free", need, free_b);
        return BPH_ERR_NOMEM;
    }

    HostCoef h;
    host_coefficients(c, h);
    std::vector<double> grid;
    grid.insert(grid.end(), h.rhf_g.begin(), h.rhf_g.end());
    grid.insert(grid.end(), h.rhfinv_g.begin(), h.rhfinv_g.end());
    grid.insert(grid.end(), h.zhf_g.begin(), h.zhf_g.end());
    // Twiddles, in long double then rounded: exact angles 2 pi k / M etc.
    const long double pil = std::acos(-1.0L);
    std::vector<double2> tw(c->M), tw2(c->M + 1), ph(g.mmax);
    for (int k = 0; k < c->M; ++k) {
        long double a = 2.0L * pil * (long double)k / (long double)c->M;
        tw[k] = make_double2((double)std::cos(a), (double)std::sin(a));
    }
    for (int k = 0; k <= c->M; ++k) {
        long double a = 2.0L * pil * (long double)k / (long double)c->N;
        tw2[k] = make_double2((double)std::cos(a), (double)std::sin(a));
    }
    for (int m = 0; m < g.mmax; ++m) {
        long double a = pil * (long double)(c->fm * m) / (long double)c->N;
        ph[m] = make_double2((double)std::cos(a), (double)std::sin(a));
    }

    if ((rc = dev_alloc(c, &c->d_green, (size_t)g.mmax * c->nb * c->np))) return rc;
    if ((rc = dev_alloc(c, &c->d_R, (size_t)c->N * c->np))) return rc;
    if ((rc = dev_alloc(c, &c->d_P, (size_t)c->N * c->nplane))) return rc;
    if ((rc = dev_alloc(c, &c->d_mom, (size_t)2 * g.mmax * c->np + compact::kMomPad))) return rc;
    if ((rc = dev_alloc(c, &c->d_S, (size_t)2 * g.mmax * c->nb))) return rc;
    if ((rc = dev_alloc(c, &c->d_brb, (size_t)c->N * g.numr))) return rc;
    if ((rc = dev_alloc(c, &c->d_elz, (size_t)c->N * g.numr))) return rc;
    if ((rc = dev_alloc(c, &c->d_alphar, (size_t)g.numr))) return rc;
    if ((rc = dev_alloc(c, &c->d_betar, (size_t)g.numr))) return rc;
    if ((rc = dev_alloc(c, &c->d_bzb, (size_t)g.numz))) return rc;
    if ((rc = dev_alloc(c, &c->d_qcoef, (size_t)g.mmax * (2 + kHyprUprBnd + 1)))) return rc;
    if ((rc = dev_alloc(c, &c->d_grid, grid.size()))) return rc;
    if ((rc = dev_alloc(c, &c->d_tw, (size_t)c->M))) return rc;
    if ((rc = dev_alloc(c, &c->d_tw2, (size_t)c->M + 1))) return rc;
    if ((rc = dev_alloc(c, &c->d_ph, (size_t)g.mmax))) return rc;
    if ((rc = dev_alloc(c, &c->d_red, (size_t)2 * c->N))) return rc;
    if ((rc = dev_alloc(c, &c->d_status, 1))) return rc;
    if ((rc = dev_alloc(c, &c->d_scf, scf_scratch_doubles()))) return rc;

    if ((rc = upload(c, c->d_brb, h.brb.data(), sizeof(double) * h.brb.size()))) return rc;
    if ((rc = upload(c, c->d_elz, h.elz.data(), sizeof(double) * h.elz.size()))) return rc;
    if ((rc = upload(c, c->d_alphar, h.alphar.data(), sizeof(double) * h.alphar.size()))) return rc;
    if ((rc = upload(c, c->d_betar, h.betar.data(), sizeof(double) * h.betar.size()))) return rc;
    if ((rc = upload(c, c->d_bzb, h.bzb.data(), sizeof(double) * h.bzb.size()))) return rc;
    if ((rc = upload(c, c->d_grid, grid.data(), sizeof(double) * grid.size()))) return rc;
    if ((rc = upload(c, c->d_tw, tw.data(), sizeof(double2) * tw.size()))) return rc;
    if ((rc = upload(c, c->d_tw2, tw2.data(), sizeof(double2) * tw2.size()))) return rc;
    if ((rc = upload(c, c->d_ph, ph.data(), sizeof(double2) * ph.size()))) return rc;
    BPH_CUDA(cudaMemsetAsync(c->d_P, 0, sizeof(double) * (size_t)c->N * c->nplane, c->stream));
    BPH_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    BPH_CUDA(cudaMemsetAsync(c->d_mom + (size_t)2 * g.mmax * c->np, 0, sizeof(double) * compact::kMomPad, c->stream));

    {
        const char *pdl = std::getenv("BPH_PDL");
        c->pdl = !(pdl && pdl[0] == '0');
    }
    {
        // slots that carry boundary data (the contraction writes them) last
        std::vector<int> map, dep;
        for (int sl = 0; sl < c->N; ++sl) {
            const int k = (sl <= c->M) ? sl : sl - c->M;
            const bool has_bc = (k < c->M) && (k % c->fm == 0) && (k / c->fm < g.mmax);
            (has_bc ? dep : map).push_back(sl);
        }
        c->nfree = (int)map.size();
        map.insert(map.end(), dep.begin(), dep.end());
        BPH_CUDA(cudaMalloc((void **)&c->d_slot_map, sizeof(int) * c->N));
        c->bytes += sizeof(int) * c->N;
        BPH_CUDA(cudaMemcpy(c->d_slot_map, map.data(), sizeof(int) * c->N, cudaMemcpyHostToDevice));
        int least = 0, greatest = 0;
        BPH_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        // the lowest priority: the contraction's CTAs take the SMs first and
        // the free slots' ADI fills SMs as its waves drain (a high-priority
        // side stream starved the contraction: 304 against 266 us per solve
        // at 130x98x256; this order gives 258)
        (void)greatest;
        BPH_CUDA(cudaStreamCreateWithPriority(&c->side_stream, cudaStreamNonBlocking, least));
        BPH_CUDA(cudaEventCreateWithFlags(&c->ev_fft, cudaEventDisableTiming));
        BPH_CUDA(cudaEventCreateWithFlags(&c->ev_free, cudaEventDisableTiming));
        BPH_CUDA(cudaEventCreateWithFlags(&c->ev_contract, cudaEventDisableTiming));
        const char *cg = std::getenv("BPH_CONV_GRAPH");
        c->conv_graph = !(cg && cg[0] == '0');
        const char *ov = std::getenv("BPH_OVERLAP");
        c->overlap = !(ov && ov[0] == '0');
    }
    BPH_CUDA(launch_qcoef(c));
    BPH_CUDA(launch_green_tables(c));
    if ((rc = compact_configure(c))) return rc;
    if ((rc = fft_configure(c))) return rc;
    if ((rc = adi_configure(c))) return rc;
    if ((rc = warp_configure(c))) return rc;
    if ((rc = direct_configure(c))) return rc;
    if ((rc = contract_configure(c))) return rc;
    if ((rc = noalloc_setup(c))) return rc;
    {
        // SM partitions for the overlapped solve: BPH_GREEN=1 turns them on,
        // BPH_GREEN_SMS sets the contraction's share (default 72 of 148)
        const char *gr = std::getenv("BPH_GREEN");
        if (gr && gr[0] == '1') {
            const char *gs = std::getenv("BPH_GREEN_SMS");
            const int sms = gs ? std::atoi(gs) : 72;
            if ((rc = green_setup(c, sms > 0 ? sms : 72))) return rc;
        }
    }
    {
        const size_t groups = (size_t)(c->nb + 7) / 8;
        if ((rc = dev_alloc(c, &c->d_ccnt, (size_t)g.mmax * groups))) return rc;
        if ((rc = dev_alloc(c, &c->d_cpart, (size_t)c->contract_split * g.mmax * c->nb * 2))) return rc;
        BPH_CUDA(cudaMemsetAsync(c->d_ccnt, 0, sizeof(unsigned int) * (size_t)g.mmax * groups, c->stream));
    }
    if (c->adi_smem == 0) {
        if (!c->large_kb[0]) {
            set_error("grid too large: an ADI panel of one row exceeds shared memory");
            return BPH_ERR_INVALID;
        }
        if ((rc = dev_alloc(c, &c->d_W, (size_t)c->N * c->nplane))) return rc;
        if ((rc = dev_alloc(c, &c->d_W2, (size_t)c->N * c->np))) return rc;
    }
    Schedule *s;
    if ((rc = get_schedule(c, 5, &s))) return rc;
    if ((rc = get_schedule(c, 20, &s))) return rc;
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    const char *tune = std::getenv("BPH_AUTOTUNE");
    if (!(tune && tune[0] == '0')) {
        if ((rc = autotune_setup(c))) return rc;
        if ((rc = autotune_mixed(c))) return rc;
    }
    return BPH_OK;
}

// Programmatic dependent launch off for the launches in its scope (kernels
// that follow a cross-stream event wait, or that must not become resident
// before another stream's kernel).
struct PdlOff {
    bph_ctx *c;
    bool keep;
    explicit PdlOff(bph_ctx *cc) : c(cc), keep(cc->pdl) { c->pdl = false; }
    ~PdlOff() { c->pdl = keep; }
};

// The solve on device arrays (see the file comment).  Overlapped form: the
// ADI of the slots without boundary data runs on the low-priority side
// stream from the end of the forward FFT, taking SMs as the contraction
// (HBM-bound, main stream) drains; the dependent slots follow the
// contraction; the inverse FFT joins both.
// Launches of its scope go to stream st (the launch wrappers use c->stream).
struct StreamSwap {
    bph_ctx *c;
    cudaStream_t keep;
    StreamSwap(bph_ctx *cc, cudaStream_t st) : c(cc), keep(cc->stream) { c->stream = st; }
    ~StreamSwap() { c->stream = keep; }
};

int solve_device(bph_ctx *c, const double *d_rho, double *d_pot, const Schedule &s, bool cold,
                 double *d_phieff = nullptr, double omega = 0.0) {
    BPH_CUDA(launch_fft_fwd_rho(c, d_rho));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (c->green) BPH_CUDA(cudaStreamIsCapturing(c->stream, &cap));
    if (c->green && cap == cudaStreamCaptureStatusNone && c->overlap && c->adi_seg && c->nfree > 0 &&
        c->nfree < c->N) {
        // contraction on partition 0, free-slot ADI on partition 1, both from the forward FFT
        BPH_CUDA(cudaEventRecord(c->ev_fft, c->stream));
        {
            PdlOff off(c);
            StreamSwap sw(c, c->green_stream[0]);
            BPH_CUDA(cudaStreamWaitEvent(c->stream, c->ev_fft, 0));
            BPH_CUDA(launch_green_contract(c));  // also writes the Dirichlet slots
            BPH_CUDA(cudaEventRecord(c->ev_contract, c->stream));
        }
        BPH_CUDA(cudaStreamWaitEvent(c->green_stream[1], c->ev_fft, 0));
        BPH_CUDA(launch_adi_slots(c, s, cold, c->d_slot_map, c->nfree, c->green_stream[1], false));
        BPH_CUDA(cudaEventRecord(c->ev_free, c->green_stream[1]));
        BPH_CUDA(cudaStreamWaitEvent(c->stream, c->ev_contract, 0));
        BPH_CUDA(launch_adi_slots(c, s, cold, c->d_slot_map + c->nfree, c->N - c->nfree, c->stream, false));
        BPH_CUDA(cudaStreamWaitEvent(c->stream, c->ev_free, 0));
        PdlOff off(c);
        BPH_CUDA(launch_fft_inv(c, d_pot, d_phieff, omega));
    } else if (c->overlap && c->adi_seg && c->nfree > 0 && c->nfree < c->N) {
        BPH_CUDA(cudaEventRecord(c->ev_fft, c->stream));
        BPH_CUDA(cudaStreamWaitEvent(c->side_stream, c->ev_fft, 0));
        BPH_CUDA(launch_adi_slots(c, s, cold, c->d_slot_map, c->nfree, c->side_stream, false));
        BPH_CUDA(cudaEventRecord(c->ev_free, c->side_stream));
        BPH_CUDA(launch_green_contract(c));  // also writes the Dirichlet slots
        BPH_CUDA(launch_adi_slots(c, s, cold, c->d_slot_map + c->nfree, c->N - c->nfree, c->stream, c->pdl));
        BPH_CUDA(cudaStreamWaitEvent(c->stream, c->ev_free, 0));
        PdlOff off(c);
        BPH_CUDA(launch_fft_inv(c, d_pot, d_phieff, omega));
    } else {
        BPH_CUDA(launch_green_contract(c));  // also writes the Dirichlet slots
        BPH_CUDA(launch_adi(c, s, 0, s.nsteps, cold));
        BPH_CUDA(launch_fft_inv(c, d_pot, d_phieff, omega));
    }
    c->have_warm = true;
    return BPH_OK;
}

int ensure_staging(bph_ctx *c) {
    int rc;
    if (!c->d_rho_stage && (rc = dev_alloc(c, &c->d_rho_stage, (size_t)c->ntot))) return rc;
    if (!c->d_pot_stage && (rc = dev_alloc(c, &c->d_pot_stage, (size_t)c->ntot))) return rc;
    return BPH_OK;
}

int read_status(bph_ctx *c) {
    int st = 0;
    BPH_CUDA(cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    BPH_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    if (st & kStatusNonFinite) {
        set_error("density contains NaN or Inf");
        return BPH_ERR_NONFINITE;
    }
    if (st & kStatusTimeout) {
        set_error("a bounded device wait expired (bulk copy of ADI factors or Green tables); results are not valid");
        return BPH_ERR_TIMEOUT;
    }
    return BPH_OK;
}

// Host-array wrapper: copy in, solve, copy out, wait, report.
int solve_host(bph_ctx *c, const double *rho, double *pot, const Schedule &s, bool cold) {
    int rc;
    if ((rc = ensure_staging(c))) return rc;
    const size_t bytes = sizeof(double) * (size_t)c->ntot;
    BPH_CUDA(cudaMemcpyAsync(c->d_rho_stage, rho, bytes, cudaMemcpyHostToDevice, c->stream));
    if ((rc = solve_device(c, c->d_rho_stage, c->d_pot_stage, s, cold))) return rc;
    BPH_CUDA(cudaMemcpyAsync(pot, c->d_pot_stage, bytes, cudaMemcpyDeviceToHost, c->stream));
    return read_status(c);
}

int check_ctx(const bph_ctx *c) {
    if (!c) {
        set_error("context is NULL");
        return BPH_ERR_INVALID;
    }
    return BPH_OK;
}


}  // namespace

int batch_schedule(bph_ctx *c, int nsteps, Schedule **out) { return get_schedule(c, nsteps, out); }
int context_status(bph_ctx *c) { return read_status(c); }

// The device state of a context, once nothing holds it.
static void ctx_free(bph_ctx *c) {
    DeviceScope scope_(c->device);
    if (c->own_stream) cudaStreamSynchronize(c->own_stream);
    if (c->stream && c->stream != c->own_stream) cudaStreamSynchronize(c->stream);
    for (auto &s : c->sched) free_schedule(c, s);
    double *bufs[] = {c->d_green, c->d_brb,  c->d_elz, c->d_alphar, c->d_betar,     c->d_bzb,
                      c->d_qcoef, c->d_grid, c->d_R,   c->d_P,      c->d_prev,      c->d_mom,
                      c->d_S,     c->d_W,    c->d_W2,  c->d_P2,     c->d_red,       c->d_rho_stage, c->d_pot_stage,
                      c->d_phieff_stage};
    for (double *p : bufs) dev_free(p);
    dev_free(c->d_tw);
    dev_free(c->d_tw2);
    dev_free(c->d_ph);
    dev_free(c->d_status);
    dev_free(c->d_ccnt);
    dev_free(c->d_cpart);
    dev_free(c->d_gtile);
    dev_free(c->d_gside);
    dev_free(c->d_kpart);
    dev_free(c->d_kcnt);
    conv_graphs_free(c);
    dev_free(c->d_work32);
    dev_free(c->d_warp_coef);
    dev_free(c->d_warp_coef32);
    dev_free(c->d_r32);
    dev_free(c->d_dir32);
    dev_free(c->d_dirS);
    dev_free(c->d_scf);
    if (c->side_stream) {
        cudaStreamSynchronize(c->side_stream);
        cudaStreamDestroy(c->side_stream);
    }
    if (c->ev_fft) cudaEventDestroy(c->ev_fft);
    if (c->ev_free) cudaEventDestroy(c->ev_free);
    if (c->ev_contract) cudaEventDestroy(c->ev_contract);
    green_free(c);
    if (c->d_slot_map) cudaFree(c->d_slot_map);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

void ctx_retain(bph_ctx *c) { c->refs.fetch_add(1, std::memory_order_relaxed); }

void ctx_release(bph_ctx *c) {
    if (c->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) ctx_free(c);
}

}  // namespace bph

using namespace bph;

extern "C" {

const char *bph_last_error(void) { return g_err; }

const char *bph_version(void) { return "bipoly_hydro_b200 0.1 (sm_100a)"; }

int bph_setup(const bph_grid_t *grid, bph_ctx_t **ctx) {
    g_err[0] = 0;
    if (!ctx) {
        set_error("ctx out-pointer is NULL");
        return BPH_ERR_INVALID;
    }
    *ctx = nullptr;
    int rc = validate(grid);
    if (rc) return rc;
    bph_ctx *c = new bph_ctx();
    c->g = *grid;
    rc = setup_impl(c);
    if (rc) {
        char keep[sizeof g_err];
        memcpy(keep, g_err, sizeof keep);
        bph_destroy(c);
        memcpy(g_err, keep, sizeof keep);
        return rc;
    }
    *ctx = c;
    return BPH_OK;
}

int bph_destroy(bph_ctx_t *c) {
    if (!c) return BPH_OK;
    ::bph::ctx_release(c);
    return BPH_OK;
}

int bph_register_host(void *ptr, size_t bytes) {
    if (!ptr || bytes == 0) {
        set_error("ptr must be non-NULL and bytes > 0");
        return BPH_ERR_INVALID;
    }
    cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterPortable);
    if (e == cudaErrorHostMemoryAlreadyRegistered) {
        (void)cudaGetLastError();  // already pinned: nothing to do
        return BPH_OK;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostRegister");
    return BPH_OK;
}

int bph_unregister_host(void *ptr) {
    if (!ptr) {
        set_error("ptr is NULL");
        return BPH_ERR_INVALID;
    }
    cudaError_t e = cudaHostUnregister(ptr);
    if (e == cudaErrorHostMemoryNotRegistered) {
        (void)cudaGetLastError();
        set_error("pointer was not registered with bph_register_host");
        return BPH_ERR_INVALID;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostUnregister");
    return BPH_OK;
}

int bph_set_stream(bph_ctx_t *c, void *stream) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    c->stream = (cudaStream_t)stream;  // NULL is CUDA's default stream
    return BPH_OK;
}

int bph_synchronize(bph_ctx_t *c) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    BPH_DEVICE_SCOPE(c);
    return read_status(c);
}

int bph_potential_solver(bph_ctx_t *c, const double *rho, double *pot, int tstep) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!rho || !pot) {
        set_error("rho and pot must be non-NULL");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    bool warm = tstep > 1;  // potential_solver.F90:80
    Schedule *s;
    if ((rc = get_schedule(c, warm ? 5 : 20, &s))) return rc;
    return solve_host(c, rho, pot, *s, !warm);
}

int bph_potential_solver_device(bph_ctx_t *c, const double *d_rho, double *d_pot, int tstep) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!d_rho || !d_pot) {
        set_error("rho and pot must be non-NULL");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    bool warm = tstep > 1;
    Schedule *s;
    if ((rc = get_schedule(c, warm ? 5 : 20, &s))) return rc;
    return solve_device(c, d_rho, d_pot, *s, !warm);
}

int bph_scf_step(bph_ctx_t *c, double *d_rho, double *d_pot, double eps, double mass, unsigned long long seed,
                 int iteration, int tstep) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!d_rho || !d_pot || !(eps >= 0.0) || !std::isfinite(eps) || !std::isfinite(mass) || iteration < 0) {
        set_error("invalid arguments (device arrays, eps >= 0, finite mass, iteration >= 0)");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    BPH_CUDA(launch_scf_update(c, d_rho, eps, mass, seed, iteration, c->d_scf));
    const bool warm = tstep > 1;  // potential_solver.F90:80
    Schedule *s;
    if ((rc = get_schedule(c, warm ? 5 : 20, &s))) return rc;
    return solve_device(c, d_rho, d_pot, *s, !warm);
}

int bph_scf_mass(bph_ctx_t *c, double *mass_out, double *scale_out) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    BPH_DEVICE_SCOPE(c);
    double h[2] = {0.0, 0.0};
    BPH_CUDA(cudaMemcpyAsync(h, c->d_scf + scf_scratch_doubles() - 2, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    if (scale_out) *scale_out = h[0];
    if (mass_out) *mass_out = h[1];
    return BPH_OK;
}

int bph_solve_nsteps(bph_ctx_t *c, const double *rho, double *pot, int nsteps, int cold, int on_device) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!rho || !pot || nsteps < 1 || nsteps > 10000) {
        set_error("invalid arguments (nsteps must be in [1, 10000])");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    Schedule *s;
    if ((rc = get_schedule(c, nsteps, &s))) return rc;
    if (on_device) return solve_device(c, rho, pot, *s, cold != 0);
    return solve_host(c, rho, pot, *s, cold != 0);
}

}  // extern "C"

namespace bph {

// Sum of the per-slot (num, den) pairs a norm kernel left in c->d_red.
int ensure_mixed_work(bph_ctx *c) {
    if (c->d_work32) return BPH_OK;
    return dev_alloc(c, &c->d_work32, (size_t)c->N * 4 * (size_t)c->np);
}

static double host_ratio(const std::vector<double> &h, int N) {
    double num = 0.0, den = 0.0;
    for (int i = 0; i < N; ++i) {
        num += h[2 * i];
        den += h[2 * i + 1];
    }
    return den > 0.0 ? std::sqrt(num / den) : std::sqrt(num);
}

// Converged FP64 (mixed = false) or mixed-precision solve.  A cold start
// zeroes the slot array before the contraction writes the Dirichlet slots,
// as the reference's cold start zeroes potp.  The cycle loop runs on the
// device as a graph while node (bph_converge.cu) unless BPH_CONV_GRAPH=0 or
// the graph cannot be built, then on the host with one synchronisation per
// cycle; both apply the same stopping rule.
static int converged_impl(bph_ctx *c, const double *rho, double *pot, int nsteps, int cold, double tol, int max_cycles,
                          int on_device, int *cycles_out, double *resid_out, bool mixed) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!rho || !pot || nsteps < 1 || nsteps > 10000 || max_cycles < 1 || !(tol >= 0.0)) {
        set_error("invalid arguments");
        return BPH_ERR_INVALID;
    }
    if (mixed && !c->adi_mixed_smem) {
        set_error("no mixed-precision ADI kernel is configured for this grid");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    Schedule *s;
    if ((rc = get_schedule(c, nsteps, &s))) return rc;
    if (mixed && c->mixed_kind == BPH_MIXED_ADI_GLOBAL && (rc = ensure_mixed_work(c))) return rc;
    if (!mixed && !c->d_prev && (rc = dev_alloc(c, &c->d_prev, (size_t)c->N * c->nplane))) return rc;
    const size_t bytes = sizeof(double) * (size_t)c->ntot;
    const double *d_rho = rho;
    double *d_pot = pot;
    if (!on_device) {
        if ((rc = ensure_staging(c))) return rc;
        BPH_CUDA(cudaMemcpyAsync(c->d_rho_stage, rho, bytes, cudaMemcpyHostToDevice, c->stream));
        d_rho = c->d_rho_stage;
        d_pot = c->d_pot_stage;
    }
    if (cold) BPH_CUDA(cudaMemsetAsync(c->d_P, 0, sizeof(double) * (size_t)c->N * c->nplane, c->stream));
    BPH_CUDA(launch_fft_fwd_rho(c, d_rho));
    BPH_CUDA(launch_green_contract(c));  // also writes the Dirichlet slots
    std::vector<double> h(2 * (size_t)c->N);
    int cyc = 0;
    double upd = 0.0;
    bool device_loop = c->conv_graph && conv_loop_device(c, *s, mixed, tol, max_cycles) == BPH_OK;
    if (!device_loop) {
        c->conv_graph = false;  // graphs unavailable: host loop from now on
        double prev_upd = INFINITY;
        for (;;) {
            if (mixed) {
                BPH_CUDA(launch_adi_defect(c, *s));
            } else if (c->adi_seg) {  // update norms from the sweep's write-back
                BPH_CUDA(launch_adi(c, *s, 0, s->nsteps, false, nullptr, nullptr, 1, nullptr, c->d_red));
            } else {
                BPH_CUDA(cudaMemcpyAsync(c->d_prev, c->d_P, bytes, cudaMemcpyDeviceToDevice, c->stream));
                BPH_CUDA(launch_adi(c, *s, 0, s->nsteps, false));
                BPH_CUDA(launch_update_norm(c, c->d_red));
            }
            ++cyc;
            BPH_CUDA(cudaMemcpyAsync(h.data(), c->d_red, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                                     c->stream));
            BPH_CUDA(cudaStreamSynchronize(c->stream));
            upd = host_ratio(h, c->N);
            bool stop = upd <= tol || cyc >= max_cycles;
            if (mixed) stop = stop || !(upd == upd) || upd > 0.5 * prev_upd;
            if (stop) break;
            prev_upd = upd;
        }
    }
    if (resid_out) BPH_CUDA(launch_residual_norm(c, c->d_red));
    BPH_CUDA(launch_fft_inv(c, d_pot));
    c->have_warm = true;
    if (!on_device) BPH_CUDA(cudaMemcpyAsync(pot, d_pot, bytes, cudaMemcpyDeviceToHost, c->stream));
    ConvState st = {};
    if (device_loop)
        BPH_CUDA(cudaMemcpyAsync(&st, c->d_conv, sizeof(ConvState), cudaMemcpyDeviceToHost, c->stream));
    if (resid_out)
        BPH_CUDA(cudaMemcpyAsync(h.data(), c->d_red, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    if ((rc = read_status(c))) return rc;  // synchronises
    if (device_loop) {
        cyc = st.cycles;
        upd = st.upd;
    }
    if (mixed && !(upd == upd)) {
        set_error("mixed-precision refinement diverged");
        return BPH_ERR_NONFINITE;
    }
    if (resid_out) *resid_out = host_ratio(h, c->N);
    if (cycles_out) *cycles_out = cyc;
    return BPH_OK;
}

}  // namespace bph

extern "C" {

int bph_solve_converged(bph_ctx_t *c, const double *rho, double *pot, int nsteps, int cold, double tol,
                        int max_cycles, int on_device, int *cycles_out, double *resid_out) {
    return converged_impl(c, rho, pot, nsteps, cold, tol, max_cycles, on_device, cycles_out, resid_out, false);
}

int bph_solve_converged_mixed(bph_ctx_t *c, const double *rho, double *pot, int nsteps, int cold, double tol,
                              int max_cycles, int on_device, int *cycles_out, double *resid_out) {
    return converged_impl(c, rho, pot, nsteps, cold, tol, max_cycles, on_device, cycles_out, resid_out, true);
}

int bph_potential_solver_phieff(bph_ctx_t *c, const double *rho, double *pot, double *phieff, double omega_frame,
                                int tstep, int on_device) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!rho || !pot || !phieff || !std::isfinite(omega_frame)) {
        set_error("rho, pot and phieff must be non-NULL and omega_frame finite");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    bool warm = tstep > 1;
    Schedule *s;
    if ((rc = get_schedule(c, warm ? 5 : 20, &s))) return rc;
    if (on_device) return solve_device(c, rho, pot, *s, !warm, phieff, omega_frame);
    if ((rc = ensure_staging(c))) return rc;
    if (!c->d_phieff_stage && (rc = dev_alloc(c, &c->d_phieff_stage, (size_t)c->ntot))) return rc;
    const size_t bytes = sizeof(double) * (size_t)c->ntot;
    BPH_CUDA(cudaMemcpyAsync(c->d_rho_stage, rho, bytes, cudaMemcpyHostToDevice, c->stream));
    if ((rc = solve_device(c, c->d_rho_stage, c->d_pot_stage, *s, !warm, c->d_phieff_stage, omega_frame))) return rc;
    BPH_CUDA(cudaMemcpyAsync(pot, c->d_pot_stage, bytes, cudaMemcpyDeviceToHost, c->stream));
    BPH_CUDA(cudaMemcpyAsync(phieff, c->d_phieff_stage, bytes, cudaMemcpyDeviceToHost, c->stream));
    return read_status(c);
}

int bph_set_potential(bph_ctx_t *c, const double *pot, int on_device) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (!pot) {
        set_error("pot must be non-NULL");
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    const double *d_pot = pot;
    if (!on_device) {
        if ((rc = ensure_staging(c))) return rc;
        BPH_CUDA(cudaMemcpyAsync(c->d_pot_stage, pot, sizeof(double) * (size_t)c->ntot, cudaMemcpyHostToDevice,
                                 c->stream));
        d_pot = c->d_pot_stage;
    }
    BPH_CUDA(launch_fft_fwd_pot(c, d_pot));
    c->have_warm = true;
    if (!on_device) BPH_CUDA(cudaStreamSynchronize(c->stream));
    return BPH_OK;
}

int bph_run_phase(bph_ctx_t *c, int phase, const double *d_rho, double *d_pot, int nsteps) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    BPH_DEVICE_SCOPE(c);
    switch (phase) {
        case BPH_PHASE_FFT_RHO:
            if (!d_rho) break;
            BPH_CUDA(launch_fft_fwd_rho(c, d_rho));
            return BPH_OK;
        case BPH_PHASE_CONTRACT:
            BPH_CUDA(launch_green_contract(c));
            return BPH_OK;
        case BPH_PHASE_SLOTS:
            BPH_CUDA(launch_boundary_slots(c));
            return BPH_OK;
        case BPH_PHASE_ADI: {
            if (nsteps < 1 || nsteps > 10000) break;
            Schedule *s;
            if ((rc = get_schedule(c, nsteps, &s))) return rc;
            BPH_CUDA(launch_adi(c, *s, 0, s->nsteps, false));
            return BPH_OK;
        }
        case BPH_PHASE_FFT_INV:
            if (!d_pot) break;
            BPH_CUDA(launch_fft_inv(c, d_pot));
            return BPH_OK;
        default:
            break;
    }
    set_error("invalid phase %d or arguments", phase);
    return BPH_ERR_INVALID;
}

int bph_num_boundary_rows(const bph_ctx_t *c) { return c ? c->nb : 0; }

int bph_copy_green(bph_ctx_t *c, double *out, size_t n) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    size_t need = (size_t)c->g.mmax * c->nb * c->np;
    if (!out || n < need) {
        set_error("output buffer too small (%zu < %zu)", n, need);
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    BPH_CUDA(cudaMemcpyAsync(out, c->d_green, sizeof(double) * need, cudaMemcpyDeviceToHost, c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    return BPH_OK;
}

int bph_copy_moments(bph_ctx_t *c, double *out, size_t n) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    size_t need = (size_t)c->g.mmax * c->nb * 2;
    if (!out || n < need) {
        set_error("output buffer too small (%zu < %zu)", n, need);
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    BPH_CUDA(cudaMemcpyAsync(out, c->d_S, sizeof(double) * need, cudaMemcpyDeviceToHost, c->stream));
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    return BPH_OK;
}

long long bph_info(const bph_ctx_t *c, int what) {
    if (!c) return -1;
    switch (what) {
        case BPH_INFO_ADI_THREADS: return c->adi_seg;
        case BPH_INFO_ADI_SMEM: return c->adi_smem;
        case BPH_INFO_MIXED_THREADS: return c->adi_mixed_threads;
        case BPH_INFO_MIXED_SMEM: return c->adi_mixed_smem;
        case BPH_INFO_MIXED_CTAS_PER_SM: return c->adi_mixed_per_sm;
        case BPH_INFO_CONTRACT_SPLIT: return c->contract_split;
        case BPH_INFO_MIXED_KIND: return c->mixed_kind;
        case BPH_INFO_MIXED_FORWARD_NS: return (long long)(1e3f * c->mixed_tuned_us[BPH_MIXED_ADI_FORWARD]);
        case BPH_INFO_MIXED_INCREMENT_NS: return (long long)(1e3f * c->mixed_tuned_us[BPH_MIXED_ADI_INCREMENT]);
        case BPH_INFO_ADI_PREFETCH: return (c->adi_pf ? 1 : 0) | (c->mixed_pf ? 2 : 0);
        case BPH_INFO_ADI_KERNEL:
            return c->adi_warp ? BPH_ADI_KERNEL_WARP
                               : c->adi_seg ? BPH_ADI_KERNEL_SEGMENTED
                                            : c->adi_smem ? BPH_ADI_KERNEL_ONCHIP : BPH_ADI_KERNEL_GRID_WIDE;
        case BPH_INFO_ADI_WARP_SMEM: return c->adi_warp_smem;
        case BPH_INFO_MIXED_WARP_NS: return (long long)(1e3f * c->mixed_tuned_us[BPH_MIXED_ADI_WARP]);
        case BPH_INFO_GREEN_SMS: return c->green ? c->green_sms[0] : -c->green_fail;
        case BPH_INFO_CONTRACT_KIND: return c->compact ? BPH_CONTRACT_COMPACT : BPH_CONTRACT_FULL;
        case BPH_INFO_FFT_DENSE: return c->fft_dense ? 1 : 0;
        case BPH_INFO_CONTRACT_FULL_NS: return (long long)(1e3f * c->tuned_contract_us[0]);
        case BPH_INFO_CONTRACT_COMPACT_NS: return (long long)(1e3f * c->tuned_contract_us[1]);
        case BPH_INFO_FFT_NS: return (long long)(1e3f * c->tuned_fft_us[0]);
        case BPH_INFO_FFT_DENSE_NS: return (long long)(1e3f * c->tuned_fft_us[1]);
        case BPH_INFO_ADI_SEG_NS: return (long long)(1e3f * c->tuned_adi_us[0]);
        case BPH_INFO_ADI_WARP_NS: return (long long)(1e3f * c->tuned_adi_us[1]);
        case BPH_INFO_MIXED_DIRECT_NS: return (long long)(1e3f * c->mixed_tuned_us[BPH_MIXED_DIRECT]);
        default: return -1;
    }
}

int bph_configure(bph_ctx_t *c, int key, int value) {
    int rc;
    if ((rc = check_ctx(c))) return rc;
    if (key != BPH_CFG_MIXED_ADI) {
        set_error("unknown configuration key %d", key);
        return BPH_ERR_INVALID;
    }
    BPH_DEVICE_SCOPE(c);
    if (value == BPH_MIXED_ADI_AUTO) return autotune_mixed(c);
    if (value != BPH_MIXED_ADI_FORWARD && value != BPH_MIXED_ADI_INCREMENT && value != BPH_MIXED_ADI_GLOBAL &&
        value != BPH_MIXED_ADI_WARP && value != BPH_MIXED_DIRECT) {
        set_error("unknown refinement ADI kind %d", value);
        return BPH_ERR_INVALID;
    }
    BPH_CUDA(cudaStreamSynchronize(c->stream));
    if (select_mixed_kind(c, value) != BPH_OK) {
        set_error("refinement ADI kind %d does not fit this grid on chip", value);
        return BPH_ERR_INVALID;
    }
    return BPH_OK;
}

long long bph_launch_count(const bph_ctx_t *c) { return c ? c->launches : 0; }

size_t bph_device_bytes(const bph_ctx_t *c) { return c ? c->bytes : 0; }

}  // extern "C"
