// bph_adi.cu -- Peaceman-Rachford ADI over every Fourier slot
// (helmadi.F90:195-355 with tridagr.F90 and tridagz.F90).
//
// The numphi slots are independent 2-D problems, so one CTA owns one slot
// for all nsteps steps.  When the slot's interior potential and a work slab
// fit in shared memory (2 x (numz-2) x (numr-2 | 1) doubles, 198 KB at
// 130x98) the whole iteration runs on chip: HBM sees one read of -4 pi
// rho_hat per half-sweep (L2-resident), and one read plus one write of the
// potential per solve, where the reference makes 2*nsteps+4 full-array
// transposes (swap_r_z / swap_z_r).  Larger slots use the same code on the
// slot array in global memory.
//
// Each half-sweep is three phases separated by CTA barriers:
//   1. right-hand side, elementwise over the slab (all threads, coalesced);
//   2. forward elimination of the line systems, one thread per line, in
//      place in the work slab: y_j = w_j/bet_j - (a_j/bet_j) y_{j-1};
//   3. back substitution into the potential: x_j = y_j - gam_{j+1} x_{j+1}.
// The factors 1/bet, a/bet, gam depend only on (step, slot) and are built
// once per schedule at setup (k_adi_factors).  The on-chip slab's row
// stride is odd (in doubles) so that line-parallel accesses along r are
// bank-conflict free.
#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kAdiThreads = 256;

struct AdiArgs {
    double *P;              // slot array [N][nplane]
    const double *R;        // [N][np]
    double *Wg;             // global work slabs [N][nplane] (global variant)
    const double *rad;      // schedule radial factors [nsteps][N][3][nr]
    const double *ver;      // schedule vertical factors [nsteps][3][nz]
    const double *dt;       // [nsteps]
    const double *elz;      // [N][numr]
    const double *alphar;   // [numr]
    const double *betar;    // [numr]
    int numr, numz, nr, nz, N, isym;
    int step0, nsteps_run, cold;
    double gamma;
};

template <bool kOnChip>
__global__ void __launch_bounds__(kAdiThreads) k_adi(AdiArgs a) {
    extern __shared__ double sm[];
    const int s = blockIdx.x;
    const int tid = threadIdx.x;
    const int nr = a.nr, nz = a.nz, numr = a.numr;
    const long long nplane = (long long)numr * a.numz;
    const long long np = (long long)nr * nz;
    double *Pg = a.P + (long long)s * nplane;  // plane of slot s
    const double *Rs = a.R + (long long)s * np;

    // Slab addressing: element (j, k) of the interior at Pw[k*ps + j].
    double *Pw, *Ww;
    int ps;
    double *smalls;
    if (kOnChip) {
        ps = nr | 1;
        Pw = sm;
        Ww = sm + (long long)nz * ps;
        smalls = Ww + (long long)nz * ps;
    } else {
        ps = numr;
        Pw = Pg + numr + 1;
        Ww = a.Wg + (long long)s * nplane + numr + 1;
        smalls = sm;
    }
    double *top = smalls;          // [nr]  phi(J, numz)
    double *side = top + nr;       // [nz]  phi(numr, K)
    double *bot = side + nz;       // [nr]  phi(J, 1) (isym 1)
    double *alz = bot + nr;        // [nr]  alphaz(J)
    double *bez = alz + nr;        // [nr]  betaz(J)
    double *elz = bez + nr;        // [nr]  elambdazb(J, slot)
    double *rf = elz + nr;         // [3][nr] radial factors of the current step
    double *vf = rf + 3 * nr;      // [3][nz] vertical factors of the current step

    for (int j = tid; j < nr; j += kAdiThreads) {
        top[j] = Pg[(j + 1) + (long long)numr * (a.numz - 1)];
        bot[j] = (a.isym == 1) ? Pg[j + 1] : 0.0;
        alz[j] = a.alphar[j + 1];
        bez[j] = a.betar[j + 1];
        elz[j] = a.elz[(long long)s * numr + j + 1];
    }
    for (int k = tid; k < nz; k += kAdiThreads) side[k] = Pg[(numr - 1) + (long long)numr * (k + 1)];
    if (kOnChip) {
        for (long long e = tid; e < np; e += kAdiThreads) {
            int j = (int)(e % nr), k = (int)(e / nr);
            Pw[k * ps + j] = a.cold ? 0.0 : Pg[(j + 1) + (long long)numr * (k + 1)];
        }
    } else if (a.cold) {
        for (long long e = tid; e < np; e += kAdiThreads) {
            int j = (int)(e % nr), k = (int)(e / nr);
            Pw[k * ps + j] = 0.0;
        }
    }
    const double gamma = a.gamma;
    const double a_side = a.alphar[numr - 2];  // alphar(numr-1)
    const bool sym_bottom = (a.isym != 1);
    __syncthreads();

    for (int it = 0; it < a.nsteps_run; ++it) {
        const int step = a.step0 + it;
        const double dtt = a.dt[step];
        const double *rsrc = a.rad + ((long long)step * a.N + s) * 3 * nr;
        const double *vsrc = a.ver + (long long)step * 3 * nz;
        for (int i = tid; i < 3 * nr; i += kAdiThreads) rf[i] = rsrc[i];
        for (int i = tid; i < 3 * nz; i += kAdiThreads) vf[i] = vsrc[i];
        // ---- radial half-sweep (helmadi.F90:203-260) ----
        const double dtm2g = dtt - 2.0 * gamma, dtmg = dtt - gamma;
        for (long long e = tid; e < np; e += kAdiThreads) {
            int j = (int)(e % nr), k = (int)(e / nr);
            double phi = Pw[k * ps + j];
            double up = (k + 1 < nz) ? Pw[(k + 1) * ps + j] : top[j];
            double v;
            if (k == 0 && sym_bottom) {
                v = Rs[e] + dtmg * phi + gamma * up;
            } else {
                double dn = (k > 0) ? Pw[(k - 1) * ps + j] : bot[j];
                v = Rs[e] + dtm2g * phi + gamma * (up + dn);
            }
            if (j == nr - 1) v = v - a_side * side[k];
            Ww[k * ps + j] = v;
        }
        __syncthreads();
        {
            const double *ib = rf, *dd = rf + nr, *gm = rf + 2 * nr;
            for (int k = tid; k < nz; k += kAdiThreads) {
                double *w = Ww + k * ps;
                double y = w[0] * ib[0];
                w[0] = y;
                for (int j = 1; j < nr; ++j) {
                    y = w[j] * ib[j] - dd[j] * y;
                    w[j] = y;
                }
                double *p = Pw + k * ps;
                double x = y;
                p[nr - 1] = x;
                for (int j = nr - 2; j >= 0; --j) {
                    x = w[j] - gm[j + 1] * x;
                    p[j] = x;
                }
            }
        }
        __syncthreads();
        // ---- vertical half-sweep (helmadi.F90:272-343) ----
        for (long long e = tid; e < np; e += kAdiThreads) {
            int j = (int)(e % nr), k = (int)(e / nr);
            double phi = Pw[k * ps + j];
            double right = (j + 1 < nr) ? Pw[k * ps + j + 1] : side[k];
            double v = Rs[e] + (elz[j] + dtt) * phi - alz[j] * right;
            if (j > 0) v = v - bez[j] * Pw[k * ps + j - 1];
            if (k == nz - 1) v = v + gamma * top[j];
            if (!sym_bottom && k == 0) v = v + gamma * bot[j];
            Ww[k * ps + j] = v;
        }
        __syncthreads();
        {
            const double *ib = vf, *dd = vf + nz, *gm = vf + 2 * nz;
            for (int j = tid; j < nr; j += kAdiThreads) {
                double y = Ww[j] * ib[0];
                Ww[j] = y;
                for (int k = 1; k < nz; ++k) {
                    y = Ww[k * ps + j] * ib[k] - dd[k] * y;
                    Ww[k * ps + j] = y;
                }
                double x = y;
                Pw[(nz - 1) * ps + j] = x;
                for (int k = nz - 2; k >= 0; --k) {
                    x = Ww[k * ps + j] - gm[k + 1] * x;
                    Pw[k * ps + j] = x;
                }
            }
        }
        __syncthreads();
    }
    if (kOnChip) {
        for (long long e = tid; e < np; e += kAdiThreads) {
            int j = (int)(e % nr), k = (int)(e / nr);
            Pg[(j + 1) + (long long)numr * (k + 1)] = Pw[k * ps + j];
        }
    }
}

size_t smalls_bytes(const bph_ctx *c) { return sizeof(double) * (size_t)(9 * c->nr + 4 * c->nz); }

// Weighted (Parseval) squared norms over the interior of the slot array:
// out[0] = sum w |P - prev|^2, out[1] = sum w |P|^2 (update test), or
// out[0] = sum w |R - A P|^2, out[1] = sum w |R|^2 (residual).
constexpr int kNormThreads = 256;

template <bool kResidual>
__global__ void __launch_bounds__(kNormThreads)
k_slot_norms(const double *__restrict__ P, const double *__restrict__ Q, const double *__restrict__ R,
             const double *__restrict__ brb, const double *__restrict__ alphar, const double *__restrict__ betar,
             const double *__restrict__ bzb, double gamma, int numr, int numz, int nr, int nz, int N, int isym,
             double *__restrict__ out) {
    const int s = blockIdx.x;
    const long long nplane = (long long)numr * numz, np = (long long)nr * nz;
    const double *Ps = P + (long long)s * nplane;
    double a0 = 0.0, a1 = 0.0;
    for (long long e = threadIdx.x; e < np; e += kNormThreads) {
        int j = (int)(e % nr), k = (int)(e / nr);
        long long q = (j + 1) + (long long)numr * (k + 1);
        if (kResidual) {
            const double *b = brb + (long long)s * numr;
            double ar = b[j + 1] * Ps[q] + alphar[j + 1] * Ps[q + 1];
            if (j > 0) ar += betar[j + 1] * Ps[q - 1];
            double az = bzb[k + 1] * Ps[q] - gamma * Ps[q + numr];
            if (k > 0 || isym == 1) az -= gamma * Ps[q - numr];
            double rhs = R[(long long)s * np + e];
            double r = rhs - ar - az;
            a0 += r * r;
            a1 += rhs * rhs;
        } else {
            double d = Ps[q] - Q[(long long)s * nplane + q];
            a0 += d * d;
            a1 += Ps[q] * Ps[q];
        }
    }
    __shared__ double red[2][kNormThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, off);
        a1 += __shfl_down_sync(0xffffffffu, a1, off);
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = a0;
        red[1][warp] = a1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0.0;
        for (int w = 0; w < kNormThreads / 32; ++w) v += red[threadIdx.x][w];
        double wgt = (s == 0 || s == N / 2) ? 1.0 : 2.0;
        out[2 * s + threadIdx.x] = wgt * v;
    }
}

}  // namespace

int adi_configure(bph_ctx *c) {
    int dev_max = 0;
    cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    size_t onchip = sizeof(double) * 2 * (size_t)c->nz * (size_t)(c->nr | 1) + smalls_bytes(c);
    if (onchip <= (size_t)dev_max) {
        c->adi_smem = (int)onchip;
        e = cudaFuncSetAttribute(k_adi<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, c->adi_smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_adi)");
    } else {
        c->adi_smem = 0;
    }
    return BPH_OK;
}

cudaError_t launch_adi(bph_ctx *c, const Schedule &sch, int step0, int nsteps_run, bool cold) {
    AdiArgs a;
    a.P = c->d_P;
    a.R = c->d_R;
    a.Wg = c->d_W;
    a.rad = sch.d_rad;
    a.ver = sch.d_ver;
    a.dt = sch.d_dt;
    a.elz = c->d_elz;
    a.alphar = c->d_alphar;
    a.betar = c->d_betar;
    a.numr = c->g.numr;
    a.numz = c->g.numz;
    a.nr = c->nr;
    a.nz = c->nz;
    a.N = c->N;
    a.isym = c->g.isym;
    a.step0 = step0;
    a.nsteps_run = nsteps_run;
    a.cold = cold ? 1 : 0;
    a.gamma = c->gamma;
    ++c->launches;
    if (c->adi_smem > 0)
        k_adi<true><<<c->N, kAdiThreads, c->adi_smem, c->stream>>>(a);
    else
        k_adi<false><<<c->N, kAdiThreads, smalls_bytes(c), c->stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_update_norm(bph_ctx *c, double *d_out) {
    ++c->launches;
    k_slot_norms<false><<<c->N, kNormThreads, 0, c->stream>>>(
        c->d_P, c->d_prev, c->d_R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz,
        c->nr, c->nz, c->N, c->g.isym, d_out);
    return cudaGetLastError();
}

cudaError_t launch_residual_norm(bph_ctx *c, double *d_out) {
    ++c->launches;
    k_slot_norms<true><<<c->N, kNormThreads, 0, c->stream>>>(
        c->d_P, c->d_prev, c->d_R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz,
        c->nr, c->nz, c->N, c->g.isym, d_out);
    return cudaGetLastError();
}

}  // namespace bph
