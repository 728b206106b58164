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
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

#include "bph_internal.cuh"
#include "bph_bulk.h"

namespace bph {
namespace {

using namespace bulk;

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
    const double *brb;      // [N][numr] (defect form: residual)
    const double *bzb;      // [numz]    (defect form: residual)
    double *norms;          // [N][2]    (defect form: |delta|^2, |phi|^2 per slot)
    const int *inst_map;    // batches: instance of each block row (nullptr: block row = instance)
    const int *slot_map;    // slot of each block within a row (nullptr: block = slot)
    int nslots;             // blocks per row (N without slot_map)
    const void *rad_pk;     // packed radial factor blocks of the kernel's type [nsteps][N][pkr]
    const void *ver_pk;     // packed vertical factor blocks [nsteps][pkz]
    int pkr, pkz;           // their sizes in elements
    int *status;            // deferred status word (bounded waits that expire)
    int numr, numz, nr, nz, N, isym;
    int step0, nsteps_run, cold;
    double gamma;
};

template <bool kOnChip>
__global__ void __launch_bounds__(kAdiThreads) k_adi(AdiArgs a) {
    extern __shared__ double sm[];
    pdl_wait();
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
        const double *rsrc = a.rad + ((long long)step * a.N + s) * kAdiFactors * nr;
        const double *vsrc = a.ver + (long long)step * kAdiFactors * nz;
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





// ---------------------------------------------------------------------------
// Segmented on-chip ADI (the fast path).  The slot's potential P and its
// right-hand side R = -4 pi rho_hat both stay in shared memory for all
// steps.  Every line system is cut into kAdiSeg-long segments, one thread
// per (line, segment):
//   A. right-hand side and forward elimination with zero carry-in, kept in
//      registers; the segment's last value goes to shared memory;
//   B. carry-in y_{s-1} folded from the preceding segments' last values and
//      forward carries, fix-up y = L + G y_{s-1}, backward elimination with
//      zero carry-in; the segment's first value goes to shared memory;
//   C. carry-in x_{e+1} folded from the following segments, x = M + K x_{e+1},
//      stored to P.
// The per-element arithmetic is the Thomas algorithm of tridagr/tridagz; the
// carries only re-associate it (results agree to rounding).

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
    using type = double2;
    static __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Vec2<float> {
    using type = float2;
    static __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
};

struct SegLayout {
    int ps, Pr, Pz, xsz;
    int fsz;                  // elements of one direction's factor block
    size_t elems;             // elements of type T in the whole layout
};

// Factor block of one direction, n = line length, in shared memory:
//   ib[n]   1/bet_j
//   dd[n]   a_j/bet_j
//   GG[n]   pairs (G_j, gam_{j+1})   forward carry and next back-substitution factor
//   K[n]    backward carry
__host__ __device__ inline int factor_block(int n) { return 5 * n + 2; }  // +2: pair alignment

__host__ __device__ inline SegLayout seg_layout(int nr, int nz) {
    SegLayout L;
    L.ps = nr | 1;
    L.Pr = (nr + kAdiSeg - 1) / kAdiSeg;
    L.Pz = (nz + kAdiSeg - 1) / kAdiSeg;
    L.xsz = max(nz * L.Pr, nr * L.Pz);
    L.fsz = factor_block(max(nr, nz));
    L.elems = 2 * (size_t)nz * L.ps + 2 * (size_t)L.fsz + 4 * (size_t)L.xsz + 5 * (size_t)nr + 4;
    return L;
}

template <typename T>
__device__ inline T *align_pair(T *p) {
    using P2 = typename Vec2<T>::type;
    while ((reinterpret_cast<uintptr_t>(p) % sizeof(P2)) != 0) ++p;
    return p;
}

template <typename T>
struct Fac {
    const T *ib, *dd, *K;
    const typename Vec2<T>::type *GG;
};

template <typename T>
__device__ inline Fac<T> fac_view(const T *base, int n) {
    Fac<T> f;
    f.ib = base;
    f.dd = base + n;
    const T *g = align_pair(const_cast<T *>(base + 2 * n));
    f.GG = reinterpret_cast<const typename Vec2<T>::type *>(g);
    f.K = g + 2 * n;
    return f;
}

// Copies one direction's factors [ib, dd, gam, G, K] (global FP64) into a block.
template <typename T>
__device__ inline void fac_load(T *base, int n, const double *src, int tid, int nthreads) {
    T *ib = base, *dd = base + n;
    T *g = align_pair(base + 2 * n);
    auto *GG = reinterpret_cast<typename Vec2<T>::type *>(g);
    T *K = g + 2 * n;
    for (int j = tid; j < n; j += nthreads) {
        ib[j] = (T)src[j];
        dd[j] = (T)src[n + j];
        GG[j] = Vec2<T>::make((T)src[3 * n + j], (T)((j + 1 < n) ? src[2 * n + j + 1] : 0.0));
        K[j] = (T)src[4 * n + j];
    }
}

// ---------------------------------------------------------------------------
// Factor prefetch by bulk copy.  The segmented kernels read one factor block
// per direction and step; with prefetch they hold two blocks per direction
// in shared memory and fill the idle one with a bulk (TMA) copy of the next
// step's packed block while the current half-steps run, completion tracked
// by an mbarrier per block (one elected thread issues, every thread waits
// before its first read).  Waits are bounded: an expired wait sets
// kStatusTimeout and the kernel runs on (its results are then reported
// invalid), so no CTA can hang on a copy.
// Shared-memory layout of the prefetching segmented kernel, byte offsets.
struct PfLayout {
    int ps, Pr, Pz, xsz, fpf;  // fpf: elements per factor block (both directions)
    size_t o_rw, o_f, o_xa, o_xb, o_eb, o_el0, o_ab, o_zrow, o_mbar, bytes;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename T>
__host__ __device__ inline PfLayout pf_layout(int nr, int nz, bool with_zrow) {
    PfLayout L;
    L.ps = nr | 1;
    L.Pr = (nr + kAdiSeg - 1) / kAdiSeg;
    L.Pz = (nz + kAdiSeg - 1) / kAdiSeg;
    L.xsz = max(nz * L.Pr, nr * L.Pz);
    L.fpf = max(packed_block<T>(nr), packed_block<T>(nz));
    const size_t e = sizeof(T);
    size_t o = (size_t)nz * L.ps * e;
    L.o_rw = o;
    o = align_up(o + (size_t)nz * L.ps * e, 16);
    L.o_f = o;  // Fr[0], Fr[1], Fz[0], Fz[1]
    o += 4 * (size_t)L.fpf * e;
    L.o_xa = o;  // the segment-edge values of phase C reuse it (dead after phase B)
    o += (size_t)L.xsz * e;
    L.o_xb = o;
    o += (size_t)L.xsz * e;
    L.o_eb = o;
    o += (size_t)L.xsz * e;
    L.o_el0 = o;
    o = align_up(o + (size_t)nr * e, 2 * e);
    L.o_ab = o;
    o += 2 * (size_t)nr * e;
    L.o_zrow = o;
    if (with_zrow) o += (size_t)nr * e;
    L.o_mbar = align_up(o, 8);
    L.bytes = L.o_mbar + 4 * sizeof(uint64_t);
    return L;
}

// The ADI of one Fourier slot per CTA, all steps on chip.
//
// kDefect = false (FP64 drop-in, T = double): nsteps Peaceman-Rachford steps
//   on the potential itself, from the initial potential P (or zero).
// kDefect = true (mixed precision, T = float): one refinement cycle.  The
//   prologue forms the FP64 residual r = -4 pi rho_hat - A phi of the current
//   potential (boundary columns included); the steps run in T on the defect
//   equation A delta = r from delta = 0 with zero Dirichlet data; the
//   epilogue adds delta to phi in FP64 and records |delta|^2, |phi|^2.
//
// Shared-memory layout (elements of T):
//   Ww  nz x ps  the line systems' right-hand sides, pre-multiplied by the
//                sweep's 1/bet: at the start of a step the radial one
//                (drop-in step 0: the initial potential), after the radial
//                sweep the vertical one, after the last sweep the solution.
//   Rw  nz x ps  the source: -4 pi rho_hat plus every Dirichlet term, folded
//                in once (drop-in): +gamma*top (K = numz-1),
//                -alphar(numr-1)*side (J = numr-1), +gamma*bottom (K = 2,
//                isym 1) -- both sweeps add exactly these terms
//                (helmadi.F90:252-256, 327-340 and the K+1 / J+1 neighbours
//                of :224-245 / :296-319) -- or the residual r (defect form);
//                either way the sweeps see a zero frame.
//   Fr, Fz  radial / vertical factor blocks
//   Xa, Xb, Ea, Eb  per (line, segment) exchange: forward ends, backward
//                starts, first and last solution values
//   el0 [nr], AB [nr] pairs (alphaz, betaz), zrow [nr]
//
// One half-sweep, threads = (line, segment), phases separated by barriers:
//   A  forward elimination with zero carry-in, values kept in registers;
//   B  carry-in folded from preceding segments, fix-up, backward elimination;
//   C  carry-in folded from following segments: the line's solution, still
//      in registers; segment edges published;
//   D  the other direction's right-hand side (or the solution after the last
//      step) from the registers and the published edges, written to Ww.
// The per-element arithmetic is the Thomas algorithm of tridagr/tridagz; the
// segment carries only re-associate it (results agree to rounding).
template <typename T, int kSegThreads, bool kFull, bool kDefect, bool kPf>
__global__ void __launch_bounds__(kSegThreads, kDefect ? 2 : 1) k_adi_seg(AdiArgs a) {
    using T2 = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sm = reinterpret_cast<T *>(smraw);
    // blockIdx.x = instance * N + slot: the slot picks the coefficients, the
    // block index the slab (batches keep instances' slot arrays contiguous)
    const int local = blockIdx.x % a.nslots, row = blockIdx.x / a.nslots, tid = threadIdx.x;
    const int s = a.slot_map ? a.slot_map[local] : local;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int lane = tid & 31, warp = tid >> 5, nwarps = kSegThreads / 32;
    const int nr = a.nr, nz = a.nz, numr = a.numr, numz = a.numz;
    const SegLayout Lo = seg_layout(nr, nz);
    const int ps = Lo.ps, Pr = Lo.Pr, Pz = Lo.Pz;
    T *Ww = sm;
    T *Rw, *Fr0, *Fr1, *Fz0, *Fz1, *Xa, *Xb, *Ea, *Eb, *el0, *abp, *zrow;
    uint64_t *mbar = nullptr;  // [4]: Fr[0], Fr[1], Fz[0], Fz[1]
    if (kPf) {
        const PfLayout P = pf_layout<T>(nr, nz, !kDefect);
        Rw = reinterpret_cast<T *>(smraw + P.o_rw);
        T *F = reinterpret_cast<T *>(smraw + P.o_f);
        Fr0 = F;
        Fr1 = F + P.fpf;
        Fz0 = F + 2 * P.fpf;
        Fz1 = F + 3 * P.fpf;
        Xa = reinterpret_cast<T *>(smraw + P.o_xa);
        Ea = Xa;
        Xb = reinterpret_cast<T *>(smraw + P.o_xb);
        Eb = reinterpret_cast<T *>(smraw + P.o_eb);
        el0 = reinterpret_cast<T *>(smraw + P.o_el0);
        abp = reinterpret_cast<T *>(smraw + P.o_ab);
        zrow = kDefect ? nullptr : reinterpret_cast<T *>(smraw + P.o_zrow);
        mbar = reinterpret_cast<uint64_t *>(smraw + P.o_mbar);
    } else {
        Rw = Ww + (size_t)nz * ps;
        Fr0 = Fr1 = Rw + (size_t)nz * ps;
        Fz0 = Fz1 = Fr0 + Lo.fsz;
        Xa = Fz0 + Lo.fsz;
        Xb = Xa + Lo.xsz;
        Ea = Xb + Lo.xsz;
        Eb = Ea + Lo.xsz;
        el0 = Eb + Lo.xsz;
        abp = align_pair(el0 + nr);
        zrow = abp + 2 * nr;
    }
    T *Fr = Fr0, *Fz = Fz0;
    // factor block of relative step j (the only block without prefetch)
    auto frb = [&](int j) -> T * { return kPf ? ((j & 1) ? Fr1 : Fr0) : Fr0; };
    auto fzb = [&](int j) -> T * { return kPf ? ((j & 1) ? Fz1 : Fz0) : Fz0; };
    T2 *AB = reinterpret_cast<T2 *>(abp);
    const long long nplane = (long long)numr * numz;
    double *Pg = a.P + blk * nplane;
    const double *Rs = a.R + blk * nr * nz;
    const double gamma = a.gamma;
    const T gam_t = (T)gamma;
    const double a_side = a.alphar[numr - 2];  // alphar(numr-1)
    const bool sym_bottom = (a.isym != 1);
    const double *rad = a.rad + (long long)s * kAdiFactors * nr;
    const long long rad_step = (long long)a.N * kAdiFactors * nr;
    const long long ver_step = (long long)kAdiFactors * nz;

    const T *rad_pk = reinterpret_cast<const T *>(a.rad_pk) + (size_t)s * a.pkr;
    const size_t rad_pk_step = (size_t)a.N * a.pkr;
    const T *ver_pk = reinterpret_cast<const T *>(a.ver_pk);
    // relative step j of a direction goes to block j % 2; its fill count there is j / 2
    auto fill_r = [&](int j) {
        bulk_fill(frb(j), rad_pk + (size_t)(a.step0 + j) * rad_pk_step, (uint32_t)(a.pkr * sizeof(T)),
                  mbar + (j & 1));
    };
    auto fill_z = [&](int j) {
        bulk_fill(fzb(j), ver_pk + (size_t)(a.step0 + j) * a.pkz, (uint32_t)(a.pkz * sizeof(T)),
                  mbar + 2 + (j & 1));
    };
    auto wait_r = [&](int j) { mbar_wait(mbar + (j & 1), (uint32_t)((j >> 1) & 1), a.status); };
    auto wait_z = [&](int j) { mbar_wait(mbar + 2 + (j & 1), (uint32_t)((j >> 1) & 1), a.status); };

    if (kPf) {
        if (tid == 0) {
            for (int i = 0; i < 4; ++i) mbar_init(mbar + i, 1);
            fence_mbar_init();
        }
        __syncthreads();
        if (tid == 0) {  // set-up data: no dependence on the previous kernel
            fill_r(0);
            fill_z(0);
            if (a.nsteps_run > 1) {
                fill_r(1);
                fill_z(1);
            }
        }
    }
    for (int j = tid; j < nr; j += kSegThreads) {
        AB[j] = Vec2<T>::make((T)a.alphar[j + 1], (T)a.betar[j + 1]);
        el0[j] = (T)a.elz[(long long)s * numr + j + 1];
        if (zrow) zrow[j] = (T)0;
    }
    if (!kPf) {
        fac_load(Fr, nr, rad + a.step0 * rad_step, tid, kSegThreads);
        fac_load(Fz, nz, a.ver + a.step0 * ver_step, tid, kSegThreads);
    }
    pdl_wait();  // P and R come from the previous kernels of the solve
    if (!kDefect) {
        // Rw (source + folded Dirichlet terms) and the initial potential: 8 rows per
        // warp pass, all loads in flight before the shared-memory stores.
        for (int k0 = warp * 8; k0 < nz; k0 += nwarps * 8) {
            double rv[8][4], pv[8][4];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int k = k0 + r;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int j = lane + 32 * c;
                    const bool ok = (k < nz) && (j < nr);
                    rv[r][c] = ok ? Rs[(long long)nr * k + j] : 0.0;
                    pv[r][c] = (ok && !a.cold) ? Pg[(long long)numr * (k + 1) + 1 + j] : 0.0;
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int k = k0 + r;
                if (k >= nz) break;
                const double side_v = Pg[(numr - 1) + (long long)numr * (k + 1)];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int j = lane + 32 * c;
                    if (j >= nr) break;
                    double r0 = rv[r][c];
                    if (k == nz - 1) r0 = r0 + gamma * Pg[(j + 1) + (long long)numr * (numz - 1)];
                    if (!sym_bottom && k == 0) r0 = r0 + gamma * Pg[j + 1];
                    if (j == nr - 1) r0 = r0 - a_side * side_v;
                    Rw[k * ps + j] = (T)r0;
                    Ww[k * ps + j] = (T)pv[r][c];
                }
            }
        }
        for (int k = warp; k < nz; k += nwarps)
            for (int j = 128 + lane; j < nr; j += 32) {
                double r0 = Rs[(long long)nr * k + j];
                if (k == nz - 1) r0 = r0 + gamma * Pg[(j + 1) + (long long)numr * (numz - 1)];
                if (!sym_bottom && k == 0) r0 = r0 + gamma * Pg[j + 1];
                if (j == nr - 1) r0 = r0 - a_side * Pg[(numr - 1) + (long long)numr * (k + 1)];
                Rw[k * ps + j] = (T)r0;
                Ww[k * ps + j] = (T)(a.cold ? 0.0 : Pg[(long long)numr * (k + 1) + 1 + j]);
            }
    } else {
        // FP64 residual r = R - (Ar + Az) phi over the interior; the Dirichlet
        // columns of phi (J = numr, K = numz, K = 1 for isym 1) enter through
        // the stencil.  delta starts at zero, so the first radial right-hand
        // side is r itself (times 1/bet).
        __syncthreads();  // Fr is read below
        if (kPf) wait_r(0);
        const Fac<T> f = fac_view(Fr, nr);
        const double *brb = a.brb + (long long)s * numr;
        for (int k = warp; k < nz; k += nwarps) {
            const double *pc = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll 2
            for (int j = lane; j < nr; j += 32) {
                const double c = pc[j], e = pc[j + 1], n = pc[j + numr];
                const double w = (j > 0) ? pc[j - 1] : 0.0;
                const double so = (k > 0 || !sym_bottom) ? pc[j - numr] : 0.0;
                const double ar = brb[j + 1] * c + a.alphar[j + 1] * e + a.betar[j + 1] * w;
                const double az = a.bzb[k + 1] * c - gamma * n - gamma * so;
                const double r0 = Rs[(long long)nr * k + j] - ar - az;
                Rw[k * ps + j] = (T)r0;
                Ww[k * ps + j] = (T)r0 * f.ib[j];
            }
        }
    }
    __syncthreads();

    const int nitem_r = nz * Pr, nitem_z = nr * Pz;
    // Half-step sequence.  Drop-in: radial(i), vertical(i) for i < nsteps
    // (helmadi.F90:195-355).  Defect form: radial(0), then vertical(i),
    // radial(i): the cycle opens and closes on a radial half-step (see
    // k_adi_delta for why T = float needs that order).
    const int nhalf = kDefect ? 2 * a.nsteps_run + 1 : 2 * a.nsteps_run;
    for (int h = 0; h < nhalf; ++h) {
        const bool radial_half = (h % 2) == 0;
        const int it = kDefect ? (radial_half ? max(h / 2 - 1, 0) : (h - 1) / 2) : h / 2;
        const int step = a.step0 + it;
        const bool last_half = (h + 1 == nhalf);
        // step of the next half-step (whose right-hand side phase D writes)
        const int it_next = kDefect ? (h + 1) / 2 - ((h + 1) % 2 == 0 ? 1 : 0) : (h + 1) / 2;
        const T dtt = (T)a.dt[step];
        const T dtn = last_half ? dtt : (T)a.dt[a.step0 + it_next];
        // reload this direction's factors when its next half-step is at another step
        const bool reload = kDefect ? (h > 0 && it + 1 < a.nsteps_run) : (it + 1 < a.nsteps_run);
        if (kPf) {
            const int n = a.nsteps_run;
            if (tid == 0) {
                // refill the block whose step was used for the last time by the half-step before
                if (!kDefect) {
                    if (radial_half && it >= 1 && it + 1 < n) fill_z(it + 1);
                    if (!radial_half && it + 2 < n) fill_r(it + 2);
                } else {
                    if (!radial_half && it >= 1 && it + 1 < n) fill_r(it + 1);
                    if (radial_half && h >= 2 && it + 2 < n) fill_z(it + 2);
                }
            }
            // the blocks this half-step reads: its own direction, and the
            // other direction's 1/bet for the next right-hand side
            if (radial_half) {
                wait_r(it);
                if (!last_half) wait_z(it_next);
            } else {
                wait_z(it);
                if (!last_half) wait_r(it_next);
            }
        }

        // ================= radial half-sweep: lines k, segments along j =================
        if (radial_half) {
            const Fac<T> f = fac_view(frb(it), nr);
            T v[kAdiSeg];
            const bool active = tid < nitem_r;
            const int k = active ? tid % nz : 0, p = active ? tid / nz : 0;
            const int j0 = p * kAdiSeg, len = kFull ? kAdiSeg : min(kAdiSeg, nr - j0);
            T *wr = Ww + k * ps + j0;
            const T *rr = Rw + k * ps + j0;
            if (active) {
                T L = (T)0;
                if (!kDefect && h == 0) {
                    // first step: the right-hand side from the initial potential
                    const bool refl = (k == 0) && sym_bottom;
                    const T cphi = refl ? dtt - gam_t : dtt - (T)2 * gam_t;
                    const T cdn = refl ? (T)0 : (T)1;
                    const T *pu = (k + 1 < nz) ? wr + ps : zrow + j0;
                    const T *pd = (k > 0) ? wr - ps : zrow + j0;
#pragma unroll
                    for (int i = 0; i < kAdiSeg; ++i)
                        if (kFull || i < len) {
                            const T rhs = rr[i] + cphi * wr[i] + gam_t * (pu[i] + cdn * pd[i]);
                            L = rhs * f.ib[j0 + i] - f.dd[j0 + i] * L;
                            v[i] = L;
                        }
                } else {
#pragma unroll
                    for (int i = 0; i < kAdiSeg; ++i)
                        if (kFull || i < len) {
                            L = wr[i] - f.dd[j0 + i] * L;
                            v[i] = L;
                        }
                }
                Xa[k + nz * p] = L;
            }
            __syncthreads();
            if (active) {
                T yin = (T)0;
                for (int q = 0; q < p; ++q) yin = Xa[k + nz * q] + f.GG[min((q + 1) * kAdiSeg, nr) - 1].x * yin;
                T M = (T)0;
#pragma unroll
                for (int i = kAdiSeg - 1; i >= 0; --i)
                    if (kFull || i < len) {
                        const T2 gg = f.GG[j0 + i];
                        M = (v[i] + gg.x * yin) - gg.y * M;
                        v[i] = M;
                    }
                Xb[k + nz * p] = M;
            }
            __syncthreads();
            if (active) {
                T xin = (T)0;
                for (int q = Pr - 1; q > p; --q) xin = Xb[k + nz * q] + f.K[q * kAdiSeg] * xin;
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) v[i] = v[i] + f.K[j0 + i] * xin;
                Ea[k + nz * p] = v[0];
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (i == len - 1) Eb[k + nz * p] = v[i];
            }
            __syncthreads();
            if (active && last_half) {
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) wr[i] = v[i];
            } else if (active) {
                // vertical right-hand side of the next half-step (helmadi.F90:276-340),
                // times the vertical 1/bet of row k
                const T ibz = fac_view(fzb(it_next), nz).ib[k];
                const T left = (p > 0) ? Eb[k + nz * (p - 1)] : (T)0;
                const T right = (p + 1 < Pr) ? Ea[k + nz * (p + 1)] : (T)0;
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) {
                        const int j = j0 + i;
                        const T pl = (i > 0) ? v[i - 1] : left;
                        const T pr = (kFull ? (i + 1 < kAdiSeg) : (i + 1 < len)) ? v[(i + 1) & (kAdiSeg - 1)] : right;
                        const T2 ab = AB[j];
                        wr[i] = (rr[i] + (el0[j] + dtn) * v[i] - ab.x * pr - ab.y * pl) * ibz;
                    }
            }
            if (!kPf && reload) {
                __syncthreads();
                fac_load(Fr, nr, rad + (step + 1) * rad_step, tid, kSegThreads);
            }
            __syncthreads();
        }
        // ================= vertical half-sweep: lines j, segments along k =================
        else {
            const Fac<T> f = fac_view(fzb(it), nz);
            T v[kAdiSeg];
            const bool active = tid < nitem_z;
            const int j = active ? tid % nr : 0, p = active ? tid / nr : 0;
            const int k0 = p * kAdiSeg, len = kFull ? kAdiSeg : min(kAdiSeg, nz - k0);
            T *wc = Ww + k0 * ps + j;
            const T *rc = Rw + k0 * ps + j;
            if (active) {
                T L = (T)0;
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) {
                        L = wc[i * ps] - f.dd[k0 + i] * L;
                        v[i] = L;
                    }
                Xa[j + nr * p] = L;
            }
            __syncthreads();
            if (active) {
                T yin = (T)0;
                for (int q = 0; q < p; ++q) yin = Xa[j + nr * q] + f.GG[min((q + 1) * kAdiSeg, nz) - 1].x * yin;
                T M = (T)0;
#pragma unroll
                for (int i = kAdiSeg - 1; i >= 0; --i)
                    if (kFull || i < len) {
                        const T2 gg = f.GG[k0 + i];
                        M = (v[i] + gg.x * yin) - gg.y * M;
                        v[i] = M;
                    }
                Xb[j + nr * p] = M;
            }
            __syncthreads();
            if (active) {
                T xin = (T)0;
                for (int q = Pz - 1; q > p; --q) xin = Xb[j + nr * q] + f.K[q * kAdiSeg] * xin;
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) v[i] = v[i] + f.K[k0 + i] * xin;
                Ea[j + nr * p] = v[0];
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (i == len - 1) Eb[j + nr * p] = v[i];
            }
            __syncthreads();
            if (active) {
                if (last_half) {
#pragma unroll
                    for (int i = 0; i < kAdiSeg; ++i)
                        if (kFull || i < len) wc[i * ps] = v[i];
                } else {
                    // radial right-hand side of the next half-step (helmadi.F90:209-256),
                    // times its radial 1/bet of column j
                    const T ibr = fac_view(frb(it_next), nr).ib[j];
                    const T dn_edge = (p > 0) ? Eb[j + nr * (p - 1)] : (T)0;
                    const T up_edge = (p + 1 < Pz) ? Ea[j + nr * (p + 1)] : (T)0;
#pragma unroll
                    for (int i = 0; i < kAdiSeg; ++i)
                        if (kFull || i < len) {
                            const int k = k0 + i;
                            const bool refl = (k == 0) && sym_bottom;
                            const T up = (kFull ? (i + 1 < kAdiSeg) : (i + 1 < len)) ? v[(i + 1) & (kAdiSeg - 1)] : up_edge;
                            const T dn = (i > 0) ? v[i - 1] : dn_edge;
                            const T cphi = refl ? dtn - gam_t : dtn - (T)2 * gam_t;
                            const T rhs = refl ? rc[i * ps] + cphi * v[i] + gam_t * up
                                               : rc[i * ps] + cphi * v[i] + gam_t * (up + dn);
                            wc[i * ps] = rhs * ibr;
                        }
                }
            }
            if (!kPf && it + 1 < a.nsteps_run) {
                __syncthreads();
                fac_load(Fz, nz, a.ver + (step + 1) * ver_step, tid, kSegThreads);
            }
            __syncthreads();
        }
    }
    pdl_trigger();
    if (!kDefect) {
        if (!a.norms) {
            for (int k = warp; k < nz; k += nwarps) {
                double *prow = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll 4
                for (int j = lane; j < nr; j += 32) prow[j] = (double)Ww[k * ps + j];
            }
        } else {
            // converged cycles: the update against the potential being
            // overwritten, |new - old|^2 and |new|^2 per slot, in the write-back
            // the old values of two rows x 4 columns per lane are loaded before any store
            // (eight global loads in flight instead of one)
            double sd = 0.0, sp = 0.0;
            constexpr int kQ = 4;
            for (int k0 = warp; k0 < nz; k0 += 2 * nwarps) {
                for (int j0 = lane; j0 < nr; j0 += 32 * kQ) {
                    double o[2][kQ];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int k = k0 + h * nwarps;
                        const double *prow = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll
                        for (int q = 0; q < kQ; ++q) {
                            const int j = j0 + 32 * q;
                            o[h][q] = (k < nz && j < nr) ? prow[j] : 0.0;
                        }
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int k = k0 + h * nwarps;
                        if (k >= nz) continue;
                        double *prow = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll
                        for (int q = 0; q < kQ; ++q) {
                            const int j = j0 + 32 * q;
                            if (j >= nr) continue;
                            const double v = (double)Ww[k * ps + j];
                            const double d = v - o[h][q];
                            prow[j] = v;
                            sd += d * d;
                            sp += v * v;
                        }
                    }
                }
            }
            for (int off = 16; off > 0; off >>= 1) {
                sd += __shfl_down_sync(0xffffffffu, sd, off);
                sp += __shfl_down_sync(0xffffffffu, sp, off);
            }
            __syncthreads();
            double *red = reinterpret_cast<double *>(smraw);
            if (lane == 0) {
                red[2 * warp] = sd;
                red[2 * warp + 1] = sp;
            }
            __syncthreads();
            if (tid < 2) {
                double t = 0.0;
                for (int w = 0; w < nwarps; ++w) t += red[2 * w + tid];
                const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
                a.norms[2 * blk + tid] = wgt * t;
            }
        }
    } else {
        // phi += delta in FP64; per-slot |delta|^2 and |phi|^2
        double sd = 0.0, sp = 0.0;
        for (int k = warp; k < nz; k += nwarps) {
            double *prow = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll 2
            for (int j = lane; j < nr; j += 32) {
                const double d = (double)Ww[k * ps + j];
                const double ph = prow[j] + d;
                prow[j] = ph;
                sd += d * d;
                sp += ph * ph;
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            sd += __shfl_down_sync(0xffffffffu, sd, off);
            sp += __shfl_down_sync(0xffffffffu, sp, off);
        }
        __syncthreads();
        double *red = reinterpret_cast<double *>(smraw);
        if (lane == 0) {
            red[2 * warp] = sd;
            red[2 * warp + 1] = sp;
        }
        __syncthreads();
        if (tid < 2) {
            double t = 0.0;
            for (int w = 0; w < nwarps; ++w) t += red[2 * w + tid];
            const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
            a.norms[2 * blk + tid] = wgt * t;
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed-precision refinement cycle (k_adi_delta, T = float).
//
// One CTA per slot, two CTAs per SM.  Prologue: the FP64 residual
// r = -4 pi rho_hat - A phi of the current potential (its Dirichlet columns
// enter through the stencil), rounded to T.  Body: nsteps ADI steps of the
// defect equation A delta = r in increment form: one radial half-step at the
// first step's dt, then for every step
//   (Az + dt) D1 = r - A delta,  delta += D1,
//   (Ar + dt) D2 = r - A delta,  delta += D2,
// which is the Peaceman-Rachford iteration of helmadi.F90 rewritten so that
// every line solve sees a residual: in the plain form the intermediate
// values of stiff near-axis components (A_r up to ~1e8 x dt) are amplified
// thousands of times and T's rounding of them would not be recoverable.
// Why the cycle starts and ends on a radial half-step: where A_r is stiff
// (A_r ~ 4 k^2 / dr^2 near the axis at high k) and A_z + dt is small, a
// vertical half-step multiplies what it is given in those components by
// A_r / (A_z + dt), up to ~1e8 at 130 x 98 x 256.  In exact arithmetic the
// next radial half-step takes it back out, but T's rounding of the
// amplified values (eps32 x 1e8 ~ 6) stays.  A vertical half-step first
// would amplify the stiff part of r (the previous cycle's rounding) and a
// vertical half-step last would leave its own rounding in delta; either way
// the outer refinement grew ~5x per cycle in high-k slots.  Opening with a
// radial half-step at the largest dt (dt >= A_z everywhere, so the extra
// factor (dt - A_z)/(dt + A_r) is a contraction) resolves the stiff residual
// before any vertical half-step sees it, and closing on a radial half-step
// removes the last vertical one's rounding.  The outer FP64 defect
// correction converges to the same discrete solution whatever the inner
// order.
// Epilogue: phi += delta in FP64, per-slot |delta|^2 and |phi|^2.
//
// Shared memory (T): D = delta, Rv = r (both nz x ps), factor blocks Fr/Fz,
// segment exchange Xa/Xb, C4 [nr] = (brb, alphar, betar, 0) of the slot,
// bz [nz] = bzb.  Per line segment: A forms the residual with a sliding
// window along the line and eliminates forward with zero carry-in; B folds
// the carry-in and eliminates backward; C folds the carry-in and adds the
// increment to D.
struct DeltaLayout {
    int ps, Pr, Pz, xsz, fsz;
    size_t elems;
};

__host__ __device__ inline DeltaLayout delta_layout(int nr, int nz) {
    DeltaLayout L;
    L.ps = nr | 1;
    L.Pr = (nr + kAdiSeg - 1) / kAdiSeg;
    L.Pz = (nz + kAdiSeg - 1) / kAdiSeg;
    L.xsz = max(nz * L.Pr, nr * L.Pz);
    L.fsz = factor_block(max(nr, nz));
    L.elems = 2 * (size_t)nz * L.ps + 2 * (size_t)L.fsz + 2 * (size_t)L.xsz + 4 * (size_t)nr + (size_t)nz + 8;
    return L;
}

template <int kThreads, bool kFull>
__global__ void __launch_bounds__(kThreads, 2) k_adi_delta(AdiArgs a) {
    using T = float;
    using T2 = float2;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sm = reinterpret_cast<T *>(smraw);
    // blockIdx.x = position * N + slot; the instance of a position through the map
    const int s = blockIdx.x % a.N, row = blockIdx.x / a.N, tid = threadIdx.x;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int lane = tid & 31, warp = tid >> 5, nwarps = kThreads / 32;
    const int nr = a.nr, nz = a.nz, numr = a.numr, numz = a.numz;
    const DeltaLayout Lo = delta_layout(nr, nz);
    const int ps = Lo.ps, Pr = Lo.Pr, Pz = Lo.Pz;
    T *D = sm;
    T *Rv = D + (size_t)nz * ps;
    T *Fr = Rv + (size_t)nz * ps;
    T *Fz = Fr + Lo.fsz;
    T *Xa = Fz + Lo.fsz;
    T *Xb = Xa + Lo.xsz;
    T *c4p = Xb + Lo.xsz;
    while ((reinterpret_cast<uintptr_t>(c4p) & 15) != 0) ++c4p;
    float4 *C4 = reinterpret_cast<float4 *>(c4p);
    T *bz = c4p + 4 * nr;
    const long long nplane = (long long)numr * numz;
    double *Pg = a.P + blk * nplane;
    const double *Rs = a.R + blk * nr * nz;
    const double gamma = a.gamma;
    const T g = (T)gamma;
    const bool sym_bottom = (a.isym != 1);
    const double *rad = a.rad + (long long)s * kAdiFactors * nr;
    const long long rad_step = (long long)a.N * kAdiFactors * nr;
    const long long ver_step = (long long)kAdiFactors * nz;
    const double *brb = a.brb + (long long)s * numr;

    for (int j = tid; j < nr; j += kThreads)
        C4[j] = make_float4((T)brb[j + 1], (T)a.alphar[j + 1], (T)a.betar[j + 1], 0.f);
    for (int k = tid; k < nz; k += kThreads) bz[k] = (T)a.bzb[k + 1];
    fac_load(Fr, nr, rad + a.step0 * rad_step, tid, kThreads);
    fac_load(Fz, nz, a.ver + a.step0 * ver_step, tid, kThreads);
    pdl_wait();
    // FP64 residual of the current potential; delta = 0
    for (int k = warp; k < nz; k += nwarps) {
        const double *pc = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll 2
        for (int j = lane; j < nr; j += 32) {
            const double c = pc[j], e = pc[j + 1], n = pc[j + numr];
            const double w = (j > 0) ? pc[j - 1] : 0.0;
            const double so = (k > 0 || !sym_bottom) ? pc[j - numr] : 0.0;
            const double ar = brb[j + 1] * c + a.alphar[j + 1] * e + a.betar[j + 1] * w;
            const double az = a.bzb[k + 1] * c - gamma * n - gamma * so;
            Rv[k * ps + j] = (T)(Rs[(long long)nr * k + j] - ar - az);
            D[k * ps + j] = 0.f;
        }
    }
    __syncthreads();

    const int nitem_r = nz * Pr, nitem_z = nr * Pz;
    // Half-steps: radial at the first step's dt, then vertical and radial at
    // every step's dt (2 nsteps + 1 line solves).
    for (int h = 0; h <= 2 * a.nsteps_run; ++h) {
        const bool radial_half = (h % 2) == 0;
        const int it = radial_half ? max(h / 2 - 1, 0) : (h - 1) / 2;
        const int step = a.step0 + it;
        const bool reload = (h > 0) && (it + 1 < a.nsteps_run);
        // ================= vertical: lines j, segments along k =================
        if (!radial_half) {
            const Fac<T> f = fac_view(Fz, nz);
            T v[kAdiSeg];
            const bool active = tid < nitem_z;
            const int j = active ? tid % nr : 0, p = active ? tid / nr : 0;
            const int k0 = p * kAdiSeg, len = kFull ? kAdiSeg : min(kAdiSeg, nz - k0);
            const float4 cc = C4[j];
            const bool has_l = j > 0, has_r = j + 1 < nr;
            if (active) {
                T L = 0.f;
                T dd_ = (k0 > 0) ? D[(k0 - 1) * ps + j] : 0.f;
                T dm = D[k0 * ps + j];
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) {
                        const int k = k0 + i;
                        const T du_ = (k + 1 < nz) ? D[(k + 1) * ps + j] : 0.f;
                        const T vl = has_l ? D[k * ps + j - 1] : 0.f, vr = has_r ? D[k * ps + j + 1] : 0.f;
                        const T czn = (k > 0 || !sym_bottom) ? g : 0.f;
                        const T rhs = Rv[k * ps + j] - (cc.x * dm + cc.y * vr + cc.z * vl) -
                                      (bz[k] * dm - g * du_ - czn * dd_);
                        L = rhs * f.ib[k] - f.dd[k] * L;
                        v[i] = L;
                        dd_ = dm;
                        dm = du_;
                    }
                Xa[j + nr * p] = L;
            }
            __syncthreads();
            if (active) {
                T yin = 0.f;
                for (int q = 0; q < p; ++q) yin = Xa[j + nr * q] + f.GG[min((q + 1) * kAdiSeg, nz) - 1].x * yin;
                T M = 0.f;
#pragma unroll
                for (int i = kAdiSeg - 1; i >= 0; --i)
                    if (kFull || i < len) {
                        const T2 gg = f.GG[k0 + i];
                        M = (v[i] + gg.x * yin) - gg.y * M;
                        v[i] = M;
                    }
                Xb[j + nr * p] = M;
            }
            __syncthreads();
            if (active) {
                T xin = 0.f;
                for (int q = Pz - 1; q > p; --q) xin = Xb[j + nr * q] + f.K[q * kAdiSeg] * xin;
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) {
                        T *dw = D + (k0 + i) * ps + j;
                        *dw = *dw + (v[i] + f.K[k0 + i] * xin);
                    }
            }
            if (reload) {
                __syncthreads();
                fac_load(Fz, nz, a.ver + (step + 1) * ver_step, tid, kThreads);
            }
            __syncthreads();
        }
        // ================= radial: lines k, segments along j =================
        else {
            const Fac<T> f = fac_view(Fr, nr);
            T v[kAdiSeg];
            const bool active = tid < nitem_r;
            const int k = active ? tid % nz : 0, p = active ? tid / nz : 0;
            const int j0 = p * kAdiSeg, len = kFull ? kAdiSeg : min(kAdiSeg, nr - j0);
            const T *dc = D + k * ps;
            const T *dn = (k > 0) ? dc - ps : nullptr;
            const T *du = (k + 1 < nz) ? dc + ps : nullptr;
            const T czn = (k > 0 || !sym_bottom) ? g : 0.f;  // K-1 neighbour weight
            const T bzk = bz[k];
            if (active) {
                T L = 0.f;
                T dl = (j0 > 0) ? dc[j0 - 1] : 0.f;
                T dm = dc[j0];
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) {
                        const int j = j0 + i;
                        const T dr_ = (j + 1 < nr) ? dc[j + 1] : 0.f;
                        const T vd = (dn ? dn[j] : 0.f), vu = (du ? du[j] : 0.f);
                        const float4 cc = C4[j];
                        const T rhs = Rv[k * ps + j] - (cc.x * dm + cc.y * dr_ + cc.z * dl) -
                                      (bzk * dm - g * vu - czn * vd);
                        L = rhs * f.ib[j] - f.dd[j] * L;
                        v[i] = L;
                        dl = dm;
                        dm = dr_;
                    }
                Xa[k + nz * p] = L;
            }
            __syncthreads();
            if (active) {
                T yin = 0.f;
                for (int q = 0; q < p; ++q) yin = Xa[k + nz * q] + f.GG[min((q + 1) * kAdiSeg, nr) - 1].x * yin;
                T M = 0.f;
#pragma unroll
                for (int i = kAdiSeg - 1; i >= 0; --i)
                    if (kFull || i < len) {
                        const T2 gg = f.GG[j0 + i];
                        M = (v[i] + gg.x * yin) - gg.y * M;
                        v[i] = M;
                    }
                Xb[k + nz * p] = M;
            }
            __syncthreads();
            if (active) {
                T xin = 0.f;
                for (int q = Pr - 1; q > p; --q) xin = Xb[k + nz * q] + f.K[q * kAdiSeg] * xin;
                T *dw = D + k * ps + j0;
#pragma unroll
                for (int i = 0; i < kAdiSeg; ++i)
                    if (kFull || i < len) dw[i] = dw[i] + (v[i] + f.K[j0 + i] * xin);
            }
            if (reload) {
                __syncthreads();
                fac_load(Fr, nr, rad + (step + 1) * rad_step, tid, kThreads);
            }
            __syncthreads();
        }
    }
    // phi += delta in FP64; per-slot |delta|^2 and |phi|^2
    double sd = 0.0, sp = 0.0;
    for (int k = warp; k < nz; k += nwarps) {
        double *prow = Pg + (long long)numr * (k + 1) + 1;
#pragma unroll 2
        for (int j = lane; j < nr; j += 32) {
            const double d = (double)D[k * ps + j];
            const double ph = prow[j] + d;
            prow[j] = ph;
            sd += d * d;
            sp += ph * ph;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        sd += __shfl_down_sync(0xffffffffu, sd, off);
        sp += __shfl_down_sync(0xffffffffu, sp, off);
    }
    __syncthreads();
    double *red = reinterpret_cast<double *>(smraw);
    if (lane == 0) {
        red[2 * warp] = sd;
        red[2 * warp + 1] = sp;
    }
    __syncthreads();
    if (tid < 2) {
        double t = 0.0;
        for (int w = 0; w < nwarps; ++w) t += red[2 * w + tid];
        const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
        a.norms[2 * blk + tid] = wgt * t;
    }
}

// Weighted (Parseval) squared norms over the interior of the slot array:
// out[0] = sum w |P - prev|^2, out[1] = sum w |P|^2 (update test), or
// out[0] = sum w |R - A P|^2, out[1] = sum w |R|^2 (residual).
constexpr int kNormThreads = 256;

template <bool kResidual>
__global__ void __launch_bounds__(kNormThreads)
k_slot_norms(const double *__restrict__ P, const double *__restrict__ Q, const double *__restrict__ R,
             const double *__restrict__ brb, const double *__restrict__ alphar, const double *__restrict__ betar,
             const double *__restrict__ bzb, double gamma, int numr, int numz, int nr, int nz, int N, int isym,
             double *__restrict__ out, const int *__restrict__ map) {
    // blockIdx.x = position * N + slot; s = instance * N + slot (batch
    // instances are contiguous; map: instance of each position)
    const int row = blockIdx.x / N, sl = blockIdx.x % N;
    const int s = (map ? map[row] : row) * N + sl;
    const long long nplane = (long long)numr * numz, np = (long long)nr * nz;
    const double *Ps = P + (long long)s * nplane;
    double a0 = 0.0, a1 = 0.0;
    for (long long e = threadIdx.x; e < np; e += kNormThreads) {
        int j = (int)(e % nr), k = (int)(e / nr);
        long long q = (j + 1) + (long long)numr * (k + 1);
        if (kResidual) {
            const double *b = brb + (long long)sl * numr;
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
        double wgt = (sl == 0 || sl == N / 2) ? 1.0 : 2.0;
        out[2 * s + threadIdx.x] = wgt * v;
    }
}

}  // namespace

template <typename T, bool kDefect, bool kPf>
const void *seg_kernel_pf(int threads, bool full) {
    if (threads == 256)
        return full ? (const void *)k_adi_seg<T, 256, true, kDefect, kPf>
                    : (const void *)k_adi_seg<T, 256, false, kDefect, kPf>;
    if (threads == 384)
        return full ? (const void *)k_adi_seg<T, 384, true, kDefect, kPf>
                    : (const void *)k_adi_seg<T, 384, false, kDefect, kPf>;
    return full ? (const void *)k_adi_seg<T, 512, true, kDefect, kPf>
                : (const void *)k_adi_seg<T, 512, false, kDefect, kPf>;
}

template <typename T, bool kDefect>
const void *seg_kernel(int threads, bool full, bool pf) {
    return pf ? seg_kernel_pf<T, kDefect, true>(threads, full) : seg_kernel_pf<T, kDefect, false>(threads, full);
}

const void *delta_kernel(int threads, bool full) {
    if (threads == 256) return full ? (const void *)k_adi_delta<256, true> : (const void *)k_adi_delta<256, false>;
    if (threads == 384) return full ? (const void *)k_adi_delta<384, true> : (const void *)k_adi_delta<384, false>;
    return full ? (const void *)k_adi_delta<512, true> : (const void *)k_adi_delta<512, false>;
}

cudaError_t raise_smem_limit(const void *fn, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> limit;  // (device, kernel) -> bytes set
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    int &cur = limit[{dev, fn}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

int adi_configure(bph_ctx *c) {
    int dev_max = 0;
    cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    const SegLayout L = seg_layout(c->nr, c->nz);
    const size_t seg_bytes = sizeof(double) * L.elems + 16;
    const size_t mixed_bytes = sizeof(float) * L.elems + 16;  // forwarding form, T = float
    const size_t onchip = sizeof(double) * 2 * (size_t)c->nz * (size_t)(c->nr | 1) + smalls_bytes(c);
    const int items = max(c->nz * L.Pr, c->nr * L.Pz);
    const int threads = (items <= 256) ? 256 : (items <= 384) ? 384 : 512;
    // Factor prefetch by bulk copy: on by default for the FP32 refinement
    // kernel (74.8 against 85.3 us per 5-step cycle at 130x98x256 on B200),
    // off for the FP64 drop-in, where it measured slower (101 against 95 us):
    // the FP64 kernel's in-place reload costs ~5 us and the extra waits more.
    // BPH_ADI_PREFETCH=0 turns it off everywhere, =1 on everywhere.
    const char *pfenv = std::getenv("BPH_ADI_PREFETCH");
    const bool pf_allowed = !(pfenv && pfenv[0] == '0');
    const bool pf_fp64 = pfenv && pfenv[0] == '1';
    c->adi_seg = 0;
    c->adi_smem = 0;
    c->adi_mixed_smem = 0;
    c->adi_pf = false;
    c->mixed_pf = false;
    c->adi_full = (c->nr % kAdiSeg == 0) && (c->nz % kAdiSeg == 0);
    const size_t seg_pf_bytes = pf_layout<double>(c->nr, c->nz, true).bytes;
    if (items <= 512 && (seg_bytes <= (size_t)dev_max || (pf_fp64 && seg_pf_bytes <= (size_t)dev_max))) {
        c->adi_seg = threads;
        c->adi_pf = pf_fp64 && seg_pf_bytes <= (size_t)dev_max;
        c->adi_smem = (int)(c->adi_pf ? seg_pf_bytes : seg_bytes);
        e = raise_smem_limit(seg_kernel<double, false>(c->adi_seg, c->adi_full, c->adi_pf), c->adi_smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_adi_seg)");
    } else if (onchip <= (size_t)dev_max) {
        c->adi_smem = (int)onchip;
        e = raise_smem_limit((const void *)k_adi<true>, c->adi_smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_adi)");
    }
    // FP32 refinement kernels: the forwarding form (k_adi_seg<float>) and the
    // increment form (k_adi_delta), both with the same thread count.
    const DeltaLayout DL = delta_layout(c->nr, c->nz);
    const size_t delta_bytes = sizeof(float) * DL.elems + 16;
    c->adi_mixed_threads = 0;
    c->mixed_kind = 0;
    // forwarding form: the prefetching variant when it keeps the resident CTAs per SM
    if (pf_allowed && items <= 512) {
        const size_t pf_bytes = pf_layout<float>(c->nr, c->nz, false).bytes;
        if (pf_bytes <= (size_t)dev_max && mixed_bytes <= (size_t)dev_max) {
            int occ_pf = 0, occ = 0;
            const void *fpf = seg_kernel<float, true>(threads, c->adi_full, true);
            const void *fno = seg_kernel<float, true>(threads, c->adi_full, false);
            e = raise_smem_limit(fpf, (int)pf_bytes);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(fpf, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            if (e == cudaSuccess) e = raise_smem_limit(fno, (int)mixed_bytes);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(fno, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_pf, fpf, threads, (int)pf_bytes);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fno, threads, (int)mixed_bytes);
            if (e != cudaSuccess) return cuda_fail(e, "refinement ADI occupancy");
            c->mixed_pf = occ_pf >= occ && occ_pf > 0;
        } else if (pf_bytes <= (size_t)dev_max) {
            c->mixed_pf = true;
        }
    }
    const size_t fwd_bytes = c->mixed_pf ? pf_layout<float>(c->nr, c->nz, false).bytes : mixed_bytes;
    for (int kind = 1; kind <= 2; ++kind) {
        c->mixed_smem_kind[kind] = 0;
        c->mixed_per_sm_kind[kind] = 0;
        const size_t bytes = (kind == BPH_MIXED_ADI_FORWARD) ? fwd_bytes : delta_bytes;
        if (bytes > (size_t)dev_max || items > 512) continue;
        const void *fn = (kind == BPH_MIXED_ADI_FORWARD) ? seg_kernel<float, true>(threads, c->adi_full, c->mixed_pf)
                                                         : delta_kernel(threads, c->adi_full);
        e = raise_smem_limit(fn, (int)bytes);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(refinement ADI)");
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->mixed_per_sm_kind[kind], fn, threads, (int)bytes);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        c->mixed_smem_kind[kind] = (int)bytes;
        c->adi_mixed_threads = threads;
        if (!c->mixed_kind) c->mixed_kind = kind;
    }
    int rc = large_configure(c);
    if (rc) return rc;
    // the grid-wide kernels fit every practical grid: the default when neither on-chip kernel does
    c->mixed_smem_kind[BPH_MIXED_ADI_GLOBAL] = c->large_kb[1] ? 1 : 0;
    c->mixed_per_sm_kind[BPH_MIXED_ADI_GLOBAL] = 0;
    if (!c->mixed_kind) c->mixed_kind = BPH_MIXED_ADI_GLOBAL;
    if (!c->adi_mixed_threads) c->adi_mixed_threads = kAdiThreads;
    return select_mixed_kind(c, c->mixed_kind);
}

int select_mixed_kind(bph_ctx *c, int kind) {
    if (kind < 1 || kind > 5 || !c->mixed_smem_kind[kind]) {
        c->adi_mixed_smem = 0;
        c->adi_mixed_per_sm = 0;
        return (kind == 0) ? BPH_OK : BPH_ERR_INVALID;
    }
    c->mixed_kind = kind;
    c->adi_mixed_smem = c->mixed_smem_kind[kind];
    c->adi_mixed_per_sm = c->mixed_per_sm_kind[kind];
    return BPH_OK;
}

AdiArgs make_args(bph_ctx *c, const Schedule &sch, int step0, int nsteps_run, bool cold) {
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
    a.brb = c->d_brb;
    a.bzb = c->d_bzb;
    a.norms = nullptr;  // FP64 sweeps: set to get update norms from the write-back
    a.inst_map = nullptr;
    a.slot_map = nullptr;
    a.nslots = c->N;
    a.rad_pk = sch.d_rad_pk[0];
    a.ver_pk = sch.d_ver_pk[0];
    a.pkr = packed_block<double>(c->nr);
    a.pkz = packed_block<double>(c->nz);
    a.status = c->d_status;
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
    return a;
}

cudaError_t launch_adi(bph_ctx *c, const Schedule &sch, int step0, int nsteps_run, bool cold, double *P,
                       const double *R, int ninst, const int *d_inst_map, double *norms) {
    AdiArgs a = make_args(c, sch, step0, nsteps_run, cold);
    if (P) a.P = P;
    if (R) a.R = R;
    a.inst_map = d_inst_map;
    if (norms && !c->adi_seg) return cudaErrorNotSupported;  // only the on-chip kernels report them
    a.norms = norms;
    if (c->adi_warp)
        return launch_adi_warp(c, sch, step0, nsteps_run, cold, a.P, a.R, ninst, d_inst_map, nullptr, c->N, norms,
                               c->stream, c->pdl);
    if (c->adi_seg) {
        ++c->launches;
        void *args[] = {&a};
        cudaLaunchAttribute attr[1];
        cudaLaunchConfig_t cfg = launch_config(c, dim3(c->N * ninst), dim3(c->adi_seg), (size_t)c->adi_smem, attr);
        return cudaLaunchKernelExC(&cfg, seg_kernel<double, false>(c->adi_seg, c->adi_full, c->adi_pf), args);
    }
    // other variants: one launch per instance (batches need the on-chip kernel)
    if (d_inst_map) return cudaErrorNotSupported;
    for (int i = 0; i < ninst; ++i) {
        AdiArgs ai = a;
        ai.P = a.P + (long long)i * c->N * c->nplane;
        ai.R = a.R + (long long)i * c->N * c->np;
        cudaError_t e;
        if (c->adi_smem > 0) {
            ++c->launches;
            k_adi<true><<<c->N, kAdiThreads, c->adi_smem, c->stream>>>(ai);
            e = cudaGetLastError();
        } else {
            e = launch_adi_large(c, sch, step0, nsteps_run, cold, ai.P, ai.R);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_adi_slots(bph_ctx *c, const Schedule &sch, bool cold, const int *d_slots, int nslots,
                             cudaStream_t st, bool pdl) {
    if (!c->adi_seg || nslots < 1) return cudaErrorNotSupported;
    if (c->adi_warp)
        return launch_adi_warp(c, sch, 0, sch.nsteps, cold, c->d_P, c->d_R, 1, nullptr, d_slots, nslots, nullptr, st,
                               pdl);
    AdiArgs a = make_args(c, sch, 0, sch.nsteps, cold);
    a.slot_map = d_slots;
    a.nslots = nslots;
    ++c->launches;
    void *args[] = {&a};
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, dim3(nslots), dim3(c->adi_seg), (size_t)c->adi_smem, attr);
    cfg.stream = st;
    if (!pdl) cfg.numAttrs = 0;
    return cudaLaunchKernelExC(&cfg, seg_kernel<double, false>(c->adi_seg, c->adi_full, c->adi_pf), args);
}

cudaError_t launch_adi_defect(bph_ctx *c, const Schedule &sch) {
    if (!c->adi_mixed_smem) return cudaErrorNotSupported;
    if (c->mixed_kind == BPH_MIXED_DIRECT) return launch_defect_direct(c, c->d_P, c->d_R, 1, nullptr, c->d_red);
    AdiArgs a = make_args(c, sch, 0, sch.nsteps, false);
    a.norms = c->d_red;
    a.rad_pk = sch.d_rad_pk[1];  // float blocks for the FP32 kernels
    a.ver_pk = sch.d_ver_pk[1];
    a.pkr = packed_block<float>(c->nr);
    a.pkz = packed_block<float>(c->nz);
    if (c->mixed_kind == BPH_MIXED_ADI_WARP) return launch_defect_warp(c, sch, c->d_P, c->d_R, 1, nullptr, c->d_red, c->d_r32);
    ++c->launches;
    void *args[] = {&a};
    if (c->mixed_kind == BPH_MIXED_ADI_GLOBAL) {
        if (!c->d_work32) return cudaErrorNotReady;  // ensure_mixed_work first
        --c->launches;  // counted per kernel there
        return launch_adi_defect_large(c, sch);
    }
    const void *fn = (c->mixed_kind == BPH_MIXED_ADI_FORWARD)
                         ? seg_kernel<float, true>(c->adi_mixed_threads, c->adi_full, c->mixed_pf)
                         : delta_kernel(c->adi_mixed_threads, c->adi_full);
    return cudaLaunchKernel(fn, dim3(c->N), dim3(c->adi_mixed_threads), args, (size_t)c->adi_mixed_smem,
                            c->stream);
}

cudaError_t launch_defect_batch(bph_ctx *c, const Schedule &sch, double *P, const double *R, int n, const int *d_map,
                                double *norms) {
    if (!c->adi_mixed_smem || c->mixed_kind == BPH_MIXED_ADI_GLOBAL) return cudaErrorNotSupported;
    if (c->mixed_kind == BPH_MIXED_ADI_WARP) return cudaErrorNotSupported;  // launch_defect_batch_warp
    if (c->mixed_kind == BPH_MIXED_DIRECT) return cudaErrorNotSupported;  // launch_defect_direct with the batch's scratch
    AdiArgs a = make_args(c, sch, 0, sch.nsteps, false);
    a.P = P;
    a.R = R;
    a.norms = norms;
    a.inst_map = d_map;
    a.rad_pk = sch.d_rad_pk[1];
    a.ver_pk = sch.d_ver_pk[1];
    a.pkr = packed_block<float>(c->nr);
    a.pkz = packed_block<float>(c->nz);
    ++c->launches;
    void *args[] = {&a};
    const void *fn = (c->mixed_kind == BPH_MIXED_ADI_FORWARD)
                         ? seg_kernel<float, true>(c->adi_mixed_threads, c->adi_full, c->mixed_pf)
                         : delta_kernel(c->adi_mixed_threads, c->adi_full);
    return cudaLaunchKernel(fn, dim3((unsigned)(c->N * n)), dim3(c->adi_mixed_threads), args,
                            (size_t)c->adi_mixed_smem, c->stream);
}

cudaError_t launch_norms_batch(bph_ctx *c, bool residual, const double *P, const double *prev, const double *R, int n,
                               const int *d_map, double *d_out) {
    ++c->launches;
    if (residual)
        k_slot_norms<true><<<c->N * n, kNormThreads, 0, c->stream>>>(
            P, prev, R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz, c->nr, c->nz,
            c->N, c->g.isym, d_out, d_map);
    else
        k_slot_norms<false><<<c->N * n, kNormThreads, 0, c->stream>>>(
            P, prev, R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz, c->nr, c->nz,
            c->N, c->g.isym, d_out, d_map);
    return cudaGetLastError();
}

cudaError_t launch_update_norm(bph_ctx *c, double *d_out) {
    ++c->launches;
    k_slot_norms<false><<<c->N, kNormThreads, 0, c->stream>>>(
        c->d_P, c->d_prev, c->d_R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz,
        c->nr, c->nz, c->N, c->g.isym, d_out, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_residual_norm(bph_ctx *c, double *d_out) {
    ++c->launches;
    k_slot_norms<true><<<c->N, kNormThreads, 0, c->stream>>>(
        c->d_P, c->d_prev, c->d_R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz,
        c->nr, c->nz, c->N, c->g.isym, d_out, nullptr);
    return cudaGetLastError();
}

}  // namespace bph
