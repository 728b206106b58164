// bph_adi_large.cu -- ADI for slots too large for shared memory.
//
// When a slot's slabs exceed an SM's shared memory (e.g. 258 x 194 x 512),
// the slots are cut into panels instead of one CTA per slot.  Every array
// stays in layout A ([k][j], j contiguous), and each half-sweep is ONE
// grid-wide kernel that also produces the next half-sweep's right-hand side:
//   k_large_radial    CTA = (slot, kb consecutive rows k): loads the radial
//       right-hand side rows (contiguous, by asynchronous copies), solves
//       the r-lines in shared memory (tridagr, each line partitioned over
//       several threads), then writes the vertical
//       right-hand side of the same rows (it needs q at j-1, j, j+1, all in
//       the CTA) -- or the result, after the last half-sweep;
//   k_large_vertical  CTA = (slot, NL consecutive columns j): loads the
//       vertical right-hand side (row segments of NL), solves the z-lines
//       (tridagz), then writes the next step's radial right-hand side (it
//       needs phi at k-1, k, k+1 of the same column) -- or the potential.
//   k_large_rhs0      the first radial right-hand side, from the warm
//       potential (zero when cold).
// Per step and zone: 8 bytes in, the source term and 8 bytes out per
// kernel (48 bytes per step), against 112 for separate right-hand-side and
// line kernels.
//
// The same kernels, in FP32 and with a zero Dirichlet frame, run the
// mixed-precision refinement cycle on the defect equation (prologue: the
// FP64 residual; body: radial at the first step's dt, then vertical and
// radial per step; epilogue: phi += delta in FP64 and the per-slot norms).
#include <cstdlib>

#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kPanelThreads = 256;
// Lines of a panel (columns of a vertical panel, at most the rows of a
// radial one): 16 for FP64, 32 for FP32, so that the lanes sharing a sweep
// segment fill the shared-memory banks once.
template <typename T>
constexpr int panel_lines() {
    return sizeof(T) == 8 ? 16 : 32;
}
constexpr int kEmit = 8;            // source loads a thread keeps in flight while emitting

template <typename T>
struct Large {
    T *phi;                 // layout A: element (k, j) of slot s at phi + s*phi_slot + phi_off + k*phi_row + j
    long long phi_slot, phi_off;
    int phi_row;
    const T *src;           // -4 pi rho_hat (drop-in) or the defect r, packed [N][nz][nr]
    T *W, *Q;               // radial and vertical right-hand sides, [rows][nz][nr]
    const double *P;        // slot array for the Dirichlet frame; nullptr: zero frame
    const double *rad, *ver;
    const double *elz, *alphar, *betar;
    const int *inst_map;    // batches: instance of each row of N slots (nullptr: row = instance)
    int numr, numz, nr, nz, N, isym;
    double gamma;
    int kb;                 // rows of a radial panel
    int ustride;            // shared-memory row stride of a radial panel (odd: no bank conflicts)
};

// blockIdx.y = row * N + slot; the slot picks coefficients and factors,
// the instance (through the map) the data, the row the scratch W/Q.
struct Where {
    int sl;             // slot within its instance
    long long sg;       // slot index of the data arrays (instance * N + slot)
    long long sw;       // slot index of the scratch arrays
};

template <typename T>
__device__ __forceinline__ Where where(const Large<T> &a) {
    Where w;
    const int row = blockIdx.y / a.N;
    w.sl = blockIdx.y % a.N;
    w.sg = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + w.sl;
    w.sw = blockIdx.y;
    return w;
}

// Asynchronous element copy global -> shared (no register round trip, so a
// thread keeps all of its panel loads in flight at once).
template <typename T>
__device__ __forceinline__ void async_copy(T *dst, const T *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

// Warms L2 with the 128-byte line holding p (the source rows that a panel
// reads after its line solves: their loads then wait on L2, not DRAM).
__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ void async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// Partitioned Thomas sweep with precomputed factors (tridagr.F90 /
// tridagz.F90) on NL lines x[0], x[st], ..., x[(n-1) st] in shared memory,
// in place:  forward  y_i = x_i ib_i - dd_i y_{i-1},  backward  x_i = y_i -
// gm_{i+1} x_{i+1}.  Thread t owns segment t / NL of line t % NL: every
// segment solves its recurrence from a zero start while tracking the
// product of its coefficients (the affine map of its incoming value), the
// maps are composed across segments through shared memory, and a second
// pass adds the incoming value times the running product.  The lanes that
// share a segment address NL different lines (no bank conflicts for an odd
// line stride: NL = 32 for 4-byte, 16 for 8-byte elements).  Every thread
// of the CTA calls it (barriers inside); lanes with active == false own
// empty segments.
template <typename T, int NL>
__device__ __forceinline__ void thomas_panel(T *x, int st, int n, const T *ib, const T *dd, const T *gm, bool active,
                                             T (*sY)[NL], T (*sP)[NL]) {
    constexpr int NS = kPanelThreads / NL;  // segments per line
    const int seg = threadIdx.x / NL, lane = threadIdx.x % NL;
    // odd segment length: the lanes of neighbouring segments read their
    // factors (and, for a line stride of 1, their elements) from different banks
    const int L = ((n + NS - 1) / NS) | 1;
    const int a = active ? min(n, seg * L) : 0, b = active ? min(n, a + L) : 0;
    // forward, local: y from zero, p = product of -dd (0 once row 0 is in)
    T y = 0, p = 1;
#pragma unroll 4
    for (int i = a; i < b; ++i) {
        const T t = x[i * st] * ib[i];
        if (i == 0) {
            y = t;
            p = 0;
        } else {
            y = t - dd[i] * y;
            p = -dd[i] * p;
        }
        x[i * st] = y;
    }
    sY[seg][lane] = y;
    sP[seg][lane] = p;
    __syncthreads();
    if (seg > 0 && a < b) {
        T cin = 0;  // true y just below the segment: maps of segments 0..seg-1
        for (int s = 0; s < seg; ++s) cin = sY[s][lane] + sP[s][lane] * cin;
        T q = 1;
#pragma unroll 4
        for (int i = a; i < b; ++i) {
            q = -dd[i] * q;
            x[i * st] += q * cin;
        }
    }
    __syncthreads();
    // backward, local: x from zero above the segment, q = product of -gm
    T xl = 0, q = 1;
#pragma unroll 4
    for (int i = b - 1; i >= a; --i) {
        if (i == n - 1) {
            xl = x[i * st];
            q = 0;
        } else {
            xl = x[i * st] - gm[i + 1] * xl;
            q = -gm[i + 1] * q;
        }
        x[i * st] = xl;
    }
    sY[seg][lane] = xl;
    sP[seg][lane] = q;
    __syncthreads();
    if (seg < NS - 1 && a < b) {
        T cin = 0;  // true x just above the segment: maps of the segments above
        for (int s = NS - 1; s > seg; --s) cin = sY[s][lane] + sP[s][lane] * cin;
        T r = 1;
#pragma unroll 4
        for (int i = b - 1; i >= a; --i) {
            r = (i == n - 1) ? (T)0 : -gm[i + 1] * r;
            x[i * st] += r * cin;
        }
    }
}

// Radial right-hand side at (k, j) (helmadi.F90:203-256) from phi at
// (k-1, j), (k, j), (k+1, j) in the interior; the frame values come from P.
template <typename T>
__device__ __forceinline__ T rhs_radial(const Large<T> &a, const double *Pg, T r, T phi, T up, T dn, int k, int j,
                                        T dt) {
    const bool sym_bottom = (a.isym != 1);
    const T g = (T)a.gamma;
    if (k + 1 >= a.nz) up = Pg ? (T)Pg[(j + 1) + (long long)a.numr * (a.numz - 1)] : (T)0;
    if (k == 0) dn = (Pg && !sym_bottom) ? (T)Pg[j + 1] : (T)0;
    T v = (k == 0 && sym_bottom) ? r + (dt - g) * phi + g * up : r + (dt - (T)2 * g) * phi + g * (up + dn);
    if (j == a.nr - 1 && Pg) v = v - (T)a.alphar[a.numr - 2] * (T)Pg[(a.numr - 1) + (long long)a.numr * (k + 1)];
    return v;
}

// First radial right-hand side of a sweep: from the potential in phi (or
// zero when cold); grid (j blocks, k blocks of kRhs0Rows, rows * N slots).
// A thread walks kRhs0Rows rows of one column, so each phi value is loaded
// once and all of its loads are in flight together.
constexpr int kRhs0Rows = 8;

template <typename T>
__global__ void __launch_bounds__(128) k_large_rhs0(Large<T> a, T dt, int cold) {
    const int j = blockIdx.x * 128 + threadIdx.x, k0 = blockIdx.y * kRhs0Rows;
    if (j >= a.nr) return;
    const int row = blockIdx.z / a.N, sl = blockIdx.z - row * a.N;
    const long long sg = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + sl;
    const long long np = (long long)a.nr * a.nz;
    const double *Pg = a.P ? a.P + sg * (long long)a.numr * a.numz : nullptr;
    const T *ph = a.phi + sg * a.phi_slot + a.phi_off + j;
    const T *src = a.src + sg * np + j;
    T *W = a.W + (long long)blockIdx.z * np + j;
    T v[kRhs0Rows + 2], r[kRhs0Rows];  // v[m] = phi at row k0 - 1 + m
#pragma unroll
    for (int m = 0; m < kRhs0Rows + 2; ++m) {
        const int k = k0 - 1 + m;
        v[m] = (!cold && k >= 0 && k < a.nz) ? ph[(long long)k * a.phi_row] : (T)0;
    }
#pragma unroll
    for (int m = 0; m < kRhs0Rows; ++m) {
        const int k = k0 + m;
        r[m] = (k < a.nz) ? src[(long long)k * a.nr] : (T)0;
    }
#pragma unroll
    for (int m = 0; m < kRhs0Rows; ++m) {
        const int k = k0 + m;
        if (k < a.nz) W[(long long)k * a.nr] = rhs_radial(a, Pg, r[m], v[m + 1], v[m + 2], v[m], k, j, dt);
    }
}

// Radial half-sweep on a panel of kb rows: W -> (r-lines) -> Q = vertical
// right-hand side at dt_next, or -> phi when last.
template <typename T, int NL>
__global__ void __launch_bounds__(kPanelThreads) k_large_radial(Large<T> a, int step, T dt_next, int last) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *U = reinterpret_cast<T *>(smem_raw);
    const Where wh = where(a);
    const int nr = a.nr, nz = a.nz, us = a.ustride;
    const int k0 = blockIdx.x * a.kb, kb = min(a.kb, nz - k0);
    T *fib = U + (long long)a.kb * us, *fdd = fib + nr, *fgm = fdd + nr;
    const long long np = (long long)nr * nz;
    const T *Wg = a.W + wh.sw * np + (long long)k0 * nr;
    for (int e = threadIdx.x; e < kb * nr; e += kPanelThreads) {
        const int kl = e / nr, j = e - kl * nr;
        async_copy(U + kl * us + j, Wg + e);
    }
    if (!last) {
        const char *sp = reinterpret_cast<const char *>(a.src + wh.sg * np + (long long)k0 * nr);
        const int lines = (int)((sizeof(T) * (size_t)kb * nr + 127) / 128);
        for (int l = threadIdx.x; l < lines; l += kPanelThreads) prefetch_l2(sp + 128 * (size_t)l);
    }
    const double *f = a.rad + ((long long)step * a.N + wh.sl) * kAdiFactors * nr;
    for (int j = threadIdx.x; j < nr; j += kPanelThreads) {
        fib[j] = (T)f[j];
        fdd[j] = (T)f[nr + j];
        fgm[j] = (T)f[2 * nr + j];
    }
    async_wait_all();
    __syncthreads();
    {  // tridagr.F90: an r-line per lane, four segments (warps)
        __shared__ T sY[kPanelThreads / NL][NL], sP[kPanelThreads / NL][NL];
        const int line = threadIdx.x % NL;
        thomas_panel<T, NL>(U + min(line, kb - 1) * us, 1, nr, fib, fdd, fgm, line < kb, sY, sP);
    }
    __syncthreads();
    if (last) {
        T *ph = a.phi + wh.sg * a.phi_slot + a.phi_off + (long long)k0 * a.phi_row;
        for (int j = threadIdx.x; j < nr; j += kPanelThreads)
            for (int kl = 0; kl < kb; ++kl) ph[(long long)kl * a.phi_row + j] = U[kl * us + j];
        return;
    }
    // vertical right-hand side (helmadi.F90:272-340) of the panel's rows:
    // a thread per column, its coefficients in registers, kEmit source rows
    // in flight at a time
    const double *Pg = a.P ? a.P + wh.sg * (long long)a.numr * a.numz : nullptr;
    const bool sym_bottom = (a.isym != 1);
    const T g = (T)a.gamma;
    const T *sgp = a.src + wh.sg * np + (long long)k0 * nr;
    T *Qg = a.Q + wh.sw * np + (long long)k0 * nr;
    const double *elz = a.elz + (long long)wh.sl * a.numr;
    for (int j = threadIdx.x; j < nr; j += kPanelThreads) {
        const T cz = (T)elz[j + 1] + dt_next, al = (T)a.alphar[j + 1], be = (T)a.betar[j + 1];
        const T top = Pg ? g * (T)Pg[(j + 1) + (long long)a.numr * (a.numz - 1)] : (T)0;
        const T bot = (Pg && !sym_bottom) ? g * (T)Pg[j + 1] : (T)0;
        for (int kl0 = 0; kl0 < kb; kl0 += kEmit) {
            T sv[kEmit];
#pragma unroll
            for (int m = 0; m < kEmit; ++m) sv[m] = (kl0 + m < kb) ? sgp[(long long)(kl0 + m) * nr + j] : (T)0;
#pragma unroll
            for (int m = 0; m < kEmit; ++m) {
                const int kl = kl0 + m, k = k0 + kl;
                if (kl >= kb) break;
                const T *qc = U + kl * us + j;
                T right;
                if (j + 1 < nr) right = qc[1];
                else right = Pg ? (T)Pg[(a.numr - 1) + (long long)a.numr * (k + 1)] : (T)0;
                T v = cz * qc[0] - al * right;
                if (j > 0) v = v - be * qc[-1];
                v = sv[m] + v;
                if (k == nz - 1) v = v + top;
                if (k == 0) v = v + bot;
                Qg[(long long)kl * nr + j] = v;
            }
        }
    }
}

// Vertical half-sweep on a panel of NL columns: Q -> (z-lines) -> W =
// radial right-hand side at dt_next, or -> phi when last.
template <typename T, int NL>
__global__ void __launch_bounds__(kPanelThreads) k_large_vertical(Large<T> a, int step, T dt_next, int last) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *V = reinterpret_cast<T *>(smem_raw);
    constexpr int vs = NL + 1;
    const Where wh = where(a);
    const int nr = a.nr, nz = a.nz;
    const int j0 = blockIdx.x * NL, jb = min(NL, nr - j0);
    T *fib = V + (long long)nz * vs, *fdd = fib + nz, *fgm = fdd + nz;
    const long long np = (long long)nr * nz;
    const T *Qg = a.Q + wh.sw * np + j0;
    for (int e = threadIdx.x; e < nz * NL; e += kPanelThreads) {
        const int k = e / NL, jl = e - k * NL;
        if (jl < jb) async_copy(V + k * vs + jl, Qg + (long long)k * nr + jl);
    }
    if (!last) {
        const T *sp = a.src + wh.sg * np + j0;
        const int per_row = (int)((sizeof(T) * (size_t)jb + 127) / 128) + 1;  // the rows need not start on a line
        for (int l = threadIdx.x; l < nz * per_row; l += kPanelThreads) {
            const int k = l / per_row, c = l - k * per_row;
            const size_t start = reinterpret_cast<size_t>(sp + (long long)k * nr), end = start + sizeof(T) * jb;
            const size_t at = c ? (start & ~(size_t)127) + 128 * (size_t)c : start;  // stays inside the row's block
            if (at < end) prefetch_l2(reinterpret_cast<const void *>(at));
        }
    }
    const double *f = a.ver + (long long)step * kAdiFactors * nz;
    for (int k = threadIdx.x; k < nz; k += kPanelThreads) {
        fib[k] = (T)f[k];
        fdd[k] = (T)f[nz + k];
        fgm[k] = (T)f[2 * nz + k];
    }
    async_wait_all();
    __syncthreads();
    {  // tridagz.F90: a z-line per lane, four segments (warps)
        __shared__ T sY[kPanelThreads / NL][NL], sP[kPanelThreads / NL][NL];
        const int line = threadIdx.x % NL;
        thomas_panel<T, NL>(V + min(line, jb - 1), vs, nz, fib, fdd, fgm, line < jb, sY, sP);
    }
    __syncthreads();
    const int jl = threadIdx.x % NL, kg = threadIdx.x / NL;
    constexpr int kRowGroups = kPanelThreads / NL;
    if (last) {
        if (jl < jb) {
            T *ph = a.phi + wh.sg * a.phi_slot + a.phi_off + j0 + jl;
            for (int k = kg; k < nz; k += kRowGroups) ph[(long long)k * a.phi_row] = V[k * vs + jl];
        }
        return;
    }
    if (jl >= jb) return;
    // next radial right-hand side (helmadi.F90:203-256): a thread per
    // (column, row group), kEmit source rows in flight at a time
    const double *Pg = a.P ? a.P + wh.sg * (long long)a.numr * a.numz : nullptr;
    const bool sym_bottom = (a.isym != 1);
    const int j = j0 + jl;
    const T g = (T)a.gamma, dt = dt_next;
    const T top = Pg ? (T)Pg[(j + 1) + (long long)a.numr * (a.numz - 1)] : (T)0;
    const T bot = (Pg && !sym_bottom) ? (T)Pg[j + 1] : (T)0;
    const bool edge = (j == nr - 1) && Pg;
    const T aedge = edge ? (T)a.alphar[a.numr - 2] : (T)0;
    const T *sgp = a.src + wh.sg * np + j;
    T *Wg = a.W + wh.sw * np + j;
    for (int k0r = kg; k0r < nz; k0r += kEmit * kRowGroups) {
        T sv[kEmit];
#pragma unroll
        for (int m = 0; m < kEmit; ++m) {
            const int k = k0r + m * kRowGroups;
            sv[m] = (k < nz) ? sgp[(long long)k * nr] : (T)0;
        }
#pragma unroll
        for (int m = 0; m < kEmit; ++m) {
            const int k = k0r + m * kRowGroups;
            if (k >= nz) break;
            const T *vc = V + k * vs + jl;
            const T phi = vc[0];
            const T up = (k + 1 < nz) ? vc[vs] : top;
            const T dn = (k > 0) ? vc[-vs] : bot;
            T v = (k == 0 && sym_bottom) ? sv[m] + (dt - g) * phi + g * up
                                         : sv[m] + (dt - (T)2 * g) * phi + g * (up + dn);
            if (edge) v = v - aedge * (T)Pg[(a.numr - 1) + (long long)a.numr * (k + 1)];
            Wg[(long long)k * nr] = v;
        }
    }
}

// FP64 residual r = -4 pi rho_hat - A phi of the current potential (its
// Dirichlet columns through the stencil), stored in T; delta = 0.  Thread
// per (position, slot, zone); P and R of instance map[position] (map
// nullptr: position = instance), r and delta by position.
template <typename T>
__global__ void k_large_defect_prologue(const double *__restrict__ P, const double *__restrict__ R,
                                        const double *__restrict__ brb, const double *__restrict__ alphar,
                                        const double *__restrict__ betar, const double *__restrict__ bzb,
                                        double gamma, int numr, int numz, int nr, int nz, int N, int isym, int npos,
                                        const int *__restrict__ map, T *__restrict__ r, T *__restrict__ delta) {
    const long long np = (long long)nr * nz, nplane = (long long)numr * numz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np * N * npos) return;
    const long long sp = t / np;  // position * N + slot
    const int row = (int)(sp / N), s = (int)(sp % N);
    const long long si = (long long)(map ? map[row] : row) * N + s;
    const long long e = t - sp * np;
    const int j = (int)(e % nr), k = (int)(e / nr);
    const bool sym_bottom = (isym != 1);
    const double *pc = P + si * nplane + (long long)numr * (k + 1) + 1;
    const double c = pc[j], east = pc[j + 1], n = pc[j + numr];
    const double w = (j > 0) ? pc[j - 1] : 0.0;
    const double so = (k > 0 || !sym_bottom) ? pc[j - numr] : 0.0;
    const double *b = brb + (long long)s * numr;
    const double ar = b[j + 1] * c + alphar[j + 1] * east + betar[j + 1] * w;
    const double az = bzb[k + 1] * c - gamma * n - gamma * so;
    r[t] = (T)(R[si * np + e] - ar - az);
    delta[t] = (T)0;
}

// phi += delta in FP64 and the per-slot |delta|^2, |phi|^2 (one CTA per
// position and slot; norms indexed by instance * N + slot)
template <typename T>
__global__ void __launch_bounds__(256) k_large_defect_epilogue(double *__restrict__ P, const T *__restrict__ delta,
                                                               int numr, int numz, int nr, int nz, int N,
                                                               const int *__restrict__ map,
                                                               double *__restrict__ norms) {
    const int row = blockIdx.x / N, s = blockIdx.x % N;
    const long long si = (long long)(map ? map[row] : row) * N + s;
    const long long np = (long long)nr * nz, nplane = (long long)numr * numz;
    double *Pg = P + si * nplane;
    const T *d = delta + (long long)blockIdx.x * np;
    double sd = 0.0, sp = 0.0;
    for (long long e = threadIdx.x; e < np; e += 256) {
        const int j = (int)(e % nr), k = (int)(e / nr);
        double *pp = Pg + (long long)numr * (k + 1) + 1 + j;
        const double dv = (double)d[e];
        const double ph = *pp + dv;
        *pp = ph;
        sd += dv * dv;
        sp += ph * ph;
    }
    for (int off = 16; off > 0; off >>= 1) {
        sd += __shfl_down_sync(0xffffffffu, sd, off);
        sp += __shfl_down_sync(0xffffffffu, sp, off);
    }
    __shared__ double red[16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[2 * warp] = sd;
        red[2 * warp + 1] = sp;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[2 * w + threadIdx.x];
        const double wgt = (s == 0 || s == N / 2) ? 1.0 : 2.0;
        norms[2 * si + threadIdx.x] = wgt * t;
    }
}

template <typename T>
size_t radial_bytes(int kb, int us, int nr) {
    return sizeof(T) * ((size_t)kb * us + 3 * (size_t)nr);
}

template <typename T>
size_t vertical_bytes(int nz) {
    return sizeof(T) * ((size_t)nz * (panel_lines<T>() + 1) + 3 * (size_t)nz);
}

template <typename T>
Large<T> base_args(bph_ctx *c, const Schedule &sch) {
    Large<T> a = {};
    a.rad = sch.d_rad;
    a.ver = sch.d_ver;
    a.elz = c->d_elz;
    a.alphar = c->d_alphar;
    a.betar = c->d_betar;
    a.numr = c->g.numr;
    a.numz = c->g.numz;
    a.nr = c->nr;
    a.nz = c->nz;
    a.N = c->N;
    a.isym = c->g.isym;
    a.gamma = c->gamma;
    const int t = (sizeof(T) == 8) ? 0 : 1;
    a.kb = c->large_kb[t];
    a.ustride = c->nr | 1;
    return a;
}

// One half-sweep: radial or vertical panels over rows * N slots.
template <typename T>
cudaError_t panel_launch(bph_ctx *c, const Large<T> &a, bool radial, int rows, int step, double dt_next, bool last) {
    ++c->launches;
    if (radial) {
        const dim3 grid((unsigned)((c->nz + a.kb - 1) / a.kb), (unsigned)rows);
        k_large_radial<T, panel_lines<T>()><<<grid, kPanelThreads, radial_bytes<T>(a.kb, a.ustride, c->nr),
                                              c->stream>>>(
            a, step, (T)dt_next, last ? 1 : 0);
    } else {
        const dim3 grid((unsigned)((c->nr + panel_lines<T>() - 1) / panel_lines<T>()), (unsigned)rows);
        k_large_vertical<T, panel_lines<T>()><<<grid, kPanelThreads, vertical_bytes<T>(c->nz), c->stream>>>(a, step, (T)dt_next,
                                                                                         last ? 1 : 0);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t rhs0_launch(bph_ctx *c, const Large<T> &a, int rows, double dt, bool cold) {
    ++c->launches;
    k_large_rhs0<T><<<dim3((unsigned)((c->nr + 127) / 128), (unsigned)((c->nz + kRhs0Rows - 1) / kRhs0Rows),
                        (unsigned)rows),
                       128, 0, c->stream>>>(a, (T)dt, cold ? 1 : 0);
    return cudaGetLastError();
}

template <typename T>
int configure_type(bph_ctx *c, int dev_max) {
    dev_max -= 4096;  // the kernels' static scan arrays
    const int t = (sizeof(T) == 8) ? 0 : 1;
    const int us = c->nr | 1;
    int kb = panel_lines<T>();  // BPH_LARGE_ROWS=1..lines overrides (rows of a radial panel)
    if (const char *env = std::getenv("BPH_LARGE_ROWS")) {
        const int v = std::atoi(env);
        if (v >= 1 && v <= panel_lines<T>()) kb = v;
    }
    while (kb > 1 && radial_bytes<T>(kb, us, c->nr) > (size_t)dev_max) kb /= 2;
    if (radial_bytes<T>(kb, us, c->nr) > (size_t)dev_max || vertical_bytes<T>(c->nz) > (size_t)dev_max) {
        c->large_kb[t] = 0;
        return BPH_OK;
    }
    cudaError_t e = raise_smem_limit((const void *)k_large_radial<T, panel_lines<T>()>, (int)radial_bytes<T>(kb, us, c->nr));
    if (e == cudaSuccess) e = raise_smem_limit((const void *)k_large_vertical<T, panel_lines<T>()>, (int)vertical_bytes<T>(c->nz));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(grid-wide ADI panels)");
    c->large_kb[t] = kb;
    return BPH_OK;
}

}  // namespace

int large_configure(bph_ctx *c) {
    int dev_max = 0;
    cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    int rc = configure_type<double>(c, dev_max);
    if (!rc) rc = configure_type<float>(c, dev_max);
    return rc;
}

cudaError_t launch_adi_large(bph_ctx *c, const Schedule &sch, int step0, int nsteps_run, bool cold, double *P,
                             const double *R, int ninst, const int *d_inst_map, double *W, double *Q) {
    if (!c->large_kb[0]) return cudaErrorNotSupported;
    Large<double> a = base_args<double>(c, sch);
    a.phi = P;
    a.phi_slot = c->nplane;
    a.phi_off = c->g.numr + 1;
    a.phi_row = c->g.numr;
    a.src = R;
    a.W = W ? W : c->d_W;
    a.Q = Q ? Q : c->d_W2;
    a.P = P;
    a.inst_map = d_inst_map;
    if (ninst < 1 || (long long)ninst * c->N > 65535) return cudaErrorInvalidConfiguration;  // grid.y limit
    const int rows = ninst * c->N;
    if (nsteps_run < 1) return cudaSuccess;
    // step i: radial (dt_i), vertical (dt_i); each emits the next right-hand side
    cudaError_t e = rhs0_launch(c, a, rows, sch.h_dt[step0], cold);
    for (int it = 0; it < nsteps_run && e == cudaSuccess; ++it) {
        const int st = step0 + it;
        const bool last = (it == nsteps_run - 1);
        e = panel_launch(c, a, true, rows, st, sch.h_dt[st], false);
        if (e == cudaSuccess) e = panel_launch(c, a, false, rows, st, last ? 0.0 : sch.h_dt[st + 1], last);
    }
    return e;
}

cudaError_t launch_adi_defect_large_batch(bph_ctx *c, const Schedule &sch, double *P, const double *R, int npos,
                                         const int *d_map, float *work, double *norms) {
    if (!c->large_kb[1]) return cudaErrorNotSupported;
    if (npos < 1 || (long long)npos * c->N > 65535) return cudaErrorInvalidConfiguration;  // grid.y limit
    const long long np = c->np, span = (long long)npos * c->N * np;
    float *r = work, *delta = r + span, *W = delta + span, *Q = W + span;
    const int rows = npos * c->N;
    ++c->launches;
    k_large_defect_prologue<float><<<(unsigned)((span + 255) / 256), 256, 0, c->stream>>>(
        P, R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz, c->nr, c->nz, c->N,
        c->g.isym, npos, d_map, r, delta);
    cudaError_t e = cudaGetLastError();
    Large<float> a = base_args<float>(c, sch);  // work arrays by position: no map
    a.phi = delta;
    a.phi_slot = np;
    a.phi_off = 0;
    a.phi_row = c->nr;
    a.src = r;
    a.W = W;
    a.Q = Q;
    a.P = nullptr;  // zero frame
    // half-sweeps h = 0..2n: radial at step 0, then (vertical, radial) at
    // steps 0..n-1; each emits the next one's right-hand side at its dt
    const int nhalf = 2 * sch.nsteps + 1;
    auto step_of = [](int h) { return (h % 2 == 0) ? (h / 2 - 1 > 0 ? h / 2 - 1 : 0) : (h - 1) / 2; };
    if (e == cudaSuccess) e = rhs0_launch(c, a, rows, sch.h_dt[0], true);  // delta = 0
    for (int h = 0; h < nhalf && e == cudaSuccess; ++h) {
        const bool last = (h == nhalf - 1);
        const double dt_next = last ? 0.0 : sch.h_dt[step_of(h + 1)];
        e = panel_launch(c, a, (h % 2) == 0, rows, step_of(h), dt_next, last);
    }
    if (e == cudaSuccess) {
        ++c->launches;
        k_large_defect_epilogue<float><<<(unsigned)rows, 256, 0, c->stream>>>(P, delta, c->g.numr, c->g.numz, c->nr,
                                                                             c->nz, c->N, d_map, norms);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_adi_defect_large(bph_ctx *c, const Schedule &sch) {
    return launch_adi_defect_large_batch(c, sch, c->d_P, c->d_R, 1, nullptr, c->d_work32, c->d_red);
}

}  // namespace bph
