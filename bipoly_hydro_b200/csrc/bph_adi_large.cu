// bph_adi_large.cu -- ADI for slots too large for shared memory.
//
// When a slot's slabs exceed an SM's shared memory (e.g. 258 x 194 x 512),
// each half-sweep is two grid-wide kernels over every slot at once instead
// of one CTA per slot:
//   k_large_rhs_r / k_large_rhs_z  the half-sweep's right-hand side, tile by
//       tile (32 x 32) through shared memory; reading one layout and writing
//       the other is where the data changes layout;
//   k_large_lines_r / k_large_lines_z  the line solves (tridagr / tridagz),
//       one thread per line over all slots.
// The potential stays in layout A ([k][j], j contiguous: the slot array);
// the radial half-sweep works in layout B ([j][k]) so that consecutive
// threads always read consecutive addresses: radial lines run along j with
// the threads on consecutive k, vertical lines along k with the threads on
// consecutive j.
//
// The same kernels, in FP32 and with a zero Dirichlet frame, run the
// mixed-precision refinement cycle on the defect equation (prologue: the
// FP64 residual; body: radial at the first step's dt, then vertical and
// radial per step; epilogue: phi += delta in FP64 and the per-slot norms).
#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kT = 32;              // tile edge
constexpr int kTileThreads = 256;
constexpr int kLineThreads = 128;

template <typename T>
struct Large {
    T *phi;                 // layout A: element (k, j) of slot s at phi + s*phi_slot + phi_off + k*phi_row + j
    long long phi_slot, phi_off;
    int phi_row;
    const T *src;           // -4 pi rho_hat (drop-in) or the defect r, packed [N][nz][nr]
    T *W, *Q;               // right-hand sides and the radial result, [N][np]
    const double *P;        // slot array for the Dirichlet frame; nullptr: zero frame
    const double *rad, *ver;
    const double *elz, *alphar, *betar;
    const int *inst_map;    // batches: instance of each row of N slots (nullptr: row = instance)
    int numr, numz, nr, nz, N, isym;
    double gamma, dt;
    int step, cold;
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

template <typename T>
__device__ __forceinline__ T phi_at(const Large<T> &a, long long s, int k, int j) {
    return a.phi[s * a.phi_slot + a.phi_off + (long long)k * a.phi_row + j];
}

// radial right-hand side (helmadi.F90:203-256): A -> B
template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_large_rhs_r(Large<T> a) {
    __shared__ T tile[kT][kT + 1];
    const Where wh = where(a);
    const long long s = wh.sg;
    const int tj = (a.nr + kT - 1) / kT;
    const int k0 = (blockIdx.x / tj) * kT, j0 = (blockIdx.x % tj) * kT;
    const long long np = (long long)a.nr * a.nz, nplane = (long long)a.numr * a.numz;
    const double *Pg = a.P ? a.P + s * nplane : nullptr;
    const bool sym_bottom = (a.isym != 1);
    const T dt = (T)a.dt, g = (T)a.gamma;
    for (int e = threadIdx.x; e < kT * kT; e += kTileThreads) {
        const int kl = e / kT, jl = e % kT, k = k0 + kl, j = j0 + jl;
        if (k >= a.nz || j >= a.nr) continue;
        const T phi = a.cold ? (T)0 : phi_at(a, s, k, j);
        T up, dn;
        if (k + 1 < a.nz) up = a.cold ? (T)0 : phi_at(a, s, k + 1, j);
        else up = Pg ? (T)Pg[(j + 1) + (long long)a.numr * (a.numz - 1)] : (T)0;
        if (k > 0) dn = a.cold ? (T)0 : phi_at(a, s, k - 1, j);
        else dn = (Pg && !sym_bottom) ? (T)Pg[j + 1] : (T)0;
        const T r = a.src[s * np + (long long)k * a.nr + j];
        T v = (k == 0 && sym_bottom) ? r + (dt - g) * phi + g * up : r + (dt - (T)2 * g) * phi + g * (up + dn);
        if (j == a.nr - 1 && Pg)
            v = v - (T)a.alphar[a.numr - 2] * (T)Pg[(a.numr - 1) + (long long)a.numr * (k + 1)];
        tile[kl][jl] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kT * kT; e += kTileThreads) {
        const int jl = e / kT, kl = e % kT, k = k0 + kl, j = j0 + jl;
        if (k < a.nz && j < a.nr) a.W[wh.sw * np + (long long)j * a.nz + k] = tile[kl][jl];
    }
}

// radial lines: thread (slot, k), W (layout B) -> Q (layout B)
template <typename T>
__global__ void __launch_bounds__(kLineThreads) k_large_lines_r(Large<T> a) {
    const Where wh = where(a);
    const int k = blockIdx.x * kLineThreads + threadIdx.x;
    if (k >= a.nz) return;
    const int nr = a.nr, nz = a.nz;
    const long long np = (long long)nr * nz;
    const double *f = a.rad + ((long long)a.step * a.N + wh.sl) * kAdiFactors * nr;
    const double *ib = f, *dd = f + nr, *gm = f + 2 * nr;
    T *w = a.W + wh.sw * np + k, *q = a.Q + wh.sw * np + k;
    T y = w[0] * (T)ib[0];
    w[0] = y;
#pragma unroll 4
    for (int j = 1; j < nr; ++j) {
        y = w[(long long)j * nz] * (T)ib[j] - (T)dd[j] * y;
        w[(long long)j * nz] = y;
    }
    T x = y;
    q[(long long)(nr - 1) * nz] = x;
#pragma unroll 4
    for (int j = nr - 2; j >= 0; --j) {
        x = w[(long long)j * nz] - (T)gm[j + 1] * x;
        q[(long long)j * nz] = x;
    }
}

// vertical right-hand side (helmadi.F90:272-340): B -> A
template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_large_rhs_z(Large<T> a) {
    __shared__ T tile[kT][kT + 1];
    const Where wh = where(a);
    const long long s = wh.sg;
    const int tj = (a.nr + kT - 1) / kT;
    const int k0 = (blockIdx.x / tj) * kT, j0 = (blockIdx.x % tj) * kT;
    const long long np = (long long)a.nr * a.nz, nplane = (long long)a.numr * a.numz;
    const double *Pg = a.P ? a.P + s * nplane : nullptr;
    const bool sym_bottom = (a.isym != 1);
    const T dt = (T)a.dt, g = (T)a.gamma;
    const T *Q = a.Q + wh.sw * np;
    for (int e = threadIdx.x; e < kT * kT; e += kTileThreads) {
        const int jl = e / kT, kl = e % kT, k = k0 + kl, j = j0 + jl;
        if (k >= a.nz || j >= a.nr) continue;
        const T *qc = Q + (long long)j * a.nz + k;
        T right;
        if (j + 1 < a.nr) right = qc[a.nz];
        else right = Pg ? (T)Pg[(a.numr - 1) + (long long)a.numr * (k + 1)] : (T)0;
        T v = ((T)a.elz[(long long)wh.sl * a.numr + j + 1] + dt) * qc[0] - (T)a.alphar[j + 1] * right;
        if (j > 0) v = v - (T)a.betar[j + 1] * qc[-a.nz];
        tile[jl][kl] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kT * kT; e += kTileThreads) {
        const int kl = e / kT, jl = e % kT, k = k0 + kl, j = j0 + jl;
        if (k >= a.nz || j >= a.nr) continue;
        T v = a.src[s * np + (long long)k * a.nr + j] + tile[jl][kl];
        if (Pg && k == a.nz - 1) v = v + g * (T)Pg[(j + 1) + (long long)a.numr * (a.numz - 1)];
        if (Pg && !sym_bottom && k == 0) v = v + g * (T)Pg[j + 1];
        a.W[wh.sw * np + (long long)k * a.nr + j] = v;
    }
}

// vertical lines: thread (slot, j), W (layout A) -> phi (layout A)
template <typename T>
__global__ void __launch_bounds__(kLineThreads) k_large_lines_z(Large<T> a) {
    const Where wh = where(a);
    const int j = blockIdx.x * kLineThreads + threadIdx.x;
    if (j >= a.nr) return;
    const int nr = a.nr, nz = a.nz;
    const long long np = (long long)nr * nz;
    const double *f = a.ver + (long long)a.step * kAdiFactors * nz;
    const double *ib = f, *dd = f + nz, *gm = f + 2 * nz;
    T *w = a.W + wh.sw * np + j;
    T *p = a.phi + wh.sg * a.phi_slot + a.phi_off + j;
    T y = w[0] * (T)ib[0];
    w[0] = y;
#pragma unroll 4
    for (int k = 1; k < nz; ++k) {
        y = w[(long long)k * nr] * (T)ib[k] - (T)dd[k] * y;
        w[(long long)k * nr] = y;
    }
    T x = y;
    p[(long long)(nz - 1) * a.phi_row] = x;
#pragma unroll 4
    for (int k = nz - 2; k >= 0; --k) {
        x = w[(long long)k * nr] - (T)gm[k + 1] * x;
        p[(long long)k * a.phi_row] = x;
    }
}

// Layout B -> A copy of the radial result (the refinement cycle ends on a
// radial half-sweep, whose result is in Q).
template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_large_b_to_a(Large<T> a) {
    __shared__ T tile[kT][kT + 1];
    const Where wh = where(a);
    const long long s = wh.sg;
    const int tj = (a.nr + kT - 1) / kT;
    const int k0 = (blockIdx.x / tj) * kT, j0 = (blockIdx.x % tj) * kT;
    const long long np = (long long)a.nr * a.nz;
    for (int e = threadIdx.x; e < kT * kT; e += kTileThreads) {
        const int jl = e / kT, kl = e % kT, k = k0 + kl, j = j0 + jl;
        if (k < a.nz && j < a.nr) tile[jl][kl] = a.Q[wh.sw * np + (long long)j * a.nz + k];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kT * kT; e += kTileThreads) {
        const int kl = e / kT, jl = e % kT, k = k0 + kl, j = j0 + jl;
        if (k < a.nz && j < a.nr) a.phi[s * a.phi_slot + a.phi_off + (long long)k * a.phi_row + j] = tile[jl][kl];
    }
}

// FP64 residual r = -4 pi rho_hat - A phi of the current potential (its
// Dirichlet columns through the stencil), stored in T; delta = 0.
template <typename T>
__global__ void k_large_defect_prologue(const double *__restrict__ P, const double *__restrict__ R,
                                        const double *__restrict__ brb, const double *__restrict__ alphar,
                                        const double *__restrict__ betar, const double *__restrict__ bzb,
                                        double gamma, int numr, int numz, int nr, int nz, int N, int isym,
                                        T *__restrict__ r, T *__restrict__ delta) {
    const long long np = (long long)nr * nz, nplane = (long long)numr * numz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np * N) return;
    const int s = (int)(t / np);
    const long long e = t - s * np;
    const int j = (int)(e % nr), k = (int)(e / nr);
    const bool sym_bottom = (isym != 1);
    const double *pc = P + s * nplane + (long long)numr * (k + 1) + 1;
    const double c = pc[j], east = pc[j + 1], n = pc[j + numr];
    const double w = (j > 0) ? pc[j - 1] : 0.0;
    const double so = (k > 0 || !sym_bottom) ? pc[j - numr] : 0.0;
    const double *b = brb + (long long)s * numr;
    const double ar = b[j + 1] * c + alphar[j + 1] * east + betar[j + 1] * w;
    const double az = bzb[k + 1] * c - gamma * n - gamma * so;
    r[t] = (T)(R[t] - ar - az);
    delta[t] = (T)0;
}

// phi += delta in FP64 and the per-slot |delta|^2, |phi|^2 (one CTA per slot)
template <typename T>
__global__ void __launch_bounds__(256) k_large_defect_epilogue(double *__restrict__ P, const T *__restrict__ delta,
                                                               int numr, int numz, int nr, int nz, int N,
                                                               double *__restrict__ norms) {
    const int s = blockIdx.x;
    const long long np = (long long)nr * nz, nplane = (long long)numr * numz;
    double *Pg = P + s * nplane;
    const T *d = delta + s * np;
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
        norms[2 * s + threadIdx.x] = wgt * t;
    }
}

template <typename T>
cudaError_t half_step(bph_ctx *c, Large<T> a, bool radial, int ninst) {
    const int tiles = ((c->nr + kT - 1) / kT) * ((c->nz + kT - 1) / kT);
    const unsigned rows = (unsigned)(c->N * ninst);
    c->launches += 2;
    if (radial) {
        k_large_rhs_r<T><<<dim3((unsigned)tiles, rows), kTileThreads, 0, c->stream>>>(a);
        k_large_lines_r<T><<<dim3((unsigned)((c->nz + kLineThreads - 1) / kLineThreads), rows), kLineThreads, 0,
                             c->stream>>>(a);
    } else {
        k_large_rhs_z<T><<<dim3((unsigned)tiles, rows), kTileThreads, 0, c->stream>>>(a);
        k_large_lines_z<T><<<dim3((unsigned)((c->nr + kLineThreads - 1) / kLineThreads), rows), kLineThreads, 0,
                             c->stream>>>(a);
    }
    return cudaGetLastError();
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
    return a;
}

}  // namespace

cudaError_t launch_adi_large(bph_ctx *c, const Schedule &sch, int step0, int nsteps_run, bool cold, double *P,
                             const double *R, int ninst, const int *d_inst_map, double *W, double *Q) {
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
    cudaError_t e = cudaSuccess;
    for (int it = 0; it < nsteps_run && e == cudaSuccess; ++it) {
        a.step = step0 + it;
        a.dt = sch.h_dt[a.step];
        a.cold = (cold && it == 0) ? 1 : 0;
        e = half_step(c, a, true, ninst);
        a.cold = 0;
        if (e == cudaSuccess) e = half_step(c, a, false, ninst);
    }
    return e;
}

cudaError_t launch_adi_defect_large(bph_ctx *c, const Schedule &sch) {
    const long long np = c->np;
    float *r = c->d_work32, *delta = r + (long long)c->N * np, *W = delta + (long long)c->N * np,
          *Q = W + (long long)c->N * np;
    const long long total = np * c->N;
    ++c->launches;
    k_large_defect_prologue<float><<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(
        c->d_P, c->d_R, c->d_brb, c->d_alphar, c->d_betar, c->d_bzb, c->gamma, c->g.numr, c->g.numz, c->nr, c->nz,
        c->N, c->g.isym, r, delta);
    cudaError_t e = cudaGetLastError();
    Large<float> a = base_args<float>(c, sch);
    a.phi = delta;
    a.phi_slot = np;
    a.phi_off = 0;
    a.phi_row = c->nr;
    a.src = r;
    a.W = W;
    a.Q = Q;
    a.P = nullptr;  // zero frame
    // radial at the first step's dt, then (vertical, radial) per step
    const int nhalf = 2 * sch.nsteps + 1;
    for (int h = 0; h < nhalf && e == cudaSuccess; ++h) {
        const bool radial = (h % 2) == 0;
        const int it = radial ? (h / 2 - 1 > 0 ? h / 2 - 1 : 0) : (h - 1) / 2;
        a.step = it;
        a.dt = sch.h_dt[it];
        e = half_step(c, a, radial, 1);
    }
    if (e == cudaSuccess) {
        const int tiles = ((c->nr + kT - 1) / kT) * ((c->nz + kT - 1) / kT);
        ++c->launches;
        k_large_b_to_a<float><<<dim3((unsigned)tiles, (unsigned)c->N), kTileThreads, 0, c->stream>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        ++c->launches;
        k_large_defect_epilogue<float><<<c->N, 256, 0, c->stream>>>(c->d_P, delta, c->g.numr, c->g.numz, c->nr, c->nz,
                                                                    c->N, c->d_red);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace bph
