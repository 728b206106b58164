// bph_fft.cu -- azimuthal real FFTs (realft.F90 + the slot reorder of
// helmadi.F90:132-183 and its inverse :357-411).
//
// A CTA takes a tile of 16 consecutive (J,K) columns and all numphi samples
// of each: every row of the tile is a 128-byte coalesced segment of the
// Fortran array (J fastest).  The N real samples of a column are packed as
// M = N/2 complex values in shared memory, transformed by in-place Stockham
// radix-4 (and one radix-2) passes -- each pass loads its butterfly inputs
// to registers, synchronises, and stores -- and post-processed into the
// real spectrum.  Results are written slot-major, which is the layout the
// ADI kernel reads: the reference's swap_phi_r / swap_r_phi transposes are
// this store / load layout.
//
// Forward convention (realft isign=+1): F_k = sum_l f_l exp(+2 pi i k l / N).
#include <cmath>
#include <cstdlib>

#include "bph_internal.cuh"

namespace bph {
namespace {

// Columns per CTA: 8 (64-byte rows) for the 64- and 128-point transforms, so
// that a grid is several short waves instead of one long one with a tail;
// 16 (128-byte rows) otherwise.
template <int M>
constexpr int tile_cols() {
    return (M >= 64 && M <= 128) ? 8 : 16;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// One in-place Stockham pass of radix R (4 or 2) over all tile columns.
// C[n*kTile + c] holds element n of column c; tw[t] = e^{+2 pi i t / M}.
// SIGN = +1 forward (e^{+i}), -1 inverse.
template <int M, int R, int SIGN, int NT>
__device__ __forceinline__ void stockham_pass(double2 *C, const double2 *tw, int Ns) {
    constexpr int kTile = tile_cols<M>();
    constexpr int kTotal = kTile * (M / R);
    constexpr int kItems = (kTotal + NT - 1) / NT;  // butterflies per thread
    double2 v[kItems][R];
    const int tid = threadIdx.x;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        int it = tid + i * NT;
        if (kTotal % NT != 0 && it >= kTotal) break;
        int c = it % kTile, j = it / kTile;
        int k = j % Ns;
        int tstep = k * (M / (Ns * R));
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double2 x = C[(j + r * (M / R)) * kTile + c];
            if (r > 0) {
                double2 w = tw[r * tstep];
                x = (SIGN > 0) ? cmul(x, w) : cmulc(x, w);
            }
            v[i][r] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        int it = tid + i * NT;
        if (kTotal % NT != 0 && it >= kTotal) break;
        int c = it % kTile, j = it / kTile;
        int k = j % Ns;
        int base = (j / Ns) * Ns * R + k;
        if (R == 4) {
            double2 a0 = cadd(v[i][0], v[i][2]), a1 = csub(v[i][0], v[i][2]);
            double2 a2 = cadd(v[i][1], v[i][3]), d = csub(v[i][1], v[i][3]);
            double2 a3 = (SIGN > 0) ? make_double2(-d.y, d.x) : make_double2(d.y, -d.x);
            C[(base + 0 * Ns) * kTile + c] = cadd(a0, a2);
            C[(base + 1 * Ns) * kTile + c] = cadd(a1, a3);
            C[(base + 2 * Ns) * kTile + c] = csub(a0, a2);
            C[(base + 3 * Ns) * kTile + c] = csub(a1, a3);
        } else {
            C[(base + 0 * Ns) * kTile + c] = cadd(v[i][0], v[i][1]);
            C[(base + 1 * Ns) * kTile + c] = csub(v[i][0], v[i][1]);
        }
    }
    __syncthreads();
}

template <int M, int SIGN, int NT>
__device__ __forceinline__ void fft_tile(double2 *C, const double2 *tw) {
    int Ns = 1;
#pragma unroll
    for (int len = M; len >= 4; len /= 4) {
        stockham_pass<M, 4, SIGN, NT>(C, tw, Ns);
        Ns *= 4;
    }
    if ((M & 0x55555555) == 0) {  // log2(M) odd: one radix-2 pass remains
        stockham_pass<M, 2, SIGN, NT>(C, tw, Ns);
    }
}

// Batched launches: blockIdx.y is the batch position.  in / outp hold each
// position's caller array (forward: rho; inverse: pot), inst its instance
// (nullptr: position = instance); instance i's slot data sits at
// i * inst_stride from the given base, position j's moments at
// j * pos_stride, its non-finite flag at status[j].
struct FftBatch {
    const double *const *in = nullptr;
    double *const *outp = nullptr;
    const int *inst = nullptr;
    long long inst_stride = 0, pos_stride = 0;
    int status_stride = 0;  // 1: a flag per position, 0: one shared flag
};

// Threads and shared bytes of a tile (the same for both register budgets).
template <int M>
struct FftTile {
    static constexpr int kThreads = (M >= 256) ? 256 : 128;
    static constexpr size_t kSmem = sizeof(double2) * ((size_t)M * tile_cols<M>() + M + (M + 1));
};

// Resident CTAs per SM the register budget is sized for (the loads of a
// tile are all in flight at once; more CTAs hide more of their latency).
// Dense = 1: eight CTAs of 64 registers per SM for the 128-thread tiles (no
// spills), chosen by the set-up autotuner or with BPH_FFT_DENSE=1.
template <int M, int Dense = 0>
struct FftShape : FftTile<M> {
    static constexpr int kMinBlocksFwd = (M >= 256) ? 2 : (Dense ? 8 : 5);
    static constexpr int kMinBlocksInv = (M >= 256) ? 1 : (Dense ? 8 : 4);
};

// Forward transform of interior columns.  kRho: write R = -4 pi rho_hat
// (zero on the rows potential_solver.F90:66-78 zeroes) and the boundary
// moments of the unzeroed density (bessel.F90:179-185, 226-274) obtained
// from the same spectrum: sum_l rho_l e^{i k (l - 1/2) dphi} = e^{i pi k/N} F_k.
// !kRho: write the warm-start potential into P's interior.
template <int M, bool kRho, int Dense = 0>
__global__ void __launch_bounds__(FftTile<M>::kThreads, (FftShape<M, Dense>::kMinBlocksFwd))
k_fft_fwd(const double *__restrict__ src, double *__restrict__ out, double *__restrict__ mom,
          const double2 *__restrict__ g_tw, const double2 *__restrict__ g_tw2, const double2 *__restrict__ g_ph,
          int numr, int numz, int nr, int nz, int mmax, int fm, int isym, double four_pi,
          int *__restrict__ status, long long mstride, FftBatch bt) {
    constexpr int kTile = tile_cols<M>();
    constexpr int NT = FftTile<M>::kThreads;
    extern __shared__ double2 smem[];
    double2 *C = smem;
    double2 *tw = C + M * kTile;
    double2 *tw2 = tw + M;
    const int tid = threadIdx.x;
    const long long np = (long long)nr * nz;
    const long long nplane = (long long)numr * numz;
    const long long p0 = (long long)blockIdx.x * kTile;
    for (int i = tid; i < M; i += NT) tw[i] = g_tw[i];
    for (int i = tid; i <= M; i += NT) tw2[i] = g_tw2[i];
    pdl_wait();
    if (bt.in) {
        const int pos = blockIdx.y;
        src = bt.in[pos];
        out += (long long)(bt.inst ? bt.inst[pos] : pos) * bt.inst_stride;
        if (kRho) {
            mom += pos * bt.pos_stride;
            status += pos * bt.status_stride;
        }
    }
    // Load: thread -> (column c fixed, sample pairs n = n0, n0 + NT/kTile, ...);
    // all global loads are issued before any shared-memory store.
    static_assert(NT % kTile == 0, "threads must cover whole tile rows");
    constexpr int kRowsPerPass = NT / kTile, kLoads = M / kRowsPerPass;
    bool bad = false;
    {
        const int c = tid % kTile, n0 = tid / kTile;
        const long long p = p0 + c;
        const bool valid = p < np;
        const double *col = src;
        if (valid) col = src + ((int)p % nr + 1) + (long long)numr * ((int)p / nr + 1);
        double2 v[kLoads];
#pragma unroll
        for (int i = 0; i < kLoads; ++i) {
            const int n = n0 + i * kRowsPerPass;
            v[i] = valid ? make_double2(__ldg(col + nplane * (2 * n)), __ldg(col + nplane * (2 * n + 1)))
                         : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int i = 0; i < kLoads; ++i) {
            if (kRho) bad |= !(isfinite(v[i].x) && isfinite(v[i].y));
            C[(n0 + i * kRowsPerPass) * kTile + c] = v[i];
        }
    }
    if (kRho && bad) atomicOr(status, kStatusNonFinite);
    __syncthreads();
    fft_tile<M, +1, NT>(C, tw);
    pdl_trigger();
    // Post-process pairs (k, M-k) into F_k, F_{M-k}; write slots.  The tile
    // column of a thread is the same in every iteration (NT % kTile == 0).
    const int c = tid % kTile;
    const long long p = p0 + c;
    if (p >= np) return;
    const int pi = (int)p;
    const int jz = pi % nr + 1, kz = pi / nr + 1;
    const bool zeroed = (jz == numr - 2) || (kz == numz - 2) || (isym == 1 && kz == 1);
    for (int k = tid / kTile; k <= M / 2; k += NT / kTile) {
        double2 Fk, Fm;  // F_k and F_{M-k} (for k = 0: F_0 and F_M, both real)
        if (k == 0) {
            double2 z = C[c];
            Fk = make_double2(z.x + z.y, 0.0);
            Fm = make_double2(z.x - z.y, 0.0);
        } else if (2 * k == M) {
            Fk = C[k * kTile + c];
            Fm = Fk;
        } else {
            double2 zk = C[k * kTile + c], zm = C[(M - k) * kTile + c];
            double2 e = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
            double2 d = make_double2(zk.x - zm.x, zk.y + zm.y);
            double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
            Fk = cadd(e, cmul(tw2[k], o));
            double2 e2 = make_double2(e.x, -e.y);
            double2 d2 = make_double2(zm.x - zk.x, zm.y + zk.y);
            double2 o2 = make_double2(0.5 * d2.y, -0.5 * d2.x);
            Fm = cadd(e2, cmul(tw2[M - k], o2));
        }
        // Slot values: s = k -> Re F_k (F_0 at 0), s = M + k -> -Im F_k, s = M -> F_M.
        const int ka = k, kb = M - k;
        double sa_re = Fk.x, sa_im = -Fk.y, sb_re = Fm.x, sb_im = -Fm.y;
        if (kRho) {
            double *o = out + p;
            if (k == 0) {
                o[0] = zeroed ? 0.0 : -(four_pi * sa_re);
                o[np * M] = zeroed ? 0.0 : -(four_pi * sb_re);
            } else {
                o[np * ka] = zeroed ? 0.0 : -(four_pi * sa_re);
                o[np * (M + ka)] = zeroed ? 0.0 : -(four_pi * sa_im);
                if (kb != ka) {
                    o[np * kb] = zeroed ? 0.0 : -(four_pi * sb_re);
                    o[np * (M + kb)] = zeroed ? 0.0 : -(four_pi * sb_im);
                }
            }
            // Moments for boundary modes m with fm*m in {ka, kb}.
#pragma unroll 1
            for (int side = 0; side < 2; ++side) {
                int kk = side ? kb : ka;
                if (side && kb == ka) break;
                if (kk == M) continue;
                if (kk % fm) continue;
                int m = kk / fm;
                if (m >= mmax) continue;
                double2 F = side ? Fm : Fk;
                double tc, ts;
                if (m == 0) {
                    tc = F.x;
                    ts = 0.0;
                } else {
                    double2 ph = g_ph[m];
                    tc = ph.x * F.x - ph.y * F.y;
                    ts = ph.y * F.x + ph.x * F.y;
                }
                mom[m * mstride + p] = tc;
                mom[m * mstride + np + p] = ts;
            }
        } else {
            double *o = out + jz + (long long)numr * kz;
            if (k == 0) {
                o[0] = sa_re;
                o[nplane * M] = sb_re;
            } else {
                o[nplane * ka] = sa_re;
                o[nplane * (M + ka)] = sa_im;
                if (kb != ka) {
                    o[nplane * kb] = sb_re;
                    o[nplane * (M + kb)] = sb_im;
                }
            }
        }
    }
}

// Inverse transform of every (J,K) column of the slot array into the
// physical potential, 1/N normalised (the reference's 2/numphi times the
// n/2-scaled NR inverse), with the axis condition phi(1,K,l) =
// phi(2,K,l+N/2) (isym 3: phi(2,K,l)) and the equator condition
// phi(J,1,l) = phi(J,2,l) (isym 2,3) taken at the source: those columns
// transform the source column's spectrum (shifted by N/2 = sign (-1)^k).
// With phieff != nullptr the epilogue also writes the effective potential
// phieff = pot - 0.5 omega^2 rhf(J)^2 that the hydro source step forms from
// pot (source.F90:156, make_source_temp.F90:121), saving it a full pass.
template <int M, int Dense = 0>
__global__ void __launch_bounds__(FftTile<M>::kThreads, (FftShape<M, Dense>::kMinBlocksInv))
k_fft_inv(const double *__restrict__ P, double *__restrict__ pot, const double2 *__restrict__ g_tw,
          const double2 *__restrict__ g_tw2, int numr, int numz, int isym, double *__restrict__ phieff,
          const double *__restrict__ rhf, double omega, FftBatch bt) {
    constexpr int kTile = tile_cols<M>();
    constexpr int NT = FftTile<M>::kThreads;
    extern __shared__ double2 smem[];
    double2 *C = smem;
    double2 *tw = C + M * kTile;
    double2 *tw2 = tw + M;
    const int tid = threadIdx.x;
    const long long nplane = (long long)numr * numz;
    const long long q0 = (long long)blockIdx.x * kTile;
    for (int i = tid; i < M; i += NT) tw[i] = g_tw[i];
    for (int i = tid; i <= M; i += NT) tw2[i] = g_tw2[i];
    pdl_wait();
    if (bt.outp) {
        const int pos = blockIdx.y;
        P += (long long)(bt.inst ? bt.inst[pos] : pos) * bt.inst_stride;
        pot = bt.outp[pos];
    }
    // Load slots: thread -> (column c fixed, slot pairs (k, M+k)); all global
    // loads are issued before any shared-memory store.
    constexpr int kRowsPerPass = NT / kTile, kLoads = M / kRowsPerPass;
    {
        const int c = tid % kTile, k0 = tid / kTile;
        const long long q = q0 + c;
        const bool valid = q < nplane;
        int jz = 0, kz = 0;
        if (valid) {
            jz = (int)q % numr;
            kz = (int)q / numr;
        }
        const int js = (jz == 0) ? 1 : jz;
        const int ks = (kz == 0 && isym != 1) ? 1 : kz;
        const bool axis = valid && (jz == 0) && (isym != 3);
        const double *col = P + js + (long long)numr * ks;
        // two batches of loads in flight (register budget of kMinBlocksInv CTAs per SM)
        constexpr int kBatch = (kLoads >= 16) ? kLoads / 2 : kLoads;
#pragma unroll
        for (int i0 = 0; i0 < kLoads; i0 += kBatch) {
            double a[kBatch], b[kBatch];
#pragma unroll
            for (int i = 0; i < kBatch; ++i) {
                const int k = k0 + (i0 + i) * kRowsPerPass;
                a[i] = valid ? __ldg(col + nplane * k) : 0.0;
                b[i] = valid ? __ldg(col + nplane * (M + k)) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < kBatch; ++i) {
                const int k = k0 + (i0 + i) * kRowsPerPass;
                double2 v;
                if (k == 0) {
                    v = make_double2(a[i], b[i]);  // (F_0, F_M): both real
                } else {
                    v = make_double2(a[i], -b[i]);  // F_k = slot_k - i slot_{M+k}
                    if (axis && (k & 1)) v = make_double2(-v.x, -v.y);
                }
                C[k * kTile + c] = v;
            }
        }
    }
    __syncthreads();
    // Pre-process into Z_k = E_k + i O_k.
    for (int it = tid; it < kTile * (M / 2 + 1); it += NT) {
        int c = it % kTile, k = it / kTile;
        if (k == 0) {
            double2 f = C[c];
            C[c] = make_double2(0.5 * (f.x + f.y), 0.5 * (f.x - f.y));
        } else if (2 * k != M) {
            double2 fk = C[k * kTile + c], fm = C[(M - k) * kTile + c];
            double2 e = make_double2(0.5 * (fk.x + fm.x), 0.5 * (fk.y - fm.y));
            double2 d = make_double2(0.5 * (fk.x - fm.x), 0.5 * (fk.y + fm.y));
            double2 o = cmulc(d, tw2[k]);
            double2 e2 = make_double2(e.x, -e.y);
            double2 d2 = make_double2(0.5 * (fm.x - fk.x), 0.5 * (fm.y + fk.y));
            double2 o2 = cmulc(d2, tw2[M - k]);
            C[k * kTile + c] = make_double2(e.x - o.y, e.y + o.x);
            C[(M - k) * kTile + c] = make_double2(e2.x - o2.y, e2.y + o2.x);
        }
    }
    __syncthreads();
    fft_tile<M, -1, NT>(C, tw);
    pdl_trigger();
    const double scale = 1.0 / (double)M;
    {
        const int c = tid % kTile, n0 = tid / kTile;
        const long long q = q0 + c;
        if (q < nplane) {
            double *col = pot + q;
#pragma unroll
            for (int i = 0; i < kLoads; ++i) {
                const int n = n0 + i * kRowsPerPass;
                const double2 z = C[n * kTile + c];
                col[nplane * (2 * n)] = z.x * scale;
                col[nplane * (2 * n + 1)] = z.y * scale;
            }
            if (phieff) {
                const double r = rhf[(int)q % numr];
                const double cen = 0.5 * omega * omega * r * r;
                double *pe = phieff + q;
#pragma unroll
                for (int i = 0; i < kLoads; ++i) {
                    const int n = n0 + i * kRowsPerPass;
                    const double2 z = C[n * kTile + c];
                    pe[nplane * (2 * n)] = z.x * scale - cen;
                    pe[nplane * (2 * n + 1)] = z.y * scale - cen;
                }
            }
        }
    }
}

template <int M>
cudaError_t set_fft_attrs(bph_ctx *c) {
    size_t smem = FftTile<M>::kSmem;
    cudaError_t e = cudaFuncSetAttribute(k_fft_fwd<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_fwd<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_inv<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_fwd<M, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_inv<M, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    c->fft_smem_fwd = c->fft_smem_inv = (int)smem;
    return e;
}

template <int M>
cudaError_t fwd_rho(bph_ctx *c, const double *rho, double *R, double *mom, long long mstride, int *status,
                    FftBatch bt, int npos) {
    constexpr int kTile = tile_cols<M>();
    unsigned blocks = (unsigned)((c->np + kTile - 1) / kTile);
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg =
        launch_config(c, dim3(blocks, (unsigned)npos), dim3(FftTile<M>::kThreads), FftTile<M>::kSmem, attr);
    if (c->fft_dense)
        return cudaLaunchKernelEx(&cfg, k_fft_fwd<M, true, 1>, rho, R, mom, (const double2 *)c->d_tw,
                                  (const double2 *)c->d_tw2, (const double2 *)c->d_ph, c->g.numr, c->g.numz, c->nr,
                                  c->nz, c->g.mmax, c->fm, c->g.isym, c->four_pi, status, mstride, bt);
    return cudaLaunchKernelEx(&cfg, k_fft_fwd<M, true>, rho, R, mom, (const double2 *)c->d_tw,
                              (const double2 *)c->d_tw2, (const double2 *)c->d_ph, c->g.numr, c->g.numz, c->nr,
                              c->nz, c->g.mmax, c->fm, c->g.isym, c->four_pi, status, mstride, bt);
}

template <int M>
cudaError_t fwd_pot(bph_ctx *c, const double *pot) {
    constexpr int kTile = tile_cols<M>();
    unsigned blocks = (unsigned)((c->np + kTile - 1) / kTile);
    k_fft_fwd<M, false><<<blocks, FftTile<M>::kThreads, FftTile<M>::kSmem, c->stream>>>(
        pot, c->d_P, nullptr, c->d_tw, c->d_tw2, c->d_ph, c->g.numr, c->g.numz, c->nr, c->nz, c->g.mmax, c->fm,
        c->g.isym, c->four_pi, c->d_status, 0, FftBatch());
    return cudaGetLastError();
}

template <int M>
cudaError_t inv(bph_ctx *c, double *pot, double *phieff, double omega, const double *P, FftBatch bt, int npos) {
    constexpr int kTile = tile_cols<M>();
    unsigned blocks = (unsigned)((c->nplane + kTile - 1) / kTile);
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg =
        launch_config(c, dim3(blocks, (unsigned)npos), dim3(FftTile<M>::kThreads), FftTile<M>::kSmem, attr);
    if (c->fft_dense)
        return cudaLaunchKernelEx(&cfg, k_fft_inv<M, 1>, P, pot, (const double2 *)c->d_tw, (const double2 *)c->d_tw2,
                                  c->g.numr, c->g.numz, c->g.isym, phieff, (const double *)c->d_grid, omega, bt);
    return cudaLaunchKernelEx(&cfg, k_fft_inv<M>, P, pot, (const double2 *)c->d_tw, (const double2 *)c->d_tw2,
                              c->g.numr, c->g.numz, c->g.isym, phieff, (const double *)c->d_grid, omega, bt);
}

#define BPH_FFT_DISPATCH(FN, ...)                  \
    switch (c->M) {                                \
        case 8: return FN<8>(__VA_ARGS__);         \
        case 16: return FN<16>(__VA_ARGS__);       \
        case 32: return FN<32>(__VA_ARGS__);       \
        case 64: return FN<64>(__VA_ARGS__);       \
        case 128: return FN<128>(__VA_ARGS__);     \
        case 256: return FN<256>(__VA_ARGS__);     \
        default: return cudaErrorInvalidValue;     \
    }

cudaError_t set_attrs_dispatch(bph_ctx *c) { BPH_FFT_DISPATCH(set_fft_attrs, c) }
cudaError_t fwd_rho_dispatch(bph_ctx *c, const double *rho, double *R, double *mom, long long mstride, int *status,
                             FftBatch bt, int npos) {
    BPH_FFT_DISPATCH(fwd_rho, c, rho, R, mom, mstride, status, bt, npos)
}
cudaError_t fwd_pot_dispatch(bph_ctx *c, const double *pot) { BPH_FFT_DISPATCH(fwd_pot, c, pot) }
cudaError_t inv_dispatch(bph_ctx *c, double *pot, double *phieff, double omega, const double *P, FftBatch bt,
                         int npos) {
    BPH_FFT_DISPATCH(inv, c, pot, phieff, omega, P, bt, npos)
}

}  // namespace

int fft_configure(bph_ctx *c) {
    const char *dense = std::getenv("BPH_FFT_DENSE");
    c->fft_dense = dense && dense[0] == '1';
    cudaError_t e = set_attrs_dispatch(c);
    if (e != cudaSuccess) return cuda_fail(e, "fft_configure");
    return BPH_OK;
}

cudaError_t launch_fft_fwd_rho(bph_ctx *c, const double *rho, double *R, double *mom, long long mstride,
                               int *status) {
    ++c->launches;
    return fwd_rho_dispatch(c, rho, R ? R : c->d_R, mom ? mom : c->d_mom, mstride ? mstride : 2 * c->np,
                            status ? status : c->d_status, FftBatch(), 1);
}

cudaError_t launch_fft_fwd_pot(bph_ctx *c, const double *pot) {
    ++c->launches;
    return fwd_pot_dispatch(c, pot);
}

cudaError_t launch_fft_inv(bph_ctx *c, double *pot, double *phieff, double omega, const double *P) {
    ++c->launches;
    return inv_dispatch(c, pot, phieff, omega, P ? P : c->d_P, FftBatch(), 1);
}

cudaError_t launch_fft_fwd_rho_batch(bph_ctx *c, int npos, const double *const *d_in, const int *d_inst, double *R,
                                     long long inst_stride, double *mom, long long mstride, long long pos_stride,
                                     int *status, bool status_per_pos) {
    FftBatch bt;
    bt.in = d_in;
    bt.status_stride = status_per_pos ? 1 : 0;
    bt.inst = d_inst;
    bt.inst_stride = inst_stride;
    bt.pos_stride = pos_stride;
    ++c->launches;
    return fwd_rho_dispatch(c, nullptr, R, mom, mstride, status, bt, npos);
}

cudaError_t launch_fft_inv_batch(bph_ctx *c, int npos, double *const *d_out, const int *d_inst, const double *P,
                                 long long inst_stride) {
    FftBatch bt;
    bt.outp = d_out;
    bt.inst = d_inst;
    bt.inst_stride = inst_stride;
    ++c->launches;
    return inv_dispatch(c, nullptr, nullptr, 0.0, P, bt, npos);
}

}  // namespace bph
