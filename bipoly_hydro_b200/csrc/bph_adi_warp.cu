// bph_adi_warp.cu -- warp-cooperative FP64 ADI of one Fourier slot per CTA
// (helmadi.F90:195-355 with tridagr.F90 and tridagz.F90), the drop-in's
// fast path on the grids whose interior is 32*NLZ x 32*NLR zones
// (128 x 96 for 130x98, 64 x 64 for 66x66).
//
// Work split.  256 threads = 8 warps x 4 groups of 8 lanes.  Group
// p = 4*warp + group (0..31) owns a set of lines; lane g of a group owns
// segment g (one eighth) of each of them:
//   radial half-step   lines k = NLR*p + l (l < NLR), lane g: j in [LR g, LR g + LR)
//   vertical half-step lines j = NLZ*p + l (l < NLZ), lane g: k in [LZ g, LZ g + LZ)
// with LR = 4 NLZ and LZ = 4 NLR, so a lane holds NLR*LR = NLZ*LZ values
// (48 at 130x98) of the slot in registers in either orientation.
//
// One half-step:
//   load   the lane's segments of the right-hand side W (premultiplied by
//          the sweep's 1/bet) from shared memory into registers;
//   A      forward elimination with zero carry-in, y = w - (a/bet) y_prev;
//   scan   the carry into each segment, y_in(g) = y_end(g-1), by a
//          Kogge-Stone scan of the affine maps y_end(g) = L(g) + G(g) y_end(g-1)
//          over the 8 lanes of the group (3 shuffle steps, the products of
//          the segment carries precomputed per schedule);
//   B      fix-up and backward substitution with zero carry-in;
//   scan   the carry out of each segment, x_in(g) = x_start(g+1) (3 steps);
//   C      x = M + K x_in: the line's solution, in registers;
//   D      after a barrier (every lane has read W): the other direction's
//          right-hand side of the next half-step, from the registers and
//          the neighbouring segments' edge values (one shuffle each), times
//          that sweep's 1/bet, stored to W; a second barrier.
// The per-element arithmetic is the Thomas algorithm of tridagr/tridagz;
// the segment carries only re-associate it (results agree to rounding).
//
// Shared memory (doubles): W and R (= -4 pi rho_hat with every Dirichlet
// term folded in, as the reference's sweeps add them: helmadi.F90:252-256,
// 327-340), each NZ x NR with an XOR swizzle of the 16-byte chunks,
//   chunk' = chunk ^ ((j / LR) ^ (k / LZ)) & 7,
// so that the 8 lanes of a group hit 8 different bank groups both when
// they read 16-byte pairs along a row (radial) and along a column pair
// (vertical); then two radial and two vertical factor blocks (the current
// and the next step, filled by cp.async one step ahead) and the slot's
// (elambdazb, alphaz, betaz) coefficients.  Factor arrays are stored
// segment-interleaved ([i][g]) so the 8 lanes of a group read 8
// consecutive values.
#include <cstdint>

#include "bph_internal.cuh"

namespace bph {

namespace {

constexpr int kWThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

template <int NLR, int NLZ>
struct WS {
    static constexpr int LR = 4 * NLZ;  // radial segment length
    static constexpr int LZ = 4 * NLR;  // vertical segment length
    static constexpr int NR = 8 * LR;   // interior zones along r (= 32 NLZ)
    static constexpr int NZ = 8 * LZ;   // interior zones along z (= 32 NLR)
    // factor block of one line system, segment length L (doubles):
    //   dd pairs [L/2][8][2], (G, gam_next) [L][8][2], K pairs [L/2][8][2],
    //   scan products [6][8] (P1 P2 P4 Q1 Q2 Q4), 1/bet [8 L] in line order
    static constexpr int block(int L) { return 40 * L + 48; }
    static constexpr int RAD = block(LR), VER = block(LZ);
    static constexpr int COEF = 24 * LR;  // elambdazb pairs [LR/2][8][2], (alphaz, betaz) [LR][8][2]
    static constexpr int O_R = NZ * NR;
    static constexpr int O_RAD = 2 * NZ * NR;
    static constexpr int O_VER = O_RAD + 2 * RAD;
    static constexpr int O_COEF = O_VER + 2 * VER;
    static constexpr int TOTAL = O_COEF + COEF;
    static_assert(RAD % 2 == 0 && VER % 2 == 0 && COEF % 2 == 0, "blocks must be whole 16-byte chunks");
    static_assert(NLZ % 2 == 0, "vertical lines are read in column pairs");
};

// Offsets inside a factor block of segment length L.
__host__ __device__ constexpr int fo_dd(int) { return 0; }
__host__ __device__ constexpr int fo_gg(int L) { return 8 * L; }
__host__ __device__ constexpr int fo_k(int L) { return 24 * L; }
__host__ __device__ constexpr int fo_scan(int L) { return 32 * L; }
__host__ __device__ constexpr int fo_ib(int L) { return 32 * L + 48; }

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// n elements of T (a whole number of 16-byte chunks), 16-byte aligned at
// both ends, copied by the whole CTA.
template <typename T>
__device__ __forceinline__ void copy_block(T *dst, const T *src, int n, int tid) {
    constexpr int E = 16 / (int)sizeof(T);
    for (int c = tid; c < n / E; c += kWThreads) cp16(dst + E * c, src + E * c);
}

template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};
// Two consecutive elements (8- or 16-byte aligned).
template <typename T>
__device__ __forceinline__ typename Pair<T>::type ldp(const T *p) {
    return *reinterpret_cast<const typename Pair<T>::type *>(p);
}

__device__ __forceinline__ double2 lds2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void sts2(double *p, double a, double b) {
    *reinterpret_cast<double2 *>(p) = make_double2(a, b);
}

// Element (k, j) of a swizzled slab, in doubles.
template <int NLR, int NLZ>
__device__ __forceinline__ int swz(int k, int j) {
    using S = WS<NLR, NLZ>;
    const int c = j >> 1;
    const int x = ((j / S::LR) ^ (k / S::LZ)) & 7;
    return k * S::NR + 2 * (c ^ x) + (j & 1);
}

// Forward carry scan over the 8 lanes of a group: in a = L_end(g), out the
// carry into segment g, y_end(g-1) (0 for g = 0).
template <typename T, int NL>
__device__ __forceinline__ void scan_forward(T (&a)[NL], const T *scan, int g) {
    const T p1 = scan[g], p2 = scan[8 + g], p4 = scan[16 + g];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        T t = __shfl_up_sync(kFull, a[l], 1, 8);
        if (g >= 1) a[l] = fma(p1, t, a[l]);
        t = __shfl_up_sync(kFull, a[l], 2, 8);
        if (g >= 2) a[l] = fma(p2, t, a[l]);
        t = __shfl_up_sync(kFull, a[l], 4, 8);
        if (g >= 4) a[l] = fma(p4, t, a[l]);
        t = __shfl_up_sync(kFull, a[l], 1, 8);
        a[l] = (g >= 1) ? t : (T)0;
    }
}

// Backward carry scan: in b = M_start(g), out the carry into segment g from
// above, x_start(g+1) (0 for g = 7).
template <typename T, int NL>
__device__ __forceinline__ void scan_backward(T (&b)[NL], const T *scan, int g) {
    const T q1 = scan[24 + g], q2 = scan[32 + g], q4 = scan[40 + g];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        T t = __shfl_down_sync(kFull, b[l], 1, 8);
        if (g <= 6) b[l] = fma(q1, t, b[l]);
        t = __shfl_down_sync(kFull, b[l], 2, 8);
        if (g <= 5) b[l] = fma(q2, t, b[l]);
        t = __shfl_down_sync(kFull, b[l], 4, 8);
        if (g <= 3) b[l] = fma(q4, t, b[l]);
        t = __shfl_down_sync(kFull, b[l], 1, 8);
        b[l] = (g <= 6) ? t : (T)0;
    }
}

// Phases A, scan, B, scan, C of NL lines of segment length L held in v,
// with the factor block f (segment-interleaved layout).
template <typename T, int NL, int L>
__device__ __forceinline__ void solve_lines(T (&v)[NL][L], const T *f, int g) {
    T c[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) c[l] = (T)0;
    // A: forward elimination, zero carry-in
#pragma unroll
    for (int t = 0; t < L / 2; ++t) {
        const auto dd = ldp(f + fo_dd(L) + (t * 8 + g) * 2);
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            c[l] = v[l][2 * t] - dd.x * c[l];
            v[l][2 * t] = c[l];
            c[l] = v[l][2 * t + 1] - dd.y * c[l];
            v[l][2 * t + 1] = c[l];
        }
    }
    scan_forward<T, NL>(c, f + fo_scan(L), g);
    // B: y = L + G y_in, backward substitution with zero carry-in
    T m[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) m[l] = (T)0;
#pragma unroll
    for (int i = L - 1; i >= 0; --i) {
        const auto gg = ldp(f + fo_gg(L) + (i * 8 + g) * 2);
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            m[l] = (v[l][i] + gg.x * c[l]) - gg.y * m[l];
            v[l][i] = m[l];
        }
    }
    scan_backward<T, NL>(m, f + fo_scan(L), g);
    // C: x = M + K x_in
#pragma unroll
    for (int t = 0; t < L / 2; ++t) {
        const auto kk = ldp(f + fo_k(L) + (t * 8 + g) * 2);
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            v[l][2 * t] = v[l][2 * t] + kk.x * m[l];
            v[l][2 * t + 1] = v[l][2 * t + 1] + kk.y * m[l];
        }
    }
}

struct WarpArgs {
    double *P;            // slot arrays [inst][N][numr*numz]
    const double *R;      // [inst][N][nr*nz]
    const double *rad;    // radial blocks [nsteps][N][RAD]
    const double *ver;    // vertical blocks [nsteps][VER]
    const double *coef;   // [N][COEF]
    const double *dt;     // [nsteps]
    const double *alphar; // [numr]
    double *norms;        // converged cycles: per (instance, slot) |new - old|^2, |new|^2 (nullptr: none)
    const int *inst_map;  // instance of each block row (nullptr: row)
    const int *slot_map;  // slot of each block in its row (nullptr: block)
    int nslots, N, numr, numz, isym;
    int step0, nsteps, cold;
    double gamma;
};

template <int NLR, int NLZ>
__global__ void __launch_bounds__(kWThreads, 1) k_adi_warp(WarpArgs a) {
    using S = WS<NLR, NLZ>;
    constexpr int LR = S::LR, LZ = S::LZ, NR = S::NR, NZ = S::NZ;
    extern __shared__ __align__(16) double smd[];
    double *W = smd;
    double *Rsh = smd + S::O_R;
    double *radb = smd + S::O_RAD;
    double *verb = smd + S::O_VER;
    const double *coefb = smd + S::O_COEF;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane & 7;
    const int p = 4 * w + (lane >> 3);  // line set
    const int x = (g ^ w) & 7;          // this lane's swizzle term (both orientations)
    const int local = blockIdx.x % a.nslots, row = blockIdx.x / a.nslots;
    const int s = a.slot_map ? a.slot_map[local] : local;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int numr = a.numr, numz = a.numz;
    double *Pg = a.P + blk * (long long)numr * numz;
    const double *Rg = a.R + blk * (long long)NR * NZ;
    const size_t rad_step = (size_t)a.N * S::RAD;
    const double *rad_src = a.rad + (size_t)s * S::RAD;
    const double gamma = a.gamma;
    const bool sym_bottom = (a.isym != 1);
    const int n = a.nsteps;

    // set-up data first (no dependence on the previous kernel of the stream)
    copy_block(radb, rad_src + (size_t)a.step0 * rad_step, S::RAD, tid);
    copy_block(verb, a.ver + (size_t)a.step0 * S::VER, S::VER, tid);
    copy_block(const_cast<double *>(coefb), a.coef + (size_t)s * S::COEF, S::COEF, tid);
    cp_commit();
    const double a_side = a.alphar[numr - 2];  // alphar(numr-1)
    pdl_wait();

    // R -> shared, 16-byte chunks straight into their swizzled places, and
    // (warm start) the initial potential's interior into W, element by
    // element: every copy of the prologue is in flight at once.
    constexpr int kTot = NR * NZ;
    for (int q = tid; q < kTot / 2; q += kWThreads) {
        const int e = 2 * q;
        cp16(Rsh + swz<NLR, NLZ>(e / NR, e % NR), Rg + e);
    }
    if (!a.cold) {
        for (int e = tid; e < kTot; e += kWThreads) {
            const int k = e / NR, j = e % NR;
            cp8(W + swz<NLR, NLZ>(k, j), Pg + (j + 1) + (long long)numr * (k + 1));
        }
    }
    cp_commit();
    // Dirichlet terms (helmadi.F90:252-256, 327-340): thread t folds the top
    // (and, isym 1, bottom) zone of column t, and the side zone of row t;
    // the corners take the top/bottom term first, then the side term.
    double top_v = 0.0, bot_v = 0.0, side_top = 0.0, side_bot = 0.0, side_v = 0.0;
    if (tid < NR) {
        top_v = Pg[(tid + 1) + (long long)numr * (numz - 1)];
        if (!sym_bottom) bot_v = Pg[tid + 1];
        if (tid == NR - 1) {
            side_top = Pg[(numr - 1) + (long long)numr * NZ];
            side_bot = Pg[(numr - 1) + (long long)numr];
        }
    }
    const bool side_row = tid < NZ && tid != NZ - 1 && !(tid == 0 && !sym_bottom);
    if (side_row) side_v = Pg[(numr - 1) + (long long)numr * (tid + 1)];
    cp_wait_all();
    __syncthreads();
    if (tid < NR) {
        double *t = Rsh + swz<NLR, NLZ>(NZ - 1, tid);
        double v = *t + gamma * top_v;
        if (tid == NR - 1) v = v - a_side * side_top;
        *t = v;
        if (!sym_bottom) {
            double *b = Rsh + swz<NLR, NLZ>(0, tid);
            double u = *b + gamma * bot_v;
            if (tid == NR - 1) u = u - a_side * side_bot;
            *b = u;
        }
    }
    if (side_row) {
        double *sd = Rsh + swz<NLR, NLZ>(tid, NR - 1);
        *sd = *sd - a_side * side_v;
    }
    __syncthreads();

    // Radial right-hand side of step `st` from a potential held in vertical
    // orientation (rows k = LZ g + i, columns j = NLZ p + l), times that
    // step's radial 1/bet (helmadi.F90:209-256), stored to W.
    auto store_radial_rhs = [&](double (&v)[NLZ][LZ], const double *ibr, double dtn) {
        double dn_e[NLZ], up_e[NLZ], ib[NLZ];
#pragma unroll
        for (int l = 0; l < NLZ; ++l) {
            dn_e[l] = __shfl_up_sync(kFull, v[l][LZ - 1], 1, 8);
            up_e[l] = __shfl_down_sync(kFull, v[l][0], 1, 8);
            if (g == 0) dn_e[l] = 0.0;
            if (g == 7) up_e[l] = 0.0;
        }
#pragma unroll
        for (int m = 0; m < NLZ / 2; ++m) {
            const double2 t = lds2(ibr + NLZ * p + 2 * m);
            ib[2 * m] = t.x;
            ib[2 * m + 1] = t.y;
        }
        const double c2 = dtn - 2.0 * gamma, c1 = dtn - gamma;
#pragma unroll
        for (int i = 0; i < LZ; ++i) {
            const int k = LZ * g + i;
            const bool refl = (k == 0) && sym_bottom;
#pragma unroll
            for (int m = 0; m < NLZ / 2; ++m) {
                const int off = k * NR + 2 * (((NLZ / 2) * p + m) ^ x);
                const double2 r = lds2(Rsh + off);
                double o[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int l = 2 * m + e;
                    const double up = (i + 1 < LZ) ? v[l][i + 1] : up_e[l];
                    const double dn = (i > 0) ? v[l][i - 1] : dn_e[l];
                    const double rr = e ? r.y : r.x;
                    const double rhs = refl ? rr + c1 * v[l][i] + gamma * up : rr + c2 * v[l][i] + gamma * (up + dn);
                    o[e] = rhs * ib[l];
                }
                sts2(W + off, o[0], o[1]);
            }
        }
    };

    // first radial right-hand side, from the initial potential (in W)
    {
        double v[NLZ][LZ];
#pragma unroll
        for (int i = 0; i < LZ; ++i) {
            const int k = LZ * g + i;
#pragma unroll
            for (int m = 0; m < NLZ / 2; ++m) {
                const double2 q = a.cold ? make_double2(0.0, 0.0)
                                         : lds2(W + k * NR + 2 * (((NLZ / 2) * p + m) ^ x));
                v[2 * m][i] = q.x;
                v[2 * m + 1][i] = q.y;
            }
        }
        __syncthreads();  // every lane has read the initial potential
        store_radial_rhs(v, radb + fo_ib(LR), a.dt[a.step0]);
    }
    __syncthreads();

#pragma unroll 1
    for (int it = 0; it < n; ++it) {
        const int step = a.step0 + it;
        const double *rb = radb + (it & 1) * S::RAD;
        const double *vb = verb + (it & 1) * S::VER;
        // prefetch the next step's blocks (their buffers were last read in step it-1)
        if (it + 1 < n) {
            copy_block(radb + ((it + 1) & 1) * S::RAD, rad_src + (size_t)(step + 1) * rad_step, S::RAD, tid);
            copy_block(verb + ((it + 1) & 1) * S::VER, a.ver + (size_t)(step + 1) * S::VER, S::VER, tid);
            cp_commit();
        }
        // ================= radial half-step: lines k, segments along j =================
        {
            double v[NLR][LR];
#pragma unroll
            for (int l = 0; l < NLR; ++l) {
                const int k = NLR * p + l;
#pragma unroll
                for (int t = 0; t < LR / 2; ++t) {
                    const double2 q = lds2(W + k * NR + 2 * (((LR / 2) * g + t) ^ x));
                    v[l][2 * t] = q.x;
                    v[l][2 * t + 1] = q.y;
                }
            }
            solve_lines<double, NLR, LR>(v, rb, g);
            // vertical right-hand side of this step (helmadi.F90:276-340) times the vertical 1/bet
            double le[NLR], re[NLR], ibz[NLR];
#pragma unroll
            for (int l = 0; l < NLR; ++l) {
                le[l] = __shfl_up_sync(kFull, v[l][LR - 1], 1, 8);
                re[l] = __shfl_down_sync(kFull, v[l][0], 1, 8);
                if (g == 0) le[l] = 0.0;
                if (g == 7) re[l] = 0.0;
                ibz[l] = vb[fo_ib(LZ) + NLR * p + l];
            }
            const double dtn = a.dt[step];
            __syncthreads();  // every lane has read W
#pragma unroll
            for (int t = 0; t < LR / 2; ++t) {
                const double2 el = lds2(coefb + (t * 8 + g) * 2);
                const double2 ab0 = lds2(coefb + 8 * LR + ((2 * t) * 8 + g) * 2);
                const double2 ab1 = lds2(coefb + 8 * LR + ((2 * t + 1) * 8 + g) * 2);
#pragma unroll
                for (int l = 0; l < NLR; ++l) {
                    const int k = NLR * p + l;
                    const int off = k * NR + 2 * (((LR / 2) * g + t) ^ x);
                    const double2 r = lds2(Rsh + off);
                    const double v0 = v[l][2 * t], v1 = v[l][2 * t + 1];
                    const double pl0 = (t > 0) ? v[l][2 * t - 1] : le[l];
                    const double pr1 = (2 * t + 2 < LR) ? v[l][2 * t + 2] : re[l];
                    const double o0 = (r.x + (el.x + dtn) * v0 - ab0.x * v1 - ab0.y * pl0) * ibz[l];
                    const double o1 = (r.y + (el.y + dtn) * v1 - ab1.x * pr1 - ab1.y * v0) * ibz[l];
                    sts2(W + off, o0, o1);
                }
            }
            __syncthreads();
        }
        // ================= vertical half-step: lines j, segments along k =================
        {
            double v[NLZ][LZ];
#pragma unroll
            for (int i = 0; i < LZ; ++i) {
                const int k = LZ * g + i;
#pragma unroll
                for (int m = 0; m < NLZ / 2; ++m) {
                    const double2 q = lds2(W + k * NR + 2 * (((NLZ / 2) * p + m) ^ x));
                    v[2 * m][i] = q.x;
                    v[2 * m + 1][i] = q.y;
                }
            }
            solve_lines<double, NLZ, LZ>(v, vb, g);
            if (it + 1 < n) {
                cp_wait_all();    // the next step's blocks (this thread's copies)
                __syncthreads();  // every lane has read W; every copy has landed
                store_radial_rhs(v, radb + ((it + 1) & 1) * S::RAD + fo_ib(LR), a.dt[step + 1]);
                __syncthreads();
            } else {
                pdl_trigger();
                double sd = 0.0, sp = 0.0;
#pragma unroll
                for (int i = 0; i < LZ; ++i) {
                    double *prow = Pg + (long long)numr * (LZ * g + i + 1) + NLZ * p + 1;
#pragma unroll
                    for (int l = 0; l < NLZ; ++l) {
                        if (a.norms) {
                            const double d = v[l][i] - prow[l];
                            sd += d * d;
                            sp += v[l][i] * v[l][i];
                        }
                        prow[l] = v[l][i];
                    }
                }
                if (a.norms) {
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) {
                        sd += __shfl_down_sync(kFull, sd, off);
                        sp += __shfl_down_sync(kFull, sp, off);
                    }
                    __syncthreads();  // W is free: the partial sums go there
                    if (lane == 0) {
                        W[2 * w] = sd;
                        W[2 * w + 1] = sp;
                    }
                    __syncthreads();
                    if (tid < 2) {
                        double tsum = 0.0;
                        for (int q = 0; q < kWThreads / 32; ++q) tsum += W[2 * q + tid];
                        const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
                        a.norms[2 * blk + tid] = wgt * tsum;
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed-precision refinement cycle, warp-cooperative, T = float (the FP32
// counterpart of k_adi_warp for the converged mixed form).  One CTA per
// slot, two CTAs per SM.
//   prologue  FP64 residual r = -4 pi rho_hat - A phi of the current
//             potential (its Dirichlet columns enter through the stencil),
//             rounded to float into Rv; delta = 0, so the first radial
//             right-hand side is r (1/bet);
//   body      2 nsteps + 1 half-steps on the defect equation A delta = r
//             with zero Dirichlet data: radial at step 0, then (vertical,
//             radial) at every step -- the cycle opens and closes on a
//             radial half-step, the order that keeps FP32 rounding of the
//             stiff near-axis components out of the result (see the
//             segmented refinement kernels in bph_adi.cu);
//   epilogue  phi += delta in FP64; per-slot |delta|^2 and |phi|^2.
// Shared memory (floats): W, Rv (NZ x NR, the 16-byte-chunk swizzle of
// k_adi_warp: 4 floats per chunk), two radial and two vertical factor
// blocks (float), the slot's (elambdazb, alphaz, betaz).
template <int NLR, int NLZ>
struct WSF {
    using S = WS<NLR, NLZ>;
    static constexpr int NR = S::NR, NZ = S::NZ, LR = S::LR, LZ = S::LZ;
    static constexpr int RAD = S::RAD, VER = S::VER, COEF = S::COEF;  // in floats
    static constexpr int O_R = NZ * NR;
    static constexpr int O_RAD = 2 * NZ * NR;
    static constexpr int O_VER = O_RAD + 2 * RAD;
    static constexpr int O_COEF = O_VER + 2 * VER;
    static constexpr int TOTAL = O_COEF + COEF;
    static_assert(RAD % 4 == 0 && VER % 4 == 0 && COEF % 4 == 0, "blocks must be whole 16-byte chunks");
    static_assert(LR % 4 == 0 && NLZ == 4, "radial segments and vertical line sets in whole float4 chunks");
};

template <int NLR, int NLZ>
__device__ __forceinline__ int swzf(int k, int j) {
    using S = WS<NLR, NLZ>;
    const int c = j >> 2;
    const int x = ((j / S::LR) ^ (k / S::LZ)) & 7;
    return k * S::NR + 4 * (c ^ x) + (j & 3);
}

struct WarpDefArgs {
    double *P;             // slot arrays [inst][N][numr*numz] (FP64, updated in place)
    const double *R;       // [inst][N][nr*nz]
    const float *rad;      // radial blocks [nsteps][N][RAD]
    const float *ver;      // vertical blocks [nsteps][VER]
    const float *coef;     // [N][COEF]
    const double *dt;      // [nsteps]
    const double *brb;     // [N][numr] radial diagonal without dt
    const double *alphar, *betar, *bzb;
    double *norms;         // per (instance, slot) |delta|^2, |phi|^2
    const int *inst_map;   // instance of each block row (nullptr: row)
    const float *r32;      // FP64 residual rounded to float, [row][N][nr*nz] (k_residual32)
    int N, numr, numz, isym, nsteps;
    double gamma;
};

// FP64 residual r = -4 pi rho_hat - A phi of the current potential (its
// Dirichlet columns enter through the stencil), rounded to float: one
// thread per zone, `bps` CTAs per (block row, slot), consecutive threads on
// consecutive zones of a row (coalesced loads of the slot plane), written
// row-major for the refinement kernel's 16-byte copies.  Enough CTAs
// (nr nz / 256 per slot) to keep every SM's loads in flight.
__global__ void __launch_bounds__(256) k_residual32(WarpDefArgs a, int nr, int nz, int bps) {
    const int q = blockIdx.x / bps;
    const int s = q % a.N, row = q / a.N;
    const int e = (blockIdx.x - q * bps) * 256 + threadIdx.x;
    const int tot = nr * nz;
    pdl_wait();
    if (e >= tot) return;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int numr = a.numr;
    const int k = e / nr, j = e - k * nr;
    const double *pc = a.P + blk * (long long)numr * a.numz + numr * (k + 1) + 1 + j;
    const double c = pc[0], ea = pc[1], no = pc[numr];
    const double we = (j > 0) ? pc[-1] : 0.0;
    const double so = (k > 0 || a.isym == 1) ? pc[-numr] : 0.0;
    const double ar = a.brb[(long long)s * numr + j + 1] * c + a.alphar[j + 1] * ea + a.betar[j + 1] * we;
    const double az = a.bzb[k + 1] * c - a.gamma * no - a.gamma * so;
    float *out = const_cast<float *>(a.r32) + ((long long)row * a.N + s) * tot;
    out[e] = (float)(a.R[blk * tot + e] - ar - az);
}

template <int NLR, int NLZ>
__global__ void __launch_bounds__(kWThreads, 2) k_adi_warp_defect(WarpDefArgs a) {
    using F = WSF<NLR, NLZ>;
    constexpr int LR = F::LR, LZ = F::LZ, NR = F::NR, NZ = F::NZ;
    extern __shared__ __align__(16) float smf[];
    float *W = smf;
    float *Rv = smf + F::O_R;
    float *radb = smf + F::O_RAD;
    float *verb = smf + F::O_VER;
    const float *coefb = smf + F::O_COEF;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane & 7;
    const int p = 4 * w + (lane >> 3);
    const int x = (g ^ w) & 7;
    const int s = blockIdx.x % a.N, row = blockIdx.x / a.N;
    const long long blk = (long long)(a.inst_map ? a.inst_map[row] : row) * a.N + s;
    const int numr = a.numr, numz = a.numz;
    double *Pg = a.P + blk * (long long)numr * numz;
    const size_t rad_step = (size_t)a.N * F::RAD;
    const float *rad_src = a.rad + (size_t)s * F::RAD;
    const double gamma = a.gamma;
    const float gf = (float)gamma;
    const bool sym_bottom = (a.isym != 1);
    const int n = a.nsteps;

    copy_block(radb, rad_src, F::RAD, tid);
    copy_block(verb, a.ver, F::VER, tid);
    copy_block(const_cast<float *>(coefb), a.coef + (size_t)s * F::COEF, F::COEF, tid);
    cp_commit();
    pdl_wait();
    // the float residual (k_residual32), 16-byte chunks into their swizzled places
    {
        constexpr int kTot = NR * NZ;
        const float *rs = a.r32 + ((long long)row * a.N + s) * (long long)kTot;
        for (int q = tid; q < kTot / 4; q += kWThreads) {
            const int e = 4 * q;
            cp16(Rv + swzf<NLR, NLZ>(e / NR, e % NR), rs + e);
        }
        cp_commit();
        cp_wait_all();
        __syncthreads();
        // first radial right-hand side: delta = 0, so r (1/bet) -- four floats of a chunk per thread
        const float *ibr = radb + fo_ib(LR);
        for (int q = tid; q < kTot / 4; q += kWThreads) {
            const int e = 4 * q;
            const int k = e / NR, j = e % NR;
            const int off = swzf<NLR, NLZ>(k, j);
            const float4 r = *reinterpret_cast<const float4 *>(Rv + off);
            const float4 ib = *reinterpret_cast<const float4 *>(ibr + j);
            *reinterpret_cast<float4 *>(W + off) = make_float4(r.x * ib.x, r.y * ib.y, r.z * ib.z, r.w * ib.w);
        }
    }
    __syncthreads();

#pragma unroll 1
    for (int h = 0; h <= 2 * n; ++h) {
        const bool radial = (h & 1) == 0;
        // prefetch: radial step i at the start of half-step 2i, vertical step i at 2i - 1
        if (radial && h >= 2 && h / 2 < n) {
            const int i = h / 2;
            copy_block(radb + (i & 1) * F::RAD, rad_src + (size_t)i * rad_step, F::RAD, tid);
            cp_commit();
        }
        if (!radial && (h + 1) / 2 < n) {
            const int i = (h + 1) / 2;
            copy_block(verb + (i & 1) * F::VER, a.ver + (size_t)i * F::VER, F::VER, tid);
            cp_commit();
        }
        if (radial) {
            const int st = (h == 0) ? 0 : h / 2 - 1;
            float v[NLR][LR];
#pragma unroll
            for (int l = 0; l < NLR; ++l) {
                const int k = NLR * p + l;
#pragma unroll
                for (int t = 0; t < LR / 4; ++t) {
                    const float4 q = *reinterpret_cast<const float4 *>(W + k * NR + 4 * (((LR / 4) * g + t) ^ x));
                    v[l][4 * t] = q.x;
                    v[l][4 * t + 1] = q.y;
                    v[l][4 * t + 2] = q.z;
                    v[l][4 * t + 3] = q.w;
                }
            }
            solve_lines<float, NLR, LR>(v, radb + (st & 1) * F::RAD, g);
            if (h == 2 * n) {
                // phi += delta in FP64, per-slot norms
                pdl_trigger();
                double sd = 0.0, sp = 0.0;
#pragma unroll
                for (int l = 0; l < NLR; ++l) {
                    double *prow = Pg + (long long)numr * (NLR * p + l + 1) + 1 + LR * g;
#pragma unroll
                    for (int i = 0; i < LR; ++i) {
                        const double d = (double)v[l][i];
                        const double ph = prow[i] + d;
                        prow[i] = ph;
                        sd += d * d;
                        sp += ph * ph;
                    }
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    sd += __shfl_down_sync(kFull, sd, off);
                    sp += __shfl_down_sync(kFull, sp, off);
                }
                __syncthreads();
                double *red = reinterpret_cast<double *>(W);
                if (lane == 0) {
                    red[2 * w] = sd;
                    red[2 * w + 1] = sp;
                }
                __syncthreads();
                if (tid < 2) {
                    double tsum = 0.0;
                    for (int q = 0; q < kWThreads / 32; ++q) tsum += red[2 * q + tid];
                    const double wgt = (s == 0 || s == a.N / 2) ? 1.0 : 2.0;
                    a.norms[2 * blk + tid] = wgt * tsum;
                }
                break;
            }
            // vertical right-hand side of the next half-step (step h / 2)
            const int sv = h / 2;
            const float *vb = verb + (sv & 1) * F::VER;
            float le[NLR], re[NLR], ibz[NLR];
            const float dtn = (float)a.dt[sv];
#pragma unroll
            for (int l = 0; l < NLR; ++l) {
                le[l] = __shfl_up_sync(kFull, v[l][LR - 1], 1, 8);
                re[l] = __shfl_down_sync(kFull, v[l][0], 1, 8);
                if (g == 0) le[l] = 0.f;
                if (g == 7) re[l] = 0.f;
            }
            cp_wait_all();
            __syncthreads();  // every lane has read W; the next blocks have landed
#pragma unroll
            for (int l = 0; l < NLR; ++l) ibz[l] = vb[fo_ib(LZ) + NLR * p + l];
#pragma unroll
            for (int t = 0; t < LR / 4; ++t) {
                float el[4], al[4], be[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int i = 4 * t + e;
                    el[e] = coefb[((i / 2) * 8 + g) * 2 + (i & 1)];
                    const float2 ab = ldp(coefb + 8 * LR + (i * 8 + g) * 2);
                    al[e] = ab.x;
                    be[e] = ab.y;
                }
#pragma unroll
                for (int l = 0; l < NLR; ++l) {
                    const int k = NLR * p + l;
                    const int off = k * NR + 4 * (((LR / 4) * g + t) ^ x);
                    const float4 r = *reinterpret_cast<const float4 *>(Rv + off);
                    const float rr[4] = {r.x, r.y, r.z, r.w};
                    float o[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int i = 4 * t + e;
                        const float pl = (i > 0) ? v[l][(i - 1) & (LR - 1)] : le[l];
                        const float pr = (i + 1 < LR) ? v[l][(i + 1) & (LR - 1)] : re[l];
                        o[e] = (rr[e] + (el[e] + dtn) * v[l][i] - al[e] * pr - be[e] * pl) * ibz[l];
                    }
                    *reinterpret_cast<float4 *>(W + off) = make_float4(o[0], o[1], o[2], o[3]);
                }
            }
            __syncthreads();
        } else {
            const int st = (h - 1) / 2;
            float v[NLZ][LZ];
#pragma unroll
            for (int i = 0; i < LZ; ++i) {
                const int k = LZ * g + i;
                const float4 q = *reinterpret_cast<const float4 *>(W + k * NR + 4 * (p ^ x));
                v[0][i] = q.x;
                v[1][i] = q.y;
                v[2][i] = q.z;
                v[3][i] = q.w;
            }
            solve_lines<float, NLZ, LZ>(v, verb + (st & 1) * F::VER, g);
            // radial right-hand side of the next half-step (the radial one of the same step)
            float dn_e[NLZ], up_e[NLZ], ib[NLZ];
#pragma unroll
            for (int l = 0; l < NLZ; ++l) {
                dn_e[l] = __shfl_up_sync(kFull, v[l][LZ - 1], 1, 8);
                up_e[l] = __shfl_down_sync(kFull, v[l][0], 1, 8);
                if (g == 0) dn_e[l] = 0.f;
                if (g == 7) up_e[l] = 0.f;
            }
            cp_wait_all();
            __syncthreads();
            {
                const float4 t4 = *reinterpret_cast<const float4 *>(radb + (st & 1) * F::RAD + fo_ib(LR) + 4 * p);
                ib[0] = t4.x;
                ib[1] = t4.y;
                ib[2] = t4.z;
                ib[3] = t4.w;
            }
            const float dtn = (float)a.dt[st];
            const float c2 = dtn - 2.f * gf, c1 = dtn - gf;
#pragma unroll
            for (int i = 0; i < LZ; ++i) {
                const int k = LZ * g + i;
                const bool refl = (k == 0) && sym_bottom;
                const int off = k * NR + 4 * (p ^ x);
                const float4 r = *reinterpret_cast<const float4 *>(Rv + off);
                const float rr[4] = {r.x, r.y, r.z, r.w};
                float o[4];
#pragma unroll
                for (int l = 0; l < NLZ; ++l) {
                    const float up = (i + 1 < LZ) ? v[l][i + 1] : up_e[l];
                    const float dn = (i > 0) ? v[l][i - 1] : dn_e[l];
                    const float rhs = refl ? rr[l] + c1 * v[l][i] + gf * up : rr[l] + c2 * v[l][i] + gf * (up + dn);
                    o[l] = rhs * ib[l];
                }
                *reinterpret_cast<float4 *>(W + off) = make_float4(o[0], o[1], o[2], o[3]);
            }
            __syncthreads();
        }
    }
}

// Factor blocks of one schedule in the segment-interleaved layout, from the
// Thomas factors [1/bet, a/bet, gam, ...] of k_adi_factors: one thread per
// (step, line system) and segment length L = n / 8.
template <typename T>
__global__ void k_pack_warp(const double *__restrict__ rad, const double *__restrict__ ver, T *__restrict__ rad_w,
                            T *__restrict__ ver_w, int nsteps, int N, int nr, int nz) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nrad = (long long)nsteps * N;
    if (t >= nrad + nsteps) return;
    const bool radial = t < nrad;
    const int n = radial ? nr : nz, L = n / 8;
    const double *src = radial ? rad + t * kAdiFactors * nr : ver + (t - nrad) * kAdiFactors * nz;
    const int bsz = 40 * L + 48;
    T *dst = radial ? rad_w + t * bsz : ver_w + (t - nrad) * bsz;
    const double *ib = src, *dd = src + n, *gam = src + 2 * n;
    double gend[8], kst[8];
    for (int g = 0; g < 8; ++g) {
        const int j0 = L * g;
        double gp = 1.0;
        for (int i = 0; i < L; ++i) {
            const int j = j0 + i;
            gp = -dd[j] * gp;
            const double gnext = (j + 1 < n) ? gam[j + 1] : 0.0;
            dst[fo_dd(L) + ((i / 2) * 8 + g) * 2 + (i & 1)] = (T)dd[j];
            dst[fo_gg(L) + (i * 8 + g) * 2] = (T)gp;
            dst[fo_gg(L) + (i * 8 + g) * 2 + 1] = (T)gnext;
        }
        gend[g] = gp;
        double kp = 1.0;
        for (int i = L - 1; i >= 0; --i) {
            const int j = j0 + i;
            const double gnext = (j + 1 < n) ? gam[j + 1] : 0.0;
            kp = -gnext * kp;
            dst[fo_k(L) + ((i / 2) * 8 + g) * 2 + (i & 1)] = (T)kp;
        }
        kst[g] = kp;
    }
    T *sc = dst + fo_scan(L);
    for (int g = 0; g < 8; ++g) {
        sc[g] = (T)gend[g];
        sc[8 + g] = (T)((g >= 1) ? gend[g] * gend[g - 1] : 0.0);
        sc[16 + g] = (T)((g >= 3) ? gend[g] * gend[g - 1] * gend[g - 2] * gend[g - 3] : 0.0);
        sc[24 + g] = (T)kst[g];
        sc[32 + g] = (T)((g <= 6) ? kst[g] * kst[g + 1] : 0.0);
        sc[40 + g] = (T)((g <= 4) ? kst[g] * kst[g + 1] * kst[g + 2] * kst[g + 3] : 0.0);
    }
    for (int j = 0; j < n; ++j) dst[fo_ib(L) + j] = (T)ib[j];
}

// (elambdazb, alphaz, betaz) of every slot in the segment-interleaved layout.
template <typename T>
__global__ void k_pack_warp_coef(const double *__restrict__ elz, const double *__restrict__ alphar,
                                 const double *__restrict__ betar, T *__restrict__ out, int N, int numr, int nr) {
    const int s = blockIdx.x;
    const int LR = nr / 8;
    T *o = out + (size_t)s * 24 * LR;
    for (int j = threadIdx.x; j < nr; j += blockDim.x) {
        const int g = j / LR, i = j % LR;
        o[((i / 2) * 8 + g) * 2 + (i & 1)] = (T)elz[(size_t)s * numr + j + 1];
        o[8 * LR + (i * 8 + g) * 2] = (T)alphar[j + 1];
        o[8 * LR + (i * 8 + g) * 2 + 1] = (T)betar[j + 1];
    }
}

template <int NLR, int NLZ>
const void *warp_kernel() {
    return (const void *)k_adi_warp<NLR, NLZ>;
}

const void *warp_kernel_for(int shape) {
    return shape == 1 ? warp_kernel<3, 4>() : warp_kernel<2, 2>();
}

const void *warp_defect_kernel() { return (const void *)k_adi_warp_defect<3, 4>; }

int warp_defect_smem() { return (int)sizeof(float) * WSF<3, 4>::TOTAL; }

int warp_smem(int shape) {
    return shape == 1 ? (int)sizeof(double) * WS<3, 4>::TOTAL : (int)sizeof(double) * WS<2, 2>::TOTAL;
}

}  // namespace

// Shape of the warp-cooperative kernel for a grid: 1 for a 128 x 96
// interior, 2 for 64 x 64, 0 when it does not apply.
int warp_shape(int nr, int nz) {
    if (nr == WS<3, 4>::NR && nz == WS<3, 4>::NZ) return 1;
    if (nr == WS<2, 2>::NR && nz == WS<2, 2>::NZ) return 2;
    return 0;
}

size_t warp_block_doubles(int n) { return (size_t)(40 * (n / 8) + 48); }

int warp_configure(bph_ctx *c) {
    c->adi_warp = 0;
    const char *env = std::getenv("BPH_ADI_WARP");
    if (env && env[0] == '0') return BPH_OK;
    const int shape = warp_shape(c->nr, c->nz);
    if (!shape) return BPH_OK;
    int dev_max = 0;
    cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    const int smem = warp_smem(shape);
    if (smem > dev_max) return BPH_OK;
    e = raise_smem_limit(warp_kernel_for(shape), smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_adi_warp)");
    const size_t coef = (size_t)c->N * 24 * (c->nr / 8);
    e = cudaMalloc((void **)&c->d_warp_coef, sizeof(double) * coef);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(warp coefficients)");
    c->bytes += sizeof(double) * coef;
    k_pack_warp_coef<double><<<c->N, 128, 0, c->stream>>>(c->d_elz, c->d_alphar, c->d_betar, c->d_warp_coef, c->N,
                                                            c->g.numr, c->nr);
    ++c->launches;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_pack_warp_coef");
    c->adi_warp = shape;
    c->adi_warp_smem = smem;
    // FP32 refinement form of the same kernel (128 x 96 interiors)
    c->mixed_warp = 0;
    if (shape == 1 && warp_defect_smem() <= dev_max) {
        const int sm32 = warp_defect_smem();
        e = raise_smem_limit(warp_defect_kernel(), sm32);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(warp_defect_kernel(), cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int per_sm = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, warp_defect_kernel(), kWThreads, sm32);
        if (e != cudaSuccess) return cuda_fail(e, "k_adi_warp_defect attributes");
        e = cudaMalloc((void **)&c->d_warp_coef32, sizeof(float) * coef);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(warp coefficients, float)");
        c->bytes += sizeof(float) * coef;
        const size_t r32 = (size_t)c->N * c->np;
        e = cudaMalloc((void **)&c->d_r32, sizeof(float) * r32);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(rounded residual)");
        c->bytes += sizeof(float) * r32;
        k_pack_warp_coef<float><<<c->N, 128, 0, c->stream>>>(c->d_elz, c->d_alphar, c->d_betar, c->d_warp_coef32, c->N,
                                                               c->g.numr, c->nr);
        ++c->launches;
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "k_pack_warp_coef<float>");
        c->mixed_warp = 1;
        c->mixed_smem_kind[BPH_MIXED_ADI_WARP] = sm32;
        c->mixed_per_sm_kind[BPH_MIXED_ADI_WARP] = per_sm;
    }
    return BPH_OK;
}

cudaError_t launch_defect_warp(bph_ctx *c, const Schedule &s, double *P, const double *R, int nrows,
                               const int *inst_map, double *norms, float *r32) {
    if (!c->mixed_warp || !s.d_warp_rad32 || !norms || !r32) return cudaErrorNotSupported;
    WarpDefArgs a;
    a.P = P;
    a.R = R;
    a.rad = s.d_warp_rad32;
    a.ver = s.d_warp_ver32;
    a.coef = c->d_warp_coef32;
    a.dt = s.d_dt;
    a.brb = c->d_brb;
    a.alphar = c->d_alphar;
    a.betar = c->d_betar;
    a.bzb = c->d_bzb;
    a.norms = norms;
    a.inst_map = inst_map;
    a.r32 = r32;
    a.N = c->N;
    a.numr = c->g.numr;
    a.numz = c->g.numz;
    a.isym = c->g.isym;
    a.nsteps = s.nsteps;
    a.gamma = c->gamma;
    c->launches += 2;
    const int bps = (c->nr * c->nz + 255) / 256;
    k_residual32<<<(unsigned)((long long)bps * c->N * nrows), 256, 0, c->stream>>>(a, c->nr, c->nz, bps);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // programmatic dependent launch: the factor-block copies of the
    // refinement kernel's prologue overlap the residual kernel's tail
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, dim3((unsigned)(c->N * nrows)), dim3(kWThreads),
                                           (size_t)warp_defect_smem(), attr);
    void *args[] = {&a};
    return cudaLaunchKernelExC(&cfg, warp_defect_kernel(), args);
}

cudaError_t launch_pack_warp(bph_ctx *c, Schedule &s) {
    const long long n = (long long)s.nsteps * c->N + s.nsteps;
    k_pack_warp<double><<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(s.d_rad, s.d_ver, s.d_warp_rad,
                                                                            s.d_warp_ver, s.nsteps, c->N, c->nr, c->nz);
    ++c->launches;
    if (c->mixed_warp) {
        k_pack_warp<float><<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(s.d_rad, s.d_ver, s.d_warp_rad32,
                                                                               s.d_warp_ver32, s.nsteps, c->N, c->nr,
                                                                               c->nz);
        ++c->launches;
    }
    return cudaGetLastError();
}

cudaError_t launch_adi_warp(bph_ctx *c, const Schedule &s, int step0, int nsteps_run, bool cold, double *P,
                            const double *R, int nrows, const int *inst_map, const int *slot_map, int nslots,
                            double *norms, cudaStream_t st, bool pdl) {
    WarpArgs a;
    a.P = P;
    a.R = R;
    a.rad = s.d_warp_rad;
    a.ver = s.d_warp_ver;
    a.coef = c->d_warp_coef;
    a.dt = s.d_dt;
    a.alphar = c->d_alphar;
    a.norms = norms;
    a.inst_map = inst_map;
    a.slot_map = slot_map;
    a.nslots = nslots;
    a.N = c->N;
    a.numr = c->g.numr;
    a.numz = c->g.numz;
    a.isym = c->g.isym;
    a.step0 = step0;
    a.nsteps = nsteps_run;
    a.cold = cold ? 1 : 0;
    a.gamma = c->gamma;
    ++c->launches;
    void *args[] = {&a};
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg =
        launch_config(c, dim3((unsigned)(nslots * nrows)), dim3(kWThreads), (size_t)c->adi_warp_smem, attr);
    cfg.stream = st;
    if (!pdl) cfg.numAttrs = 0;
    return cudaLaunchKernelExC(&cfg, warp_kernel_for(c->adi_warp), args);
}

}  // namespace bph
