// bph_boundary.cu -- the boundary potential (bessel.F90:170-488).
//
// k_green_contract: S[m][b] = sum_p G[m][b][p] * (cos, sin moment)[m][p],
// the per-mode contraction of the Green tables with the interior density
// moments (bessel.F90:186-296).  The tables (8 bytes per element, read once
// per solve) dominate the compulsory bytes of a solve, so the kernel is a
// streaming GEMV with two right-hand sides: 16-byte evict-first loads of the
// table rows, the moment vectors (small, L2-resident) read once per CTA
// for BR rows, and a fixed-order CTA reduction (deterministic results).
//
// k_boundary_slots: the Dirichlet data of the ADI sweeps in Fourier-slot
// space.  The reference synthesises the physical boundary potential
//   Phi_B(l) = factor [S_C0 + 2 sum_{m>=1} (S_Cm cos k th_l + S_Sm sin k th_l)],
// th_l = (l - 1/2) dphi, k = fm*m (bessel.F90:399-488), writes it into potp
// and transforms it with the rest of potp (helmadi.F90:159).  For k < N/2
// that transform is exact in closed form:
//   F_0 = N factor S_C0,  F_k = e^{-i pi k/N} N factor (S_Cm + i S_Sm),
// and zero at every other frequency, so the slots are written directly.
#include <cmath>
#include <cstdlib>

#include "bph_compact.h"
#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kContractRows = 8;
constexpr int kContractThreads = 256;

// Grid (row groups, mmax, nsplit).  CTA (g, m, k) reduces table rows
// b0..b0+7 of mode m over the k-th slice of the interior zones; the number
// of slices is chosen at setup so that the launch fills whole waves of the
// GPU.  Slices write partial sums, and the last CTA of each (m, group) to
// arrive adds them in slice order (deterministic) and writes S; it also
// resets its arrival counter for the next launch.
// Dirichlet slots of one boundary row, written by the CTA that finishes the
// row's moments (the closed form of k_boundary_slots below, fused so that
// the solve needs no separate launch).  Slots of modes without boundary
// data and the corner columns are zero from set-up and never written.
struct SlotOut {
    double *P;          // slot array [N][nplane], or nullptr: S only
    const double2 *ph;  // (cos, sin) of pi fm m / N
    int numr, numz, nr, nz, M, fm;
    double nfactor;     // N * factor
};

// Dirichlet slot of boundary row b, mode m from (S_C, S_S): the cosine
// slot fm m (part 0) or the sine slot M + fm m (part 1, m > 0).
__device__ __forceinline__ void write_slot(const SlotOut &so, int m, int b, double sc, double ss, int part) {
    int jz, kz;
    if (b < so.nr) {
        jz = b + 1;
        kz = so.numz - 1;
    } else if (b < so.nr + so.nz) {
        jz = so.numr - 1;
        kz = b - so.nr + 1;
    } else {
        jz = b - so.nr - so.nz + 1;
        kz = 0;
    }
    const long long nplane = (long long)so.numr * so.numz;
    const long long pos = jz + (long long)so.numr * kz;
    const int k = so.fm * m;
    const double2 w = so.ph[m];
    if (part == 0)
        so.P[(long long)k * nplane + pos] = so.nfactor * (w.x * sc + w.y * ss);
    else if (m > 0)
        so.P[(long long)(so.M + k) * nplane + pos] = so.nfactor * (w.y * sc - w.x * ss);
}

template <bool kVec>
__global__ void __launch_bounds__(kContractThreads, 2)
k_green_contract(const double *__restrict__ G, const double *__restrict__ mom, double *__restrict__ S,
                 long long np, int nb, unsigned int *__restrict__ counters, double *__restrict__ partials,
                 SlotOut so) {
    const int m = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
    const int b0 = blockIdx.x * kContractRows;
    const int nrows = min(kContractRows, nb - b0);
    // slice bounds in units of 2 doubles (16-byte loads) when vectorised
    const long long unit = kVec ? 2 : 1, nu = np / unit;
    const long long chunk = (nu + nsplit - 1) / nsplit;
    const long long u0 = split * chunk, u1 = min(nu, u0 + chunk);
    const double *mc = mom + (2LL * m) * np;
    const double *ms = mom + (2LL * m + 1) * np;
    const double *g0 = G + ((long long)m * nb + b0) * np;
    double ac[kContractRows], as[kContractRows];
#pragma unroll
    for (int r = 0; r < kContractRows; ++r) ac[r] = as[r] = 0.0;
    pdl_wait();
    if (kVec) {
        const double2 *mc2 = reinterpret_cast<const double2 *>(mc);
        const double2 *ms2 = reinterpret_cast<const double2 *>(ms);
        for (long long i = u0 + threadIdx.x; i < u1; i += kContractThreads) {
            double2 g[kContractRows];
#pragma unroll
            for (int r = 0; r < kContractRows; ++r)
                g[r] = (r < nrows) ? __ldcs(reinterpret_cast<const double2 *>(g0 + r * np) + i) : make_double2(0.0, 0.0);
            const double2 vc = __ldg(mc2 + i), vs = __ldg(ms2 + i);
#pragma unroll
            for (int r = 0; r < kContractRows; ++r) {
                ac[r] = fma(g[r].x, vc.x, ac[r]);
                ac[r] = fma(g[r].y, vc.y, ac[r]);
                as[r] = fma(g[r].x, vs.x, as[r]);
                as[r] = fma(g[r].y, vs.y, as[r]);
            }
        }
    } else {
        for (long long i = u0 + threadIdx.x; i < u1; i += kContractThreads) {
            const double vc = __ldg(mc + i), vs = __ldg(ms + i);
#pragma unroll
            for (int r = 0; r < kContractRows; ++r) {
                if (r < nrows) {
                    const double g = __ldcs(g0 + r * np + i);
                    ac[r] = fma(g, vc, ac[r]);
                    as[r] = fma(g, vs, as[r]);
                }
            }
        }
    }
    pdl_trigger();
    __shared__ double red[kContractThreads / 32][2 * kContractRows];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < kContractRows; ++r) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            ac[r] += __shfl_down_sync(0xffffffffu, ac[r], off);
            as[r] += __shfl_down_sync(0xffffffffu, as[r], off);
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < kContractRows; ++r) {
            red[warp][2 * r] = ac[r];
            red[warp][2 * r + 1] = as[r];
        }
    }
    __syncthreads();
    const long long slice_stride = (long long)gridDim.y * nb * 2;
    double v = 0.0;
    if (threadIdx.x < 2 * nrows) {
#pragma unroll
        for (int w = 0; w < kContractThreads / 32; ++w) v += red[w][threadIdx.x];
    }
    // Threads 2r, 2r+1 of warp 0 hold (S_C, S_S) of row b0 + r.
    auto finish = [&](double val) {
        const double other = __shfl_xor_sync(0xffffffffu, val, 1);
        if (threadIdx.x >= 2 * nrows) return;
        const int r = threadIdx.x >> 1, cs = threadIdx.x & 1;
        const double mine = (m == 0 && cs == 1) ? 0.0 : val;
        S[((long long)m * nb + b0 + r) * 2 + cs] = mine;
        if (!so.P) return;
        const double sc = cs ? other : mine;
        const double ss = (m == 0) ? 0.0 : (cs ? mine : other);
        write_slot(so, m, b0 + r, sc, ss, cs);
    };
    if (nsplit == 1) {
        if (threadIdx.x < 32) finish(v);
        return;
    }
    if (threadIdx.x < 2 * nrows) partials[split * slice_stride + ((long long)m * nb + b0) * 2 + threadIdx.x] = v;
    __threadfence();
    __syncthreads();
    const int tile = m * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) last = (atomicAdd(counters + tile, 1u) == (unsigned)(nsplit - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 32) {
        double t = 0.0;
        if (threadIdx.x < 2 * nrows)
            for (int k = 0; k < nsplit; ++k)
                t += __ldcg(partials + k * slice_stride + ((long long)m * nb + b0) * 2 + threadIdx.x);
        finish(t);
    }
    if (threadIdx.x == 0) counters[tile] = 0u;
}

// One thread per (boundary row b, slot s); rows nb.. write the corner
// columns, which stay zero (bessel.F90:417,452: pott(numr)=pots(numz)=0).
__global__ void k_boundary_slots(const double *__restrict__ S, const double2 *__restrict__ ph,
                                 double *__restrict__ P, int numr, int numz, int nr, int nz, int nb, int N,
                                 int mmax, int fm, int isym, double nfactor) {
    const int M = N / 2;
    const int ncorner = (isym == 1) ? 2 : 1;
    pdl_wait();
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)(nb + ncorner) * N) return;
    const int s = (int)(t % N), b = (int)(t / N);
    const long long nplane = (long long)numr * numz;
    int jz, kz;
    if (b < nr) {
        jz = b + 1;
        kz = numz - 1;
    } else if (b < nr + nz) {
        jz = numr - 1;
        kz = b - nr + 1;
    } else if (b < nb) {
        jz = b - nr - nz + 1;
        kz = 0;
    } else {
        jz = numr - 1;
        kz = (b == nb) ? numz - 1 : 0;
        P[(long long)s * nplane + jz + (long long)numr * kz] = 0.0;
        return;
    }
    const bool imag = s > M;
    const int k = imag ? s - M : s;
    double v = 0.0;
    if (k < M && k % fm == 0 && k / fm < mmax) {
        const int m = k / fm;
        const double sc = S[((long long)m * nb + b) * 2], ss = S[((long long)m * nb + b) * 2 + 1];
        const double2 w = ph[m];  // (cos, sin) of pi k / N
        v = imag ? nfactor * (w.y * sc - w.x * ss) : nfactor * (w.x * sc + w.y * ss);
    }
    P[(long long)s * nplane + jz + (long long)numr * kz] = v;
}

// ---------------------------------------------------------------------------
// k_green_compact: the same S (and Dirichlet slots) from the compact tables
// of bph_compact.h.  One CTA of 8 warps per work item, items mode-major;
// an item is one height part (compact::kHeightParts of them; splitting
// the heights evens out the last wave but costs more than it saves at
// 130x98, so one part is the default) of a mode's set of 8 tiles or of a
// group of 8 side zones.
// Both roles stage what they read in shared memory with cp.async, so the
// bytes in flight do not cost registers.
//
// Tile warps (one tile (I, J) over the item's heights): a ring of kRing
// stages of kStageH heights per warp; lane l copies its 16 bytes of each
// height's 512 (evict-first) and one of the 32 moments a height needs
// ((cos, sin) pairs of the rows 8I.. and the columns 8J..).  Lane
// (r = l / 4, c0 = 2 (l % 4)) then accumulates
//   row part:    sum_k H(8I + r, 8J + c, k) mom(8J + c, k)   -> S[8I + r]
//   column part: sum_k H(8I + r, 8J + c, k) mom(8I + r, k)   -> S[8J + c]
// for c = c0, c0 + 1 (the column part is the mirrored tile (J, I), unused
// when I == J).  The radii r_j of G = H r_j scale the sums at the end;
// shuffles reduce them over the tile's rows and columns in a fixed order.
//
// Side warps (one radial zone j over the item's heights): the CTA stages
// the moments of its eight zones and each warp its U and V vectors; lane
// holds side rows kb = KPL lane + i and slides windows of U_j(kb - k),
// V_j(kb + k) over k (one new U and one new V value per height), so the
// side rows cost compute, not table bytes.  The CTA adds its eight zones in
// shared memory.
//
// Reduction in three fixed-order levels (deterministic): every item writes
// its partial sums; the last of a tile set's (or side group's) height parts
// to arrive adds the parts; the last of a mode's tile sets and side groups
// adds those per boundary row, writes S and the slots, and resets the
// counters for the next launch.
struct CompactArgs {
    const double *T;    // tiles [m][set][k < nzp][tile][64]
    const double *U;    // side vectors [m][j][U | V][stride]
    const double *mom;  // moments [2m + cs][np]
    const double *rw;   // r_j, j < nr
    double *S;          // [m][nb][2]
    double *part;       // per mode and height part: tile parts [set][tile][32], then side parts [group][nz][2]
    unsigned int *cnt;  // arrival counters (compact::counters)
    long long np, part_m, part_h;
    int nr, nz, nzp, nb, nb8, npair, nsets, stride, top_ctas, side_ctas, mmax, nh, hp;
    SlotOut so;
};

constexpr int kRing = 4;                            // stages in a tile warp's ring
constexpr int kStageH = compact::kStageHeights;     // heights per stage
constexpr int kHeightDoubles = 64 + 32;     // a height: 64 tile elements, 16 (cos, sin) moment pairs
constexpr int kStageDoubles = kStageH * kHeightDoubles;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cpa16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa16_ef_u(uint32_t dst, const void *src, unsigned long long pol) {
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cpa8_u(uint32_t dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Dynamic shared bytes: the larger of the tile rings and the side staging
// (moment pairs of eight zones over a height part, U and V of each warp).
inline size_t compact_smem(int hp, int stride) {
    const size_t ring = sizeof(double) * compact::kWarps * kRing * kStageDoubles;
    const size_t side = sizeof(double) * ((size_t)2 * compact::kWarps * hp + (size_t)compact::kWarps * 2 * stride);
    return ring > side ? ring : side;
}

// One work item (see k_green_compact below); `it` is the item's index.
template <int KPL>
__device__ __forceinline__ void compact_item(const CompactArgs &a, int it, double *csm, double (*red)[64],
                                             bool &last) {
    using namespace compact;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nr = a.nr, nz = a.nz;
    const long long np = a.np;
    const int per_m = a.top_ctas + a.side_ctas;
    const int per_mode_items = a.nh * per_m;
    const int m = it / per_mode_items;
    const int rem = it % per_mode_items;
    const int h = rem / per_m, role = rem % per_m;
    const int k0 = min(h * a.hp, nz), k1 = min(k0 + a.hp, nz);
    const double *mc = a.mom + 2LL * m * np;
    double *pmode = a.part + (long long)m * a.part_m;
    double *part = pmode + (long long)h * a.part_h;
    const long long top_doubles = (long long)a.nsets * a.npair * kPartPair;
    if (role < a.top_ctas) {
        const int q = role * kWarps + warp;
        if (q < a.nsets * a.npair && k1 > k0) {
            const int set = q / a.npair, tile = q % a.npair;
            int I, J;
            pair_blocks(tile, a.nb8, &I, &J);
            double *ring = csm + warp * kRing * kStageDoubles;
            const long long hstride = (long long)a.npair * 64;  // doubles between heights of a tile
            const int nst = (k1 - k0 + kStageH - 1) / kStageH;
            const int r = lane >> 2, c0 = 2 * (lane & 3);
            double r0c = 0.0, r0s = 0.0, r1c = 0.0, r1s = 0.0, k0c = 0.0, k0s = 0.0, k1c = 0.0, k1s = 0.0;
            unsigned long long evict_first;
            asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(evict_first));
            // the lane's table bytes and moment of height k0; both advance by fixed strides per height
            const double *tnext =
                a.T + ((long long)m * a.nsets + set) * a.nzp * hstride + (long long)k0 * hstride + tile * 64 + 2 * lane;
            // moment lane l stages per height: pair l / 2 (rows 8I.. for l / 2 < 8, columns 8J.. after),
            // component l % 2 (cos, sin), at slot l of the height's 32; heights past nz (zero tiles)
            // read the last height's moment
            const int idx = lane >> 1, cs_l = lane & 1;
            const int jl = min(idx < 8 ? kTile * I + idx : kTile * J + idx - 8, nr - 1);
            const double *mnext = mc + (long long)cs_l * np + jl + (long long)nr * k0;
            const double *mlast = mc + (long long)cs_l * np + jl + (long long)nr * (nz - 1);
            int knext = k0;
            const uint32_t tdst = smem_u32(ring) + 16 * lane, mdst = smem_u32(ring) + 8 * (64 + lane);
            constexpr uint32_t kStageBytes = 8 * kStageDoubles, kHeightBytes = 8 * kHeightDoubles;
            // the first stages' table bytes, then their moments
            {
                const double *t = tnext;
#pragma unroll
                for (int u = 0; u < kRing - 1; ++u)
#pragma unroll
                    for (int hh = 0; hh < kStageH; ++hh) {
                        if (u < nst) cpa16_ef_u(tdst + u * kStageBytes + hh * kHeightBytes, t, evict_first);
                        t += hstride;
                    }
            }
            pdl_wait();  // the moments come from the forward transform
#pragma unroll
            for (int u = 0; u < kRing - 1; ++u) {
                if (u < nst) {
#pragma unroll
                    for (int hh = 0; hh < kStageH; ++hh) {
                        cpa8_u(mdst + u * kStageBytes + hh * kHeightBytes, knext < nz ? mnext : mlast);
                        tnext += hstride;
                        mnext += nr;
                        ++knext;
                    }
                }
                cpa_commit();
            }
            for (int sidx = 0; sidx < nst; ++sidx) {
                cpa_wait<kRing - 2>();
                __syncwarp();  // stage sidx has landed for every lane; stage sidx - 1 is consumed
                if (sidx + kRing - 1 < nst) {
                    const uint32_t so = ((sidx + kRing - 1) & (kRing - 1)) * kStageBytes;
#pragma unroll
                    for (int hh = 0; hh < kStageH; ++hh) {
                        cpa16_ef_u(tdst + so + hh * kHeightBytes, tnext, evict_first);
                        cpa8_u(mdst + so + hh * kHeightBytes, knext < nz ? mnext : mlast);
                        tnext += hstride;
                        mnext += nr;
                        ++knext;
                    }
                }
                cpa_commit();
                const double *st = ring + (sidx & (kRing - 1)) * kStageDoubles;
#pragma unroll
                for (int hh = 0; hh < kStageH; ++hh) {
                    // heights past k1 within the last stage are zero tiles (padding above nz)
                    const double *sh = st + hh * kHeightDoubles;
                    const double2 t = *reinterpret_cast<const double2 *>(sh + 2 * lane);
                    const double2 x0 = *reinterpret_cast<const double2 *>(sh + 64 + 2 * (8 + c0));
                    const double2 x1 = *reinterpret_cast<const double2 *>(sh + 64 + 2 * (9 + c0));
                    const double2 y = *reinterpret_cast<const double2 *>(sh + 64 + 2 * r);
                    r0c = fma(t.x, x0.x, r0c);
                    r0s = fma(t.x, x0.y, r0s);
                    r1c = fma(t.y, x1.x, r1c);
                    r1s = fma(t.y, x1.y, r1s);
                    k0c = fma(t.x, y.x, k0c);
                    k0s = fma(t.x, y.y, k0s);
                    k1c = fma(t.y, y.x, k1c);
                    k1s = fma(t.y, y.y, k1s);
                }
            }
            cpa_wait<0>();
            // G = H r_j: the row part takes the columns' radii, the column part the row's
            const int jr = min(kTile * I + r, nr - 1);
            const int jc0 = min(kTile * J + c0, nr - 1), jc1 = min(kTile * J + c0 + 1, nr - 1);
            const double wr = a.rw[jr], w0 = a.rw[jc0], w1 = a.rw[jc1];
            double rc = w0 * r0c + w1 * r1c, rs = w0 * r0s + w1 * r1s;
            double cc0 = wr * k0c, cs0 = wr * k0s, cc1 = wr * k1c, cs1 = wr * k1s;
#pragma unroll
            for (int off = 1; off <= 2; off <<= 1) {
                rc += __shfl_xor_sync(0xffffffffu, rc, off);
                rs += __shfl_xor_sync(0xffffffffu, rs, off);
            }
#pragma unroll
            for (int off = 4; off <= 16; off <<= 1) {
                cc0 += __shfl_xor_sync(0xffffffffu, cc0, off);
                cs0 += __shfl_xor_sync(0xffffffffu, cs0, off);
                cc1 += __shfl_xor_sync(0xffffffffu, cc1, off);
                cs1 += __shfl_xor_sync(0xffffffffu, cs1, off);
            }
            double *pp = part + (long long)q * kPartPair;  // [row | column][8][cos, sin]
            if ((lane & 3) == 0) {
                pp[2 * r] = rc;
                pp[2 * r + 1] = rs;
            }
            if (lane < 4) {
                pp[16 + 2 * c0] = cc0;
                pp[16 + 2 * c0 + 1] = cs0;
                pp[16 + 2 * c0 + 2] = cc1;
                pp[16 + 2 * c0 + 3] = cs1;
            }
        } else {
            pdl_wait();
            if (q < a.nsets * a.npair) part[(long long)q * kPartPair + lane] = 0.0;  // an empty height part
        }
    } else {
        const int g = role - a.top_ctas;
        const int j = g * kWarps + warp;
        const int hk = k1 - k0;
        // staging: moment pairs [k - k0][8 zones][cos, sin], then U | V of each warp
        double *msh = csm;
        double *uvw = csm + 2 * kWarps * a.hp + (long long)warp * 2 * a.stride;
        if (j < nr) {
            const double *Uv = a.U + ((long long)m * nr + j) * 2 * a.stride;
            for (int c = lane; c < a.stride; c += 32) cpa16(uvw + 2 * c, Uv + 2 * c);  // 2 stride doubles
        }
        pdl_wait();
        for (int e = threadIdx.x; e < 2 * kWarps * hk; e += blockDim.x) {
            const int cs = e & 1, jj = (e >> 1) & (kWarps - 1), kk = e >> 4;
            const int jz = min(g * kWarps + jj, nr - 1);
            cpa8(msh + e, mc + (long long)cs * np + jz + (long long)nr * (k0 + kk));
        }
        cpa_commit();
        cpa_wait<0>();
        __syncthreads();
        double acc_c[KPL], acc_s[KPL];
#pragma unroll
        for (int i = 0; i < KPL; ++i) acc_c[i] = acc_s[i] = 0.0;
        if (j < nr && hk > 0) {
            const double *Uv = uvw, *Vv = uvw + a.stride;
            const int base = KPL * lane;
            // windows as rings: at step s = k - kb of a block of KPL heights,
            // U_j(kb_i - k) = uu[(i - s) mod KPL] and V_j(kb_i + k) = vv[(i + s) mod KPL];
            // the value that leaves each window is replaced in place (no moves)
            double uu[KPL], vv[KPL];
#pragma unroll
            for (int i = 0; i < KPL; ++i) {
                uu[i] = Uv[base + i + nz - 1 - k0];
                vv[i] = Vv[base + i + k0];
            }
            const double2 *mp = reinterpret_cast<const double2 *>(msh) + warp;
            // the values entering the windows at the next height; after the last height the U
            // pointer reads one element before this warp's vectors (staged memory, never used)
            const double *up = Uv + base + nz - 2 - k0, *vp = Vv + base + KPL + k0;
            for (int kb = k0; kb < k1; kb += KPL) {
#pragma unroll
                for (int st = 0; st < KPL; ++st) {
                    if (kb + st < k1) {
                        const double2 x = *mp;
                        const double un = *up, vn = *vp;
                        mp += kWarps;
                        --up;
                        ++vp;
#pragma unroll
                        for (int i = 0; i < KPL; ++i) {
                            const double w = uu[(i - st + KPL) % KPL] + vv[(i + st) % KPL];
                            acc_c[i] = fma(w, x.x, acc_c[i]);
                            acc_s[i] = fma(w, x.y, acc_s[i]);
                        }
                        uu[KPL - 1 - st] = un;
                        vv[st] = vn;
                    }
                }
            }
        }
        // the CTA's eight zones, added in warp order, one window position at a time
        double *ps = part + top_doubles + (long long)g * nz * 2;
#pragma unroll
        for (int i = 0; i < KPL; ++i) {
            red[warp][2 * lane] = acc_c[i];
            red[warp][2 * lane + 1] = acc_s[i];
            __syncthreads();
            if (threadIdx.x < 64) {
                double val = 0.0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) val += red[w][threadIdx.x];
                const int kb = KPL * (threadIdx.x >> 1) + i;
                if (kb < nz) ps[2 * kb + (threadIdx.x & 1)] = val;
            }
            __syncthreads();
        }
    }
    pdl_trigger();
    // level 2: the last height part of this tile set / side group adds the parts
    unsigned int *mcnt = a.cnt, *rcnt = a.cnt + a.mmax;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(rcnt + (long long)m * per_m + role, 1u) == (unsigned)(a.nh - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    double *merged = pmode + (long long)a.nh * a.part_h;
    if (role < a.top_ctas) {
        const int q = role * kWarps + warp;
        if (q < a.nsets * a.npair) {
            double t = 0.0;
            for (int hh = 0; hh < a.nh; ++hh) t += __ldcg(pmode + (long long)hh * a.part_h + (long long)q * kPartPair + lane);
            merged[(long long)q * kPartPair + lane] = t;
        }
    } else {
        const long long off = top_doubles + (long long)(role - a.top_ctas) * nz * 2;
        for (int e = threadIdx.x; e < 2 * nz; e += blockDim.x) {
            double t = 0.0;
            for (int hh = 0; hh < a.nh; ++hh) t += __ldcg(pmode + (long long)hh * a.part_h + off + e);
            merged[off + e] = t;
        }
    }
    if (threadIdx.x == 0) rcnt[(long long)m * per_m + role] = 0u;
    // level 3: the last tile set / side group of the mode adds the merged parts per boundary row
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(mcnt + m, 1u) == (unsigned)(per_m - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int b = threadIdx.x; b < a.nb; b += blockDim.x) {
        double sc = 0.0, ss = 0.0;
        if (b < nr || b >= nr + nz) {
            const int set = (b < nr) ? 0 : 1;
            const int jb = (b < nr) ? b : b - nr - nz;
            const int I = jb / kTile, r = jb % kTile;
            const double *pt = merged + (long long)set * a.npair * kPartPair;
            // column parts of tiles (I', I), I' < I, then row parts of tiles (I, J), J >= I
#pragma unroll 8
            for (int t = 0; t < a.nb8; ++t) {
                const double *pp = (t < I) ? pt + (long long)pair_index(t, I, a.nb8) * kPartPair + 16 + 2 * r
                                           : pt + (long long)pair_index(I, t, a.nb8) * kPartPair + 2 * r;
                const double2 v = __ldcg(reinterpret_cast<const double2 *>(pp));
                sc += v.x;
                ss += v.y;
            }
        } else {
            const double *pside = merged + top_doubles + 2 * (b - nr);
#pragma unroll 8
            for (int gg = 0; gg < a.side_ctas; ++gg) {
                const double2 v = __ldcg(reinterpret_cast<const double2 *>(pside + (long long)gg * nz * 2));
                sc += v.x;
                ss += v.y;
            }
        }
        if (m == 0) ss = 0.0;
        a.S[((long long)m * a.nb + b) * 2] = sc;
        a.S[((long long)m * a.nb + b) * 2 + 1] = ss;
        if (a.so.P) {
            write_slot(a.so, m, b, sc, ss, 0);
            write_slot(a.so, m, b, sc, ss, 1);
        }
    }
    if (threadIdx.x == 0) mcnt[m] = 0u;
}

// One CTA per work item.  (A persistent grid that fetched items from a
// counter balanced the last wave but cost more in per-item overhead at
// 130x98.)
template <int KPL>
__global__ void __launch_bounds__(256, KPL <= 4 ? 3 : 2) k_green_compact(CompactArgs a) {
    extern __shared__ __align__(16) double csm[];
    __shared__ double red[compact::kWarps][64];
    __shared__ bool last;
    compact_item<KPL>(a, (int)blockIdx.x, csm, red, last);  // waits for the previous kernel before its first write
}

const void *compact_kernel(int kpl) {
    switch (kpl) {
        case 1: return (const void *)k_green_compact<1>;
        case 2: return (const void *)k_green_compact<2>;
        case 3: return (const void *)k_green_compact<3>;
        case 4: return (const void *)k_green_compact<4>;
        case 5: return (const void *)k_green_compact<5>;
        case 6: return (const void *)k_green_compact<6>;
        case 7: return (const void *)k_green_compact<7>;
        default: return (const void *)k_green_compact<8>;
    }
}

}  // namespace

int contract_configure(bph_ctx *c) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_green_contract<true>, kContractThreads, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const long long slots = (long long)sms * (per_sm > 0 ? per_sm : 1);
    const long long tiles = (long long)c->g.mmax * ((c->nb + kContractRows - 1) / kContractRows);
    // smallest slice count whose last wave is >= 90% full, at least 2048 zones per slice
    int best = 1;
    double best_eff = 0.0;
    for (int k = 1; k <= 16; ++k) {
        if (k > 1 && c->np / k < 2048) break;
        double waves = (double)(tiles * k) / (double)slots;
        double eff = waves / std::ceil(waves);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = k;
        }
        if (eff >= 0.9) break;
    }
    c->contract_split = best;
    return BPH_OK;
}

int compact_configure(bph_ctx *c) {
    c->compact = 0;
    const char *env = std::getenv("BPH_COMPACT");
    if (env && env[0] == '0') return BPH_OK;
    const compact::Dims d = compact::dims(c->nr, c->nz, c->g.isym);
    if (!d.ok) return BPH_OK;
    const size_t mm = (size_t)c->g.mmax;
    const size_t nt = mm * (size_t)compact::pair_doubles(d), ns = mm * (size_t)compact::side_doubles(d),
                 np = mm * (size_t)compact::part_doubles(d);
    cudaError_t e = cudaMalloc((void **)&c->d_gtile, sizeof(double) * nt);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_gside, sizeof(double) * ns);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_kpart, sizeof(double) * np);
    const size_t ncnt = (size_t)compact::counters(d, c->g.mmax);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_kcnt, sizeof(unsigned int) * ncnt);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_kcnt, 0, sizeof(unsigned int) * ncnt, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "compact Green tables");
    c->bytes += sizeof(double) * (nt + ns + np) + sizeof(unsigned int) * ncnt;
    const int smem = (int)compact_smem(d.hp, d.stride);
    e = raise_smem_limit(compact_kernel(d.kpl), smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_green_compact)");

    e = launch_green_compact(c);
    if (e != cudaSuccess) return cuda_fail(e, "k_green_compact_tiles / k_green_compact_side");
    c->compact = 1;
    return BPH_OK;
}

cudaError_t launch_green_compact_contract(bph_ctx *c, bool write_slots) {
    const compact::Dims d = compact::dims(c->nr, c->nz, c->g.isym);
    CompactArgs a;
    a.T = c->d_gtile;
    a.U = c->d_gside;
    a.mom = c->d_mom;
    a.rw = c->d_grid + 1;  // rhf[j + 1]
    a.S = c->d_S;
    a.part = c->d_kpart;
    a.cnt = c->d_kcnt;
    a.np = c->np;
    a.part_m = compact::part_doubles(d);
    a.nr = c->nr;
    a.nz = c->nz;
    a.nb = c->nb;
    a.nb8 = d.nb8;
    a.npair = d.npair;
    a.nsets = d.nsets;
    a.stride = d.stride;
    a.top_ctas = d.top_ctas;
    a.side_ctas = d.side_ctas;
    a.so.P = write_slots ? c->d_P : nullptr;
    a.so.ph = c->d_ph;
    a.so.numr = c->g.numr;
    a.so.numz = c->g.numz;
    a.so.nr = c->nr;
    a.so.nz = c->nz;
    a.so.M = c->M;
    a.so.fm = c->fm;
    a.so.nfactor = (double)c->N * c->factor;
    a.mmax = c->g.mmax;
    a.nh = d.nh;
    a.hp = d.hp;
    a.nzp = d.nzp;

    a.part_h = compact::part_height_doubles(d);
    ++c->launches;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, dim3((unsigned)compact::items(d, c->g.mmax)), dim3(256),
                                           compact_smem(d.hp, d.stride), attr);
    void *args[] = {&a};
    return cudaLaunchKernelExC(&cfg, compact_kernel(d.kpl), args);
}

cudaError_t launch_green_contract(bph_ctx *c, bool write_slots) {
    if (c->compact) return launch_green_compact_contract(c, write_slots);
    dim3 grid((unsigned)((c->nb + kContractRows - 1) / kContractRows), (unsigned)c->g.mmax,
              (unsigned)c->contract_split);
    SlotOut so;
    so.P = write_slots ? c->d_P : nullptr;
    so.ph = c->d_ph;
    so.numr = c->g.numr;
    so.numz = c->g.numz;
    so.nr = c->nr;
    so.nz = c->nz;
    so.M = c->M;
    so.fm = c->fm;
    so.nfactor = (double)c->N * c->factor;
    ++c->launches;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, grid, dim3(kContractThreads), 0, attr);
    const double *G = c->d_green, *mom = c->d_mom;
    if (c->np % 2 == 0)
        return cudaLaunchKernelEx(&cfg, k_green_contract<true>, G, mom, c->d_S, c->np, c->nb, c->d_ccnt, c->d_cpart,
                                  so);
    return cudaLaunchKernelEx(&cfg, k_green_contract<false>, G, mom, c->d_S, c->np, c->nb, c->d_ccnt, c->d_cpart, so);
}

cudaError_t launch_boundary_slots(bph_ctx *c) {
    int ncorner = (c->g.isym == 1) ? 2 : 1;
    long long n = (long long)(c->nb + ncorner) * c->N;
    int threads = 256;
    ++c->launches;
    k_boundary_slots<<<(unsigned)((n + threads - 1) / threads), threads, 0, c->stream>>>(
        c->d_S, c->d_ph, c->d_P, c->g.numr, c->g.numz, c->nr, c->nz, c->nb, c->N, c->g.mmax, c->fm, c->g.isym,
        (double)c->N * c->factor);
    return cudaGetLastError();
}

}  // namespace bph
