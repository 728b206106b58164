// bph_compact.h -- layout of the compact Green tables.
//
// The boundary tables G[m][b][p] (tm.F90, sm.F90, bm.F90) hold, for every
// boundary row b and interior zone p = (j, k), the mode-m Green function
// coef * Q(chi) with chi = (r_b^2 + r_j^2 + (z_b - z_k)^2) / (2 r_b r_j)
// (plus the reflected-image term at z_b + z_k for isym 2 and 3), coef =
// sqrt(r_j / r_b) / pi.  Two symmetries make most of the table redundant:
//
//   * top (and, for isym 1, bottom) rows: the boundary point sits at a
//     grid radius r_jb of the same set as r_j and at a fixed height, so
//     H(jb, j, k) = G(jb, j, k) / r_j = Q / (pi sqrt(r_jb r_j)) is symmetric
//     in (jb, j).  Only the 8 x 8 tiles (I, J), I <= J, of the jb x j plane
//     are stored, one per interior height k: tile[k][r][c] = H(8I + r,
//     8J + c, k), the tiles of one height contiguous.  A tile serves row jb = 8I + r with columns 8J + c and, by
//     symmetry, row 8J + c with columns 8I + r.
//   * side rows: the boundary point sits at r_B = r_{numr} and height
//     z_kb, so on the uniform vertical grid G depends on k only through
//     kb - k and kb + k: G(kb, j, k) = U_j(kb - k) + V_j(kb + k).  Per mode
//     and radial zone j, U and V are vectors of about 2 nz values.
//
// For the 130 x 98 grid (30 modes) this stores 212 MB of the 660 MB, and
// the boundary contraction that streams them per solve moves that much less.
// Plain C++ shared by the kernels and a host-side check.
#pragma once

#if defined(__CUDACC__)
#define BPH_CHD __host__ __device__
#else
#define BPH_CHD
#endif

namespace bph {
namespace compact {

constexpr int kTile = 8;         // rows and columns of a tile
constexpr int kWarps = 8;        // warps of a contraction CTA
constexpr int kMaxKpl = 8;       // side rows per lane: nz <= 256
constexpr int kPartPair = 32;    // partial sums of a tile: row / column x 8 x (cos, sin)
constexpr int kHeightParts = 1;  // height ranges a tile or side group is split into (work items)
constexpr int kStageHeights = 2; // heights per stage of the contraction's ring; the tiles are padded to a multiple
constexpr int kMomPad = 8;       // zeroed doubles after the moment array: an 8-zone run of the last row stays in bounds

struct Dims {
    int nr = 0, nz = 0;
    int nb8 = 0;        // tiles along jb and j
    int npair = 0;      // stored tiles (I <= J) per height
    int nsets = 0;      // 1: top rows, 2: top and bottom (isym 1)
    int kpl = 0;        // side rows per lane (ceil(nz / 32))
    int stride = 0;     // doubles per U or V vector (zero-padded)
    int top_ctas = 0;   // CTAs of tiles per mode (8 tiles each)
    int side_ctas = 0;  // CTAs of side vectors per mode (8 radial zones each)
    int nh = 0;         // height parts (kHeightParts, or nz when smaller)
    int hp = 0;         // heights per part, a multiple of kStageHeights (the last part may be shorter)
    int nzp = 0;        // heights of the tile table: nz rounded up to kStageHeights (zero tiles above nz)
    bool ok = false;    // the compact form applies to this grid
};

BPH_CHD inline Dims dims(int nr, int nz, int isym) {
    Dims d;
    d.nr = nr;
    d.nz = nz;
    d.nb8 = (nr + kTile - 1) / kTile;
    d.npair = d.nb8 * (d.nb8 + 1) / 2;
    d.nsets = (isym == 1) ? 2 : 1;
    d.kpl = (nz + 31) / 32;
    d.stride = nz + 32 * d.kpl;
    d.top_ctas = (d.nsets * d.npair + kWarps - 1) / kWarps;
    d.side_ctas = (nr + kWarps - 1) / kWarps;
    d.nh = nz < kHeightParts ? nz : kHeightParts;
    d.hp = d.nh > 0 ? (nz + d.nh - 1) / d.nh : 0;
    d.hp = ((d.hp + kStageHeights - 1) / kStageHeights) * kStageHeights;
    d.nzp = ((nz + kStageHeights - 1) / kStageHeights) * kStageHeights;
    d.ok = nr >= 1 && nz >= 1 && d.kpl <= kMaxKpl;
    return d;
}

// Tile index of blocks (I, J), I <= J: row-major over the upper triangle.
BPH_CHD inline int pair_index(int I, int J, int nb8) { return I * nb8 - I * (I - 1) / 2 + (J - I); }

BPH_CHD inline void pair_blocks(int q, int nb8, int *I, int *J) {
    int i = 0, first = 0;
    while (q >= first + (nb8 - i)) {
        first += nb8 - i;
        ++i;
    }
    *I = i;
    *J = i + (q - first);
}

// Positions in the U and V vectors of side row kb and height k.
BPH_CHD inline int side_u(int kb, int k, int nz) { return kb - k + nz - 1; }
BPH_CHD inline int side_v(int kb, int k) { return kb + k; }

// Doubles of each table and of the partial-sum scratch, per mode.
BPH_CHD inline long long pair_doubles(const Dims &d) { return (long long)d.nsets * d.npair * d.nzp * kTile * kTile; }
BPH_CHD inline long long side_doubles(const Dims &d) { return (long long)d.nr * 2 * d.stride; }
// Partial sums of one mode: per height part, the tiles' then the side
// groups'; after the nh parts, the same block once more for their sums.
BPH_CHD inline long long part_height_doubles(const Dims &d) {
    return (long long)d.nsets * d.npair * kPartPair + (long long)d.side_ctas * d.nz * 2;
}
BPH_CHD inline long long part_doubles(const Dims &d) { return (long long)(d.nh + 1) * part_height_doubles(d); }

// Arrival counters: one per mode, then one per (mode, tile set or side group).
BPH_CHD inline long long counters(const Dims &d, int mmax) {
    return (long long)mmax * (1 + d.top_ctas + d.side_ctas);
}

// Heights [k0, k1) of part h (empty when k0 >= nz).
BPH_CHD inline void height_range(const Dims &d, int h, int *k0, int *k1) {
    const int a = h * d.hp, b = a + d.hp;
    *k0 = a < d.nz ? a : d.nz;
    *k1 = b < d.nz ? b : d.nz;
}

// Work items of one launch: mode-major, then height part, then the mode's
// tile sets and side groups.
BPH_CHD inline long long items(const Dims &d, int mmax) {
    return (long long)mmax * d.nh * (d.top_ctas + d.side_ctas);
}

}  // namespace compact
}  // namespace bph
