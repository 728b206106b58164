// bph_slices.h -- slices of the interior zones of the split-K contractions.
//
// The tensor-core batched contraction splits the np interior zones of a
// mode into nsplit slices, one CTA per (row group, mode, slice), and
// streams each slice in chunks of `chunk_steps` steps of 8 zones.  A slice
// is a whole number of chunks, so that the chunks of one slice never read
// zones of the next one (which the next slice's CTA adds as well); zones at
// or past z_end are zero-filled.  Plain C++, shared by the kernel and the
// host-side check that runs without a GPU.
#pragma once

#if defined(__CUDACC__)
#define BPH_HD __host__ __device__
#else
#define BPH_HD
#endif

namespace bph {

struct ZoneSlice {
    long long k_begin;  // first 8-zone step of the slice
    long long k_end;    // one past its last step (== k_begin: empty slice)
    long long z_end;    // one past its last zone (<= np)
};

BPH_HD inline ZoneSlice zone_slice(long long np, int nsplit, int split, int chunk_steps) {
    const long long nk = (np + 7) / 8;  // 8-zone steps; the last one may be partial
    long long per = (nk + nsplit - 1) / nsplit;
    per = ((per + chunk_steps - 1) / chunk_steps) * chunk_steps;
    ZoneSlice s;
    s.k_begin = (long long)split * per;
    long long e = s.k_begin + per;
    if (e > nk) e = nk;
    s.k_end = e > s.k_begin ? e : s.k_begin;
    const long long z = 8 * s.k_end;
    s.z_end = z < np ? z : np;
    return s;
}

}  // namespace bph
