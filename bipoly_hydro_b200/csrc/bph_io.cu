// bph_io.cu -- the reference's continuation record, read back into the
// solver's warm state.
//
// ritecont_frac_new.F90:151-160 writes, per rank, one Fortran unformatted
// sequential record to output/conts/fort.12.<tstep>.<rank>:
//     write(12) s, t, a, rho, tau, pot, tempa, frac1, frac2
// nine real(8) arrays of (numr_dd, numz_dd, numphi) in column-major order,
// framed by the compiler's 4-byte record-length markers; setup_frac.F90:
// 647-648 reads the same record back for a continued run (model_type 1).
// Records longer than 2^31 - 9 bytes are split into subrecords whose
// leading marker is negative (gfortran's convention; a single rank of
// the grids here stays below that).  The file is little endian (the
// reference's note for its cluster); a big-endian file is recognised by
// its marker and swapped.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kContArrays = 9;  // s, t, a, rho, tau, pot, tempa, frac1, frac2
constexpr int kContRho = 3;
constexpr int kContPot = 5;

uint32_t bswap32(uint32_t v) {
    return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}

uint64_t bswap64(uint64_t v) {
    return ((uint64_t)bswap32((uint32_t)v) << 32) | bswap32((uint32_t)(v >> 32));
}

struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

}  // namespace
}  // namespace bph

using namespace bph;

extern "C" {

int bph_read_continuation(const char *path, const bph_grid_t *grid, double *rho_out, double *pot_out) {
    if (!path || !grid) {
        set_error("path and grid must be non-NULL");
        return BPH_ERR_INVALID;
    }
    if (grid->numr < 1 || grid->numz < 1 || grid->numphi < 1) {
        set_error("invalid grid");
        return BPH_ERR_INVALID;
    }
    const size_t n = (size_t)grid->numr * grid->numz * grid->numphi;
    const uint64_t want = (uint64_t)kContArrays * n * sizeof(double);
    File fh;
    fh.f = fopen(path, "rb");
    if (!fh.f) {
        set_error("cannot open continuation file %s", path);
        return BPH_ERR_INVALID;
    }
    // Walk the (sub)records, keeping the bytes of arrays rho and pot.
    const uint64_t rho0 = (uint64_t)kContRho * n * 8, pot0 = (uint64_t)kContPot * n * 8, arr = (uint64_t)n * 8;
    uint64_t pos = 0;  // payload bytes consumed so far
    bool swap = false, first = true, more = true;
    std::vector<unsigned char> buf;
    while (more) {
        uint32_t raw;
        if (fread(&raw, 4, 1, fh.f) != 1) {
            set_error("%s: truncated record marker", path);
            return BPH_ERR_INVALID;
        }
        if (first) {
            // the first marker tells the byte order: a plausible length either way
            const int32_t le = (int32_t)raw, be = (int32_t)bswap32(raw);
            const uint64_t ale = (uint64_t)(le < 0 ? -(int64_t)le : le), abe = (uint64_t)(be < 0 ? -(int64_t)be : be);
            const bool le_ok = ale > 0 && ale <= want, be_ok = abe > 0 && abe <= want;
            if (!le_ok && be_ok) swap = true;
            first = false;
        }
        int32_t m = (int32_t)(swap ? bswap32(raw) : raw);
        more = m < 0;  // a negative leading marker: more subrecords follow
        const uint64_t len = (uint64_t)(m < 0 ? -(int64_t)m : m);
        if (len == 0 || pos + len > want) {
            set_error("%s: record of %llu bytes does not hold nine %dx%dx%d real(8) arrays (%llu bytes)", path,
                      (unsigned long long)(pos + len), grid->numr, grid->numz, grid->numphi,
                      (unsigned long long)want);
            return BPH_ERR_INVALID;
        }
        buf.resize((size_t)len);
        if (fread(buf.data(), 1, (size_t)len, fh.f) != (size_t)len) {
            set_error("%s: truncated record payload", path);
            return BPH_ERR_INVALID;
        }
        for (int which = 0; which < 2; ++which) {
            double *out = which ? pot_out : rho_out;
            const uint64_t a0 = which ? pot0 : rho0;
            if (!out) continue;
            const uint64_t lo = pos > a0 ? pos : a0, hi = (pos + len < a0 + arr) ? pos + len : a0 + arr;
            if (lo < hi) memcpy(reinterpret_cast<unsigned char *>(out) + (lo - a0), buf.data() + (lo - pos), hi - lo);
        }
        pos += len;
        uint32_t tail;
        if (fread(&tail, 4, 1, fh.f) != 1) {
            set_error("%s: truncated trailing record marker", path);
            return BPH_ERR_INVALID;
        }
        const int32_t t = (int32_t)(swap ? bswap32(tail) : tail);
        if ((uint64_t)(t < 0 ? -(int64_t)t : t) != len) {
            set_error("%s: record markers disagree (%d vs %d)", path, (int)m, (int)t);
            return BPH_ERR_INVALID;
        }
    }
    if (pos != want) {
        set_error("%s: record of %llu bytes, expected nine %dx%dx%d real(8) arrays (%llu bytes)", path,
                  (unsigned long long)pos, grid->numr, grid->numz, grid->numphi, (unsigned long long)want);
        return BPH_ERR_INVALID;
    }
    if (swap) {
        for (double *out : {rho_out, pot_out}) {
            if (!out) continue;
            uint64_t *u = reinterpret_cast<uint64_t *>(out);
            for (size_t i = 0; i < n; ++i) u[i] = bswap64(u[i]);
        }
    }
    return BPH_OK;
}

int bph_restore_continuation(bph_ctx_t *c, const char *path, double *rho_out) {
    if (!c) {
        set_error("context is NULL");
        return BPH_ERR_INVALID;
    }
    std::vector<double> pot((size_t)c->ntot);
    int rc = bph_read_continuation(path, &c->g, rho_out, pot.data());
    if (rc) return rc;
    return bph_set_potential(c, pot.data(), 0);
}

}  // extern "C"
