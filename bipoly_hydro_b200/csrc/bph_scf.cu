// bph_scf.cu -- one SCF-like iteration on device-resident arrays.
//
// The reference reads its initial models from disk (scfin_frac.F90:105-125);
// the self-consistent-field code that makes them is not part of it.  A model
// sweep (mass ratio, separation) is a sequence of density updates, each
// followed by a potential solve warm-started from the previous potential.
// bph_scf_step does one such iteration in one call, without the density
// leaving the device:
//   1. rho <- 0.9 rho + 0.1 rho (1 + eps xi), xi ~ N(0,1) per zone, from a
//      counter-based generator (SplitMix64 of seed, iteration and zone; two
//      32-bit uniforms; Box-Muller), so a sequence is reproducible anywhere;
//   2. renormalised to a fixed mass M = sum over interior zones of
//      rho(J,K,L) rhf(J) dr dz dphi (the zone volume of the cylindrical
//      grid, setup_frac.F90:429-456), summed in a fixed order (results do
//      not depend on the launch);
//   3. the potential_solver step (tstep > 1 warm, else cold).
#include <cstdint>

#include "bph_internal.cuh"

namespace bph {
namespace {

constexpr int kScfThreads = 256;
constexpr int kScfBlocks = 512;  // fixed: the mass reduction order does not depend on the device

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Standard normal deviate of zone i at (seed, iteration).
__device__ __forceinline__ double scf_normal(uint64_t seed, int iteration, long long i) {
    const uint64_t key = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(iteration + 1));
    const uint64_t z = splitmix64(key + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1));
    const double u1 = ((double)(z >> 32) + 0.5) * (1.0 / 4294967296.0);
    const double u2 = ((double)(z & 0xffffffffull) + 0.5) * (1.0 / 4294967296.0);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// Update every zone; per-block partial masses of the interior before
// (part[2b]) and after (part[2b+1]) the update.
__global__ void __launch_bounds__(kScfThreads) k_scf_update(double *__restrict__ rho, const double *__restrict__ rhf,
                                                            int numr, int numz, long long ntot, double eps,
                                                            uint64_t seed, int iteration, double *__restrict__ part) {
    double m0 = 0.0, m1 = 0.0;
    const long long nplane = (long long)numr * numz;
    for (long long i = (long long)blockIdx.x * kScfThreads + threadIdx.x; i < ntot;
         i += (long long)kScfBlocks * kScfThreads) {
        const double r = rho[i];
        const double xi = scf_normal(seed, iteration, i);
        const double rn = 0.9 * r + 0.1 * (r * (1.0 + eps * xi));
        rho[i] = rn;
        const int J = (int)(i % numr), K = (int)((i % nplane) / numr);  // 0-based
        if (J >= 1 && J <= numr - 2 && K >= 1 && K <= numz - 2) {
            m0 += r * rhf[J];
            m1 += rn * rhf[J];
        }
    }
    __shared__ double red[2][kScfThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        m0 += __shfl_down_sync(0xffffffffu, m0, off);
        m1 += __shfl_down_sync(0xffffffffu, m1, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = m0;
        red[1][warp] = m1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int w = 0; w < kScfThreads / 32; ++w) t += red[threadIdx.x][w];
        part[2 * blockIdx.x + threadIdx.x] = t;
    }
}

// Every block sums the partials in the same order, then scales its zones so
// that the interior mass becomes `mass` (mass <= 0: the mass before the update).
__global__ void __launch_bounds__(kScfThreads) k_scf_scale(double *__restrict__ rho, long long ntot,
                                                           const double *__restrict__ part, double vol, double mass,
                                                           double *__restrict__ scale_out) {
    __shared__ double sc;
    if (threadIdx.x == 0) {
        double before = 0.0, after = 0.0;
        for (int b = 0; b < kScfBlocks; ++b) {
            before += part[2 * b];
            after += part[2 * b + 1];
        }
        before *= vol;
        after *= vol;
        const double target = (mass > 0.0) ? mass : before;
        sc = (after > 0.0) ? target / after : 1.0;
        if (blockIdx.x == 0 && scale_out) {
            scale_out[0] = sc;
            scale_out[1] = (mass > 0.0) ? mass : before;
        }
    }
    __syncthreads();
    const double s = sc;
    for (long long i = (long long)blockIdx.x * kScfThreads + threadIdx.x; i < ntot;
         i += (long long)kScfBlocks * kScfThreads)
        rho[i] *= s;
}

}  // namespace

cudaError_t launch_scf_update(bph_ctx *c, double *d_rho, double eps, double mass, unsigned long long seed,
                              int iteration, double *d_part) {
    const double *rhf = c->d_grid;  // rhf_g[numr] leads the grid block
    k_scf_update<<<kScfBlocks, kScfThreads, 0, c->stream>>>(d_rho, rhf, c->g.numr, c->g.numz, c->ntot, eps,
                                                            (uint64_t)seed, iteration, d_part);
    const double vol = c->g.dr * c->dz * c->dphi;
    k_scf_scale<<<kScfBlocks, kScfThreads, 0, c->stream>>>(d_rho, c->ntot, d_part, vol, mass,
                                                           d_part + 2 * kScfBlocks);
    c->launches += 2;
    return cudaGetLastError();
}

size_t scf_scratch_doubles() { return 2 * kScfBlocks + 2; }

}  // namespace bph
