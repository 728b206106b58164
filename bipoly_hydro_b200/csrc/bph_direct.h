// bph_direct.h -- eigen-decomposition of the vertical ADI operator, for the
// direct defect solve of the mixed-precision converged forms.
//
// After the azimuthal transform every Fourier slot is a 2-D (r, z) system
// A = A_r (x) I + I (x) A_z: A_r is the radial tridiagonal of the slot
// (diagonal brb, off-diagonals alphar / betar, helmadi.F90:195-260) and
// A_z = gamma T with T the constant vertical second difference
// (bzb = 2 gamma, and gamma in the first row when the equatorial plane
// reflects: helmadi.F90:285-340), Dirichlet at the top.  T is diagonalised
// in closed form:
//   reflecting bottom (isym 2, 3): v_q(k) = cos((k + 1/2) theta_q),
//                                   theta_q = (q + 1/2) pi / (nz + 1/2);
//   Dirichlet bottom (isym 1):      v_q(k) = sin((k + 1) theta_q),
//                                   theta_q = (q + 1) pi / (nz + 1);
//   eigenvalue lambda_q = 2 - 2 cos theta_q.
// With E the orthonormal eigenvector matrix (rows q), A x = r becomes
// (A_r + gamma lambda_q) y_q = (E r)_q for every vertical mode q, and
// x = E^T y: one transform, nz radial tridiagonal solves, one transform.
// Plain C++ (long double), shared by the set-up and a host-side check.
#pragma once

#include <cmath>
#include <vector>

namespace bph {
namespace direct {

// E (nz x nz, row q = eigenvector q, orthonormal) and lambda (nz) of T.
inline void vertical_eigen(int nz, int isym, std::vector<long double> &E, std::vector<long double> &lambda) {
    const long double pi = std::acos(-1.0L);
    E.assign((size_t)nz * nz, 0.0L);
    lambda.assign((size_t)nz, 0.0L);
    for (int q = 0; q < nz; ++q) {
        const long double th = (isym == 1) ? (q + 1.0L) * pi / (nz + 1.0L) : (q + 0.5L) * pi / (nz + 0.5L);
        long double norm = 0.0L;
        for (int k = 0; k < nz; ++k) {
            const long double v = (isym == 1) ? std::sin((k + 1.0L) * th) : std::cos((k + 0.5L) * th);
            E[(size_t)q * nz + k] = v;
            norm += v * v;
        }
        norm = std::sqrt(norm);
        for (int k = 0; k < nz; ++k) E[(size_t)q * nz + k] /= norm;
        lambda[q] = 2.0L - 2.0L * std::cos(th);
    }
}

// T applied to x (the operator the eigen-decomposition diagonalises).
inline void apply_vertical(int nz, int isym, const long double *x, long double *y) {
    for (int k = 0; k < nz; ++k) {
        const long double dn = (k > 0) ? x[k - 1] : 0.0L;
        const long double up = (k + 1 < nz) ? x[k + 1] : 0.0L;
        const long double diag = (k == 0 && isym != 1) ? 1.0L : 2.0L;
        y[k] = diag * x[k] - dn - up;
    }
}

}  // namespace direct
}  // namespace bph
