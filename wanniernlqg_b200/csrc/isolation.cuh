// isolation.cuh - the spectral isolation contract of the exact geometry, per k-point on the device.
//
// The reference refuses a k-point whose spectrum the requested geometry cannot resolve:
//   * geometry_isolated_spectrum_minimum_gap (MatrixElements/Interpolated/OrthogonalBandDerivatives.jl:66-82)
//     throws GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED unless every pair of bands is split by more
//     than the tolerance; the Berry dipole calls it with degeneracy_threshold
//     (Responses/QuantumGeometry/BerryMultipoleGeometry.jl:81), the exact (eta = 0) gauge
//     correction with spectral_gap_tolerance (PositionMatrixElements.jl:447-452);
//   * spectral_subspace_blocks (SubspacePositionMatrixElements.jl:5-22) groups levels within
//     32 eps max(1, max|E|) of a block's first level and throws SPECTRAL_CROSS_BLOCK_GAP_UNRESOLVED
//     when a distinct level is split from its neighbour by no more than the tolerance.
// Energies come out of the eigensolvers in ascending order, so the smallest pair gap is the
// smallest adjacent gap.  A failing point records (row << 24 | batch entry) with atomicMin, so
// the smallest caller row wins; a one-thread kernel then stores, for that row, the first failing
// pair in the reference's loop order (m ascending, then l ascending) and its gap.  One row can be
// checked on several spectra (the centre and the shifted points of a finite-difference stencil):
// each check carries a priority in the reference's order (0 = the centre) and the record keeps
// the failing spectrum of the smallest priority.
#pragma once

#include <math_constants.h>

#include "common.cuh"

enum { ISO_ALL_PAIRS = 0, ISO_SPECTRAL_BLOCKS = 1 };

// No failure recorded.
#define ISO_NONE 0xFFFFFFFFFFFFFFFFull
#define ISO_LOCAL_BITS 24

struct IsoRecord {
    int l, m;       // 0-based bands of the first failing pair
    double gap;     // their energy difference (eV)
    int64_t row;    // caller row (mesh index or point index) of the failing k-point; -1 = none
    int prio;       // priority of the spectrum that failed (0 = the centre)
};

// First failing pair of one sorted spectrum in the reference's loop order; false when none fails.
WNLQG_HD bool iso_first_failure(const double *E, int n, double tol, int mode, int &l_out, int &m_out,
                                       double &gap_out) {
    if (mode == ISO_ALL_PAIRS) {
        for (int m = 0; m < n; ++m)
            for (int l = 0; l < m; ++l) {
                const double gap = fabs(E[m] - E[l]);
                if (!(gap > tol)) { l_out = l; m_out = m; gap_out = gap; return true; }
            }
        return false;
    }
    double emax = 0.0;
    for (int i = 0; i < n; ++i) emax = fmax(emax, fabs(E[i]));
    const double exact = 32.0 * 2.220446049250313e-16 * fmax(1.0, emax);
    int start = 0;
    for (int m = 1; m < n; ++m) {
        if (E[m] - E[start] > exact) {
            const double adjacent = E[m] - E[m - 1];
            if (!(adjacent > tol)) { l_out = m - 1; m_out = m; gap_out = adjacent; return true; }
            start = m;
        }
    }
    return false;
}

// One thread per k-point of the batch: flag the first failing row.
__global__ void isolation_check_kernel(const double *__restrict__ E, int64_t nb, int nw, double tol, int mode,
                                       int64_t row_base, const int *__restrict__ perm,
                                       unsigned long long *__restrict__ key) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const double *e = E + i * nw;
    bool bad = false;
    for (int j = 0; j < nw && !bad; ++j) bad = !isfinite(e[j]);
    if (!bad) {
        if (mode == ISO_ALL_PAIRS) {
            for (int j = 1; j < nw && !bad; ++j) bad = !(e[j] - e[j - 1] > tol);
        } else {
            int l, m;
            double g;
            bad = iso_first_failure(e, nw, tol, mode, l, m, g);
        }
    }
    if (bad) {
        const int64_t row = row_base + (perm ? (int64_t)perm[i] : i);
        atomicMin(key, ((unsigned long long)row << ISO_LOCAL_BITS) | (unsigned long long)i);
    }
}

// The record of the winning row, when it belongs to this batch (rows of later batches are larger,
// so the record of an earlier batch is never overwritten by a later one).
__global__ void isolation_record_kernel(const double *__restrict__ E, int64_t nb, int nw, double tol, int mode,
                                        int64_t row_base, const unsigned long long *__restrict__ key,
                                        IsoRecord *__restrict__ rec, int prio) {
    const unsigned long long k = *key;
    if (k == ISO_NONE) return;
    const int64_t row = (int64_t)(k >> ISO_LOCAL_BITS);
    const int64_t i = (int64_t)(k & ((1ull << ISO_LOCAL_BITS) - 1));
    if (row < row_base || i >= nb) return;
    if (rec->row == row && rec->prio <= prio) return;   // an earlier spectrum of this row failed
    const double *e = E + i * nw;
    int l = -1, m = -1;
    double gap = 0.0;
    bool nonfinite = false;
    for (int j = 0; j < nw; ++j) nonfinite |= !isfinite(e[j]);
    if (!nonfinite && !iso_first_failure(e, nw, tol, mode, l, m, gap)) return;   // this spectrum passes
    rec->l = l;
    rec->m = m;
    rec->gap = nonfinite ? CUDART_NAN : gap;
    rec->row = row;
    rec->prio = prio;
}
