// fdsea.cuh - the Fermi-sea Berry-curvature dipole on the finite-difference geometry.
//
// The reference's default BCD geometry backend (derivative_backend = :finite_difference,
// Runtime/Config.jl:113) evaluates, for a Fermi-sea moment, the band curvature at k +- delta_c
// and takes the central difference (berry_curvature_dipole_component!,
// Responses/QuantumGeometry/QuantumGeometryDerivatives.jl:193-228, called per band from
// prepare_berry_multipole_geometry!, BerryMultipoleGeometry.jl:67-161); delta_c is the
// fractional image lattice * (h e_c) / 2 pi of the Cartesian step (finite_difference_step_matrix,
// Core/Coordinates.jl:15-44).  The moment is D[mu,a,b,c] = sum_n f(E_n; mu, T) d_c Omega_n^{ab}
// (berry_dipole_moments!, BerryMultipoleMoments.jl:7-47; berry_multipole_sea_weight,
// BerryMultipoleDC.jl:56-62).
//
// On the device a batch's shifted points go through the arbitrary-k front (Fourier, eigensolve,
// isolation check) and the response kernel's band-curvature items, which leave Omega_n^{ab} in a
// per-batch buffer [entry][2 nd][npair][nw] (slot 2 j: +delta of derivative axis j, 2 j + 1:
// -delta); the centre's front then supplies E_n and sea_dipole_kernel combines the two.
#pragma once

#include "common.cuh"
#include "response.cuh"

#define SEA_MAX_ITEMS 96

// Shifted k-points of one batch: k_i + sign delta, k_i from caller k-points, a mesh index list
// or a run of mesh indices (the same three sources as the front's phase kernels).
__global__ void fd_shift_kernel(const double *__restrict__ kpts, const int64_t *__restrict__ kidx, int64_t k_begin,
                                int64_t n1, int64_t n2, int64_t n3, int64_t nb, double d0, double d1, double d2,
                                double *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    double k0, k1, k2;
    if (kpts) {
        k0 = kpts[3 * i];
        k1 = kpts[3 * i + 1];
        k2 = kpts[3 * i + 2];
    } else {
        const int64_t idx = kidx ? kidx[i] : k_begin + i;
        k0 = (double)(idx % n1) / (double)n1;
        k1 = (double)((idx / n1) % n2) / (double)n2;
        k2 = (double)(idx / (n1 * n2)) / (double)n3;
    }
    out[3 * i] = k0 + d0;
    out[3 * i + 1] = k1 + d1;
    out[3 * i + 2] = k2 + d2;
}

struct SeaParams {
    int nw;
    int64_t batch;
    const double *E;         // centre energies [batch][nw]
    const double *curv;      // shifted band curvatures [batch][2 nd][npair][nw]
    int nd, npair;
    int n_items;
    int item_pair[SEA_MAX_ITEMS], item_dir[SEA_MAX_ITEMS];
    int64_t item_out[SEA_MAX_ITEMS];
    int nmu;
    const double *mus;
    double temperature;
    double two_h;            // 2 h (1/Angstrom)
    double scale;
    const double *weights;   // mode 0 per-k weights; nullptr: scale
    int mode;                // 0: partial sums [gridDim][vc][4]; 1: per-point values
    int64_t vc;
    double *partials;
    double2 *out_points;
    int64_t point_offset;
    const int *out_perm;
};

// One CTA per contiguous range of the batch and one partial-sum slot per CTA (the response
// kernel's rule, so the sum does not depend on scheduling); a thread per (item, mu) value.
__global__ void __launch_bounds__(128) sea_dipole_kernel(SeaParams p) {
    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x;
    const int64_t ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    const int nw = p.nw;
    const int64_t pstride = (int64_t)2 * p.nd * p.npair * nw;
    const int nval = p.n_items * p.nmu;
    for (int v = threadIdx.x; v < nval; v += blockDim.x) {
        const int it = v / p.nmu, im = v % p.nmu;
        const double mu = p.mus[im];
        const int64_t plus = (int64_t)(2 * p.item_dir[it]) * p.npair * nw + (int64_t)p.item_pair[it] * nw;
        const int64_t minus = plus + (int64_t)p.npair * nw;
        const int64_t idx = p.item_out[it] + im;
        double *acc = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
        for (int64_t b = kb; b < ke; ++b) {
            const double *e = p.E + b * nw;
            const double *c = p.curv + b * pstride;
            double value = 0.0;
            for (int n = 0; n < nw; ++n)
                value += response_occ(e[n], mu, p.temperature) * ((c[plus + n] - c[minus + n]) / p.two_h);
            if (p.mode == 0) {
                const double wk = p.weights ? p.weights[b] * p.scale : p.scale;
                neumaier_add(acc[0], acc[2], value * wk);
            } else {
                const int64_t row = p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : b);
                p.out_points[row * p.vc + idx] = make_double2(value * p.scale, 0.0);
            }
        }
    }
}
