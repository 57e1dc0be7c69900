// bcd_analytic.cuh - the Fermi-sea Berry-curvature dipole on the analytic geometry
// (derivative_backend = :analytic): the local dipole d_c Omega_n^{ab} of every band from the
// central point alone.
//
// Reference: orthogonal_bcd_partition_matrices! and orthogonal_geometry_partition_diagonal
// (Responses/QuantumGeometry/OrthogonalGeometryDerivatives.jl:24-113) over the Hamiltonian-frame
// jets of prepare_orthogonal_geometry_jets! (MatrixElements/Interpolated/OrthogonalGeometryJets.jl:
// 176-218) and the band derivatives D_a = U^H d_a U, D_ac = U^H d_a d_c U of
// orthogonal_band_first_derivative! / orthogonal_band_second_derivative!
// (OrthogonalBandDerivatives.jl:123-245); the moment D[mu, a, b, c] = sum_n f(E_n; mu, T) d_c Omega_n
// (berry_dipole_moments!, BerryMultipoleMoments.jl:7-47).
//
// Only the diagonals of the six partitions are consumed, so every term X Y enters as
// sum_l X_nl Y_ln (O(nw) per band) and every triple X Y Z as (X Y) then sum_l (X Y)_nl Z_ln: eight
// full products (Dc Db, Db Dc, Dc Da, Da Dc, Dc Aa, Dc Ab, Db Aa, Da Ab) per component, beside the
// rotations of the jets (two products each; one for the jets whose diagonal alone is used) and
// the four products of the two second band derivatives.  One CTA per point range, the matrices
// in a per-CTA global working set (L2-resident up to ~40 orbitals), products on the FP64 tensor
// cores (dmma_product); FP64 in both precision modes.
#pragma once

#include "common.cuh"
#include "dmma.cuh"
#include "response.cuh"

#define BCDA_MAX_ITEMS 32
#define BCDA_MAX_NW 128
#define BCDA_SLOTS 19

struct BcdaParams {
    int nw, ld;
    int64_t batch;
    int64_t xw_stride;          // complex entries per point in xw (C nw^2)
    const double2 *xw;          // Wannier-gauge channels [batch][C][nw][nw]
    const double *E;            // [batch][nw]
    const double2 *U;           // [batch][nw][nw]
    int n_items;
    int item_a[BCDA_MAX_ITEMS], item_b[BCDA_MAX_ITEMS], item_c[BCDA_MAX_ITEMS];
    int64_t item_out[BCDA_MAX_ITEMS];
    // Channel indices: dH[a], A[a], ddH[a * 3 + c] (symmetric), dA[p * 3 + d] = d_d A_p,
    // ddA[p * 9 + c * 3 + g] = d_c d_g A_p (symmetric in c, g).
    int ch_dH[3], ch_A[3], ch_ddH[9], ch_dA[9], ch_ddA[27];
    int nmu;
    const double *mus;
    double temperature;
    double scale;
    const double *weights;      // mode 0 per-k weights; nullptr: scale
    int mode;                   // 0: partial sums [gridDim][vc][4]; 1: per-point values
    int64_t vc;
    double *partials;
    double2 *out_points;
    int64_t point_offset;
    const int *out_perm;
    unsigned char *gscratch;    // BCDA_SLOTS matrices of nw x ld per CTA
    int64_t gscratch_stride;
};

__global__ void __launch_bounds__(256) bcd_analytic_kernel(BcdaParams p) {
    const int nw = p.nw, ld = p.ld, nn = nw * nw;
    const int tid = threadIdx.x;
    const size_t mat = (size_t)nw * ld;
    double2 *slots = reinterpret_cast<double2 *>(p.gscratch + (int64_t)blockIdx.x * p.gscratch_stride);
    double2 *U = slots, *T1 = slots + mat, *T2 = slots + 2 * mat;
    double2 *dHa = slots + 3 * mat, *dHb = slots + 4 * mat, *dHc = slots + 5 * mat;
    double2 *ddHac = slots + 6 * mat, *ddHbc = slots + 7 * mat;
    double2 *Aa = slots + 8 * mat, *Ab = slots + 9 * mat, *Ac = slots + 10 * mat;
    double2 *Aac = slots + 11 * mat, *Abc = slots + 12 * mat, *Om = slots + 13 * mat;
    double2 *Da = slots + 14 * mat, *Db = slots + 15 * mat, *Dc = slots + 16 * mat;
    double2 *Dac = slots + 17 * mat, *Dbc = slots + 18 * mat;
    __shared__ double sE[BCDA_MAX_NW], sTot[BCDA_MAX_NW];
    __shared__ double sdEa[BCDA_MAX_NW], sdEb[BCDA_MAX_NW], sdEc[BCDA_MAX_NW];
    __shared__ double2 sAca[BCDA_MAX_NW], sAcb[BCDA_MAX_NW], sOmc[BCDA_MAX_NW];

    // sum_l X_nl Y_ln
    auto diag2 = [&](const double2 *X, const double2 *Y, int n) {
        double2 s = make_double2(0.0, 0.0);
        for (int l = 0; l < nw; ++l) s = cadd(s, cmul(X[n + ld * l], Y[l + ld * n]));
        return s;
    };
    // T2 <- X0 - X1 (Wannier-gauge channels, X1 optional), laid out with ld.
    auto load = [&](const double2 *xw, int c0, int c1) {
        const double2 *x0 = xw + (int64_t)c0 * nn, *x1 = c1 >= 0 ? xw + (int64_t)c1 * nn : nullptr;
        for (int e = tid; e < nn; e += blockDim.x) {
            double2 v = x0[e];
            if (x1) v = csub(v, x1[e]);
            T2[(e % nw) + ld * (e / nw)] = v;
        }
        __syncthreads();
    };
    // dst = U^H (X0 - X1) U
    auto rotate = [&](const double2 *xw, int c0, int c1, double2 *dst) {
        load(xw, c0, c1);
        dmma_product<0>(T2, U, T1, nw, ld);
        __syncthreads();
        dmma_product<1>(U, T1, dst, nw, ld);
        __syncthreads();
    };
    // dst0 = U^H X0 U and dst1 = U^H X1 U in two paired DMMA passes, the channels read straight
    // from the Wannier-gauge input (leading dimension nw).
    auto rotate2 = [&](const double2 *xw, int c0, int c1, double2 *dst0, double2 *dst1) {
        dmma_product_pair<0>(xw + (int64_t)c0 * nn, nw, U, T1, xw + (int64_t)c1 * nn, nw, U, T2, nw, ld);
        __syncthreads();
        dmma_product_pair<1>(U, ld, T1, dst0, U, ld, T2, dst1, nw, ld);
        __syncthreads();
    };
    // diag[n] = (U^H (X0 - X1) U)_nn
    auto rotate_diag = [&](const double2 *xw, int c0, int c1, double2 *diag) {
        load(xw, c0, c1);
        dmma_product<0>(T2, U, T1, nw, ld);
        __syncthreads();
        for (int n = tid; n < nw; n += blockDim.x) {
            double2 s = make_double2(0.0, 0.0);
            for (int l = 0; l < nw; ++l) s = cadd(s, cmul(cconj(U[l + ld * n]), T1[l + ld * n]));
            diag[n] = s;
        }
        __syncthreads();
    };
    // D_x = U^H d_x U: dH_nm / (E_m - E_n) off the diagonal, i A_nn on it.
    auto first = [&](const double2 *dH, const double2 *A, double2 *D) {
        for (int e = tid; e < nn; e += blockDim.x) {
            const int i = e % nw, m = e / nw;
            D[i + ld * m] = i == m ? cmuli(A[i + ld * i]) : cscale(dH[i + ld * m], 1.0 / (sE[m] - sE[i]));
        }
    };
    // D_xc = U^H d_x d_c U (orthogonal_band_second_derivative! with alpha = x, beta = c).
    auto second = [&](const double2 *dHx, const double2 *ddHxc, const double2 *Ax, const double2 *Dx,
                      const double *dEx, const double2 *Axc, const double2 *Acx_diag, double2 *out) {
        dmma_product_pair<0>(dHx, ld, Dc, T1, dHc, ld, Dx, T2, nw, ld);
        __syncthreads();
        for (int e = tid; e < nn; e += blockDim.x) {
            const int i = e % nw, m = e / nw;
            if (i == m) continue;
            double2 num = cadd(cadd(ddHxc[i + ld * m], T1[i + ld * m]), T2[i + ld * m]);
            num = csub(num, cadd(cscale(Dc[i + ld * m], dEx[m]), cscale(Dx[i + ld * m], sdEc[m])));
            out[i + ld * m] = cscale(num, 1.0 / (sE[m] - sE[i]));
        }
        for (int i = tid; i < nw; i += blockDim.x) {
            double2 cxc = make_double2(0.0, 0.0), ccx = make_double2(0.0, 0.0), dd = make_double2(0.0, 0.0);
            for (int l = 0; l < nw; ++l) {
                cxc = cadd(cxc, csub(cmul(Dc[i + ld * l], Ax[l + ld * i]), cmul(Ax[i + ld * l], Dc[l + ld * i])));
                ccx = cadd(ccx, csub(cmul(Dx[i + ld * l], Ac[l + ld * i]), cmul(Ac[i + ld * l], Dx[l + ld * i])));
            }
            for (int l = 0; l < nw; ++l)
                dd = cadd(dd, cadd(cmul(Dc[i + ld * l], Dx[l + ld * i]), cmul(Dx[i + ld * l], Dc[l + ld * i])));
            const double jet = 0.5 * (Axc[i + ld * i].x - cxc.x + Acx_diag[i].x - ccx.x);
            out[i + ld * i] = make_double2(0.5 * dd.x, jet);
        }
        __syncthreads();
    };

    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x, ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *xw = p.xw + b * p.xw_stride;
        for (int e = tid; e < nn; e += blockDim.x) U[(e % nw) + ld * (e / nw)] = p.U[b * nn + e];
        for (int i = tid; i < nw; i += blockDim.x) sE[i] = p.E[b * nw + i];
        __syncthreads();
        const double wk = p.weights ? p.weights[b] * p.scale : p.scale;
        for (int it = 0; it < p.n_items; ++it) {
            const int a = p.item_a[it], bb = p.item_b[it], c = p.item_c[it];
            auto sym = [](int x, int y) { return x <= y ? x * 3 + y : y * 3 + x; };
            rotate2(xw, p.ch_dH[a], p.ch_dH[bb], dHa, dHb);
            rotate2(xw, p.ch_dH[c], p.ch_ddH[sym(a, c)], dHc, ddHac);
            rotate2(xw, p.ch_ddH[sym(bb, c)], p.ch_A[a], ddHbc, Aa);
            rotate2(xw, p.ch_A[bb], p.ch_A[c], Ab, Ac);
            rotate2(xw, p.ch_dA[a * 3 + c], p.ch_dA[bb * 3 + c], Aac, Abc);  // d_c A_a, d_c A_b
            rotate(xw, p.ch_dA[bb * 3 + a], p.ch_dA[a * 3 + bb], Om);         // d_a A_b - d_b A_a
            rotate_diag(xw, p.ch_dA[c * 3 + a], -1, sAca);                   // d_a A_c
            rotate_diag(xw, p.ch_dA[c * 3 + bb], -1, sAcb);                  // d_b A_c
            rotate_diag(xw, p.ch_ddA[bb * 9 + sym(a, c)], p.ch_ddA[a * 9 + sym(bb, c)], sOmc);   // d_a d_c A_b - d_b d_c A_a
            for (int i = tid; i < nw; i += blockDim.x) {
                sdEa[i] = dHa[i + ld * i].x;
                sdEb[i] = dHb[i + ld * i].x;
                sdEc[i] = dHc[i + ld * i].x;
            }
            first(dHa, Aa, Da);
            first(dHb, Ab, Db);
            first(dHc, Ac, Dc);
            __syncthreads();
            second(dHa, ddHac, Aa, Da, sdEa, Aac, sAca, Dac);
            second(dHb, ddHbc, Ab, Db, sdEb, Abc, sAcb, Dbc);
            // Terms with at most two factors.
            for (int n = tid; n < nw; n += blockDim.x) {
                double t = sOmc[n].x;                                                    // omega derivative
                t += diag2(Dbc, Aa, n).x - diag2(Aac, Db, n).x - diag2(Dac, Ab, n).x + diag2(Abc, Da, n).x;   // second
                t += diag2(Db, Aac, n).x - diag2(Aa, Dbc, n).x - diag2(Da, Abc, n).x + diag2(Ab, Dac, n).x;   // first
                t += -diag2(Dc, Om, n).x + diag2(Om, Dc, n).x;                           // omega transport
                t += diag2(Da, Dbc, n).y + diag2(Dac, Db, n).y - diag2(Db, Dac, n).y - diag2(Dbc, Da, n).y;   // pure D
                sTot[n] = t;
            }
            __syncthreads();
            // Triples through one full product each, two products per paired DMMA pass (into T1, T2).
            const double2 *L[8] = {Dc, Db, Dc, Da, Dc, Dc, Db, Da};
            const double2 *R[8] = {Db, Dc, Da, Dc, Aa, Ab, Aa, Ab};
            #pragma unroll
            for (int q = 0; q < 8; q += 2) {
                dmma_product_pair<0>(L[q], ld, R[q], T1, L[q + 1], ld, R[q + 1], T2, nw, ld);
                __syncthreads();
                for (int n = tid; n < nw; n += blockDim.x) {
                    double t;
                    switch (q) {
                    case 0:   // Dc Db, Db Dc: second, pure D
                        t = -diag2(T1, Aa, n).x + diag2(T1, Da, n).y - diag2(T2, Aa, n).x + diag2(T2, Da, n).y;
                        break;
                    case 2:   // Dc Da, Da Dc
                        t = diag2(T1, Ab, n).x - diag2(T1, Db, n).y + diag2(T2, Ab, n).x - diag2(T2, Db, n).y;
                        break;
                    case 4:   // Dc Aa, Dc Ab: mixed
                        t = diag2(T1, Db, n).x - diag2(T2, Da, n).x;
                        break;
                    default:  // Db Aa, Da Ab
                        t = diag2(T1, Dc, n).x - diag2(T2, Dc, n).x;
                        break;
                    }
                    sTot[n] += t;
                }
                __syncthreads();
            }
            // D[mu] = sum_n f(E_n; mu, T) d_c Omega_n.
            for (int im = tid; im < p.nmu; im += blockDim.x) {
                const double mu = p.mus[im];
                double value = 0.0;
                for (int n = 0; n < nw; ++n) value += response_occ(sE[n], mu, p.temperature) * sTot[n];
                const int64_t idx = p.item_out[it] + im;
                if (p.mode == 0) {
                    double *acc = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
                    neumaier_add(acc[0], acc[2], value * wk);
                } else {
                    const int64_t row = p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : b);
                    p.out_points[row * p.vc + idx] = make_double2(value * p.scale, 0.0);
                }
            }
            __syncthreads();
        }
    }
}
