// nonorth.cuh - metric (nonorthogonal) k-point geometry for the conventional currents, FP64.
//
// Restates _nonorthogonal_geometry (NonorthogonalMatrixElements.jl:560-817) on the device for
// models with an overlap S(R).  Inputs per k: the localized channels from the Fourier step
// (dH_a, dS_a, r_a and, per requested (position p, derivative d) pair, d2H_pd, d2S_pd, dr_pd) and
// the S-orthonormal canonical eigenvectors C with energies E from the generalised eigensolve.
// Per axis a (gap = E_m - E_l, f = gap/(gap^2 + eta^2) or 1/gap when eta = 0):
//   dh_a = C^H dH_a C,  ds_a = C^H dS_a C,  B_a = C^H (r_a + i dS_a) C,
//   N_a[l,m] = dh_a[l,m] - (E_l + E_m) ds_a[l,m] / 2,
//   D_a[l,m] = -ds_a[l,m]/2 + N_a[l,m] f (l != m),  D_a[l,l] = -ds_a[l,l]/2 + i Re B_a[l,l],
//   r_a = i D_a + B_a (Berry connection),  v_a[l] = Re(dh_a[l,l] - E_l ds_a[l,l]).
// Per pair (p, d), with hd = D_d^H dh_p + dh_p D_d + C^H d2H_pd C, sd likewise with dS and
// bd = D_d^H B_p + B_p D_d + C^H (dr_pd + i d2S_pd) C, for l != m:
//   nd = hd - (E_l + E_m) sd / 2 - (v_d[l] + v_d[m]) ds_p / 2,
//   dd = -sd/2 + nd f + N_p fp (v_d[m] - v_d[l]),  fp = (eta^2 - gap^2)/(gap^2 + eta^2)^2 (-1/gap^2),
//   G_pd = i dd + bd - i (r_d[l,l] - r_d[m,m]) r_p[l,m].
// Outputs per k: r (3 axes), v (3 axes) and G for the listed pairs; the response kernel consumes
// them in place of its orthogonal geometry (shift current from G and r, injection current from
// v and r).  One CTA per contiguous range of the batch; every matrix sits in the CTA's global
// working set (L1/L2-resident).
#pragma once
#include "common.cuh"
#include "response.cuh"

#define NG_MAX_PAIRS 9

struct NonorthParams {
    int nw, ld;
    int64_t batch;
    int64_t xw_stride;
    const double2 *xw;
    const double *E;
    const double2 *U;
    int ch_dH[3], ch_dS[3], ch_A[3];
    int npairs;
    int pair_p[NG_MAX_PAIRS], pair_d[NG_MAX_PAIRS];
    int ch_ddH[NG_MAX_PAIRS], ch_ddS[NG_MAX_PAIRS], ch_dA[NG_MAX_PAIRS];
    double eta;
    double2 *r_out;      // [batch][3][nn]
    double *v_out;       // [batch][3][nw]
    double2 *g_out;      // [batch][npairs][nn]
    unsigned char *ws;   // per-CTA working set
    int64_t ws_stride;
};

struct NonorthWs {
    // U, T1, T2, dh[3], ds[3], B[3], D[3], r[3], hd, sd, bd: 20 matrices of nw x (nw + 1).
    static __host__ __device__ int64_t bytes(int nw) { return 20 * (int64_t)nw * (nw + 1) * (int64_t)sizeof(double2) + 64; }
};

// dst = C^H (X + i Y) C for Wannier-gauge channels X, Y in global memory (Y may be null).
WNLQG_D void ng_rotate(const double2 *__restrict__ X, const double2 *__restrict__ Y, double2 *T1, double2 *T2,
                       const double2 *U, double2 *dst, int nw, int ld) {
    const int nn = nw * nw;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        double2 v = X[e];
        if (Y) v = cadd(v, cmuli(Y[e]));
        T1[(e % nw) + ld * (e / nw)] = v;
    }
    __syncthreads();
    mm_xy(T1, U, T2, nw, ld);
    __syncthreads();
    mm_xhy(U, T2, dst, nw, ld);
    __syncthreads();
}

__global__ void __launch_bounds__(256) nonorth_geometry_kernel(NonorthParams p) {
    const int nw = p.nw, ld = p.ld, nn = nw * nw;
    const int64_t mat = (int64_t)nw * ld;
    double2 *base = reinterpret_cast<double2 *>(p.ws + (int64_t)blockIdx.x * p.ws_stride);
    double2 *U = base, *T1 = base + mat, *T2 = base + 2 * mat;
    double2 *dh = base + 3 * mat, *ds = base + 6 * mat, *B = base + 9 * mat, *D = base + 12 * mat;
    double2 *r = base + 15 * mat, *hd = base + 18 * mat, *sd = base + 19 * mat;
    double2 *bd = T2;   // reuses T2 once the rotations of a pair are done (see below)
    __shared__ double sE[128];
    __shared__ double sv[3 * 128];
    const double eta = p.eta;
    auto fgap = [&](double g) { return eta == 0.0 ? 1.0 / g : g / (g * g + eta * eta); };
    auto fpgap = [&](double g) {
        const double q = g * g + eta * eta;
        return eta == 0.0 ? -1.0 / (g * g) : (eta * eta - g * g) / (q * q);
    };
    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x;
    const int64_t ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *xw = p.xw + b * p.xw_stride;
        for (int e = threadIdx.x; e < nn; e += blockDim.x) U[(e % nw) + ld * (e / nw)] = p.U[b * nn + e];
        for (int i = threadIdx.x; i < nw; i += blockDim.x) sE[i] = p.E[b * nw + i];
        __syncthreads();
        for (int a = 0; a < 3; ++a) {
            double2 *dha = dh + a * mat, *dsa = ds + a * mat, *Ba = B + a * mat, *Da = D + a * mat, *ra = r + a * mat;
            ng_rotate(xw + (int64_t)p.ch_dH[a] * nn, nullptr, T1, T2, U, dha, nw, ld);
            ng_rotate(xw + (int64_t)p.ch_dS[a] * nn, nullptr, T1, T2, U, dsa, nw, ld);
            ng_rotate(xw + (int64_t)p.ch_A[a] * nn, xw + (int64_t)p.ch_dS[a] * nn, T1, T2, U, Ba, nw, ld);
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int l = e % nw, m = e / nw, o = l + ld * m;
                double2 dv;
                if (l == m) {
                    dv = make_double2(-0.5 * dsa[o].x, -0.5 * dsa[o].y + Ba[o].x);
                } else {
                    const double2 num = csub(dha[o], cscale(dsa[o], 0.5 * (sE[l] + sE[m])));
                    dv = cadd(cscale(dsa[o], -0.5), cscale(num, fgap(sE[m] - sE[l])));
                }
                Da[o] = dv;
                const double2 rv = cadd(cmuli(dv), Ba[o]);
                ra[o] = rv;
                p.r_out[(b * 3 + a) * nn + e] = rv;
            }
            for (int l = threadIdx.x; l < nw; l += blockDim.x) {
                const int o = l + ld * l;
                const double v = dha[o].x - sE[l] * dsa[o].x;
                sv[a * nw + l] = v;
                p.v_out[(b * 3 + a) * nw + l] = v;
            }
            __syncthreads();
        }
        for (int g = 0; g < p.npairs; ++g) {
            const int pp = p.pair_p[g], dd = p.pair_d[g];
            const double2 *Dd = D + dd * mat, *dhp = dh + pp * mat, *dsp = ds + pp * mat, *Bp = B + pp * mat;
            const double2 *rp = r + pp * mat, *rd = r + dd * mat;
            // hd = C^H d2H C + D^H dh + dh D, sd likewise; T1/T2 serve the rotations.
            ng_rotate(xw + (int64_t)p.ch_ddH[g] * nn, nullptr, T1, T2, U, hd, nw, ld);
            ng_rotate(xw + (int64_t)p.ch_ddS[g] * nn, nullptr, T1, T2, U, sd, nw, ld);
            ng_rotate(xw + (int64_t)p.ch_dA[g] * nn, xw + (int64_t)p.ch_ddS[g] * nn, T1, T2, U, T1, nw, ld);
            // T1 = C^H (dr + i d2S) C; accumulate the D products elementwise per output.
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int l = e % nw, m = e / nw, o = l + ld * m;
                double2 h = hd[o], s = sd[o], q = T1[o];
                for (int k = 0; k < nw; ++k) {
                    const double2 dkl = Dd[k + ld * l], dkm = Dd[k + ld * m];
                    h = cfmaconj(dkl, dhp[k + ld * m], h);
                    h = cfma(dhp[l + ld * k], dkm, h);
                    s = cfmaconj(dkl, dsp[k + ld * m], s);
                    s = cfma(dsp[l + ld * k], dkm, s);
                    q = cfmaconj(dkl, Bp[k + ld * m], q);
                    q = cfma(Bp[l + ld * k], dkm, q);
                }
                bd[o] = q;   // bd aliases T2, free after the rotations
                hd[o] = h;
                sd[o] = s;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int l = e % nw, m = e / nw, o = l + ld * m;
                double2 gv = make_double2(0.0, 0.0);
                if (l != m) {
                    const double gap = sE[m] - sE[l];
                    const double vl = sv[dd * nw + l], vm = sv[dd * nw + m];
                    const double2 num = csub(dhp[o], cscale(dsp[o], 0.5 * (sE[l] + sE[m])));
                    const double2 nd = csub(csub(hd[o], cscale(sd[o], 0.5 * (sE[l] + sE[m]))), cscale(dsp[o], 0.5 * (vl + vm)));
                    const double2 dv = cadd(cadd(cscale(sd[o], -0.5), cscale(nd, fgap(gap))), cscale(num, fpgap(gap) * (vm - vl)));
                    const double2 diagdiff = csub(rd[l + ld * l], rd[m + ld * m]);
                    gv = csub(cadd(cmuli(dv), bd[o]), cmuli(cmul(diagdiff, rp[o])));
                }
                p.g_out[(b * p.npairs + g) * nn + e] = gv;
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Metric (nonorthogonal) second-harmonic inputs per k-point, FP64.
//
// Restates, for the SHG of models with an overlap S(R):
//   the normalized local source jets of _prepare_nonorthogonal_optical_cutoff!
//     (NonorthogonalOpticalCutoffVertices.jl:67-186): with k_a = C^H dH_a C, g_a = C^H dS_a C,
//     raw_a = C^H (r_a + i dS_a) C and z_ab = -C^H d2S_ab C / 2 + 3 (g_a g_b + g_b g_a) / 8,
//       V_a = k_a - (E_i + E_j) g_a / 2,  A_a = raw_a - i g_a / 2,
//       W_ab = C^H d2H_ab C - (g_a k_b + k_b g_a + g_b k_a + k_a g_b) / 2
//              + (g_a E g_b + g_b E g_a) / 4 + (E_i + E_j) z_ab,
//       dA_ab = C^H (dr_ab + i d2S_ab) C - (g_b raw_a + raw_a g_b) / 2 + i (z_ab - g_b g_a / 4);
//   the metric Berry connection r_a = i D_a + raw_a (r_eta of metric SHG,
//     NonorthogonalMatrixElements.jl:1088-1139), D_a the metric eigenvector derivative;
//   the metric energy Hessians (_nonorthogonal_geometry, NonorthogonalMatrixElements.jl:660-727)
//     esd[l, a, b] = Re(hd_ll - E_l sd_ll - v_l^b g_a,ll), hd = D_b^H k_a + k_a D_b + C^H d2H_ab C,
//     sd likewise from g_a and d2S_ab;
//   the isolated-band curvature (isolated_band_curvature, NonorthogonalMatrixElements.jl:1141-1185)
//     with the band-frame ambient metric curvature (_nonorthogonal_ambient_curvature, :819-878),
//     whose diagonal is (B_b;a - g_a raw_b - B_a;b + g_b raw_a - i [raw_a, raw_b])_nn with
//     B_a;b = C^H (dr_ab + i d2S_ab) C (S^-1 = C C^H for the S-orthonormal eigenvectors).
// Channel index [a * 3 + b]: position / first axis a, derivative / second axis b.
// Outputs per k: src[27][nn] (V 0-2, A 3-5, W 6-14, dA 15-23, r 24-26, column-major nw x nw) and
// diag[18][nw] (esd at (a * 3 + b) nw + l, curvature at (9 + a * 3 + b) nw + l).
// ---------------------------------------------------------------------------------------------
struct MetricShgParams {
    int nw, ld;
    int64_t batch;
    int64_t xw_stride;
    const double2 *xw;
    const double *E;
    const double2 *U;
    int ch_dH[3], ch_dS[3], ch_A[3], ch_ddH[9], ch_ddS[9], ch_dA[9];
    double eta;                 // geometry width (the task's denominator regularization)
    double2 *src;
    double *diag;
    unsigned char *ws;
    int64_t ws_stride;
};

struct MetricShgWs {
    // U, T1, T2, k[3], g[3], raw[3], D[3], Z, P, Q, R2H, R2S, RB: 21 matrices of nw x (nw + 1).
    static __host__ __device__ int64_t bytes(int nw) { return 21 * (int64_t)nw * (nw + 1) * (int64_t)sizeof(double2) + 64; }
    static __host__ __device__ int64_t src_entries(int nw) { return 27 * (int64_t)nw * nw; }
    static __host__ __device__ int64_t diag_entries(int nw) { return 18 * (int64_t)nw; }
};

__global__ void __launch_bounds__(256) metric_shg_kernel(MetricShgParams p) {
    const int nw = p.nw, ld = p.ld, nn = nw * nw;
    const int64_t mat = (int64_t)nw * ld;
    double2 *base = reinterpret_cast<double2 *>(p.ws + (int64_t)blockIdx.x * p.ws_stride);
    double2 *U = base, *T1 = base + mat, *T2 = base + 2 * mat;
    double2 *K = base + 3 * mat, *Gm = base + 6 * mat, *Rw = base + 9 * mat, *D = base + 12 * mat;
    double2 *Z = base + 15 * mat, *P = base + 16 * mat, *Q = base + 17 * mat;
    double2 *R2H = base + 18 * mat, *R2S = base + 19 * mat, *RB = base + 20 * mat;
    __shared__ double sE[128];
    __shared__ double sv[3 * 128];
    __shared__ double2 rbd[9 * 128];
    __shared__ double hdiag[9 * 128];   // diagonal of C^H d2H_ab C (symmetric in a, b)
    const double eta = p.eta;
    auto fgap = [&](double g) { return eta == 0.0 ? 1.0 / g : g / (g * g + eta * eta); };
    auto at = [&](double2 *M, int a) { return M + a * mat; };
    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x;
    const int64_t ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *xw = p.xw + b * p.xw_stride;
        double2 *src = p.src + b * MetricShgWs::src_entries(nw);
        double *dg = p.diag + b * MetricShgWs::diag_entries(nw);
        for (int e = threadIdx.x; e < nn; e += blockDim.x) U[(e % nw) + ld * (e / nw)] = p.U[b * nn + e];
        for (int i = threadIdx.x; i < nw; i += blockDim.x) sE[i] = p.E[b * nw + i];
        __syncthreads();
        for (int a = 0; a < 3; ++a) {
            ng_rotate(xw + (int64_t)p.ch_dH[a] * nn, nullptr, T1, T2, U, at(K, a), nw, ld);
            ng_rotate(xw + (int64_t)p.ch_dS[a] * nn, nullptr, T1, T2, U, at(Gm, a), nw, ld);
            ng_rotate(xw + (int64_t)p.ch_A[a] * nn, xw + (int64_t)p.ch_dS[a] * nn, T1, T2, U, at(Rw, a), nw, ld);
            const double2 *ka = at(K, a), *ga = at(Gm, a), *ra = at(Rw, a);
            double2 *Da = at(D, a);
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int l = e % nw, m = e / nw, o = l + ld * m;
                const double2 num = csub(ka[o], cscale(ga[o], 0.5 * (sE[l] + sE[m])));
                const double2 dv = l == m ? make_double2(-0.5 * ga[o].x, -0.5 * ga[o].y + ra[o].x)
                                          : cadd(cscale(ga[o], -0.5), cscale(num, fgap(sE[m] - sE[l])));
                Da[o] = dv;
                src[(int64_t)(0 + a) * nn + e] = num;
                src[(int64_t)(3 + a) * nn + e] = csub(ra[o], cmuli(cscale(ga[o], 0.5)));
                src[(int64_t)(24 + a) * nn + e] = cadd(cmuli(dv), ra[o]);
            }
            for (int l = threadIdx.x; l < nw; l += blockDim.x)
                sv[a * nw + l] = ka[l + ld * l].x - sE[l] * ga[l + ld * l].x;
            __syncthreads();
        }
        for (int ab = 0; ab < 9; ++ab) {
            const int a = ab / 3, bb = ab % 3;
            const double2 *ga = at(Gm, a), *gb = at(Gm, bb), *ka = at(K, a), *kbm = at(K, bb);
            const double2 *ra = at(Rw, a), *Db = at(D, bb);
            // W_ab = W_ba (d2H, d2S and z are symmetric): for a > b only dA and the diagonals are new.
            const bool wnew = a <= bb;
            if (wnew) ng_rotate(xw + (int64_t)p.ch_ddH[ab] * nn, nullptr, T1, T2, U, R2H, nw, ld);
            ng_rotate(xw + (int64_t)p.ch_ddS[ab] * nn, nullptr, T1, T2, U, R2S, nw, ld);
            ng_rotate(xw + (int64_t)p.ch_dA[ab] * nn, xw + (int64_t)p.ch_ddS[ab] * nn, T1, T2, U, RB, nw, ld);
            // Energy Hessian diagonal and the B_a;b diagonal (before W and dA overwrite R2H, RB).
            for (int l = threadIdx.x; l < nw; l += blockDim.x) {
                if (wnew) hdiag[ab * 128 + l] = R2H[l + ld * l].x;
                double2 hd = make_double2(wnew ? R2H[l + ld * l].x : hdiag[(bb * 3 + a) * 128 + l], 0.0);
                double2 sd = R2S[l + ld * l];
                for (int q = 0; q < nw; ++q) {
                    const double2 dql = Db[q + ld * l];
                    hd = cfma(ka[l + ld * q], dql, cfmaconj(dql, ka[q + ld * l], hd));
                    sd = cfma(ga[l + ld * q], dql, cfmaconj(dql, ga[q + ld * l], sd));
                }
                dg[ab * nw + l] = hd.x - sE[l] * sd.x - sv[bb * nw + l] * ga[l + ld * l].x;
                rbd[ab * 128 + l] = RB[l + ld * l];
            }
            // z = -C^H d2S C / 2 + 3 (g_a g_b + g_b g_a) / 8 into Z; Q = g_b g_a kept for dA.
            mm_xy(ga, gb, P, nw, ld);
            mm_xy(gb, ga, Q, nw, ld);
            __syncthreads();
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int l = e % nw, m = e / nw, o = l + ld * m;
                const double2 z = cadd(cscale(R2S[o], -0.5), cscale(cadd(P[o], Q[o]), 0.375));
                Z[o] = z;
                // W starts as C^H d2H C + (E_l + E_m) z; dA as C^H (dr + i d2S) C + i (z - g_b g_a / 4).
                if (wnew) R2H[o] = cadd(R2H[o], cscale(z, sE[l] + sE[m]));
                RB[o] = cadd(RB[o], cmuli(csub(z, cscale(Q[o], 0.25))));
            }
            __syncthreads();
            // W -= (g_a k_b + k_b g_a + g_b k_a + k_a g_b) / 2.
            const double2 *pairs[4][2] = {{ga, kbm}, {kbm, ga}, {gb, ka}, {ka, gb}};
            for (int t = 0; t < (wnew ? 4 : 0); ++t) {
                mm_xy(pairs[t][0], pairs[t][1], P, nw, ld);
                __syncthreads();
                for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                    const int o = (e % nw) + ld * (e / nw);
                    R2H[o] = csub(R2H[o], cscale(P[o], 0.5));
                }
                __syncthreads();
            }
            // W += (g_a (E g_b) + g_b (E g_a)) / 4.
            for (int t = 0; t < (wnew ? 2 : 0); ++t) {
                const double2 *left = t == 0 ? ga : gb, *right = t == 0 ? gb : ga;
                for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                    const int l = e % nw, o = l + ld * (e / nw);
                    T1[o] = cscale(right[o], sE[l]);
                }
                __syncthreads();
                mm_xy(left, T1, P, nw, ld);
                __syncthreads();
                for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                    const int o = (e % nw) + ld * (e / nw);
                    R2H[o] = cadd(R2H[o], cscale(P[o], 0.25));
                }
                __syncthreads();
            }
            // dA -= (g_b raw_a + raw_a g_b) / 2.
            mm_xy(gb, ra, P, nw, ld);
            mm_xy(ra, gb, Q, nw, ld);
            __syncthreads();
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int o = (e % nw) + ld * (e / nw);
                src[(int64_t)(6 + ab) * nn + e] = wnew ? R2H[o] : src[(int64_t)(6 + bb * 3 + a) * nn + e];
                src[(int64_t)(15 + ab) * nn + e] = csub(RB[o], cscale(cadd(P[o], Q[o]), 0.5));
            }
            __syncthreads();
        }
        // Isolated-band curvature, one (band, a, b) per thread.
        for (int it = threadIdx.x; it < nw * 9; it += blockDim.x) {
            const int l = it / 9, ab = it % 9, a = ab / 3, bb = ab % 3;
            double value = 0.0;
            if (a != bb) {
                const double2 *ga = at(Gm, a), *gb = at(Gm, bb), *ra = at(Rw, a), *rb = at(Rw, bb);
                const double2 *ka = at(K, a), *kbm = at(K, bb);
                double2 band = csub(rbd[(bb * 3 + a) * 128 + l], rbd[(a * 3 + bb) * 128 + l]);
                for (int q = 0; q < nw; ++q) {
                    band = csub(band, cmul(ga[l + ld * q], rb[q + ld * l]));
                    band = cadd(band, cmul(gb[l + ld * q], ra[q + ld * l]));
                    band = csub(band, cmuli(csub(cmul(ra[l + ld * q], rb[q + ld * l]), cmul(rb[l + ld * q], ra[q + ld * l]))));
                }
                value = band.x;
                for (int m = 0; m < nw; ++m) {
                    if (m == l) continue;
                    const double inv = fabs(sE[m] - sE[l]) < 1.0e-7 ? 0.0 : 1.0 / (sE[m] - sE[l]);
                    const double rinv = fabs(sE[l] - sE[m]) < 1.0e-7 ? 0.0 : 1.0 / (sE[l] - sE[m]);
                    const double avg = 0.5 * (sE[l] + sE[m]);
                    auto rowcol = [&](const double2 *r, const double2 *k, double2 &row, double2 &col) {
                        const double2 fw = r[l + ld * m], rv = r[m + ld * l];
                        const double2 mf = cmulmi(csub(fw, cconj(rv))), mr = cmulmi(csub(rv, cconj(fw)));
                        const double2 ff = cscale(cadd(fw, cconj(rv)), 0.5), fr = cscale(cadd(rv, cconj(fw)), 0.5);
                        const double2 nf = csub(k[l + ld * m], cscale(mf, avg)), nr = csub(k[m + ld * l], cscale(mr, avg));
                        row = inv == 0.0 ? ff : cadd(ff, cmuli(cscale(nf, inv)));
                        col = rinv == 0.0 ? fr : cadd(fr, cmuli(cscale(nr, rinv)));
                    };
                    double2 row_a, col_a, row_b, col_b;
                    rowcol(ra, ka, row_a, col_a);
                    rowcol(rb, kbm, row_b, col_b);
                    value -= 2.0 * cmul(row_a, col_b).y;
                }
            }
            dg[(9 + ab) * nw + l] = value;
        }
        __syncthreads();
    }
}
