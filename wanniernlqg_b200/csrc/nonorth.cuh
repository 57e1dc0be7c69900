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
