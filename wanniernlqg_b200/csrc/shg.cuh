// shg.cuh - second-harmonic generation per k-point: cutoff optical vertices, the seven SHG terms
// and their deterministic accumulation.  FP64 throughout (both precision modes).
//
// Reference routines restated here (file:line in the WannierNLQG project):
//   bare / regularised inverse, C weight   PositionVertexRegularization.jl:7-50
//   r0, r_eta, Gcut (cutoff derivative)    optical_position_vertices!, OpticalPositionDerivatives.jl:13-91
//   delta, principal value, resonance      SecondHarmonicKernels.jl:86-98
//   occupations                            second_harmonic_occupation, SecondHarmonicKernels.jl:101-105
//   five pair terms + three-band sums      second_harmonic_response!, SecondHarmonicKernels.jl:115-236
//   one-band terms (BCD, semiclassical)    second_harmonic_one_band!, SecondHarmonicKernels.jl:245-294
//
// One CTA per k-point (a fixed contiguous range of the batch per CTA).  Stages per k:
//   1. U, energies, occupations and the nw x nw energy tables (bare inverse, regularised inverse,
//      C weight) into shared memory; dH_a and A_a rotated to the Hamiltonian gauge (shared).
//   2. For each of the nine (a, b): U'ddH_ab U and U'dA_ab U (shared, transient), their diagonals
//      kept for the one-band terms, and G^{ab}_{nm} for all n != m written to the CTA's global
//      scratch (nine nw x nw matrices).
//   3. Active pairs (|f_n - f_m| >= 1e-10) are compacted; per pair and component the seven
//      k-local coefficients (first ... fifth, the two three-band sums) go to global scratch.
//   4. Frequency contraction: a thread owns one photon energy and SHG_CB components and streams
//      the pair list once, evaluating the three resonance kernels per pair; the five pair terms of
//      both quantities follow from nine accumulators per component plus three frequency-independent
//      sums.
//   5. T > 1e-7 K: one-band terms from the band curvature and Hessian near the Fermi level.
// Output per k: value[out + w + nom * (comp + nc * (term + 7 * quantity))].
#pragma once
#include "common.cuh"
#include "response.cuh"

#define SHG_MAX_COMPONENTS 81
#define SHG_CB 3                         // components per thread in the frequency contraction
#define SHG_KB_EV 8.617333262145e-5      // RESPONSE_KB_EV of the reference's SHG occupations

struct ShgParams {
    int nw, ld;
    int64_t batch;
    int64_t xw_stride;
    const double2 *xw;
    const double *E;
    const double2 *U;
    int ch_dH[3], ch_A[3], ch_ddH[9], ch_dA[9];   // ch_dA[p*3+d]: position p, derivative d
    int nc;
    int comp[SHG_MAX_COMPONENTS][3];
    int64_t out;
    int nom;
    const double *omegas;
    double mu, T, width, low_width, eta, degeneracy;
    int gaussian, eta_correction;
    double scale;
    const double *weights;
    int mode;
    int64_t vc;
    double *partials;
    double2 *out_points;
    int64_t point_offset;
    const int *out_perm;         // mode 1: batch entry b is written to row out_perm[b]; nullptr: row b
    double2 *scratch;            // per CTA: G[9][nn] | coef[nn][nc][7] | pinfo[nn] (fo, inv, diff, 0)
    int64_t scratch_stride;      // double2 entries per CTA
    unsigned char *gscratch;     // per-CTA matrix working set in global memory (large nw); nullptr: shared
    int64_t gscratch_stride;
    // Metric (nonorthogonal) models: V, A, d2H, dA come as the normalized source jets of
    // metric_shg_kernel (m_src, [27][nn] per point), the vertices take the geometry width
    // vertex_eta, r_eta is the metric Berry connection, and the one-band Hessians and
    // isolated-band curvatures are the metric ones (m_diag, [18][nw] per point).
    int metric;
    double vertex_eta;
    const double2 *m_src;
    const double *m_diag;
};

struct ShgSmem {
    size_t U, T1, T2, X, V, A, I0, Rg, Wt, E, f, dAd, ddHd, curv, plist, S, red, total;
    static __host__ __device__ ShgSmem layout(int nw, int nc) {
        ShgSmem s;
        const int ld = nw + 1;
        const size_t mat = (size_t)nw * ld * sizeof(double2);
        const size_t nn = (size_t)nw * nw;
        size_t off = 0;
        auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 15) & ~(size_t)15; return o; };
        s.U = take(mat);
        s.T1 = take(mat);
        s.T2 = take(mat);
        s.X = take(mat);
        s.V = take(3 * mat);
        s.A = take(3 * mat);
        s.I0 = take(nn * sizeof(double));
        s.Rg = take(nn * sizeof(double));
        s.Wt = take(nn * sizeof(double));
        s.E = take(nw * sizeof(double));
        s.f = take(nw * sizeof(double));
        s.dAd = take(9 * (size_t)nw * sizeof(double2));
        s.ddHd = take(9 * (size_t)nw * sizeof(double2));
        s.curv = take(9 * (size_t)nw * sizeof(double));
        s.plist = take(nn * sizeof(int));
        s.S = take(3 * (size_t)(nc > 0 ? nc : 1) * sizeof(double2));
        s.red = take(64 * sizeof(double) + 64 * sizeof(int));
        s.total = off;
        return s;
    }
    static __host__ __device__ int64_t scratch_entries(int nw, int nc) {
        const int64_t nn = (int64_t)nw * nw;
        return 9 * nn + nn * nc * 7 + 2 * nn;
    }
};

// bare_energy_inverse (PositionVertexRegularization.jl:7-8).
WNLQG_D double shg_bare_inverse(double d) { return fabs(d) < 1.0e-7 ? 0.0 : 1.0 / d; }

// regularized_energy_weight (PositionVertexRegularization.jl:37-50): eta^2 / (d^2 + eta^2).
WNLQG_D double shg_weight(double d, double eta) {
    const double w2 = eta * eta, den = d * d + w2;
    if (isfinite(den) && den != 0.0 && w2 != 0.0) return w2 / den;
    if (!(isfinite(d) && isfinite(eta) && eta > 0)) return w2 / den;
    const double sc = fmax(fabs(d), eta), sd = d / sc, sw = eta / sc;
    return sw * sw / (sd * sd + sw * sw);
}

WNLQG_D double shg_principal(double e, double w) { return e / (e * e + w * w); }

WNLQG_D double shg_delta(double e, double w, int gaussian) {
    const double x = e / w;
    return gaussian ? exp(-x * x) / (1.7724538509055160273 * w) : 1.0 / (WNLQG_PI * w * (1.0 + x * x));
}

// second_harmonic_resonance: PV(1/x) + i pi delta(x).
template <bool GAUSS>
WNLQG_D double2 shg_resonance(double x, double w, double w2, double gpref) {
    const double r = 1.0 / (x * x + w2);
    if (GAUSS) {
        const double y = x / w;
        return make_double2(x * r, gpref * exp(-y * y));   // gpref = sqrt(pi) / w
    }
    return make_double2(x * r, w * r);                      // pi * lorentzian = w / (x^2 + w^2)
}

WNLQG_D double shg_occupation(double e, double mu, double T) {
    if (T <= 1.0e-7) return e <= mu ? 1.0 : 0.0;
    const double x = (e - mu) / (SHG_KB_EV * T);
    return x >= 0 ? exp(-x) / (1.0 + exp(-x)) : 1.0 / (1.0 + exp(x));
}

WNLQG_D void shg_emit(const ShgParams &p, int64_t b, int64_t idx, double2 v, double wk) {
    if (p.mode == 0) {
        double *a4 = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
        neumaier_add(a4[0], a4[2], v.x * wk);
        neumaier_add(a4[1], a4[3], v.y * wk);
    } else {
        p.out_points[(p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : b)) * p.vc + idx] = cscale(v, p.scale);
    }
}

// Frequency contraction for one thread: photon energy `om`, components c0 .. c0+SHG_CB-1.
template <bool GAUSS>
WNLQG_D void shg_contract(const ShgParams &p, const double2 *__restrict__ coef, const double *__restrict__ pinfo,
                          int npairs, double om, int c0, double2 (*acc)[9]) {
    const double w = p.width, w2 = w * w, gpref = 1.7724538509055160273 / w;
    const int nc = p.nc;
    for (int q = 0; q < npairs; ++q) {
        const double fo = pinfo[4 * q], inv = pinfo[4 * q + 1], diff = pinfo[4 * q + 2];
        const double2 d1 = shg_resonance<GAUSS>(diff - om, w, w2, gpref);
        const double2 d2 = shg_resonance<GAUSS>(diff - 2.0 * om, w, w2, gpref);
        const double2 dn = shg_resonance<GAUSS>(-diff - om, w, w2, gpref);
        const double fi = fo * inv, fd = fo * diff;
#pragma unroll
        for (int j = 0; j < SHG_CB; ++j) {
            const int c = c0 + j;
            if (c >= nc) break;
            const double2 *cf = coef + ((int64_t)q * nc + c) * 7;
            const double2 first = cf[0], second = cf[1], third = cf[2], fourth = cf[3], fifth = cf[4];
            const double2 tf = cf[5], to = cf[6];
            const double2 t1 = cmul(first, d2), t2 = cmul(second, d1);
            const double2 t3 = cmul(third, d1), t4 = cmul(third, d2);
            const double2 t5 = cmul(tf, d2), t6 = cmul(to, dn);
            const double2 t7 = cmul(fourth, d1), t8 = cmul(fifth, d1);
            // P1 = sum fo inv (2 first d2 + second d1)      P2 = sum fo inv third (d1 - 4 d2)
            // P3 = sum fo (2 tf d2 + to dn)                 P4 = sum fo inv fourth d1
            // P5 = sum fo fifth d1                          P6 = sum fo (first d2 + second d1)
            // P7 = sum fo third (d1 - 2 d2)                 P8 = sum fo diff (tf d2 - to dn)
            // P9 = sum fo fourth d1
            acc[j][0] = cadd(acc[j][0], cscale(cadd(cscale(t1, 2.0), t2), fi));
            acc[j][1] = cadd(acc[j][1], cscale(csub(t3, cscale(t4, 4.0)), fi));
            acc[j][2] = cadd(acc[j][2], cscale(cadd(cscale(t5, 2.0), t6), fo));
            acc[j][3] = cadd(acc[j][3], cscale(t7, fi));
            acc[j][4] = cadd(acc[j][4], cscale(t8, fo));
            acc[j][5] = cadd(acc[j][5], cscale(cadd(t1, t2), fo));
            acc[j][6] = cadd(acc[j][6], cscale(csub(t3, cscale(t4, 2.0)), fo));
            acc[j][7] = cadd(acc[j][7], cscale(csub(t5, t6), fd));
            acc[j][8] = cadd(acc[j][8], cscale(t7, fo));
        }
    }
}

// GW: matrices in the per-CTA global working set (large nw); else dynamic shared memory.
template <bool GW>
__global__ void __launch_bounds__(256) shg_kernel(ShgParams p) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *sm;
    if constexpr (GW) sm = p.gscratch + (int64_t)blockIdx.x * p.gscratch_stride;
    else sm = smem_dyn;
    const int nw = p.nw, ld = p.ld, nn = nw * nw, nc = p.nc;
    const ShgSmem L = ShgSmem::layout(nw, nc);
    double2 *sU = reinterpret_cast<double2 *>(sm + L.U);
    double2 *T1 = reinterpret_cast<double2 *>(sm + L.T1);
    double2 *T2 = reinterpret_cast<double2 *>(sm + L.T2);
    double2 *X = reinterpret_cast<double2 *>(sm + L.X);
    double2 *sV = reinterpret_cast<double2 *>(sm + L.V);
    double2 *sA = reinterpret_cast<double2 *>(sm + L.A);
    double *I0 = reinterpret_cast<double *>(sm + L.I0);
    double *Rg = reinterpret_cast<double *>(sm + L.Rg);
    double *Wt = reinterpret_cast<double *>(sm + L.Wt);
    double *sE = reinterpret_cast<double *>(sm + L.E);
    double *sf = reinterpret_cast<double *>(sm + L.f);
    double2 *dAd = reinterpret_cast<double2 *>(sm + L.dAd);
    double2 *ddHd = reinterpret_cast<double2 *>(sm + L.ddHd);
    double *curv = reinterpret_cast<double *>(sm + L.curv);
    int *plist = reinterpret_cast<int *>(sm + L.plist);
    double2 *sS = reinterpret_cast<double2 *>(sm + L.S);
    double *red = reinterpret_cast<double *>(sm + L.red);
    int *ired = reinterpret_cast<int *>(red + 64);
    const size_t matsz = (size_t)nw * ld;
    double2 *G = p.scratch + (int64_t)blockIdx.x * p.scratch_stride;
    double2 *coef = G + 9 * (int64_t)nn;
    double *pinfo = reinterpret_cast<double *>(coef + (int64_t)nn * nc * 7);
    auto V = [&](int a, int i, int j) { return sV[matsz * a + i + ld * j]; };
    auto A = [&](int a, int i, int j) { return sA[matsz * a + i + ld * j]; };
    // r0 = A + i D0 with D0_ij = dH_ij I0(E_j - E_i); r_eta with the regularised inverse.
    auto d0 = [&](int a, int i, int j) { return cscale(V(a, i, j), I0[i + nw * j]); };
    auto dip = [&](int a, int i, int j) { return cadd(A(a, i, j), cmuli(d0(a, i, j))); };
    const double2 *msrc = nullptr;
    const double *mdiag = nullptr;
    auto rdip = [&](int a, int i, int j) {
        if (p.metric) return msrc[(int64_t)(24 + a) * nn + i + nw * j];
        return cadd(A(a, i, j), cmuli(cscale(V(a, i, j), Rg[i + nw * j])));
    };
    auto gel = [&](int a, int b, int i, int j) { return G[(int64_t)(a + 3 * b) * nn + i + nw * j]; };
    const double eta = p.eta;

    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x;
    const int64_t ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *xw = p.xw + b * p.xw_stride;
        const double wk = p.weights ? p.weights[b] * p.scale : p.scale;
        if (p.metric) {
            msrc = p.m_src + b * 27 * (int64_t)nn;
            mdiag = p.m_diag + b * 18 * (int64_t)nw;
        }
        for (int e = threadIdx.x; e < nn; e += blockDim.x) sU[(e % nw) + ld * (e / nw)] = p.U[b * nn + e];
        for (int i = threadIdx.x; i < nw; i += blockDim.x) {
            const double e = p.E[b * nw + i];
            sE[i] = e;
            sf[i] = shg_occupation(e, p.mu, p.T);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            const int i = e % nw, j = e / nw;
            I0[e] = shg_bare_inverse(sE[j] - sE[i]);
            Rg[e] = reg_inverse(sE[j] - sE[i], p.metric ? p.vertex_eta : eta);
            Wt[e] = shg_weight(sE[i] - sE[j], eta);
        }
        if (p.metric) {
            for (int e = threadIdx.x; e < 3 * nn; e += blockDim.x) {
                const int a = e / nn, r = e % nn, o = (r % nw) + ld * (r / nw);
                sV[matsz * a + o] = msrc[(int64_t)a * nn + r];
                sA[matsz * a + o] = msrc[(int64_t)(3 + a) * nn + r];
            }
            __syncthreads();
        } else {
            for (int a = 0; a < 3; ++a) {
                rotate_to_hamiltonian(xw + (int64_t)p.ch_dH[a] * nn, T1, T2, sU, sV + matsz * a, nw, ld);
                rotate_to_hamiltonian(xw + (int64_t)p.ch_A[a] * nn, T1, T2, sU, sA + matsz * a, nw, ld);
            }
        }

        // Stage 2: G^{ab} (optical_position_vertices!, OpticalPositionDerivatives.jl:36-89).
        for (int ab = 0; ab < 9; ++ab) {
            const int a = ab % 3, bb = ab / 3;
            if (p.metric) {
                for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                    const int o = (e % nw) + ld * (e / nw);
                    X[o] = msrc[(int64_t)(6 + a * 3 + bb) * nn + e];
                    T1[o] = msrc[(int64_t)(15 + a * 3 + bb) * nn + e];
                }
                __syncthreads();
            } else {
                rotate_to_hamiltonian(xw + (int64_t)p.ch_ddH[a * 3 + bb] * nn, T1, T2, sU, X, nw, ld);
                rotate_to_hamiltonian(xw + (int64_t)p.ch_dA[a * 3 + bb] * nn, T1, T2, sU, T1, nw, ld);
            }
            for (int n = threadIdx.x; n < nw; n += blockDim.x) {
                ddHd[ab * nw + n] = X[n + ld * n];
                dAd[ab * nw + n] = T1[n + ld * n];
            }
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int n = e % nw, m = e / nw;
                if (n == m) continue;
                double2 comA = make_double2(0.0, 0.0), comH = comA, corr = comA;
                const double En = sE[n], Em = sE[m];
                for (int l = 0; l < nw; ++l) {
                    const double2 Drlm = cscale(V(bb, l, m), Rg[l + nw * m]);
                    const double2 Drnl = cscale(V(bb, n, l), Rg[n + nw * l]);
                    const double2 Aanl = A(a, n, l), Aalm = A(a, l, m);
                    const double2 Vanl = V(a, n, l), Valm = V(a, l, m);
                    comA = cadd(comA, csub(cmul(Aanl, Drlm), cmul(Drnl, Aalm)));
                    comH = cadd(comH, csub(cmul(Vanl, Drlm), cmul(Drnl, Valm)));
                    if (p.eta_correction && l != n && l != m) {
                        const double El = sE[l];
                        const double2 t1 = csub(cmul(Aanl, V(bb, l, m)),
                                                cmul(cadd(Vanl, cmuli(cscale(Aanl, En - El))), A(bb, l, m)));
                        const double2 t2 = csub(cmul(V(bb, n, l), Aalm),
                                                cmul(A(bb, n, l), cadd(Valm, cmuli(cscale(Aalm, El - Em)))));
                        corr = cadd(corr, csub(cscale(t1, Wt[l + nw * m]), cscale(t2, Wt[n + nw * l])));
                    }
                }
                const double2 Drnm = cscale(V(bb, n, m), Rg[e]);
                const double2 dAa = csub(A(a, n, n), A(a, m, m)), dAb = csub(A(bb, n, n), A(bb, m, m));
                const double2 sum_a = csub(comA, cmul(dAa, Drnm));
                const double2 sum_h = csub(comH, cmul(csub(V(a, n, n), V(a, m, m)), Drnm));
                const double2 D0a = d0(a, n, m), D0b = d0(bb, n, m);
                double2 finite = cadd(T1[n + ld * m], sum_a);
                finite = cadd(finite, cadd(cmul(dAa, D0b), cmul(dAb, D0a)));
                finite = csub(finite, cmuli(cmul(A(a, n, m), dAb)));
                double2 num = cadd(X[n + ld * m], sum_h);
                num = cadd(num, cadd(cscale(D0a, V(bb, n, n).x - V(bb, m, m).x), cscale(D0b, V(a, n, n).x - V(a, m, m).x)));
                num = cadd(cmuli(num), corr);
                const double inv = I0[e];
                G[(int64_t)ab * nn + e] = inv == 0.0 ? finite : cadd(finite, cscale(num, inv));
            }
            __syncthreads();
        }

        // Stage 3: active pairs in column-major order (n fastest), then per-pair coefficients.
        if (threadIdx.x == 0) ired[0] = 0;
        __syncthreads();
        for (int base = 0; base < nn; base += blockDim.x) {
            const int e = base + threadIdx.x;
            bool keep = false;
            if (e < nn) {
                const int n = e % nw, m = e / nw;
                keep = n != m && fabs(sf[n] - sf[m]) >= 1.0e-10;
            }
            const unsigned ball = __ballot_sync(0xffffffffu, keep);
            const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
            if (lane == 0) ired[8 + wid] = __popc(ball);
            __syncthreads();
            int before = ired[0];
            for (int w = 0; w < wid; ++w) before += ired[8 + w];
            before += __popc(ball & ((1u << lane) - 1u));
            if (keep) plist[before] = e;
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += ired[8 + w];
                ired[0] += tot;
            }
            __syncthreads();
        }
        const int npairs = ired[0];
        for (int it = threadIdx.x; it < npairs * nc; it += blockDim.x) {
            const int q = it / nc, c = it % nc;
            const int e = plist[q], n = e % nw, m = e / nw;
            const int a = p.comp[c][0], bb = p.comp[c][1], cc = p.comp[c][2];
            const double inv = I0[n + nw * m];   // bare inverse of E_m - E_n
            const double2 r_nm_a = dip(a, n, m), r_mn_b = dip(bb, m, n), r_mn_c = dip(cc, m, n);
            const double2 r_nm_b = dip(bb, n, m), r_nm_c = dip(cc, n, m);
            const double2 first = cmul(r_nm_a, cadd(gel(bb, cc, m, n), gel(cc, bb, m, n)));
            const double2 second = cadd(cmul(gel(a, bb, n, m), r_mn_c), cmul(gel(a, cc, n, m), r_mn_b));
            const double2 third = cscale(cmul(r_nm_a, cadd(cscale(r_mn_b, V(cc, m, m).x - V(cc, n, n).x),
                                                            cscale(r_mn_c, V(bb, m, m).x - V(bb, n, n).x))), inv);
            const double2 fourth = cadd(cmul(gel(bb, a, n, m), r_mn_c), cmul(gel(cc, a, n, m), r_mn_b));
            const double2 fifth = cscale(cadd(cmul(r_nm_b, r_mn_c), cmul(r_nm_c, r_mn_b)), V(a, n, n).x - V(a, m, m).x);
            double2 tf = make_double2(0.0, 0.0), to = tf;
            for (int l = 0; l < nw; ++l) {
                if (l == n || l == m) continue;
                const double2 rml_b = rdip(bb, m, l), rml_c = rdip(cc, m, l);
                const double2 rln_b = rdip(bb, l, n), rln_c = rdip(cc, l, n);
                tf = cadd(tf, cscale(cmul(r_nm_a, cadd(cmul(rml_b, rln_c), cmul(rml_c, rln_b))),
                                     shg_principal(2.0 * sE[l] - sE[n] - sE[m], eta)));
                to = cadd(to, cscale(cmul(rdip(a, m, l), cadd(cmul(rln_b, r_nm_c), cmul(rln_c, r_nm_b))),
                                     shg_principal(2.0 * sE[n] - sE[m] - sE[l], eta)));
                to = cadd(to, cscale(cmul(rdip(a, l, n), cadd(cmul(r_nm_b, rml_c), cmul(r_nm_c, rml_b))),
                                     shg_principal(2.0 * sE[m] - sE[l] - sE[n], eta)));
            }
            double2 *cf = coef + ((int64_t)q * nc + c) * 7;
            cf[0] = first; cf[1] = second; cf[2] = third; cf[3] = fourth; cf[4] = fifth; cf[5] = tf; cf[6] = to;
            if (c == 0) {
                pinfo[4 * q] = sf[n] - sf[m];
                pinfo[4 * q + 1] = inv;
                pinfo[4 * q + 2] = sE[m] - sE[n];
                pinfo[4 * q + 3] = 0.0;
            }
        }
        __syncthreads();
        // Frequency-independent sums S1 = sum fo inv (first + second), S2 = sum fo inv third,
        // S4 = sum fo inv fourth (the low-frequency parts of terms 1, 2 and 4).
        for (int c = threadIdx.x; c < nc; c += blockDim.x) {
            double2 s1 = make_double2(0.0, 0.0), s2 = s1, s4 = s1;
            for (int q = 0; q < npairs; ++q) {
                const double fi = pinfo[4 * q] * pinfo[4 * q + 1];
                const double2 *cf = coef + ((int64_t)q * nc + c) * 7;
                s1 = cadd(s1, cscale(cadd(cf[0], cf[1]), fi));
                s2 = cadd(s2, cscale(cf[2], fi));
                s4 = cadd(s4, cscale(cf[3], fi));
            }
            sS[3 * c] = s1; sS[3 * c + 1] = s2; sS[3 * c + 2] = s4;
        }
        __syncthreads();

        // Stage 4: pair terms 1-5 of both quantities.
        const int nchunks = (nc + SHG_CB - 1) / SHG_CB;
        for (int it = threadIdx.x; it < p.nom * nchunks; it += blockDim.x) {
            const int w = it % p.nom, c0 = (it / p.nom) * SHG_CB;
            const double om = p.omegas[w];
            double2 acc[SHG_CB][9];
#pragma unroll
            for (int j = 0; j < SHG_CB; ++j)
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[j][t] = make_double2(0.0, 0.0);
            if (p.gaussian) shg_contract<true>(p, coef, pinfo, npairs, om, c0, acc);
            else shg_contract<false>(p, coef, pinfo, npairs, om, c0, acc);
            if (p.mode == 0 && npairs == 0) continue;
            const double low = shg_principal(om, p.low_width);
#pragma unroll
            for (int j = 0; j < SHG_CB; ++j) {
                const int c = c0 + j;
                if (c >= nc) break;
                const double2 s1 = sS[3 * c], s2 = sS[3 * c + 1], s4 = sS[3 * c + 2];
                double2 o[10];
                o[0] = cscale(cmuli(cadd(acc[j][0], cscale(s1, low))), 0.5);
                o[1] = cscale(cmuli(csub(acc[j][1], cscale(s2, low))), 0.5);
                o[2] = cscale(acc[j][2], 0.5);
                o[3] = cscale(cmuli(cadd(acc[j][3], cscale(s4, low))), -0.25);
                o[4] = cscale(cmuli(acc[j][4]), -0.125 * low * low);
                o[5] = acc[j][5];
                o[6] = acc[j][6];
                o[7] = cmulmi(acc[j][7]);
                o[8] = cscale(acc[j][8], -0.5);
                o[9] = cscale(acc[j][4], -0.25 * low);
                for (int t = 0; t < 5; ++t) {
                    shg_emit(p, b, p.out + w + (int64_t)p.nom * (c + (int64_t)nc * t), o[t], wk);
                    shg_emit(p, b, p.out + w + (int64_t)p.nom * (c + (int64_t)nc * (t + 7)), o[5 + t], wk);
                }
            }
        }

        // Stage 5: one-band terms 6-7 (second_harmonic_one_band!).
        const bool warm = p.T > 1.0e-7;
        if (warm) {
            const double kt = SHG_KB_EV * p.T;
            for (int it = threadIdx.x; it < nw * 9; it += blockDim.x) {
                const int n = it / 9, ab = it % 9, a = ab % 3, bb = ab / 3;
                double value = 0.0;
                const bool isolated = (n == 0 || sE[n] - sE[n - 1] > p.degeneracy) &&
                                      (n == nw - 1 || sE[n + 1] - sE[n] > p.degeneracy);
                if (a != bb && isolated && fabs(sE[n] - p.mu) <= 5.0 * kt && p.metric) {
                    value = mdiag[(9 + a * 3 + bb) * nw + n];
                } else if (a != bb && isolated && fabs(sE[n] - p.mu) <= 5.0 * kt) {
                    double2 v = csub(dAd[(bb + 3 * a) * nw + n], dAd[(a + 3 * bb) * nw + n]);
                    for (int l = 0; l < nw; ++l) {
                        const double2 t = csub(cadd(csub(cmul(A(bb, n, l), d0(a, l, n)), cmul(d0(a, n, l), A(bb, l, n))),
                                                    cmul(d0(bb, n, l), A(a, l, n))),
                                               cmul(A(a, n, l), d0(bb, l, n)));
                        const double2 u = csub(cmul(d0(a, n, l), d0(bb, l, n)), cmul(d0(bb, n, l), d0(a, l, n)));
                        v = csub(cadd(v, t), cmuli(u));
                    }
                    value = v.x;
                }
                curv[n * 9 + ab] = value;
            }
            __syncthreads();
            for (int c = threadIdx.x; c < nc; c += blockDim.x) {
                const int a = p.comp[c][0], bb = p.comp[c][1], cc = p.comp[c][2];
                double semi = 0.0, bcd = 0.0;
                for (int n = 0; n < nw; ++n) {
                    const double offset = sE[n] - p.mu;
                    if (fabs(offset) > 5.0 * kt) continue;
                    const double fd = -exp(-0.5 * (offset / kt) * (offset / kt)) / (kt * 2.5066282746310005024);
                    const double sd = -offset / (kt * kt) * fd;
                    const bool isolated = (n == 0 || sE[n] - sE[n - 1] > p.degeneracy) &&
                                          (n == nw - 1 || sE[n + 1] - sE[n] > p.degeneracy);
                    double hess;
                    if (p.metric) {
                        hess = mdiag[(bb * 3 + cc) * nw + n];
                    } else {
                        hess = ddHd[(bb + 3 * cc) * nw + n].x;
                        for (int l = 0; l < nw; ++l)
                            if (l != n) hess += 2.0 * cmul(V(bb, n, l), V(cc, l, n)).x * shg_principal(sE[n] - sE[l], eta);
                    }
                    const double va = V(a, n, n).x, vb = V(bb, n, n).x, vc = V(cc, n, n).x;
                    semi += sd * va * vb * vc + fd * va * hess;
                    if (isolated) bcd += fd * (vb * curv[n * 9 + a + 3 * cc] + vc * curv[n * 9 + a + 3 * bb]);
                }
                sS[3 * c] = make_double2(bcd, semi);
            }
            __syncthreads();
        }
        if (warm || p.mode == 1) {
            for (int it = threadIdx.x; it < p.nom * nc; it += blockDim.x) {
                const int w = it % p.nom, c = it / p.nom;
                double2 o6 = make_double2(0.0, 0.0), o6s = o6, o7 = o6, o7s = o6;
                if (warm) {
                    const double bcd = sS[3 * c].x, semi = sS[3 * c].y;
                    const double low = shg_principal(p.omegas[w], p.low_width);
                    const double2 kern = make_double2(low, -shg_delta(p.omegas[w], p.low_width, p.gaussian));
                    o6 = cscale(kern, -0.25 * bcd * low);
                    o6s = cmuli(cscale(kern, 0.5 * bcd));
                    o7 = cmuli(cscale(kern, -0.25 * semi * low * low));
                    o7s = cscale(kern, -0.5 * semi * low);
                }
                shg_emit(p, b, p.out + w + (int64_t)p.nom * (c + (int64_t)nc * 5), o6, wk);
                shg_emit(p, b, p.out + w + (int64_t)p.nom * (c + (int64_t)nc * 12), o6s, wk);
                shg_emit(p, b, p.out + w + (int64_t)p.nom * (c + (int64_t)nc * 6), o7, wk);
                shg_emit(p, b, p.out + w + (int64_t)p.nom * (c + (int64_t)nc * 13), o7s, wk);
            }
        }
        __syncthreads();
    }
}
