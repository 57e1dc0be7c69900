// response.cuh - fused per-k response kernel: gauge rotation, geometry, integrands, transition
// screen, frequency contraction and deterministic accumulation.  One CTA per k-point; each CTA
// owns a fixed contiguous range of the batch and a fixed slot of the partial-sum buffer, so the
// result does not depend on scheduling.
//
// Reference routines restated here (file:line in the WannierNLQG project):
//   U' X U                      transform_to_hamiltonian_gauge!, HamiltonianMatrixElements.jl:61-71
//   inverse energy differences  PositionMatrixElements.jl:444-461; PositionVertexRegularization.jl:7-29
//   D = -dH .* inv, r = A + iD  PositionMatrixElements.jl:462-483
//   generalised derivative      conventional_generalized_position_derivative_element, ConventionalShiftCurrent.jl:191-229
//   shift-current kernel        ConventionalShiftCurrent.jl:716-729
//   injection-current kernel    ConventionalInjectionCurrent.jl:23-97
//   occupations                 fermi_dirac!, CalculationUtils.jl:28-46
//   transition screen           _fill_transition_screen!, TransitionScreening.jl:32-94
//   frequency accumulation      accumulate_conventional_response!, ConventionalShiftCurrent.jl:864-882
//   Berry curvature (occupied)  berry_curvature_occupied_sum_component, ConventionalQuantumGeometry.jl:188-215
//   Wannier curvature           PositionMatrixElements.jl:485-556 (evaluated as U'dA U - i[A^H_a, A^H_b])
//   quantum metric (band sum)   quantum_metric_band_sum_component, ConventionalQuantumGeometry.jl:321-355
#pragma once
#include "common.cuh"

#define RS_MAX_FREQ 8
#define RS_MAX_SCALAR 16
#define RS_MAX_G 9

enum { RS_FC_SHIFT = 1, RS_FC_INJECTION = 2 };
enum { RS_SC_BERRY = 1, RS_SC_METRIC = 2 };

struct RespParams {
    int nw, ld;
    int64_t batch;
    int64_t xw_stride;          // complex entries per k in xw
    const double2 *xw;          // Wannier-gauge channels [batch][C][nw][nw]
    const double *E;            // [batch][nw]
    const double2 *U;           // [batch][nw][nw]
    // Channel index inside xw (-1: absent).
    int ch_dH[3], ch_A[3], ch_ddH[9], ch_dA[9];   // [p*3+d]: position p, derivative d
    // Shared-memory matrix slots (-1: absent).
    int slot_dH[3], slot_A[3];
    int n_g;
    int g_p[RS_MAX_G], g_d[RS_MAX_G], g_slot[RS_MAX_G];
    // Frequency-axis components (shift / injection).
    int n_fc;
    int fc_kind[RS_MAX_FREQ], fc_a[RS_MAX_FREQ], fc_b[RS_MAX_FREQ], fc_c[RS_MAX_FREQ];
    int fc_g1[RS_MAX_FREQ], fc_g2[RS_MAX_FREQ];   // index into the g list: G(c,a), G(b,a)
    double fc_pref[RS_MAX_FREQ];
    int64_t fc_out[RS_MAX_FREQ];
    // Scalar components (Berry curvature, quantum metric).
    int n_sc;
    int sc_kind[RS_MAX_SCALAR], sc_a[RS_MAX_SCALAR], sc_b[RS_MAX_SCALAR];
    int64_t sc_out[RS_MAX_SCALAR];
    // Frequencies and screen parameters.
    int nom;
    const double *omegas;
    double mu, kT;
    int gaussian;
    double width, cutoff, gscale, thr;
    int window_interval;        // 1: the sorted omega grid is dense enough for the interval test
    double om_lo, om_hi;
    double eta_reg;
    double scale;               // 1/Nk (mesh mode) or 1 (point mode)
    const double *weights;      // per-k weights (mode 0); nullptr: every k uses `scale`
    int mode;                   // 0: accumulate into partials[cta]; 1: write per-point values
    int64_t vc;                 // values per k
    double *partials;           // [gridDim][vc][4]: (sum re, sum im, comp re, comp im)
    double2 *out_points;        // [batch][vc]
    int64_t point_offset;       // global index of batch entry 0 (mode 1)
    int n_slots;
};

struct RespSmem {
    // Byte offsets inside the dynamic shared memory.
    size_t U, T1, T2, slots, inv, E, f, te, fnm, Q, fd, red, total;
    static __host__ __device__ RespSmem layout(int nw, int n_slots, int n_fc, int n_berry, int csize) {
        RespSmem s;
        int ld = nw + 1;
        size_t mat = (size_t)nw * ld * csize;
        size_t off = 0;
        auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 15) & ~(size_t)15; return o; };
        s.U = take(mat);
        s.T1 = take(mat);
        s.T2 = take(mat);
        s.slots = take(mat * n_slots);
        s.inv = take((size_t)nw * nw * sizeof(double));
        s.E = take(nw * sizeof(double));
        s.f = take(nw * sizeof(double));
        s.te = take((size_t)nw * nw * sizeof(double));
        s.fnm = take((size_t)nw * nw * sizeof(double));
        s.Q = take((size_t)nw * nw * (n_fc > 0 ? n_fc : 1) * sizeof(double2));
        s.fd = take((size_t)nw * (n_berry > 0 ? n_berry : 1) * sizeof(double2));
        s.red = take(64 * sizeof(double) + 64 * sizeof(int));
        s.total = off;
        return s;
    }
};

// regularized_energy_inverse (PositionVertexRegularization.jl:17-29).
WNLQG_D double reg_inverse(double d, double eta) {
    double den = d * d + eta * eta;
    if (isfinite(den) && den != 0.0) return d / den;
    if (!(isfinite(d) && isfinite(eta) && eta > 0)) return d / den;
    double sc = fmax(fabs(d), eta);
    double sd = d / sc, sw = eta / sc;
    return (sd / (sd * sd + sw * sw)) / sc;
}

WNLQG_D double fermi_occ(double e, double mu, double kT) {
    if (kT == 0.0) return e <= mu ? 1.0 : 0.0;
    double arg = fmin(700.0, fmax(-700.0, (e - mu) / kT));
    return 1.0 / (exp(arg) + 1.0);
}

// dst = U^H X U for one Wannier-gauge matrix X read from global memory (column-major nw x nw).
// All threads participate; shared matrices use leading dimension ld = nw + 1.
WNLQG_D void rotate_to_hamiltonian(const double2 *__restrict__ src, double2 *T1, double2 *T2, const double2 *U,
                                   double2 *dst, int nw, int ld) {
    const int nn = nw * nw;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        int i = e % nw, j = e / nw;
        T1[i + ld * j] = src[e];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        int i = e % nw, j = e / nw;
        double2 acc = make_double2(0.0, 0.0);
        for (int l = 0; l < nw; ++l) acc = cfma(T1[i + ld * l], U[l + ld * j], acc);
        T2[i + ld * j] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        int i = e % nw, j = e / nw;
        double2 acc = make_double2(0.0, 0.0);
        for (int l = 0; l < nw; ++l) acc = cfmaconj(U[l + ld * i], T2[l + ld * j], acc);
        dst[i + ld * j] = acc;
    }
    __syncthreads();
}

// Deterministic block sum of one double per thread (fixed shuffle tree, warps in order).
WNLQG_D double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += red[w];
        red[32] = total;
    }
    __syncthreads();
    total = red[32];
    __syncthreads();
    return total;
}

// Does any photon energy lie within `half` of transition energy te (|te - omega| < half)?
WNLQG_D bool any_within(double te, double half, const RespParams &p) {
    if (p.window_interval) return te > p.om_lo - half && te < p.om_hi + half;
    for (int w = 0; w < p.nom; ++w)
        if (fabs(te - p.omegas[w]) < half) return true;
    return false;
}

__global__ void __launch_bounds__(256) response_kernel_f64(RespParams p) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int nw = p.nw, ld = p.ld, nn = nw * nw;
    const RespSmem L = RespSmem::layout(nw, p.n_slots, p.n_fc, 1, sizeof(double2));
    double2 *sU = reinterpret_cast<double2 *>(sm + L.U);
    double2 *T1 = reinterpret_cast<double2 *>(sm + L.T1);
    double2 *T2 = reinterpret_cast<double2 *>(sm + L.T2);
    double2 *slots = reinterpret_cast<double2 *>(sm + L.slots);
    double *sinv = reinterpret_cast<double *>(sm + L.inv);
    double *sE = reinterpret_cast<double *>(sm + L.E);
    double *sf = reinterpret_cast<double *>(sm + L.f);
    double *ste = reinterpret_cast<double *>(sm + L.te);
    double *sfnm = reinterpret_cast<double *>(sm + L.fnm);
    double2 *sQ = reinterpret_cast<double2 *>(sm + L.Q);
    double2 *sFd = reinterpret_cast<double2 *>(sm + L.fd);
    double *red = reinterpret_cast<double *>(sm + L.red);
    int *ired = reinterpret_cast<int *>(red + 64);
    const size_t matsz = (size_t)nw * ld;
    auto slot = [&](int s) { return slots + matsz * s; };

    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x;
    const int64_t ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *xw = p.xw + b * p.xw_stride;
        const double wk = p.weights ? p.weights[b] * p.scale : p.scale;
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            int i = e % nw, j = e / nw;
            sU[i + ld * j] = p.U[b * nn + e];
        }
        for (int i = threadIdx.x; i < nw; i += blockDim.x) {
            double e = p.E[b * nw + i];
            sE[i] = e;
            sf[i] = fermi_occ(e, p.mu, p.kT);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            int i = e % nw, j = e / nw;
            double d = sE[i] - sE[j];
            sinv[e] = p.eta_reg == 0.0 ? (d == 0.0 ? 0.0 : 1.0 / d) : reg_inverse(d, p.eta_reg);
        }
        for (int a = 0; a < 3; ++a)
            if (p.slot_dH[a] >= 0) rotate_to_hamiltonian(xw + (int64_t)p.ch_dH[a] * nn, T1, T2, sU, slot(p.slot_dH[a]), nw, ld);
        for (int a = 0; a < 3; ++a)
            if (p.slot_A[a] >= 0) rotate_to_hamiltonian(xw + (int64_t)p.ch_A[a] * nn, T1, T2, sU, slot(p.slot_A[a]), nw, ld);

        // Generalised derivatives r^p_{nm;d} (ConventionalShiftCurrent.jl:191-229).
        for (int g = 0; g < p.n_g; ++g) {
            const int pp = p.g_p[g], dd = p.g_d[g];
            double2 *G = slot(p.g_slot[g]);
            rotate_to_hamiltonian(xw + (int64_t)p.ch_dA[pp * 3 + dd] * nn, T1, T2, sU, G, nw, ld);
            rotate_to_hamiltonian(xw + (int64_t)p.ch_ddH[pp * 3 + dd] * nn, T1, T2, sU, T1, nw, ld);
            const double2 *Ap = slot(p.slot_A[pp]), *Ad = slot(p.slot_A[dd]);
            const double2 *Hp = slot(p.slot_dH[pp]), *Hd = slot(p.slot_dH[dd]);
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int n = e % nw, m = e / nw;
                double2 sum_AD = make_double2(0.0, 0.0), sum_HD = make_double2(0.0, 0.0);
                for (int l = 0; l < nw; ++l) {
                    if (l == n || l == m) continue;
                    // D_d[l,m] = -dH_d[l,m] inv[l,m];  D_d[n,l] = -dH_d[n,l] inv[n,l]
                    double2 Dlm = cscale(Hd[l + ld * m], -sinv[l + nw * m]);
                    double2 Dnl = cscale(Hd[n + ld * l], -sinv[n + nw * l]);
                    sum_AD = cadd(sum_AD, csub(cmul(Ap[n + ld * l], Dlm), cmul(Dnl, Ap[l + ld * m])));
                    sum_HD = cadd(sum_HD, csub(cmul(Hp[n + ld * l], Dlm), cmul(Dnl, Hp[l + ld * m])));
                }
                const double inm = sinv[n + nw * m];
                double2 Da = cscale(Hp[n + ld * m], -inm);   // D_p[n,m]
                double2 Db = cscale(Hd[n + ld * m], -inm);   // D_d[n,m]
                double2 dAdn = csub(Ad[n + ld * n], Ad[m + ld * m]);
                double2 dApn = csub(Ap[n + ld * n], Ap[m + ld * m]);
                double2 AD_bit = cadd(cmul(dAdn, Da), cmul(dApn, Db));
                double2 AA_bit = cmul(dAdn, Ap[n + ld * m]);
                double2 DV_bit = cadd(cmul(csub(Hd[n + ld * n], Hd[m + ld * m]), Da),
                                      cmul(csub(Hp[n + ld * n], Hp[m + ld * m]), Db));
                double2 h = cadd(cadd(T1[n + ld * m], sum_HD), DV_bit);
                double2 v = cadd(cadd(G[n + ld * m], AD_bit), csub(sum_AD, cmuli(AA_bit)));
                v = cadd(v, cmuli(cscale(h, -inm)));
                G[n + ld * m] = v;
            }
            __syncthreads();
        }

        // Scalar responses.
        for (int s = 0; s < p.n_sc; ++s) {
            const int a = p.sc_a[s], bb = p.sc_b[s];
            const double2 *Aa = slot(p.slot_A[a]), *Ab = slot(p.slot_A[bb]);
            const double2 *Ha = slot(p.slot_dH[a]), *Hb = slot(p.slot_dH[bb]);
            double local = 0.0;
            if (p.sc_kind[s] == RS_SC_BERRY) {
                // Diagonals of U^H (dA_b/dk_a) U (kept in sFd) and U^H (dA_a/dk_b) U (left in T1).
                rotate_to_hamiltonian(xw + (int64_t)p.ch_dA[bb * 3 + a] * nn, T1, T2, sU, T1, nw, ld);
                for (int n = threadIdx.x; n < nw; n += blockDim.x) sFd[n] = T1[n + ld * n];
                __syncthreads();
                rotate_to_hamiltonian(xw + (int64_t)p.ch_dA[a * 3 + bb] * nn, T1, T2, sU, T1, nw, ld);
            }
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int n = e % nw, m = e / nw;
                const double inm = sinv[e];
                double2 ra = cadd(Aa[n + ld * m], cmuli(cscale(Ha[n + ld * m], -inm)));
                const double imn = sinv[m + nw * n];
                double2 rb = cadd(Ab[m + ld * n], cmuli(cscale(Hb[m + ld * n], -imn)));
                if (p.sc_kind[s] == RS_SC_BERRY) {
                    if (n == m) {
                        // F_nn = (U'dA_b/dk_a U)_nn - (U'dA_a/dk_b U)_nn - i sum_l (A_a[n,l]A_b[l,n] - A_b[n,l]A_a[l,n])
                        double2 fnn = csub(sFd[n], T1[n + ld * n]);
                        double2 comm = make_double2(0.0, 0.0);
                        for (int l = 0; l < nw; ++l)
                            comm = cadd(comm, csub(cmul(Aa[n + ld * l], Ab[l + ld * n]), cmul(Ab[n + ld * l], Aa[l + ld * n])));
                        fnn = csub(fnn, cmuli(comm));
                        local += sf[n] * fnn.x;
                    } else {
                        double2 t = cmuli(cmul(ra, rb));
                        local += (sf[n] - sf[m]) * t.x;
                    }
                } else if (n != m) {
                    local += 0.5 * (sf[n] + sf[m]) * cmul(ra, rb).x;
                }
            }
            double total = block_sum(local, red);
            if (threadIdx.x == 0) {
                if (p.mode == 0) {
                    double *acc = p.partials + ((int64_t)blockIdx.x * p.vc + p.sc_out[s]) * 4;
                    neumaier_add(acc[0], acc[2], total * wk);
                } else {
                    p.out_points[(p.point_offset + b) * p.vc + p.sc_out[s]] = make_double2(total * p.scale, 0.0);
                }
            }
        }

        if (p.n_fc > 0) {
            // Transition screen and per-pair kernels, pairs in column-major (n fastest) order.
            if (threadIdx.x == 0) { ired[0] = 0; ired[1] = 0; }
            __syncthreads();
            for (int base = 0; base < nn; base += blockDim.x) {
                const int e = base + threadIdx.x;
                bool keep = false;
                int n = 0, m = 0;
                double fnm = 0.0, te = 0.0;
                if (e < nn) {
                    n = e % nw; m = e / nw;
                    fnm = sf[n] - sf[m];
                    te = sE[m] - sE[n];
                    const bool occ = fabs(fnm) > 1.0e-10;
                    if (occ) {
                        if (p.gaussian) {
                            keep = any_within(te, p.cutoff, p);
                            if (keep) ired[1] = 1;
                        } else {
                            keep = true;
                            if (p.thr <= 0.0 || any_within(te, p.thr, p)) ired[1] = 1;
                        }
                    }
                }
                // Ordered compaction: warp ballots, warps in order.
                unsigned ball = __ballot_sync(0xffffffffu, keep);
                int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
                if (lane == 0) ired[8 + wid] = __popc(ball);
                __syncthreads();
                int before = ired[0];
                for (int w = 0; w < wid; ++w) before += ired[8 + w];
                before += __popc(ball & ((1u << lane) - 1u));
                if (keep) {
                    ste[before] = te;
                    sfnm[before] = fnm;
                    for (int c = 0; c < p.n_fc; ++c) {
                        const int a = p.fc_a[c], bb = p.fc_b[c], cc = p.fc_c[c];
                        const double2 *Ab = slot(p.slot_A[bb]), *Ac = slot(p.slot_A[cc]);
                        const double2 *Hb = slot(p.slot_dH[bb]), *Hc = slot(p.slot_dH[cc]);
                        // r_c[n,m] and r_b[m,n]
                        double2 rc_nm = cadd(Ac[n + ld * m], cmuli(cscale(Hc[n + ld * m], -sinv[n + nw * m])));
                        double2 rb_mn = cadd(Ab[m + ld * n], cmuli(cscale(Hb[m + ld * n], -sinv[m + nw * n])));
                        double2 q;
                        if (p.fc_kind[c] == RS_FC_SHIFT) {
                            const double2 *G1 = slot(p.g_slot[p.fc_g1[c]]), *G2 = slot(p.g_slot[p.fc_g2[c]]);
                            q = cmulmi(csub(cmul(G1[n + ld * m], rb_mn), cmul(G2[m + ld * n], rc_nm)));
                        } else {
                            const double2 *Ha = slot(p.slot_dH[a]);
                            double2 vd = csub(Ha[m + ld * m], Ha[n + ld * n]);
                            q = cmul(cmul(vd, rc_nm), rb_mn);
                        }
                        sQ[(size_t)c * nn + before] = q;
                    }
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    int tot = 0;
                    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += ired[8 + w];
                    ired[0] += tot;
                }
                __syncthreads();
            }
            const int npairs = ired[0];
            const bool active = ired[1] != 0;
            for (int w = threadIdx.x; w < p.nom; w += blockDim.x) {
                const double om = p.omegas[w];
                double2 acc[RS_MAX_FREQ];
                for (int c = 0; c < RS_MAX_FREQ; ++c) acc[c] = make_double2(0.0, 0.0);
                if (active) {
                    for (int q = 0; q < npairs; ++q) {
                        const double x = ste[q] - om;
                        double delta;
                        if (p.gaussian) {
                            if (!(fabs(x) < p.cutoff)) continue;
                            const double y = x / p.width;
                            delta = p.gscale * exp(-y * y);
                        } else {
                            delta = (p.width / WNLQG_PI) / (x * x + p.width * p.width);
                        }
                        const double weight = sfnm[q] * delta;
                        if (weight == 0.0) continue;
                        for (int c = 0; c < p.n_fc; ++c) {
                            const double cw = p.fc_pref[c] * weight;
                            const double2 qq = sQ[(size_t)c * nn + q];
                            acc[c].x = fma(cw, qq.x, acc[c].x);
                            acc[c].y = fma(cw, qq.y, acc[c].y);
                        }
                    }
                }
                for (int c = 0; c < p.n_fc; ++c) {
                    const int64_t idx = p.fc_out[c] + w;
                    if (p.mode == 0) {
                        if (active) {
                            double *a4 = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
                            neumaier_add(a4[0], a4[2], acc[c].x * wk);
                            neumaier_add(a4[1], a4[3], acc[c].y * wk);
                        }
                    } else {
                        p.out_points[(p.point_offset + b) * p.vc + idx] = cscale(acc[c], p.scale);
                    }
                }
            }
        }
        __syncthreads();
    }
}

// out[v] = sum over CTAs g (in order) of partials[g][v], compensated.
__global__ void reduce_partials_kernel(const double *__restrict__ partials, int64_t nslots, int64_t vc,
                                       double2 *__restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < vc; v += (int64_t)gridDim.x * blockDim.x) {
        double sr = 0.0, cr = 0.0, si = 0.0, ci = 0.0;
        for (int64_t g = 0; g < nslots; ++g) {
            const double *a = partials + (g * vc + v) * 4;
            neumaier_add(sr, cr, a[0]);
            neumaier_add(sr, cr, a[2]);
            neumaier_add(si, ci, a[1]);
            neumaier_add(si, ci, a[3]);
        }
        out[v] = make_double2(sr + cr, si + ci);
    }
}
