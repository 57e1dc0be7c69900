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
#include "dmma.cuh"

#define RS_MAX_FREQ 8
#define RS_MAX_SCALAR 16
#define RS_MAX_G 9

enum { RS_FC_SHIFT = 1, RS_FC_INJECTION = 2, RS_FC_JERK = 3 };
enum { RS_SC_BERRY = 1, RS_SC_METRIC = 2 };
enum { RS_MU_AHC = 1, RS_MU_DIPOLE = 2, RS_MU_LT = 3, RS_MU_BANDCURV = 4 };
#define RS_MAX_HESS 9
#define RS_MU_CHUNK 8

struct RespParams {
    int nw, ld;
    int omb_force;              // photon energies per thread in the contraction: 1, 2, 4; 0 = sized to the axis
    int64_t batch;
    int64_t xw_stride;          // complex entries per k in xw
    const double2 *xw;          // Wannier-gauge channels [batch][C][nw][nw]
    const double *E;            // [batch][nw]
    const double2 *U;           // [batch][nw][nw]
    // Channel index inside xw (-1: absent).
    int ch_dH[3], ch_A[3], ch_ddH[9], ch_dA[9];   // [p*3+d]: position p, derivative d
    // Shared-memory matrix slots (-1: absent).
    int slot_dH[3], slot_A[3], slot_D[3];
    int n_g;
    int g_p[RS_MAX_G], g_d[RS_MAX_G], g_slot[RS_MAX_G];
    // Frequency-axis components (shift / injection).
    int n_fc;
    int fc_kind[RS_MAX_FREQ], fc_a[RS_MAX_FREQ], fc_b[RS_MAX_FREQ], fc_c[RS_MAX_FREQ];
    int fc_g1[RS_MAX_FREQ], fc_g2[RS_MAX_FREQ];   // index into the g list: G(c,a), G(b,a)
    double fc_pref[RS_MAX_FREQ];
    int64_t fc_out[RS_MAX_FREQ];
    // Pair family of the frequency components: 0 = transition screen (shift/injection),
    // 1 = positive-gap pairs with a windowed delta (jerk).
    int pair_mode;
    int fc_hess[RS_MAX_FREQ];                     // jerk: index into the Hessian list (a,d)
    int n_hess;
    int hess_a[RS_MAX_HESS], hess_d[RS_MAX_HESS];
    // Fermi-energy-axis components (intrinsic AHC, Berry-curvature dipole).
    int n_mu;
    int mu_kind[RS_MAX_SCALAR], mu_a[RS_MAX_SCALAR], mu_b[RS_MAX_SCALAR], mu_c[RS_MAX_SCALAR];
    int64_t mu_out[RS_MAX_SCALAR];
    int nmu;
    const double *mus;
    double temperature, fs_width;
    double lt_gamma, lt_factor;   // linear transport Berry channel: interband rate (eV), e^2/hbar 1e-20
    // Band curvature items (RS_MU_BANDCURV, the shifted points of the finite-difference Fermi-sea
    // dipole): Omega_n^{ab} of batch entry b goes to curv_out[b * curv_stride + mu_out * nw + n].
    double *curv_out;
    int64_t curv_stride;
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
    const int *out_perm;        // mode 1: batch entry b is written to row out_perm[b]; nullptr: row b
    int n_slots;
    // Per-CTA working set in global memory (L1/L2-resident) when it exceeds shared memory
    // (large nw); nullptr: dynamic shared memory.
    unsigned char *gscratch;
    int64_t gscratch_stride;
    // Shift/injection band window (-1: all bands) and the response degeneracy threshold.
    int band_window;
    int use_sel;                         // explicit interband selection (valence n, conduction m)
    unsigned vsel[4], csel[4];
    double degeneracy_threshold;
    // Nonorthogonal models: per-k geometry precomputed by nonorth_geometry_kernel (Berry
    // connection r [batch][3][nn], Hellmann-Feynman slopes v [batch][3][nw], generalized
    // derivatives [batch][ng_pairs][nn] with g_ng[g] the pair index of G slot g).  nullptr: the
    // orthogonal geometry of this kernel.
    const double2 *ng_r;
    const double *ng_v;
    const double2 *ng_G;
    int ng_pairs;
    int g_ng[RS_MAX_G];
};

// Effective band window [lo, hi) (0-based) around mu: select_band_window (CalculationUtils.jl:71-90),
// widened for a finite window to whole degeneracy groups (TransitionScreening.jl:201-233,
// ResponseDegeneracyGroups.jl:10-33).  lo = hi = 0: the Fermi level is outside the spectrum.
WNLQG_D void band_window(const double *E, int n, double mu, int size, double thr, int &lo, int &hi) {
    if (size == -1 || 2 * size > n) { lo = 0; hi = n; return; }
    int valence = 0;
    while (valence < n && E[valence] <= mu) ++valence;
    if (valence < 1 || valence >= n) { lo = 0; hi = 0; return; }
    int start = max(1, valence - size + 1), end = min(n, valence + size);
    double emax = 0.0;
    for (int i = 0; i < n; ++i) emax = fmax(emax, fabs(E[i]));
    const double equal = 32.0 * 2.220446049250313e-16 * fmax(1.0, emax);
    while (start > 1 && (E[start - 1] - E[start - 2] < thr || E[start - 1] - E[start - 2] <= equal)) --start;
    while (end < n && (E[end] - E[end - 1] < thr || E[end] - E[end - 1] <= equal)) ++end;
    lo = start - 1;
    hi = end;
}

struct RespSmem {
    // Byte offsets inside the dynamic shared memory.
    size_t U, T1, T2, slots, inv, E, f, te, fnm, Q, fd, hess, red, total;
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
        s.Q = take((size_t)nw * nw * (n_fc > 0 ? n_fc : 1) * csize);
        s.fd = take((size_t)4 * nw * (n_berry > 0 ? n_berry : 1) * sizeof(double2));
        s.hess = take((size_t)RS_MAX_HESS * nw * sizeof(double));
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

// response_occupation (Responses/Shared/ResponseOccupations.jl:8-14): strict step with one half
// at equality at T = 0, the stable logistic form above.
WNLQG_D double response_occ(double e, double mu, double T) {
    if (T == 0.0) return e < mu ? 1.0 : (e > mu ? 0.0 : 0.5);
    const double x = (e - mu) / (8.617333262145e-5 * T);
    const double z = exp(-fabs(x));
    return x >= 0.0 ? z / (1.0 + z) : 1.0 / (1.0 + z);
}

WNLQG_D double fermi_occ(double e, double mu, double kT) {
    if (kT == 0.0) return e <= mu ? 1.0 : 0.0;
    double arg = fmin(700.0, fmax(-700.0, (e - mu) / kT));
    return 1.0 / (exp(arg) + 1.0);
}

// ---- shared-memory matrix products (all threads participate; ld = nw + 1) -------------------
// Complex FP64 (double2): FP64 tensor cores (dmma_product).  Complex FP32 (float2): CUDA cores,
// work item w -> row i = w % nw and four columns 4*(w / nw) .. +3: the row operand is read
// conflict-free across lanes, the column operand is a broadcast.
#define RS_JB 4

WNLQG_D double2 load_c(const double2 *p) { return *p; }
template <typename C> WNLQG_D C conv_c(double2 v);
template <> WNLQG_D double2 conv_c<double2>(double2 v) { return v; }
template <> WNLQG_D float2 conv_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

// out = X * Y
template <typename C> WNLQG_D void mm_xy(const C *X, const C *Y, C *out, int nw, int ld) {
    if constexpr (same_type<C, double2>::value) {
        dmma_product<0>(X, Y, out, nw, ld);
        return;
    }
    const int ng = (nw + RS_JB - 1) / RS_JB;
    for (int w = threadIdx.x; w < nw * ng; w += blockDim.x) {
        const int i = w % nw, j0 = (w / nw) * RS_JB;
        C acc[RS_JB];
#pragma unroll
        for (int q = 0; q < RS_JB; ++q) acc[q] = czero<C>();
        for (int l = 0; l < nw; ++l) {
            const C x = X[i + ld * l];
#pragma unroll
            for (int q = 0; q < RS_JB; ++q)
                if (j0 + q < nw) acc[q] = cfma(x, Y[l + ld * (j0 + q)], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < RS_JB; ++q)
            if (j0 + q < nw) out[i + ld * (j0 + q)] = acc[q];
    }
}

// out = X^H * Y
template <typename C> WNLQG_D void mm_xhy(const C *X, const C *Y, C *out, int nw, int ld) {
    if constexpr (same_type<C, double2>::value) {
        dmma_product<1>(X, Y, out, nw, ld);
        return;
    }
    const int ng = (nw + RS_JB - 1) / RS_JB;
    for (int w = threadIdx.x; w < nw * ng; w += blockDim.x) {
        const int i = w % nw, j0 = (w / nw) * RS_JB;
        C acc[RS_JB];
#pragma unroll
        for (int q = 0; q < RS_JB; ++q) acc[q] = czero<C>();
        for (int l = 0; l < nw; ++l) {
            const C x = X[l + ld * i];
#pragma unroll
            for (int q = 0; q < RS_JB; ++q)
                if (j0 + q < nw) acc[q] = cfmaconj(x, Y[l + ld * (j0 + q)], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < RS_JB; ++q)
            if (j0 + q < nw) out[i + ld * (j0 + q)] = acc[q];
    }
}

// out = X * Y - Y * X
template <typename C> WNLQG_D void mm_comm(const C *X, const C *Y, C *out, int nw, int ld) {
    if constexpr (same_type<C, double2>::value) {
        dmma_product<2>(X, Y, out, nw, ld);
        return;
    }
    const int ng = (nw + RS_JB - 1) / RS_JB;
    for (int w = threadIdx.x; w < nw * ng; w += blockDim.x) {
        const int i = w % nw, j0 = (w / nw) * RS_JB;
        C acc[RS_JB];
#pragma unroll
        for (int q = 0; q < RS_JB; ++q) acc[q] = czero<C>();
        for (int l = 0; l < nw; ++l) {
            const C x = X[i + ld * l], y = Y[i + ld * l];
#pragma unroll
            for (int q = 0; q < RS_JB; ++q)
                if (j0 + q < nw) {
                    acc[q] = cfma(x, Y[l + ld * (j0 + q)], acc[q]);
                    const C xl = X[l + ld * (j0 + q)];
                    acc[q] = cfma(make_neg(y), xl, acc[q]);
                }
        }
#pragma unroll
        for (int q = 0; q < RS_JB; ++q)
            if (j0 + q < nw) out[i + ld * (j0 + q)] = acc[q];
    }
}

// Prefetch of one 128-byte line into L2 (a hint: no value, no fault on the line's contents).
WNLQG_D void l2_prefetch(const void *ptr) { asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr)); }

// dst0 = X0 - Y0 (and dst1 = X1 when X1 is given) for column-major nw x nw matrices in global
// memory (Y0 optional), into shared matrices of leading dimension ld.  Each thread issues all the
// loads of four elements per matrix before its first store, so that the global-memory latency is
// paid once per four elements instead of once per element.  No closing barrier.
template <typename C>
WNLQG_D void stage_from_global(const double2 *__restrict__ X0, C *dst0, int nw, int ld,
                               const double2 *__restrict__ Y0 = nullptr, const double2 *__restrict__ X1 = nullptr,
                               C *dst1 = nullptr) {
    constexpr int B = 4;
    const int nn = nw * nw;
    const double2 zero = make_double2(0.0, 0.0);
    for (int e0 = threadIdx.x; e0 < nn; e0 += B * blockDim.x) {
        double2 v0[B], v1[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int e = e0 + j * blockDim.x;
            v0[j] = e < nn ? (Y0 ? csub(X0[e], Y0[e]) : X0[e]) : zero;
            v1[j] = (X1 && e < nn) ? X1[e] : zero;
        }
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int e = e0 + j * blockDim.x;
            if (e < nn) {
                const int o = (e % nw) + ld * (e / nw);
                dst0[o] = conv_c<C>(v0[j]);
                if (X1) dst1[o] = conv_c<C>(v1[j]);
            }
        }
    }
}

// dst = U^H X U for a Wannier-gauge matrix X in global memory (FP64, column-major nw x nw).
// dst may alias T1.
template <typename C>
WNLQG_D void rotate_to_hamiltonian(const double2 *__restrict__ src, C *T1, C *T2, const C *U, C *dst, int nw, int ld) {
    stage_from_global(src, T1, nw, ld);
    __syncthreads();
    mm_xy(T1, U, T2, nw, ld);
    __syncthreads();
    mm_xhy(U, T2, dst, nw, ld);
    __syncthreads();
}

// dst0 = U^H X0 U and dst1 = U^H X1 U for two Wannier-gauge channels in global memory.  FP64: the
// channels are staged in dst0 and dst1 (eight loads in flight per thread), then two paired DMMA
// passes (four accumulator tiles per warp; three barriers for both channels); dst0 and dst1 must
// not alias T1, T2 or U.  FP32: two single rotations.
template <typename C>
WNLQG_D void rotate_two_to_hamiltonian(const double2 *__restrict__ src0, const double2 *__restrict__ src1, C *T1,
                                       C *T2, const C *U, C *dst0, C *dst1, int nw, int ld) {
    if constexpr (same_type<C, double2>::value) {
        stage_from_global(src0, dst0, nw, ld, (const double2 *)nullptr, src1, dst1);
        __syncthreads();
        dmma_product_pair<0>(dst0, ld, U, T1, dst1, ld, U, T2, nw, ld);
        __syncthreads();
        dmma_product_pair<1>(U, ld, T1, dst0, U, ld, T2, dst1, nw, ld);
        __syncthreads();
    } else {
        rotate_to_hamiltonian(src0, T1, T2, U, dst0, nw, ld);
        rotate_to_hamiltonian(src1, T1, T2, U, dst1, nw, ld);
    }
}

// Per-band sums out(n, sum_l term(n, l)) for n < nw, by groups of g threads per band (g the largest
// power of two up to 32 with g nw <= blockDim.x): each thread of a group sums the terms l = part,
// part + g, ... in order, then a fixed shuffle butterfly adds the group's partials, so the order of
// the additions is fixed and the result reproducible.  A band's group is g consecutive lanes of one
// warp.  All threads of the CTA call it (every lane takes every shuffle); no closing barrier.
template <typename F, typename S>
WNLQG_D void band_sums(int nw, F term, S out) {
    int g = 32;
    while (g > 1 && g * nw > (int)blockDim.x) g >>= 1;
    const int part = threadIdx.x & (g - 1);
    const int per = (int)blockDim.x / g;
    for (int n0 = 0; n0 < nw; n0 += per) {
        const int n = n0 + (int)threadIdx.x / g;
        double2 acc = make_double2(0.0, 0.0);
        if (n < nw)
            for (int l = part; l < nw; l += g) acc = cadd(acc, term(n, l));
        for (int o = g >> 1; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (part == 0 && n < nw) out(n, acc);
    }
}

// diag[n] = (U^H (X - Y) U)_nn for Wannier-gauge X and optional Y (nullptr: 0); uses T1, T2.
template <typename C>
WNLQG_D void rotate_diagonal(const double2 *__restrict__ src, C *T1, C *T2, const C *U, double2 *diag, int nw, int ld,
                             const double2 *__restrict__ sub = nullptr) {
    stage_from_global(src, T1, nw, ld, sub);
    __syncthreads();
    mm_xy(T1, U, T2, nw, ld);
    __syncthreads();
    band_sums(
        nw, [&](int n, int l) { return cfmaconj(to_c64(U[l + ld * n]), to_c64(T2[l + ld * n]), make_double2(0.0, 0.0)); },
        [&](int n, double2 v) { diag[n] = v; });
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

#define RS_OMB 4   // largest number of photon energies per thread per pass of the pair loop

// Reciprocal of a Lorentzian denominator den >= w2 > 0.  FP32 path: the fast hardware quotient.
// FP64 path: one cubically convergent step r <- r (1 + e + e^2), e = 1 - den r (the series of
// 1 / (1 - e), truncated after e^2), seeded by the PTX instruction rcp.approx.ftz.f64 (a hardware
// approximation), so that no FP64 <-> FP32 conversions are needed.  The seed's relative error
// measured on B200 is at most 2^-19.96 (4M denominators from 1e-10 to 1e4), so the step leaves
// e^3 < 2^-59 plus a few ulp of rounding, in three FMAs (two Newton steps took four).  The
// denominators are normal numbers (den >= w2 > 0), so flushing subnormals changes nothing.
WNLQG_D float lorentz_recip(float den) { return __fdividef(1.0f, den); }
WNLQG_D double lorentz_recip(double den) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(den));
    const double e = fma(-den, r, 1.0);
    return fma(r, fma(e, e, e), r);
}
WNLQG_D float lorentz(float num, float den) { return __fdividef(num, den); }
WNLQG_D double lorentz(double num, double den) { return num * lorentz_recip(den); }

// One pair's contribution to a thread's OMB photon energies.  KIND 0: Gaussian with the
// sqrt(200) cutoff (transition screen); 1: Lorentzian (q0, q1 already carry f_nm width / pi);
// 2: jerk's windowed delta (Gaussian or Lorentzian by `gaussian`).
template <typename R, typename C, int KIND, int OMB, bool TWO>
WNLQG_D void contract_one(double te, R fq, C q0, C q1, const double *om, C (*acc)[2], R gsc, R cut, R invw,
                          R w2, R lor, R win, int gaussian) {
#pragma unroll
    for (int j = 0; j < OMB; ++j) {
        const R x = (R)(te - om[j]);
        R weight;
        if (KIND == 0) {
            if (!(fabs(x) < cut)) continue;
            const R y = x * invw;
            weight = fq * (gsc * exp(-y * y));
        } else if (KIND == 1) {
            weight = lorentz_recip(x * x + w2);
        } else {
            if (win > (R)0 && fabs(x) > win) continue;
            const R y = x * invw;
            weight = fq * (gaussian ? gsc * exp(-y * y) : lorentz(lor, x * x + w2));
        }
        acc[j][0].x = fma(weight, q0.x, acc[j][0].x);
        acc[j][0].y = fma(weight, q0.y, acc[j][0].y);
        if (TWO) {
            acc[j][1].x = fma(weight, q1.x, acc[j][1].x);
            acc[j][1].y = fma(weight, q1.y, acc[j][1].y);
        }
    }
}

// Frequency contraction of one thread's OMB photon energies over the pair list, for one or two
// components (TWO).  Pairs are streamed two at a time into separate accumulators (two independent
// dependency chains per energy), which are added at the end.
template <typename R, typename C, int KIND, int OMB, bool TWO>
WNLQG_D void contract_pairs(const double *ste, const double *sfnm, const C *Q0, const C *Q1, int npairs,
                            const double *om, C (*acc)[2], R gsc, R cut, R invw, R w2, R lor, R win, int gaussian) {
    C odd[OMB][2];
#pragma unroll
    for (int j = 0; j < OMB; ++j) { odd[j][0] = czero<C>(); odd[j][1] = czero<C>(); }
    int q = 0;
    for (; q + 1 < npairs; q += 2) {
        contract_one<R, C, KIND, OMB, TWO>(ste[q], (R)sfnm[q], Q0[q], TWO ? Q1[q] : Q0[q], om, acc, gsc, cut, invw,
                                           w2, lor, win, gaussian);
        contract_one<R, C, KIND, OMB, TWO>(ste[q + 1], (R)sfnm[q + 1], Q0[q + 1], TWO ? Q1[q + 1] : Q0[q + 1], om, odd,
                                           gsc, cut, invw, w2, lor, win, gaussian);
    }
    if (q < npairs)
        contract_one<R, C, KIND, OMB, TWO>(ste[q], (R)sfnm[q], Q0[q], TWO ? Q1[q] : Q0[q], om, acc, gsc, cut, invw, w2,
                                           lor, win, gaussian);
#pragma unroll
    for (int j = 0; j < OMB; ++j) {
        acc[j][0] = cadd(acc[j][0], odd[j][0]);
        acc[j][1] = cadd(acc[j][1], odd[j][1]);
    }
}

template <typename R, typename C, int OMB, bool TWO>
WNLQG_D void contract_dispatch(int pair_mode, int gaussian, const double *ste, const double *sfnm, const C *Q0,
                               const C *Q1, int npairs, const double *om, C (*acc)[2], R gsc, R cut, R invw, R w2,
                               R lor, R win) {
    if (pair_mode == 1)
        contract_pairs<R, C, 2, OMB, TWO>(ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win, gaussian);
    else if (gaussian)
        contract_pairs<R, C, 0, OMB, TWO>(ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win, 1);
    else
        contract_pairs<R, C, 1, OMB, TWO>(ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win, 0);
}

// R: storage/arithmetic type of the per-k matrices (double: plain FP64 path; float: mixed path).
// Energies, inverse energy differences, occupations and every accumulation across pairs of a
// scalar response and across k-points stay FP64.
// NG: the per-k geometry comes precomputed (nonorthogonal models); a separate instantiation so the
// orthogonal kernel carries no code for it.  The FP64 kernel runs one CTA per SM (its shared
// memory), the FP32 kernel two: the register budgets follow.
// GW: the per-k working set lives in global memory (p.gscratch); a separate instantiation so that
// the shared-memory kernel addresses shared memory directly.
// WIDE: 512 threads per CTA (16 warps to hide the FP64 latencies of the one CTA an SM holds) at
// 128 registers per thread instead of 256 threads at up to 255; the autotuner picks the width.
template <typename R, bool NG, bool GW, bool WIDE = false>
__global__ void __launch_bounds__(WIDE ? 512 : 256, WIDE ? 1 : (sizeof(R) == 8 ? 1 : 2)) response_kernel(RespParams p) {
    typedef typename cplx_of<R>::type C;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *sm;
    if constexpr (GW) sm = p.gscratch + (int64_t)blockIdx.x * p.gscratch_stride;
    else sm = smem_dyn;
    const int nw = p.nw, ld = p.ld, nn = nw * nw;
    const RespSmem L = RespSmem::layout(nw, p.n_slots, p.n_fc, 1, sizeof(C));
    C *sU = reinterpret_cast<C *>(sm + L.U);
    C *T1 = reinterpret_cast<C *>(sm + L.T1);
    C *T2 = reinterpret_cast<C *>(sm + L.T2);
    C *slots = reinterpret_cast<C *>(sm + L.slots);
    double *sinv = reinterpret_cast<double *>(sm + L.inv);
    double *sE = reinterpret_cast<double *>(sm + L.E);
    double *sf = reinterpret_cast<double *>(sm + L.f);
    double *ste = reinterpret_cast<double *>(sm + L.te);
    double *sfnm = reinterpret_cast<double *>(sm + L.fnm);
    C *sQ = reinterpret_cast<C *>(sm + L.Q);
    double2 *sFd = reinterpret_cast<double2 *>(sm + L.fd);
    double *sHess = reinterpret_cast<double *>(sm + L.hess);
    double *red = reinterpret_cast<double *>(sm + L.red);
    int *ired = reinterpret_cast<int *>(red + 64);
    const size_t matsz = (size_t)nw * ld;
    auto slot = [&](int s) { return slots + matsz * s; };
    // r_a[n,m] = A_a[n,m] + i D_a[n,m], D_a = -dH_a .* inv
    auto r_elem = [&](int a, int n, int m) -> C {
        const C A = slot(p.slot_A[a])[n + ld * m];
        const C H = slot(p.slot_dH[a])[n + ld * m];
        const R s = (R)(-sinv[n + nw * m]);
        return cadd(A, cmuli(cscale(H, s)));
    };

    const int64_t kb = (p.batch * blockIdx.x) / gridDim.x;
    const int64_t ke = (p.batch * (blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *xw = p.xw + b * p.xw_stride;
        const double wk = p.weights ? p.weights[b] * p.scale : p.scale;
        if (!NG && p.xw && b + 1 < ke) {
            // The next point's channels and eigenvectors into L2 (128-byte lines) while this
            // point computes: its staging loads then wait on L2 instead of HBM.
            const char *nx = reinterpret_cast<const char *>(xw + p.xw_stride);
            const char *nu = reinterpret_cast<const char *>(p.U + (b + 1) * nn);
            const int64_t lx = p.xw_stride * (int64_t)sizeof(double2) / 128, lu = (int64_t)nn * sizeof(double2) / 128;
            for (int64_t l = threadIdx.x; l < lx + lu; l += blockDim.x)
                l2_prefetch(l < lx ? nx + 128 * l : nu + 128 * (l - lx));
        }
        stage_from_global(p.U + b * nn, sU, nw, ld);
        for (int i = threadIdx.x; i < nw; i += blockDim.x) {
            const double e = p.E[b * nw + i];
            sE[i] = e;
            sf[i] = fermi_occ(e, p.mu, p.kT);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            const int i = e % nw, j = e / nw;
            const double d = sE[i] - sE[j];
            sinv[e] = p.eta_reg == 0.0 ? (d == 0.0 ? 0.0 : 1.0 / d) : reg_inverse(d, p.eta_reg);
        }
        if constexpr (NG) {
            // Nonorthogonal model: Berry connection into the A slots, slopes on the dH diagonals,
            // generalized derivatives into the G slots; r_elem then reads r directly (inv = 0).
            for (int e = threadIdx.x; e < nn; e += blockDim.x) sinv[e] = 0.0;
            for (int a = 0; a < 3; ++a) {
                if (p.slot_A[a] >= 0) {
                    C *dst = slot(p.slot_A[a]);
                    const double2 *src = p.ng_r + (b * 3 + a) * (int64_t)nn;
                    for (int e = threadIdx.x; e < nn; e += blockDim.x) dst[(e % nw) + ld * (e / nw)] = conv_c<C>(src[e]);
                }
                if (p.slot_dH[a] >= 0) {
                    C *dst = slot(p.slot_dH[a]);
                    const double *v = p.ng_v + (b * 3 + a) * (int64_t)nw;
                    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                        const int i = e % nw, j = e / nw;
                        dst[i + ld * j] = conv_c<C>(make_double2(i == j ? v[i] : 0.0, 0.0));
                    }
                }
            }
            for (int g = 0; g < p.n_g; ++g) {
                C *dst = slot(p.g_slot[g]);
                const double2 *src = p.ng_G + (b * p.ng_pairs + p.g_ng[g]) * (int64_t)nn;
                for (int e = threadIdx.x; e < nn; e += blockDim.x) dst[(e % nw) + ld * (e / nw)] = conv_c<C>(src[e]);
            }
            __syncthreads();
        } else {
            // The velocity and connection channels, two rotations per paired pass.
            {
                const double2 *src[6];
                C *dst[6];
                int nrot = 0;
                for (int a = 0; a < 3; ++a)
                    if (p.slot_dH[a] >= 0) { src[nrot] = xw + (int64_t)p.ch_dH[a] * nn; dst[nrot++] = slot(p.slot_dH[a]); }
                for (int a = 0; a < 3; ++a)
                    if (p.slot_A[a] >= 0) { src[nrot] = xw + (int64_t)p.ch_A[a] * nn; dst[nrot++] = slot(p.slot_A[a]); }
                int r = 0;
                for (; r + 1 < nrot; r += 2) rotate_two_to_hamiltonian(src[r], src[r + 1], T1, T2, sU, dst[r], dst[r + 1], nw, ld);
                if (r < nrot) rotate_to_hamiltonian(src[r], T1, T2, sU, dst[r], nw, ld);
            }
            // Gauge corrections D_d = -dH_d .* inv for the derivative axes of the generalised derivatives.
            for (int a = 0; a < 3; ++a)
                if (p.slot_D[a] >= 0) {
                    C *D = slot(p.slot_D[a]);
                    const C *H = slot(p.slot_dH[a]);
                    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                        const int i = e % nw, j = e / nw;
                        D[i + ld * j] = cscale(H[i + ld * j], (R)(-sinv[e]));
                    }
                }
            __syncthreads();

            // Generalised derivatives r^p_{nm;d} (ConventionalShiftCurrent.jl:191-229), with the
            // l != n,m sums written as commutators (exact: D_nn = 0):
            //   sum_AD + AD_bit = [A_p, D_d]_nm + (A_d,nn - A_d,mm) D_p,nm
            //   sum_HD + DV_bit = [dH_p, D_d]_nm + (dH_d,nn - dH_d,mm) D_p,nm
            // The pair-data region (transition energies, occupations, pair kernels: at least
            // 32 nw^2 bytes) is unused until the pairs are built, so it holds the rotated ddH.
            C *Hpd = reinterpret_cast<C *>(sm + L.te);
            for (int g = 0; g < p.n_g; ++g) {
                const int pp = p.g_p[g], dd = p.g_d[g];
                C *G = slot(p.g_slot[g]);
                rotate_two_to_hamiltonian(xw + (int64_t)p.ch_dA[pp * 3 + dd] * nn, xw + (int64_t)p.ch_ddH[pp * 3 + dd] * nn,
                                          T1, T2, sU, G, Hpd, nw, ld);
                const C *Ap = slot(p.slot_A[pp]), *Ad = slot(p.slot_A[dd]);
                const C *Hp = slot(p.slot_dH[pp]), *Hd = slot(p.slot_dH[dd]);
                const C *Dd = slot(p.slot_D[dd]);
                // T1 = [A_p, D_d], T2 = [dH_p, D_d] in one pass.
                if constexpr (same_type<C, double2>::value) {
                    dmma_product_pair<2>(Ap, ld, Dd, T1, Hp, ld, Dd, T2, nw, ld);
                } else {
                    mm_comm(Ap, Dd, T1, nw, ld);
                    mm_comm(Hp, Dd, T2, nw, ld);
                }
                __syncthreads();
                for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                    const int n = e % nw, m = e / nw;
                    const int o = n + ld * m;
                    const C Dp = cscale(Hp[o], (R)(-sinv[e]));
                    const C dAd = csub(Ad[n + ld * n], Ad[m + ld * m]);
                    const C dHd = csub(Hd[n + ld * n], Hd[m + ld * m]);
                    // G = dA + (A_d,nn - A_d,mm)(D_p - i A_p) + [A_p, D_d]
                    //     + i (ddH + (dH_d,nn - dH_d,mm) D_p + [dH_p, D_d]) (-inv)
                    const C h = cadd(cadd(Hpd[o], cmul(dHd, Dp)), T2[o]);
                    G[o] = cadd(cadd(cadd(G[o], cmul(dAd, csub(Dp, cmuli(Ap[o])))), T1[o]),
                                cmuli(cscale(h, (R)(-sinv[e]))));
                }
                __syncthreads();
            }
        }

        // Scalar responses (FP64 block sums).
        for (int s = 0; s < p.n_sc; ++s) {
            const int a = p.sc_a[s], bb = p.sc_b[s];
            if (p.sc_kind[s] == RS_SC_BERRY) {
                // F_nn = (U' (dA_b/dk_a - dA_a/dk_b) U)_nn - i [A_a, A_b]_nn (one rotation of the
                // difference; sFd[nw + n] = 0 keeps the two-term form below).
                rotate_diagonal(xw + (int64_t)p.ch_dA[bb * 3 + a] * nn, T1, T2, sU, sFd, nw, ld,
                                xw + (int64_t)p.ch_dA[a * 3 + bb] * nn);
                // sFd[nw + n] = i [A_a, A_b]_nn.
                const C *Aa = slot(p.slot_A[a]), *Ab = slot(p.slot_A[bb]);
                band_sums(
                    nw,
                    [&](int n, int l) {
                        return to_c64(csub(cmul(Aa[n + ld * l], Ab[l + ld * n]), cmul(Ab[n + ld * l], Aa[l + ld * n])));
                    },
                    [&](int n, double2 v) { sFd[nw + n] = cmuli(v); });
                __syncthreads();
            }
            double local = 0.0;
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const int n = e % nw, m = e / nw;
                if (p.sc_kind[s] == RS_SC_BERRY) {
                    if (n == m) {
                        const double2 fnn = csub(sFd[n], sFd[nw + n]);
                        local += sf[n] * fnn.x;
                    } else {
                        const double2 t = cmuli(to_c64(cmul(r_elem(a, n, m), r_elem(bb, m, n))));
                        local += (sf[n] - sf[m]) * t.x;
                    }
                } else if (n != m) {
                    local += 0.5 * (sf[n] + sf[m]) * (double)cmul(r_elem(a, n, m), r_elem(bb, m, n)).x;
                }
            }
            const double total = block_sum(local, red);
            if (threadIdx.x == 0) {
                if (p.mode == 0) {
                    double *acc = p.partials + ((int64_t)blockIdx.x * p.vc + p.sc_out[s]) * 4;
                    neumaier_add(acc[0], acc[2], total * wk);
                } else {
                    p.out_points[(p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : (int64_t)b)) * p.vc + p.sc_out[s]] = make_double2(total * p.scale, 0.0);
                }
            }
        }


        // Fermi-energy-axis responses.
        for (int s = 0; s < p.n_mu; ++s) {
            const int a = p.mu_a[s], bb = p.mu_b[s], cc = p.mu_c[s];
            // F_nn^{ab} (Hamiltonian-gauge Wannier curvature diagonal) into sFd[2nw .. 3nw).
            rotate_diagonal(xw + (int64_t)p.ch_dA[bb * 3 + a] * nn, T1, T2, sU, sFd, nw, ld,
                            xw + (int64_t)p.ch_dA[a * 3 + bb] * nn);
            for (int n = threadIdx.x; n < nw; n += blockDim.x) sFd[nw + n] = make_double2(0.0, 0.0);
            __syncthreads();
            const C *Aa = slot(p.slot_A[a]), *Ab = slot(p.slot_A[bb]);
            const C *Ha = slot(p.slot_dH[a]), *Hb = slot(p.slot_dH[bb]);
            band_sums(
                nw,
                [&](int n, int l) {
                    return to_c64(csub(cmul(Aa[n + ld * l], Ab[l + ld * n]), cmul(Ab[n + ld * l], Aa[l + ld * n])));
                },
                [&](int n, double2 comm) { sFd[2 * nw + n] = csub(csub(sFd[n], sFd[nw + n]), cmuli(comm)); });
            __syncthreads();
            if (p.mu_kind[s] == RS_MU_BANDCURV) {
                // berry_curvature_group_sum_component with the group {n} (ConventionalQuantumGeometry.jl:
                // 530-557): Re F_nn + sum_{m != n} -Im(r^a_nm r^b_mn - r^b_nm r^a_mn).
                double *dst = p.curv_out + b * p.curv_stride + p.mu_out[s] * nw;
                band_sums(
                    nw,
                    [&](int n, int m) {
                        if (m == n) return make_double2(0.0, 0.0);
                        return make_double2(-to_c64(csub(cmul(r_elem(a, n, m), r_elem(bb, m, n)),
                                                         cmul(r_elem(bb, n, m), r_elem(a, m, n)))).y, 0.0);
                    },
                    [&](int n, double2 om) { dst[n] = sFd[2 * nw + n].x + om.x; });
                __syncthreads();
            } else if (p.mu_kind[s] == RS_MU_DIPOLE) {
                // Band Berry curvature Omega_n = -2 sum_m Im(r^a_nm r^b_mn) + Re F_nn
                // (berry_curvature_component, ConventionalQuantumGeometry.jl:166-180) into sFd[3nw..).
                band_sums(
                    nw,
                    [&](int n, int m) {
                        if (m == n) return make_double2(0.0, 0.0);
                        return make_double2(-to_c64(cmul(r_elem(a, n, m), r_elem(bb, m, n))).y, 0.0);
                    },
                    [&](int n, double2 om) { sFd[3 * nw + n] = make_double2(2.0 * om.x + sFd[2 * nw + n].x, 0.0); });
                __syncthreads();
                if (threadIdx.x == 0) {
                    const C *Hc = slot(p.slot_dH[cc]);
                    for (int im = 0; im < p.nmu; ++im) {
                        const double mu = p.mus[im];
                        double value = 0.0;
                        for (int n = 0; n < nw; ++n) {
                            double w;
                            if (p.temperature > 0.0) {
                                const double scale = 8.617333262145e-5 * p.temperature;
                                const double z = exp(-fabs((sE[n] - mu) / scale));
                                w = z / (scale * (1.0 + z) * (1.0 + z));
                            } else {
                                const double x = (sE[n] - mu) / p.fs_width;
                                w = exp(-x * x) / (sqrt(WNLQG_PI) * p.fs_width);
                            }
                            value += w * sFd[3 * nw + n].x * (double)Hc[n + ld * n].x;
                        }
                        const int64_t idx = p.mu_out[s] + im;
                        if (p.mode == 0) {
                            double *a4 = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
                            neumaier_add(a4[0], a4[2], value * wk);
                        } else {
                            p.out_points[(p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : (int64_t)b)) * p.vc + idx] = make_double2(value * p.scale, 0.0);
                        }
                    }
                }
                __syncthreads();
            } else {
                for (int m0 = 0; m0 < p.nmu; m0 += RS_MU_CHUNK) {
                    double loc[RS_MU_CHUNK];
                    int nocc[RS_MU_CHUNK];
#pragma unroll
                    for (int j = 0; j < RS_MU_CHUNK; ++j) {
                        loc[j] = 0.0;
                        nocc[j] = 0;
                        if (m0 + j < p.nmu) {
                            const double mu = p.mus[m0 + j];
                            for (int n = 0; n < nw; ++n) nocc[j] += sE[n] <= mu ? 1 : 0;
                        }
                    }
                    double exact = 0.0;   // spectral blocks: levels within 32 eps max(1, max|E|)
                    if (p.mu_kind[s] == RS_MU_LT) {
                        for (int n = 0; n < nw; ++n) exact = fmax(exact, fabs(sE[n]));
                        exact = 32.0 * 2.220446049250313e-16 * fmax(1.0, exact);
                    }
                    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                        const int l = e % nw, m = e / nw;
                        if (p.mu_kind[s] == RS_MU_LT) {
                            // Berry channel of _linear_transport_response (LinearTransportKernels.jl:
                            // 100-163): contact -f(E_l) Re F_ll and, over ordered pairs of distinct
                            // spectral blocks, (f_l - f_m) gap^2/(gap^2 + gamma^2) Im(r^a_lm r^b_ml)
                            // (both orders give the reference's 2 Im q of each unordered pair); the
                            // common factor -e^2/hbar 1e-20 is applied to the sum.
                            const double gap = sE[m] - sE[l];
                            const bool joined = l != m && fabs(gap) <= exact;
                            const double rate = gap * gap / (gap * gap + p.lt_gamma * p.lt_gamma);
                            const double2 t = (l == m || joined)
                                                  ? make_double2(0.0, 0.0)
                                                  : cmuli(to_c64(cmul(r_elem(a, l, m), r_elem(bb, m, l))));
#pragma unroll
                            for (int j = 0; j < RS_MU_CHUNK; ++j) {
                                if (m0 + j >= p.nmu) continue;
                                const double mu = p.mus[m0 + j];
                                const double fl = response_occ(sE[l], mu, p.temperature);
                                if (l == m) loc[j] += fl * sFd[2 * nw + l].x;
                                else if (!joined) loc[j] += (fl - response_occ(sE[m], mu, p.temperature)) * rate * t.x;
                            }
                        } else {
                            // Zero temperature (the only AHC temperature, checked at plan creation):
                            // matrix curvature with bare occupied/empty links
                            // (IntrinsicHallCurvature.jl:2-29, IntrinsicHallGeometry.jl:117-136).
                            double pair = 0.0;
                            if (l != m) {
                                const double g = sE[l] - sE[m];
                                auto link = [&](int ax, int x, int y, double inv) {
                                    const double2 A = to_c64(slot(p.slot_A[ax])[x + ld * y]);
                                    const double2 H = to_c64(slot(p.slot_dH[ax])[x + ld * y]);
                                    return cadd(A, cmuli(cscale(H, -inv)));
                                };
                                const double ilm = 1.0 / g, iml = -1.0 / g;
                                const double2 left = cmul(link(a, l, m, ilm), link(bb, m, l, iml));
                                const double2 right = cmul(link(bb, l, m, ilm), link(a, m, l, iml));
                                pair = -(left.y - right.y);
                            }
#pragma unroll
                            for (int j = 0; j < RS_MU_CHUNK; ++j) {
                                if (m0 + j >= p.nmu) continue;
                                if (l == m) { if (l < nocc[j]) loc[j] += sFd[2 * nw + l].x; }
                                else if (l < nocc[j] && m >= nocc[j]) loc[j] += pair;
                            }
                        }
                    }
                    const double mu_scale = p.mu_kind[s] == RS_MU_LT ? -p.lt_factor : 1.0;
                    for (int j = 0; j < RS_MU_CHUNK && m0 + j < p.nmu; ++j) {
                        const double total = mu_scale * block_sum(loc[j], red);
                        if (threadIdx.x == 0) {
                            const int64_t idx = p.mu_out[s] + m0 + j;
                            if (p.mode == 0) {
                                double *a4 = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
                                neumaier_add(a4[0], a4[2], total * wk);
                            } else {
                                p.out_points[(p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : (int64_t)b)) * p.vc + idx] = make_double2(total * p.scale, 0.0);
                            }
                        }
                    }
                }
            }
        }

        // Band Hessians for jerk: H_n^{ad} = Re ddH_ad[n,n] + 2 sum_{l!=n} Re(dH_a[n,l] dH_d[l,n]) reg(E_n-E_l)
        // (prepare_third_order_band_geometry!, ThirdOrderGeometry.jl:131-160).
        for (int h = 0; h < p.n_hess; ++h) {
            const int a = p.hess_a[h], dd = p.hess_d[h];
            rotate_diagonal(xw + (int64_t)p.ch_ddH[a * 3 + dd] * nn, T1, T2, sU, sFd, nw, ld);
            const C *Ha = slot(p.slot_dH[a]), *Hd = slot(p.slot_dH[dd]);
            band_sums(
                nw,
                [&](int n, int l) {
                    if (l == n) return make_double2(0.0, 0.0);
                    return make_double2(2.0 * to_c64(cmul(Ha[n + ld * l], Hd[l + ld * n])).x * sinv[n + nw * l], 0.0);
                },
                [&](int n, double2 v) { sHess[h * nw + n] = sFd[n].x + v.x; });
            __syncthreads();
        }

        if (p.n_fc > 0) {
            // Transition screen and per-pair kernels; pairs kept in column-major (n fastest) order.
            if (threadIdx.x == 0) {
                ired[0] = 0;
                ired[1] = 0;
                int lo = 0, hi = nw;
                if (p.pair_mode == 0) band_window(sE, nw, p.mu, p.band_window, p.degeneracy_threshold, lo, hi);
                ired[2] = lo;
                ired[3] = hi;
            }
            __syncthreads();
            const int wlo = ired[2], whi = ired[3];
            for (int base = 0; base < nn; base += blockDim.x) {
                const int e = base + threadIdx.x;
                bool keep = false;
                int n = 0, m = 0;
                double fnm = 0.0, te = 0.0;
                if (e < nn && p.pair_mode == 1) {
                    // Jerk: ordered pairs with E_n > E_m, weight (f_m - f_n) delta(E_n - E_m - omega)
                    // (ConventionalJerkCurrent.jl:39-61); exactly-zero occupation differences add zero.
                    n = e % nw; m = e / nw;
                    te = sE[n] - sE[m];
                    fnm = sf[m] - sf[n];
                    keep = te > 0.0 && fnm != 0.0;
                    if (keep) ired[1] = 1;
                } else if (e < nn) {
                    n = e % nw; m = e / nw;
                    fnm = sf[n] - sf[m];
                    te = sE[m] - sE[n];
                    const bool selected = !p.use_sel || (((p.vsel[n >> 5] >> (n & 31)) & 1u) &&
                                                         ((p.csel[m >> 5] >> (m & 31)) & 1u));
                    if (selected && fabs(fnm) > 1.0e-10 && n >= wlo && n < whi && m >= wlo && m < whi) {
                        if (p.gaussian) {
                            keep = any_within(te, p.cutoff, p);
                            if (keep) ired[1] = 1;
                        } else {
                            keep = true;
                            if (p.thr <= 0.0 || any_within(te, p.thr, p)) ired[1] = 1;
                        }
                    }
                }
                const unsigned ball = __ballot_sync(0xffffffffu, keep);
                const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
                        const C rc_nm = r_elem(cc, n, m), rb_mn = r_elem(bb, m, n);
                        C q;
                        if (p.fc_kind[c] == RS_FC_JERK) {
                            const int hh = p.fc_hess[c];
                            const R dh = (R)(sHess[hh * nw + n] - sHess[hh * nw + m]);
                            q = cscale(cmul(r_elem(bb, n, m), r_elem(cc, m, n)), dh);
                        } else if (p.fc_kind[c] == RS_FC_SHIFT) {
                            const C *G1 = slot(p.g_slot[p.fc_g1[c]]), *G2 = slot(p.g_slot[p.fc_g2[c]]);
                            q = cmulmi(csub(cmul(G1[n + ld * m], rb_mn), cmul(G2[m + ld * n], rc_nm)));
                        } else {
                            const C *Ha = slot(p.slot_dH[a]);
                            q = cmul(cmul(csub(Ha[m + ld * m], Ha[n + ld * n]), rc_nm), rb_mn);
                        }
                        // Lorentzian kernel (pair mode 0): the pair factor f_nm width / pi is
                        // folded into Q here, once per pair instead of once per photon energy.
                        if (p.pair_mode == 0 && !p.gaussian) q = cscale(q, (R)(fnm * p.width / WNLQG_PI));
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
            // Frequency contraction: each thread owns OMB photon energies per pass (OMB = 1, 2 or 4,
            // the fewest that cover the energy axis with the CTA's threads) and streams the pair list
            // once per pass; threads past the end of the axis skip the pass.
            const R w2 = (R)(p.width * p.width), lor = (R)(p.width / WNLQG_PI);
            const R gsc = (R)p.gscale, cut = (R)p.cutoff, invw = (R)(1.0 / p.width);
            const R win = (R)(p.thr > 0.0 ? p.thr : 0.0);
            const int omb = p.omb_force == 1 || p.omb_force == 2 || p.omb_force == RS_OMB
                                ? p.omb_force
                                : (p.nom <= (int)blockDim.x ? 1 : (p.nom <= 2 * (int)blockDim.x ? 2 : RS_OMB));
            for (int w0 = 0; w0 < p.nom; w0 += omb * blockDim.x) {
                if (w0 + (int)threadIdx.x >= p.nom) continue;
                double om[RS_OMB];
#pragma unroll
                for (int j = 0; j < RS_OMB; ++j) {
                    const int w = w0 + threadIdx.x + j * blockDim.x;
                    om[j] = (j < omb && w < p.nom) ? p.omegas[w] : 0.0;
                }
                // Components in chunks of two keep the accumulators in registers.
                for (int c0 = 0; c0 < p.n_fc; c0 += 2) {
                    const bool two = c0 + 1 < p.n_fc;
                    C acc[RS_OMB][2];
#pragma unroll
                    for (int j = 0; j < RS_OMB; ++j) { acc[j][0] = czero<C>(); acc[j][1] = czero<C>(); }
                    if (active) {
                        const C *Q0 = sQ + (size_t)c0 * nn;
                        const C *Q1 = sQ + (size_t)(two ? c0 + 1 : c0) * nn;
                        if (omb == 1) {
                            if (two) contract_dispatch<R, C, 1, true>(p.pair_mode, p.gaussian, ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win);
                            else contract_dispatch<R, C, 1, false>(p.pair_mode, p.gaussian, ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win);
                        } else if (omb == 2) {
                            if (two) contract_dispatch<R, C, 2, true>(p.pair_mode, p.gaussian, ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win);
                            else contract_dispatch<R, C, 2, false>(p.pair_mode, p.gaussian, ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win);
                        } else {
                            if (two) contract_dispatch<R, C, RS_OMB, true>(p.pair_mode, p.gaussian, ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win);
                            else contract_dispatch<R, C, RS_OMB, false>(p.pair_mode, p.gaussian, ste, sfnm, Q0, Q1, npairs, om, acc, gsc, cut, invw, w2, lor, win);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < RS_OMB; ++j) {
                        const int w = w0 + threadIdx.x + j * blockDim.x;
                        if (j >= omb || w >= p.nom) continue;
#pragma unroll
                        for (int cc = 0; cc < 2; ++cc) {
                            if (cc == 1 && !two) continue;
                            const int c = c0 + cc;
                            const int64_t idx = p.fc_out[c] + w;
                            const double2 v = cscale(to_c64(acc[j][cc]), p.fc_pref[c]);
                            if (p.mode == 0) {
                                if (active) {
                                    double *a4 = p.partials + ((int64_t)blockIdx.x * p.vc + idx) * 4;
                                    neumaier_add(a4[0], a4[2], v.x * wk);
                                    neumaier_add(a4[1], a4[3], v.y * wk);
                                }
                            } else {
                                p.out_points[(p.point_offset + (p.out_perm ? (int64_t)p.out_perm[b] : (int64_t)b)) * p.vc + idx] = cscale(v, p.scale);
                            }
                        }
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
