// wnlqg_oracle.cpp -- CPU FP64 restatement of the WannierNLQG k-mesh response hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, __graft_entry__.smoke()
// and the CPU-baseline leg of bench.py call it as the checker and as the timed CPU path.  The
// product (wanniernlqg_b200) never links, imports or calls it.
//
// Each routine restates the reference's Julia code (paths relative to the WannierNLQG project)
// with plain loops in the reference's own summation order, FP64 / complex<double> throughout:
//   Fourier factors             src/MatrixElements/Interpolated/HamiltonianMatrixElements.jl:28-39
//   direct Fourier sums         HamiltonianMatrixElements.jl:42-58, 426-462; PositionMatrixElements.jl:239-334
//   real-space derivative tiles HamiltonianMatrixElements.jl:92-177; PositionMatrixElements.jl:8-84
//   Hermitian eigensolve        src/Core/ESKernel/DenseSpectra.jl:14-16 (LAPACK there; cyclic Jacobi here)
//   phase canonicalisation      HamiltonianMatrixElements.jl:6-25
//   generalised eigensolve      DenseSpectra.jl:33-39 (LAPACK hegv there; Cholesky + Jacobi here),
//                               NonorthogonalMatrixElements.jl:349-385
//   gauge rotation U'XU         HamiltonianMatrixElements.jl:61-71
//   gauge correction, r, F      PositionMatrixElements.jl:416-556; PositionVertexRegularization.jl:7-29
//   transition screen           src/Runtime/Execution/TransitionScreening.jl:32-94; CalculationUtils.jl:21-46
//   shift current               src/Responses/ShiftCurrent/ConventionalShiftCurrent.jl:191-229, 686-884
//   injection current           src/Responses/InjectionCurrent/ConventionalInjectionCurrent.jl:23-211
//   prefactors                  src/Runtime/Execution/ConventionalCurrentIntegralExecution.jl:241-245, 294-298
//   Berry curvature / metric    src/Responses/QuantumGeometry/ConventionalQuantumGeometry.jl:188-215, 321-355
//   intrinsic AHC (T = 0)       src/Responses/IntrinsicHall/IntrinsicHallOccupations.jl:8-44,
//                               IntrinsicHallCurvature.jl:2-29; MatrixElements/IntrinsicHallGeometry.jl:117-136
//   Berry-curvature dipole      src/Responses/QuantumGeometry/BerryMultipoleMoments.jl:7-47,
//                               BerryMultipoleGeometry.jl:66-161, BerryMultipoleDC.jl:64-75;
//                               Responses/Shared/ResponseOccupations.jl:10-36
//   second harmonic             src/Responses/SecondHarmonicGeneration/SecondHarmonicKernels.jl:1-294;
//                               MatrixElements/Interpolated/OpticalPositionDerivatives.jl:13-123,
//                               PositionVertexRegularization.jl:7-50
//   jerk                        src/Responses/JerkCurrent/ConventionalJerkCurrent.jl:14-65;
//                               MatrixElements/Interpolated/ThirdOrderGeometry.jl:28-41, 131-160
//   mesh + lanes                src/Core/CalculationUtils.jl:280-292; Runtime/Setup/BundleAssembly.jl:35-53;
//                               Runtime/Execution/IntegralDriver.jl:820-874; Reduction/DeterministicReduction.jl:2-38
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <omp.h>

#include "../include/wnlqg_b200.h"

namespace {

using cd = std::complex<double>;
const cd I1(0.0, 1.0);
const double PI = 3.14159265358979323846;

// Constants of src/Core/Constants.jl:1-4.
const double ELEMENTARY_CHARGE_C = 1.602176634e-19;
const double REDUCED_PLANCK_CONSTANT_J_S = 1.054571817e-34;
const double REDUCED_PLANCK_CONSTANT_EV_S = 6.582119569e-16;
const double BOLTZMANN_CONSTANT_EV_K = 8.617333262e-5;
const double RESPONSE_KB_EV = 8.617333262145e-5;   // Responses/Shared/ResponseOccupations.jl:4

thread_local std::string g_error;

struct Mat {
    int n = 0;
    std::vector<cd> v;
    void init(int size) { n = size; v.assign((size_t)size * size, cd(0.0, 0.0)); }
    cd &operator()(int i, int j) { return v[(size_t)i + (size_t)n * j]; }
    const cd &operator()(int i, int j) const { return v[(size_t)i + (size_t)n * j]; }
};

struct Model {
    int nw = 0, nr = 0;
    double lattice[9];
    std::vector<int64_t> rvec;    // [3*NR]
    std::vector<int64_t> deg;     // [NR]
    std::vector<cd> H;            // [nw*nw*NR]
    std::vector<cd> A;            // [nw*nw*3*NR] (zeros when absent)
    std::vector<cd> S;            // [nw*nw*NR] overlap (nonorthogonal models)
    bool has_position = false;
    bool has_overlap = false;
    // Convention I centres (_initialize_wannier_center_scratch!, WannierCenterConventionTransforms.jl:15-56).
    int home = -1;
    std::string centers_error;           // empty: centres valid
    std::vector<double> tau_cart, tau_frac;   // [3 * nw], index a * nw + i
};

// Which Cartesian channels a task needs (the reference's MatrixElementPlan direction
// requirements, MatrixElementPlan.jl:1-18, restated as masks).
struct Needs {
    bool dH[3] = {false, false, false};
    bool ddH[3][3] = {};
    bool A[3] = {false, false, false};
    bool dA[3][3] = {};   // [position][derivative]
    bool ddA[3][3][3] = {};   // [position][derivative][derivative]: d_c d_g A_p
    bool F[3][3] = {};
    bool shg = false;     // second harmonic generation (metric models: the source jets below)
    int convention = 0;   // 0: Convention II, 1: Convention I
    void need_r(int a) { A[a] = true; dH[a] = true; }
    void need_gder(int p, int d) {   // r^p_{nm;d}
        dA[p][d] = true; ddH[p][d] = true; ddH[d][p] = true;
        need_r(p); need_r(d);
    }
};

struct KData {
    int nw = 0;
    std::vector<double> E;
    Mat U, Uadj;
    Mat dH[3], ddH[3][3], Aint[3], dA[3][3], F[3][3], inv, D[3], r[3];
    Mat ddA[3][3][3];   // U' (d_c d_g A_p) U where requested
    // Nonorthogonal models: r = Berry connection, dH diagonal = Hellmann-Feynman slopes and the
    // metric generalized derivatives G[p][d] (position p, derivative d) replace gder.
    bool nonorth = false;
    Mat G[3][3];
    // Metric SHG inputs (nonorthogonal models with an SHG request): the normalized local source
    // jets (hamiltonian derivatives, internal connection, their derivatives), the metric energy
    // Hessians esd[l + n (a + 3 b)] and the isolated-band curvatures iso[l + n (a + 3 b)].
    Mat srcV[3], srcA[3], srcW[3][3], srcdA[3][3];
    std::vector<double> esd, iso;
};

void set_error(const std::string &s) { g_error = s; }

// _r_vector_cartesian (HamiltonianMatrixElements.jl:74-83): R_cart = sum_i r_i * lattice[i,:].
void r_cartesian(const Model &m, int ir, double out[3]) {
    const int64_t *r = &m.rvec[3 * (size_t)ir];
    for (int j = 0; j < 3; ++j)
        out[j] = (double)r[0] * m.lattice[0 + 3 * j] + (double)r[1] * m.lattice[1 + 3 * j] +
                 (double)r[2] * m.lattice[2 + 3 * j];
}

// U' * X * U (transform_to_hamiltonian_gauge!, HamiltonianMatrixElements.jl:61-71).
void rotate(const KData &d, const Mat &x, Mat &out) {
    int n = d.nw;
    Mat t; t.init(n);
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < n; ++l) {
            cd xl = x(l, j);
            for (int i = 0; i < n; ++i) t(i, j) += d.Uadj(i, l) * xl;
        }
    out.init(n);
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < n; ++l) {
            cd ul = d.U(l, j);
            for (int i = 0; i < n; ++i) out(i, j) += t(i, l) * ul;
        }
}

// Cyclic Jacobi eigensolver for the Hermitian matrix given by the upper triangle of `h`
// (Julia's Hermitian(H, :U) view), FP64.  Eigenvalues ascending (stable for ties),
// eigenvector columns in U.  Stands in for LAPACK (DenseSpectra.jl:14-16); both are
// backward stable, so eigenvalues agree to O(eps*||H||).
void hermitian_eigen(const Mat &h, std::vector<double> &evals, Mat &U) {
    int n = h.n;
    Mat a; a.init(n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            if (i == j) a(i, i) = cd(h(i, i).real(), 0.0);
            else { a(i, j) = h(i, j); a(j, i) = std::conj(h(i, j)); }
        }
    Mat v; v.init(n);
    for (int i = 0; i < n; ++i) v(i, i) = 1.0;
    double fro = 0.0;
    for (auto &z : a.v) fro += std::norm(z);
    fro = std::sqrt(fro);
    const double tol = fro * 8.673617379884035e-19;  // 2^-60 * ||H||_F
    for (int sweep = 0; sweep < 60; ++sweep) {
        bool rotated = false;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                cd apq = a(p, q);
                double g = std::abs(apq);
                if (!(g > tol)) continue;
                rotated = true;
                double app = a(p, p).real(), aqq = a(q, q).real();
                cd ph = apq / g;   // e^{i phi}
                double theta = (aqq - app) / (2.0 * g);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0);
                double s = t * c;
                cd sp = s * ph, sm = s * std::conj(ph);
                // A <- A J, J = [[c, s e^{i phi}], [-s e^{-i phi}, c]] on (p,q)
                for (int i = 0; i < n; ++i) {
                    cd aip = a(i, p), aiq = a(i, q);
                    a(i, p) = c * aip - sm * aiq;
                    a(i, q) = sp * aip + c * aiq;
                }
                // A <- J^H A
                for (int j = 0; j < n; ++j) {
                    cd apj = a(p, j), aqj = a(q, j);
                    a(p, j) = c * apj - sp * aqj;
                    a(q, j) = sm * apj + c * aqj;
                }
                a(p, q) = 0.0; a(q, p) = 0.0;
                a(p, p) = cd(a(p, p).real(), 0.0);
                a(q, q) = cd(a(q, q).real(), 0.0);
                for (int i = 0; i < n; ++i) {
                    cd vip = v(i, p), viq = v(i, q);
                    v(i, p) = c * vip - sm * viq;
                    v(i, q) = sp * vip + c * viq;
                }
            }
        if (!rotated) break;
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return a(x, x).real() < a(y, y).real(); });
    evals.resize(n);
    U.init(n);
    for (int j = 0; j < n; ++j) {
        evals[j] = a(order[j], order[j]).real();
        for (int i = 0; i < n; ++i) U(i, j) = v(i, order[j]);
    }
}

// canonicalize_eigenvectors! (HamiltonianMatrixElements.jl:6-25).
void canonicalize(Mat &U) {
    int n = U.n;
    for (int j = 0; j < n; ++j) {
        int pivot = 0;
        double pm = std::abs(U(0, j));
        for (int i = 1; i < n; ++i) {
            double m = std::abs(U(i, j));
            if (m > pm) { pivot = i; pm = m; }
        }
        if (pm > 0.0) {
            cd phase = std::conj(U(pivot, j)) / pm;
            for (int i = 0; i < n; ++i) U(i, j) *= phase;
        }
    }
}

// Generalised Hermitian eigensolve of (H, S) from their upper triangles: S = L L^H, Jacobi on
// L^-1 H L^-H, C = L^-H U (so C^H S C = I), eigenvalues ascending.  Returns false when S is not
// positive definite.
bool generalized_eigen(const Mat &h, const Mat &sm, std::vector<double> &evals, Mat &C) {
    int n = h.n;
    Mat S; S.init(n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            if (i == j) S(i, i) = cd(sm(i, i).real(), 0.0);
            else { S(i, j) = sm(i, j); S(j, i) = std::conj(sm(i, j)); }
        }
    Mat L; L.init(n);
    for (int j = 0; j < n; ++j) {
        double d = S(j, j).real();
        for (int k = 0; k < j; ++k) d -= std::norm(L(j, k));
        if (!(d > 0)) return false;
        L(j, j) = std::sqrt(d);
        for (int i = j + 1; i < n; ++i) {
            cd v = S(i, j);
            for (int k = 0; k < j; ++k) v -= L(i, k) * std::conj(L(j, k));
            L(i, j) = v / L(j, j).real();
        }
    }
    Mat H; H.init(n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            if (i == j) H(i, i) = cd(h(i, i).real(), 0.0);
            else { H(i, j) = h(i, j); H(j, i) = std::conj(h(i, j)); }
        }
    Mat X; X.init(n);   // X = L^-1 H
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            cd v = H(r, c);
            for (int k = 0; k < r; ++k) v -= L(r, k) * X(k, c);
            X(r, c) = v / L(r, r).real();
        }
    Mat Ht; Ht.init(n);   // Ht = X L^-H = (L^-1 X^H)^H
    for (int c = 0; c < n; ++c) {
        std::vector<cd> y(n);
        for (int r = 0; r < n; ++r) {
            cd v = std::conj(X(c, r));
            for (int k = 0; k < r; ++k) v -= L(r, k) * y[k];
            y[r] = v / L(r, r).real();
        }
        for (int r = 0; r < n; ++r) Ht(c, r) = std::conj(y[r]);
    }
    Mat U;
    hermitian_eigen(Ht, evals, U);
    C.init(n);
    for (int c = 0; c < n; ++c)
        for (int r = n - 1; r >= 0; --r) {
            cd v = U(r, c);
            for (int k = r + 1; k < n; ++k) v -= std::conj(L(k, r)) * C(k, c);
            C(r, c) = v / L(r, r).real();
        }
    canonicalize(C);
    return true;
}

// regularized_energy_inverse (PositionVertexRegularization.jl:17-29).
double regularized_inverse(double d, double eta) {
    double den = d * d + eta * eta;
    if (std::isfinite(den) && den != 0.0) return d / den;
    if (!(std::isfinite(d) && std::isfinite(eta) && eta > 0)) return d / den;
    double scale = std::max(std::fabs(d), eta);
    double sd = d / scale, sw = eta / scale;
    return (sd / (sd * sd + sw * sw)) / scale;
}

// Fourier interpolation, eigensolve and Hamiltonian-gauge geometry at one k
// (compute_spectrum! + compute_remaining!, HamiltonianMatrixElements.jl:279-300, 532-563).
void nonorth_kpoint(const Model &m, const Needs &need, const double k[3], double eta, KData &d);

void compute_kpoint(const Model &m, const Needs &need, const double k[3], double eta, KData &d) {
    if (m.has_overlap) { nonorth_kpoint(m, need, k, eta, d); return; }
    int n = m.nw;
    d.nw = n;
    size_t nn = (size_t)n * n;
    // Fourier factors exp(2 pi i R.k)/deg (HamiltonianMatrixElements.jl:28-39).
    std::vector<cd> f(m.nr);
    for (int ir = 0; ir < m.nr; ++ir) {
        const int64_t *r = &m.rvec[3 * (size_t)ir];
        double phase = (double)r[0] * k[0] + (double)r[1] * k[1] + (double)r[2] * k[2];
        f[ir] = std::polar(1.0, 2.0 * PI * phase) / (double)m.deg[ir];
    }
    const bool conv1 = need.convention == 1;
    Mat Hw; Hw.init(n);
    Mat dHw[3], ddHw[3][3], Aw[3], dAw[3][3];
    bool needAw[3];
    for (int a = 0; a < 3; ++a) {
        needAw[a] = need.A[a];
        for (int b = 0; b < 3; ++b) if (need.F[a][b]) { needAw[a] = true; needAw[b] = true; }
    }
    bool needdAw[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            needdAw[a][b] = need.dA[a][b] || need.F[a][b] || need.F[b][a];
    Mat ddAw[3][3][3];
    for (int p = 0; p < 3; ++p)
        for (int c = 0; c < 3; ++c)
            for (int g = 0; g < 3; ++g)
                if (need.ddA[p][c][g]) ddAw[p][c][g].init(n);
    for (int a = 0; a < 3; ++a) {
        if (need.dH[a]) dHw[a].init(n);
        if (needAw[a]) Aw[a].init(n);
        for (int b = 0; b < 3; ++b) {
            if (need.ddH[a][b]) ddHw[a][b].init(n);
            if (needdAw[a][b]) dAw[a][b].init(n);
        }
    }
    // Direct sums in R order (HamiltonianMatrixElements.jl:42-58, 428-460; PositionMatrixElements.jl:294-332).
    // Convention I: per-element displacement R + tau_j - tau_i (_convention_displacement_component,
    // WannierCenterConventionTransforms.jl:85-96) and the centred home-cell connection A - tau
    // (_convention_position_value, :99-113).
    auto disp = [&](const double rc[3], int a, size_t e) {
        if (!conv1) return rc[a];
        const int i = (int)(e % n), j = (int)(e / n);
        return rc[a] + m.tau_cart[a * n + j] - m.tau_cart[a * n + i];
    };
    for (int ir = 0; ir < m.nr; ++ir) {
        double rc[3];
        r_cartesian(m, ir, rc);
        const cd fr = f[ir];
        const cd *h = &m.H[nn * ir];
        for (size_t e = 0; e < nn; ++e) {
            cd fh = fr * h[e];
            Hw.v[e] += fh;
        }
        for (int a = 0; a < 3; ++a) {
            if (need.dH[a]) {
                for (size_t e = 0; e < nn; ++e) dHw[a].v[e] += fr * (I1 * disp(rc, a, e) * h[e]);
            }
            for (int b = 0; b < 3; ++b)
                if (need.ddH[a][b])
                    for (size_t e = 0; e < nn; ++e) ddHw[a][b].v[e] += fr * (-disp(rc, a, e) * disp(rc, b, e) * h[e]);
        }
        if (m.has_position) {
            for (int a = 0; a < 3; ++a) {
                const cd *pa = &m.A[nn * (a + 3 * (size_t)ir)];
                auto pos = [&](size_t e) {
                    cd v = pa[e];
                    if (conv1 && ir == m.home && e % n == e / n) v -= m.tau_cart[a * n + (int)(e % n)];
                    return v;
                };
                if (needAw[a])
                    for (size_t e = 0; e < nn; ++e) Aw[a].v[e] += fr * pos(e);
                for (int b = 0; b < 3; ++b)
                    if (needdAw[a][b])
                        for (size_t e = 0; e < nn; ++e) dAw[a][b].v[e] += fr * (I1 * disp(rc, b, e) * pos(e));
                for (int c = 0; c < 3; ++c)
                    for (int g = 0; g < 3; ++g)
                        if (need.ddA[a][c][g])
                            for (size_t e = 0; e < nn; ++e)
                                ddAw[a][c][g].v[e] += fr * (-disp(rc, c, e) * disp(rc, g, e) * pos(e));
            }
        }
    }
    if (conv1) {
        // D(k)^H X D(k), D = diag(exp(2 pi i k.tau_frac)) (_apply_wannier_center_similarity!, :68-81).
        std::vector<cd> phi(n);
        for (int i = 0; i < n; ++i)
            phi[i] = std::polar(1.0, 2.0 * PI * (k[0] * m.tau_frac[i] + k[1] * m.tau_frac[n + i] + k[2] * m.tau_frac[2 * n + i]));
        auto sim = [&](Mat &X) {
            if (X.n != n) return;
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) X(i, j) *= std::conj(phi[i]) * phi[j];
        };
        sim(Hw);
        for (int a = 0; a < 3; ++a) {
            sim(dHw[a]);
            sim(Aw[a]);
            for (int b = 0; b < 3; ++b) {
                sim(ddHw[a][b]);
                sim(dAw[a][b]);
                for (int g = 0; g < 3; ++g) sim(ddAw[a][b][g]);
            }
        }
    }
    std::vector<double> ev;
    hermitian_eigen(Hw, ev, d.U);
    canonicalize(d.U);
    d.E = ev;
    d.Uadj.init(n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) d.Uadj(i, j) = std::conj(d.U(j, i));
    for (int a = 0; a < 3; ++a) {
        if (need.dH[a]) rotate(d, dHw[a], d.dH[a]);
        if (needAw[a]) rotate(d, Aw[a], d.Aint[a]);
        for (int b = 0; b < 3; ++b) {
            if (need.ddH[a][b]) rotate(d, ddHw[a][b], d.ddH[a][b]);
            if (need.dA[a][b]) rotate(d, dAw[a][b], d.dA[a][b]);
            for (int g = 0; g < 3; ++g)
                if (need.ddA[a][b][g]) rotate(d, ddAw[a][b][g], d.ddA[a][b][g]);
        }
    }
    // Wannier curvature F_ab = dA_b/dk_a - dA_a/dk_b - i[A_a, A_b], then U'FU
    // (PositionMatrixElements.jl:485-556, non-curl branch).
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            if (!need.F[a][b]) continue;
            Mat fw; fw.init(n);
            for (int col = 0; col < n; ++col)
                for (int row = 0; row < n; ++row) {
                    cd val = dAw[b][a](row, col) - dAw[a][b](row, col);
                    for (int l = 0; l < n; ++l)
                        val -= I1 * (Aw[a](row, l) * Aw[b](l, col) - Aw[b](row, l) * Aw[a](l, col));
                    fw(row, col) = val;
                }
            rotate(d, fw, d.F[a][b]);
        }
    // Inverse energy differences (PositionMatrixElements.jl:444-461).
    d.inv.init(n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double diff = d.E[i] - d.E[j];
            if (eta == 0.0) d.inv(i, j) = diff == 0.0 ? 0.0 : 1.0 / diff;
            else d.inv(i, j) = regularized_inverse(diff, eta);
        }
    for (int a = 0; a < 3; ++a) {
        if (!need.dH[a]) continue;
        d.D[a].init(n);
        for (size_t e = 0; e < nn; ++e) d.D[a].v[e] = -d.dH[a].v[e] * d.inv.v[e];
        if (need.A[a]) {
            d.r[a].init(n);
            for (size_t e = 0; e < nn; ++e) d.r[a].v[e] = d.Aint[a].v[e] + I1 * d.D[a].v[e];
        }
    }
}

// Nonorthogonal k-point geometry for the conventional currents: the localized operator sums of
// nonorthogonal_operator_matrices (NonorthogonalMatrixElements.jl:223-283, Convention II), the
// S-orthonormal canonical eigenvectors C, and _nonorthogonal_geometry (:560-817): band-frame
// dH, dS and connection B = r + i dS, the metric eigenvector derivative D, the Berry connection
// i D + B (-> d.r), the Hellmann-Feynman slopes Re(dH_ll - E_l dS_ll) (-> diagonal of d.dH) and
// the generalized derivatives for the requested (position, derivative) pairs (-> d.G).
void nonorth_kpoint(const Model &m, const Needs &need, const double k[3], double eta, KData &d) {
    const int n = m.nw;
    const size_t nn = (size_t)n * n;
    d.nw = n;
    d.nonorth = true;
    Mat h, sm, r[3], dh[3], ds[3], d2h[3][3], d2s[3][3], dr[3][3];
    h.init(n); sm.init(n);
    for (int a = 0; a < 3; ++a) {
        r[a].init(n); dh[a].init(n); ds[a].init(n);
        for (int b = 0; b < 3; ++b) { d2h[a][b].init(n); d2s[a][b].init(n); dr[a][b].init(n); }
    }
    for (int ir = 0; ir < m.nr; ++ir) {
        const int64_t *rv = &m.rvec[3 * (size_t)ir];
        const double phase = (double)rv[0] * k[0] + (double)rv[1] * k[1] + (double)rv[2] * k[2];
        const cd f = std::polar(1.0, 2.0 * PI * phase) / (double)m.deg[ir];
        double rc[3];
        r_cartesian(m, ir, rc);
        const cd *H = &m.H[nn * ir];
        const cd *S = &m.S[nn * ir];
        for (size_t e = 0; e < nn; ++e) { h.v[e] += f * H[e]; sm.v[e] += f * S[e]; }
        for (int a = 0; a < 3; ++a) {
            const cd fa = f * (I1 * rc[a]);
            for (size_t e = 0; e < nn; ++e) { dh[a].v[e] += fa * H[e]; ds[a].v[e] += fa * S[e]; }
            if (m.has_position) {
                const cd *A = &m.A[nn * (a + 3 * (size_t)ir)];
                for (size_t e = 0; e < nn; ++e) r[a].v[e] += f * A[e];
            }
            for (int b = 0; b < 3; ++b) {
                const cd fab = f * (-rc[a] * rc[b]);
                for (size_t e = 0; e < nn; ++e) { d2h[a][b].v[e] += fab * H[e]; d2s[a][b].v[e] += fab * S[e]; }
                if (m.has_position) {
                    const cd *A = &m.A[nn * (a + 3 * (size_t)ir)];
                    const cd fb = f * (I1 * rc[b]);
                    for (size_t e = 0; e < nn; ++e) dr[a][b].v[e] += fb * A[e];
                }
            }
        }
    }
    std::vector<double> ev;
    Mat C;
    if (!generalized_eigen(h, sm, ev, C)) {
        for (double &x : ev) x = std::nan("");
        d.E.assign(n, std::nan(""));
        return;
    }
    d.E = ev;
    d.U = C;
    d.Uadj.init(n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) d.Uadj(i, j) = std::conj(C(j, i));
    auto mulh = [&](const Mat &X, const Mat &Y) {   // X^H Y
        Mat o; o.init(n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                cd v(0.0, 0.0);
                for (int l = 0; l < n; ++l) v += std::conj(X(l, i)) * Y(l, j);
                o(i, j) = v;
            }
        return o;
    };
    auto mul = [&](const Mat &X, const Mat &Y) {
        Mat o; o.init(n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                cd v(0.0, 0.0);
                for (int l = 0; l < n; ++l) v += X(i, l) * Y(l, j);
                o(i, j) = v;
            }
        return o;
    };
    auto f_of = [&](double gap) { return eta == 0.0 ? 1.0 / gap : gap / (gap * gap + eta * eta); };
    auto fp_of = [&](double gap) {
        return eta == 0.0 ? -1.0 / (gap * gap) : (eta * eta - gap * gap) / ((gap * gap + eta * eta) * (gap * gap + eta * eta));
    };
    Mat dhb[3], dsb[3], conn[3], numer[3];
    std::vector<double> ed((size_t)n * 3);
    for (int a = 0; a < 3; ++a) {
        rotate(d, dh[a], dhb[a]);
        rotate(d, ds[a], dsb[a]);
        Mat B; B.init(n);
        for (size_t e = 0; e < nn; ++e) B.v[e] = r[a].v[e] + I1 * ds[a].v[e];
        rotate(d, B, conn[a]);
        numer[a].init(n);
        d.D[a].init(n);
        for (int mm = 0; mm < n; ++mm)
            for (int l = 0; l < n; ++l) {
                numer[a](l, mm) = dhb[a](l, mm) - (ev[l] + ev[mm]) * dsb[a](l, mm) / 2.0;
                if (l == mm) d.D[a](l, l) = -dsb[a](l, l) / 2.0 + I1 * conn[a](l, l).real();
                else d.D[a](l, mm) = -dsb[a](l, mm) / 2.0 + numer[a](l, mm) * f_of(ev[mm] - ev[l]);
            }
        for (int l = 0; l < n; ++l) ed[l + (size_t)n * a] = (dhb[a](l, l) - ev[l] * dsb[a](l, l)).real();
        d.r[a].init(n);
        for (size_t e = 0; e < nn; ++e) d.r[a].v[e] = I1 * d.D[a].v[e] + conn[a].v[e];
        d.dH[a] = dhb[a];
        for (int l = 0; l < n; ++l) d.dH[a](l, l) = ed[l + (size_t)n * a];
        d.Aint[a] = conn[a];
    }
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) {
            if (!need.dA[p][q]) continue;
            const Mat &Dd = d.D[q];
            Mat hd = mulh(Dd, dhb[p]), sd = mulh(Dd, dsb[p]), bd = mulh(Dd, conn[p]);
            Mat t1 = mul(dhb[p], Dd), t2 = mul(dsb[p], Dd), t3 = mul(conn[p], Dd);
            Mat rh, rs, rb, X;
            rotate(d, d2h[p][q], rh);
            rotate(d, d2s[p][q], rs);
            X.init(n);
            for (size_t e = 0; e < nn; ++e) X.v[e] = dr[p][q].v[e] + I1 * d2s[p][q].v[e];
            rotate(d, X, rb);
            for (size_t e = 0; e < nn; ++e) {
                hd.v[e] += t1.v[e] + rh.v[e];
                sd.v[e] += t2.v[e] + rs.v[e];
                bd.v[e] += t3.v[e] + rb.v[e];
            }
            Mat &G = d.G[p][q];
            G.init(n);
            for (int mm = 0; mm < n; ++mm)
                for (int l = 0; l < n; ++l) {
                    if (l == mm) continue;
                    const double gap = ev[mm] - ev[l];
                    const double edl = ed[l + (size_t)n * q], edm = ed[mm + (size_t)n * q];
                    const cd nd = hd(l, mm) - (ev[l] + ev[mm]) * sd(l, mm) / 2.0 - (edl + edm) * dsb[p](l, mm) / 2.0;
                    const cd dd = -sd(l, mm) / 2.0 + nd * f_of(gap) + numer[p](l, mm) * fp_of(gap) * (edm - edl);
                    G(l, mm) = I1 * dd + bd(l, mm) - I1 * (d.r[q](l, l) - d.r[q](mm, mm)) * d.r[p](l, mm);
                }
        }
    if (!need.shg) return;
    // Metric SHG inputs.
    Mat rot2h[3][3], rot2s[3][3], rotB[3][3];   // C^H d2H_ab C, C^H d2S_ab C, C^H (dr_ab + i d2S_ab) C
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            rotate(d, d2h[a][b], rot2h[a][b]);
            rotate(d, d2s[a][b], rot2s[a][b]);
            Mat X; X.init(n);
            for (size_t e = 0; e < nn; ++e) X.v[e] = dr[a][b].v[e] + I1 * d2s[a][b].v[e];
            rotate(d, X, rotB[a][b]);
        }
    // Normalized local source jets (_prepare_nonorthogonal_optical_cutoff!,
    // NonorthogonalOpticalCutoffVertices.jl:67-186): with k_a = C^H dH_a C, g_a = C^H dS_a C and
    // raw_a = C^H (r_a + i dS_a) C,
    //   V_a = k_a - (E_i + E_j) g_a / 2,   A_a = raw_a - i g_a / 2,
    //   z_ab = -C^H d2S_ab C / 2 + 3 (g_a g_b + g_b g_a) / 8,
    //   W_ab = C^H d2H_ab C - (g_a k_b + k_b g_a + g_b k_a + k_a g_b) / 2
    //          + (g_a E g_b + g_b E g_a) / 4 + (E_i + E_j) z_ab,
    //   dA_ab = C^H (dr_ab + i d2S_ab) C - (g_b raw_a + raw_a g_b) / 2 + i (z_ab - g_b g_a / 4).
    for (int a = 0; a < 3; ++a) {
        d.srcV[a] = numer[a];
        d.srcA[a].init(n);
        for (size_t e = 0; e < nn; ++e) d.srcA[a].v[e] = conn[a].v[e] - 0.5 * I1 * dsb[a].v[e];
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const Mat &ga = dsb[a], &gb = dsb[b], &ka = dhb[a], &kb = dhb[b];
            Mat gagb = mul(ga, gb), gbga = mul(gb, ga);
            Mat z; z.init(n);
            for (size_t e = 0; e < nn; ++e) z.v[e] = -0.5 * rot2s[a][b].v[e] + 0.375 * (gagb.v[e] + gbga.v[e]);
            Mat Egb, Ega;
            Egb.init(n); Ega.init(n);
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) { Egb(i, j) = ev[i] * gb(i, j); Ega(i, j) = ev[i] * ga(i, j); }
            Mat p1 = mul(ga, kb), p2 = mul(kb, ga), p3 = mul(gb, ka), p4 = mul(ka, gb);
            Mat q1 = mul(ga, Egb), q2 = mul(gb, Ega);
            Mat &W = d.srcW[a][b];
            W.init(n);
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    const size_t e = (size_t)i + (size_t)n * j;
                    W.v[e] = rot2h[a][b].v[e] - 0.5 * (p1.v[e] + p2.v[e] + p3.v[e] + p4.v[e]) +
                             0.25 * (q1.v[e] + q2.v[e]) + (ev[i] + ev[j]) * z.v[e];
                }
            Mat r1 = mul(gb, conn[a]), r2 = mul(conn[a], gb);
            Mat &dA = d.srcdA[a][b];
            dA.init(n);
            for (size_t e = 0; e < nn; ++e)
                dA.v[e] = rotB[a][b].v[e] - 0.5 * (r1.v[e] + r2.v[e]) + I1 * (z.v[e] - 0.25 * gbga.v[e]);
        }
    // Metric energy Hessians (_nonorthogonal_geometry, NonorthogonalMatrixElements.jl:660-727):
    // with hd = D_b^H dh_a + dh_a D_b + C^H d2H_ab C and sd likewise from ds,
    // esd[l, a, b] = Re(hd_ll - E_l sd_ll - v_l^b ds_ll^a).
    d.esd.assign((size_t)n * 9, 0.0);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const Mat &Db = d.D[b];
            for (int l = 0; l < n; ++l) {
                cd hd = rot2h[a][b](l, l), sd = rot2s[a][b](l, l);
                for (int q = 0; q < n; ++q) {
                    hd += std::conj(Db(q, l)) * dhb[a](q, l) + dhb[a](l, q) * Db(q, l);
                    sd += std::conj(Db(q, l)) * dsb[a](q, l) + dsb[a](l, q) * Db(q, l);
                }
                d.esd[l + (size_t)n * (a + 3 * b)] =
                    (hd - ev[l] * sd - ed[l + (size_t)n * b] * dsb[a](l, l)).real();
            }
        }
    // Isolated-band curvature (isolated_band_curvature, NonorthogonalMatrixElements.jl:1141-1185)
    // with the band-frame ambient metric curvature (_nonorthogonal_ambient_curvature, :819-878):
    // using S^-1 = C C^H, its diagonal is
    //   (B_b;a - g_a B_b - B_a;b + g_b B_a - i (B_a B_b - B_b B_a))_nn,
    // B_a = C^H (r_a + i dS_a) C and B_a;b = C^H (dr_ab + i d2S_ab) C.
    auto bare_inv = [](double x) { return std::fabs(x) < 1.0e-7 ? 0.0 : 1.0 / x; };
    d.iso.assign((size_t)n * 9, 0.0);
    for (int l = 0; l < n; ++l) {
        cd row[3][128], col[3][128];
        for (int mm = 0; mm < n; ++mm) {
            if (mm == l) continue;
            const double inv = bare_inv(ev[mm] - ev[l]), rinv = bare_inv(ev[l] - ev[mm]);
            const double avg = 0.5 * (ev[l] + ev[mm]);
            for (int a = 0; a < 3; ++a) {
                const cd fw = conn[a](l, mm), rv = conn[a](mm, l);
                const cd mf = -I1 * (fw - std::conj(rv)), mr = -I1 * (rv - std::conj(fw));
                const cd ff = 0.5 * (fw + std::conj(rv)), fr = 0.5 * (rv + std::conj(fw));
                const cd nf = dhb[a](l, mm) - avg * mf, nr = dhb[a](mm, l) - avg * mr;
                row[a][mm] = inv == 0.0 ? ff : ff + I1 * nf * inv;
                col[a][mm] = rinv == 0.0 ? fr : fr + I1 * nr * rinv;
            }
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                if (a == b) continue;
                cd band = rotB[b][a](l, l) - rotB[a][b](l, l);
                for (int q = 0; q < n; ++q) {
                    band += -dsb[a](l, q) * conn[b](q, l) + dsb[b](l, q) * conn[a](q, l) -
                            I1 * (conn[a](l, q) * conn[b](q, l) - conn[b](l, q) * conn[a](q, l));
                }
                double value = band.real();
                for (int mm = 0; mm < n; ++mm) {
                    if (mm == l) continue;
                    value -= 2.0 * (row[a][mm] * col[b][mm]).imag();
                }
                d.iso[l + (size_t)n * (a + 3 * b)] = value;
            }
    }
}

// conventional_generalized_position_derivative_element (ConventionalShiftCurrent.jl:191-229):
// r^a_{nm;b} with a the position axis and b the derivative axis.
cd gder(const KData &d, int n, int m, int a, int b) {
    if (d.nonorth) return d.G[a][b](n, m);
    cd sum_AD(0.0, 0.0), sum_HD(0.0, 0.0);
    for (int l = 0; l < d.nw; ++l) {
        if (l != n && l != m) {
            sum_AD += d.Aint[a](n, l) * d.D[b](l, m) - d.D[b](n, l) * d.Aint[a](l, m);
            sum_HD += d.dH[a](n, l) * d.D[b](l, m) - d.D[b](n, l) * d.dH[a](l, m);
        }
    }
    cd AD_bit = (d.Aint[b](n, n) - d.Aint[b](m, m)) * d.D[a](n, m) +
                (d.Aint[a](n, n) - d.Aint[a](m, m)) * d.D[b](n, m);
    cd AA_bit = (d.Aint[b](n, n) - d.Aint[b](m, m)) * d.Aint[a](n, m);
    cd DV_bit = (d.dH[b](n, n) - d.dH[b](m, m)) * d.D[a](n, m) +
                (d.dH[a](n, n) - d.dH[a](m, m)) * d.D[b](n, m);
    return d.dA[a][b](n, m) + AD_bit - I1 * AA_bit + sum_AD +
           I1 * (d.ddH[a][b](n, m) + sum_HD + DV_bit) * (-d.inv(n, m));
}

// fermi_dirac! (CalculationUtils.jl:28-46).
void fermi(const std::vector<double> &E, double mu, double T, std::vector<double> &f) {
    double kt = BOLTZMANN_CONSTANT_EV_K * T;
    f.resize(E.size());
    for (size_t i = 0; i < E.size(); ++i) {
        if (kt == 0.0) f[i] = E[i] <= mu ? 1.0 : 0.0;
        else {
            double arg = std::min(700.0, std::max(-700.0, (E[i] - mu) / kt));
            f[i] = 1.0 / (std::exp(arg) + 1.0);
        }
    }
}

struct Screen {
    bool active = false;
    std::vector<double> fnm;     // [n + nw*m]
    std::vector<double> delta;   // [w + nom*(n + nw*m)]
    std::vector<char> mask;      // [n + nw*m]
};

// Effective band window [lo, hi) (0-based) of _prepare_transition_selection_window!
// (TransitionScreening.jl:201-233): select_band_window (CalculationUtils.jl:71-90) around mu, then,
// for a finite window, widened to whole response degeneracy groups
// (_mark_response_degeneracy_groups!, ResponseDegeneracyGroups.jl:10-33).  lo = hi = 0: no bands.
void band_window(const std::vector<double> &E, const wnlqg_task_desc &t, int &lo, int &hi) {
    const int n = (int)E.size();
    const int size = t.band_window_size;
    if (size == -1 || 2 * size > n) { lo = 0; hi = n; return; }
    int valence = 0;   // searchsortedlast: number of energies <= mu
    while (valence < n && E[valence] <= t.fermi_energy) ++valence;
    if (valence < 1 || valence >= n) { lo = 0; hi = 0; return; }
    int start = std::max(1, valence - size + 1), end = std::min(n, valence + size);   // 1-based inclusive
    double emax = 0.0;
    for (double e : E) emax = std::max(emax, std::fabs(e));
    const double equal = 32.0 * 2.220446049250313e-16 * std::max(1.0, emax);
    auto joined = [&](int b) {   // bands b and b+1 (1-based) in one group
        const double gap = E[b] - E[b - 1];
        return gap < t.degeneracy_threshold || gap <= equal;
    };
    while (start > 1 && joined(start - 1)) --start;
    while (end < n && joined(end)) ++end;
    lo = start - 1;
    hi = end;
}

// _fill_transition_screen! (TransitionScreening.jl:32-94) with the pair lists of
// _record_active_transition_pairs! (:126-162) restricted to the effective band window.
void fill_screen(const std::vector<double> &E, const std::vector<double> &f,
                 const wnlqg_task_desc &t, Screen &s) {
    int n = (int)E.size();
    int wlo = 0, whi = 0;
    band_window(E, t, wlo, whi);
    int64_t nom = t.num_photon_energies;
    bool gaussian = t.broadening_type == WNLQG_GAUSSIAN;
    double eta = t.broadening;
    double cutoff = eta * std::sqrt(200.0);
    double gscale = gaussian ? 1.0 / (std::sqrt(PI) * eta) : 0.0;
    double thr = t.transition_window_factor * eta;
    s.active = false;
    s.fnm.assign((size_t)n * n, 0.0);
    s.delta.assign((size_t)nom * n * n, 0.0);
    s.mask.assign((size_t)n * n, 0);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            double od = f[a] - f[b];
            s.fnm[a + (size_t)n * b] = od;
            double te = E[b] - E[a];
            // Explicit interband selection (_fill_transition_screen!, TransitionScreening.jl:57-61):
            // source (valence) band a, target (conduction) band b.
            const bool selected = !t.use_band_selection || (((t.valence_bands[a >> 5] >> (a & 31)) & 1u) &&
                                                            ((t.conduction_bands[b >> 5] >> (b & 31)) & 1u));
            bool occ = selected && std::fabs(od) > 1.0e-10 && a >= wlo && a < whi && b >= wlo && b < whi;
            bool pair_active = occ && !gaussian;
            if (occ && !gaussian && thr <= 0) s.active = true;
            for (int64_t w = 0; w < nom; ++w) {
                double x = te - t.photon_energies[w];
                bool inside = false;
                double dv;
                if (gaussian) {
                    inside = std::fabs(x) < cutoff;
                    dv = inside ? gscale * std::exp(-(x / eta) * (x / eta)) : 0.0;
                    pair_active = pair_active || (occ && inside);
                } else {
                    dv = (eta / PI) / (x * x + eta * eta);
                }
                s.delta[w + nom * (a + (size_t)n * b)] = dv;
                if (occ && (gaussian ? inside : (thr > 0 && std::fabs(x) < thr))) s.active = true;
            }
            s.mask[a + (size_t)n * b] = pair_active ? 1 : 0;
        }
}

struct Task {
    wnlqg_task_desc desc;
    std::vector<double> omegas, mus;
    Needs need;
    int64_t value_count = 0;
    // Spectral isolation contract: -1 none, 0 every pair split by more than iso_tol
    // (geometry_isolated_spectrum_minimum_gap), 1 spectral blocks (spectral_subspace_blocks).
    int iso_mode = -1;
    double iso_tol = 0.0;
};

// geometry_isolated_spectrum_minimum_gap (MatrixElements/Interpolated/OrthogonalBandDerivatives.jl:66-82):
// every pair (l < m, loop over m then l) must be split by more than the tolerance.
std::string isolated_spectrum_error(const std::vector<double> &E, double tol) {
    for (double e : E)
        if (!std::isfinite(e)) return "empty/nonfinite geometry spectrum";
    char buf[200];
    for (size_t m = 0; m < E.size(); ++m)
        for (size_t l = 0; l < m; ++l) {
            const double gap = std::fabs(E[m] - E[l]);
            if (!(gap > tol)) {
                std::snprintf(buf, sizeof(buf),
                              "GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED: bands=(%d,%d), gap_ev=%.17g, threshold_ev=%.17g",
                              (int)l + 1, (int)m + 1, gap, tol);
                return buf;
            }
        }
    return "";
}

// spectral_subspace_blocks (MatrixElements/Interpolated/SubspacePositionMatrixElements.jl:5-22):
// levels within 32 eps max(1, max|E|) of a block's first level join it; a new block must be split
// from the previous level by more than the tolerance.  Returns the 0-based first index of each
// block followed by E.size(), or sets err.
std::vector<int> spectral_blocks(const std::vector<double> &E, double tol, std::string &err) {
    std::vector<int> starts;
    for (double e : E)
        if (!std::isfinite(e)) { err = "Invalid spectrum"; return starts; }
    double emax = 0.0;
    for (double e : E) emax = std::max(emax, std::fabs(e));
    const double exact = 32.0 * 2.220446049250313e-16 * std::max(1.0, emax);
    int start = 0;
    starts.push_back(0);
    for (int n = 1; n < (int)E.size(); ++n) {
        if (E[n] - E[start] > exact) {
            const double adjacent = E[n] - E[n - 1];
            if (!(adjacent > tol)) {
                char buf[120];
                std::snprintf(buf, sizeof(buf), "SPECTRAL_CROSS_BLOCK_GAP_UNRESOLVED: gap=%.17g eV", adjacent);
                err = buf;
                return starts;
            }
            starts.push_back(n);
            start = n;
        }
    }
    starts.push_back((int)E.size());
    return starts;
}

// response_occupation (Responses/Shared/ResponseOccupations.jl:8-14).
double response_occupation(double e, double mu, double T) {
    if (T == 0.0) return e < mu ? 1.0 : (e > mu ? 0.0 : 0.5);
    const double x = (e - mu) / (RESPONSE_KB_EV * T);
    const double z = std::exp(-std::fabs(x));
    return x >= 0 ? z / (1 + z) : 1 / (1 + z);
}

bool build_task(const wnlqg_task_desc *t, Task &task) {
    task.desc = *t;
    if (t->num_photon_energies < 0 || t->num_fermi_energies < 0) { set_error("negative axis length"); return false; }
    if (t->wannier_center_convention != 0 && t->wannier_center_convention != 1) {
        set_error("wannier_center_convention must be 0 (II) or 1 (I)");
        return false;
    }
    task.need.convention = t->wannier_center_convention;
    if (t->use_band_selection) {
        // validate_interband_band_selection (CalculationUtils.jl:501-522).
        bool any_v = false, any_c = false, overlap = false;
        for (int w = 0; w < 4; ++w) {
            any_v |= t->valence_bands[w] != 0;
            any_c |= t->conduction_bands[w] != 0;
            overlap |= (t->valence_bands[w] & t->conduction_bands[w]) != 0;
        }
        if (!any_v || !any_c) { set_error("band_selection groups must be nonempty and inside the orbitals"); return false; }
        if (overlap) { set_error("band_selection groups must not overlap"); return false; }
        if (t->band_window_size != -1) { set_error("band_selection together with a band window is not built"); return false; }
    }
    task.omegas.assign(t->photon_energies, t->photon_energies + t->num_photon_energies);
    if (t->num_fermi_energies > 0) task.mus.assign(t->fermi_energies, t->fermi_energies + t->num_fermi_energies);
    task.desc.photon_energies = task.omegas.data();
    task.desc.fermi_energies = task.mus.data();
    if (!(t->broadening > 0) || !std::isfinite(t->broadening)) { set_error("broadening must be finite and positive"); return false; }
    if (!(t->denominator_regularization >= 0)) { set_error("denominator_regularization must be >= 0"); return false; }
    if (!(std::isfinite(t->spectral_gap_tolerance) && t->spectral_gap_tolerance >= 0)) {
        set_error("invalid spectral isolation threshold");
        return false;
    }
    if (t->num_responses < 1 || t->num_responses > WNLQG_MAX_RESPONSES) { set_error("num_responses out of range"); return false; }
    int64_t count = 0;
    for (int r = 0; r < t->num_responses; ++r) {
        const wnlqg_response_request &q = t->responses[r];
        if (q.num_components < 1 || q.num_components > WNLQG_MAX_COMPONENTS) { set_error("num_components out of range"); return false; }
        for (int c = 0; c < q.num_components; ++c) {
            const int32_t *x = q.components[c];
            for (int i = 0; i < 4; ++i)
                if (x[i] < 0 || x[i] > 2) { set_error("component axis out of range"); return false; }
            int a = x[0], b = x[1], cc = x[2], dd = x[3];
            switch (q.kind) {
            case WNLQG_SHIFT_CURRENT:
                task.need.need_gder(cc, a); task.need.need_gder(b, a);
                task.need.need_r(b); task.need.need_r(cc);
                break;
            case WNLQG_INJECTION_CURRENT:
                task.need.dH[a] = true; task.need.need_r(b); task.need.need_r(cc);
                break;
            case WNLQG_BERRY_CURVATURE:
                task.need.F[a][b] = true; task.need.need_r(a); task.need.need_r(b);
                break;
            case WNLQG_QUANTUM_METRIC:
                task.need.need_r(a); task.need.need_r(b);
                break;
            case WNLQG_INTRINSIC_AHC:
            case WNLQG_BERRY_DIPOLE:
            case WNLQG_LINEAR_TRANSPORT_BERRY:
            case WNLQG_BERRY_DIPOLE_SEA:
                task.need.F[a][b] = true; task.need.need_r(a); task.need.need_r(b);
                if (q.kind == WNLQG_BERRY_DIPOLE_SEA && t->derivative_backend == 1) {
                    // Jets of orthogonal_bcd_partition_matrices! (OrthogonalGeometryDerivatives.jl:24-102)
                    // and of the band derivatives D_a, D_c, D_ac, D_bc (OrthogonalBandDerivatives.jl:123-245).
                    task.need.need_r(cc);
                    task.need.ddH[a][cc] = task.need.ddH[cc][a] = true;
                    task.need.ddH[b][cc] = task.need.ddH[cc][b] = true;
                    task.need.dA[a][cc] = task.need.dA[b][cc] = true;
                    task.need.dA[b][a] = task.need.dA[a][b] = true;
                    task.need.dA[cc][a] = task.need.dA[cc][b] = true;
                    task.need.ddA[b][a][cc] = task.need.ddA[a][b][cc] = true;
                }
                if (q.kind == WNLQG_BERRY_DIPOLE) task.need.dH[cc] = true;
                break;
            case WNLQG_SECOND_HARMONIC:
                task.need.shg = true;
                for (int x = 0; x < 3; ++x) {
                    task.need.dH[x] = true; task.need.A[x] = true;
                    for (int y = 0; y < 3; ++y) { task.need.dA[x][y] = true; task.need.ddH[x][y] = true; }
                }
                break;
            case WNLQG_JERK_CURRENT:
                task.need.need_r(b); task.need.need_r(cc);
                task.need.dH[a] = true; task.need.dH[dd] = true;
                task.need.ddH[a][dd] = true;
                break;
            default:
                set_error("response kind not implemented by the oracle"); return false;
            }
        }
        if (q.kind == WNLQG_SHIFT_CURRENT || q.kind == WNLQG_INJECTION_CURRENT || q.kind == WNLQG_JERK_CURRENT)
            count += q.num_components * t->num_photon_energies;
        else if (q.kind == WNLQG_SECOND_HARMONIC) {
            // second_harmonic_response! argument checks (SecondHarmonicKernels.jl:129-138).
            const double eta = t->shg_intermediate_regularization > 0 ? t->shg_intermediate_regularization
                                                                      : t->denominator_regularization;
            if (!(std::isfinite(t->shg_low_frequency_broadening) && t->shg_low_frequency_broadening > 0 &&
                  std::isfinite(eta) && eta > 0)) {
                set_error("SHG optical widths and intermediate_regularization must be finite and positive in eV");
                return false;
            }
            if (!(std::isfinite(t->degeneracy_threshold) && t->degeneracy_threshold >= 0)) {
                set_error("SHG degeneracy_threshold must be finite and nonnegative in eV");
                return false;
            }
            count += q.num_components * t->num_photon_energies * 14;
        }
        else if (q.kind == WNLQG_INTRINSIC_AHC || q.kind == WNLQG_BERRY_DIPOLE || q.kind == WNLQG_LINEAR_TRANSPORT_BERRY ||
                 q.kind == WNLQG_BERRY_DIPOLE_SEA) {
            // intrinsic_hall_fermi_sea (IntrinsicHallOccupations.jl:15-16) is zero-temperature only.
            if (q.kind == WNLQG_INTRINSIC_AHC && t->temperature != 0.0) {
                set_error("INTRINSIC_HALL_REQUIRES_ZERO_TEMPERATURE"); return false;
            }
            if (q.kind == WNLQG_LINEAR_TRANSPORT_BERRY) {
                // spectral_response_geometry(data) (SpectralResponseGeometry.jl:61-66).
                if (!(std::isfinite(t->denominator_regularization) && t->denominator_regularization > 0)) {
                    set_error("spectral position regularization must be finite and positive"); return false;
                }
                if (!(std::isfinite(t->linear_transport_gamma_inter) && t->linear_transport_gamma_inter >= 0)) {
                    set_error("gamma_inter_ev must be finite and nonnegative"); return false;
                }
            }
            if (t->num_fermi_energies < 1) { set_error("a Fermi-energy axis is required"); return false; }
            if (q.kind == WNLQG_BERRY_DIPOLE_SEA && t->derivative_backend != 0 && t->derivative_backend != 1) {
                set_error("derivative_backend must be 0 (finite difference) or 1 (analytic)"); return false;
            }
            if (q.kind == WNLQG_BERRY_DIPOLE_SEA && t->derivative_backend == 0 &&
                !(std::isfinite(t->finite_difference_step) && t->finite_difference_step > 0)) {
                set_error("finite_difference_step must be finite and positive"); return false;
            }
            if (q.kind == WNLQG_BERRY_DIPOLE && t->temperature == 0.0 && !(t->fermi_surface_broadening > 0)) {
                set_error("T=0 requires positive eta_fs_ev"); return false;
            }
            count += q.num_components * t->num_fermi_energies;
        } else
            count += q.num_components;
    }
    task.value_count = count;
    // Isolation contract (BerryMultipoleGeometry.jl:81 with degeneracy_threshold; the eta = 0 gauge
    // correction, PositionMatrixElements.jl:447-452, with spectral_gap_tolerance; the linear
    // transport Berry channel's spectral blocks with spectral_gap_tolerance).
    bool dipole = false, exact = false, blocks = false;
    for (int r = 0; r < t->num_responses; ++r) {
        const int kind = t->responses[r].kind;
        dipole |= kind == WNLQG_BERRY_DIPOLE || kind == WNLQG_BERRY_DIPOLE_SEA;
        exact |= t->denominator_regularization == 0.0 &&
                 (kind == WNLQG_SHIFT_CURRENT || kind == WNLQG_INJECTION_CURRENT || kind == WNLQG_BERRY_CURVATURE ||
                  kind == WNLQG_QUANTUM_METRIC || kind == WNLQG_BERRY_DIPOLE || kind == WNLQG_BERRY_DIPOLE_SEA);
        blocks |= kind == WNLQG_LINEAR_TRANSPORT_BERRY;
    }
    if (dipole && !(std::isfinite(t->degeneracy_threshold) && t->degeneracy_threshold >= 0)) {
        set_error("invalid spectral isolation threshold");
        return false;
    }
    if (dipole || exact) {
        task.iso_mode = 0;
        task.iso_tol = std::max(dipole ? t->degeneracy_threshold : 0.0, exact ? t->spectral_gap_tolerance : 0.0);
    } else if (blocks) {
        task.iso_mode = 1;
        task.iso_tol = t->spectral_gap_tolerance;
    }
    return true;
}

// Jerk Eq. 9.20 from prepared band data (ConventionalJerkCurrent.jl:14-65 with
// prepare_third_order_band_geometry!, ThirdOrderGeometry.jl:131-160, and
// _fill_jerk_current_dipoles!, ThirdOrderGeometry.jl:28-41).  B = dH, A = internal
// connection, C = ddH, all in the Hamiltonian gauge; out[w + nom*comp].
void jerk_response(int n, const double *E, const cd *B, const cd *A, const cd *C, int64_t nom,
                   const double *om, double mu, double T, double width, bool gaussian, double reg,
                   double window, int ncomp, const int32_t (*comps)[4], cd *out) {
    auto b3 = [&](int i, int j, int a) { return B[i + n * (j + n * a)]; };
    auto a3 = [&](int i, int j, int a) { return A[i + n * (j + n * a)]; };
    auto c4 = [&](int i, int j, int a, int dd) { return C[i + n * (j + n * (a + 3 * dd))]; };
    std::vector<double> hess((size_t)n * 9);
    std::vector<cd> dip((size_t)n * n * 3);
    for (int nn = 0; nn < n; ++nn)
        for (int a = 0; a < 3; ++a)
            for (int dd = 0; dd < 3; ++dd) {
                double value = c4(nn, nn, a, dd).real();
                for (int l = 0; l < n; ++l) {
                    if (l == nn) continue;
                    double gap = E[nn] - E[l];
                    double inverse = gap / (gap * gap + reg * reg);
                    value += 2.0 * (b3(nn, l, a) * b3(l, nn, dd)).real() * inverse;
                }
                hess[nn + n * (a + 3 * dd)] = value;
            }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int a = 0; a < 3; ++a) {
                double gap = E[i] - E[j];
                dip[i + n * (j + n * a)] = i == j ? cd(0.0, 0.0)
                                                  : a3(i, j, a) - I1 * b3(i, j, a) * gap / (gap * gap + reg * reg);
            }
    std::vector<double> occ;
    std::vector<double> Ev(E, E + n);
    fermi(Ev, mu, T, occ);
    for (int64_t e = 0; e < nom * ncomp; ++e) out[e] = 0.0;
    for (int m = 0; m < n; ++m)
        for (int nn = 0; nn < n; ++nn) {
            double gap = E[nn] - E[m];
            if (!(gap > 0)) continue;
            double o = occ[m] - occ[nn];
            for (int64_t w = 0; w < nom; ++w) {
                double energy = om[w];
                if (window > 0 && std::fabs(gap - energy) > window * width) continue;
                double x = (gap - energy) / width;
                double delta = gaussian ? std::exp(-x * x) / (std::sqrt(PI) * width)
                                        : 1.0 / (PI * width * (1 + x * x));
                double weight = o * delta;
                for (int c = 0; c < ncomp; ++c) {
                    int a = comps[c][0], b = comps[c][1], cc = comps[c][2], dd = comps[c][3];
                    cd optical = dip[nn + n * (m + n * b)] * dip[m + n * (nn + n * cc)];
                    out[w + nom * c] += weight * optical *
                                        (hess[nn + n * (a + 3 * dd)] - hess[m + n * (a + 3 * dd)]);
                }
            }
        }
}

// ---------------------------------------------------------------------------------------------
// Second-harmonic generation (src/Responses/SecondHarmonicGeneration/SecondHarmonicKernels.jl).
// Inputs are prepared Hamiltonian-gauge band data at one k, all [n,n,...] column-major:
// V = dH (velocity, [n,n,3]), A = internal connection ([n,n,3]), dA = connection derivatives
// ([n,n,3,3], position axis then derivative axis), W = second Hamiltonian derivatives ([n,n,3,3]).
// out[w + nom*(c + nc*(term + 7*q))] for term 0..6 (SECOND_HARMONIC_TERMS order) and quantity q
// (0 = susceptibility, 1 = conductivity, both before their physical prefactors).

// bare_energy_inverse (PositionVertexRegularization.jl:7-8): zero strictly below 1e-7 eV.
double bare_inverse(double d) { return std::fabs(d) < 1.0e-7 ? 0.0 : 1.0 / d; }

// regularized_energy_weight (PositionVertexRegularization.jl:37-50): eta^2/(d^2+eta^2).
double regularized_weight(double d, double eta) {
    double w2 = eta * eta, den = d * d + w2;
    if (std::isfinite(den) && den != 0.0 && w2 != 0.0) return w2 / den;
    if (!(std::isfinite(d) && std::isfinite(eta) && eta > 0)) return w2 / den;
    double scale = std::max(std::fabs(d), eta), sd = d / scale, sw = eta / scale;
    return sw * sw / (sd * sd + sw * sw);
}

// second_harmonic_delta / _principal / _resonance (SecondHarmonicKernels.jl:86-98).
double shg_delta(double e, double width, bool gaussian) {
    double x = e / width;
    return gaussian ? std::exp(-x * x) / (std::sqrt(PI) * width) : 1.0 / (PI * width * (1 + x * x));
}
double shg_principal(double e, double width) { return e / (e * e + width * width); }
cd shg_resonance(double e, double width, bool gaussian) {
    return cd(shg_principal(e, width), PI * shg_delta(e, width, gaussian));
}

// second_harmonic_occupation (SecondHarmonicKernels.jl:101-105).
double shg_occupation(double e, double mu, double T) {
    if (T <= 1.0e-7) return e <= mu ? 1.0 : 0.0;
    double x = (e - mu) / (RESPONSE_KB_EV * T);
    return x >= 0 ? std::exp(-x) / (1 + std::exp(-x)) : 1.0 / (1 + std::exp(x));
}

struct ShgParams {
    double mu, T, width, low_width, eta, degeneracy;
    bool gaussian, eta_correction;
    // Metric (nonorthogonal) models: the vertices take the geometry width vertex_eta, r_eta is
    // the metric Berry connection, and the Hessians and isolated-band curvatures are the metric
    // ones (SecondHarmonicKernels.jl:47-68, NonorthogonalMatrixElements.jl:1088-1139).
    double vertex_eta = -1.0;                 // < 0: the energy-sum width eta
    const cd *rdip = nullptr;                  // [n*n*3]
    const double *hess = nullptr, *curv = nullptr;   // [n*9], index l + n (a + 3 b)
};

void shg_response(int n, const double *E, const cd *V, const cd *A, const cd *dA, const cd *W, int64_t nom,
                  const double *om, int nc, const int32_t (*comps)[4], const ShgParams &p, cd *out) {
    auto v3 = [&](int i, int j, int a) { return V[i + n * (j + n * a)]; };
    auto a3 = [&](int i, int j, int a) { return A[i + n * (j + n * a)]; };
    auto da4 = [&](int i, int j, int a, int b) { return dA[i + n * (j + n * (a + 3 * b))]; };
    auto w4 = [&](int i, int j, int a, int b) { return W[i + n * (j + n * (a + 3 * b))]; };
    const size_t nn = (size_t)n * n;
    for (int64_t e = 0; e < nom * nc * 14; ++e) out[e] = 0.0;
    std::vector<double> occ(n);
    for (int i = 0; i < n; ++i) occ[i] = shg_occupation(E[i], p.mu, p.T);
    std::vector<char> active(nn, 0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) active[i + n * j] = i != j && std::fabs(occ[i] - occ[j]) >= 1.0e-10;
    // optical_position_vertices! (OpticalPositionDerivatives.jl:13-91): bare D0, regularised
    // D_eta, r0 = A + i D0, r_eta = A + i D_eta and the cutoff derivative G for active pairs.
    std::vector<cd> D0(nn * 3), Dr(nn * 3), r0(nn * 3), re(nn * 3), G(nn * 9, cd(0.0, 0.0));
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                size_t e = i + n * (j + (size_t)n * a);
                double inv = bare_inverse(E[j] - E[i]);
                D0[e] = inv == 0.0 ? cd(0.0, 0.0) : V[e] * inv;
                Dr[e] = V[e] * regularized_inverse(E[j] - E[i], p.vertex_eta >= 0.0 ? p.vertex_eta : p.eta);
                r0[e] = A[e] + I1 * D0[e];
                re[e] = p.rdip ? p.rdip[e] : A[e] + I1 * Dr[e];
            }
    auto d0 = [&](int i, int j, int a) { return D0[i + n * (j + n * a)]; };
    auto dr = [&](int i, int j, int a) { return Dr[i + n * (j + n * a)]; };
    auto dip = [&](int i, int j, int a) { return r0[i + n * (j + n * a)]; };
    auto rdip = [&](int i, int j, int a) { return re[i + n * (j + n * a)]; };
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int m = 0; m < n; ++m)
                for (int i = 0; i < n; ++i) {
                    if (!active[i + n * m]) continue;
                    cd comA(0.0, 0.0), comH(0.0, 0.0);
                    for (int l = 0; l < n; ++l) {
                        comA += a3(i, l, a) * dr(l, m, b) - dr(i, l, b) * a3(l, m, a);
                        comH += v3(i, l, a) * dr(l, m, b) - dr(i, l, b) * v3(l, m, a);
                    }
                    cd sum_a = comA - (a3(i, i, a) - a3(m, m, a)) * dr(i, m, b);
                    cd sum_h = comH - (v3(i, i, a) - v3(m, m, a)) * dr(i, m, b);
                    cd finite = da4(i, m, a, b) + sum_a + (a3(i, i, a) - a3(m, m, a)) * d0(i, m, b) +
                                (a3(i, i, b) - a3(m, m, b)) * d0(i, m, a) -
                                I1 * a3(i, m, a) * (a3(i, i, b) - a3(m, m, b));
                    cd numerator = I1 * (w4(i, m, a, b) + sum_h +
                                         d0(i, m, a) * (v3(i, i, b) - v3(m, m, b)).real() +
                                         d0(i, m, b) * (v3(i, i, a) - v3(m, m, a)).real());
                    if (p.eta_correction)
                        for (int q = 0; q < n; ++q) {
                            if (q == i || q == m) continue;
                            numerator += regularized_weight(E[q] - E[m], p.eta) *
                                         (a3(i, q, a) * v3(q, m, b) -
                                          (v3(i, q, a) + I1 * (E[i] - E[q]) * a3(i, q, a)) * a3(q, m, b));
                            numerator -= regularized_weight(E[i] - E[q], p.eta) *
                                         (v3(i, q, b) * a3(q, m, a) -
                                          a3(i, q, b) * (v3(q, m, a) + I1 * (E[q] - E[m]) * a3(q, m, a)));
                        }
                    double inv = bare_inverse(E[m] - E[i]);
                    G[i + n * (m + n * (a + 3 * (size_t)b))] = inv == 0.0 ? finite : finite + inv * numerator;
                }
    auto g4 = [&](int i, int j, int a, int b) { return G[i + n * (j + n * (a + 3 * b))]; };
    auto o = [&](int64_t w, int c, int term, int q) -> cd & { return out[w + nom * (c + nc * (term + 7 * q))]; };
    // Pair terms (SecondHarmonicKernels.jl:149-220).
    for (int i = 0; i < n; ++i)
        for (int m = 0; m < n; ++m) {
            if (i == m) continue;
            const double fo = occ[i] - occ[m];
            if (std::fabs(fo) < 1.0e-10) continue;
            const double diff = E[m] - E[i];
            const double inv = bare_inverse(diff);
            for (int c = 0; c < nc; ++c) {
                const int a = comps[c][0], b = comps[c][1], cc = comps[c][2];
                cd first = dip(i, m, a) * (g4(m, i, b, cc) + g4(m, i, cc, b));
                cd second = g4(i, m, a, b) * dip(m, i, cc) + g4(i, m, a, cc) * dip(m, i, b);
                cd third = dip(i, m, a) *
                           (dip(m, i, b) * (v3(m, m, cc) - v3(i, i, cc)).real() +
                            dip(m, i, cc) * (v3(m, m, b) - v3(i, i, b)).real()) * inv;
                cd fourth = g4(i, m, b, a) * dip(m, i, cc) + g4(i, m, cc, a) * dip(m, i, b);
                cd fifth = (v3(i, i, a) - v3(m, m, a)).real() *
                           (dip(i, m, b) * dip(m, i, cc) + dip(i, m, cc) * dip(m, i, b));
                cd tfirst(0.0, 0.0), tother(0.0, 0.0);
                for (int q = 0; q < n; ++q) {
                    if (q == i || q == m) continue;
                    tfirst += dip(i, m, a) * (rdip(m, q, b) * rdip(q, i, cc) + rdip(m, q, cc) * rdip(q, i, b)) *
                              shg_principal(2 * E[q] - E[i] - E[m], p.eta);
                    tother += rdip(m, q, a) * (rdip(q, i, b) * dip(i, m, cc) + rdip(q, i, cc) * dip(i, m, b)) *
                              shg_principal(2 * E[i] - E[m] - E[q], p.eta);
                    tother += rdip(q, i, a) * (dip(i, m, b) * rdip(m, q, cc) + dip(i, m, cc) * rdip(m, q, b)) *
                              shg_principal(2 * E[m] - E[q] - E[i], p.eta);
                }
                for (int64_t w = 0; w < nom; ++w) {
                    const double energy = om[w];
                    cd d1 = shg_resonance(diff - energy, p.width, p.gaussian);
                    cd d2 = shg_resonance(diff - 2 * energy, p.width, p.gaussian);
                    cd dn = shg_resonance(-diff - energy, p.width, p.gaussian);
                    double low = shg_principal(energy, p.low_width);
                    cd factor = 0.5 * I1 * fo;
                    o(w, c, 0, 0) += factor * inv * (2.0 * first * d2 + second * d1 + (first + second) * low);
                    o(w, c, 1, 0) += factor * inv * third * (d1 - 4.0 * d2 - low);
                    o(w, c, 2, 0) += 0.5 * fo * (2.0 * tfirst * d2 + tother * dn);
                    o(w, c, 3, 0) -= factor * inv * 0.5 * fourth * (d1 + low);
                    o(w, c, 4, 0) -= factor * 0.25 * fifth * d1 * (low * low);
                    o(w, c, 0, 1) += fo * (first * d2 + second * d1);
                    o(w, c, 1, 1) += fo * third * (d1 - 2.0 * d2);
                    o(w, c, 2, 1) -= I1 * fo * diff * (tfirst * d2 - tother * dn);
                    o(w, c, 3, 1) -= fo * 0.5 * fourth * d1;
                    o(w, c, 4, 1) -= fo * 0.25 * fifth * d1 * low;
                }
            }
        }
    if (p.T <= 1.0e-7) return;
    // One-band terms (second_harmonic_one_band!, SecondHarmonicKernels.jl:245-294).
    const double kt = RESPONSE_KB_EV * p.T;
    for (int i = 0; i < n; ++i) {
        const double offset = E[i] - p.mu;
        if (std::fabs(offset) > 5 * kt) continue;
        const double fd = -std::exp(-0.5 * (offset / kt) * (offset / kt)) / (kt * std::sqrt(2 * PI));
        const double sd = -offset / (kt * kt) * fd;
        // _second_harmonic_bcd_enabled: a singleton of the adjacent-gap partition.
        const bool isolated = (i == 0 || E[i] - E[i - 1] > p.degeneracy) && (i == n - 1 || E[i + 1] - E[i] > p.degeneracy);
        double curv[3][3] = {};
        if (isolated && p.curv)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) curv[a][b] = a == b ? 0.0 : p.curv[i + n * (a + 3 * b)];
        else if (isolated)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    if (a == b) continue;
                    cd value = da4(i, i, b, a) - da4(i, i, a, b);
                    for (int q = 0; q < n; ++q)
                        value += a3(i, q, b) * d0(q, i, a) - d0(i, q, a) * a3(q, i, b) - a3(i, q, a) * d0(q, i, b) +
                                 d0(i, q, b) * a3(q, i, a) - I1 * (d0(i, q, a) * d0(q, i, b) - d0(i, q, b) * d0(q, i, a));
                    curv[a][b] = value.real();
                }
        for (int c = 0; c < nc; ++c) {
            const int a = comps[c][0], b = comps[c][1], cc = comps[c][2];
            double hess = w4(i, i, b, cc).real();
            if (p.hess) {
                hess = p.hess[i + n * (b + 3 * cc)];
            } else {
                for (int q = 0; q < n; ++q) {
                    if (q == i) continue;
                    hess += 2.0 * (v3(i, q, b) * v3(q, i, cc)).real() * shg_principal(E[i] - E[q], p.eta);
                }
            }
            const double va = v3(i, i, a).real(), vb = v3(i, i, b).real(), vc = v3(i, i, cc).real();
            const double semi = sd * va * vb * vc + fd * va * hess;
            const double bcd = isolated ? fd * (vb * curv[a][cc] + vc * curv[a][b]) : 0.0;
            for (int64_t w = 0; w < nom; ++w) {
                const double low = shg_principal(om[w], p.low_width);
                const cd kernel = low - I1 * shg_delta(om[w], p.low_width, p.gaussian);
                o(w, c, 5, 0) -= 0.25 * bcd * kernel * low;
                o(w, c, 5, 1) += 0.5 * I1 * bcd * kernel;
                o(w, c, 6, 0) -= 0.25 * I1 * semi * kernel * (low * low);
                o(w, c, 6, 1) -= 0.5 * semi * kernel * low;
            }
        }
    }
}

// ---- analytic local Berry-curvature dipole (derivative_backend = :analytic) ----------------------

Mat mat_mul(const Mat &X, const Mat &Y) {
    const int n = X.n;
    Mat out;
    out.init(n);
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < n; ++l) {
            const cd y = Y(l, j);
            for (int i = 0; i < n; ++i) out(i, j) += X(i, l) * y;
        }
    return out;
}

// D_a = U' d_a U (orthogonal_band_first_derivative!, MatrixElements/Interpolated/
// OrthogonalBandDerivatives.jl:123-141): dH_nm / (E_m - E_n) off the diagonal, i A_nn on it.
Mat band_first_derivative(const KData &d, int a) {
    const int n = d.nw;
    Mat D;
    D.init(n);
    for (int m = 0; m < n; ++m)
        for (int i = 0; i < n; ++i)
            D(i, m) = i == m ? I1 * d.Aint[a](i, i) : d.dH[a](i, m) * (1.0 / (d.E[m] - d.E[i]));
    return D;
}

// D_ag = U' d_a d_g U (orthogonal_band_second_derivative!, OrthogonalBandDerivatives.jl:183-245).
Mat band_second_derivative(const KData &d, const Mat &Da, const Mat &Dg, int a, int g) {
    const int n = d.nw;
    Mat T = mat_mul(d.dH[a], Dg), S = mat_mul(d.dH[g], Da);
    for (size_t e = 0; e < T.v.size(); ++e) T.v[e] += S.v[e];
    const Mat &Aa = d.Aint[a], &Ag = d.Aint[g];
    const Mat &dAag = d.dA[a][g], &dAga = d.dA[g][a];   // d_g A_a and d_a A_g
    Mat out;
    out.init(n);
    for (int m = 0; m < n; ++m)
        for (int i = 0; i < n; ++i) {
            if (i != m) {
                const double delta = d.E[m] - d.E[i];
                cd num = d.ddH[a][g](i, m) + T(i, m);
                num -= d.dH[a](m, m).real() * Dg(i, m) + d.dH[g](m, m).real() * Da(i, m);
                out(i, m) = num * (1.0 / delta);
            } else {
                cd cag(0.0, 0.0), cga(0.0, 0.0), dd(0.0, 0.0);
                for (int l = 0; l < n; ++l) {
                    cag += Dg(i, l) * Aa(l, i);
                    cag -= Aa(i, l) * Dg(l, i);
                    cga += Da(i, l) * Ag(l, i);
                    cga -= Ag(i, l) * Da(l, i);
                }
                for (int l = 0; l < n; ++l) {
                    dd += Dg(i, l) * Da(l, i);
                    dd += Da(i, l) * Dg(l, i);
                }
                const double jet = 0.5 * (dAag(i, i) - cag + dAga(i, i) - cga).real();
                out(i, i) = cd(0.5 * dd.real(), jet);
            }
        }
    return out;
}

// Per band the total of the six partitions of orthogonal_bcd_partition_matrices! (omega derivative,
// second derivative, first derivative, omega transport, mixed products, pure D) at their diagonal
// (orthogonal_geometry_partition_diagonal), Responses/QuantumGeometry/OrthogonalGeometryDerivatives.jl:
// 24-113, for the component (alpha, beta, gamma): d_gamma Omega_n^{alpha beta}.
std::vector<double> analytic_local_dipole(const KData &d, int al, int be, int ga) {
    const int n = d.nw;
    const Mat &Aa = d.Aint[al], &Ab = d.Aint[be];
    const Mat &Aag = d.dA[al][ga], &Abg = d.dA[be][ga];
    Mat Om, Omg;
    Om.init(n);
    Omg.init(n);
    for (size_t e = 0; e < Om.v.size(); ++e) {
        Om.v[e] = d.dA[be][al].v[e] - d.dA[al][be].v[e];
        Omg.v[e] = d.ddA[be][al][ga].v[e] - d.ddA[al][be][ga].v[e];
    }
    const Mat Da = band_first_derivative(d, al), Db = band_first_derivative(d, be), Dg = band_first_derivative(d, ga);
    const Mat Dag = band_second_derivative(d, Da, Dg, al, ga), Dbg = band_second_derivative(d, Db, Dg, be, ga);
    auto M = mat_mul;
    std::vector<Mat> parts;
    parts.push_back(Omg);   // omega_derivative
    {
        std::vector<std::pair<double, Mat>> t = {
            {-1, M(M(Dg, Db), Aa)}, {1, M(Dbg, Aa)}, {-1, M(M(Db, Dg), Aa)}, {-1, M(Aag, Db)},
            {1, M(M(Dg, Da), Ab)}, {-1, M(Dag, Ab)}, {1, M(M(Da, Dg), Ab)}, {1, M(Abg, Da)}};
        Mat s;
        s.init(n);
        for (auto &x : t)
            for (size_t e = 0; e < s.v.size(); ++e) s.v[e] += x.first * x.second.v[e];
        parts.push_back(s);   // second_derivative
    }
    {
        Mat s;
        s.init(n);
        const Mat t1 = M(Db, Aag), t2 = M(Aa, Dbg), t3 = M(Da, Abg), t4 = M(Ab, Dag);
        for (size_t e = 0; e < s.v.size(); ++e) s.v[e] = t1.v[e] - t2.v[e] - t3.v[e] + t4.v[e];
        parts.push_back(s);   // first_derivative
    }
    {
        Mat s;
        s.init(n);
        const Mat t1 = M(Dg, Om), t2 = M(Om, Dg);
        for (size_t e = 0; e < s.v.size(); ++e) s.v[e] = -t1.v[e] + t2.v[e];
        parts.push_back(s);   // omega_transport
    }
    {
        Mat s;
        s.init(n);
        const Mat t1 = M(M(Dg, Aa), Db), t2 = M(M(Dg, Ab), Da), t3 = M(M(Db, Aa), Dg), t4 = M(M(Da, Ab), Dg);
        for (size_t e = 0; e < s.v.size(); ++e) s.v[e] = t1.v[e] - t2.v[e] + t3.v[e] - t4.v[e];
        parts.push_back(s);   // mixed_products
    }
    {
        Mat s;
        s.init(n);
        const Mat t1 = M(Da, Dbg), t2 = M(Dag, Db), t3 = M(M(Dg, Da), Db), t4 = M(M(Da, Dg), Db), t5 = M(Db, Dag),
                  t6 = M(Dbg, Da), t7 = M(M(Dg, Db), Da), t8 = M(M(Db, Dg), Da);
        for (size_t e = 0; e < s.v.size(); ++e)
            s.v[e] = I1 * (-t1.v[e] - t2.v[e] + t3.v[e] + t4.v[e] + t5.v[e] + t6.v[e] - t7.v[e] - t8.v[e]);
        parts.push_back(s);   // pure_D
    }
    std::vector<double> out(n);
    for (int i = 0; i < n; ++i) {
        double total = 0.0;
        for (const Mat &p : parts) total += p(i, i).real();
        out[i] = total;
    }
    return out;
}

// One k-point's concatenated response values (point_value!, IntegralDriver.jl:596-...), with
// num_kpoints = 1 in every prefactor (the 1/Nk scale is applied by the lane consumer).
std::string point_values(const Model &m, const Task &task, const double k[3], cd *out) {
    const wnlqg_task_desc &t = task.desc;
    KData d;
    compute_kpoint(m, task.need, k, t.denominator_regularization, d);
    int n = d.nw;
    if (task.iso_mode == 0) {
        std::string err = isolated_spectrum_error(d.E, task.iso_tol);
        if (!err.empty()) return err;
    } else if (task.iso_mode == 1) {
        std::string err;
        spectral_blocks(d.E, task.iso_tol, err);
        if (!err.empty()) return err;
    }
    std::vector<double> f;
    fermi(d.E, t.fermi_energy, t.temperature, f);
    Screen s;
    bool need_screen = false;
    for (int r = 0; r < t.num_responses; ++r)
        need_screen |= t.responses[r].kind == WNLQG_SHIFT_CURRENT || t.responses[r].kind == WNLQG_INJECTION_CURRENT;
    if (need_screen) fill_screen(d.E, f, t, s);
    double vol = 0.0;
    {
        const double *L = m.lattice;  // det of lattice[i,j] = L[i + 3j]
        auto e = [&](int i, int j) { return L[i + 3 * j]; };
        vol = e(0, 0) * (e(1, 1) * e(2, 2) - e(1, 2) * e(2, 1)) - e(0, 1) * (e(1, 0) * e(2, 2) - e(1, 2) * e(2, 0)) +
              e(0, 2) * (e(1, 0) * e(2, 1) - e(1, 1) * e(2, 0));
    }
    int64_t nom = t.num_photon_energies;
    cd *o = out;
    for (int r = 0; r < t.num_responses; ++r) {
        const wnlqg_response_request &q = t.responses[r];
        int nc = q.num_components;
        if (q.kind == WNLQG_SHIFT_CURRENT || q.kind == WNLQG_INJECTION_CURRENT) {
            for (int64_t e = 0; e < nom * nc; ++e) o[e] = 0.0;
            if (s.active) {
                double P = q.kind == WNLQG_SHIFT_CURRENT
                               ? REDUCED_PLANCK_CONSTANT_EV_S * PI * std::pow(-ELEMENTARY_CHARGE_C, 3) /
                                     (2.0 * REDUCED_PLANCK_CONSTANT_J_S * REDUCED_PLANCK_CONSTANT_J_S * vol)
                               : -PI * std::pow(ELEMENTARY_CHARGE_C, 3) /
                                     (REDUCED_PLANCK_CONSTANT_J_S * REDUCED_PLANCK_CONSTANT_J_S * vol);
                // Per-pair kernels for the requested components (compute_*_kernel!).
                std::vector<cd> kern((size_t)n * n * nc, cd(0.0, 0.0));
                for (int c = 0; c < nc; ++c) {
                    int a = q.components[c][0], b = q.components[c][1], cc = q.components[c][2];
                    for (int nn = 0; nn < n; ++nn)
                        for (int mm = 0; mm < n; ++mm) {
                            if (!s.mask[nn + (size_t)n * mm]) continue;
                            cd val;
                            if (q.kind == WNLQG_SHIFT_CURRENT) {
                                cd dnm = gder(d, nn, mm, cc, a);
                                cd dmn = gder(d, mm, nn, b, a);
                                val = -I1 * (dnm * d.r[b](mm, nn) - dmn * d.r[cc](nn, mm));
                            } else {
                                // (v_mm^a - v_nn^a) r^c_nm r^b_mn with v = diag dH (ConventionalInjectionCurrent.jl:4-5).
                                cd vdc = d.dH[a](mm, mm) - d.dH[a](nn, nn);
                                val = vdc * d.r[cc](nn, mm) * d.r[b](mm, nn);
                            }
                            kern[nn + (size_t)n * (mm + (size_t)n * c)] = val;
                        }
                }
                // accumulate_conventional_response! (ConventionalShiftCurrent.jl:864-882).
                for (int64_t w = 0; w < nom; ++w)
                    for (int mm = 0; mm < n; ++mm)
                        for (int nn = 0; nn < n; ++nn) {
                            if (!s.mask[nn + (size_t)n * mm]) continue;
                            double weight = s.fnm[nn + (size_t)n * mm] * s.delta[w + nom * (nn + (size_t)n * mm)];
                            if (weight == 0.0) continue;
                            double cw = P * weight;
                            for (int c = 0; c < nc; ++c)
                                o[w + nom * c] += cw * kern[nn + (size_t)n * (mm + (size_t)n * c)];
                        }
            }
            o += nom * nc;
        } else if (q.kind == WNLQG_BERRY_CURVATURE) {
            for (int c = 0; c < nc; ++c) {
                int a = q.components[c][0], b = q.components[c][1];
                cd value(0.0, 0.0);
                for (int nn = 0; nn < n; ++nn) {
                    double fn = f[nn];
                    value += fn * d.F[a][b](nn, nn);
                    for (int mm = 0; mm < n; ++mm) {
                        if (mm == nn) continue;
                        value += (fn - f[mm]) * I1 * d.r[a](nn, mm) * d.r[b](mm, nn);
                    }
                }
                o[c] = cd(value.real(), 0.0);
            }
            o += nc;
        } else if (q.kind == WNLQG_QUANTUM_METRIC) {
            for (int c = 0; c < nc; ++c) {
                int a = q.components[c][0], b = q.components[c][1];
                double value = 0.0;
                for (int nn = 0; nn < n; ++nn)
                    for (int mm = 0; mm < n; ++mm) {
                        if (mm == nn) continue;
                        value += 0.5 * (f[nn] + f[mm]) * (d.r[a](nn, mm) * d.r[b](mm, nn)).real();
                    }
                o[c] = cd(value, 0.0);
            }
            o += nc;
        } else if (q.kind == WNLQG_LINEAR_TRANSPORT_BERRY) {
            // Berry-curvature channel of _linear_transport_response (LinearTransportKernels.jl:100-163,
            // kernel from linear_transport_kernel, :4-62, conventional_spectral_pair,
            // SpectralResponseGeometry.jl:79-85): summands 1 (contact) and 4 (interband imaginary
            // part), each accumulated in the reference's order, then added.
            const int64_t nmu = t.num_fermi_energies;
            const double factor = ELEMENTARY_CHARGE_C * ELEMENTARY_CHARGE_C / REDUCED_PLANCK_CONSTANT_J_S * 1e-20;
            const double gamma = t.linear_transport_gamma_inter;
            std::string berr;
            const std::vector<int> starts = spectral_blocks(d.E, t.spectral_gap_tolerance, berr);
            if (!berr.empty()) return berr;
            const int nblocks = (int)starts.size() - 1;
            for (int c = 0; c < nc; ++c) {
                const int a = q.components[c][0], b = q.components[c][1];
                for (int64_t im = 0; im < nmu; ++im) {
                    const double mu = t.fermi_energies[im];
                    double contact = 0.0, interband = 0.0;
                    for (int nn = 0; nn < n; ++nn)
                        contact -= factor * response_occupation(d.E[nn], mu, t.temperature) * d.F[a][b](nn, nn).real();
                    for (int i = 0; i < nblocks; ++i)
                        for (int j = i + 1; j < nblocks; ++j) {
                            const double el = d.E[starts[i]], er = d.E[starts[j]];
                            const double gap = er - el;
                            cd qv(0.0, 0.0);
                            for (int mm = starts[j]; mm < starts[j + 1]; ++mm)
                                for (int nn = starts[i]; nn < starts[i + 1]; ++nn)
                                    qv += d.r[a](nn, mm) * d.r[b](mm, nn);
                            const double occ = response_occupation(el, mu, t.temperature) -
                                               response_occupation(er, mu, t.temperature);
                            interband += 2 * factor * occ * gap * gap / (gap * gap + gamma * gamma) * qv.imag();
                        }
                    o[im + nmu * c] = cd(contact + interband, 0.0);
                }
            }
            o += nmu * nc;
        } else if (q.kind == WNLQG_BERRY_DIPOLE_SEA) {
            // Fermi-sea dipole on the finite-difference geometry (prepare_berry_multipole_geometry!,
            // BerryMultipoleGeometry.jl:67-161): per band n the central difference of the band
            // curvature (berry_curvature_group_sum_component with the group {n},
            // ConventionalQuantumGeometry.jl:530-557) at k +- delta_c, where delta_c is the
            // fractional image lattice * (h e_c) / 2pi of the Cartesian step (finite_difference_step_matrix,
            // Core/Coordinates.jl:15-44; berry_curvature_dipole_component!,
            // QuantumGeometryDerivatives.jl:193-228).  Every shifted spectrum passes the centre's
            // isolation check (isolation_threshold_ev = gap_tolerance, BerryMultipoleGeometry.jl:38-39).
            // D[mu,a,b,c] = sum_n f(E_n; mu, T) d_c Omega_n^{ab} (berry_dipole_moments!,
            // BerryMultipoleMoments.jl:7-47, with berry_multipole_sea_weight, BerryMultipoleDC.jl:56-62).
            const int64_t nmu = t.num_fermi_energies;
            if (t.derivative_backend == 1) {
                for (int c = 0; c < nc; ++c) {
                    const int a = q.components[c][0], b = q.components[c][1], cc = q.components[c][2];
                    const std::vector<double> ld = analytic_local_dipole(d, a, b, cc);
                    for (double v : ld)
                        if (!std::isfinite(v)) return "nonfinite consumed BCD/BCQ geometry";
                    for (int64_t im = 0; im < nmu; ++im) {
                        double value = 0.0;
                        for (int nu = 0; nu < n; ++nu)
                            value += response_occupation(d.E[nu], t.fermi_energies[im], t.temperature) * ld[nu];
                        o[im + nmu * c] = cd(value, 0.0);
                    }
                }
                o += nmu * nc;
                continue;
            }
            const double h = t.finite_difference_step;
            KData shifted[3][2];
            bool have[3] = {false, false, false};
            for (int c = 0; c < nc; ++c) {
                const int cc = q.components[c][2];
                if (have[cc]) continue;
                have[cc] = true;
                for (int sgn = 0; sgn < 2; ++sgn) {
                    double ks[3];
                    for (int i = 0; i < 3; ++i)
                        ks[i] = k[i] + (sgn == 0 ? 1.0 : -1.0) * (m.lattice[i + 3 * cc] * h / (2.0 * PI));
                    compute_kpoint(m, task.need, ks, t.denominator_regularization, shifted[cc][sgn]);
                    if (task.iso_mode == 0) {
                        std::string err = isolated_spectrum_error(shifted[cc][sgn].E, task.iso_tol);
                        if (!err.empty()) return err;
                    }
                }
            }
            auto band_curvature = [&](const KData &s, int a, int b, int nu) {
                double value = s.F[a][b](nu, nu).real();
                for (int mm = 0; mm < n; ++mm) {
                    if (mm == nu) continue;
                    const cd qab = s.r[a](nu, mm) * s.r[b](mm, nu);
                    const cd qba = s.r[b](nu, mm) * s.r[a](mm, nu);
                    value += -(qab - qba).imag();
                }
                return value;
            };
            for (int c = 0; c < nc; ++c) {
                const int a = q.components[c][0], b = q.components[c][1], cc = q.components[c][2];
                std::vector<double> dO(n);
                for (int nu = 0; nu < n; ++nu)
                    dO[nu] = (band_curvature(shifted[cc][0], a, b, nu) - band_curvature(shifted[cc][1], a, b, nu)) /
                             (2.0 * h);
                for (int64_t im = 0; im < nmu; ++im) {
                    double value = 0.0;
                    for (int nu = 0; nu < n; ++nu)
                        value += response_occupation(d.E[nu], t.fermi_energies[im], t.temperature) * dO[nu];
                    o[im + nmu * c] = cd(value, 0.0);
                }
            }
            o += nmu * nc;
        } else if (q.kind == WNLQG_INTRINSIC_AHC || q.kind == WNLQG_BERRY_DIPOLE) {
            const int64_t nmu = t.num_fermi_energies;
            for (int c = 0; c < nc; ++c) {
                const int a = q.components[c][0], b = q.components[c][1], cc = q.components[c][2];
                for (int64_t im = 0; im < nmu; ++im) {
                    const double mu = t.fermi_energies[im];
                    double value = 0.0;
                    if (q.kind == WNLQG_INTRINSIC_AHC && t.temperature == 0.0) {
                        // Occupied-space matrix curvature with bare occupied/empty links
                        // r_lm = A_lm - i dH_lm/(E_l - E_m) (IntrinsicHallGeometry.jl:117-136).
                        int occ = 0;
                        while (occ < n && d.E[occ] <= mu) ++occ;
                        for (int l = 0; l < occ; ++l) {
                            value += d.F[a][b](l, l).real();
                            for (int m = occ; m < n; ++m) {
                                auto link = [&](int x, int y, int ax) {
                                    return d.Aint[ax](x, y) - I1 * d.dH[ax](x, y) / (d.E[x] - d.E[y]);
                                };
                                cd left = link(l, m, a) * link(m, l, b);
                                cd right = link(l, m, b) * link(m, l, a);
                                value -= (left - right).imag();
                            }
                        }
                    } else {
                        // D[mu,a,b,c] = sum_n (-f'(E_n)) Omega_n^{ab} dE_n/dk_c.
                        for (int nn = 0; nn < n; ++nn) {
                            double omega = 0.0;
                            for (int mm = 0; mm < n; ++mm)
                                if (mm != nn) omega += -(d.r[a](nn, mm) * d.r[b](mm, nn)).imag();
                            omega = 2.0 * omega + d.F[a][b](nn, nn).real();
                            double w;
                            if (t.temperature > 0) {
                                const double scale = RESPONSE_KB_EV * t.temperature;
                                const double z = std::exp(-std::fabs((d.E[nn] - mu) / scale));
                                w = z / (scale * (1 + z) * (1 + z));
                            } else {
                                const double x = (d.E[nn] - mu) / t.fermi_surface_broadening;
                                w = std::exp(-x * x) / (std::sqrt(PI) * t.fermi_surface_broadening);
                            }
                            value += w * omega * d.dH[cc](nn, nn).real();
                        }
                    }
                    o[im + nmu * c] = cd(value, 0.0);
                }
            }
            o += nmu * nc;
        } else if (q.kind == WNLQG_SECOND_HARMONIC) {
            const size_t nn = (size_t)n * n;
            std::vector<cd> V(nn * 3), A(nn * 3), dA(nn * 9), W(nn * 9), R;
            for (int a = 0; a < 3; ++a) {
                const Mat &va = d.nonorth ? d.srcV[a] : d.dH[a], &aa = d.nonorth ? d.srcA[a] : d.Aint[a];
                for (size_t e = 0; e < nn; ++e) { V[e + nn * a] = va.v[e]; A[e + nn * a] = aa.v[e]; }
                for (int b = 0; b < 3; ++b) {
                    const Mat &dab = d.nonorth ? d.srcdA[a][b] : d.dA[a][b], &wab = d.nonorth ? d.srcW[a][b] : d.ddH[a][b];
                    for (size_t e = 0; e < nn; ++e) {
                        dA[e + nn * (a + 3 * b)] = dab.v[e];
                        W[e + nn * (a + 3 * b)] = wab.v[e];
                    }
                }
            }
            if (d.nonorth) {
                R.resize(nn * 3);
                for (int a = 0; a < 3; ++a)
                    for (size_t e = 0; e < nn; ++e) R[e + nn * a] = d.r[a].v[e];
            }
            ShgParams p;
            p.mu = t.fermi_energy; p.T = t.temperature; p.width = t.broadening;
            p.low_width = t.shg_low_frequency_broadening;
            p.eta = t.shg_intermediate_regularization > 0 ? t.shg_intermediate_regularization : t.denominator_regularization;
            p.degeneracy = t.degeneracy_threshold;
            p.gaussian = t.broadening_type == WNLQG_GAUSSIAN;
            p.eta_correction = t.shg_eta_correction != 0;
            if (d.nonorth) {
                p.vertex_eta = t.denominator_regularization;
                p.rdip = R.data();
                p.hess = d.esd.data();
                p.curv = d.iso.data();
            }
            shg_response(n, d.E.data(), V.data(), A.data(), dA.data(), W.data(), nom, t.photon_energies, nc,
                         q.components, p, o);
            o += nom * nc * 14;
        } else if (q.kind == WNLQG_JERK_CURRENT) {
            std::vector<cd> B((size_t)n * n * 3, 0.0), A((size_t)n * n * 3, 0.0), C((size_t)n * n * 9, 0.0);
            for (int a = 0; a < 3; ++a) {
                if (task.need.dH[a])
                    for (size_t e = 0; e < (size_t)n * n; ++e) B[e + (size_t)n * n * a] = d.dH[a].v[e];
                if (task.need.A[a])
                    for (size_t e = 0; e < (size_t)n * n; ++e) A[e + (size_t)n * n * a] = d.Aint[a].v[e];
                for (int b = 0; b < 3; ++b)
                    if (task.need.ddH[a][b])
                        for (size_t e = 0; e < (size_t)n * n; ++e) C[e + (size_t)n * n * (a + 3 * b)] = d.ddH[a][b].v[e];
            }
            jerk_response(n, d.E.data(), B.data(), A.data(), C.data(), nom, t.photon_energies, t.fermi_energy,
                          t.temperature, t.broadening, t.broadening_type == WNLQG_GAUSSIAN,
                          t.denominator_regularization > 0 ? t.denominator_regularization : 0.001,
                          t.transition_window_factor, nc, q.components, o);
            o += nom * nc;
        }
    }
    return "";
}

bool build_model(const wnlqg_model_desc *desc, Model &m) {
    if (!desc || desc->num_orbitals <= 0 || desc->num_r_vectors <= 0) { set_error("invalid model dimensions"); return false; }
    if (!desc->lattice || !desc->r_vectors || !desc->r_degeneracies || !desc->hamiltonian_r) { set_error("null model array"); return false; }
    m.nw = (int)desc->num_orbitals;
    m.nr = (int)desc->num_r_vectors;
    std::memcpy(m.lattice, desc->lattice, sizeof(m.lattice));
    m.rvec.assign(desc->r_vectors, desc->r_vectors + 3 * (size_t)m.nr);
    m.deg.assign(desc->r_degeneracies, desc->r_degeneracies + m.nr);
    size_t nn = (size_t)m.nw * m.nw;
    m.H.resize(nn * m.nr);
    for (size_t e = 0; e < nn * m.nr; ++e) m.H[e] = cd(desc->hamiltonian_r[2 * e], desc->hamiltonian_r[2 * e + 1]);
    m.has_position = desc->position_r != nullptr;
    if (m.has_position) {
        m.A.resize(nn * 3 * m.nr);
        for (size_t e = 0; e < nn * 3 * m.nr; ++e) m.A[e] = cd(desc->position_r[2 * e], desc->position_r[2 * e + 1]);
    }
    m.has_overlap = desc->overlap_r != nullptr;
    if (m.has_overlap) {
        m.S.resize(nn * m.nr);
        for (size_t e = 0; e < nn * m.nr; ++e) m.S[e] = cd(desc->overlap_r[2 * e], desc->overlap_r[2 * e + 1]);
    }
    for (auto &z : m.H) if (!std::isfinite(z.real()) || !std::isfinite(z.imag())) { set_error("hamiltonian_r contains non-finite values"); return false; }
    for (int64_t g : m.deg) if (g <= 0) { set_error("r_degeneracies must be positive"); return false; }
    // Convention I centres: tau = Re diag A(R = 0) and its fractional coordinates.
    int homes = 0;
    for (int r = 0; r < m.nr; ++r)
        if (m.rvec[3 * (size_t)r] == 0 && m.rvec[3 * (size_t)r + 1] == 0 && m.rvec[3 * (size_t)r + 2] == 0) { m.home = r; ++homes; }
    m.tau_cart.assign(3 * (size_t)m.nw, 0.0);
    m.tau_frac.assign(3 * (size_t)m.nw, 0.0);
    if (homes != 1) {
        m.centers_error = homes == 0 ? "Convention_I requires one R=(0,0,0) position block in the TB model."
                                     : "TB model contains more than one R=(0,0,0) block.";
    } else {
        for (int i = 0; i < m.nw && m.centers_error.empty(); ++i)
            for (int a = 0; a < 3; ++a) {
                const cd v = m.has_position ? m.A[nn * (a + 3 * (size_t)m.home) + i + (size_t)m.nw * i] : cd(0.0, 0.0);
                if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) { m.centers_error = "Convention_I Wannier center is non-finite"; break; }
                if (std::fabs(v.imag()) > 1.0e-10) { m.centers_error = "Convention_I Wannier center has an imaginary part"; break; }
                m.tau_cart[a * m.nw + i] = v.real();
            }
        // tau_cart[j] = sum_r tau_frac[r] * lattice[r + 3 j]: Gaussian elimination with pivoting.
        for (int i = 0; i < m.nw; ++i) {
            double M[3][4];
            for (int j = 0; j < 3; ++j) {
                for (int r = 0; r < 3; ++r) M[j][r] = m.lattice[r + 3 * j];
                M[j][3] = m.tau_cart[j * m.nw + i];
            }
            for (int c = 0; c < 3; ++c) {
                int piv = c;
                for (int r = c + 1; r < 3; ++r) if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
                for (int q = 0; q < 4; ++q) std::swap(M[c][q], M[piv][q]);
                for (int r = 0; r < 3; ++r) {
                    if (r == c || M[c][c] == 0.0) continue;
                    const double fct = M[r][c] / M[c][c];
                    for (int q = 0; q < 4; ++q) M[r][q] -= fct * M[c][q];
                }
            }
            for (int c = 0; c < 3; ++c) m.tau_frac[c * m.nw + i] = M[c][3] / M[c][c];
        }
    }
    return true;
}

}  // namespace

// The failing point with the smallest row among parallel workers; reported like the GPU engine's
// message (the reference's text followed by the k-point row).
struct FirstError {
    int64_t row = -1;
    std::string msg;
    void record(int64_t r, const std::string &m) {
#pragma omp critical(oracle_first_error)
        if (row < 0 || r < row) { row = r; msg = m; }
    }
    int report() const {
        set_error(msg + " (k-point row " + std::to_string(row) + ")");
        return WNLQG_ERR_INVALID_ARGUMENT;
    }
};

extern "C" {

const char *oracle_last_error(void) { return g_error.c_str(); }

int64_t oracle_value_count(const wnlqg_task_desc *t) {
    Task task;
    if (!build_task(t, task)) return -1;
    return task.value_count;
}

// Per-point values: k[3*n] -> out[n*value_count] complex (interleaved).
bool nonorth_kinds_ok(const Model &m, const wnlqg_task_desc *t) {
    if (t->wannier_center_convention == 1) {
        if (m.has_overlap) { set_error("Convention I with an overlap is not built"); return false; }
        if (!m.centers_error.empty()) { set_error(m.centers_error); return false; }
    }
    if (!m.has_overlap) return true;
    for (int r = 0; r < t->num_responses; ++r) {
        const int kind = t->responses[r].kind;
        if (kind == WNLQG_SECOND_HARMONIC) {
            // Metric SHG preconditions (NonorthogonalMatrixElements.jl:1088-1110).
            if (t->shg_eta_correction) { set_error("NONORTHOGONAL_SHG_ETA_CORRECTION_UNSUPPORTED"); return false; }
            if (!(std::isfinite(t->denominator_regularization) && t->denominator_regularization > 0)) {
                set_error("NONORTHOGONAL_SHG_POSITIVE_GEOMETRY_REQUIRED");
                return false;
            }
            continue;
        }
        if (kind != WNLQG_SHIFT_CURRENT && kind != WNLQG_INJECTION_CURRENT) {
            set_error("nonorthogonal models: shift current, injection current and second harmonic generation only");
            return false;
        }
    }
    return true;
}

int oracle_point_values(const wnlqg_model_desc *md, const wnlqg_task_desc *td, const double *k,
                        int64_t n, int threads, double *out) {
    Model m; Task task;
    if (!build_model(md, m) || !build_task(td, task)) return WNLQG_ERR_INVALID_ARGUMENT;
    if (!nonorth_kinds_ok(m, td)) return WNLQG_ERR_UNSUPPORTED;
    int64_t vc = task.value_count;
    if (threads <= 0) threads = omp_get_max_threads();
    FirstError first;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int64_t i = 0; i < n; ++i) {
        std::vector<cd> vals((size_t)vc);
        std::string err = point_values(m, task, &k[3 * i], vals.data());
        if (!err.empty()) first.record(i, err);
        for (int64_t e = 0; e < vc; ++e) { out[2 * (i * vc + e)] = vals[e].real(); out[2 * (i * vc + e) + 1] = vals[e].imag(); }
    }
    if (first.row >= 0) return first.report();
    return WNLQG_OK;
}

// Uniform Gamma-centred mesh integral with the reference's 64 deterministic lanes:
// lane L owns the contiguous indices [fld((L-1)Nk, NL)+1, fld(L Nk, NL)] (1-based), adds
// value/Nk in k order; lanes are summed in lane order.  Only indices in [k_begin, k_end)
// are evaluated (a bounded sample when the range is a sub-range); Nk stays the full mesh size.
int oracle_integrate_mesh(const wnlqg_model_desc *md, const wnlqg_task_desc *td, const int64_t mesh[3],
                          int64_t k_begin, int64_t k_end, int threads, double *out) {
    Model m; Task task;
    if (!build_model(md, m) || !build_task(td, task)) return WNLQG_ERR_INVALID_ARGUMENT;
    if (!nonorth_kinds_ok(m, td)) return WNLQG_ERR_UNSUPPORTED;
    int64_t nk = mesh[0] * mesh[1] * mesh[2];
    if (nk <= 0 || k_begin < 0 || k_end > nk || k_begin > k_end) { set_error("invalid mesh range"); return WNLQG_ERR_INVALID_ARGUMENT; }
    int64_t vc = task.value_count;
    int64_t lanes = std::min<int64_t>(nk, 64);
    std::vector<std::vector<cd>> lane_sum((size_t)lanes, std::vector<cd>((size_t)vc, cd(0.0, 0.0)));
    if (threads <= 0) threads = omp_get_max_threads();
    const double scale = 1.0 / (double)nk;
    FirstError failed;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int64_t L = 0; L < lanes; ++L) {
        int64_t first = (L * nk) / lanes;          // 0-based inclusive
        int64_t last = ((L + 1) * nk) / lanes;      // exclusive
        first = std::max(first, k_begin);
        last = std::min(last, k_end);
        std::vector<cd> vals((size_t)vc);
        for (int64_t idx = first; idx < last; ++idx) {
            double k[3];
            k[0] = (double)(idx % mesh[0]) / (double)mesh[0];
            k[1] = (double)((idx / mesh[0]) % mesh[1]) / (double)mesh[1];
            k[2] = (double)(idx / (mesh[0] * mesh[1])) / (double)mesh[2];
            std::string err = point_values(m, task, k, vals.data());
            if (!err.empty()) { failed.record(idx, err); break; }
            for (int64_t e = 0; e < vc; ++e) lane_sum[L][e] += scale * vals[e];
        }
    }
    if (failed.row >= 0) return failed.report();
    for (int64_t e = 0; e < vc; ++e) {
        cd acc(0.0, 0.0);
        for (int64_t L = 0; L < lanes; ++L) acc += lane_sum[L][e];
        out[2 * e] = acc.real();
        out[2 * e + 1] = acc.imag();
    }
    return WNLQG_OK;
}

// Band data at one k for tests: energies[nw], U[nw*nw] (canonical, column-major complex),
// and the Hamiltonian-gauge velocity matrices dH[a] (complex [nw,nw,3]).
int oracle_kpoint_spectrum(const wnlqg_model_desc *md, const double k[3], int convention, double *energies,
                           double *eigenvectors, double *dh) {
    Model m;
    if (!build_model(md, m)) return WNLQG_ERR_INVALID_ARGUMENT;
    if (convention == 1 && (m.has_overlap || !m.centers_error.empty())) {
        set_error(m.has_overlap ? "Convention I with an overlap is not built" : m.centers_error);
        return WNLQG_ERR_INVALID_ARGUMENT;
    }
    if (m.has_overlap) {
        // Nonorthogonal spectrum: H(k), S(k) by the direct sums, then the generalised eigensolve.
        const size_t nn = (size_t)m.nw * m.nw;
        Mat Hk, Sk;
        Hk.init(m.nw);
        Sk.init(m.nw);
        for (int ir = 0; ir < m.nr; ++ir) {
            const int64_t *r = &m.rvec[3 * (size_t)ir];
            double phase = (double)r[0] * k[0] + (double)r[1] * k[1] + (double)r[2] * k[2];
            cd f = std::polar(1.0, 2.0 * PI * phase) / (double)m.deg[ir];
            for (size_t e = 0; e < nn; ++e) { Hk.v[e] += f * m.H[nn * ir + e]; Sk.v[e] += f * m.S[nn * ir + e]; }
        }
        std::vector<double> ev;
        Mat C;
        if (!generalized_eigen(Hk, Sk, ev, C)) { set_error("effective S(k) is not positive definite"); return WNLQG_ERR_INVALID_ARGUMENT; }
        for (int i = 0; i < m.nw; ++i) energies[i] = ev[i];
        for (size_t e = 0; e < nn; ++e) { eigenvectors[2 * e] = C.v[e].real(); eigenvectors[2 * e + 1] = C.v[e].imag(); }
        return WNLQG_OK;
    }
    Needs need;
    for (int a = 0; a < 3; ++a) need.dH[a] = true;
    need.convention = convention;
    KData d;
    compute_kpoint(m, need, k, 0.001, d);
    size_t nn = (size_t)m.nw * m.nw;
    for (int i = 0; i < m.nw; ++i) energies[i] = d.E[i];
    for (size_t e = 0; e < nn; ++e) { eigenvectors[2 * e] = d.U.v[e].real(); eigenvectors[2 * e + 1] = d.U.v[e].imag(); }
    if (dh)
        for (int a = 0; a < 3; ++a)
            for (size_t e = 0; e < nn; ++e) { dh[2 * (e + nn * a)] = d.dH[a].v[e].real(); dh[2 * (e + nn * a) + 1] = d.dH[a].v[e].imag(); }
    return WNLQG_OK;
}

// Hermitian eigensolve of one matrix (upper triangle), canonicalised: for pinning the
// eigensolver against LAPACK through numpy.
int oracle_hermitian_eigen(int64_t n, const double *h, double *energies, double *eigenvectors) {
    Mat a; a.init((int)n);
    for (int64_t e = 0; e < n * n; ++e) a.v[e] = cd(h[2 * e], h[2 * e + 1]);
    std::vector<double> ev; Mat U;
    hermitian_eigen(a, ev, U);
    canonicalize(U);
    for (int64_t i = 0; i < n; ++i) energies[i] = ev[i];
    for (int64_t e = 0; e < n * n; ++e) { eigenvectors[2 * e] = U.v[e].real(); eigenvectors[2 * e + 1] = U.v[e].imag(); }
    return WNLQG_OK;
}

// Generalised eigensolve of one (H, S) pair (upper triangles), canonicalised: for pinning
// against LAPACK hegv through scipy.
int oracle_generalized_eigen(int64_t n, const double *h, const double *s, double *energies, double *eigenvectors) {
    Mat a, b;
    a.init((int)n);
    b.init((int)n);
    for (int64_t e = 0; e < n * n; ++e) { a.v[e] = cd(h[2 * e], h[2 * e + 1]); b.v[e] = cd(s[2 * e], s[2 * e + 1]); }
    std::vector<double> ev;
    Mat C;
    if (!generalized_eigen(a, b, ev, C)) { set_error("effective S(k) is not positive definite"); return WNLQG_ERR_INVALID_ARGUMENT; }
    for (int64_t i = 0; i < n; ++i) energies[i] = ev[i];
    for (int64_t e = 0; e < n * n; ++e) { eigenvectors[2 * e] = C.v[e].real(); eigenvectors[2 * e + 1] = C.v[e].imag(); }
    return WNLQG_OK;
}

// Jerk Eq. 9.20 on prepared Hamiltonian-gauge inputs (the reference's algebra fixture form):
// B, A complex [n,n,3]; C complex [n,n,3,3]; out complex [nom, ncomp].
int oracle_jerk_algebra(int64_t n, const double *E, const double *B, const double *A, const double *C,
                        int64_t nom, const double *omegas, double mu, double T, double width, int gaussian,
                        double reg, double window, int64_t ncomp, const int32_t *comps, double *out) {
    std::vector<cd> b((size_t)n * n * 3), a((size_t)n * n * 3), c((size_t)n * n * 9), o((size_t)nom * ncomp);
    for (size_t e = 0; e < b.size(); ++e) { b[e] = cd(B[2 * e], B[2 * e + 1]); a[e] = cd(A[2 * e], A[2 * e + 1]); }
    for (size_t e = 0; e < c.size(); ++e) c[e] = cd(C[2 * e], C[2 * e + 1]);
    jerk_response((int)n, E, b.data(), a.data(), c.data(), nom, omegas, mu, T, width, gaussian != 0, reg, window,
                  (int)ncomp, reinterpret_cast<const int32_t(*)[4]>(comps), o.data());
    for (size_t e = 0; e < o.size(); ++e) { out[2 * e] = o[e].real(); out[2 * e + 1] = o[e].imag(); }
    return WNLQG_OK;
}

// Hamiltonian-gauge band data at one k for tests: energies[nw]; dH, A [nw,nw,3]; dA, ddH
// [nw,nw,3,3] (dA: position axis, then derivative axis), all complex column-major.
int oracle_kpoint_data(const wnlqg_model_desc *md, const double k[3], double *energies, double *dh, double *a,
                       double *da, double *ddh) {
    Model m;
    if (!build_model(md, m)) return WNLQG_ERR_INVALID_ARGUMENT;
    if (m.has_overlap) { set_error("orthogonal models only"); return WNLQG_ERR_UNSUPPORTED; }
    Needs need;
    for (int x = 0; x < 3; ++x) {
        need.dH[x] = need.A[x] = true;
        for (int y = 0; y < 3; ++y) need.dA[x][y] = need.ddH[x][y] = true;
    }
    KData d;
    compute_kpoint(m, need, k, 0.001, d);
    const size_t nn = (size_t)m.nw * m.nw;
    for (int i = 0; i < m.nw; ++i) energies[i] = d.E[i];
    auto put = [](double *dst, size_t off, const Mat &x, size_t nn_) {
        for (size_t e = 0; e < nn_; ++e) { dst[2 * (off + e)] = x.v[e].real(); dst[2 * (off + e) + 1] = x.v[e].imag(); }
    };
    for (int x = 0; x < 3; ++x) {
        put(dh, nn * x, d.dH[x], nn);
        put(a, nn * x, d.Aint[x], nn);
        for (int y = 0; y < 3; ++y) { put(da, nn * (x + 3 * y), d.dA[x][y], nn); put(ddh, nn * (x + 3 * y), d.ddH[x][y], nn); }
    }
    return WNLQG_OK;
}

// Hamiltonian-gauge geometry at one k for the parity pins: energies[nw], canonical U[nw,nw],
// r[nw,nw,3] (Berry connection A + i D) and the generalized derivatives gder[nw,nw,3,3] with
// element (n, m, a, b) = r^a_{nm;b} (conventional_generalized_position_derivative_element,
// ConventionalShiftCurrent.jl:191-229) and F[nw,nw,3,3] (Wannier curvature, (a, b) order), all at
// the given denominator regularization (0 = bare inverses).
int oracle_kpoint_geometry(const wnlqg_model_desc *md, const double k[3], double eta, double *energies, double *u,
                           double *r, double *gd, double *f) {
    Model m;
    if (!build_model(md, m)) return WNLQG_ERR_INVALID_ARGUMENT;
    if (m.has_overlap) { set_error("orthogonal models only"); return WNLQG_ERR_UNSUPPORTED; }
    Needs need;
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) { need.need_gder(x, y); need.F[x][y] = true; }
    KData d;
    compute_kpoint(m, need, k, eta, d);
    const size_t nn = (size_t)m.nw * m.nw;
    auto put = [](double *dst, size_t off, const Mat &x, size_t nn_) {
        for (size_t e = 0; e < nn_; ++e) { dst[2 * (off + e)] = x.v[e].real(); dst[2 * (off + e) + 1] = x.v[e].imag(); }
    };
    for (int i = 0; i < m.nw; ++i) energies[i] = d.E[i];
    put(u, 0, d.U, nn);
    for (int a = 0; a < 3; ++a) {
        put(r, nn * a, d.r[a], nn);
        for (int b = 0; b < 3; ++b) {
            put(f, nn * (a + 3 * b), d.F[a][b], nn);
            for (int n = 0; n < m.nw; ++n)
                for (int mm = 0; mm < m.nw; ++mm) {
                    const cd g = gder(d, n, mm, a, b);
                    const size_t e = nn * (a + 3 * b) + n + (size_t)m.nw * mm;
                    gd[2 * e] = g.real();
                    gd[2 * e + 1] = g.imag();
                }
        }
    }
    return WNLQG_OK;
}

// Seven-term SHG on prepared Hamiltonian-gauge inputs (the reference's unit-test form):
// out complex [nom, ncomp, 7, 2].
int oracle_shg_algebra(int64_t n, const double *E, const double *V, const double *A, const double *dA,
                       const double *W, int64_t nom, const double *omegas, int64_t ncomp, const int32_t *comps,
                       double mu, double T, double width, double low_width, int gaussian, double eta,
                       int eta_correction, double degeneracy, double *out) {
    if (!(std::isfinite(width) && width > 0 && std::isfinite(low_width) && low_width > 0 && std::isfinite(eta) && eta > 0)) {
        set_error("SHG optical widths and intermediate_regularization must be finite and positive in eV");
        return WNLQG_ERR_INVALID_ARGUMENT;
    }
    if (!(std::isfinite(degeneracy) && degeneracy >= 0)) {
        set_error("SHG degeneracy_threshold must be finite and nonnegative in eV");
        return WNLQG_ERR_INVALID_ARGUMENT;
    }
    const size_t nn = (size_t)n * n;
    auto load = [](const double *src, size_t count) {
        std::vector<cd> v(count);
        for (size_t e = 0; e < count; ++e) v[e] = cd(src[2 * e], src[2 * e + 1]);
        return v;
    };
    std::vector<cd> v = load(V, nn * 3), a = load(A, nn * 3), da = load(dA, nn * 9), w = load(W, nn * 9);
    std::vector<cd> o((size_t)nom * ncomp * 14);
    ShgParams p;
    p.mu = mu; p.T = T; p.width = width; p.low_width = low_width; p.eta = eta; p.degeneracy = degeneracy;
    p.gaussian = gaussian != 0; p.eta_correction = eta_correction != 0;
    shg_response((int)n, E, v.data(), a.data(), da.data(), w.data(), nom, omegas, (int)ncomp,
                 reinterpret_cast<const int32_t(*)[4]>(comps), p, o.data());
    for (size_t e = 0; e < o.size(); ++e) { out[2 * e] = o[e].real(); out[2 * e + 1] = o[e].imag(); }
    return WNLQG_OK;
}

}  // extern "C"
