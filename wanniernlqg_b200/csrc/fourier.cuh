// fourier.cuh - Fourier interpolation of the real-space channel tiles onto a batch of k-points.
//
// X_c(k)[i,j] = sum_R f_R(k) * T_c(R)[i,j],   f_R(k) = exp(2 pi i R.k) / deg_R
// (HamiltonianMatrixElements.jl:28-58 and :426-462, PositionMatrixElements.jl:294-332).
// The batch is a complex GEMM  X[k, n] = sum_R F[k, R] * T[R, n]  with n = channel*nw^2 + i + nw*j.
#pragma once
#include "common.cuh"

// Phase table F[k, R] for a batch.  Mesh mode (kpts == nullptr): batch entry b is mesh index
// kidx[b] (or k_begin + b without an index list) of the Gamma-centred mesh (first axis fastest, CalculationUtils.jl:280-292); the
// phase R.k is reduced exactly with integer arithmetic before sincospi.  Point mode: k from kpts.
__global__ void phase_kernel(double2 *__restrict__ phases, const int64_t *__restrict__ rvec,
                             const int64_t *__restrict__ deg, int nr, int64_t batch, int64_t k_begin,
                             int64_t n1, int64_t n2, int64_t n3, const double *__restrict__ kpts,
                             const int64_t *__restrict__ kidx = nullptr) {
    int64_t total = batch * (int64_t)nr;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int64_t b = e / nr;
        int r = (int)(e - b * nr);
        int64_t r1 = rvec[3 * r], r2 = rvec[3 * r + 1], r3 = rvec[3 * r + 2];
        double x;
        if (kpts == nullptr) {
            int64_t idx = kidx ? kidx[b] : k_begin + b;
            int64_t i1 = idx % n1, i2 = (idx / n1) % n2, i3 = idx / (n1 * n2);
            int64_t p1 = ((r1 * i1) % n1 + n1) % n1, p2 = ((r2 * i2) % n2 + n2) % n2, p3 = ((r3 * i3) % n3 + n3) % n3;
            x = (double)p1 / (double)n1 + (double)p2 / (double)n2 + (double)p3 / (double)n3;
        } else {
            const double *k = kpts + 3 * b;
            x = (double)r1 * k[0] + (double)r2 * k[1] + (double)r3 * k[2];
        }
        x -= rint(x);
        double s, c;
        sincospi(2.0 * x, &s, &c);
        double inv = 1.0 / (double)deg[r];
        phases[e] = make_double2(c * inv, s * inv);
    }
}

// FP64 complex GEMM  X[M x N] = F[M x K] * T[K x N], all row-major, 64x64x8 tiles, 256 threads,
// 4x4 complex outputs per thread (rows ty*4+i, columns tx+16*j: conflict-free shared reads and
// 256-byte coalesced stores).
constexpr int FG_BM = 64, FG_BN = 64, FG_BK = 8;

__global__ void __launch_bounds__(256) fourier_gemm_f64(const double2 *__restrict__ F, const double2 *__restrict__ T,
                                                        double2 *__restrict__ X, int64_t M, int64_t N, int K) {
    __shared__ double2 As[FG_BK][FG_BM];
    __shared__ double2 Bs[FG_BK][FG_BN];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int64_t m0 = (int64_t)blockIdx.y * FG_BM, n0 = (int64_t)blockIdx.x * FG_BN;
    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
    for (int r0 = 0; r0 < K; r0 += FG_BK) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            int e = tid + l * 256;           // 0..511
            int mm = e >> 3, kk = e & 7;     // A tile: 64 rows x 8
            int64_t gm = m0 + mm;
            int gr = r0 + kk;
            As[kk][mm] = (gm < M && gr < K) ? F[gm * K + gr] : make_double2(0.0, 0.0);
            int kb = e >> 6, nb = e & 63;    // B tile: 8 rows x 64
            int64_t gn = n0 + nb;
            int grb = r0 + kb;
            Bs[kb][nb] = (grb < K && gn < N) ? T[(int64_t)grb * N + gn] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < FG_BK; ++kk) {
            double2 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int64_t gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int64_t gn = n0 + tx + 16 * j;
            if (gn < N) X[gm * N + gn] = acc[i][j];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Staged (separable) Fourier contraction on the uniform Gamma-centred mesh.
//
// exp(2 pi i R.k) = exp(2 pi i r1 i1/N1) exp(2 pi i r2 i2/N2) exp(2 pi i r3 i3/N3), so
//   Y[i3][(r1,r2)] = sum_{r3} e3 T(R)/deg          (once per k3 plane touched by the batch)
//   Z[line][r1]    = sum_{r2} e2 Y[i3][(r1,r2)]     (once per (i2,i3) line touched)
//   X[k]           = sum_{r1} e1 Z[line(k)][r1]     (per k-point)
// give the direct sum of HamiltonianMatrixElements.jl:42-58 on every mesh point with
// 8*P1*C*nw^2 flops per k instead of 8*NR*C*nw^2 (P1 = number of distinct r1).  This is the
// dense-mesh role of the reference's Mixed-FFT backend (MixedFourierMatrixElements.jl:954-1126).
// R-vectors are grouped on the host: q12 = distinct (r1,r2) with its R list, q1 = distinct r1
// with its q12 list.
// ---------------------------------------------------------------------------------------------
struct StagedGroups {
    int P12, P1;
    const int *q12_start;   // [P12+1] offsets into q12_ridx
    const int *q12_ridx;    // [NR] R indices grouped by (r1,r2)
    const int *q12_r2;      // [P12]
    const int *q1_start;    // [P1+1] offsets into q1_q12
    const int *q1_q12;      // [P12] q12 indices grouped by r1
    const int *q1_r1;       // [P1]
};

WNLQG_D double2 mesh_phase(int64_t r, int64_t i, int64_t n) {
    int64_t p = ((r * i) % n + n) % n;
    double s, c;
    sincospi(2.0 * (double)p / (double)n, &s, &c);
    return make_double2(c, s);
}

// Y[t3][q12][col] for t3 = 0..n3-1 (i3 = i3_first + t3).  Grid: (col blocks, P12, n3).
__global__ void staged_r3_kernel(const double2 *__restrict__ T, int64_t N, StagedGroups g,
                                 const int64_t *__restrict__ rvec, const int64_t *__restrict__ deg, int64_t i3_first,
                                 int64_t n3mesh, double2 *__restrict__ Y) {
    const int q12 = blockIdx.y, t3 = blockIdx.z;
    const int64_t col = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t i3 = i3_first + t3;
    __shared__ double2 ph[64];
    const int s0 = g.q12_start[q12], s1 = g.q12_start[q12 + 1];
    double2 acc = make_double2(0.0, 0.0);
    for (int base = s0; base < s1; base += 64) {
        const int cnt = min(64, s1 - base);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const int r = g.q12_ridx[base + threadIdx.x];
            ph[threadIdx.x] = cscale(mesh_phase(rvec[3 * r + 2], i3, n3mesh), 1.0 / (double)deg[r]);
        }
        __syncthreads();
        if (col < N)
            for (int j = 0; j < cnt; ++j) acc = cfma(ph[j], T[(int64_t)g.q12_ridx[base + j] * N + col], acc);
    }
    if (col < N) Y[((int64_t)t3 * g.P12 + q12) * N + col] = acc;
}

// Z[l][q1][col] for lines l = 0..nlines-1 (global line = line_first + l, i2 = line % N2,
// i3 = line / N2).  Grid: (col blocks, P1, nlines).
__global__ void staged_r2_kernel(const double2 *__restrict__ Y, int64_t N, StagedGroups g, int64_t line_first,
                                 int64_t n2mesh, int64_t i3_first, double2 *__restrict__ Z) {
    const int q1 = blockIdx.y;
    const int64_t l = blockIdx.z;
    const int64_t col = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t line = line_first + l;
    const int64_t i2 = line % n2mesh, t3 = line / n2mesh - i3_first;
    __shared__ double2 ph[64];
    __shared__ int qq[64];
    const int s0 = g.q1_start[q1], s1 = g.q1_start[q1 + 1];
    double2 acc = make_double2(0.0, 0.0);
    for (int base = s0; base < s1; base += 64) {
        const int cnt = min(64, s1 - base);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const int q12 = g.q1_q12[base + threadIdx.x];
            qq[threadIdx.x] = q12;
            ph[threadIdx.x] = mesh_phase(g.q12_r2[q12], i2, n2mesh);
        }
        __syncthreads();
        if (col < N)
            for (int j = 0; j < cnt; ++j) acc = cfma(ph[j], Y[((int64_t)t3 * g.P12 + qq[j]) * N + col], acc);
    }
    if (col < N) Z[((int64_t)l * g.P1 + q1) * N + col] = acc;
}

// X[b][col] = sum_q1 e1(b, q1) Z[line(b)][q1][col] for batch entries b (mesh index k_begin + b).
// Grid: (col blocks, ceil(nb / 16)); each CTA handles 16 consecutive batch entries.
constexpr int STAGED_BT = 16;
constexpr int STAGED_MAX_P1 = 32;

__global__ void __launch_bounds__(256) staged_r1_kernel(const double2 *__restrict__ Z, int64_t N, StagedGroups g,
                                                        int64_t k_begin, int64_t nb, int64_t n1mesh,
                                                        int64_t line_first, double2 *__restrict__ X) {
    __shared__ double2 ph[STAGED_BT][STAGED_MAX_P1];
    const int64_t b0 = (int64_t)blockIdx.y * STAGED_BT;
    const int64_t col = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int P1 = g.P1;
    for (int e = threadIdx.x; e < STAGED_BT * P1; e += blockDim.x) {
        const int bb = e / P1, q1 = e % P1;
        const int64_t idx = k_begin + b0 + bb;
        ph[bb][q1] = mesh_phase(g.q1_r1[q1], idx % n1mesh, n1mesh);
    }
    __syncthreads();
    if (col >= N) return;
    const int64_t bend = min((int64_t)STAGED_BT, nb - b0);
    const int64_t l_first = (k_begin + b0) / n1mesh - line_first;
    const int64_t l_last = (k_begin + b0 + bend - 1) / n1mesh - line_first;
    if (l_first == l_last) {
        // One line: each Z element is loaded once and feeds the CTA's STAGED_BT outputs, which stay
        // in registers (static indices), so nothing goes through local memory.
        const double2 *zl = Z + (l_first * P1) * N + col;
        double2 acc[STAGED_BT];
#pragma unroll
        for (int bb = 0; bb < STAGED_BT; ++bb) acc[bb] = make_double2(0.0, 0.0);
        for (int q1 = 0; q1 < P1; ++q1) {
            const double2 z = zl[(int64_t)q1 * N];
#pragma unroll
            for (int bb = 0; bb < STAGED_BT; ++bb) acc[bb] = cfma(ph[bb][q1], z, acc[bb]);
        }
#pragma unroll
        for (int bb = 0; bb < STAGED_BT; ++bb)
            if (bb < bend) X[(b0 + bb) * N + col] = acc[bb];
    } else {
        for (int bb = 0; bb < bend; ++bb) {
            const int64_t l = (k_begin + b0 + bb) / n1mesh - line_first;
            const double2 *zl = Z + (l * P1) * N + col;
            double2 acc = make_double2(0.0, 0.0);
            for (int q1 = 0; q1 < P1; ++q1) acc = cfma(ph[bb][q1], zl[(int64_t)q1 * N], acc);
            X[(b0 + bb) * N + col] = acc;
        }
    }
}
