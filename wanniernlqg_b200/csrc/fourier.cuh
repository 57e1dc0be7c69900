// fourier.cuh - Fourier interpolation of the real-space channel tiles onto a batch of k-points.
//
// X_c(k)[i,j] = sum_R f_R(k) * T_c(R)[i,j],   f_R(k) = exp(2 pi i R.k) / deg_R
// (HamiltonianMatrixElements.jl:28-58 and :426-462, PositionMatrixElements.jl:294-332).
// The batch is a complex GEMM  X[k, n] = sum_R F[k, R] * T[R, n]  with n = channel*nw^2 + i + nw*j.
#pragma once
#include "common.cuh"

// Phase table F[k, R] for a batch.  Mesh mode (kpts == nullptr): batch entry b is mesh index
// k_begin + b of the Gamma-centred mesh (first axis fastest, CalculationUtils.jl:280-292); the
// phase R.k is reduced exactly with integer arithmetic before sincospi.  Point mode: k from kpts.
__global__ void phase_kernel(double2 *__restrict__ phases, const int64_t *__restrict__ rvec,
                             const int64_t *__restrict__ deg, int nr, int64_t batch, int64_t k_begin,
                             int64_t n1, int64_t n2, int64_t n3, const double *__restrict__ kpts) {
    int64_t total = batch * (int64_t)nr;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int64_t b = e / nr;
        int r = (int)(e - b * nr);
        int64_t r1 = rvec[3 * r], r2 = rvec[3 * r + 1], r3 = rvec[3 * r + 2];
        double x;
        if (kpts == nullptr) {
            int64_t idx = k_begin + b;
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
