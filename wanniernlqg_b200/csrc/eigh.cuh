// eigh.cuh - batched Hermitian eigensolver: one CTA per k-point, parallel cyclic Jacobi in
// shared memory.
//
// Replaces DenseSpectra.hermitian_spectrum (src/Core/ESKernel/DenseSpectra.jl:14-16, LAPACK) and
// canonicalize_eigenvectors! (HamiltonianMatrixElements.jl:6-25).  The input is read as
// Hermitian(H, :U): only the upper triangle is used.  Eigenvalues come out ascending (ties keep
// index order) with every eigenvector column rotated so that its largest-magnitude entry (first
// on ties) is real and non-negative.
//
// Parallel ordering: the nw (padded to even np) indices are paired by the circle method, np/2
// disjoint pairs per round, np-1 rounds per sweep.  The rotations of one round commute, so the
// whole round is A <- J^H A J with J block-diagonal; each thread updates whole 2x2 blocks
// (rows of pair k1, columns of pair k2), and V <- V J likewise.
#pragma once
#include "common.cuh"
#include "dmma.cuh"

#define WNLQG_JACOBI_MAX_SWEEPS 30

struct EighSmem {
    static __host__ __device__ size_t bytes(int nw, int csize) {
        int np = nw + (nw & 1);
        int ld = np + 1;
        size_t s = 2 * (size_t)np * ld * csize;            // A, V
        s += (size_t)(np / 2) * (csize + 2 * sizeof(double) + 2 * sizeof(int));
        s += 64;
        return s;
    }
};

// One parallel-Jacobi sweep on (A, V) of real type T.  Returns after np-1 rounds; the caller
// measures convergence.  Pairs are computed by threads tid < np/2.
template <typename T>
WNLQG_D void jacobi_sweep(typename cplx_of<T>::type *A, typename cplx_of<T>::type *V, int np, int ld, T tol,
                          typename cplx_of<T>::type *rot_s, T *rot_c, int *rot_p, int *rot_q, int *rotated) {
    typedef typename cplx_of<T>::type C;
    const int half = np / 2;
    const int tid = threadIdx.x;
    for (int round = 0; round < np - 1; ++round) {
        if (tid < half) {
            int s1 = tid, s2 = np - 1 - tid;
            int i1 = s1 == 0 ? 0 : ((s1 - 1 + round) % (np - 1)) + 1;
            int i2 = ((s2 - 1 + round) % (np - 1)) + 1;
            int p = min(i1, i2), q = max(i1, i2);
            C apq = A[p + ld * q];
            T g = (T)hypot((double)apq.x, (double)apq.y);
            T c = (T)1;
            C sp = czero<C>();
            if (g > tol) {
                T app = A[p + ld * p].x, aqq = A[q + ld * q].x;
                T theta = (aqq - app) / ((T)2 * g);
                T t = (theta >= (T)0 ? (T)1 : (T)-1) / (fabs(theta) + sqrt(theta * theta + (T)1));
                c = (T)1 / sqrt(t * t + (T)1);
                T s = t * c;
                sp.x = s * (apq.x / g);
                sp.y = s * (apq.y / g);
                *rotated = 1;
            }
            rot_c[tid] = c;
            rot_s[tid] = sp;
            rot_p[tid] = p;
            rot_q[tid] = q;
        }
        __syncthreads();
        const int nblk = half * (half + 1) / 2;
        for (int w = tid; w < nblk + half * half; w += blockDim.x) {
            if (w < nblk) {
                // Upper-triangular block index (k1 <= k2) of the pair grid.
                int k2 = (int)((sqrtf(8.0f * w + 1.0f) - 1.0f) * 0.5f);
                while (k2 * (k2 + 1) / 2 > w) --k2;
                while ((k2 + 1) * (k2 + 2) / 2 <= w) ++k2;
                const int k1 = w - k2 * (k2 + 1) / 2;
                const int p1 = rot_p[k1], q1 = rot_q[k1], p2 = rot_p[k2], q2 = rot_q[k2];
                const T c1 = rot_c[k1], c2 = rot_c[k2];
                const C s1 = rot_s[k1], s2 = rot_s[k2];
                const C s2c = cconj(s2), s1c = cconj(s1);
                C a00 = A[p1 + ld * p2], a01 = A[p1 + ld * q2], a10 = A[q1 + ld * p2], a11 = A[q1 + ld * q2];
                C t00 = csub(cscale(a00, c2), cmul(a01, s2c));
                C t01 = cadd(cmul(a00, s2), cscale(a01, c2));
                C t10 = csub(cscale(a10, c2), cmul(a11, s2c));
                C t11 = cadd(cmul(a10, s2), cscale(a11, c2));
                C o00 = csub(cscale(t00, c1), cmul(s1, t10));
                C o01 = csub(cscale(t01, c1), cmul(s1, t11));
                C o10 = cadd(cmul(s1c, t00), cscale(t10, c1));
                C o11 = cadd(cmul(s1c, t01), cscale(t11, c1));
                if (k1 == k2) {
                    if (s1.x != (T)0 || s1.y != (T)0) {
                        o01 = czero<C>();
                        o10 = czero<C>();
                    } else {
                        o10 = cconj(o01);
                    }
                    o00.y = (T)0;
                    o11.y = (T)0;
                    A[p1 + ld * p2] = o00; A[p1 + ld * q2] = o01; A[q1 + ld * p2] = o10; A[q1 + ld * q2] = o11;
                } else {
                    A[p1 + ld * p2] = o00; A[p1 + ld * q2] = o01; A[q1 + ld * p2] = o10; A[q1 + ld * q2] = o11;
                    // Mirrored block (rows of pair k2, columns of pair k1) = conjugate transpose.
                    A[p2 + ld * p1] = cconj(o00); A[q2 + ld * p1] = cconj(o01);
                    A[p2 + ld * q1] = cconj(o10); A[q2 + ld * q1] = cconj(o11);
                }
            } else {
                const int v = w - nblk;
                const int k1 = v % half, k2 = v / half;
                const int p1 = rot_p[k1], q1 = rot_q[k1], p2 = rot_p[k2], q2 = rot_q[k2];
                const T c2 = rot_c[k2];
                const C s2 = rot_s[k2], s2c = cconj(s2);
                C v00 = V[p1 + ld * p2], v01 = V[p1 + ld * q2], v10 = V[q1 + ld * p2], v11 = V[q1 + ld * q2];
                V[p1 + ld * p2] = csub(cscale(v00, c2), cmul(v01, s2c));
                V[p1 + ld * q2] = cadd(cmul(v00, s2), cscale(v01, c2));
                V[q1 + ld * p2] = csub(cscale(v10, c2), cmul(v11, s2c));
                V[q1 + ld * q2] = cadd(cmul(v10, s2), cscale(v11, c2));
            }
        }
        __syncthreads();
    }
}

// Off-diagonal Frobenius norm (fixed-order block reduction); all threads get the value.
template <typename C>
WNLQG_D double offdiag_norm(const C *A, int np, int ld, double *red) {
    double local = 0.0;
    for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
        const int i = e % np, j = e / np;
        if (i != j) {
            const double2 z = to_c64(A[i + ld * j]);
            local += z.x * z.x + z.y * z.y;
        }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        red[40] = sqrt(s);
    }
    __syncthreads();
    const double r = red[40];
    __syncthreads();
    return r;
}

// T: real type of the iteration (double for the FP64 path, float for the mixed path).
// Input H(k) for batch entry b at h_in + b*h_stride (complex double, column-major nw x nw).
// Outputs: energies E[b*nw + n] (double) and U[b*nw*nw + i + nw*n] (complex double).
// gscratch (optional): a per-CTA working set of EighSmem::bytes in global memory, used when the
// matrices do not fit shared memory (large nw).
template <typename T, bool GW = false>
__global__ void __launch_bounds__(256, 4) jacobi_eigh_kernel(const double2 *__restrict__ h_in, int64_t h_stride, int64_t batch, int nw,
                                   double *__restrict__ E_out, double2 *__restrict__ U_out, T tol_scale,
                                   unsigned char *gscratch = nullptr, int64_t gscratch_stride = 0) {
    typedef typename cplx_of<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *smraw;
    if constexpr (GW) smraw = gscratch + (int64_t)blockIdx.x * gscratch_stride;
    else smraw = smem_dyn;
    const int np = nw + (nw & 1);
    const int ld = np + 1;
    const int half = np / 2;
    C *A = reinterpret_cast<C *>(smraw);
    C *V = A + (size_t)np * ld;
    C *rot_s = V + (size_t)np * ld;                          // s * e^{i phi} per pair
    double *scratch = reinterpret_cast<double *>(rot_s + half);
    T *rot_c = reinterpret_cast<T *>(scratch + 2);           // c per pair
    int *rot_p = reinterpret_cast<int *>(rot_c + half);
    int *rot_q = rot_p + half;
    __shared__ double red[48];
    __shared__ int rot_flag;

    const int tid = threadIdx.x;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const double2 *h = h_in + b * h_stride;
        double local = 0.0;
        for (int e = tid; e < np * np; e += blockDim.x) {
            int i = e % np, j = e / np;
            double2 v = make_double2(0.0, 0.0);
            if (i < nw && j < nw) {
                if (i < j) v = h[i + (size_t)nw * j];
                else if (i > j) v = cconj(h[j + (size_t)nw * i]);
                else v = make_double2(h[i + (size_t)nw * i].x, 0.0);
            }
            local += v.x * v.x + v.y * v.y;
            A[i + ld * j] = from_c64<C>(v);
            V[i + ld * j] = from_c64<C>(make_double2(i == j ? 1.0 : 0.0, 0.0));
        }
        // Frobenius norm (fixed-order reduction).
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((tid & 31) == 0) red[tid >> 5] = local;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
            scratch[0] = sqrt(s) * (double)tol_scale;
        }
        __syncthreads();
        const T tol = (T)scratch[0];

        // Sweep until a sweep applies no rotation (every |a_pq| <= tol) or the off-diagonal norm is
        // below np * tol (then every element is too).
        for (int sweep = 0; sweep < WNLQG_JACOBI_MAX_SWEEPS; ++sweep) {
            if (offdiag_norm(A, np, ld, red) <= (double)tol * np) break;
            if (tid == 0) rot_flag = 0;
            __syncthreads();
            jacobi_sweep<T>(A, V, np, ld, tol, rot_s, rot_c, rot_p, rot_q, &rot_flag);
            const int any = rot_flag;
            __syncthreads();
            if (!any) break;
        }
        // Ascending order (stable), then phase canonicalisation per column.
        for (int i = tid; i < nw; i += blockDim.x) {
            T di = A[i + ld * i].x;
            int rank = 0;
            for (int j = 0; j < nw; ++j) {
                T dj = A[j + ld * j].x;
                rank += (dj < di) || (dj == di && j < i);
            }
            int pivot = 0;
            double pm = hypot((double)V[0 + ld * i].x, (double)V[0 + ld * i].y);
            for (int r = 1; r < nw; ++r) {
                double mg = hypot((double)V[r + ld * i].x, (double)V[r + ld * i].y);
                if (mg > pm) { pm = mg; pivot = r; }
            }
            double2 phase = make_double2(1.0, 0.0);
            if (pm > 0.0) {
                double2 pv = to_c64(V[pivot + ld * i]);
                phase = make_double2(pv.x / pm, -pv.y / pm);
            }
            E_out[b * nw + rank] = (double)di;
            double2 *u = U_out + b * (int64_t)nw * nw + (int64_t)nw * rank;
            for (int r = 0; r < nw; ++r) {
                u[r] = cmul(to_c64(V[r + ld * i]), phase);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Mixed-precision eigensolver, one team of TEAM threads per matrix, in two kernels:
//   stage 1 (jacobi_f32_team_kernel): FP32 parallel Jacobi until the off-diagonal norm is below
//     2^-17 ||H||, warm-started along runs of consecutive mesh points from the previous point's
//     eigenvectors (V <- V (3I - V^H V)/2, A <- V^H H V);
//   stage 2 (eigh_refine_f64_team_kernel): FP64 Rayleigh-Ritz refinement, W = second-order
//     Loewdin orthonormalisation of V, H' = W^H H W, FP64 Jacobi sweeps (quadratic
//     convergence), U = W J, ascending order and canonical phases.
// A team is one warp (TEAM = 32: several teams per CTA, synchronised with __syncwarp) or one
// CTA of 64 or 128 threads (two or four warps share a matrix, synchronised with __syncthreads;
// each thread then holds a half or a quarter of a column in the products and does that share of
// a round's updates, and an SM holds more warps for the same shared memory).  A and V sit in the team's own shared
// memory.  The off-diagonal 2x2 block updates of a round take their (k1 < k2) pair indices from a
// fixed table (the order w = k2 (k2 - 1) / 2 + k1 is a prefix for every np <= 32); V <- V J
// runs one row per thread, the pairs of a round split between the warps.
// ---------------------------------------------------------------------------------------------
__constant__ unsigned char c_jacobi_offdiag[120][2];   // k1 < k2 < 16 in the order w = k2 (k2 - 1) / 2 + k1

template <int TEAM> struct Team {
    static_assert(TEAM == 32 || TEAM == 64 || TEAM == 128, "a team is one warp or one CTA of 2 or 4 warps");
    static constexpr int ROWS = 32 / (TEAM / 32);   // rows of a product column held per thread: 32, 16 or 8
    static WNLQG_D int rank() { return TEAM == 32 ? (int)(threadIdx.x & 31) : (int)threadIdx.x; }
    static WNLQG_D void sync() {
        if constexpr (TEAM == 32) __syncwarp();
        else __syncthreads();
    }
    static WNLQG_D bool any(bool v) {
        if constexpr (TEAM == 32) return __any_sync(0xffffffffu, v);
        else return __syncthreads_or(v ? 1 : 0) != 0;
    }
    // Sum of one double per thread over the team, the same value in every thread (fixed order).
    static WNLQG_D double sum(double v, double *red) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if constexpr (TEAM == 32) {
            return v;
        } else {
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
            __syncthreads();
            double t = red[0];
#pragma unroll
            for (int w = 1; w < TEAM / 32; ++w) t += red[w];
            __syncthreads();
            return t;
        }
    }
};

struct WarpJacobiSmem {
    // Per team: A, V (np x ld complex float), rotation sines, cosines and pair indices.
    // The team kernels pad rows to ld = np + 3 (measured 1% faster than np + 1 at nw = 32 in both
    // the FP32 sweep and the FP64 refinement; np + 5 was slower).
    static __host__ __device__ size_t per_team(int nw) {
        const int np = nw + (nw & 1);
        const int ld = np + 3;
        size_t s = 2 * (size_t)np * ld * sizeof(float2) + 16 * (sizeof(float2) + sizeof(float) + 2 * sizeof(int));
        return (s + 15) & ~(size_t)15;
    }
};

// One team-synchronous parallel-Jacobi sweep (np - 1 rounds); returns true (in every thread)
// when a rotation was applied.
WNLQG_D float recip_sqrt(float x) { return rsqrtf(x); }
WNLQG_D double recip_sqrt(double x) { return 1.0 / sqrt(x); }

template <typename T, int TEAM>
WNLQG_D bool team_jacobi_sweep(typename cplx_of<T>::type *A, typename cplx_of<T>::type *V, int np, int ld, T tol,
                               typename cplx_of<T>::type *rot_s, T *rot_c) {
    typedef typename cplx_of<T>::type C;
    const int t = Team<TEAM>::rank();
    const int half = np / 2;
    const int noff = half * (half - 1) / 2;
    // V <- V J: thread t handles row t % 32 and the pairs [kb, ke) of its warp.
    const int vrow = t & 31;
    const int kper = (half + TEAM / 32 - 1) / (TEAM / 32);
    const int kb = (t >> 5) * kper, ke = min(half, kb + kper);
    bool rotated = false;
    for (int round = 0; round < np - 1; ++round) {
        // Pair k of this round rotates indices (p, q) of slots k and np - 1 - k: slot 0 holds index
        // 0, slot s >= 1 holds ((s - 1 + round) mod (np - 1)) + 1.  Every thread computes the
        // indices it needs in registers, so its shared-memory loads wait on nothing else.
        auto slot_index = [&](int sl) -> int {
            if (sl == 0) return 0;
            int v = sl - 1 + round;
            if (v >= np - 1) v -= np - 1;
            return v + 1;
        };
        auto pair_pq = [&](int k, int &p, int &q) {
            const int i1 = slot_index(k), i2 = slot_index(np - 1 - k);
            p = min(i1, i2);
            q = max(i1, i2);
        };
        if (t < half) {
            int p, q;
            pair_pq(t, p, q);
            const C apq = A[p + ld * q];
            T c = (T)1;
            C sp = czero<C>();
            if constexpr (sizeof(T) == 4) {
                // FP32 preconditioner: the rotation from one reciprocal square root of |a_pq|^2
                // (no divisions; the FP64 stage absorbs the few-ulp differences).  |a_pq| >= tol
                // >= 2^-20 ||H|| keeps the squares far from the FP32 range limits.
                const T g2 = apq.x * apq.x + apq.y * apq.y;
                if (g2 > tol * tol) {
                    const T ginv = rsqrtf(g2);
                    const T app = A[p + ld * p].x, aqq = A[q + ld * q].x;
                    const T theta = (aqq - app) * ((T)0.5 * ginv);
                    const T tt = copysignf(__frcp_rn(fabsf(theta) + sqrtf(theta * theta + (T)1)), theta);
                    c = rsqrtf(tt * tt + (T)1);
                    const T sg = tt * c * ginv;
                    sp.x = sg * apq.x;
                    sp.y = sg * apq.y;
                    rotated = true;
                }
            } else {
                const T g = hypot(apq.x, apq.y);
                if (g > tol) {
                    const T app = A[p + ld * p].x, aqq = A[q + ld * q].x;
                    const T theta = (aqq - app) / ((T)2 * g);
                    const T tt = (theta >= (T)0 ? (T)1 : (T)-1) / (fabs(theta) + sqrt(theta * theta + (T)1));
                    c = recip_sqrt(tt * tt + (T)1);
                    const T sn = tt * c;
                    sp.x = sn * (apq.x / g);
                    sp.y = sn * (apq.y / g);
                    rotated = true;
                }
            }
            rot_c[t] = c;
            rot_s[t] = sp;
        }
        Team<TEAM>::sync();
        // 2x2 block updates: the off-diagonal blocks (k1 < k2, table order) go to threads 0, 1, ...
        // and the cheaper diagonal blocks (k1 == k2) to the last threads of the team, so that no
        // thread takes two off-diagonal blocks before every thread has one.
        auto block = [&](int k1, int k2) {
            int p1, q1, p2, q2;
            pair_pq(k1, p1, q1);
            pair_pq(k2, p2, q2);
            const T c1 = rot_c[k1], c2 = rot_c[k2];
            const C s1 = rot_s[k1], s2 = rot_s[k2];
            const C s2c = cconj(s2), s1c = cconj(s1);
            const C a00 = A[p1 + ld * p2], a01 = A[p1 + ld * q2], a10 = A[q1 + ld * p2], a11 = A[q1 + ld * q2];
            const C t00 = csub(cscale(a00, c2), cmul(a01, s2c));
            const C t01 = cadd(cmul(a00, s2), cscale(a01, c2));
            const C t10 = csub(cscale(a10, c2), cmul(a11, s2c));
            const C t11 = cadd(cmul(a10, s2), cscale(a11, c2));
            C o00 = csub(cscale(t00, c1), cmul(s1, t10));
            C o01 = csub(cscale(t01, c1), cmul(s1, t11));
            C o10 = cadd(cmul(s1c, t00), cscale(t10, c1));
            C o11 = cadd(cmul(s1c, t01), cscale(t11, c1));
            if (k1 == k2) {
                if (s1.x != (T)0 || s1.y != (T)0) {
                    o01 = czero<C>();
                    o10 = o01;
                } else {
                    o10 = cconj(o01);
                }
                o00.y = (T)0;
                o11.y = (T)0;
                A[p1 + ld * p2] = o00; A[p1 + ld * q2] = o01; A[q1 + ld * p2] = o10; A[q1 + ld * q2] = o11;
            } else {
                A[p1 + ld * p2] = o00; A[p1 + ld * q2] = o01; A[q1 + ld * p2] = o10; A[q1 + ld * q2] = o11;
                A[p2 + ld * p1] = cconj(o00); A[q2 + ld * p1] = cconj(o01);
                A[p2 + ld * q1] = cconj(o10); A[q2 + ld * q1] = cconj(o11);
            }
        };
        for (int w = t; w < noff; w += TEAM) block(c_jacobi_offdiag[w][0], c_jacobi_offdiag[w][1]);
        for (int k = TEAM - 1 - t; k < half; k += TEAM) block(k, k);
        if (vrow < np) {
            for (int k = kb; k < ke; ++k) {
                int p, q;
                pair_pq(k, p, q);
                const T c = rot_c[k];
                const C sk = rot_s[k], skc = cconj(sk);
                const C vp = V[vrow + ld * p], vq = V[vrow + ld * q];
                V[vrow + ld * p] = csub(cscale(vp, c), cmul(vq, skc));
                V[vrow + ld * q] = cadd(cmul(vp, sk), cscale(vq, c));
            }
        }
        Team<TEAM>::sync();
    }
    return Team<TEAM>::any(rotated);
}

// out[r] = (op(X) * Y)[r0 + r, col] for the team's np x np shared matrices (op = conjugate
// transpose when xh), with col = t % 32 and rows r0 = (t / 32) * ROWS .. + ROWS: each thread's
// part of one column of the product, in registers (static indices only).
template <int TEAM, typename C>
WNLQG_D void team_column_product(const C *X, const C *Y, C (&out)[Team<TEAM>::ROWS], int np, int ld, bool xh) {
    constexpr int ROWS = Team<TEAM>::ROWS;
    const int t = Team<TEAM>::rank();
    const int col = t & 31, r0 = (t >> 5) * ROWS;
#pragma unroll
    for (int i = 0; i < ROWS; ++i) out[i] = czero<C>();
    if (col >= np) return;
    for (int l = 0; l < np; ++l) {
        const C y = Y[l + ld * col];
        if (xh) {
#pragma unroll
            for (int i = 0; i < ROWS; ++i)
                if (r0 + i < np) out[i] = cfmaconj(X[l + ld * (r0 + i)], y, out[i]);
        } else {
#pragma unroll
            for (int i = 0; i < ROWS; ++i)
                if (r0 + i < np) out[i] = cfma(X[(r0 + i) + ld * l], y, out[i]);
        }
    }
}

// FP64 team of 128 threads (four warps), np <= 32: P = op(X) Y on the FP64 tensor cores (op = X^H
// when XH), warp w taking the 8 x 32 row block w as four 8 x 8 tiles (one A fragment per K step
// shared by the four tiles, twelve DMMA chains, dmma.cuh's three-product form); then a team
// barrier and out[r + ld c] = f(r, c, P[r][c]) for r, c < np.  out may alias X or Y (every
// operand read precedes the barrier), and f may read out[r + ld c] itself, which only the
// calling lane writes.  No closing barrier.
template <bool XH, typename F>
WNLQG_D void team128_dmma(const double2 *X, const double2 *Y, double2 *out, int np, int ld, F f) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int fr = lane >> 2, fk = lane & 3;
    const int r = 8 * w + fr;
    const double2 zero = make_double2(0.0, 0.0);
    Dmma3 acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q].zero();
    for (int k0 = 0; k0 < np; k0 += 4) {
        const int ka = k0 + fk;
        double2 a = zero;
        if (r < np && ka < np) {
            if (XH) {
                const double2 v = X[ka + ld * r];
                a = make_double2(v.x, -v.y);
            } else {
                a = X[r + ld * ka];
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = 8 * q + fr;
            acc[q].mac(a, (ka < np && c < np) ? Y[ka + ld * c] : zero);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int c = 8 * q + 2 * fk + i;
            if (r < np && c < np) out[r + ld * c] = f(r, c, acc[q].value(i));
        }
}

template <int TEAM, typename C>
WNLQG_D void team_store_column(C *M, const C (&v)[Team<TEAM>::ROWS], int np, int ld) {
    constexpr int ROWS = Team<TEAM>::ROWS;
    const int t = Team<TEAM>::rank();
    const int col = t & 31, r0 = (t >> 5) * ROWS;
    if (col < np) {
#pragma unroll
        for (int i = 0; i < ROWS; ++i)
            if (r0 + i < np) M[(r0 + i) + ld * col] = v[i];
    }
}

// A <- H(k) from the upper triangle of the stored matrix (lower = conjugate, real diagonal),
// zero-padded to np; returns the Frobenius norm (the same value in every thread).
template <int TEAM, typename C>
WNLQG_D double team_load_hermitian(C *A, const double2 *__restrict__ h, int nw, int np, int ld, double *red) {
    const int t = Team<TEAM>::rank();
    const int row = t & 31, j0 = t >> 5;
    for (int j = j0; j < np; j += TEAM / 32) {
        double2 v = make_double2(0.0, 0.0);
        if (row < nw && j < nw) v = h[row + (size_t)nw * j];
        if (row < np) A[row + ld * j] = from_c64<C>(v);
    }
    Team<TEAM>::sync();
    if (row < np)
        for (int i = row + j0; i < np; i += TEAM / 32) {
            if (i > row) A[i + ld * row] = cconj(A[row + ld * i]);
            else A[i + ld * i].y = 0;
        }
    Team<TEAM>::sync();
    double local = 0.0;
    if (row < np)
        for (int i = j0; i < np; i += TEAM / 32) {
            const C z = A[i + ld * row];
            local += (double)z.x * z.x + (double)z.y * z.y;
        }
    return sqrt(Team<TEAM>::sum(local, red));
}

// Squared off-diagonal Frobenius norm of the team's matrix (the same value in every thread).
template <int TEAM, typename C>
WNLQG_D double team_offdiag2(const C *A, int np, int ld, double *red) {
    const int t = Team<TEAM>::rank();
    const int row = t & 31, j0 = t >> 5;
    double off = 0.0;
    if (row < np)
        for (int i = j0; i < np; i += TEAM / 32)
            if (i != row) {
                const C z = A[i + ld * row];
                off += (double)z.x * z.x + (double)z.y * z.y;
            }
    return Team<TEAM>::sum(off, red);
}

// TEAM = 32: blocks of 128 threads (four teams); otherwise blocks of TEAM threads (one team).
template <int TEAM>
__global__ void __launch_bounds__(TEAM == 32 ? 128 : TEAM, TEAM == 32 ? 4 : (TEAM == 64 ? 12 : 8)) jacobi_f32_team_kernel(const double2 *__restrict__ h_in, int64_t h_stride,
                                                              int64_t batch, int nw, float2 *__restrict__ V_out,
                                                              int warm_start) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int ROWS = Team<TEAM>::ROWS;
    __shared__ double red[4];
    const int np = nw + (nw & 1);
    const int ld = np + 3;
    const int team = TEAM == 32 ? (int)(threadIdx.x >> 5) : 0;
    const int teams = TEAM == 32 ? (int)(blockDim.x >> 5) : 1;
    unsigned char *base = smraw + (size_t)team * WarpJacobiSmem::per_team(nw);
    float2 *A = reinterpret_cast<float2 *>(base);
    float2 *V = A + (size_t)np * ld;
    float2 *rot_s = V + (size_t)np * ld;
    float *rot_c = reinterpret_cast<float *>(rot_s + 16);
    const int t = Team<TEAM>::rank();
    const int64_t nteams = (int64_t)gridDim.x * teams;
    const int64_t gt = (int64_t)blockIdx.x * teams + team;
    const int64_t kb = (batch * gt) / nteams, ke = (batch * (gt + 1)) / nteams;
    float2 col[ROWS];
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *h = h_in + b * h_stride;
        double fro;
        if (b == kb || !warm_start) {
            fro = team_load_hermitian<TEAM>(A, h, nw, np, ld, red);
            for (int e = t; e < np * np; e += TEAM) {
                const int i = e % np, j = e / np;
                V[i + ld * j] = make_float2(i == j ? 1.0f : 0.0f, 0.0f);
            }
            Team<TEAM>::sync();
        } else {
            // Warm start from the previous point's V: V <- V (3I - V^H V)/2 and A <- V^H H V; the
            // second factor of every product is read from shared memory (A serves as scratch).
            const int c0 = t & 31, r0 = (t >> 5) * ROWS;
            team_column_product<TEAM>(V, V, col, np, ld, true);                // (V^H V)[:, c0]
#pragma unroll
            for (int i = 0; i < ROWS; ++i)
                col[i] = make_float2((r0 + i == c0 ? 1.5f : 0.0f) - 0.5f * col[i].x, -0.5f * col[i].y);
            team_store_column<TEAM>(A, col, np, ld);                           // A <- M
            Team<TEAM>::sync();
            team_column_product<TEAM>(V, A, col, np, ld, false);               // (V M)[:, c0]
            Team<TEAM>::sync();
            team_store_column<TEAM>(V, col, np, ld);
            fro = team_load_hermitian<TEAM>(A, h, nw, np, ld, red);            // A <- H
            team_column_product<TEAM>(A, V, col, np, ld, false);               // (H V)[:, c0]
            Team<TEAM>::sync();
            team_store_column<TEAM>(A, col, np, ld);                           // A <- H V
            Team<TEAM>::sync();
            team_column_product<TEAM>(V, A, col, np, ld, true);                // (V^H H V)[:, c0]
            Team<TEAM>::sync();
            team_store_column<TEAM>(A, col, np, ld);
            Team<TEAM>::sync();
            const int row = t & 31;
            if (row < np)
                for (int i = row + (t >> 5); i < np; i += TEAM / 32) {
                    if (i > row) A[i + ld * row] = cconj(A[row + ld * i]);
                    else A[i + ld * i].y = 0.0f;
                }
            Team<TEAM>::sync();
        }
        // The FP64 stage converges quadratically from here: the FP32 stage stops once the
        // off-diagonal norm is below 2^-17 ||H|| (rotating elements above 2^-20 ||H||).
        const float tol32 = (float)(fro * 9.5367431640625e-07);
        for (int sweep = 0; sweep < WNLQG_JACOBI_MAX_SWEEPS; ++sweep) {
            const double off = team_offdiag2<TEAM>(A, np, ld, red);
            if (sqrt(off) <= fro * 7.62939453125e-06) break;
            if (!team_jacobi_sweep<float, TEAM>(A, V, np, ld, tol32, rot_s, rot_c)) break;
        }
        float2 *vo = V_out + b * (int64_t)np * np;
        for (int e = t; e < np * np; e += TEAM) {
            const int i = e % np, j = e / np;
            vo[i + (int64_t)np * j] = V[i + ld * j];
        }
        Team<TEAM>::sync();
    }
}

// First-order completion of the FP64 refinement.  After one FP64 sweep the off-diagonal of A is
// quadratically small; when every |a_ij| <= tau |d_i - d_j| (tau = 2^-26), the eigenvectors of A are
// e_j + sum_{i != j} e_i a_ij / (d_j - d_i) and its eigenvalues d_j + sum_{i != j} |a_ij|^2 / (d_j - d_i)
// up to terms in products of two such ratios (<= tau^2 = 2^-52: first-order perturbation theory),
// so W (I + E) with E_ij = a_ij / (d_j - d_i) (anti-Hermitian, hence unitary to the same order)
// reaches what a further sweep would, for one product instead of np - 1 rotation rounds.  The
// mixed path, whose response arithmetic is FP32, takes tau = 2^-13 straight after the FP32 stage
// (eigenvector error <= 2^-26, below that arithmetic) in place of its one FP64 sweep; there E is
// no longer negligible against FP64 rounding, so the rotation is I + E + E^2 / 2 = ((I + E)^2 + I) / 2,
// whose deviation from unitarity is |E|^4 / 4 instead of |E|^2.  Returns false, with A and W
// untouched, when some pair is too close for the bound (the caller then sweeps).  dnew: np
// doubles of the team's scratch.
template <int TEAM>
WNLQG_D bool team_first_order_completion(double2 *A, double2 *W, int np, int ld, double *dnew, double tau) {
    const int t = Team<TEAM>::rank();
    bool bad = false;
    for (int e = t; e < np * np; e += TEAM) {
        const int i = e % np, j = e / np;
        const double2 a = A[i + ld * j];
        if (i == j || (a.x == 0.0 && a.y == 0.0)) continue;
        if (!(hypot(a.x, a.y) <= tau * fabs(A[j + ld * j].x - A[i + ld * i].x))) bad = true;
    }
    if (Team<TEAM>::any(bad)) return false;
    if (t < np) {
        const double dj = A[t + ld * t].x;
        double s = 0.0;
        for (int i = 0; i < np; ++i) {
            const double2 a = A[i + ld * t];
            if (i == t || (a.x == 0.0 && a.y == 0.0)) continue;
            s += (a.x * a.x + a.y * a.y) / (dj - A[i + ld * i].x);
        }
        dnew[t] = dj + s;
    }
    Team<TEAM>::sync();
    // A <- I + E: the off-diagonal in place (reading only the unchanged diagonal), then the diagonal.
    for (int e = t; e < np * np; e += TEAM) {
        const int i = e % np, j = e / np;
        const double2 a = A[i + ld * j];
        if (i == j || (a.x == 0.0 && a.y == 0.0)) continue;
        const double g = A[j + ld * j].x - A[i + ld * i].x;
        A[i + ld * j] = make_double2(a.x / g, a.y / g);
    }
    Team<TEAM>::sync();
    if (t < np) A[t + ld * t] = make_double2(1.0, 0.0);
    Team<TEAM>::sync();
    if constexpr (TEAM == 128) {
        if (tau > 1.4901161193847656e-08) {
            team128_dmma<false>(A, A, A, np, ld, [](int r, int c, double2 v) {   // A <- I + E + E^2 / 2
                return make_double2(0.5 * (v.x + (r == c ? 1.0 : 0.0)), 0.5 * v.y);
            });
            Team<TEAM>::sync();
        }
        team128_dmma<false>(W, A, W, np, ld, [](int, int, double2 v) { return v; });   // W <- W A
        if (t < np) A[t + ld * t] = make_double2(dnew[t], 0.0);
        Team<TEAM>::sync();
        return true;
    }
    double2 col[Team<TEAM>::ROWS];
    if (tau > 1.4901161193847656e-08) {
        constexpr int ROWS = Team<TEAM>::ROWS;
        const int c0 = t & 31, r0 = (t >> 5) * ROWS;
        team_column_product<TEAM>(A, A, col, np, ld, false);                // ((I + E)^2)[:, c0]
        Team<TEAM>::sync();
#pragma unroll
        for (int i = 0; i < ROWS; ++i)
            col[i] = make_double2(0.5 * (col[i].x + (r0 + i == c0 ? 1.0 : 0.0)), 0.5 * col[i].y);
        team_store_column<TEAM>(A, col, np, ld);                            // A <- I + E + E^2 / 2
        Team<TEAM>::sync();
    }
    team_column_product<TEAM>(W, A, col, np, ld, false);                    // (W A)[:, c0]
    Team<TEAM>::sync();
    team_store_column<TEAM>(W, col, np, ld);
    if (t < np) A[t + ld * t] = make_double2(dnew[t], 0.0);
    Team<TEAM>::sync();
    return true;
}

// Stage 2: FP64 A and W in the team's shared memory.
// W = V (I - E/2 + 3E^2/8) with E = V^H V - I (second-order Loewdin), H' = W^H H W, then FP64
// Jacobi sweeps on H' (quadratic convergence: the off-diagonal goes from the FP32 stage's
// 2^-17 ||H|| to the square of that over the gap), then ascending order and canonical phases.
// converge = 0 (mixed path): one sweep unless H' is already diagonal to 1e-13 ||H||, or the
// first-order completion with tau = 2^-13 in its place.
// converge = 1 (FP64 path): sweeps until the FP64 CTA Jacobi's stopping rule holds (off-diagonal
// norm <= np 2^-60 ||H||, or a sweep with every |a_pq| <= 2^-60 ||H||), so the FP32 stage only
// preconditions and the result carries the FP64 solver's accuracy; from the second sweep on, a
// first-order completion replaces the sweep whenever its bound holds (team_first_order_completion;
// measured on the nw = 32 workload: 6.8 ms of the 33.0 ms eigensolve per 65536 points is one sweep).
struct WarpRefineSmem {
    static __host__ __device__ size_t per_team(int nw) {
        const int np = nw + (nw & 1);
        const int ld = np + 3;
        size_t s = 2 * (size_t)np * ld * sizeof(double2) + 16 * (sizeof(double2) + sizeof(double) + 2 * sizeof(int)) +
                   32 * (sizeof(double2) + sizeof(int));
        return (s + 15) & ~(size_t)15;
    }
};

// Blocks of 64 threads holding two teams (TEAM = 32), otherwise blocks of TEAM threads (one team).
template <int TEAM>
__global__ void __launch_bounds__(TEAM == 128 ? 128 : 64, TEAM == 32 ? 1 : (TEAM == 128 ? 5 : 6)) eigh_refine_f64_team_kernel(const double2 *__restrict__ h_in, int64_t h_stride,
                                                                  const float2 *__restrict__ V_in, int64_t batch, int nw,
                                                                  double *__restrict__ E_out, double2 *__restrict__ U_out,
                                                                  int converge) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int ROWS = Team<TEAM>::ROWS;
    __shared__ double red[4];
    const int np = nw + (nw & 1);
    const int ld = np + 3;
    const int team = TEAM == 32 ? (int)(threadIdx.x >> 5) : 0;
    const int teams = TEAM == 32 ? (int)(blockDim.x >> 5) : 1;
    unsigned char *base = smraw + (size_t)team * WarpRefineSmem::per_team(nw);
    double2 *A = reinterpret_cast<double2 *>(base);
    double2 *W = A + (size_t)np * ld;
    double2 *rot_s = W + (size_t)np * ld;
    double2 *phase = rot_s + 16;
    double *rot_c = reinterpret_cast<double *>(phase + 32);
    int *rank = reinterpret_cast<int *>(rot_c + 16) + 32;
    const int t = Team<TEAM>::rank();
    const int c0 = t & 31, r0 = (t >> 5) * ROWS;
    const int64_t nteams = (int64_t)gridDim.x * teams;
    double2 col[ROWS];
    for (int64_t b = (int64_t)blockIdx.x * teams + team; b < batch; b += nteams) {
        const float2 *vi = V_in + b * (int64_t)np * np;
        for (int e = t; e < np * np; e += TEAM) {
            const int i = e % np, j = e / np;
            W[i + ld * j] = to_c64(vi[i + np * j]);
        }
        Team<TEAM>::sync();
        // E = V^H V - I into A; then M = I - E/2 + 3 E^2 / 8 into A; W <- V M.
        if constexpr (TEAM == 128) {
            team128_dmma<true>(W, W, A, np, ld, [](int r, int c, double2 v) {
                return make_double2(v.x - (r == c ? 1.0 : 0.0), v.y);
            });
            Team<TEAM>::sync();
            team128_dmma<false>(A, A, A, np, ld, [&](int r, int c, double2 v) {      // (E^2), then M
                const double2 e = A[r + ld * c];
                return make_double2((r == c ? 1.0 : 0.0) - 0.5 * e.x + 0.375 * v.x, -0.5 * e.y + 0.375 * v.y);
            });
            Team<TEAM>::sync();
            team128_dmma<false>(W, A, W, np, ld, [](int, int, double2 v) { return v; });   // W <- V M
        } else {
        team_column_product<TEAM>(W, W, col, np, ld, true);
#pragma unroll
        for (int i = 0; i < ROWS; ++i)
            if (r0 + i == c0) col[i].x -= 1.0;
        team_store_column<TEAM>(A, col, np, ld);
        Team<TEAM>::sync();
        team_column_product<TEAM>(A, A, col, np, ld, false);                 // (E^2)[:, c0]
#pragma unroll
        for (int i = 0; i < ROWS; ++i) {
            if (r0 + i < np && c0 < np) {
                const double2 e = A[(r0 + i) + ld * c0];
                col[i] = make_double2((r0 + i == c0 ? 1.0 : 0.0) - 0.5 * e.x + 0.375 * col[i].x, -0.5 * e.y + 0.375 * col[i].y);
            }
        }
        Team<TEAM>::sync();
        team_store_column<TEAM>(A, col, np, ld);
        Team<TEAM>::sync();
        team_column_product<TEAM>(W, A, col, np, ld, false);                 // (V M)[:, c0]
        Team<TEAM>::sync();
        team_store_column<TEAM>(W, col, np, ld);
        }
        // A <- W^H H W (exactly Hermitian); returns ||H||_F.
        auto project = [&]() {
            const double f = team_load_hermitian<TEAM>(A, h_in + b * h_stride, nw, np, ld, red);   // A <- H
            if constexpr (TEAM == 128) {
                team128_dmma<false>(A, W, A, np, ld, [](int, int, double2 v) { return v; });   // A <- H W
                Team<TEAM>::sync();
                team128_dmma<true>(W, A, A, np, ld, [](int, int, double2 v) { return v; });    // A <- W^H H W
                Team<TEAM>::sync();
            } else {
            team_column_product<TEAM>(A, W, col, np, ld, false);             // (H W)[:, c0]
            Team<TEAM>::sync();
            team_store_column<TEAM>(A, col, np, ld);
            Team<TEAM>::sync();
            team_column_product<TEAM>(W, A, col, np, ld, true);              // (W^H H W)[:, c0]
            Team<TEAM>::sync();
            team_store_column<TEAM>(A, col, np, ld);
            Team<TEAM>::sync();
            }
            const int row = t & 31;
            if (row < np)
                for (int i = row + (t >> 5); i < np; i += TEAM / 32) {
                    if (i > row) A[i + ld * row] = cconj(A[row + ld * i]);
                    else A[i + ld * i].y = 0.0;
                }
            Team<TEAM>::sync();
            return f;
        };
        const double fro = project();
        const double tol = fro * 8.673617379884035e-19;
        double *dnew = reinterpret_cast<double *>(phase);
        // FP64 path: a loose completion (2^-13) straight from the FP32 stage and a fresh projection
        // square the off-diagonal ratios, after which the strict completion (2^-26) normally holds
        // without any sweep; the sweeps remain the fallback of either bound.
        bool loose = false;
        if (converge && team_first_order_completion<TEAM>(A, W, np, ld, dnew, 1.220703125e-04)) {
            loose = true;
            project();
        }
        for (int sweep = 0; sweep < (converge ? WNLQG_JACOBI_MAX_SWEEPS : 1); ++sweep) {
            const double off = team_offdiag2<TEAM>(A, np, ld, red);
            if (sqrt(off) <= (converge ? tol * np : fro * 1.0e-13)) break;
            if ((converge ? (sweep > 0 || loose) : sweep == 0) &&
                team_first_order_completion<TEAM>(A, W, np, ld, dnew, converge ? 1.4901161193847656e-08 : 1.220703125e-04))
                break;
            if (!team_jacobi_sweep<double, TEAM>(A, W, np, ld, tol, rot_s, rot_c)) break;
        }
        // Ascending order (stable) and canonical phases: thread i handles eigenpair i, then the
        // columns are written row-wise (coalesced), the warps taking alternate columns.
        if (t < nw) {
            const double di = A[t + ld * t].x;
            int r = 0;
            for (int j = 0; j < nw; ++j) {
                const double dj = A[j + ld * j].x;
                r += (dj < di) || (dj == di && j < t);
            }
            int pivot = 0;
            double pm = hypot(W[0 + ld * t].x, W[0 + ld * t].y);
            for (int rr = 1; rr < nw; ++rr) {
                const double mg = hypot(W[rr + ld * t].x, W[rr + ld * t].y);
                if (mg > pm) { pm = mg; pivot = rr; }
            }
            phase[t] = pm > 0.0 ? make_double2(W[pivot + ld * t].x / pm, -W[pivot + ld * t].y / pm)
                                : make_double2(1.0, 0.0);
            rank[t] = r;
            E_out[b * nw + r] = di;
        }
        Team<TEAM>::sync();
        double2 *u = U_out + b * (int64_t)nw * nw;
        const int row = t & 31;
        for (int c = t >> 5; c < nw; c += TEAM / 32)
            if (row < nw) u[row + (int64_t)nw * rank[c]] = cmul(W[row + ld * c], phase[c]);
        Team<TEAM>::sync();
    }
}
// ---------------------------------------------------------------------------------------------
// Mixed-precision eigensolver above 32 orbitals, one CTA per matrix, in two kernels (the same
// scheme as the team kernels, for matrices a warp team cannot hold):
//   stage 1 (jacobi_f32_cta_kernel): FP32 parallel Jacobi until the off-diagonal norm is below
//     2^-17 ||H|| (rotating elements above 2^-20 ||H||), eigenvectors written unsorted; each CTA
//     takes a contiguous range of points and, along mesh runs and Morton-ordered point batches,
//     warm-starts each point from the previous one's eigenvectors;
//   stage 2 (eigh_refine_f64_cta_kernel): W = second-order Loewdin orthonormalisation of V
//     (E = W^H W - I, W <- W (I - E/2 + 3E^2/8)), H' = W^H H W, FP64 Jacobi sweeps (mixed path:
//     one, unless H' is diagonal to 1e-13 ||H||; FP64 path: until the FP64 CTA Jacobi's stopping
//     rule holds, np 2^-60 ||H||, from the second sweep on replaced by the first-order completion
//     when its bound holds), U = W J, ascending order and canonical phases.  The products run on
//     the FP64 tensor cores (dmma_product).
// GW: the working set lives in global memory (gscratch, one stride per CTA) when it does not fit
// shared memory.
// ---------------------------------------------------------------------------------------------
// out = op(X) Y for np x np FP32 complex matrices with leading dimensions ldx, ldy, ldo (either
// input may live in global memory), op = conjugate transpose when xh; the CTA's threads take
// out's elements in turn, rows fastest.
WNLQG_D void cta_product_f32(const float2 *X, int ldx, const float2 *Y, int ldy, float2 *out, int ldo, int np, bool xh) {
    for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
        const int i = e % np, j = e / np;
        float2 acc = make_float2(0.0f, 0.0f);
        if (xh)
            for (int l = 0; l < np; ++l) acc = cfmaconj(X[l + ldx * i], Y[l + ldy * j], acc);
        else
            for (int l = 0; l < np; ++l) acc = cfma(X[i + ldx * l], Y[l + ldy * j], acc);
        out[i + ldo * j] = acc;
    }
}

// Each CTA takes a contiguous range of the batch.  warm_start: every point after the first of the
// range starts from the previous point's eigenvectors Vp (already in V_out; this point's V_out
// slot serves as the scratch W): W = Vp (3I - Vp^H Vp)/2, A = W^H H W, V = W.
template <bool GW>
__global__ void __launch_bounds__(256, 3) jacobi_f32_cta_kernel(const double2 *__restrict__ h_in, int64_t h_stride,
                                                              int64_t batch, int nw, float2 *V_out,
                                                              unsigned char *gscratch, int64_t gscratch_stride,
                                                              int warm_start) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *smraw;
    if constexpr (GW) smraw = gscratch + (int64_t)blockIdx.x * gscratch_stride;
    else smraw = smem_dyn;
    const int np = nw + (nw & 1);
    const int ld = np + 1;
    const int half = np / 2;
    float2 *A = reinterpret_cast<float2 *>(smraw);
    float2 *V = A + (size_t)np * ld;
    float2 *rot_s = V + (size_t)np * ld;
    double *scratch = reinterpret_cast<double *>(rot_s + half);
    float *rot_c = reinterpret_cast<float *>(scratch + 2);
    int *rot_p = reinterpret_cast<int *>(rot_c + half);
    int *rot_q = rot_p + half;
    __shared__ double red[48];
    __shared__ int rot_flag;
    const int tid = threadIdx.x;
    const int64_t nn = (int64_t)np * np;
    const int64_t kb = (batch * (int64_t)blockIdx.x) / gridDim.x, ke = (batch * ((int64_t)blockIdx.x + 1)) / gridDim.x;
    for (int64_t b = kb; b < ke; ++b) {
        const double2 *h = h_in + b * h_stride;
        const bool warm = warm_start && b > kb;
        float2 *Wg = V_out + b * nn;
        const float2 *Vp = warm ? V_out + (b - 1) * nn : nullptr;
        if (warm) {
            cta_product_f32(Vp, np, Vp, np, V, ld, np, true);                  // V <- Vp^H Vp
            __syncthreads();
            for (int e = tid; e < np * np; e += blockDim.x) {                   // V <- M = (3I - V)/2
                const int i = e % np, j = e / np;
                const float2 m = V[i + ld * j];
                V[i + ld * j] = make_float2((i == j ? 1.5f : 0.0f) - 0.5f * m.x, -0.5f * m.y);
            }
            __syncthreads();
            cta_product_f32(Vp, np, V, ld, Wg, np, np, false);                 // W <- Vp M (global)
        }
        double local = 0.0;
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int i = e % np, j = e / np;
            double2 v = make_double2(0.0, 0.0);
            if (i < nw && j < nw) {
                if (i < j) v = h[i + (size_t)nw * j];
                else if (i > j) v = cconj(h[j + (size_t)nw * i]);
                else v = make_double2(h[i + (size_t)nw * i].x, 0.0);
            }
            local += v.x * v.x + v.y * v.y;
            A[i + ld * j] = make_float2((float)v.x, (float)v.y);
            if (!warm) V[i + ld * j] = make_float2(i == j ? 1.0f : 0.0f, 0.0f);
        }
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((tid & 31) == 0) red[tid >> 5] = local;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
            scratch[0] = sqrt(s);
        }
        __syncthreads();
        if (warm) {
            cta_product_f32(A, ld, Wg, np, V, ld, np, false);                  // V <- H W
            __syncthreads();
            cta_product_f32(Wg, np, V, ld, A, ld, np, true);                   // A <- W^H H W
            __syncthreads();
            for (int e = tid; e < np * np; e += blockDim.x) {                   // V <- W; A Hermitian
                const int i = e % np, j = e / np;
                V[i + ld * j] = Wg[i + (int64_t)np * j];
                if (i > j) A[i + ld * j] = cconj(A[j + ld * i]);
                else if (i == j) A[i + ld * i].y = 0.0f;
            }
            __syncthreads();
        }
        const double fro = scratch[0];
        const float tol32 = (float)(fro * 9.5367431640625e-07);
        for (int sweep = 0; sweep < WNLQG_JACOBI_MAX_SWEEPS; ++sweep) {
            if (offdiag_norm(A, np, ld, red) <= fro * 7.62939453125e-06) break;
            if (tid == 0) rot_flag = 0;
            __syncthreads();
            jacobi_sweep<float>(A, V, np, ld, tol32, rot_s, rot_c, rot_p, rot_q, &rot_flag);
            const int any = rot_flag;
            __syncthreads();
            if (!any) break;
        }
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int i = e % np, j = e / np;
            Wg[i + (int64_t)np * j] = V[i + ld * j];
        }
        __syncthreads();
    }
}

struct RefineCtaSmem {
    // A, W, T (np x ld complex double), rotation sines, cosines and pair indices, scratch.
    static __host__ __device__ size_t bytes(int nw) {
        const int np = nw + (nw & 1);
        const int ld = np + 1;
        const int half = np / 2;
        size_t s = 3 * (size_t)np * ld * sizeof(double2);
        s += (size_t)half * (sizeof(double2) + sizeof(double) + 2 * sizeof(int));
        return (s + 15) & ~(size_t)15;
    }
};

// The CTA form of team_first_order_completion (the same bound and algebra, the product on the
// FP64 tensor cores): on success W <- W (I + E) (Wc and Tc swap roles) and A's diagonal holds the
// second-order eigenvalues.  dnew: np doubles of shared scratch.
WNLQG_D bool cta_first_order_completion(double2 *A, double2 *&Wc, double2 *&Tc, int np, int ld, double *dnew,
                                        double tau) {
    const int tid = threadIdx.x;
    int bad = 0;
    for (int e = tid; e < np * np; e += blockDim.x) {
        const int i = e % np, j = e / np;
        const double2 a = A[i + ld * j];
        if (i == j || (a.x == 0.0 && a.y == 0.0)) continue;
        if (!(hypot(a.x, a.y) <= tau * fabs(A[j + ld * j].x - A[i + ld * i].x))) bad = 1;
    }
    if (__syncthreads_or(bad)) return false;
    for (int j = tid; j < np; j += blockDim.x) {
        const double dj = A[j + ld * j].x;
        double s = 0.0;
        for (int i = 0; i < np; ++i) {
            const double2 a = A[i + ld * j];
            if (i == j || (a.x == 0.0 && a.y == 0.0)) continue;
            s += (a.x * a.x + a.y * a.y) / (dj - A[i + ld * i].x);
        }
        dnew[j] = dj + s;
    }
    __syncthreads();
    for (int e = tid; e < np * np; e += blockDim.x) {
        const int i = e % np, j = e / np;
        const double2 a = A[i + ld * j];
        if (i == j || (a.x == 0.0 && a.y == 0.0)) continue;
        const double g = A[j + ld * j].x - A[i + ld * i].x;
        A[i + ld * j] = make_double2(a.x / g, a.y / g);
    }
    __syncthreads();
    for (int i = tid; i < np; i += blockDim.x) A[i + ld * i] = make_double2(1.0, 0.0);
    __syncthreads();
    if (tau > 1.4901161193847656e-08) {                      // A <- ((I + E)^2 + I) / 2
        dmma_product<0>(A, A, Tc, np, ld);
        __syncthreads();
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int i = e % np, j = e / np;
            const double2 v = Tc[i + ld * j];
            A[i + ld * j] = make_double2(0.5 * (v.x + (i == j ? 1.0 : 0.0)), 0.5 * v.y);
        }
        __syncthreads();
    }
    dmma_product<0>(Wc, A, Tc, np, ld);                      // T = W A
    __syncthreads();
    double2 *x = Wc;
    Wc = Tc;
    Tc = x;
    for (int i = tid; i < np; i += blockDim.x) A[i + ld * i] = make_double2(dnew[i], 0.0);
    __syncthreads();
    return true;
}

template <bool GW>
__global__ void __launch_bounds__(512, 1) eigh_refine_f64_cta_kernel(const double2 *__restrict__ h_in, int64_t h_stride,
                                                                   const float2 *__restrict__ V_in, int64_t batch, int nw,
                                                                   double *__restrict__ E_out, double2 *__restrict__ U_out,
                                                                   int converge, unsigned char *gscratch,
                                                                   int64_t gscratch_stride) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *smraw;
    if constexpr (GW) smraw = gscratch + (int64_t)blockIdx.x * gscratch_stride;
    else smraw = smem_dyn;
    const int np = nw + (nw & 1);
    const int ld = np + 1;
    const int half = np / 2;
    const size_t mat = (size_t)np * ld;
    double2 *A = reinterpret_cast<double2 *>(smraw);
    double2 *W = A + mat;
    double2 *T = W + mat;
    double2 *rot_s = T + mat;
    double *rot_c = reinterpret_cast<double *>(rot_s + half);
    int *rot_p = reinterpret_cast<int *>(rot_c + half);
    int *rot_q = rot_p + half;
    __shared__ double red[48];
    __shared__ int rot_flag;
    const int tid = threadIdx.x;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        double2 *Wc = W, *Tc = T;
        const float2 *vi = V_in + b * (int64_t)np * np;
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int i = e % np, j = e / np;
            Wc[i + ld * j] = to_c64(vi[i + np * j]);
        }
        __syncthreads();
        dmma_product<1>(Wc, Wc, Tc, np, ld);                 // T = W^H W
        __syncthreads();
        for (int i = tid; i < np; i += blockDim.x) Tc[i + ld * i].x -= 1.0;   // E = W^H W - I
        __syncthreads();
        dmma_product<0>(Tc, Tc, A, np, ld);                  // A = E^2
        __syncthreads();
        for (int e = tid; e < np * np; e += blockDim.x) {    // A = M = I - E/2 + 3 E^2 / 8
            const int i = e % np, j = e / np, o = i + ld * j;
            const double2 ev = Tc[o], e2 = A[o];
            A[o] = make_double2((i == j ? 1.0 : 0.0) - 0.5 * ev.x + 0.375 * e2.x, -0.5 * ev.y + 0.375 * e2.y);
        }
        __syncthreads();
        dmma_product<0>(Wc, A, Tc, np, ld);                  // T = W M
        __syncthreads();
        { double2 *x = Wc; Wc = Tc; Tc = x; }                // W <- W M
        // A <- H (Hermitian from the upper triangle, zero-padded), Frobenius norm.
        const double2 *h = h_in + b * h_stride;
        double local = 0.0;
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int i = e % np, j = e / np;
            double2 v = make_double2(0.0, 0.0);
            if (i < nw && j < nw) {
                if (i < j) v = h[i + (size_t)nw * j];
                else if (i > j) v = cconj(h[j + (size_t)nw * i]);
                else v = make_double2(h[i + (size_t)nw * i].x, 0.0);
            }
            local += v.x * v.x + v.y * v.y;
            A[i + ld * j] = v;
        }
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((tid & 31) == 0) red[tid >> 5] = local;
        __syncthreads();
        double fro = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) fro += red[w];
        fro = sqrt(fro);
        dmma_product<0>(A, Wc, Tc, np, ld);                  // T = H W
        __syncthreads();
        dmma_product<1>(Wc, Tc, A, np, ld);                  // A = W^H H W
        __syncthreads();
        for (int e = tid; e < np * np; e += blockDim.x) {    // exact Hermitian symmetry
            const int i = e % np, j = e / np;
            if (i > j) A[i + ld * j] = cconj(A[j + ld * i]);
            else if (i == j) A[i + ld * i].y = 0.0;
        }
        __syncthreads();
        const double tol = fro * 8.673617379884035e-19;
        for (int sweep = 0; sweep < (converge ? WNLQG_JACOBI_MAX_SWEEPS : 1); ++sweep) {
            const double off = offdiag_norm(A, np, ld, red);
            if (off <= (converge ? tol * np : fro * 1.0e-13)) break;
            if ((converge ? sweep > 0 : sweep == 0) &&
                cta_first_order_completion(A, Wc, Tc, np, ld, reinterpret_cast<double *>(rot_s),
                                           converge ? 1.4901161193847656e-08 : 1.220703125e-04))
                break;
            if (tid == 0) rot_flag = 0;
            __syncthreads();
            jacobi_sweep<double>(A, Wc, np, ld, tol, rot_s, rot_c, rot_p, rot_q, &rot_flag);
            const int any = rot_flag;
            __syncthreads();
            if (!any) break;
        }
        // Ascending order (stable), then phase canonicalisation per column.
        for (int i = tid; i < nw; i += blockDim.x) {
            const double di = A[i + ld * i].x;
            int rank = 0;
            for (int j = 0; j < nw; ++j) {
                const double dj = A[j + ld * j].x;
                rank += (dj < di) || (dj == di && j < i);
            }
            int pivot = 0;
            double pm = hypot(Wc[0 + ld * i].x, Wc[0 + ld * i].y);
            for (int r = 1; r < nw; ++r) {
                const double mg = hypot(Wc[r + ld * i].x, Wc[r + ld * i].y);
                if (mg > pm) { pm = mg; pivot = r; }
            }
            double2 phase = make_double2(1.0, 0.0);
            if (pm > 0.0) phase = make_double2(Wc[pivot + ld * i].x / pm, -Wc[pivot + ld * i].y / pm);
            E_out[b * nw + rank] = di;
            double2 *u = U_out + b * (int64_t)nw * nw + (int64_t)nw * rank;
            for (int r = 0; r < nw; ++r) u[r] = cmul(Wc[r + ld * i], phase);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Generalised Hermitian eigensolve H C = S C E for nonorthogonal models, FP64
// (generalized_hermitian_spectrum, DenseSpectra.jl:33-39: eigen(Hermitian(H,:U), Hermitian(S,:U))).
// S = L L^H (Cholesky, lower), Ht = L^-1 H L^-H, Jacobi on Ht, C = L^-H Ut, so C^H S C = I; then
// ascending order and the canonical phase rule (NonorthogonalMatrixElements.jl:382-385).
// A non-positive pivot of S sets the k-point's status word to 1 (S(k) not positive definite).
// ---------------------------------------------------------------------------------------------
struct GenEighSmem {
    static __host__ __device__ size_t bytes(int nw) {
        int np = nw + (nw & 1);
        int ld = np + 1;
        return 3 * (size_t)np * ld * sizeof(double2) + (size_t)(np / 2) * (sizeof(double2) + sizeof(double) + 2 * sizeof(int)) + 64;
    }
};

// S = L L^H (lower Cholesky factor in Lm) and A = L^-1 H L^-H (Hermitian, full) for one padded
// np x np matrix, CTA-wide; V is scratch.  Sets *bad when a pivot of S is not positive.
WNLQG_D void gen_cholesky_reduce(const double2 *__restrict__ h, const double2 *__restrict__ sk, int nw, int np,
                                 int ld, double2 *A, double2 *V, double2 *Lm, int *bad) {
    const int tid = threadIdx.x;
    if (tid == 0) *bad = 0;
    for (int e = tid; e < np * np; e += blockDim.x) {
        const int i = e % np, j = e / np;
        double2 hv = make_double2(0.0, 0.0), sv = make_double2(i == j ? 1.0 : 0.0, 0.0);
        if (i < nw && j < nw) {
            if (i < j) { hv = h[i + (size_t)nw * j]; sv = sk[i + (size_t)nw * j]; }
            else if (i > j) { hv = cconj(h[j + (size_t)nw * i]); sv = cconj(sk[j + (size_t)nw * i]); }
            else { hv = make_double2(h[i + (size_t)nw * i].x, 0.0); sv = make_double2(sk[i + (size_t)nw * i].x, 0.0); }
        }
        A[i + ld * j] = hv;
        Lm[i + ld * j] = sv;
    }
    __syncthreads();
    // Right-looking Cholesky in place (lower triangle of Lm).
    for (int j = 0; j < np; ++j) {
        if (tid == 0) {
            const double d = Lm[j + ld * j].x;
            if (!(d > 0.0)) *bad = 1;
            Lm[j + ld * j] = make_double2(d > 0.0 ? sqrt(d) : 1.0, 0.0);
        }
        __syncthreads();
        const double ljj = Lm[j + ld * j].x;
        for (int i = j + 1 + tid; i < np; i += blockDim.x) Lm[i + ld * j] = cscale(Lm[i + ld * j], 1.0 / ljj);
        __syncthreads();
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int r = e % np, c = e / np;
            if (c > j && r >= c) Lm[r + ld * c] = csub(Lm[r + ld * c], cmul(Lm[r + ld * j], cconj(Lm[c + ld * j])));
        }
        __syncthreads();
    }
    // X = L^-1 H (forward substitution, one thread per column), stored in V.
    for (int c = tid; c < np; c += blockDim.x)
        for (int r = 0; r < np; ++r) {
            double2 acc = A[r + ld * c];
            for (int k = 0; k < r; ++k) acc = csub(acc, cmul(Lm[r + ld * k], V[k + ld * c]));
            V[r + ld * c] = cscale(acc, 1.0 / Lm[r + ld * r].x);
        }
    __syncthreads();
    // Ht = X L^-H = (L^-1 X^H)^H: solve L Y = X^H column by column (column c of X^H is row c
    // of X, conjugated); Ht[c][r] = conj(Y[r][c]).
    for (int c = tid; c < np; c += blockDim.x)
        for (int r = 0; r < np; ++r) {
            double2 acc = cconj(V[c + ld * r]);
            for (int k = 0; k < r; ++k) acc = csub(acc, cmul(Lm[r + ld * k], cconj(A[c + ld * k])));
            A[c + ld * r] = cconj(cscale(acc, 1.0 / Lm[r + ld * r].x));
        }
    __syncthreads();
    // Hermitian part from the upper triangle.
    for (int e = tid; e < np * np; e += blockDim.x) {
        const int i = e % np, j = e / np;
        if (i > j) A[i + ld * j] = cconj(A[j + ld * i]);
        if (i == j) A[i + ld * i].y = 0.0;
    }
    __syncthreads();
}

template <bool GW = false>
__global__ void generalized_eigh_kernel(const double2 *__restrict__ h_in, const double2 *__restrict__ s_in,
                                        int64_t stride, int64_t batch, int nw, double *__restrict__ E_out,
                                        double2 *__restrict__ U_out, int *__restrict__ status,
                                        unsigned char *gscratch = nullptr, int64_t gscratch_stride = 0) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *smraw;
    if constexpr (GW) smraw = gscratch + (int64_t)blockIdx.x * gscratch_stride;
    else smraw = smem_dyn;
    const int np = nw + (nw & 1);
    const int ld = np + 1;
    const int half = np / 2;
    double2 *A = reinterpret_cast<double2 *>(smraw);     // H, then Ht, then the Jacobi matrix
    double2 *V = A + (size_t)np * ld;                    // Jacobi eigenvectors
    double2 *Lm = V + (size_t)np * ld;                   // S, then its Cholesky factor
    double2 *rot_s = Lm + (size_t)np * ld;
    double *rot_c = reinterpret_cast<double *>(rot_s + half);
    int *rot_p = reinterpret_cast<int *>(rot_c + half);
    int *rot_q = rot_p + half;
    __shared__ double red[48];
    __shared__ int rot_flag, bad;
    const int tid = threadIdx.x;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const double2 *h = h_in + b * stride;
        const double2 *sk = s_in + b * stride;
        gen_cholesky_reduce(h, sk, nw, np, ld, A, V, Lm, &bad);
        // Identity for the eigenvector accumulation.
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int i = e % np, j = e / np;
            V[i + ld * j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
        }
        __syncthreads();
        double local = 0.0;
        for (int e = tid; e < np * np; e += blockDim.x) {
            const double2 z = A[(e % np) + ld * (e / np)];
            local += z.x * z.x + z.y * z.y;
        }
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((tid & 31) == 0) red[tid >> 5] = local;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w];
            red[41] = sqrt(sum);
        }
        __syncthreads();
        const double tol = red[41] * 8.673617379884035e-19;
        for (int sweep = 0; sweep < WNLQG_JACOBI_MAX_SWEEPS; ++sweep) {
            if (offdiag_norm(A, np, ld, red) <= tol * np) break;
            if (tid == 0) rot_flag = 0;
            __syncthreads();
            jacobi_sweep<double>(A, V, np, ld, tol, rot_s, rot_c, rot_p, rot_q, &rot_flag);
            const int any = rot_flag;
            __syncthreads();
            if (!any) break;
        }
        // C = L^-H Ut (back substitution with L^H, one thread per column), in place in V.
        for (int c = tid; c < np; c += blockDim.x)
            for (int r = np - 1; r >= 0; --r) {
                double2 acc = V[r + ld * c];
                for (int k = r + 1; k < np; ++k) acc = csub(acc, cmul(cconj(Lm[k + ld * r]), V[k + ld * c]));
                V[r + ld * c] = cscale(acc, 1.0 / Lm[r + ld * r].x);
            }
        __syncthreads();
        for (int i = tid; i < nw; i += blockDim.x) {
            const double di = A[i + ld * i].x;
            int rank = 0;
            for (int j = 0; j < nw; ++j) {
                const double dj = A[j + ld * j].x;
                rank += (dj < di) || (dj == di && j < i);
            }
            int pivot = 0;
            double pm = hypot(V[0 + ld * i].x, V[0 + ld * i].y);
            for (int r = 1; r < nw; ++r) {
                const double mg = hypot(V[r + ld * i].x, V[r + ld * i].y);
                if (mg > pm) { pm = mg; pivot = r; }
            }
            double2 phase = make_double2(1.0, 0.0);
            if (pm > 0.0) phase = make_double2(V[pivot + ld * i].x / pm, -V[pivot + ld * i].y / pm);
            E_out[b * nw + rank] = di;
            double2 *u = U_out + b * (int64_t)nw * nw + (int64_t)nw * rank;
            for (int r = 0; r < nw; ++r) u[r] = cmul(V[r + ld * i], phase);
        }
        if (tid == 0 && status) status[b] = bad;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Mixed-precision generalised eigensolve (nonorthogonal models on the mixed path): the FP64
// Cholesky S = L L^H and reduction C = L^-1 H L^-H (cholesky_reduce_kernel, the same arithmetic
// as generalized_eigh_kernel), the orthogonal mixed-precision stages on C (FP32 Jacobi, FP64
// refinement, ascending order and canonical phases of C's eigenvectors V), then U = L^-H V and
// the canonical phase rule on U (gen_back_substitute_kernel), so U^H S U = I.
// ---------------------------------------------------------------------------------------------
struct GenReduceSmem {
    static __host__ __device__ size_t bytes(int nw) {
        const int np = nw + (nw & 1);
        return 3 * (size_t)np * (np + 1) * sizeof(double2);
    }
};

template <bool GW>
__global__ void __launch_bounds__(256) cholesky_reduce_kernel(const double2 *__restrict__ h_in,
                                                              const double2 *__restrict__ s_in, int64_t stride,
                                                              int64_t batch, int nw, double2 *__restrict__ C_out,
                                                              double2 *__restrict__ L_out, int *__restrict__ status,
                                                              unsigned char *gscratch, int64_t gscratch_stride) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char *smraw;
    if constexpr (GW) smraw = gscratch + (int64_t)blockIdx.x * gscratch_stride;
    else smraw = smem_dyn;
    const int np = nw + (nw & 1);
    const int ld = np + 1;
    double2 *A = reinterpret_cast<double2 *>(smraw);
    double2 *V = A + (size_t)np * ld;
    double2 *Lm = V + (size_t)np * ld;
    __shared__ int bad;
    const int64_t nn = (int64_t)nw * nw;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        gen_cholesky_reduce(h_in + b * stride, s_in + b * stride, nw, np, ld, A, V, Lm, &bad);
        double2 *c = C_out + b * nn;
        double2 *l = L_out + b * nn;
        for (int e = threadIdx.x; e < nw * nw; e += blockDim.x) {
            const int i = e % nw, j = e / nw;
            c[e] = A[i + ld * j];
            l[e] = i >= j ? Lm[i + ld * j] : make_double2(0.0, 0.0);
        }
        if (threadIdx.x == 0) status[b] = bad;
        __syncthreads();
    }
}

// U <- L^-H U for each point's nw x nw eigenvector matrix (columns), L lower; then each column
// is rotated so that its largest-modulus entry is real and positive (first such entry on ties).
// One thread per column; L is read from global memory (every thread of a warp reads the same
// element at once).
__global__ void __launch_bounds__(128) gen_back_substitute_kernel(const double2 *__restrict__ L_in, double2 *U,
                                                                  int64_t batch, int nw) {
    const int64_t nn = (int64_t)nw * nw;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const double2 *L = L_in + b * nn;
        double2 *u = U + b * nn;
        for (int c = threadIdx.x; c < nw; c += blockDim.x) {
            double2 *col = u + (int64_t)nw * c;
            for (int r = nw - 1; r >= 0; --r) {
                double2 acc = col[r];
                for (int k = r + 1; k < nw; ++k) acc = csub(acc, cmul(cconj(L[k + (int64_t)nw * r]), col[k]));
                col[r] = cscale(acc, 1.0 / L[r + (int64_t)nw * r].x);
            }
            int pivot = 0;
            double pm = hypot(col[0].x, col[0].y);
            for (int r = 1; r < nw; ++r) {
                const double mg = hypot(col[r].x, col[r].y);
                if (mg > pm) { pm = mg; pivot = r; }
            }
            if (pm > 0.0) {
                const double2 ph = make_double2(col[pivot].x / pm, -col[pivot].y / pm);
                for (int r = 0; r < nw; ++r) col[r] = cmul(col[r], ph);
            }
        }
    }
}
