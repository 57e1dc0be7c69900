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

// T: real type of the iteration (double for the FP64 path, float for the mixed path).
// Input H(k) for batch entry b at h_in + b*h_stride (complex double, column-major nw x nw).
// Outputs: energies E[b*nw + n] (double) and U[b*nw*nw + i + nw*n] (complex double).
template <typename T>
__global__ void jacobi_eigh_kernel(const double2 *__restrict__ h_in, int64_t h_stride, int64_t batch, int nw,
                                   double *__restrict__ E_out, double2 *__restrict__ U_out, T tol_scale) {
    typedef typename cplx_of<T>::type C;
    extern __shared__ __align__(16) unsigned char smraw[];
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
    __shared__ int any_rotation;
    __shared__ double red[32];

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

        for (int sweep = 0; sweep < WNLQG_JACOBI_MAX_SWEEPS; ++sweep) {
            if (tid == 0) any_rotation = 0;
            __syncthreads();
            for (int round = 0; round < np - 1; ++round) {
                if (tid < half) {
                    // Circle method: slot 0 holds index 0, slots 1..np-1 hold ((j-1+round) mod (np-1)) + 1.
                    int s1 = tid, s2 = np - 1 - tid;
                    int i1 = s1 == 0 ? 0 : ((s1 - 1 + round) % (np - 1)) + 1;
                    int i2 = ((s2 - 1 + round) % (np - 1)) + 1;
                    int p = min(i1, i2), q = max(i1, i2);
                    C apq = A[p + ld * q];
                    T g = (T)hypot((double)apq.x, (double)apq.y);
                    T c = (T)1, s = (T)0;
                    C ph = from_c64<C>(make_double2(1.0, 0.0));
                    if (g > tol) {
                        T app = A[p + ld * p].x, aqq = A[q + ld * q].x;
                        T theta = (aqq - app) / ((T)2 * g);
                        T t = (theta >= (T)0 ? (T)1 : (T)-1) / (fabs(theta) + sqrt(theta * theta + (T)1));
                        c = (T)1 / sqrt(t * t + (T)1);
                        s = t * c;
                        ph.x = apq.x / g;
                        ph.y = apq.y / g;
                        any_rotation = 1;
                    }
                    rot_c[tid] = c;
                    rot_s[tid] = cscale(ph, s);
                    rot_p[tid] = p;
                    rot_q[tid] = q;
                }
                __syncthreads();
                for (int blk = tid; blk < half * half; blk += blockDim.x) {
                    int k1 = blk % half, k2 = blk / half;
                    int p1 = rot_p[k1], q1 = rot_q[k1], p2 = rot_p[k2], q2 = rot_q[k2];
                    T c1 = rot_c[k1], c2 = rot_c[k2];
                    C s1 = rot_s[k1], s2 = rot_s[k2];
                    C s2c = cconj(s2), s1c = cconj(s1);
                    // A block rows (p1,q1), cols (p2,q2): J1^H * a * J2.
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
                        // Diagonal 2x2 block: the rotated pair's coupling is zero by construction.
                        if (rot_s[k1].x != (T)0 || rot_s[k1].y != (T)0) {
                            o01 = czero<C>();
                            o10 = czero<C>();
                        }
                        o00.y = (T)0;
                        o11.y = (T)0;
                    }
                    A[p1 + ld * p2] = o00; A[p1 + ld * q2] = o01; A[q1 + ld * p2] = o10; A[q1 + ld * q2] = o11;
                    // V rows (p1,q1), cols (p2,q2): v * J2.
                    C v00 = V[p1 + ld * p2], v01 = V[p1 + ld * q2], v10 = V[q1 + ld * p2], v11 = V[q1 + ld * q2];
                    V[p1 + ld * p2] = csub(cscale(v00, c2), cmul(v01, s2c));
                    V[p1 + ld * q2] = cadd(cmul(v00, s2), cscale(v01, c2));
                    V[q1 + ld * p2] = csub(cscale(v10, c2), cmul(v11, s2c));
                    V[q1 + ld * q2] = cadd(cmul(v10, s2), cscale(v11, c2));
                }
                __syncthreads();
            }
            int done = any_rotation == 0;
            __syncthreads();
            if (done) break;
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
                double2 v = cmul(to_c64(V[r + ld * i]), phase);
                if (r == pivot) v.y = 0.0;
                u[r] = v;
            }
        }
        __syncthreads();
    }
}
