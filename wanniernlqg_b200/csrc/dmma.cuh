// dmma.cuh - CTA-wide products of complex FP64 matrices in shared memory on the FP64 tensor
// cores (DMMA: mma.sync.aligned.m8n8k4.row.col.f64, sm_80 and later, sm_100a included; tcgen05
// has no FP64 kind).
//
// A complex product C = op(X) Y is three real products (Gauss's three-multiplication form):
// P1 = Re A Re B, P2 = Im A Im B, P3 = (Re A + Im A)(Re B + Im B), each accumulated in FP64 by the
// tensor core, then Re C = P1 - P2 and Im C = P3 - P1 - P2.  Against the four-product form it
// issues a quarter fewer DMMAs and every accumulator chain takes one DMMA per K step instead of
// two; the imaginary part's error bound grows from eps sum(|Re a Im b| + |Im a Re b|) to about
// eps sum(|Re a| + |Im a|)(|Re b| + |Im b|), still eps times the operands' norms.  Outputs are cut
// into 8 x 8 tiles; each warp takes two tiles at a time and walks K in steps of 4.  Fragment layout of m8n8k4 (PTX ISA, "Matrix fragments for mma.m8n8k4 with
// .f64"): A (8 x 4, row) lane t holds A[t / 4][t % 4]; B (4 x 8, col) lane t holds B[t % 4][t / 4];
// C/D (8 x 8) lane t holds C[t / 4][2 (t % 4) + i], i = 0, 1.  Every operand load is masked to
// the nw x nw block (zero outside), so nw need not be a multiple of 8 and no access leaves the
// matrices; stores are masked the same way.  All lanes of a warp execute every mma (the masks act
// on values, never on control flow).
#pragma once
#include "common.cuh"

WNLQG_D void dmma_m8n8k4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Three-product accumulators of one 8 x 8 tile: P[0] += Re a Re b, P[1] += Im a Im b,
// P[2] += (Re a + Im a)(Re b + Im b); a and b one fragment element each.
struct Dmma3 {
    double p[3][2];
    WNLQG_D void zero() {
#pragma unroll
        for (int j = 0; j < 3; ++j) p[j][0] = p[j][1] = 0.0;
    }
    WNLQG_D void mac(double2 a, double2 b) {
        dmma_m8n8k4(p[0][0], p[0][1], a.x, b.x);
        dmma_m8n8k4(p[1][0], p[1][1], a.y, b.y);
        dmma_m8n8k4(p[2][0], p[2][1], a.x + a.y, b.x + b.y);
    }
    WNLQG_D double2 value(int i) const { return make_double2(p[0][i] - p[1][i], p[2][i] - p[0][i] - p[1][i]); }
};

// MODE 0: out = X Y;  MODE 1: out = X^H Y;  MODE 2: out = X Y - Y X.
// X, Y, out: column-major nw x nw, leading dimension ld, in shared memory (or a CTA's global
// working set); out must not alias X or Y.  All threads of the CTA call it; it ends without a
// barrier (callers synchronise before reading out).
template <int MODE>
WNLQG_D void dmma_product(const double2 *X, const double2 *Y, double2 *out, int nw, int ld) {
    const int nt = (nw + 7) >> 3;
    const int ntiles = nt * nt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int fr = lane >> 2, fk = lane & 3;   // A: row fr, column fk; B: row fk, column fr
    const double2 zero = make_double2(0.0, 0.0);
    auto a_elem = [&](const double2 *M, int i, int k) -> double2 {
        if (i >= nw || k >= nw) return zero;
        if (MODE == 1) {
            const double2 v = M[k + ld * i];
            return make_double2(v.x, -v.y);
        }
        return M[i + ld * k];
    };
    auto b_elem = [&](const double2 *M, int k, int j) -> double2 {
        return (k < nw && j < nw) ? M[k + ld * j] : zero;
    };
    for (int t0 = 2 * warp; t0 < ntiles; t0 += 2 * nwarps) {
        const int t1 = t0 + 1 < ntiles ? t0 + 1 : t0;   // a lone last tile is computed twice, stored once
        const int r0 = 8 * (t0 / nt), c0 = 8 * (t0 % nt);
        const int r1 = 8 * (t1 / nt), c1 = 8 * (t1 % nt);
        Dmma3 acc0, acc1;
        acc0.zero();
        acc1.zero();
        for (int k0 = 0; k0 < nw; k0 += 4) {
            const int ka = k0 + fk;
            const double2 a0 = a_elem(X, r0 + fr, ka), b0 = b_elem(Y, ka, c0 + fr);
            const double2 a1 = a_elem(X, r1 + fr, ka), b1 = b_elem(Y, ka, c1 + fr);
            acc0.mac(a0, b0);
            acc1.mac(a1, b1);
            if (MODE == 2) {
                // - Y X: A = -Y, B = X.
                const double2 y0 = a_elem(Y, r0 + fr, ka), x0 = b_elem(X, ka, c0 + fr);
                const double2 y1 = a_elem(Y, r1 + fr, ka), x1 = b_elem(X, ka, c1 + fr);
                acc0.mac(make_double2(-y0.x, -y0.y), x0);
                acc1.mac(make_double2(-y1.x, -y1.y), x1);
            }
        }
        const int orow = fr, ocol = 2 * fk;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            if (r0 + orow < nw && c0 + ocol + i < nw) out[(r0 + orow) + ld * (c0 + ocol + i)] = acc0.value(i);
            if (t1 != t0 && r1 + orow < nw && c1 + ocol + i < nw)
                out[(r1 + orow) + ld * (c1 + ocol + i)] = acc1.value(i);
        }
    }
}

// Two independent products in one pass: out0 = op(X0, Y0) and out1 = op(X1, Y1) (MODE 0: X Y,
// MODE 1: X^H Y, MODE 2: X Y - Y X, where X must have leading dimension ld).  Each warp takes the same tile pair of both products, so it keeps four
// accumulator tiles (twelve independent DMMA chains) in flight instead of two.  X0 and X1 have
// their own leading dimensions (a Wannier-gauge channel can be read straight from global memory,
// ldx = nw); Y and out use ld.  out0 and out1 must not alias any operand.  No closing barrier.
template <int MODE>
WNLQG_D void dmma_product_pair(const double2 *X0, int ldx0, const double2 *Y0, double2 *out0, const double2 *X1,
                               int ldx1, const double2 *Y1, double2 *out1, int nw, int ld) {
    const int nt = (nw + 7) >> 3;
    const int ntiles = nt * nt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int fr = lane >> 2, fk = lane & 3;
    const double2 zero = make_double2(0.0, 0.0);
    auto a_elem = [&](const double2 *M, int ldm, int i, int k) -> double2 {
        if (i >= nw || k >= nw) return zero;
        if (MODE == 1) {
            const double2 v = M[k + ldm * i];
            return make_double2(v.x, -v.y);
        }
        return M[i + ldm * k];
    };
    auto b_elem = [&](const double2 *M, int k, int j) -> double2 {
        return (k < nw && j < nw) ? M[k + ld * j] : zero;
    };
    for (int t0 = 2 * warp; t0 < ntiles; t0 += 2 * nwarps) {
        const int t1 = t0 + 1 < ntiles ? t0 + 1 : t0;
        const int r0 = 8 * (t0 / nt), c0 = 8 * (t0 % nt);
        const int r1 = 8 * (t1 / nt), c1 = 8 * (t1 % nt);
        Dmma3 acc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q].zero();
        for (int k0 = 0; k0 < nw; k0 += 4) {
            const int ka = k0 + fk;
            const double2 a0 = a_elem(X0, ldx0, r0 + fr, ka), b0 = b_elem(Y0, ka, c0 + fr);
            const double2 a1 = a_elem(X0, ldx0, r1 + fr, ka), b1 = b_elem(Y0, ka, c1 + fr);
            const double2 a2 = a_elem(X1, ldx1, r0 + fr, ka), b2 = b_elem(Y1, ka, c0 + fr);
            const double2 a3 = a_elem(X1, ldx1, r1 + fr, ka), b3 = b_elem(Y1, ka, c1 + fr);
            acc[0].mac(a0, b0);
            acc[1].mac(a1, b1);
            acc[2].mac(a2, b2);
            acc[3].mac(a3, b3);
            if (MODE == 2) {
                // - Y X: A = -Y, B = X (X stored with leading dimension ld).
                const double2 y0 = a_elem(Y0, ld, r0 + fr, ka), x0 = b_elem(X0, ka, c0 + fr);
                const double2 y1 = a_elem(Y0, ld, r1 + fr, ka), x1 = b_elem(X0, ka, c1 + fr);
                const double2 y2 = a_elem(Y1, ld, r0 + fr, ka), x2 = b_elem(X1, ka, c0 + fr);
                const double2 y3 = a_elem(Y1, ld, r1 + fr, ka), x3 = b_elem(X1, ka, c1 + fr);
                acc[0].mac(make_double2(-y0.x, -y0.y), x0);
                acc[1].mac(make_double2(-y1.x, -y1.y), x1);
                acc[2].mac(make_double2(-y2.x, -y2.y), x2);
                acc[3].mac(make_double2(-y3.x, -y3.y), x3);
            }
        }
        const int orow = fr, ocol = 2 * fk;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            if (r0 + orow < nw && c0 + ocol + i < nw) {
                out0[(r0 + orow) + ld * (c0 + ocol + i)] = acc[0].value(i);
                out1[(r0 + orow) + ld * (c0 + ocol + i)] = acc[2].value(i);
            }
            if (t1 != t0 && r1 + orow < nw && c1 + ocol + i < nw) {
                out0[(r1 + orow) + ld * (c1 + ocol + i)] = acc[1].value(i);
                out1[(r1 + orow) + ld * (c1 + ocol + i)] = acc[3].value(i);
            }
        }
    }
}
