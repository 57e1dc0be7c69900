// tc_fourier.cuh - Fourier interpolation on the tcgen05 tensor cores (arbitrary k-points).
//
// X[k, n] = sum_R F[k, R] T[R, n] (HamiltonianMatrixElements.jl:28-58, 426-462;
// PositionMatrixElements.jl:294-332) as a real GEMM D[M x N'] = A[M x K'] B[N' x K']^T with
//   A[k, 2R] = Re F, A[k, 2R+1] = Im F,
//   B[2n, 2R] = Re T, B[2n, 2R+1] = -Im T, B[2n+1, 2R] = Im T, B[2n+1, 2R+1] = Re T,
// so that D[k, 2n] + i D[k, 2n+1] = X[k, n] lands as one complex double per output.
//
// Precision: fixed-point slicing (an Ozaki-type split).  Every operand value y with |y| <= 1
// (A: |F| <= 1/deg <= 1; B: each row scaled by a power of two 2^e_n) is written as
//   y = sum_{i<S} a_i 2^(-6-7i) + r,   a_i integer in [-64, 64],   |r| <= 2^(-7S),
// by S round-to-nearest steps that are exact in FP64.  The product of two sliced values is
// sum_{i,j} a_i b_j 2^(-12-7(i+j)); the pairs with level L = i + j < S are kept (the dropped ones
// are below 2^(-7S) relative).  Each level is accumulated EXACTLY by tcgen05.mma kind::i8 in an
// int32 TMEM accumulator (|a_i b_j| <= 4096, so K' * S * 4096 < 2^31 for K' < 74000), and the
// epilogue forms D = 2^(e_n - 12) sum_L 2^(-7L) acc_L in FP64.  S = 7 leaves 2^-49 of the row
// scale (the FP64 path); the mixed path uses fewer slices.
//
// Kernel structure (one CTA per SM, persistent over 128 x NT output tiles):
//   warp 4        TMA producer: per K block of 64 int8, one 3D box of all S slices of A
//                 (128 x 64 each) and one of B (NT x 64 each), 64-byte swizzle, into a ring of
//                 ST stages guarded by full/empty mbarriers;
//   warp 5        MMA issuer: per K block and 32-byte K step, the S(S+1)/2 slice pairs into the
//                 S level accumulators (TMEM columns L*NT .. L*NT+NT-1), tcgen05.commit frees
//                 the stage; after the last block it signals the epilogue;
//   warps 0-3     epilogue: tcgen05.ld of their 32 TMEM lanes (rows), FP64 combination of the
//                 levels, row/column scaling and the complex-double store into the channel
//                 buffer; then they release the accumulators for the next tile.
// Every mbarrier wait is bounded; a wait that gives up sets *err and the CTA winds down (TMEM is
// freed on every exit path).
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace tcf {

constexpr int BM = 128;        // output rows (k-points) per tile = TMEM lanes
constexpr int BK = 64;         // int8 K elements per pipeline stage (one 64-byte swizzled row)
constexpr int GROUP_M = 16;    // m-tiles per L2 group in the tile order
constexpr long long WAIT_CYCLES = 4000000000LL;
constexpr int THREADS = 192;

template <int S> struct Cfg;
template <> struct Cfg<7> { static constexpr int NT = 64;  static constexpr int ST = 2; };
template <> struct Cfg<5> { static constexpr int NT = 64;  static constexpr int ST = 3; };
template <> struct Cfg<4> { static constexpr int NT = 128; static constexpr int ST = 3; };

template <int S> struct Layout {
    static constexpr int NT = Cfg<S>::NT, ST = Cfg<S>::ST;
    static constexpr uint32_t A_BYTES = (uint32_t)S * BM * BK;
    static constexpr uint32_t B_BYTES = (uint32_t)S * NT * BK;
    static constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr uint32_t BAR_OFF = ST * STAGE_BYTES;           // after the stages
    static constexpr uint32_t SMEM_BYTES = BAR_OFF + 128 + 1024;     // barriers + alignment slack
    static constexpr uint32_t TMEM_COLS = 512;
    static_assert(S * NT <= 512, "level accumulators exceed TMEM");
    static_assert(STAGE_BYTES % 1024 == 0, "stages must keep 1024-byte alignment");
};

// ---- PTX wrappers ------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of parity `parity`: false when about WAIT_CYCLES SM cycles (~2 s)
// passed or another role of the CTA aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag) {
    const long long start = clock64();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag || clock64() - start > WAIT_CYCLES) return false;
    }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot_addr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_addr), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major operand, rows of 64 bytes with the 64-byte swizzle,
// 8-row groups 512 bytes apart (stride byte offset), descriptor version 1, layout SWIZZLE_64B (4).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused by swizzled K-major layouts)
    d |= (uint64_t)(512 >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1 << 46;             // version
    d |= (uint64_t)4 << 61;             // SWIZZLE_64B
    return d;
}

// Instruction descriptor of kind::i8: D s32, A and B signed int8, both K-major, M = 128, N = NT.
template <int NT> __host__ __device__ constexpr uint32_t idesc_i8() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

// ---- slicing -----------------------------------------------------------------------------------
template <int S> __host__ __device__ inline void slice_value(double y, int8_t *out) {
    double unit = 0.015625;   // 2^-6
    for (int i = 0; i < S; ++i) {
        const double a = rint(y / unit);
        out[i] = (int8_t)a;
        y -= a * unit;
        unit *= 0.0078125;    // 2^-7
    }
}

// Phase slices Aq[i][b][2R + {0,1}] (re, im) for a batch; padded R columns (R >= nr) are zero.
// Phase arithmetic as phase_kernel (exact integer reduction on meshes, sincospi).
template <int S>
__global__ void phase_slices_kernel(int8_t *__restrict__ Aq, int64_t Mpad, int64_t Kpad, const int64_t *__restrict__ rvec,
                                    const int64_t *__restrict__ deg, int nr, int64_t batch, int64_t k_begin, int64_t n1,
                                    int64_t n2, int64_t n3, const double *__restrict__ kpts,
                                    const int64_t *__restrict__ kidx) {
    const int64_t half = Kpad / 2;
    const int64_t total = batch * half;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = e / half;
        const int r = (int)(e - b * half);
        double re = 0.0, im = 0.0;
        if (r < nr) {
            const int64_t r1 = rvec[3 * r], r2 = rvec[3 * r + 1], r3 = rvec[3 * r + 2];
            double x;
            if (kpts == nullptr) {
                const int64_t idx = kidx ? kidx[b] : k_begin + b;
                const int64_t i1 = idx % n1, i2 = (idx / n1) % n2, i3 = idx / (n1 * n2);
                const int64_t p1 = ((r1 * i1) % n1 + n1) % n1, p2 = ((r2 * i2) % n2 + n2) % n2,
                              p3 = ((r3 * i3) % n3 + n3) % n3;
                x = (double)p1 / (double)n1 + (double)p2 / (double)n2 + (double)p3 / (double)n3;
            } else {
                const double *k = kpts + 3 * b;
                x = (double)r1 * k[0] + (double)r2 * k[1] + (double)r3 * k[2];
            }
            x -= rint(x);
            double s, c;
            sincospi(2.0 * x, &s, &c);
            const double inv = 1.0 / (double)deg[r];
            re = c * inv;
            im = s * inv;
        }
        int8_t sr[S], si[S];
        slice_value<S>(re, sr);
        slice_value<S>(im, si);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            char2 v;
            v.x = sr[i];
            v.y = si[i];
            *reinterpret_cast<char2 *>(Aq + ((int64_t)i * Mpad + b) * Kpad + 2 * r) = v;
        }
    }
}

// ---- the GEMM ----------------------------------------------------------------------------------
struct TcArgs {
    const double *colscale;   // [Npad]: 2^(e_n - 12)
    double2 *xw;              // [nb][ncols / 2]
    int64_t nb;
    int64_t ncols;            // real output columns N' (= 2 * C * nw^2)
    int kblocks;
    int mtiles, ntiles;
    int *err;                 // set to 1 when a bounded wait gave up
};

__device__ __forceinline__ void tile_coords(int t, int mtiles, int ntiles, int &m, int &n) {
    const int per_group = GROUP_M * ntiles;
    const int g = t / per_group;
    const int within = t - g * per_group;
    const int gs = min(GROUP_M, mtiles - g * GROUP_M);
    n = within / gs;
    m = g * GROUP_M + within % gs;
}

template <int S>
__global__ void __launch_bounds__(THREADS, 1)
    tc_fourier_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcArgs args) {
    typedef Layout<S> L;
    constexpr int NT = L::NT, ST = L::ST;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char *gbase = smem_raw + (base - raw);
    const uint32_t bar_full = base + L::BAR_OFF;           // ST x 8 bytes
    const uint32_t bar_empty = bar_full + 8 * ST;         // ST x 8 bytes
    const uint32_t bar_done = bar_empty + 8 * ST;
    const uint32_t bar_tmem_empty = bar_done + 8;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gbase + L::BAR_OFF + 16 * ST + 16);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(gbase + L::BAR_OFF + 16 * ST + 20);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        mbar_init(bar_done, 1);
        mbar_init(bar_tmem_empty, 4 * 32);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(smem_u32(tmem_slot), L::TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int total_tiles = args.mtiles * args.ntiles;

    if (warp == 4) {
        if (lane == 0) {
            uint32_t it = 0;
            for (int t = blockIdx.x; t < total_tiles && !*abort_flag; t += gridDim.x) {
                int m, n;
                tile_coords(t, args.mtiles, args.ntiles, m, n);
                for (int kb = 0; kb < args.kblocks; ++kb, ++it) {
                    const uint32_t s = it % ST, round = it / ST;
                    if (!mbar_wait(bar_empty + 8 * s, (round & 1u) ^ 1u, abort_flag)) {
                        *abort_flag = 1;
                        atomicExch(args.err, 1);
                        break;
                    }
                    const uint32_t sa = base + s * L::STAGE_BYTES;
                    mbar_expect_tx(bar_full + 8 * s, L::STAGE_BYTES);
                    tma_load_3d(sa, &mapA, bar_full + 8 * s, kb * BK, m * BM, 0);
                    tma_load_3d(sa + L::A_BYTES, &mapB, bar_full + 8 * s, kb * BK, n * NT, 0);
                }
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_i8<NT>();
            uint32_t it = 0, tl = 0;
            for (int t = blockIdx.x; t < total_tiles && !*abort_flag; t += gridDim.x, ++tl) {
                if (!mbar_wait(bar_tmem_empty, (tl & 1u) ^ 1u, abort_flag)) {
                    *abort_flag = 1;
                    atomicExch(args.err, 1);
                    break;
                }
                tc_fence_after();
                uint32_t wrote = 0;
                bool ok = true;
                for (int kb = 0; kb < args.kblocks; ++kb, ++it) {
                    const uint32_t s = it % ST, round = it / ST;
                    if (!mbar_wait(bar_full + 8 * s, round & 1u, abort_flag)) {
                        *abort_flag = 1;
                        atomicExch(args.err, 1);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = base + s * L::STAGE_BYTES, sb = sa + L::A_BYTES;
#pragma unroll
                    for (int ks = 0; ks < BK / 32; ++ks) {
#pragma unroll
                        for (int i = 0; i < S; ++i) {
#pragma unroll
                            for (int j = 0; j < S - i; ++j) {
                                const int lv = i + j;
                                const uint64_t ad = smem_desc(sa + (uint32_t)i * BM * BK + 32u * ks);
                                const uint64_t bd = smem_desc(sb + (uint32_t)j * NT * BK + 32u * ks);
                                mma_i8(tmem + (uint32_t)(lv * NT), ad, bd, idesc, (wrote >> lv) & 1u);
                                wrote |= 1u << lv;
                            }
                        }
                    }
                    mma_commit(bar_empty + 8 * s);
                }
                if (!ok) break;
                mma_commit(bar_done);
            }
        }
    } else {
        // Epilogue: warps 0-3 own TMEM lanes 32*warp .. 32*warp + 31 (tile rows).
        uint32_t tl = 0;
        const int64_t half = args.ncols / 2;
        for (int t = blockIdx.x; t < total_tiles; t += gridDim.x, ++tl) {
            int m, n;
            tile_coords(t, args.mtiles, args.ntiles, m, n);
            const bool ok = __all_sync(0xffffffffu, mbar_wait(bar_done, tl & 1u, abort_flag) ? 1 : 0) != 0;
            if (!ok) {
                if (lane == 0) { *abort_flag = 1; atomicExch(args.err, 1); }
                break;
            }
            tc_fence_after();
            const int64_t row = (int64_t)m * BM + warp * 32 + lane;
            const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
            for (int c0 = 0; c0 < NT; c0 += 16) {
                double v[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) v[q] = 0.0;
                double w = 1.0;
#pragma unroll
                for (int lv = 0; lv < S; ++lv) {
                    uint32_t r[16];
                    tmem_ld16(lane_addr + (uint32_t)(lv * NT + c0), r);
#pragma unroll
                    for (int q = 0; q < 16; ++q) v[q] = fma((double)(int)r[q], w, v[q]);
                    w *= 0.0078125;
                }
                const int64_t col0 = (int64_t)n * NT + c0;
                if (row < args.nb) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int64_t c = col0 + 2 * q;
                        if (c < args.ncols)
                            args.xw[row * half + c / 2] =
                                make_double2(v[2 * q] * args.colscale[c], v[2 * q + 1] * args.colscale[c + 1]);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(bar_tmem_empty);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, L::TMEM_COLS);
    }
}

}  // namespace tcf
