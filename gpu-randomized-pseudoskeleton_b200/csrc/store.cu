// Compressed store and its far-field matvec on the 5th-generation tensor cores.
//
// After the recompression every far block is C'_b diag(S_b) R'_b. The store regroups the
// factors so that the matvec Y = sum_b P_t(b) C'_b S_b R'_b P_s(b)^T X (16 complex right-hand
// sides) becomes two grouped GEMMs:
//   phase 1, per source group s:  T_s = [S_b R'_b ; b with gs(b) = s] X(ids_s)
//   phase 2, per test group t:    Y(ids_t) = [C'_b ; b with gt(b) = t] [T_b ; b with gt(b) = t]
// (the reference's C(U(R v)) of codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:
// 1929-1960, for all blocks and 16 vectors, on the recompressed form of
// codes/ACA_vs_CUR/seed/svd_compress.m:19-33).
//
// Complex products run as real GEMMs. Phase 1: A' = [Re A | Im A] (K doubled) times
// B' = [[Re X, Im X]; [-Im X, Re X]] gives [Re(AX) | Im(AX)] (N = 2 x 16 = 32). Phase 2: the
// rows are doubled instead, A' = [Re C' ; Im C'] times B' = [Re T | Im T], and each output row
// combines its two rows (Re Y = Re C' Re T - Im C' Im T, Im Y = Re C' Im T + Im C' Re T) in the
// FP32 atomics that write Y: a test group of m rows pads 2m rows to the 128-row tile (154 -> 256
// instead of 154 -> 128 x 2 on a doubled K), and B' is half the size. The phase-1 epilogue
// writes its rows straight into B' (no separate T and no builder kernel).
// Operand formats (pskel_store_build_mode), all accumulated in FP32 in TMEM:
//   BF16X3 (default): every real operand split into bf16 hi + lo (hi = bf16(x), lo = bf16(x -
//            hi)), hi*hi + hi*lo + lo*hi with tcgen05.mma kind::f16 (relative error ~1e-5);
//   TF32:    one TF32 plane (x rounded to 10 mantissa bits), one product with kind::tf32
//            (~5e-4 relative); the same bytes as BF16X3, a third of the MMAs;
//   TF32X3:  TF32 hi + lo planes, three products with kind::tf32 (~1e-6 relative), twice the
//            bytes.
//
// Layout: both operands are stored K-major in the canonical no-swizzle UMMA layout: 16-byte
// chunks of consecutive K values (8 bf16 or 4 TF32) for all rows of a 128-row tile (A) or of the
// 32 columns (B), so that one pipeline stage (8 chunks: 64 bf16 or 32 TF32 K values) of a tile is
// one contiguous range of global memory, fetched with one bulk copy (cp.async.bulk, the TMA
// engine's linear mode) per plane. The hi and lo planes are two arrays of the same shape.
//
// Kernels of one matvec: build_b1_kernel (phase-1 B' from X; also clears Y), then the grouped
// GEMM store_gemm_kernel twice (phase 1, phase 2): persistent, one CTA of 192 threads per SM
// over 128-row work items. Warp 0 allocates two 32-column TMEM accumulators (128 x 32 FP32
// each) and its lane 0 issues the bulk copies of a 4-stage ring; lane 0 of warp 1 issues
// tcgen05.mma (M = 128, N = 32) and commits each stage back to the producer through an
// mbarrier; warps 2-5 read their 32 TMEM lanes (tcgen05.ld 32x32b) and write the rows while the
// next item accumulates into the other accumulator. Every mbarrier wait is bounded: a wait that
// runs out sets the error word, the CTA stops issuing, waits (bounded) for what it issued,
// frees its TMEM and returns.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "engine_internal.cuh"
#include "tcgen05.cuh"

namespace pskel {

constexpr int kStTileM = 128;      // rows per output tile (UMMA M)
constexpr int kStN = 32;           // real columns: 16 right-hand sides x (re, im)
constexpr int kStRhs = 16;
constexpr int kStStages = 4;
constexpr int kStStageABytes = 8 * kStTileM * 16;  // 16 KB per plane: 8 chunks of 128 rows
constexpr int kStStageBBytes = 8 * kStN * 16;      // 4 KB per plane: 8 chunks of 32 columns
constexpr int kStStageBytes = 2 * kStStageABytes + 2 * kStStageBBytes;  // two planes at most
constexpr size_t kStSmem = (size_t)kStStages * kStStageBytes + 1024;
constexpr int kStSliceStages = 8;             // phase-2 K slice per work item (512 K values)

// Element type, elements per 16-byte chunk and planes of each format
template <int MODE> struct StFmt;
template <> struct StFmt<PSKEL_STORE_BF16X3> {
    using E = __nv_bfloat16;
    static constexpr int kEpc = 8, kPlanes = 2;
};
template <> struct StFmt<PSKEL_STORE_TF32> {
    using E = float;
    static constexpr int kEpc = 4, kPlanes = 1;
};
template <> struct StFmt<PSKEL_STORE_TF32X3> {
    using E = float;
    static constexpr int kEpc = 4, kPlanes = 2;
};
inline int st_epc(int mode) { return mode == PSKEL_STORE_BF16X3 ? 8 : 4; }
inline int st_planes(int mode) { return mode == PSKEL_STORE_TF32 ? 1 : 2; }
inline size_t st_esize(int mode) { return mode == PSKEL_STORE_BF16X3 ? 2 : 4; }

// canonical offset (elements) of A(row, k) inside a group whose tiles have kc chunks each
template <int EPC>
__host__ __device__ __forceinline__ long long st_a_off(long long base, int kc, int row, int k) {
    return base + (((long long)(row >> 7) * kc + k / EPC) * kStTileM + (row & 127)) * EPC + k % EPC;
}
// canonical offset of B(col, k) (col < 32)
template <int EPC>
__host__ __device__ __forceinline__ long long st_b_off(long long base, int col, int k) {
    return base + ((long long)(k / EPC) * kStN + col) * EPC + k % EPC;
}

// x as the format's hi (and lo) plane values
__device__ __forceinline__ void st_split(float x, __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    *hi = h;
    *lo = __float2bfloat16_rn(x - __bfloat162float(h));
}
__device__ __forceinline__ void st_split(float x, float *hi, float *lo) {
    const float h = tf32_round(x);
    *hi = h;
    if (lo) *lo = tf32_round(x - h);
}

// ---------------------------------------------------------------- pack (once per recompression)
struct PackBlock {
    const double2 *Cp;  // m x r (ld ldcp), first k columns
    const double2 *Rp;  // r x n (ld r), first k rows
    const double *S;    // k
    int m, n, r, k;     // r: leading dimension of Rp
    int trans, ldcp;    // trans: mirror block, Cp and Rp are its primary's (C' = R'_p^T, R' = C'_p^T)
    long long a1_base;  // phase-1 group base (elements) and the block's first row in it
    int a1_kc, a1_row0;
    long long a2_base;  // phase-2 group base and the block's first K column
    int a2_kc, a2_col0, a2_m;  // a2_m: rows of the test group (imaginary parts start there)
};

template <int MODE>
__global__ void __launch_bounds__(256) pack_kernel(const PackBlock *__restrict__ blocks,
                                                   typename StFmt<MODE>::E *A1h,
                                                   typename StFmt<MODE>::E *A1l,
                                                   typename StFmt<MODE>::E *A2h,
                                                   typename StFmt<MODE>::E *A2l) {
    constexpr int EPC = StFmt<MODE>::kEpc;
    const bool two = StFmt<MODE>::kPlanes == 2;
    const PackBlock w = blocks[blockIdx.x];
    // phase 1: rows S_i R'(i, :) of the source group's stack, [re | im] along K
    for (int e = threadIdx.x; e < w.k * w.n; e += blockDim.x) {
        const int i = e % w.k, j = e / w.k;
        const double2 v = w.trans ? w.Cp[j + (size_t)i * w.ldcp] : w.Rp[i + (size_t)j * w.r];
        const double s = w.S[i];
        const int row = w.a1_row0 + i;
        const long long o_re = st_a_off<EPC>(w.a1_base, w.a1_kc, row, j);
        const long long o_im = st_a_off<EPC>(w.a1_base, w.a1_kc, row, w.n + j);
        st_split((float)(s * v.x), A1h + o_re, two ? A1l + o_re : nullptr);
        st_split((float)(s * v.y), A1h + o_im, two ? A1l + o_im : nullptr);
    }
    // phase 2: columns C'(:, i) in the test group's stack
    for (int e = threadIdx.x; e < w.m * w.k; e += blockDim.x) {
        const int i = e % w.m, j = e / w.m;
        const double2 v = w.trans ? w.Rp[j + (size_t)i * w.r] : w.Cp[i + (size_t)j * w.ldcp];
        const long long o_re = st_a_off<EPC>(w.a2_base, w.a2_kc, i, w.a2_col0 + j);
        const long long o_im = st_a_off<EPC>(w.a2_base, w.a2_kc, w.a2_m + i, w.a2_col0 + j);
        st_split((float)v.x, A2h + o_re, two ? A2l + o_re : nullptr);
        st_split((float)v.y, A2h + o_im, two ? A2l + o_im : nullptr);
    }
}

// ---------------------------------------------------------------- B operands (every matvec)
struct StGroupB {
    long long b_base;  // B buffer offset (elements)
    int kc;            // chunks of the group's K (padded)
    int K;             // real K (phase 1: group size; phase 2: sum of the blocks' ranks)
    const int *src;    // phase 1: RWG ids of the group; phase 2: T row of each real K index
};

// One work item of a B-operand builder: 8 chunks (8 x EPC consecutive K values) of a group.
struct StBItem {
    int g;   // group (index into the phase's StGroupB table)
    int kb;  // 8-chunk block within the group's K
};

// the hi (and lo) plane values of v in a thread's chunk slot e
template <int MODE>
__device__ __forceinline__ void st_split_at(float v, typename StFmt<MODE>::E (&hi)[StFmt<MODE>::kEpc],
                                            typename StFmt<MODE>::E (&lo)[StFmt<MODE>::kEpc], int e) {
    st_split(v, &hi[e], StFmt<MODE>::kPlanes == 2 ? &lo[e] : nullptr);
}

// one 16-byte chunk of each plane at element offset o
template <int MODE>
__device__ __forceinline__ void st_store_chunk(typename StFmt<MODE>::E *Bh, typename StFmt<MODE>::E *Bl,
                                               long long o, const typename StFmt<MODE>::E (&hi)[StFmt<MODE>::kEpc],
                                               const typename StFmt<MODE>::E (&lo)[StFmt<MODE>::kEpc]) {
    *reinterpret_cast<uint4 *>(Bh + o) = *reinterpret_cast<const uint4 *>(hi);
    if (StFmt<MODE>::kPlanes == 2) *reinterpret_cast<uint4 *>(Bl + o) = *reinterpret_cast<const uint4 *>(lo);
}

// phase 1: B'(k, c) from X (complex64, entry (i, rhs) at X[i xr + rhs xc]), columns >= nrhs
// are zero. A CTA stages the X rows of its 8 x EPC K values in shared memory; thread (q, c) then
// writes chunk q of column c: EPC consecutive K values, 16 bytes per plane, each warp one
// contiguous 512-byte row. The grid also clears Y (ne x nrhs entries at Y[i yr + rhs yc], the
// phase-2 atomics' target; the unit stride runs fastest) and the error word.
template <int MODE>
__global__ void __launch_bounds__(256) build_b1_kernel(const StBItem *__restrict__ items,
                                                       const StGroupB *__restrict__ groups,
                                                       const float2 *__restrict__ X, long long xr,
                                                       long long xc, int nrhs, typename StFmt<MODE>::E *Bh,
                                                       typename StFmt<MODE>::E *Bl, float2 *Y, int ne,
                                                       long long yr, long long yc, int *err) {
    using E = typename StFmt<MODE>::E;
    constexpr int EPC = StFmt<MODE>::kEpc, KB = 8 * EPC;
    __shared__ float2 xs[KB][kStRhs + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0;
    const long long ny = (long long)ne * nrhs;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ny; e += (long long)gridDim.x * blockDim.x) {
        const long long i = yr == 1 ? e % ne : e / nrhs, rhs = yr == 1 ? e / ne : e % nrhs;
        Y[i * yr + rhs * yc] = make_float2(0.f, 0.f);
    }
    const StBItem it = items[blockIdx.x];
    const StGroupB g = groups[it.g];
    const int k0 = it.kb * KB;
    for (int e = threadIdx.x; e < KB * kStRhs; e += blockDim.x) {
        // the unit stride of X runs fastest across the threads
        const int kk = xc == 1 ? e / kStRhs : e % KB, rhs = xc == 1 ? e % kStRhs : e / KB, k = k0 + kk;
        float2 x = make_float2(0.f, 0.f);
        if (k < 2 * g.K && rhs < nrhs) x = X[(long long)g.src[k < g.K ? k : k - g.K] * xr + rhs * xc];
        xs[kk][rhs] = x;
    }
    __syncthreads();
    const int q = threadIdx.x >> 5, c = threadIdx.x & 31, rhs = c & (kStRhs - 1);
    alignas(16) E hi[EPC];
    alignas(16) E lo[EPC];
#pragma unroll
    for (int e = 0; e < EPC; ++e) {
        const int kk = q * EPC + e;
        const bool re_half = k0 + kk < g.K;
        const float2 x = xs[kk][rhs];
        // column rhs: [re X; -im X], column 16 + rhs: [im X; re X]
        const float v = c < kStRhs ? (re_half ? x.x : -x.y) : (re_half ? x.y : x.x);
        st_split_at<MODE>(v, hi, lo, e);
    }
    st_store_chunk<MODE>(Bh, Bl, st_b_off<EPC>(g.b_base, c, k0 + q * EPC), hi, lo);
}

// Place of a phase-1 output row (block b's i-th rank row of T_s) in the phase-2 B operand
// [Re T | Im T] of its test group t = gt(b): row k, the row's position in the test group's
// stack of ranks.
struct StT2 {
    long long b_base;  // the test group's B region (elements, phase-2 region included)
    int k, pad;
};

// ---------------------------------------------------------------- tcgen05 grouped GEMM
// One work item of the grouped GEMM: a 128-row output tile and a range of its K stages.
struct StItem {
    long long a_off;  // first A chunk of the item (bf16 elements)
    long long b_off;  // first B chunk of the item
    int nst;          // stages (64 K values each)
    int rows;         // valid rows of the tile
    int out0;         // phase 1: first T row of the tile; phase 2: first row of the 2m stack
    const int *ids;   // phase 2: RWG ids of the test group (null in phase 1)
    int m;            // phase 2: rows of the test group (stack rows m + i: imaginary parts)
};

// instruction descriptors, FP32 D, both operands K-major, M = 128, N = 32:
// kind::f16 with bf16 A and B (format 1), kind::tf32 with TF32 A and B (format 2)
constexpr uint32_t kStIdescBf16 = umma_idesc(1, kStTileM, kStN);
constexpr uint32_t kStIdescTf32 = umma_idesc(2, kStTileM, kStN);

// one MMA of the format: kind::f16 (bf16, K = 16) or kind::tf32 (K = 8); 32 bytes of K per row
template <int MODE>
__device__ __forceinline__ void umma_st(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t accumulate) {
    if constexpr (MODE == PSKEL_STORE_BF16X3) umma_f16(tmem_d, adesc, bdesc, kStIdescBf16, accumulate);
    else umma_tf32(tmem_d, adesc, bdesc, kStIdescTf32, accumulate);
}

// Persistent grouped GEMM, one CTA per SM, warp-specialised:
//   warp 0 lane 0   producer: bulk copies of the A and B planes into a 4-stage ring;
//   warp 1 lane 0   MMA issuer: 3 x 4 tcgen05.mma per stage into one of two TMEM accumulators;
//   warps 2-5       epilogue: tcgen05.ld of their TMEM lane quadrant, then the rows go out
//                   (phase 1: each row T(b, i) straight into the phase-2 B operand, as its
//                   format's planes, at rows k and K + k of its test group; phase 2: FP32
//                   atomics into Y, the items of a tile being K slices of it).
// The two accumulators let the epilogue of one item overlap the MMAs of the next.
template <int MODE>
__global__ void __launch_bounds__(192, 1)
    store_gemm_kernel(const StItem *__restrict__ items, int nitems,
                      const typename StFmt<MODE>::E *__restrict__ Ah,
                      const typename StFmt<MODE>::E *__restrict__ Al,
                      const typename StFmt<MODE>::E *__restrict__ Bh,
                      const typename StFmt<MODE>::E *__restrict__ Bl,
                      const StT2 *__restrict__ t2, typename StFmt<MODE>::E *B2h,
                      typename StFmt<MODE>::E *B2l, float *Y, long long yr, long long yc, int nrhs,
                      int *err) {
    constexpr int EPC = StFmt<MODE>::kEpc;
    constexpr bool kTwo = StFmt<MODE>::kPlanes == 2;
    constexpr int kChunkA = kStTileM * EPC, kChunkB = kStN * EPC;  // elements per chunk block
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kStStages], empty_bar[kStStages];
    __shared__ __align__(8) uint64_t tfull_bar[2], tempty_bar[2], final_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int s_abort;
    unsigned char *ring = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull_bar[a], 1);
            mbar_init(&tempty_bar[a], 4);  // one arrival per epilogue warp
        }
        mbar_init(&final_bar, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        tmem_alloc(&tmem_slot, 2 * kStN);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            long long g = 0;  // stages issued by this CTA
            for (int it = blockIdx.x; it < nitems && !s_abort; it += gridDim.x) {
                const StItem w = items[it];
                for (int s = 0; s < w.nst; ++s, ++g) {
                    const int slot = (int)(g % kStStages);
                    if (g >= kStStages &&
                        !mbar_wait(&empty_bar[slot], (uint32_t)(((g / kStStages) - 1) & 1), &s_abort)) {
                        atomicExch(err, 1);
                        s_abort = 1;
                        break;
                    }
                    unsigned char *st = ring + (size_t)slot * kStStageBytes;
                    mbar_expect_tx(&full_bar[slot], (kTwo ? 2 : 1) * (kStStageABytes + kStStageBBytes));
                    const long long ao = w.a_off + (long long)s * 8 * kChunkA;
                    const long long bo = w.b_off + (long long)s * 8 * kChunkB;
                    bulk_g2s(st, Ah + ao, kStStageABytes, &full_bar[slot]);
                    bulk_g2s(st + 2 * kStStageABytes, Bh + bo, kStStageBBytes, &full_bar[slot]);
                    if (kTwo) {
                        bulk_g2s(st + kStStageABytes, Al + ao, kStStageABytes, &full_bar[slot]);
                        bulk_g2s(st + 2 * kStStageABytes + kStStageBBytes, Bl + bo, kStStageBBytes,
                                 &full_bar[slot]);
                    }
                }
            }
            // no copy may still be in flight when the CTA leaves
            for (long long q = (g > kStStages ? g - kStStages : 0); q < g; ++q)
                mbar_wait(&full_bar[q % kStStages], (uint32_t)((q / kStStages) & 1), &s_abort);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            long long g = 0;
            int n = 0;  // items handled
            for (int it = blockIdx.x; it < nitems && !s_abort; it += gridDim.x, ++n) {
                const StItem w = items[it];
                const int acc = n & 1;
                if (n >= 2 && !mbar_wait(&tempty_bar[acc], (uint32_t)(((n >> 1) - 1) & 1), &s_abort)) {
                    atomicExch(err, 1);
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(acc * kStN);
                for (int s = 0; s < w.nst; ++s, ++g) {
                    const int slot = (int)(g % kStStages);
                    if (!mbar_wait(&full_bar[slot], (uint32_t)((g / kStStages) & 1), &s_abort)) {
                        atomicExch(err, 1);
                        s_abort = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    unsigned char *st = ring + (size_t)slot * kStStageBytes;
                    const uint32_t a_hi = smem_u32(st), a_lo = smem_u32(st + kStStageABytes);
                    const uint32_t b_hi = smem_u32(st + 2 * kStStageABytes);
                    const uint32_t b_lo = smem_u32(st + 2 * kStStageABytes + kStStageBBytes);
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks) {  // one MMA reads two chunks (32 bytes) of K
                        // byte offsets: two chunk blocks of 128 rows (A) / 32 columns (B)
                        const uint32_t ao = ks * 2 * kStTileM * 16, bo = ks * 2 * kStN * 16;
                        const uint64_t dah = umma_desc(a_hi + ao, kStTileM * 16, 128);
                        const uint64_t dbh = umma_desc(b_hi + bo, kStN * 16, 128);
                        umma_st<MODE>(d, dah, dbh, (s > 0 || ks > 0) ? 1u : 0u);
                        if (kTwo) {
                            const uint64_t dal = umma_desc(a_lo + ao, kStTileM * 16, 128);
                            const uint64_t dbl = umma_desc(b_lo + bo, kStN * 16, 128);
                            umma_st<MODE>(d, dah, dbl, 1u);
                            umma_st<MODE>(d, dal, dbh, 1u);
                        }
                    }
                    umma_commit(&empty_bar[slot]);  // the slot is free once these MMAs have read it
                }
                if (s_abort) break;
                umma_commit(&tfull_bar[acc]);  // the accumulator is complete
            }
            // every MMA issued has finished before TMEM may be released
            umma_commit(&final_bar);
            if (!mbar_wait(&final_bar, 0, &s_abort)) atomicExch(err, 1);
        }
    } else {
        const int quad = warp & 3;  // TMEM lanes 32 quad .. 32 quad + 31
        int n = 0;
        for (int it = blockIdx.x; it < nitems; it += gridDim.x, ++n) {
            const StItem w = items[it];
            const int acc = n & 1;
            int okw = mbar_wait(&tfull_bar[acc], (uint32_t)((n >> 1) & 1), &s_abort) ? 1 : 0;
            okw = __all_sync(0xffffffffu, okw);
            if (!okw) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    s_abort = 1;
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t v[32];
            const uint32_t taddr = tmem + (uint32_t)(acc * kStN) + ((uint32_t)(quad * 32) << 16);
            tmem_ld32(taddr, v);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[acc]);  // the accumulator may be reused
            const int row = quad * 32 + lane;
            if (row < w.rows) {
                if (!w.ids) {
                    // T(b, i) = [re of the 16 sides | im] is row k of its test group's B'
                    const StT2 d = t2[w.out0 + row];
#pragma unroll
                    for (int c = 0; c < kStN; ++c) {
                        typename StFmt<MODE>::E h, l;
                        const long long o = st_b_off<EPC>(d.b_base, c, d.k);
                        st_split(__uint_as_float(v[c]), &h, kTwo ? &l : nullptr);
                        B2h[o] = h;
                        if (kTwo) B2l[o] = l;
                    }
                } else {
                    // stack row rho: Re C'(i, :) [Re T | Im T] (rho = i) or Im C'(i, :) [Re T | Im T]
                    // (rho = m + i)
                    const int rho = w.out0 + row;
                    const bool im = rho >= w.m;
                    const int id = w.ids[im ? rho - w.m : rho];
#pragma unroll
                    for (int c = 0; c < kStRhs; ++c)
                        if (c < nrhs) {
                            float *y = Y + 2 * ((long long)id * yr + (long long)c * yc);
                            const float a = __uint_as_float(v[c]), b = __uint_as_float(v[c + kStRhs]);
                            atomicAdd(y, im ? -b : a);
                            atomicAdd(y + 1, im ? a : b);
                        }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, 2 * kStN);
}

}  // namespace pskel

using namespace pskel;

// ---------------------------------------------------------------- host side
namespace {
template <int MODE>
void launch_pack(pskel_ctx *c, long long a1) {
    using E = typename StFmt<MODE>::E;
    E *ah = c->st_ah.as<E>(), *al = StFmt<MODE>::kPlanes == 2 ? c->st_al.as<E>() : nullptr;
    pack_kernel<MODE><<<c->n_blocks, 256, 0, c->stream>>>(c->st_tab.as<PackBlock>(), ah, al, ah + a1,
                                                          al ? al + a1 : nullptr);
}
}  // namespace

extern "C" int pskel_store_build_mode(pskel_ctx *c, int mode, long long *bytes) {
    if (!c || c->n_blocks <= 0 || (int)c->recomp_slots.size() != c->n_blocks) {
        set_error(PSKEL_ERR_STATE, "store_build: run pskel_recompress first");
        return PSKEL_ERR_STATE;
    }
    if (mode != PSKEL_STORE_BF16X3 && mode != PSKEL_STORE_TF32 && mode != PSKEL_STORE_TF32X3) {
        set_error(PSKEL_ERR_ARG, "store_build: unknown operand format %d", mode);
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const int nb = c->n_blocks, ng = c->n_groups;
    StoreLayout &L = c->store;
    L = StoreLayout();
    L.mode = mode;
    const int epc = st_epc(mode), planes = st_planes(mode);
    const size_t esize = st_esize(mode);
    const long long chunkA = (long long)kStTileM * epc, chunkB = (long long)kStN * epc;
    const long long stageK = 8LL * epc;  // K values per pipeline stage
    std::vector<std::vector<int>> by_src(ng), by_test(ng);
    for (int b = 0; b < nb; ++b) {
        by_src[c->gs[b]].push_back(b);
        by_test[c->gt[b]].push_back(b);
    }
    auto gsize = [&](int g) { return c->gptr[g + 1] - c->gptr[g]; };
    auto pad = [](long long x, long long a) { return (x + a - 1) / a * a; };
    std::vector<PackBlock> pb(nb);
    // phase 1: per source group
    long long a1 = 0, b1 = 0;
    int trow = 0;
    std::vector<int> t_row0(nb);  // first T row of each block
    for (int g = 0; g < ng; ++g) {
        if (by_src[g].empty()) continue;
        int K = 0;
        for (int b : by_src[g]) K += c->recomp_slots[b].k;
        if (K == 0) continue;
        const int n = gsize(g);
        const int kc = (int)(pad(2 * (long long)n, stageK) / epc);
        const int mpad = (int)pad(K, kStTileM);
        int row = 0;
        for (int b : by_src[g]) {
            PackBlock &w = pb[b];
            w.a1_base = a1;
            w.a1_kc = kc;
            w.a1_row0 = row;
            t_row0[b] = trow + row;
            row += c->recomp_slots[b].k;
        }
        for (int mt = 0; mt < mpad / kStTileM; ++mt)
            L.tiles1.push_back(StoreTile{a1 + (long long)mt * kc * chunkA, b1, kc,
                                         std::min(kStTileM, K - mt * kStTileM), trow + mt * kStTileM, -1});
        L.groups1.push_back(StoreGroup{b1, kc, n, c->gptr[g]});
        a1 += (long long)mpad * kc * epc;
        b1 += (long long)kc * chunkB;
        trow += mpad;
    }
    // phase 2: per test group; the place of every phase-1 output row in its B operand
    std::vector<StT2> tplace(std::max(trow, 1), StT2{0, 0, 0});
    long long a2 = 0, b2 = 0;
    for (int g = 0; g < ng; ++g) {
        if (by_test[g].empty()) continue;
        int K = 0;
        for (int b : by_test[g]) K += c->recomp_slots[b].k;
        if (K == 0) continue;
        const int m = gsize(g);
        const int kc = (int)(pad((long long)K, stageK) / epc);
        const int mpad = (int)pad(2 * (long long)m, kStTileM);  // Re C' rows, then Im C' rows
        int col = 0;
        for (int b : by_test[g]) {
            PackBlock &w = pb[b];
            w.a2_base = a2;
            w.a2_kc = kc;
            w.a2_col0 = col;
            w.a2_m = m;
            for (int i = 0; i < c->recomp_slots[b].k; ++i) tplace[t_row0[b] + i] = StT2{b1 + b2, col + i, 0};
            col += c->recomp_slots[b].k;
        }
        for (int mt = 0; mt < mpad / kStTileM; ++mt)
            L.tiles2.push_back(StoreTile{a2 + (long long)mt * kc * chunkA, b2, kc,
                                         std::min(kStTileM, 2 * m - mt * kStTileM), mt * kStTileM, 1,
                                         c->gptr[g], m});
        a2 += (long long)mpad * kc * epc;
        b2 += (long long)kc * chunkB;
    }
    for (int b = 0; b < nb; ++b) {
        const RecompSlot &sl = c->recomp_slots[b];
        const BlockResult &res = c->results[b];
        PackBlock &w = pb[b];
        w.Cp = sl.Cp;
        w.Rp = sl.Rp;
        w.S = sl.S;
        w.m = res.m;
        w.n = res.n;
        w.r = sl.ldrp;  // leading dimension of the (primary's) R
        w.k = sl.k;
        w.trans = sl.mirror >= 0 ? 1 : 0;
        w.ldcp = sl.mirror >= 0 ? c->results[sl.mirror].m : res.m;
    }
    L.a1 = a1;
    L.a2 = a2;
    L.b1 = b1;
    L.b2 = b2;
    L.trows = trow;
    // device buffers: A planes (phase 1 then phase 2), B planes, T, tables
    const size_t abytes = (size_t)(a1 + a2) * esize;
    PSKEL_TRY(c->st_ah.reserve(abytes));
    PSKEL_TRY(c->st_bh.reserve((size_t)(b1 + b2) * esize + 256));
    if (planes == 2) {
        PSKEL_TRY(c->st_al.reserve(abytes));
        PSKEL_TRY(c->st_bl.reserve((size_t)(b1 + b2) * esize + 256));
    }
    PSKEL_TRY(c->st_t.reserve(sizeof(StT2) * tplace.size()));
    PSKEL_CUDA(cudaMemcpyAsync(c->st_t.ptr, tplace.data(), sizeof(StT2) * tplace.size(), cudaMemcpyHostToDevice,
                               c->stream));
    PSKEL_CUDA(cudaMemsetAsync(c->st_ah.ptr, 0, abytes, c->stream));
    if (planes == 2) PSKEL_CUDA(cudaMemsetAsync(c->st_al.ptr, 0, abytes, c->stream));
    // the B planes' K padding stays zero: every matvec rewrites the phase-1 region whole and
    // the phase-2 rows k < 2K of each test group
    PSKEL_CUDA(cudaMemsetAsync(c->st_bh.ptr, 0, (size_t)(b1 + b2) * esize, c->stream));
    if (planes == 2) PSKEL_CUDA(cudaMemsetAsync(c->st_bl.ptr, 0, (size_t)(b1 + b2) * esize, c->stream));
    PSKEL_TRY(c->st_tab.reserve(sizeof(PackBlock) * nb + 256));
    PSKEL_CUDA(cudaMemcpyAsync(c->st_tab.ptr, pb.data(), sizeof(PackBlock) * nb, cudaMemcpyHostToDevice,
                               c->stream));
    if (mode == PSKEL_STORE_BF16X3) launch_pack<PSKEL_STORE_BF16X3>(c, a1);
    else if (mode == PSKEL_STORE_TF32) launch_pack<PSKEL_STORE_TF32>(c, a1);
    else launch_pack<PSKEL_STORE_TF32X3>(c, a1);
    PSKEL_LAUNCHED(1);
    // device tile and group tables (pointers resolved here)
    const int *gids = c->d_gids.as<int>();
    // work items: phase-1 tiles whole (their K is one source group); phase-2 tiles cut into K
    // slices of at most kStSliceStages stages, accumulated with atomics
    std::vector<StItem> t1, t2;
    for (const StoreTile &t : L.tiles1)
        t1.push_back(StItem{t.a_off, t.b_off, t.kc / 8, t.rows, t.out0, nullptr, 0});
    for (const StoreTile &t : L.tiles2)
        for (int s0 = 0; s0 < t.kc / 8; s0 += kStSliceStages)
            t2.push_back(StItem{a1 + t.a_off + (long long)s0 * 8 * chunkA,
                                b1 + t.b_off + (long long)s0 * 8 * chunkB,
                                std::min(kStSliceStages, t.kc / 8 - s0), t.rows, t.out0, gids + t.ids0, t.m});
    L.n_items1 = (int)t1.size();
    L.n_items2 = (int)t2.size();
    std::vector<StGroupB> g1;
    for (const StoreGroup &g : L.groups1) g1.push_back(StGroupB{g.b_base, g.kc, g.K, gids + g.ids0});
    // phase-1 B-builder items: every 8-chunk block of every source group (kc is a multiple of 8)
    std::vector<StBItem> bi1;
    for (size_t g = 0; g < g1.size(); ++g)
        for (int kb = 0; kb < g1[g].kc / 8; ++kb) bi1.push_back(StBItem{(int)g, kb});
    L.n_bitems1 = (int)bi1.size();
    const size_t s1 = sizeof(StItem) * t1.size(), s2 = sizeof(StItem) * t2.size();
    const size_t s3 = sizeof(StGroupB) * g1.size(), s5 = sizeof(StBItem) * bi1.size();
    auto al256 = [](size_t x) { return (x + 255) & ~size_t(255); };
    PSKEL_TRY(c->st_tiles.reserve(al256(s1) + al256(s2) + al256(s3) + al256(s5) + 256));
    char *d = c->st_tiles.as<char>();
    L.d_t1 = d;
    L.d_t2 = d + al256(s1);
    L.d_g1 = d + al256(s1) + al256(s2);
    L.d_bi1 = d + al256(s1) + al256(s2) + al256(s3);
    if (s1) PSKEL_CUDA(cudaMemcpyAsync(L.d_t1, t1.data(), s1, cudaMemcpyHostToDevice, c->stream));
    if (s2) PSKEL_CUDA(cudaMemcpyAsync(L.d_t2, t2.data(), s2, cudaMemcpyHostToDevice, c->stream));
    if (s3) PSKEL_CUDA(cudaMemcpyAsync(L.d_g1, g1.data(), s3, cudaMemcpyHostToDevice, c->stream));
    if (s5) PSKEL_CUDA(cudaMemcpyAsync(L.d_bi1, bi1.data(), s5, cudaMemcpyHostToDevice, c->stream));
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    L.ready = true;
    L.generation = c->generation;
    if (bytes) *bytes = (long long)(planes * abytes);
    return PSKEL_OK;
}

extern "C" int pskel_store_build(pskel_ctx *c, long long *bytes) {
    return pskel_store_build_mode(c, PSKEL_STORE_BF16X3, bytes);
}

namespace {
// The three launches of one matvec over a store of format MODE: the phase-1 B operand (with the
// clear of Y and of the error word), the phase-1 GEMM (writing the phase-2 B operand), the
// phase-2 GEMM (atomics into Y).
template <int MODE>
int store_matvec_t(pskel_ctx *c, const void *X, long long xr, long long xc, void *Y, long long yr,
                   long long yc, int nrhs, cudaStream_t st) {
    using E = typename StFmt<MODE>::E;
    const bool two = StFmt<MODE>::kPlanes == 2;
    const StoreLayout &L = c->store;
    PSKEL_TRY(ensure_smem_attr(store_gemm_kernel<MODE>, kStSmem));
    E *ah = c->st_ah.as<E>(), *al = two ? c->st_al.as<E>() : nullptr;
    E *bh = c->st_bh.as<E>(), *bl = two ? c->st_bl.as<E>() : nullptr;
    int *err = c->st_err.as<int>();
    const int n1 = L.n_items1, n2 = L.n_items2;
    const int nb1 = L.n_bitems1;
    const int sms = sm_count();
    if (nb1 > 0) {
        build_b1_kernel<MODE><<<nb1, 256, 0, st>>>(reinterpret_cast<const StBItem *>(L.d_bi1),
                                                   reinterpret_cast<const StGroupB *>(L.d_g1),
                                                   reinterpret_cast<const float2 *>(X), xr, xc, nrhs, bh, bl,
                                                   reinterpret_cast<float2 *>(Y), c->mesh.ne, yr, yc, err);
        PSKEL_LAUNCHED(1);
    }
    if (n1 > 0) {
        store_gemm_kernel<MODE><<<std::min(n1, sms), 192, kStSmem, st>>>(
            reinterpret_cast<const StItem *>(L.d_t1), n1, ah, al, bh, bl, c->st_t.as<StT2>(), bh, bl,
            nullptr, 0, 0, kStRhs, err);
        PSKEL_LAUNCHED(1);
    }
    if (n2 > 0) {
        store_gemm_kernel<MODE><<<std::min(n2, sms), 192, kStSmem, st>>>(
            reinterpret_cast<const StItem *>(L.d_t2), n2, ah, al, bh, bl, nullptr, nullptr, nullptr,
            reinterpret_cast<float *>(Y), yr, yc, nrhs, err);
        PSKEL_LAUNCHED(1);
    }
    return PSKEL_OK;
}
}  // namespace

extern "C" int pskel_store_matvec_strided(pskel_ctx *c, const void *X, long long x_row_stride,
                                          long long x_col_stride, void *Y, long long y_row_stride,
                                          long long y_col_stride, int nrhs, void *stream) {
    if (!c || !X || !Y || nrhs <= 0 || nrhs > kStRhs || x_row_stride <= 0 || x_col_stride <= 0 ||
        !((y_row_stride == 1 && y_col_stride >= c->mesh.ne) || (y_col_stride == 1 && y_row_stride >= nrhs))) {
        set_error(PSKEL_ERR_ARG, "store_matvec: bad arguments (nrhs=%d, at most %d; positive X strides; Y "
                                 "column-major or row-major without overlap)", nrhs, kStRhs);
        return PSKEL_ERR_ARG;
    }
    const StoreLayout &L = c->store;
    if (!L.ready || L.generation != c->generation) {
        set_error(PSKEL_ERR_STATE, "store_matvec: build the store after the last compression");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PSKEL_TRY(c->st_err.reserve(256));
    if (L.n_bitems1 == 0) {  // no phase-1 work: Y and the error word are cleared here
        PSKEL_CUDA(cudaMemsetAsync(c->st_err.ptr, 0, sizeof(int), st));
        if (y_row_stride == 1)
            PSKEL_CUDA(cudaMemsetAsync(Y, 0, sizeof(float2) * (size_t)y_col_stride * nrhs, st));
        else
            PSKEL_CUDA(cudaMemsetAsync(Y, 0, sizeof(float2) * (size_t)y_row_stride * c->mesh.ne, st));
    }
    const long long xr = x_row_stride, xc = x_col_stride, yr = y_row_stride, yc = y_col_stride;
    if (L.mode == PSKEL_STORE_BF16X3) return store_matvec_t<PSKEL_STORE_BF16X3>(c, X, xr, xc, Y, yr, yc, nrhs, st);
    if (L.mode == PSKEL_STORE_TF32) return store_matvec_t<PSKEL_STORE_TF32>(c, X, xr, xc, Y, yr, yc, nrhs, st);
    return store_matvec_t<PSKEL_STORE_TF32X3>(c, X, xr, xc, Y, yr, yc, nrhs, st);
}

extern "C" int pskel_store_matvec(pskel_ctx *c, const void *X, int ldx, void *Y, int ldy, int nrhs,
                                  void *stream) {
    if (!c || ldx < c->mesh.ne || ldy < c->mesh.ne) {
        set_error(PSKEL_ERR_ARG, "store_matvec: bad arguments (ldx=%d, ldy=%d)", ldx, ldy);
        return PSKEL_ERR_ARG;
    }
    return pskel_store_matvec_strided(c, X, 1, ldx, Y, 1, ldy, nrhs, stream);
}

extern "C" int pskel_store_status(pskel_ctx *c, int *error_word) {
    if (!c || !error_word) {
        set_error(PSKEL_ERR_ARG, "store_status: null argument");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    *error_word = 0;
    if (c->st_err.ptr) PSKEL_CUDA(cudaMemcpy(error_word, c->st_err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    return PSKEL_OK;
}
