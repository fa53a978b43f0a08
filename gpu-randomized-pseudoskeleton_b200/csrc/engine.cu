// Handle API: resident mesh and groups, batched compression of many far-field blocks.
//
// One compression call processes every block of the block list in rounds. A round runs, for
// all still-active blocks at once:
//   sample   - seeded Philox/Floyd index sets I, J and extra estimator rows Ix (one CTA/block);
//   fill     - C = Z(group_t, J) and Rx = Z([I; Ix], group_s) in one batched fill launch;
//   pinv     - core = C(I, :) gathered and promoted to FP64, batched one-sided Jacobi SVD,
//              U = V diag(1/s) W^H over the kept singular values;
//   estimate - est = ||Z(Ix,:) - C(Ix,:) U R||_F / ||Z(Ix,:)||_F (one CTA/block).
// Blocks whose estimate is within tolerance (or that reached r = min(m, n), or the round cap)
// are done; the others double r and go to the next round with fresh samples - the reference's
// adaptive growth rule (compres_single_block_spheres_for_sweep2.jl:878-973), judged by the
// extra-row estimate instead of the successive-estimate difference. The first round's kernel
// sequence can be captured once into a CUDA graph and replayed on identical calls.
//
// The core Z(I, J) is taken from the filled C instead of a third fill: the values are the same
// entries, and in complex FP32 mode the pinv then inverts exactly the numbers that C and R hold.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>

#include "pskel_internal.cuh"
#include "zgemm.cuh"
#include "engine_internal.cuh"

namespace pskel {


// ------------------------------------------------------------------ sampler
__device__ __forceinline__ uint32_t philox_word(uint32_t i, uint32_t block, uint32_t round,
                                                uint32_t stream, uint64_t seed) {
    uint32_t c0 = i, c1 = block, c2 = round, c3 = stream;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int rr = 0; rr < 10; ++rr) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c0;
}

// r distinct values of [0, D) (Floyd), left as a bitmap in bits[]; then the sorted values are
// written to out (if not null). Must be called by all threads of the CTA.
__device__ void draw_bitmap(uint32_t *words, uint32_t *bits, int *scan, int r, int D,
                            uint32_t block, uint32_t round, uint32_t stream, uint64_t seed,
                            int *out) {
    const int nw = (D + 31) / 32;
    for (int i = threadIdx.x; i < r; i += blockDim.x)
        words[i] = philox_word((uint32_t)i, block, round, stream, seed);
    for (int i = threadIdx.x; i < nw; i += blockDim.x) bits[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0, j = D - r; j < D; ++i, ++j) {
            const uint32_t t = (uint32_t)(((uint64_t)words[i] * (uint64_t)(j + 1)) >> 32);
            const uint32_t b = (bits[t >> 5] >> (t & 31)) & 1u;
            const uint32_t v = b ? (uint32_t)j : t;
            bits[v >> 5] |= 1u << (v & 31);
        }
        int acc = 0;
        for (int w = 0; w < nw; ++w) {
            scan[w] = acc;
            acc += __popc(bits[w]);
        }
    }
    __syncthreads();
    if (out) {
        for (int w = threadIdx.x; w < nw; w += blockDim.x) {
            uint32_t x = bits[w];
            int pos = scan[w];
            while (x) {
                const int b = __ffs(x) - 1;
                out[pos++] = w * 32 + b;
                x &= x - 1;
            }
        }
    }
    __syncthreads();
}

// p extra draws out of the D - r values not set in bits_set (D bits valid); the k-th unset
// value is taken for draw k, results sorted. All threads of the CTA must call it.
__device__ void draw_extra(uint32_t *words, const uint32_t *bits_set, uint32_t *bitsX, int *scan,
                           int *pick, int p, int D, int r, uint32_t block, uint32_t round,
                           uint32_t stream, uint64_t seed, int *out) {
    if (p <= 0) return;
    draw_bitmap(words, bitsX, scan, p, D - r, block, round, stream, seed, pick);
    const int nw = (D + 31) / 32;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int q = 0; q < nw; ++q) {
            const uint32_t valid = (q == nw - 1 && (D & 31)) ? ((1u << (D & 31)) - 1u) : 0xffffffffu;
            scan[q] = acc;
            acc += __popc(~bits_set[q] & valid);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < p; e += blockDim.x) {
        const int kk = pick[e];
        int q = 0;
        while (q + 1 < nw && scan[q + 1] <= kk) ++q;
        const uint32_t valid = (q == nw - 1 && (D & 31)) ? ((1u << (D & 31)) - 1u) : 0xffffffffu;
        uint32_t z = ~bits_set[q] & valid;
        int left = kk - scan[q];
        while (left-- > 0) z &= z - 1;
        out[e] = q * 32 + __ffs(z) - 1;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(128) sample_kernel(const BlockWork *__restrict__ works,
                                                     uint64_t seed) {
    extern __shared__ __align__(16) uint32_t sh[];
    uint32_t *words = sh;                       // kMaxGroup
    uint32_t *bitsI = words + kMaxGroup;        // kMaxGroup/32 each
    uint32_t *bitsJ = bitsI + kMaxGroup / 32;
    uint32_t *bitsX = bitsJ + kMaxGroup / 32;
    int *scan = reinterpret_cast<int *>(bitsX + kMaxGroup / 32);
    int *pick = scan + kMaxGroup / 32;          // kMaxExtra
    const BlockWork w = works[blockIdx.x];
    // streams: 0 rows I, 1 columns J, 2 extra rows, 3 extra columns
    draw_bitmap(words, bitsJ, scan, w.r, w.n, w.block_id, w.round, 1u, seed, w.J);
    draw_bitmap(words, bitsI, scan, w.r, w.m, w.block_id, w.round, 0u, seed, w.I);
    draw_extra(words, bitsI, bitsX, scan, pick, w.pe, w.m, w.r, w.block_id, w.round, 2u, seed, w.Ix);
    draw_extra(words, bitsJ, bitsX, scan, pick, w.pc, w.n, w.r, w.block_id, w.round, 3u, seed, w.Jx);
    for (int i = threadIdx.x; i < w.r; i += blockDim.x) {
        w.Ig[i] = w.rows_g[w.I[i]];
        w.Jg[i] = w.cols_g[w.J[i]];
    }
    for (int e = threadIdx.x; e < w.pe; e += blockDim.x) w.Ig[w.r + e] = w.rows_g[w.Ix[e]];
    for (int e = threadIdx.x; e < w.pc; e += blockDim.x) w.Jg[w.r + e] = w.cols_g[w.Jx[e]];
}

static size_t sample_smem() {
    return sizeof(uint32_t) * (kMaxGroup + 4 * (kMaxGroup / 32)) + sizeof(int) * kMaxExtra;
}

// Re-check of a block accepted with little margin: pe2 fresh extra rows and pc2 fresh extra
// columns, drawn outside every row / column the block's round already used (I and Ix, J and
// Jx), from Philox streams 4 (rows) and 5 (columns) of that round. Every block that may need one
// is planned with its round; *gate, set on the device once the round's estimate is known,
// says whether it runs.
struct VerifyWork {
    const int *rows_g, *cols_g;
    const int *I, *J, *Ix, *Jx;  // the round's local samples
    int *Ix2, *Jx2;              // the new local samples (sorted)
    int *Ig2, *Jg2;              // their global ids
    int m, n, r, pe, pc, pe2, pc2;
    int block_id, round;
    const int *gate;
};

__global__ void __launch_bounds__(128) verify_sample_kernel(const VerifyWork *__restrict__ works,
                                                            uint64_t seed) {
    __shared__ uint32_t words[kMaxExtra];
    __shared__ uint32_t bits_used[kMaxGroup / 32];
    __shared__ uint32_t bits_x[kMaxGroup / 32];
    __shared__ int scan[kMaxGroup / 32];
    __shared__ int pick[kMaxExtra];
    const VerifyWork w = works[blockIdx.x];
    if (*w.gate == 0) return;
    for (int side = 0; side < 2; ++side) {
        const int D = side == 0 ? w.m : w.n;
        const int *S0 = side == 0 ? w.I : w.J;
        const int *S1 = side == 0 ? w.Ix : w.Jx;
        const int n1 = side == 0 ? w.pe : w.pc;
        const int p = side == 0 ? w.pe2 : w.pc2;
        int *out = side == 0 ? w.Ix2 : w.Jx2;
        const int nw = (D + 31) / 32;
        for (int i = threadIdx.x; i < nw; i += blockDim.x) bits_used[i] = 0u;
        __syncthreads();
        for (int i = threadIdx.x; i < w.r + n1; i += blockDim.x) {
            const int v = i < w.r ? S0[i] : S1[i - w.r];
            atomicOr(&bits_used[v >> 5], 1u << (v & 31));
        }
        __syncthreads();
        draw_extra(words, bits_used, bits_x, scan, pick, p, D, w.r + n1, w.block_id, w.round,
                   4u + side, seed, out);
    }
    for (int e = threadIdx.x; e < w.pe2; e += blockDim.x) w.Ig2[e] = w.rows_g[w.Ix2[e]];
    for (int e = threadIdx.x; e < w.pc2; e += blockDim.x) w.Jg2[e] = w.cols_g[w.Jx2[e]];
}

// ------------------------------------------------------------------ core gather
__device__ __forceinline__ double2 promote(double2 v) { return v; }
__device__ __forceinline__ double2 promote(float2 v) { return make_double2(v.x, v.y); }

// The core Z(I, J) = C(I, :) in FP64 for the SVD, and the same numbers written into R(:, J):
// C and R come from two fills (Z(group_t, J) and the transposed Z(group_s, I)) whose complex-FP32
// roundings of the shared entries Z(I, J) differ, and the pinv of an ill-conditioned core
// amplifies any difference between the core and R(:, J) (at r = min(m, n) with a near-exact
// inverse, to 1e-4 of the block). With one set of numbers C U R interpolates its own samples.
template <typename S>
__global__ void __launch_bounds__(256) gather_core_kernel(const BlockWork *__restrict__ works) {
    const BlockWork w = works[blockIdx.x];
    const S *C = reinterpret_cast<const S *>(w.C);
    S *Rx = reinterpret_cast<S *>(w.Rx);
    const int r = w.r, ldr = w.r + w.pe;
    for (int idx = threadIdx.x; idx < r * r; idx += blockDim.x) {
        const int i = idx % r, j = idx / r;
        const S v = C[w.I[i] + (size_t)j * w.m];
        w.AV[idx] = promote(v);
        Rx[i + (size_t)w.J[j] * ldr] = v;
    }
}

// ------------------------------------------------------------------ randomized estimate
// Residual of a block's C U R on pe extra rows and pc extra columns that were not sampled:
//   rows: ||Z(Ix,:) - C(Ix,:) U R||_F^2 and ||Z(Ix,:)||_F^2,
//   cols: ||Z(:,Jx) - C U R(:,Jx)||_F^2 and ||Z(:,Jx)||_F^2,
// and est = the larger of the two relative errors (0 where a side has no extra samples).
// The extra rows / columns live in their own buffers (the first round's are stacked below R and
// beside C in the round's storage; a re-check's are separate), so one kernel serves both.
struct EstJob {
    const void *C;    // m x >= r, ld m (the first r columns are C)
    const void *R;    // >= r rows x n, ld ldr (the first r rows are R)
    const double2 *U; // r x r
    const void *Xr;   // Z(Ix, :): row e, column j at Xr[e + j * ldxr]
    const void *Xc;   // Z(:, Jx): column c at Xc + c * m
    const int *Ix, *Jx;
    int m, n, r, ldr, ldxr, pe, pc;
    double2 *T;       // scratch: C(Ix, :) U (pe x r), then U R(:, Jx) (r x pc)
    double *out;      // est, then the four sums (rows num, den, cols num, den)
    const int *gate = nullptr;  // non-null: nothing is done while *gate is 0 (a re-check)
};

// SM: U and the scratch Tr, Sc live in shared memory (est_smem_bytes of the launch's largest
// r, pe, pc); otherwise U is read from global memory and Tr, Sc use the job's scratch. The
// arithmetic and its order are the same in both.
template <typename S, bool SM>
__global__ void __launch_bounds__(256) estimate_kernel(const EstJob *__restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char est_smem[];
    __shared__ double s_red[4][256];
    const EstJob w = jobs[blockIdx.x];
    if (w.gate && *w.gate == 0) return;
    const int r = w.r, pe = w.pe, pc = w.pc, n = w.n, m = w.m, ldr = w.ldr, ldxr = w.ldxr;
    const S *C = reinterpret_cast<const S *>(w.C);
    const S *Rm = reinterpret_cast<const S *>(w.R);
    const S *Xr = reinterpret_cast<const S *>(w.Xr);
    const S *Xc = reinterpret_cast<const S *>(w.Xc);
    const double2 *Uc = w.U;
    double2 *Tr = w.T;             // pe x r
    double2 *Sc = w.T + pe * r;    // r x pc
    if (SM) {
        double2 *sU = reinterpret_cast<double2 *>(est_smem);
        for (int e0 = threadIdx.x; e0 < r * r; e0 += 8 * blockDim.x) {
            double2 v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {  // loads first, then the stores
                const int e = e0 + u * blockDim.x;
                if (e < r * r) v[u] = w.U[e];
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (e0 + u * blockDim.x < r * r) sU[e0 + u * blockDim.x] = v[u];
        }
        Uc = sU;
        Tr = sU + r * r;
        Sc = Tr + pe * r;
        __syncthreads();
    }
    // Tr = C(Ix, :) U ; Sc = U R(:, Jx)
    for (int idx = threadIdx.x; idx < pe * r + r * pc; idx += blockDim.x) {
        double sx = 0, sy = 0;
        if (idx < pe * r) {
            const int e = idx % pe, k = idx / pe;
            const int row = w.Ix[e];
            for (int l = 0; l < r; ++l) {
                const double2 c = promote(C[row + (size_t)l * m]);
                const double2 u = Uc[l + (size_t)k * r];
                sx = fma(c.x, u.x, fma(-c.y, u.y, sx));
                sy = fma(c.x, u.y, fma(c.y, u.x, sy));
            }
            Tr[idx] = make_double2(sx, sy);
        } else {
            const int q = idx - pe * r;
            const int k = q % r, cc = q / r;
            const int col = w.Jx[cc];
            for (int l = 0; l < r; ++l) {
                const double2 u = Uc[k + (size_t)l * r];
                const double2 rv = promote(Rm[l + (size_t)col * ldr]);
                sx = fma(u.x, rv.x, fma(-u.y, rv.y, sx));
                sy = fma(u.x, rv.y, fma(u.y, rv.x, sy));
            }
            Sc[q] = make_double2(sx, sy);
        }
    }
    __syncthreads();
    // residuals on the extra rows (Z(Ix, j) - Tr R(:, j)) and the extra columns
    // (Z(i, Jx) - C(i, :) Sc): each thread keeps up to kEstChunk independent complex accumulators,
    // reading each factor value once per k
    constexpr int kEstChunk = 8;
    double nr_ = 0, dr_ = 0, nc_ = 0, dc_ = 0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {  // extra rows, column j
        const S *col = Rm + (size_t)j * ldr;
        const S *xcol = Xr + (size_t)j * ldxr;
        for (int e0 = 0; e0 < pe; e0 += kEstChunk) {
            double zx[kEstChunk], zy[kEstChunk];
#pragma unroll
            for (int q = 0; q < kEstChunk; ++q) zx[q] = zy[q] = 0.0;
            for (int k = 0; k < r; ++k) {
                const double2 rv = promote(col[k]);
#pragma unroll
                for (int q = 0; q < kEstChunk; ++q) {
                    if (e0 + q < pe) {
                        const double2 t = Tr[e0 + q + k * pe];
                        zx[q] = fma(t.x, rv.x, fma(-t.y, rv.y, zx[q]));
                        zy[q] = fma(t.x, rv.y, fma(t.y, rv.x, zy[q]));
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < kEstChunk; ++q) {
                if (e0 + q < pe) {
                    const double2 x = promote(xcol[e0 + q]);
                    const double dx = x.x - zx[q], dy = x.y - zy[q];
                    nr_ = fma(dx, dx, fma(dy, dy, nr_));
                    dr_ = fma(x.x, x.x, fma(x.y, x.y, dr_));
                }
            }
        }
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) {  // extra columns, row i
        for (int c0 = 0; c0 < pc; c0 += kEstChunk) {
            double zx[kEstChunk], zy[kEstChunk];
#pragma unroll
            for (int q = 0; q < kEstChunk; ++q) zx[q] = zy[q] = 0.0;
            for (int k = 0; k < r; ++k) {
                const double2 cv = promote(C[i + (size_t)k * m]);
#pragma unroll
                for (int q = 0; q < kEstChunk; ++q) {
                    if (c0 + q < pc) {
                        const double2 t = Sc[k + (c0 + q) * r];
                        zx[q] = fma(cv.x, t.x, fma(-cv.y, t.y, zx[q]));
                        zy[q] = fma(cv.x, t.y, fma(cv.y, t.x, zy[q]));
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < kEstChunk; ++q) {
                if (c0 + q < pc) {
                    const double2 x = promote(Xc[i + (size_t)(c0 + q) * m]);
                    const double dx = x.x - zx[q], dy = x.y - zy[q];
                    nc_ = fma(dx, dx, fma(dy, dy, nc_));
                    dc_ = fma(x.x, x.x, fma(x.y, x.y, dc_));
                }
            }
        }
    }
    s_red[0][threadIdx.x] = nr_;
    s_red[1][threadIdx.x] = dr_;
    s_red[2][threadIdx.x] = nc_;
    s_red[3][threadIdx.x] = dc_;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int q = 0; q < 4; ++q) s_red[q][threadIdx.x] += s_red[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double er = s_red[1][0] > 0 ? sqrt(s_red[0][0] / s_red[1][0]) : 0.0;
        const double ec = s_red[3][0] > 0 ? sqrt(s_red[2][0] / s_red[3][0]) : 0.0;
        w.out[0] = fmax(er, ec);
        for (int q = 0; q < 4; ++q) w.out[1 + q] = s_red[q][0];
    }
}

// Shared memory of the estimate for cores up to r, pe extra rows, pc extra columns.
inline size_t est_smem_bytes(int r, int pe, int pc) {
    return sizeof(double2) * ((size_t)r * r + (size_t)(pe + pc) * r);
}
constexpr size_t kEstSmemMax = 96 * 1024;

// One estimate launch of cnt jobs whose largest r, pe, pc are given.
int launch_estimate(const EstJob *d_jobs, int cnt, int precision, int rmax, int pemax, int pcmax,
                    cudaStream_t st) {
    if (cnt <= 0) return PSKEL_OK;
    const size_t sm = est_smem_bytes(rmax, pemax, pcmax);
    if (sm <= kEstSmemMax) {
        if (precision == PSKEL_C64) {
            PSKEL_TRY(ensure_smem_attr(estimate_kernel<float2, true>, kEstSmemMax));
            estimate_kernel<float2, true><<<cnt, 256, sm, st>>>(d_jobs);
        } else {
            PSKEL_TRY(ensure_smem_attr(estimate_kernel<double2, true>, kEstSmemMax));
            estimate_kernel<double2, true><<<cnt, 256, sm, st>>>(d_jobs);
        }
    } else if (precision == PSKEL_C64) {
        estimate_kernel<float2, false><<<cnt, 256, 0, st>>>(d_jobs);
    } else {
        estimate_kernel<double2, false><<<cnt, 256, 0, st>>>(d_jobs);
    }
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

// per-block outcome gather: est, rank, svd status into one compact array for a single D2H
struct RoundOut {
    double est;
    double sums[4];  // residual and norm sums of the estimate (rows num, den, cols num, den)
    int rank;
    int status;
    int sweeps;  // Jacobi sweeps of the core SVD
    int pad;
};
__global__ void collect_kernel(const BlockWork *__restrict__ works, const SvdJob *__restrict__ svd,
                               int nb, RoundOut *out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    out[b].est = works[b].est[0];
    for (int q = 0; q < 4; ++q) out[b].sums[q] = works[b].est[1 + q];
    out[b].rank = *works[b].rank;
    out[b].status = svd[b].status;
    out[b].sweeps = svd[b].sweeps;
}

// Which of the round's re-check candidates run: candidate v (the round's block idx[v]) passed
// with little margin (status OK, est <= hi, not est <= lo).
__global__ void verify_select_kernel(const int *__restrict__ idx, int nv, const RoundOut *__restrict__ outs,
                                     double hi, double lo, int *gate) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const RoundOut q = outs[idx[v]];
    gate[v] = (q.status == PSKEL_OK && q.est <= hi && !(q.est <= lo)) ? 1 : 0;
}

// Extra rows and columns of a re-check: as many as are left outside the round's samples, up to
// the option's counts.
void verify_extent(int m, int n, int r, int pe, int pc, const pskel_opts_t &o, int *pe2, int *pc2) {
    *pe2 = std::max(0, std::min(o.extra_rows, m - r - pe));
    *pc2 = std::max(0, std::min(o.extra_cols, n - r - pc));
}

// The round's outcome buffer: RoundOut per block, then 8 doubles per re-check candidate (est on
// the new samples alone, the four residual sums), then each candidate's gate.
size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
size_t outs_vouts_offset(int nb) { return al256(sizeof(RoundOut) * (size_t)nb); }
size_t outs_gates_offset(int nb, int nv) { return outs_vouts_offset(nb) + al256(sizeof(double) * 8 * (size_t)nv); }
size_t outs_bytes(int nb, int nv) { return outs_gates_offset(nb, nv) + al256(sizeof(int) * (size_t)nv); }

// ------------------------------------------------------------------ true errors
__global__ void block_norm_kernel(const double2 *const *mats, const long long *sizes, double *out) {
    __shared__ double s[256];
    const double2 *a = mats[blockIdx.x];
    const long long n = sizes[blockIdx.x];
    double acc = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) acc = fma(a[i].x, a[i].x, fma(a[i].y, a[i].y, acc));
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s[0]);
}

template <typename S>
__global__ void promote_kernel(const S *in, double2 *out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = promote(in[i]);
}

// ------------------------------------------------------------------ dense reference product
// Y(rows_b, :) += Z_b X(cols_b, :) for the densely filled blocks of a batch (complex FP64):
// one CTA per block, one (row, right-hand side) pair per thread and step, FP64 atomics into Y.
struct DenseApply {
    const double2 *Z;   // m x n, column-major
    const int *rows, *cols;
    int m, n;
};
__global__ void __launch_bounds__(256) dense_apply_kernel(const DenseApply *__restrict__ jobs,
                                                          const double2 *__restrict__ X, int ldx,
                                                          double2 *Y, int ldy, int nrhs) {
    const DenseApply w = jobs[blockIdx.x];
    for (int e = threadIdx.x; e < w.m * nrhs; e += blockDim.x) {
        const int i = e % w.m, q = e / w.m;
        double ax = 0, ay = 0;
        for (int j = 0; j < w.n; ++j) {
            const double2 z = w.Z[i + (size_t)j * w.m];
            const double2 x = X[w.cols[j] + (size_t)q * ldx];
            ax = fma(z.x, x.x, fma(-z.y, x.y, ax));
            ay = fma(z.x, x.y, fma(z.y, x.x, ay));
        }
        double *y = reinterpret_cast<double *>(Y + w.rows[i] + (size_t)q * ldy);
        atomicAdd(y, ax);
        atomicAdd(y + 1, ay);
    }
}

}  // namespace pskel

// ====================================================================== context
using namespace pskel;

namespace {

// columns per tile of a triangle-moment fill job: the context's fixed width, or (width 0) the
// balanced width of tri_tile_cols up to the widest variant
int tri_cols_for(const pskel_ctx *c, int nt) {
    return c->tri_cols > 0 ? c->tri_cols : tri_tile_cols(nt, kTriFillCols);
}


// the per-(triangle, slot) table of group g for the triangle-moment fill
const double *guse_of(const pskel_ctx *c, int g) {
    return c->d_guse.as<double>() + 12 * (size_t)c->gtri_ptr[g];
}

// fill variant actually used for a precision: the triangle-moment kernel when asked for and
// every group fits it, else the per-entry kernel (two rows per thread when 8 was asked for)
bool tri_for(const pskel_ctx *c, int precision) {
    return c->split[precision == PSKEL_C64 ? 1 : 0] == 8 && c->use_tri;
}
int entry_split_for(const pskel_ctx *c, int precision) {
    const int s = c->split[precision == PSKEL_C64 ? 1 : 0];
    return s == 8 ? 0 : s;
}

int ctx_ok(pskel_ctx *c) {
    if (!c) {
        set_error(PSKEL_ERR_ARG, "null context");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    return PSKEL_OK;
}

size_t al16(size_t x) { return (x + 15) & ~size_t(15); }


struct RoundPlan {
    std::vector<int> blocks;     // block ids of this round
    std::vector<int> r, pe, pc;
    int round = 0;
    // device table views (inside arena.tables)
    BlockWork *d_works = nullptr;
    FillJob *d_fill = nullptr;            // per-entry fill jobs (groups too large for tri)
    GroupFillJob *d_gfill = nullptr;      // triangle-moment fill jobs
    bool tri = false;
    int tri_rows = 0;                     // largest group among the triangle-moment jobs
    int *d_fill_prefix = nullptr;
    int fill_jobs = 0, fill_tiles = 0;
    SvdJob *d_svd = nullptr;
    int *d_svd_idx = nullptr;
    SvdPlan svd;
    PinvJob *d_pinv = nullptr;
    EstJob *d_est = nullptr;
    int pinv_tiles = 0;
    int nb = 0;
    // pipeline chunks: blocks [cb[k], cb[k+1]) of the works order; each chunk has its own fill
    // tile prefix (from 0), SVD plan (index map into the round's SvdJob table) and pinv tiles
    std::vector<int> cb;
    std::vector<int> ch_tiles, ch_pinv_tiles;
    std::vector<int *> ch_prefix, ch_idx;
    std::vector<SvdPlan> ch_svd;
    // re-check candidates (round indices; set before planning) and the selection thresholds
    std::vector<int> vcand;
    double v_hi = 0, v_lo = 0;
    // their tables (inside arena.tables), gated by the selection after the round's estimate
    int nv = 0;
    VerifyWork *d_vworks = nullptr;
    FillJob *d_vfill = nullptr;
    GroupFillJob *d_vgfill = nullptr;
    int *d_vidx = nullptr, *d_gates = nullptr;
    const int *const *d_vjgate = nullptr;  // per re-check fill job: its candidate's gate
    // per pipeline chunk: its candidates [vc[k], vc[k+1]), fill jobs [vj[k], vj[k+1]) with their
    // own tile prefix (from 0) and tile count
    std::vector<int> vc, vj, vch_tiles;
    std::vector<int *> vch_prefix;
    EstJob *d_vest = nullptr;
    int vtri_rows = 0, vrmax = 0, vpemax = 0, vpcmax = 0;
};

constexpr int kPipeMinBlocks = 2048;  // smaller rounds run as one chunk

// f(lo, hi) over [0, n) split into contiguous ranges run on up to kPlanThreads host threads
// (one range per thread of at least min_each items; the calling thread takes the first)
constexpr int kPlanThreads = 8;
template <typename F>
void parallel_ranges(int n, int min_each, F f) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min({kPlanThreads, hw, n / std::max(1, min_each)}));
    if (nt <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (int t = 1; t < nt; ++t) {
        const int lo = (int)((long long)n * t / nt), hi = (int)((long long)n * (t + 1) / nt);
        try {
            th.emplace_back(f, lo, hi);
        } catch (...) {  // no thread to be had: the range runs here
            f(lo, hi);
        }
    }
    f(0, (int)((long long)n / nt));
    for (std::thread &x : th) x.join();
}

// Lay out the round's storage, build all job tables on the host and upload them in one copy.
// A first pass sizes everything (storage, fill tiles, pipeline chunks, re-check extents), so
// that the second writes every table once, straight into the context's page-locked staging
// buffer, from which one asynchronous copy uploads them.
int plan_round(pskel_ctx *c, RoundPlan &p, const pskel_opts_t &o) {
    const int nb = (int)p.blocks.size();
    p.nb = nb;
    if ((int)c->arenas.size() <= p.round) c->arenas.resize(p.round + 1);
    RoundArena &ar = c->arenas[p.round];
    const size_t es = o.precision == PSKEL_C64 ? sizeof(float2) : sizeof(double2);
    const int nv = (int)p.vcand.size();
    p.nv = nv;
    p.tri = tri_for(c, o.precision);
    int tm, tn;
    fill_tile_shape(o.precision, c->em.q_test, entry_split_for(c, o.precision), &tm, &tn);
    auto rows_of = [&](int g) { return c->gptr[g + 1] - c->gptr[g]; };
    auto tris_of = [&](int g) { return c->gtri_ptr[g + 1] - c->gtri_ptr[g]; };
    // triangle-moment tile width of each group's jobs
    std::vector<int> gtc;
    if (p.tri) {
        gtc.resize(c->gptr.size() - 1);
        for (size_t g = 0; g < gtc.size(); ++g) gtc[g] = tri_cols_for(c, tris_of((int)g));
    }
    // tiles of a fill job of nr rows (group g) and nc columns
    auto job_tiles = [&](int g, int nr, int nc) {
        if (p.tri) return (nc + gtc[g] - 1) / gtc[g];
        return ((nr + tm - 1) / tm) * ((nc + tn - 1) / tn);
    };
    // ---- first pass: keep arena, scratch, fill tiles (C, then Rx, of each block): sizes per
    // block on the planning threads, then the running offsets
    std::vector<size_t> off(nb + 1, 0), soffs(nb + 1, 0);
    std::vector<int> prefix(2 * (size_t)nb + 1, 0);
    int max_pinv_tiles = 0;
    p.tri_rows = 0;
    std::mutex red;  // the per-range maxima
    parallel_ranges(nb, 2048, [&](int lo, int hi) {
        int pt = 0, rm = 0;
        for (int i = lo; i < hi; ++i) {
            const int b = p.blocks[i], gt = c->gt[b], gs = c->gs[b];
            const size_t m = rows_of(gt), n = rows_of(gs);
            const size_t r = p.r[i], pe = p.pe[i], pc = p.pc[i];
            size_t sz = 0;
            sz += al16(m * (r + pc) * es);       // C (+ extra columns)
            sz += al16((r + pe) * n * es);       // Rx
            sz += al16(r * r * sizeof(double2)); // U
            sz += al16(sizeof(int) * r) * 2;     // I, J
            sz += al16(sizeof(int) * (pe + 1));  // Ix
            sz += al16(sizeof(int) * (pc + 1));  // Jx
            sz += al16(sizeof(int) * (r + pe));  // Ig
            sz += al16(sizeof(int) * (r + pc));  // Jg
            sz += al16(sizeof(double) * r);      // sigma
            sz += al16(sizeof(int) * r);         // perm
            sz += 16 + 64;                       // rank; est and its four sums
            off[i + 1] = (sz + 255) & ~size_t(255);
            soffs[i + 1] = 2 * al16(r * r * sizeof(double2)) + al16((pe + pc) * r * sizeof(double2));
            prefix[2 * i + 1] = job_tiles(gt, (int)m, (int)(r + pc));
            prefix[2 * i + 2] = job_tiles(gs, (int)n, (int)(r + pe));
            if (p.tri) rm = std::max(rm, (int)std::max(m, n));
            pt = std::max(pt, (int)(((r + 31) / 32) * ((r + 31) / 32)));
        }
        std::lock_guard<std::mutex> lk(red);
        max_pinv_tiles = std::max(max_pinv_tiles, pt);
        p.tri_rows = std::max(p.tri_rows, rm);
    });
    for (int i = 0; i < nb; ++i) {
        off[i + 1] += off[i];
        soffs[i + 1] += soffs[i];
    }
    for (size_t j = 1; j < prefix.size(); ++j) prefix[j] += prefix[j - 1];
    size_t scratch_total = soffs[nb];
    // re-check storage of every candidate after the blocks' scratch: the fresh extra columns
    // (m x pc2) and rows (pe2 x n), their local and global ids, the estimate's scratch; its fill
    // jobs (extra columns, then extra rows, where there are any) and their tiles
    std::vector<int> vpe2(nv), vpc2(nv), vjob0(nv + 1, 0), vtc(nv), vtr(nv);
    std::vector<size_t> voff(nv + 1, 0);
    p.vrmax = p.vpemax = p.vpcmax = p.vtri_rows = 0;
    parallel_ranges(nv, 2048, [&](int lo, int hi) {
        int rmax = 0, pemax = 0, pcmax = 0, trows = 0;
        for (int v = lo; v < hi; ++v) {
            const int i = p.vcand[v], b = p.blocks[i], gt = c->gt[b], gs = c->gs[b];
            const int m = rows_of(gt), n = rows_of(gs);
            verify_extent(m, n, p.r[i], p.pe[i], p.pc[i], o, &vpe2[v], &vpc2[v]);
            size_t q = al16((size_t)m * vpc2[v] * es) + al16((size_t)vpe2[v] * n * es);
            q += 4 * al16(sizeof(int) * (kMaxExtra + 1));
            q += al16(sizeof(double2) * (size_t)(vpe2[v] + vpc2[v]) * p.r[i]);
            voff[v + 1] = al256(q);
            vtc[v] = vpc2[v] > 0 ? job_tiles(gt, m, vpc2[v]) : -1;  // -1: no job
            vtr[v] = vpe2[v] > 0 ? job_tiles(gs, n, vpe2[v]) : -1;
            if (p.tri && vpc2[v] > 0) trows = std::max(trows, m);
            if (p.tri && vpe2[v] > 0) trows = std::max(trows, n);
            rmax = std::max(rmax, p.r[i]);
            pemax = std::max(pemax, vpe2[v]);
            pcmax = std::max(pcmax, vpc2[v]);
        }
        std::lock_guard<std::mutex> lk(red);
        p.vrmax = std::max(p.vrmax, rmax);
        p.vpemax = std::max(p.vpemax, pemax);
        p.vpcmax = std::max(p.vpcmax, pcmax);
        p.vtri_rows = std::max(p.vtri_rows, trows);
    });
    // running offsets; each candidate's fill jobs (extra columns, then extra rows, where there
    // are any) and their tiles
    std::vector<int> vprefix(1, 0);
    vprefix.reserve(2 * (size_t)nv + 1);
    for (int v = 0; v < nv; ++v) {
        voff[v + 1] += voff[v];
        vjob0[v] = (int)vprefix.size() - 1;
        if (vtc[v] >= 0) vprefix.push_back(vprefix.back() + vtc[v]);
        if (vtr[v] >= 0) vprefix.push_back(vprefix.back() + vtr[v]);
    }
    const int nvf = (int)vprefix.size() - 1;
    vjob0[nv] = nvf;
    scratch_total = al256(scratch_total);
    PSKEL_TRY(ar.keep.reserve(off[nb] + 256));
    PSKEL_TRY(ar.work.reserve(scratch_total + voff[nv] + 256));
    PSKEL_TRY(ar.outs.reserve(outs_bytes(nb, nv) + 256));
    // pipeline chunks, each with its own tables, of decreasing fill work: chunk k ends at the
    // fraction 1 - (1 - k/K)^2 of the tiles, so the early chunks' pinv and estimate run beside
    // the many later fills and the last chunk, whose pinv and estimate run alone, is small
    const int K = (nb >= kPipeMinBlocks && c->pipe_chunks > 1) ? std::min(c->pipe_chunks, pskel_ctx::kMaxChunks) : 1;
    p.cb.assign(1, 0);
    {
        const long long total = prefix.back();
        int b = 0;
        for (int k = 1; k < K; ++k) {
            const double left = 1.0 - (double)k / K;
            const long long want = (long long)((1.0 - left * left) * (double)total);
            while (b < nb && prefix[2 * (size_t)b] < want) ++b;
            if (b > p.cb.back()) p.cb.push_back(b);
        }
        p.cb.push_back(nb);
    }
    const int nch = (int)p.cb.size() - 1;
    // the re-checks by pipeline chunk (candidates are in round order, so each chunk's candidates
    // and their fill jobs are contiguous)
    p.vc.assign(nch + 1, nv);
    p.vj.assign(nch + 1, nvf);
    p.vch_tiles.assign(nch, 0);
    for (int k = 0; k < nch; ++k) {
        p.vc[k] = (int)(std::lower_bound(p.vcand.begin(), p.vcand.end(), p.cb[k]) - p.vcand.begin());
        p.vj[k] = vjob0[p.vc[k]];
    }
    // ---- table layout in the staging buffer (and, at the same offsets, on the device)
    size_t t = 0;
    auto slot = [&](size_t bytes) { size_t x = t; t += (bytes + 255) & ~size_t(255); return x; };
    const size_t o_works = slot(sizeof(BlockWork) * nb);
    const size_t o_fill = p.tri ? slot(sizeof(GroupFillJob) * 2 * (size_t)nb) : slot(sizeof(FillJob) * 2 * (size_t)nb);
    const size_t o_pref = slot(sizeof(int) * prefix.size());
    const size_t o_svd = slot(sizeof(SvdJob) * nb);
    const size_t o_idx = slot(sizeof(int) * nb);
    const size_t o_pinv = slot(sizeof(PinvJob) * nb);
    const size_t o_est = slot(sizeof(EstJob) * nb);
    const size_t o_cpref = slot(sizeof(int) * (2 * (size_t)nb + nch));
    const size_t o_cidx = slot(sizeof(int) * (nb + 1));
    const size_t o_vw = slot(sizeof(VerifyWork) * nv);
    const size_t o_vf = p.tri ? slot(sizeof(GroupFillJob) * (nvf + 1)) : slot(sizeof(FillJob) * (nvf + 1));
    const size_t o_vp = slot(sizeof(int) * (nvf + nch));
    const size_t o_ve = slot(sizeof(EstJob) * nv);
    const size_t o_vi = slot(sizeof(int) * (nv + 1));
    const size_t o_vg = slot(sizeof(const int *) * (nvf + 1));
    PSKEL_TRY(c->plan_host.reserve(t + 256));
    char *h = c->plan_host.as<char>();
    BlockWork *works = reinterpret_cast<BlockWork *>(h + o_works);
    FillJob *fills = reinterpret_cast<FillJob *>(h + o_fill);
    GroupFillJob *gfills = reinterpret_cast<GroupFillJob *>(h + o_fill);
    SvdJob *svds = reinterpret_cast<SvdJob *>(h + o_svd);
    PinvJob *pinvs = reinterpret_cast<PinvJob *>(h + o_pinv);
    EstJob *ests = reinterpret_cast<EstJob *>(h + o_est);
    std::memcpy(h + o_pref, prefix.data(), sizeof(int) * prefix.size());
    // ---- second pass: every block's storage pointers and jobs
    char *kb = ar.keep.as<char>();
    char *sb = ar.work.as<char>();
    const int *tri_ids = c->d_gtri.as<int>(), *tri_adj = c->d_gadj.as<int>();
    parallel_ranges(nb, 2048, [&](int lo, int hi) {
    for (int i = lo; i < hi; ++i) {
        const int b = p.blocks[i];
        BlockWork w{};
        BlockResult &res = c->results[b];
        w.rows_g = c->d_gids.as<int>() + c->gptr[c->gt[b]];
        w.cols_g = c->d_gids.as<int>() + c->gptr[c->gs[b]];
        w.m = rows_of(c->gt[b]);
        w.n = rows_of(c->gs[b]);
        w.r = p.r[i];
        w.pe = p.pe[i];
        w.pc = p.pc[i];
        w.block_id = b;
        w.round = p.round;
        char *q = kb + off[i];
        auto take = [&](size_t bytes) { char *x = q; q += al16(bytes); return x; };
        const size_t m = w.m, n = w.n, r = w.r, pe = w.pe, pc = w.pc;
        w.C = take(m * (r + pc) * es);
        w.Rx = take((r + pe) * n * es);
        w.U = reinterpret_cast<double2 *>(take(r * r * sizeof(double2)));
        w.I = reinterpret_cast<int *>(take(sizeof(int) * r));
        w.J = reinterpret_cast<int *>(take(sizeof(int) * r));
        w.Ix = reinterpret_cast<int *>(take(sizeof(int) * (pe + 1)));
        w.Jx = reinterpret_cast<int *>(take(sizeof(int) * (pc + 1)));
        w.Ig = reinterpret_cast<int *>(take(sizeof(int) * (r + pe)));
        w.Jg = reinterpret_cast<int *>(take(sizeof(int) * (r + pc)));
        w.sigma = reinterpret_cast<double *>(take(sizeof(double) * r));
        w.perm = reinterpret_cast<int *>(take(sizeof(int) * r));
        w.rank = reinterpret_cast<int *>(take(16));
        w.est = reinterpret_cast<double *>(take(64));
        size_t soff = soffs[i];
        w.AV = reinterpret_cast<double2 *>(sb + soff);
        soff += al16(r * r * sizeof(double2));
        w.V = reinterpret_cast<double2 *>(sb + soff);
        soff += al16(r * r * sizeof(double2));
        w.T = reinterpret_cast<double2 *>(sb + soff);
        works[i] = w;
        // C = Z(group_t, [J; Jx]); Rx = Z([I; Ix], group_s) filled as the transpose of
        // Z(group_s, [I; Ix]) (the Galerkin block is symmetric for equal test and source rules),
        // so the long side is on rows
        if (p.tri) {
            const int gt = c->gt[b], gs = c->gs[b];
            gfills[2 * i] = GroupFillJob{w.rows_g, tri_ids + c->gtri_ptr[gt], tri_adj + 3 * (size_t)c->gtri_ptr[gt],
                                         w.Jg, w.C, w.m, tris_of(gt), w.r + w.pc, w.m, 0,
                                         gtc[gt], guse_of(c, gt)};
            gfills[2 * i + 1] = GroupFillJob{w.cols_g, tri_ids + c->gtri_ptr[gs], tri_adj + 3 * (size_t)c->gtri_ptr[gs],
                                             w.Ig, w.Rx, w.n, tris_of(gs), w.r + w.pe, w.r + w.pe, 1,
                                             gtc[gs], guse_of(c, gs)};
        } else {
            fills[2 * i] = FillJob{w.rows_g, w.Jg, w.C, w.m, w.r + w.pc, w.m, 0};
            fills[2 * i + 1] = FillJob{w.cols_g, w.Ig, w.Rx, w.n, w.r + w.pe, w.r + w.pe, 1};
        }
        svds[i] = SvdJob{w.AV, w.V, w.sigma, w.perm, w.r, w.r, 0, 0};
        // a block sampled on every row or every column of its smaller side cannot gain from more
        // samples: its pinv keeps every singular value above full_tau of the largest, so that
        // C U R reproduces the block instead of losing the truncated directions
        double tau_i = o.tau;
        int rel_i = o.tau_relative;
        if (w.r >= std::min(w.m, w.n) && o.full_tau > 0) {
            tau_i = rel_i ? std::min(o.tau, o.full_tau) : o.full_tau;
            rel_i = 1;
        }
        pinvs[i] = PinvJob{w.AV, w.V, w.sigma, w.U, w.rank, w.r, w.r, tau_i, rel_i};
        ests[i] = EstJob{w.C, w.Rx, w.U, (const char *)w.Rx + r * es, (const char *)w.C + m * r * es,
                         w.Ix, w.Jx, w.m, w.n, w.r, w.r + w.pe, w.r + w.pe, w.pe, w.pc, w.T, w.est};
        res.m = w.m;
        res.n = w.n;
        res.r = w.r;
        res.pe = w.pe;
        res.pc = w.pc;
        res.round = p.round;
        res.arena = p.round;
        res.offC = (char *)w.C - kb;
        res.offRx = (char *)w.Rx - kb;
        res.offU = (char *)w.U - kb;
        res.offI = (char *)w.I - kb;
        res.offJ = (char *)w.J - kb;
        res.offAV = (char *)w.AV - sb;
        res.offV = (char *)w.V - sb;
        res.offSig = (char *)w.sigma - kb;
        res.offPerm = (char *)w.perm - kb;
    }
    });
    // SVD plans of the round and of each chunk (index maps into the round's SvdJob table)
    PSKEL_TRY(svd_plan(svds, nb, p.svd));
    std::memcpy(h + o_idx, p.svd.idx.data(), sizeof(int) * nb);
    std::vector<size_t> ch_pref_off(nch), ch_idx_off(nch);
    p.ch_svd.assign(nch, SvdPlan());
    p.ch_tiles.assign(nch, 0);
    p.ch_pinv_tiles.assign(nch, 0);
    {
        int *cpref = reinterpret_cast<int *>(h + o_cpref);
        int *cidx = reinterpret_cast<int *>(h + o_cidx);
        size_t np = 0, ni = 0;
        for (int k = 0; k < nch; ++k) {
            const int b0 = p.cb[k], b1 = p.cb[k + 1];
            ch_pref_off[k] = np;
            for (int j = 2 * b0; j <= 2 * b1; ++j) cpref[np++] = prefix[j] - prefix[2 * b0];
            p.ch_tiles[k] = prefix[2 * b1] - prefix[2 * b0];
            PSKEL_TRY(svd_plan(svds + b0, b1 - b0, p.ch_svd[k]));
            for (int &x : p.ch_svd[k].idx) x += b0;  // into the round's SvdJob table
            ch_idx_off[k] = ni;
            for (int x : p.ch_svd[k].idx) cidx[ni++] = x;
            for (int i = b0; i < b1; ++i)
                p.ch_pinv_tiles[k] = std::max(p.ch_pinv_tiles[k], ((p.r[i] + 31) / 32) * ((p.r[i] + 31) / 32));
        }
    }
    // ---- re-check tables of every candidate; the gates and outputs live in the outcome buffer
    {
        VerifyWork *vws = reinterpret_cast<VerifyWork *>(h + o_vw);
        EstJob *vests = reinterpret_cast<EstJob *>(h + o_ve);
        FillJob *vfills = reinterpret_cast<FillJob *>(h + o_vf);
        GroupFillJob *vgfills = reinterpret_cast<GroupFillJob *>(h + o_vf);
        const int **vjgate = reinterpret_cast<const int **>(h + o_vg);
        std::memcpy(h + o_vi, p.vcand.data(), sizeof(int) * nv);
        char *vb = sb + scratch_total;
        char *ob = ar.outs.as<char>();
        double *vouts = reinterpret_cast<double *>(ob + outs_vouts_offset(nb));
        int *gates = reinterpret_cast<int *>(ob + outs_gates_offset(nb, nv));
        p.d_gates = gates;
        parallel_ranges(nv, 2048, [&](int lo, int hi) {
        for (int v = lo; v < hi; ++v) {
            int f = vjob0[v];  // the candidate's first re-check fill job
            const int i = p.vcand[v];
            const BlockWork &w = works[i];
            const int b = w.block_id, pe2 = vpe2[v], pc2 = vpc2[v];
            char *q = vb + voff[v];
            auto take = [&](size_t bytes) { char *x = q; q += al16(bytes); return x; };
            VerifyWork x{};
            x.rows_g = w.rows_g;
            x.cols_g = w.cols_g;
            x.I = w.I;
            x.J = w.J;
            x.Ix = w.Ix;
            x.Jx = w.Jx;
            x.m = w.m;
            x.n = w.n;
            x.r = w.r;
            x.pe = w.pe;
            x.pc = w.pc;
            x.pe2 = pe2;
            x.pc2 = pc2;
            x.block_id = b;
            x.round = w.round;
            x.gate = gates + v;
            void *Xc = take((size_t)w.m * pc2 * es);
            void *Xr = take((size_t)pe2 * w.n * es);
            x.Ix2 = reinterpret_cast<int *>(take(sizeof(int) * (kMaxExtra + 1)));
            x.Jx2 = reinterpret_cast<int *>(take(sizeof(int) * (kMaxExtra + 1)));
            x.Ig2 = reinterpret_cast<int *>(take(sizeof(int) * (kMaxExtra + 1)));
            x.Jg2 = reinterpret_cast<int *>(take(sizeof(int) * (kMaxExtra + 1)));
            double2 *T = reinterpret_cast<double2 *>(take(sizeof(double2) * (size_t)(pe2 + pc2) * w.r));
            vws[v] = x;
            vests[v] = EstJob{w.C, w.Rx, w.U, Xr, Xc, x.Ix2, x.Jx2, w.m, w.n, w.r, w.r + w.pe,
                              std::max(pe2, 1), pe2, pc2, T, vouts + 8 * (size_t)v, gates + v};
            const int gt = c->gt[b], gs = c->gs[b];
            if (pc2 > 0) {
                if (p.tri)
                    vgfills[f] = GroupFillJob{w.rows_g, tri_ids + c->gtri_ptr[gt], tri_adj + 3 * (size_t)c->gtri_ptr[gt],
                                              x.Jg2, Xc, w.m, tris_of(gt), pc2, w.m, 0,
                                              gtc[gt], guse_of(c, gt)};
                else
                    vfills[f] = FillJob{w.rows_g, x.Jg2, Xc, w.m, pc2, w.m, 0};
                vjgate[f++] = gates + v;
            }
            if (pe2 > 0) {
                if (p.tri)
                    vgfills[f] = GroupFillJob{w.cols_g, tri_ids + c->gtri_ptr[gs], tri_adj + 3 * (size_t)c->gtri_ptr[gs],
                                              x.Ig2, Xr, w.n, tris_of(gs), pe2, pe2, 1,
                                              gtc[gs], guse_of(c, gs)};
                else
                    vfills[f] = FillJob{w.cols_g, x.Ig2, Xr, w.n, pe2, pe2, 1};
                vjgate[f++] = gates + v;
            }
        }
        });
    }
    std::vector<size_t> vch_off(nch);
    {
        int *vp = reinterpret_cast<int *>(h + o_vp);
        size_t np = 0;
        for (int k = 0; k < nch; ++k) {
            vch_off[k] = np;
            for (int j = p.vj[k]; j <= p.vj[k + 1]; ++j) vp[np++] = vprefix[j] - vprefix[p.vj[k]];
            p.vch_tiles[k] = vprefix[p.vj[k + 1]] - vprefix[p.vj[k]];
        }
    }
    // ---- one asynchronous upload from the staging buffer (the previous round's upload from it
    // completed before that round's outcome was read)
    PSKEL_TRY(ar.tables.reserve(t + 256));
    PSKEL_CUDA(cudaMemcpyAsync(ar.tables.ptr, h, t, cudaMemcpyHostToDevice, c->stream));
    char *d = ar.tables.as<char>();
    p.d_works = reinterpret_cast<BlockWork *>(d + o_works);
    p.d_fill = reinterpret_cast<FillJob *>(d + o_fill);
    p.d_gfill = reinterpret_cast<GroupFillJob *>(d + o_fill);
    p.d_fill_prefix = reinterpret_cast<int *>(d + o_pref);
    p.fill_jobs = 2 * nb;
    p.fill_tiles = prefix.back();
    p.d_svd = reinterpret_cast<SvdJob *>(d + o_svd);
    p.d_svd_idx = reinterpret_cast<int *>(d + o_idx);
    p.d_pinv = reinterpret_cast<PinvJob *>(d + o_pinv);
    p.d_est = reinterpret_cast<EstJob *>(d + o_est);
    p.d_vworks = reinterpret_cast<VerifyWork *>(d + o_vw);
    p.d_vfill = reinterpret_cast<FillJob *>(d + o_vf);
    p.d_vgfill = reinterpret_cast<GroupFillJob *>(d + o_vf);
    p.d_vest = reinterpret_cast<EstJob *>(d + o_ve);
    p.d_vidx = reinterpret_cast<int *>(d + o_vi);
    p.d_vjgate = reinterpret_cast<const int *const *>(d + o_vg);
    p.vch_prefix.assign(nch, nullptr);
    for (int k = 0; k < nch; ++k) p.vch_prefix[k] = reinterpret_cast<int *>(d + o_vp) + vch_off[k];
    p.ch_prefix.assign(nch, nullptr);
    p.ch_idx.assign(nch, nullptr);
    for (int k = 0; k < nch; ++k) {
        p.ch_prefix[k] = reinterpret_cast<int *>(d + o_cpref) + ch_pref_off[k];
        p.ch_idx[k] = reinterpret_cast<int *>(d + o_cidx) + ch_idx_off[k];
    }
    p.pinv_tiles = max_pinv_tiles;
    return PSKEL_OK;
}

// All kernels of one round (no host synchronisation inside: capturable). A round of several
// chunks is pipelined: the fill of chunk k + 1 (one CTA per tile) on the context's stream
// overlaps the gather, SVD, pinv and estimate of chunk k on the high-priority pipeline stream,
// whose CTAs take the SMs' free slots as fill CTAs retire (the fill is bound by FP32 issue, the
// Jacobi SVD by FP64 latency).
int launch_round(pskel_ctx *c, const RoundPlan &p, const pskel_opts_t &o, bool events) {
    cudaStream_t s = c->stream;
    if (events) PSKEL_CUDA(cudaEventRecord(c->ev[0], s));
    sample_kernel<<<p.nb, 128, sample_smem(), s>>>(p.d_works, o.seed);
    PSKEL_LAUNCHED(1);
    if (events) PSKEL_CUDA(cudaEventRecord(c->ev[1], s));
    FillParams fp;
    fp.k = c->em.k;
    fp.eta = c->em.eta;
    fp.r_near = 0.0;
    fp.q_test = c->em.q_test;
    fp.q_src = c->em.q_src;
    fp.precision = o.precision;
    fp.split = entry_split_for(c, o.precision);
    fp.tri_cols = c->tri_cols;
    fp.geom32 = c->geom32;
    fp.max_rows = p.tri_rows;
    const int nch = (int)p.cb.size() - 1;
    auto fill = [&](int job0, const int *prefix, int njobs, int tiles, cudaStream_t st) -> int {
        if (p.tri)
            return launch_tri_fill(c->mesh, fp, p.d_gfill + job0, prefix, njobs, tiles, st);
        return launch_fill(c->mesh, fp, p.d_fill + job0, prefix, njobs, tiles, c->flags.as<int>(), st);
    };
    auto pinv_est = [&](int b0, int cnt, const SvdPlan &plan, const int *idx, int ptiles,
                        cudaStream_t st, cudaEvent_t between) -> int {
        if (o.precision == PSKEL_C64)
            gather_core_kernel<float2><<<cnt, 256, 0, st>>>(p.d_works + b0);
        else
            gather_core_kernel<double2><<<cnt, 256, 0, st>>>(p.d_works + b0);
        PSKEL_LAUNCHED(1);
        PSKEL_TRY(svd_launch(p.d_svd, idx, plan, 60, st, &c->svd_par));
        PSKEL_TRY(batched_pinv(p.d_pinv + b0, cnt, ptiles, st));
        if (between) PSKEL_CUDA(cudaEventRecord(between, st));
        int rmax = 0, pemax = 0, pcmax = 0;
        for (int i = b0; i < b0 + cnt; ++i) {
            rmax = std::max(rmax, p.r[i]);
            pemax = std::max(pemax, p.pe[i]);
            pcmax = std::max(pcmax, p.pc[i]);
        }
        return launch_estimate(p.d_est + b0, cnt, o.precision, rmax, pemax, pcmax, st);
    };
    const RoundOut *outs = c->arenas[p.round].outs.as<RoundOut>();
    auto collect = [&](int b0, int cnt, cudaStream_t st) -> int {
        collect_kernel<<<(cnt + 255) / 256, 256, 0, st>>>(p.d_works + b0, p.d_svd + b0, cnt,
                                                          c->arenas[p.round].outs.as<RoundOut>() + b0);
        PSKEL_LAUNCHED(1);
        return PSKEL_OK;
    };
    // the re-check of chunk k's blocks accepted with little margin, selected on the device from
    // their estimates: every candidate's launches are planned, the unselected return at once
    auto verify = [&](int k, cudaStream_t st) -> int {
        const int v0 = p.vc[k], cnt = p.vc[k + 1] - v0;
        if (cnt <= 0) return PSKEL_OK;
        verify_select_kernel<<<(cnt + 255) / 256, 256, 0, st>>>(p.d_vidx + v0, cnt, outs, p.v_hi, p.v_lo,
                                                                p.d_gates + v0);
        PSKEL_LAUNCHED(1);
        verify_sample_kernel<<<cnt, 128, 0, st>>>(p.d_vworks + v0, o.seed);
        PSKEL_LAUNCHED(1);
        const int j0 = p.vj[k], nj = p.vj[k + 1] - j0;
        if (p.vch_tiles[k] > 0) {
            FillParams vf = fp;
            vf.persistent = false;  // one CTA per tile: the tiles of unselected blocks retire at once
            vf.max_rows = p.vtri_rows;
            vf.gates = p.d_vjgate + j0;
            if (p.tri)
                PSKEL_TRY(launch_tri_fill(c->mesh, vf, p.d_vgfill + j0, p.vch_prefix[k], nj, p.vch_tiles[k], st));
            else
                PSKEL_TRY(launch_fill(c->mesh, vf, p.d_vfill + j0, p.vch_prefix[k], nj, p.vch_tiles[k],
                                      c->flags.as<int>(), st));
        }
        return launch_estimate(p.d_vest + v0, cnt, o.precision, p.vrmax, p.vpemax, p.vpcmax, st);
    };
    if (nch <= 1) {
        PSKEL_TRY(fill(0, p.d_fill_prefix, p.fill_jobs, p.fill_tiles, s));
        if (events) PSKEL_CUDA(cudaEventRecord(c->ev[2], s));
        PSKEL_TRY(pinv_est(0, p.nb, p.svd, p.d_svd_idx, p.pinv_tiles, s, events ? c->ev[3] : nullptr));
        PSKEL_TRY(collect(0, p.nb, s));
        if (p.nv > 0) PSKEL_TRY(verify(0, s));
    } else {
        cudaStream_t s2 = c->pipe_stream;
        fp.persistent = false;
        for (int k = 0; k < nch; ++k) {
            const int b0 = p.cb[k], cnt = p.cb[k + 1] - b0;
            PSKEL_TRY(fill(2 * b0, p.ch_prefix[k], 2 * cnt, p.ch_tiles[k], s));
            PSKEL_CUDA(cudaEventRecord(c->pipe_ev[k], s));
            PSKEL_CUDA(cudaStreamWaitEvent(s2, c->pipe_ev[k], 0));
            PSKEL_TRY(pinv_est(b0, cnt, p.ch_svd[k], p.ch_idx[k], p.ch_pinv_tiles[k], s2, nullptr));
            PSKEL_TRY(collect(b0, cnt, s2));
            PSKEL_CUDA(cudaEventRecord(c->chunk_ev[k], s2));
        }
        if (events) PSKEL_CUDA(cudaEventRecord(c->ev[2], s));  // the last fill
        // chunk k's re-check on the context's stream, beside the later chunks' SVD, pinv and
        // estimate on the pipeline stream
        if (p.nv > 0)
            for (int k = 0; k < nch; ++k) {
                PSKEL_CUDA(cudaStreamWaitEvent(s, c->chunk_ev[k], 0));
                PSKEL_TRY(verify(k, s));
            }
        PSKEL_CUDA(cudaEventRecord(c->pipe_ev[pskel_ctx::kMaxChunks], s2));
        PSKEL_CUDA(cudaStreamWaitEvent(s, c->pipe_ev[pskel_ctx::kMaxChunks], 0));
        if (events) PSKEL_CUDA(cudaEventRecord(c->ev[3], s));  // the last chunk's pinv and estimate
    }
    // (pipelined: ev[1..2] = the fills with the earlier chunks' pinv and estimate beside them,
    // ev[2..3] = the last chunk's pinv, estimate and the re-checks, ev[3..4] = nothing)
    if (events) PSKEL_CUDA(cudaEventRecord(c->ev[4], s));
    return PSKEL_OK;
}

int set_kernel_attrs() { return ensure_smem_attr(sample_kernel, sample_smem()); }

// Relative error from pooled residual sums (rows num, den, cols num, den): the larger side.
double pooled_est(const double *a, const double *b) {
    const double nr = a[0] + b[0], dr = a[1] + b[1], nc = a[2] + b[2], dc = a[3] + b[3];
    const double er = dr > 0 ? std::sqrt(nr / dr) : 0.0;
    const double ec = dc > 0 ? std::sqrt(nc / dc) : 0.0;
    return std::max(er, ec);
}

}  // namespace

extern "C" int pskel_create(pskel_ctx **out, int device) {
    if (!out) {
        set_error(PSKEL_ERR_ARG, "null output pointer");
        return PSKEL_ERR_ARG;
    }
    pskel_ctx *c = new pskel_ctx();
    c->device = device;
    auto fail = [&](int st) { delete c; return st; };
    if (cudaSetDevice(device) != cudaSuccess) {
        set_error(PSKEL_ERR_CUDA, "cudaSetDevice(%d) failed", device);
        return fail(PSKEL_ERR_CUDA);
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error(PSKEL_ERR_CUDA, "stream creation failed");
        return fail(PSKEL_ERR_CUDA);
    }
    for (auto &e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            set_error(PSKEL_ERR_CUDA, "event creation failed");
            return fail(PSKEL_ERR_CUDA);
        }
    int lo_pri = 0, hi_pri = 0;
    cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri);
    if (cudaStreamCreateWithPriority(&c->pipe_stream, cudaStreamNonBlocking, hi_pri) != cudaSuccess) {
        set_error(PSKEL_ERR_CUDA, "stream creation failed");
        return fail(PSKEL_ERR_CUDA);
    }
    for (auto &e : c->chunk_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            set_error(PSKEL_ERR_CUDA, "event creation failed");
            return fail(PSKEL_ERR_CUDA);
        }
    for (auto &e : c->pipe_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            set_error(PSKEL_ERR_CUDA, "event creation failed");
            return fail(PSKEL_ERR_CUDA);
        }
    int st = c->flags.reserve(256);
    if (st != PSKEL_OK) return fail(st);
    st = svd_streams_create(c->svd_par);
    if (st != PSKEL_OK) return fail(st);
    cudaMemsetAsync(c->flags.ptr, 0, 256, c->stream);
    *out = c;
    return PSKEL_OK;
}

extern "C" int pskel_destroy(pskel_ctx *c) {
    if (!c) return PSKEL_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->pipe_stream) cudaStreamSynchronize(c->pipe_stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    c->mesh.vertex.release(); c->mesh.topol.release(); c->mesh.edges.release();
    c->mesh.ln.release(); c->mesh.cent.release();
    c->mesh.rec1.f64.release();
    c->mesh.rec7.f64.release();
    c->flags.release(); c->d_gids.release();
    c->tmp.release(); c->tmp2.release(); c->tmp3.release(); c->recomp.release(); c->recomp64.release(); c->recomp64b.release(); c->rc_work.release(); c->rc_tab.release(); c->rc_idx.release(); c->rc_host.release(); c->plan_host.release(); c->mv_table.release();
    for (DevBuf *d : {&c->st_ah, &c->st_al, &c->st_bh, &c->st_bl, &c->st_t, &c->st_tab, &c->st_tiles, &c->st_err}) d->release();
    for (auto &a : c->arenas) { a.keep.release(); a.work.release(); a.tables.release(); a.outs.release(); }
    svd_streams_destroy(c->svd_par);
    octree_release(c->octree);
    c->near_jobs.release(); c->near_mom.release(); c->near_data.release(); c->near_tab.release();
    c->aca_buf.release(); c->aca_tab.release();
    for (auto &e : c->pipe_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->chunk_ev)
        if (e) cudaEventDestroy(e);
    if (c->pipe_stream) cudaStreamDestroy(c->pipe_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PSKEL_OK;
}

extern "C" int pskel_upload_mesh(pskel_ctx *c, const double *vertex, int nv, const double *topol,
                                 int nt, const double *edges, int ne, const double *ln,
                                 const double *cent, const pskel_em_t *em) {
    PSKEL_TRY(ctx_ok(c));
    if (!em || em->k <= 0 || (em->q_test != 1 && em->q_test != 7) || em->q_src != em->q_test) {
        set_error(PSKEL_ERR_ARG, "em: k > 0 and q_test == q_src in {1, 7} required");
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(upload_mesh_arrays(c->mesh, vertex, nv, topol, nt, edges, ne, ln, cent, c->stream));
    PSKEL_CUDA(cudaMemsetAsync(c->flags.ptr, 0, 256, c->stream));
    PSKEL_TRY(build_records(c->mesh, em->q_test, c->stream, c->flags.as<int>()));
    int h = 0;
    PSKEL_CUDA(cudaMemcpyAsync(&h, c->flags.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    if (h & 2) {
        set_error(PSKEL_ERR_RANGE, "mesh: triangle or vertex id out of range");
        return PSKEL_ERR_RANGE;
    }
    c->h_edges.resize(4 * (size_t)ne);
    for (size_t i = 0; i < 4 * (size_t)ne; ++i) c->h_edges[i] = (int)edges[i] - 1;
    c->h_vertex.assign(vertex, vertex + 3 * (size_t)nv);
    c->h_ln.assign(ln, ln + ne);
    c->h_cent.assign(cent, cent + 3 * (size_t)nt);
    c->em = *em;
    c->have_mesh = true;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
        c->graph_key.clear();
    }
    return PSKEL_OK;
}

extern "C" int pskel_fill_device(pskel_ctx *c, const int *rows_dev, int nr, const int *cols_dev,
                                 int nc, void *Z_dev, int ld, int precision) {
    PSKEL_TRY(ctx_ok(c));
    if (!c->have_mesh) {
        set_error(PSKEL_ERR_STATE, "no mesh uploaded");
        return PSKEL_ERR_STATE;
    }
    if (nr < 0 || nc < 0 || ld < nr || (precision != PSKEL_C128 && precision != PSKEL_C64)) {
        set_error(PSKEL_ERR_ARG, "fill: nr=%d nc=%d ld=%d precision=%d", nr, nc, ld, precision);
        return PSKEL_ERR_ARG;
    }
    if ((size_t)nr * nc == 0) return PSKEL_OK;
    int tm, tn;
    fill_tile_shape(precision, c->em.q_test, entry_split_for(c, precision), &tm, &tn);
    FillJob job{rows_dev, cols_dev, Z_dev, nr, nc, ld, 0};
    int prefix[2] = {0, ((nr + tm - 1) / tm) * ((nc + tn - 1) / tn)};
    PSKEL_TRY(c->tmp3.reserve(512));
    PSKEL_CUDA(cudaMemcpyAsync(c->tmp3.ptr, &job, sizeof(job), cudaMemcpyHostToDevice, c->stream));
    PSKEL_CUDA(cudaMemcpyAsync(c->tmp3.as<char>() + 256, prefix, sizeof(prefix),
                               cudaMemcpyHostToDevice, c->stream));
    FillParams fp;
    fp.k = c->em.k;
    fp.eta = c->em.eta;
    fp.r_near = 0;
    fp.q_test = c->em.q_test;
    fp.q_src = c->em.q_src;
    fp.precision = precision;
    fp.split = entry_split_for(c, precision);
    return launch_fill(c->mesh, fp, c->tmp3.as<FillJob>(),
                       reinterpret_cast<int *>(c->tmp3.as<char>() + 256), 1, prefix[1],
                       c->flags.as<int>(), c->stream);
}

extern "C" int pskel_set_blocks(pskel_ctx *c, const int *group_ptr, const int *group_ids,
                                int n_groups, const int *gt, const int *gs, int n_blocks) {
    PSKEL_TRY(ctx_ok(c));
    if (!c->have_mesh || !group_ptr || !group_ids || n_groups <= 0 || n_blocks < 0 ||
        (n_blocks > 0 && (!gt || !gs))) {
        set_error(PSKEL_ERR_ARG, "set_blocks: bad arguments (mesh uploaded: %d)", (int)c->have_mesh);
        return PSKEL_ERR_ARG;
    }
    const int nids = group_ptr[n_groups];
    if (group_ptr[0] != 0 || nids <= 0) {
        set_error(PSKEL_ERR_ARG, "set_blocks: group_ptr must start at 0 and be non-empty");
        return PSKEL_ERR_ARG;
    }
    for (int g = 0; g < n_groups; ++g) {
        const int sz = group_ptr[g + 1] - group_ptr[g];
        if (sz <= 0 || sz > kMaxGroup) {
            set_error(PSKEL_ERR_ARG, "group %d has %d members (1..%d allowed)", g, sz, kMaxGroup);
            return PSKEL_ERR_ARG;
        }
    }
    for (int i = 0; i < nids; ++i)
        if (group_ids[i] < 0 || group_ids[i] >= c->mesh.ne) {
            set_error(PSKEL_ERR_RANGE, "group id %d out of range", group_ids[i]);
            return PSKEL_ERR_RANGE;
        }
    for (int b = 0; b < n_blocks; ++b)
        if (gt[b] < 0 || gt[b] >= n_groups || gs[b] < 0 || gs[b] >= n_groups) {
            set_error(PSKEL_ERR_RANGE, "block %d refers to a missing group", b);
            return PSKEL_ERR_RANGE;
        }
    c->gptr.assign(group_ptr, group_ptr + n_groups + 1);
    c->gids.assign(group_ids, group_ids + nids);
    c->gt.assign(gt, gt + n_blocks);
    c->gs.assign(gs, gs + n_blocks);
    c->n_groups = n_groups;
    c->n_blocks = n_blocks;
    {  // the block with swapped groups, for the symmetric mode (the last block listed for a pair)
        c->partner.assign(n_blocks, -1);
        const long long G = n_groups;
        if (G * G <= (1LL << 24)) {  // dense group-pair table
            std::vector<int> where((size_t)(G * G), -1);
            for (int b = 0; b < n_blocks; ++b) where[(size_t)(gt[b] * G + gs[b])] = b;
            for (int b = 0; b < n_blocks; ++b) {
                const int p = where[(size_t)(gs[b] * G + gt[b])];
                if (p >= 0 && p != b) c->partner[b] = p;
            }
        } else {  // sorted keys
            std::vector<std::pair<long long, int>> keys(n_blocks);
            for (int b = 0; b < n_blocks; ++b) keys[b] = {gt[b] * G + gs[b], b};
            std::stable_sort(keys.begin(), keys.end(),
                             [](const std::pair<long long, int> &a, const std::pair<long long, int> &b) {
                                 return a.first < b.first;
                             });
            for (int b = 0; b < n_blocks; ++b) {
                const long long want = gs[b] * G + gt[b];
                auto it = std::upper_bound(keys.begin(), keys.end(), want,
                                           [](long long v, const std::pair<long long, int> &e) { return v < e.first; });
                if (it != keys.begin() && (it - 1)->first == want && (it - 1)->second != b)
                    c->partner[b] = (it - 1)->second;
            }
        }
    }
    PSKEL_TRY(c->d_gids.reserve(sizeof(int) * nids));
    PSKEL_CUDA(cudaMemcpyAsync(c->d_gids.ptr, group_ids, sizeof(int) * nids, cudaMemcpyHostToDevice,
                               c->stream));
    // triangles of each group and, per triangle, the (local RWG, side) pairs that use it
    {
        std::vector<int> tri, adj;
        c->gtri_ptr.assign(n_groups + 1, 0);
        int max_rows = 0;
        std::vector<int> local(c->mesh.nt, -1);
        for (int g = 0; g < n_groups; ++g) {
            const int b0 = group_ptr[g], b1 = group_ptr[g + 1];
            max_rows = std::max(max_rows, b1 - b0);
            const size_t t0 = tri.size();
            for (int i = b0; i < b1; ++i)
                for (int side = 0; side < 2; ++side) {
                    const int t = c->h_edges[4 * (size_t)group_ids[i] + side];
                    if (t < 0 || t >= c->mesh.nt) {
                        set_error(PSKEL_ERR_RANGE, "edges: triangle id out of range");
                        return PSKEL_ERR_RANGE;
                    }
                    if (local[t] < 0) {
                        local[t] = (int)(tri.size() - t0);
                        tri.push_back(t);
                        adj.insert(adj.end(), {-1, -1, -1});
                    }
                    int *a = &adj[3 * (t0 + local[t])];
                    int u = 0;
                    while (u < 3 && a[u] >= 0) ++u;
                    if (u == 3) {
                        set_error(PSKEL_ERR_ARG, "triangle %d is used by more than three RWG", t);
                        return PSKEL_ERR_ARG;
                    }
                    a[u] = 2 * (i - b0) + side;
                }
            for (size_t q = t0; q < tri.size(); ++q) local[tri[q]] = -1;
            c->gtri_ptr[g + 1] = (int)tri.size();
        }
        c->use_tri = max_rows <= kTriFillMaxRows;
        // per (triangle, slot) of each group: the RWG's free vertex minus the triangle centroid
        // and the signed edge length, the numbers the fill's per-item scatter needs (looked up
        // here once instead of through dependent loads in every item)
        std::vector<double> use(12 * tri.size(), 0.0);
        for (int g = 0; g < n_groups; ++g)
            for (int sl = c->gtri_ptr[g]; sl < c->gtri_ptr[g + 1]; ++sl)
                for (int u = 0; u < 3; ++u) {
                    const int a = adj[3 * (size_t)sl + u];
                    if (a < 0) continue;
                    const int ml = a >> 1, side = a & 1;
                    const int e = group_ids[group_ptr[g] + ml], t = tri[sl];
                    const int vo = c->h_edges[4 * (size_t)e + 2 + side];
                    if (vo < 0 || 3 * (size_t)vo + 2 >= c->h_vertex.size()) {
                        set_error(PSKEL_ERR_RANGE, "edges: vertex id out of range");
                        return PSKEL_ERR_RANGE;
                    }
                    double *o = &use[12 * (size_t)sl + 4 * u];
                    for (int d = 0; d < 3; ++d)
                        o[d] = c->h_vertex[3 * (size_t)vo + d] - c->h_cent[3 * (size_t)t + d];
                    o[3] = (side ? -1.0 : 1.0) * c->h_ln[e];
                }
        PSKEL_TRY(c->d_guse.reserve(sizeof(double) * (use.size() + 1)));
        PSKEL_CUDA(cudaMemcpyAsync(c->d_guse.ptr, use.data(), sizeof(double) * use.size(),
                                   cudaMemcpyHostToDevice, c->stream));
        PSKEL_TRY(c->d_gtri.reserve(sizeof(int) * (tri.size() + 1)));
        PSKEL_TRY(c->d_gadj.reserve(sizeof(int) * (adj.size() + 1)));
        PSKEL_CUDA(cudaMemcpyAsync(c->d_gtri.ptr, tri.data(), sizeof(int) * tri.size(),
                                   cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(c->d_gadj.ptr, adj.data(), sizeof(int) * adj.size(),
                                   cudaMemcpyHostToDevice, c->stream));
    }
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    c->results.assign(n_blocks, BlockResult());
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
        c->graph_key.clear();
    }
    return PSKEL_OK;
}

extern "C" int pskel_compress_blocks(pskel_ctx *c, const pskel_opts_t *opts, const int *r0,
                                     pskel_block_stat_t *stats) {
    PSKEL_TRY(ctx_ok(c));
    if (!opts || !c->have_mesh || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_STATE, "compress: options, mesh and blocks are required");
        return PSKEL_ERR_STATE;
    }
    const pskel_opts_t o = *opts;
    if (!(o.tol > 0) || o.tau < 0 || o.full_tau < 0 || (o.precision != PSKEL_C128 && o.precision != PSKEL_C64) ||
        o.extra_rows < 0 || o.extra_rows > kMaxExtra || o.extra_cols < 0 ||
        o.extra_cols > kMaxExtra || o.max_rounds < 1 ||
        (o.start == PSKEL_START_GIVEN && !r0)) {
        set_error(PSKEL_ERR_ARG, "compress: bad options");
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(set_kernel_attrs());
    const double safety = o.est_safety >= 1.0 ? o.est_safety : 1.0;
    c->precision = o.precision;
    ++c->generation;
    c->recomp_slots.clear();
    for (double &t : c->timing) t = 0;
    const int nb = c->n_blocks;
    // first sample counts
    std::vector<int> r_cur(nb), Dmin(nb), mrows(nb), ncols(nb);
    for (int b = 0; b < nb; ++b) {
        const int m = c->gptr[c->gt[b] + 1] - c->gptr[c->gt[b]];
        const int n = c->gptr[c->gs[b] + 1] - c->gptr[c->gs[b]];
        const int D = std::min(m, n);
        Dmin[b] = D;
        mrows[b] = m;
        ncols[b] = n;
        int r;
        if (o.start == PSKEL_START_GIVEN) r = r0[b] + o.oversample;
        else r = D < 10 ? 1 : D / 10;
        r_cur[b] = std::max(1, std::min(r, D));
    }
    std::vector<int> rounds_used(nb, 0);
    cudaEvent_t t0, t1;
    PSKEL_CUDA(cudaEventCreate(&t0));
    PSKEL_CUDA(cudaEventCreate(&t1));
    PSKEL_CUDA(cudaEventRecord(t0, c->stream));
    std::vector<RoundOut> hout;
    std::vector<char> hbuf;
    // rounds of an active set until every block of it is done
    auto run_rounds = [&](std::vector<int> active, bool allow_graph) -> int {
    int round = 0;
    while (!active.empty()) {
        RoundPlan p;
        p.round = round;
        p.blocks = active;
        p.r.resize(active.size());
        p.pe.resize(active.size());
        p.pc.resize(active.size());
        for (size_t i = 0; i < active.size(); ++i) {
            const int b = active[i];
            p.r[i] = r_cur[b];
            p.pe[i] = std::min(o.extra_rows, mrows[b] - r_cur[b]);
            p.pc[i] = std::min(o.extra_cols, ncols[b] - r_cur[b]);
        }
        // blocks whose estimate may pass with little margin (est within a factor est_verify of
        // the acceptance threshold) are re-checked on fresh extra rows and columns, inside the
        // round; candidates are the blocks that could still go on to another round
        if (o.est_verify > 1.0) {
            p.v_hi = o.tol / safety;
            p.v_lo = o.tol / (safety * o.est_verify);
            for (size_t i = 0; i < active.size(); ++i) {
                const int b = active[i];
                const bool more = mrows[b] - p.r[i] - p.pe[i] > 0 || ncols[b] - p.r[i] - p.pc[i] > 0;
                if (more && r_cur[b] < Dmin[b] && round + 1 < o.max_rounds) p.vcand.push_back((int)i);
            }
        }
        const int nv = (int)p.vcand.size();
        {
            double ent = 0;
            for (size_t i = 0; i < active.size(); ++i) {
                const int b = active[i];
                ent += (double)mrows[b] * (p.r[i] + p.pc[i]) + (double)(p.r[i] + p.pe[i]) * ncols[b];
            }
            const double q2 = 4.0 * c->em.q_test * c->em.q_src;
            c->timing[6] += ent;
            c->timing[7] += ent * q2;
            c->timing[8] += 1;
            c->timing[9] += 1;
        }
        // graph of the first round: key = the sample counts and options that shape it
        bool try_graph = allow_graph && o.use_graph && round == 0;
        std::vector<int> key;
        if (try_graph) {
            key = p.r;
            key.push_back(o.precision);
            key.push_back((int)(o.seed & 0x7fffffff));
            key.push_back(o.extra_rows);
            key.push_back(o.extra_cols);
            key.push_back((int)std::lround(std::log10(std::max(o.tau, 1e-300)) * 1000));
            key.push_back(o.tau_relative);
            key.push_back(c->split[0] * 8 + c->split[1] + (c->use_tri ? 1000 : 0));
            key.push_back(c->tri_cols + 100 * c->geom32);
            key.push_back(c->pipe_chunks);
            key.push_back(o.max_rounds);
            for (double x : {p.v_hi, p.v_lo}) {  // the re-check's thresholds, bit for bit
                int h[2];
                std::memcpy(h, &x, sizeof(h));
                key.push_back(h[0]);
                key.push_back(h[1]);
            }
            // capture only when the same first round ran eagerly before (warm, attributes set)
            const bool seen = key == c->last_key || (c->graph && key == c->graph_key);
            c->last_key = key;
            try_graph = seen;
        }
        if (try_graph && c->graph && key == c->graph_key) {
            // tables and arenas from the capturing call are still in place: replay
            for (size_t i = 0; i < active.size(); ++i) c->results[active[i]] = c->graph_results[active[i]];
            PSKEL_CUDA(cudaEventRecord(c->ev[0], c->stream));
            PSKEL_CUDA(cudaGraphLaunch(c->graph, c->stream));
            count_launch(c->graph_kernels);
            PSKEL_CUDA(cudaEventRecord(c->ev[4], c->stream));
        } else {
            if (round == 0 && c->graph) {
                // a new round-0 plan may move the buffers a captured graph points into
                cudaGraphExecDestroy(c->graph);
                c->graph = nullptr;
                c->graph_key.clear();
            }
            PSKEL_TRY(plan_round(c, p, o));
            if (try_graph) {
                if (c->graph) {
                    cudaGraphExecDestroy(c->graph);
                    c->graph = nullptr;
                }
                PSKEL_CUDA(cudaStreamSynchronize(c->stream));
                cudaGraph_t g;
                PSKEL_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                const long long before = launches_so_far();
                int st = launch_round(c, p, o, false);
                c->graph_kernels = launches_so_far() - before;
                count_launch(-c->graph_kernels);  // captured, not run
                cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
                if (st != PSKEL_OK) return st;
                if (ce != cudaSuccess) {
                    set_error(PSKEL_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
                    return PSKEL_ERR_CUDA;
                }
                PSKEL_CUDA(cudaGraphInstantiate(&c->graph, g, 0));
                cudaGraphDestroy(g);
                c->graph_key = key;
                c->graph_results = c->results;
                PSKEL_CUDA(cudaEventRecord(c->ev[0], c->stream));
                PSKEL_CUDA(cudaGraphLaunch(c->graph, c->stream));
                count_launch(c->graph_kernels);
                PSKEL_CUDA(cudaEventRecord(c->ev[4], c->stream));
            } else {
                PSKEL_TRY(launch_round(c, p, o, true));
            }
        }
        // the round's outcome, the re-checks' sums and gates in one read-back
        const int na = (int)active.size();
        hbuf.resize(outs_bytes(na, nv));
        PSKEL_CUDA(cudaMemcpyAsync(hbuf.data(), c->arenas[round].outs.ptr, hbuf.size(), cudaMemcpyDeviceToHost,
                                   c->stream));
        PSKEL_CUDA(cudaStreamSynchronize(c->stream));
        hout.resize(na);
        std::memcpy(hout.data(), hbuf.data(), sizeof(RoundOut) * na);
        const double *vouts = reinterpret_cast<const double *>(hbuf.data() + outs_vouts_offset(na));
        const int *gates = reinterpret_cast<const int *>(hbuf.data() + outs_gates_offset(na, nv));
        {
            float ms = 0;
            const bool per_phase = !(try_graph);
            if (per_phase) {
                for (int k = 0; k < 4; ++k) {
                    cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]);
                    c->timing[k] += ms;
                }
            } else {
                cudaEventElapsedTime(&ms, c->ev[0], c->ev[4]);
                c->timing[1] += ms;  // graph replays are not split by phase
            }
        }
        // the re-checked blocks pass on the estimate pooled over both sample sets
        std::vector<double> est(na);
        for (int i = 0; i < na; ++i) est[i] = hout[i].est;
        {
            double ent = 0;
            for (int v = 0; v < nv; ++v) {
                if (!gates[v]) continue;
                const int i = p.vcand[v], b = active[i];
                int pe2, pc2;
                verify_extent(mrows[b], ncols[b], p.r[i], p.pe[i], p.pc[i], o, &pe2, &pc2);
                ent += (double)mrows[b] * pc2 + (double)pe2 * ncols[b];
                est[i] = pooled_est(hout[i].sums, vouts + 8 * (size_t)v + 1);
            }
            if (ent > 0) {
                c->timing[6] += ent;
                c->timing[7] += ent * 4.0 * c->em.q_test * c->em.q_src;
                c->timing[8] += 1;
            }
        }
        std::vector<int> next;
        for (size_t i = 0; i < active.size(); ++i) {
            const int b = active[i];
            BlockResult &res = c->results[b];
            res.est = est[i];
            res.rank = hout[i].rank;
            res.status = hout[i].status;
            c->timing[10] += hout[i].sweeps;
            c->timing[11] = std::max(c->timing[11], (double)hout[i].sweeps);
            c->timing[12] += 1;
            rounds_used[b] = round + 1;
            const bool ok = hout[i].status == PSKEL_OK && est[i] <= o.tol / safety;
            if (ok || r_cur[b] >= Dmin[b] || round + 1 >= o.max_rounds) continue;
            r_cur[b] = std::min(std::max(r_cur[b] + 1, (int)std::ceil(c->growth * r_cur[b])), Dmin[b]);
            next.push_back(b);
        }
        active.swap(next);
        ++round;
    }
    return PSKEL_OK;
    };
    for (int b = 0; b < nb; ++b) c->results[b].mirror = -1;
    if (o.per_block) {
        for (int b = 0; b < nb; ++b) PSKEL_TRY(run_rounds(std::vector<int>{b}, false));
        // each block reused the round arenas: only the last block's factors are still there
        for (int b = 0; b + 1 < nb; ++b) c->results[b].arena = -1;
    } else {
        // symmetric mode: the block of a (t, s) / (s, t) pair with the smaller index is compressed,
        // the other takes its transpose (Z(s, t) = Z(t, s)^T for a Galerkin EFIE matrix)
        const bool sym = c->symmetric != 0;
        std::vector<int> all;
        all.reserve(nb);
        for (int b = 0; b < nb; ++b)
            if (!sym || c->partner[b] < 0 || b < c->partner[b]) all.push_back(b);
        PSKEL_TRY(run_rounds(all, true));
        if (sym)
            for (int b = 0; b < nb; ++b) {
                const int pb = c->partner[b];
                if (pb < 0 || b < pb) continue;
                BlockResult res = c->results[pb];
                res.mirror = pb;
                res.m = c->results[pb].n;
                res.n = c->results[pb].m;
                c->results[b] = res;
                rounds_used[b] = rounds_used[pb];
            }
    }
    PSKEL_CUDA(cudaEventRecord(t1, c->stream));
    PSKEL_CUDA(cudaEventSynchronize(t1));
    float total = 0;
    cudaEventElapsedTime(&total, t0, t1);
    c->timing[5] = total;
    if (c->timing[12] > 0) c->timing[10] /= c->timing[12];
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    int h = 0;
    PSKEL_CUDA(cudaMemcpy(&h, c->flags.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (h & 6) {
        set_error(PSKEL_ERR_RANGE, "an id was out of range during the fill");
        return PSKEL_ERR_RANGE;
    }
    // per-block statuses are reported in stats (the call itself succeeds)
    for (int b = 0; b < nb; ++b) {
        const BlockResult &res = c->results[b];
        if (stats) {
            pskel_block_stat_t &s = stats[b];
            s.m = res.m;
            s.n = res.n;
            s.r = res.r;
            s.rank = res.rank;
            s.rank_recompressed = 0;
            s.rounds = rounds_used[b];
            s.status = res.status;
            s.est = res.est;
        }
    }
    return PSKEL_OK;
}

extern "C" int pskel_set_fill_split(pskel_ctx *c, int split_c128, int split_c64) {
    PSKEL_TRY(ctx_ok(c));
    auto ok = [](int v) { return v == -1 || v == 0 || v == 1 || v == 2 || v == 4 || v == 8; };
    if (!ok(split_c128) || !ok(split_c64)) {
        set_error(PSKEL_ERR_ARG, "fill variant must be -1 (unchanged), 0, 1, 2, 4 or 8");
        return PSKEL_ERR_ARG;
    }
    if (split_c128 >= 0) c->split[0] = split_c128;
    if (split_c64 >= 0) c->split[1] = split_c64;
    return PSKEL_OK;
}

extern "C" int pskel_set_tri_cols(pskel_ctx *c, int cols) {
    PSKEL_TRY(ctx_ok(c));
    if (cols != 0 && cols != 4 && cols != 8 && cols != 16) {
        set_error(PSKEL_ERR_ARG, "triangle-moment fill: %d columns per tile (0 = balanced, 4, 8 or 16)", cols);
        return PSKEL_ERR_ARG;
    }
    c->tri_cols = cols;
    return PSKEL_OK;
}

extern "C" int pskel_set_round_growth(pskel_ctx *c, double factor) {
    if (!c || !(factor > 1.0 && factor <= 4.0)) {
        set_error(PSKEL_ERR_ARG, "set_round_growth: factor must be in (1, 4]");
        return PSKEL_ERR_ARG;
    }
    c->growth = factor;
    return PSKEL_OK;
}

extern "C" int pskel_set_pipeline(pskel_ctx *c, int chunks) {
    PSKEL_TRY(ctx_ok(c));
    if (chunks < 1 || chunks > pskel_ctx::kMaxChunks) {
        set_error(PSKEL_ERR_ARG, "pipeline chunks must be 1 .. %d", pskel_ctx::kMaxChunks);
        return PSKEL_ERR_ARG;
    }
    c->pipe_chunks = chunks;
    return PSKEL_OK;
}

extern "C" int pskel_set_symmetric(pskel_ctx *c, int on) {
    PSKEL_TRY(ctx_ok(c));
    if (on != 0 && on != 1) {
        set_error(PSKEL_ERR_ARG, "symmetric: 0 or 1");
        return PSKEL_ERR_ARG;
    }
    c->symmetric = on;
    return PSKEL_OK;
}

extern "C" int pskel_set_fill_geometry(pskel_ctx *c, int fp32_offsets) {
    PSKEL_TRY(ctx_ok(c));
    if (fp32_offsets != 0 && fp32_offsets != 1) {
        set_error(PSKEL_ERR_ARG, "fill geometry: 0 (FP64) or 1 (FP32 offsets)");
        return PSKEL_ERR_ARG;
    }
    c->geom32 = fp32_offsets;
    return PSKEL_OK;
}

extern "C" int pskel_last_timing(pskel_ctx *c, double *out, int n) {
    PSKEL_TRY(ctx_ok(c));
    if (!out || n < 0) {
        set_error(PSKEL_ERR_ARG, "null output");
        return PSKEL_ERR_ARG;
    }
    for (int i = 0; i < n && i < 12; ++i) out[i] = c->timing[i];
    return PSKEL_OK;
}

extern "C" int pskel_get_block(pskel_ctx *c, int b, pskel_c128 *C, pskel_c128 *U, pskel_c128 *R,
                               int *I, int *J) {
    PSKEL_TRY(ctx_ok(c));
    if (b < 0 || b >= c->n_blocks || c->results[b].arena < 0) {
        set_error(PSKEL_ERR_ARG, "block %d has no result", b);
        return PSKEL_ERR_ARG;
    }
    const BlockResult &res = c->results[b];
    if (res.mirror >= 0) {
        // the transpose of the primary's factors: C = R_p^T, U = U_p^T, R = C_p^T, I = J_p, J = I_p
        const size_t mb = res.m, nb_ = res.n, r = res.r;
        std::vector<pskel_c128> Cp(nb_ * r), Up(r * r), Rp(r * mb);
        std::vector<int> Ip(r), Jp(r);
        PSKEL_TRY(pskel_get_block(c, res.mirror, Cp.data(), Up.data(), Rp.data(), Ip.data(), Jp.data()));
        if (C)
            for (size_t k = 0; k < r; ++k)
                for (size_t i = 0; i < mb; ++i) C[i + k * mb] = Rp[k + i * r];
        if (U)
            for (size_t k = 0; k < r; ++k)
                for (size_t i = 0; i < r; ++i) U[i + k * r] = Up[k + i * r];
        if (R)
            for (size_t j = 0; j < nb_; ++j)
                for (size_t k = 0; k < r; ++k) R[k + j * r] = Cp[j + k * nb_];
        if (I) std::copy(Jp.begin(), Jp.end(), I);
        if (J) std::copy(Ip.begin(), Ip.end(), J);
        return PSKEL_OK;
    }
    const char *base = c->arenas[res.arena].keep.as<char>();
    const size_t m = res.m, n = res.n, r = res.r, ldr = res.r + res.pe;
    const bool f32 = c->precision == PSKEL_C64;
    const size_t es = f32 ? sizeof(float2) : sizeof(double2);
    std::vector<char> h;
    auto fetch = [&](size_t off, size_t count, pskel_c128 *dst, size_t rows, size_t ld) -> int {
        h.resize(count * es);
        PSKEL_CUDA(cudaMemcpy(h.data(), base + off, count * es, cudaMemcpyDeviceToHost));
        const size_t cols = count / ld;
        for (size_t j = 0; j < cols; ++j)
            for (size_t i = 0; i < rows; ++i) {
                const size_t src = i + j * ld;
                pskel_c128 v;
                if (f32) {
                    const float2 x = reinterpret_cast<const float2 *>(h.data())[src];
                    v.re = x.x;
                    v.im = x.y;
                } else {
                    const double2 x = reinterpret_cast<const double2 *>(h.data())[src];
                    v.re = x.x;
                    v.im = x.y;
                }
                dst[i + j * rows] = v;
            }
        return PSKEL_OK;
    };
    if (C) PSKEL_TRY(fetch(res.offC, m * r, C, m, m));
    if (R) PSKEL_TRY(fetch(res.offRx, ldr * n, R, r, ldr));
    if (U) PSKEL_CUDA(cudaMemcpy(U, base + res.offU, sizeof(double2) * r * r, cudaMemcpyDeviceToHost));
    if (I) PSKEL_CUDA(cudaMemcpy(I, base + res.offI, sizeof(int) * r, cudaMemcpyDeviceToHost));
    if (J) PSKEL_CUDA(cudaMemcpy(J, base + res.offJ, sizeof(int) * r, cudaMemcpyDeviceToHost));
    return PSKEL_OK;
}

namespace {
// ||Z_b - C_b U_b R_b||_F / ||Z_b||_F of the blocks in `list` (err[i] for list[i]), Z_b filled
// densely in complex FP64, in batches of at most 2^28 dense entries.
int true_errors_list(pskel_ctx *c, const std::vector<int> &list, double *err) {
    const int nb = (int)list.size();
    for (int b : list)
        if (c->results[b].arena < 0) {
            set_error(PSKEL_ERR_STATE, "true_errors: block %d has no retained factors (run the "
                                       "batched mode to keep every block)", b);
            return PSKEL_ERR_STATE;
        }
    const bool f32 = c->precision == PSKEL_C64;
    const size_t budget = (size_t)1 << 28;  // complex elements of dense blocks per batch
    int b0 = 0;
    while (b0 < nb) {
        // choose a batch
        size_t dense = 0, work = 0;
        int b1 = b0;
        while (b1 < nb) {
            const BlockResult &res = c->results[list[b1]];
            const BlockResult &pr = res.mirror >= 0 ? c->results[res.mirror] : res;  // factor storage
            const size_t d = (size_t)res.m * res.n;
            const size_t wsz = (size_t)res.r * res.n + (f32 ? (size_t)pr.m * pr.r + (size_t)(pr.r + pr.pe) * pr.n : 0);
            if (b1 > b0 && dense + d > budget) break;
            dense += d;
            work += wsz;
            ++b1;
        }
        const int nbb = b1 - b0;
        PSKEL_TRY(c->tmp.reserve(sizeof(double2) * (dense + work) + 256 * (size_t)(4 * nbb + 8)));
        double2 *Zb = c->tmp.as<double2>();
        double2 *Wb = Zb + dense;
        std::vector<FillJob> fills(nbb);
        std::vector<GroupFillJob> gfills(nbb);
        std::vector<ZgemmJob> g1, g2;
        std::vector<const double2 *> mats(nbb);
        std::vector<long long> sizes(nbb);
        size_t zo = 0, wo = 0;
        int tm, tn;
        fill_tile_shape(PSKEL_C128, c->em.q_test, entry_split_for(c, PSKEL_C128), &tm, &tn);
        const bool tri = tri_for(c, PSKEL_C128);
        std::vector<int> prefix(nbb + 1, 0);
        for (int i = 0; i < nbb; ++i) {
            const int b = list[b0 + i];
            const BlockResult &res = c->results[b];
            const char *base = c->arenas[res.arena].keep.as<char>();
            double2 *Z = Zb + zo;
            fills[i] = FillJob{c->d_gids.as<int>() + c->gptr[c->gt[b]],
                               c->d_gids.as<int>() + c->gptr[c->gs[b]], Z, res.m, res.n, res.m, 0};
            const int gt = c->gt[b];
            gfills[i] = GroupFillJob{c->d_gids.as<int>() + c->gptr[gt],
                                     c->d_gtri.as<int>() + c->gtri_ptr[gt],
                                     c->d_gadj.as<int>() + 3 * (size_t)c->gtri_ptr[gt],
                                     c->d_gids.as<int>() + c->gptr[c->gs[b]], Z, res.m,
                                     c->gtri_ptr[gt + 1] - c->gtri_ptr[gt], res.n, res.m, 0,
                                     tri_cols_for(c, c->gtri_ptr[gt + 1] - c->gtri_ptr[gt]),
                                     guse_of(c, gt)};
            prefix[i + 1] = prefix[i] + (tri ? (res.n + gfills[i].tc - 1) / gfills[i].tc
                                                     : ((res.m + tm - 1) / tm) * ((res.n + tn - 1) / tn));
            mats[i] = Z;
            sizes[i] = (long long)res.m * res.n;
            const BlockResult &pr = res.mirror >= 0 ? c->results[res.mirror] : res;  // factor storage
            const bool mir = res.mirror >= 0;
            const double2 *Cd;
            const double2 *Rd;
            int ldr = pr.r + pr.pe;
            double2 *T = Wb + wo;
            wo += (size_t)res.r * res.n;
            if (f32) {
                double2 *Cc = Wb + wo;
                wo += (size_t)pr.m * pr.r;
                double2 *Rc = Wb + wo;
                wo += (size_t)ldr * pr.n;
                const long long nC = (long long)pr.m * pr.r, nR = (long long)ldr * pr.n;
                promote_kernel<float2><<<(unsigned)((nC + 255) / 256), 256, 0, c->stream>>>(
                    reinterpret_cast<const float2 *>(base + pr.offC), Cc, nC);
                promote_kernel<float2><<<(unsigned)((nR + 255) / 256), 256, 0, c->stream>>>(
                    reinterpret_cast<const float2 *>(base + pr.offRx), Rc, nR);
                count_launch(2);
                Cd = Cc;
                Rd = Rc;
            } else {
                Cd = reinterpret_cast<const double2 *>(base + pr.offC);
                Rd = reinterpret_cast<const double2 *>(base + pr.offRx);
            }
            const double2 *Ud = reinterpret_cast<const double2 *>(base + pr.offU);
            // Z - C U R, or for a mirror block Z - R_p^T U_p^T C_p^T
            if (!mir)
                g1.push_back(zjob(Ud, res.r, ZOP_N, Rd, ldr, ZOP_N, T, res.r, res.r, res.n, res.r));
            else
                g1.push_back(zjob(Ud, res.r, ZOP_T, Cd, pr.m, ZOP_T, T, res.r, res.r, res.n, res.r));
            ZgemmJob j2 = !mir ? zjob(Cd, res.m, ZOP_N, T, res.r, ZOP_N, Z, res.m, res.m, res.n, res.r)
                               : zjob(Rd, ldr, ZOP_T, T, res.r, ZOP_N, Z, res.m, res.m, res.n, res.r);
            j2.alpha = make_double2(-1.0, 0.0);
            j2.beta = make_double2(1.0, 0.0);
            g2.push_back(j2);
            zo += (size_t)res.m * res.n;
        }
        PSKEL_CUDA(cudaGetLastError());
        // dense FP64 fill of the batch
        const size_t jb = std::max(sizeof(FillJob), sizeof(GroupFillJob)) * nbb;
        PSKEL_TRY(c->tmp2.reserve(jb + sizeof(int) * (nbb + 1) + sizeof(void *) * nbb +
                                  sizeof(long long) * nbb + sizeof(double) * 2 * nbb + 8 * 256));
        char *d = c->tmp2.as<char>();
        size_t t = 0;
        auto slot = [&](size_t bytes) { size_t x = t; t += (bytes + 255) & ~size_t(255); return d + x; };
        FillJob *d_f = reinterpret_cast<FillJob *>(slot(jb));
        int *d_p = reinterpret_cast<int *>(slot(sizeof(int) * (nbb + 1)));
        const double2 **d_m = reinterpret_cast<const double2 **>(slot(sizeof(void *) * nbb));
        long long *d_s = reinterpret_cast<long long *>(slot(sizeof(long long) * nbb));
        double *d_nz = reinterpret_cast<double *>(slot(sizeof(double) * nbb));
        double *d_ne = reinterpret_cast<double *>(slot(sizeof(double) * nbb));
        if (tri)
            PSKEL_CUDA(cudaMemcpyAsync(d_f, gfills.data(), sizeof(GroupFillJob) * nbb,
                                       cudaMemcpyHostToDevice, c->stream));
        else
            PSKEL_CUDA(cudaMemcpyAsync(d_f, fills.data(), sizeof(FillJob) * nbb,
                                       cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_p, prefix.data(), sizeof(int) * (nbb + 1), cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_m, mats.data(), sizeof(void *) * nbb, cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_s, sizes.data(), sizeof(long long) * nbb, cudaMemcpyHostToDevice, c->stream));
        FillParams fp;
        fp.k = c->em.k;
        fp.eta = c->em.eta;
        fp.r_near = 0;
        fp.q_test = c->em.q_test;
        fp.q_src = c->em.q_src;
        fp.precision = PSKEL_C128;
        fp.split = entry_split_for(c, PSKEL_C128);
        fp.tri_cols = c->tri_cols;
            if (tri)
            PSKEL_TRY(launch_tri_fill(c->mesh, fp, reinterpret_cast<GroupFillJob *>(d_f), d_p, nbb,
                                      prefix.back(), c->stream));
        else
            PSKEL_TRY(launch_fill(c->mesh, fp, d_f, d_p, nbb, prefix.back(), c->flags.as<int>(), c->stream));
        block_norm_kernel<<<nbb, 256, 0, c->stream>>>(d_m, d_s, d_nz);
        PSKEL_LAUNCHED(1);
        PSKEL_TRY(launch_zgemm(g1, c->stream, c->tmp3));
        PSKEL_TRY(launch_zgemm(g2, c->stream, c->tmp3));
        block_norm_kernel<<<nbb, 256, 0, c->stream>>>(d_m, d_s, d_ne);
        PSKEL_LAUNCHED(1);
        std::vector<double> nz(nbb), ne(nbb);
        PSKEL_CUDA(cudaMemcpyAsync(nz.data(), d_nz, sizeof(double) * nbb, cudaMemcpyDeviceToHost, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(ne.data(), d_ne, sizeof(double) * nbb, cudaMemcpyDeviceToHost, c->stream));
        PSKEL_CUDA(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < nbb; ++i) err[b0 + i] = nz[i] > 0 ? ne[i] / nz[i] : 0.0;
        b0 = b1;
    }
    return PSKEL_OK;
}
}  // namespace

extern "C" int pskel_true_errors(pskel_ctx *c, double *err) {
    PSKEL_TRY(ctx_ok(c));
    if (!err || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_ARG, "true_errors: null output or no blocks");
        return PSKEL_ERR_ARG;
    }
    std::vector<int> all(c->n_blocks);
    std::iota(all.begin(), all.end(), 0);
    return true_errors_list(c, all, err);
}

extern "C" int pskel_true_errors_blocks(pskel_ctx *c, const int *blocks, int n, double *err) {
    PSKEL_TRY(ctx_ok(c));
    if (!blocks || !err || n <= 0 || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_ARG, "true_errors_blocks: null argument or empty list");
        return PSKEL_ERR_ARG;
    }
    std::vector<int> list(blocks, blocks + n);
    for (int b : list)
        if (b < 0 || b >= c->n_blocks) {
            set_error(PSKEL_ERR_ARG, "true_errors_blocks: block %d out of range", b);
            return PSKEL_ERR_ARG;
        }
    return true_errors_list(c, list, err);
}

extern "C" int pskel_dense_far_matvec(pskel_ctx *c, const void *X, int ldx, void *Y, int ldy,
                                      int nrhs) {
    PSKEL_TRY(ctx_ok(c));
    if (!X || !Y || nrhs <= 0 || ldx < c->mesh.ne || ldy < c->mesh.ne || c->n_blocks <= 0 ||
        !c->have_mesh) {
        set_error(PSKEL_ERR_ARG, "dense_far_matvec: bad arguments or no blocks");
        return PSKEL_ERR_ARG;
    }
    const int nb = c->n_blocks;
    PSKEL_CUDA(cudaMemsetAsync(Y, 0, sizeof(double2) * (size_t)ldy * nrhs, c->stream));
    const size_t budget = (size_t)1 << 28;  // dense entries per batch
    int tm, tn;
    fill_tile_shape(PSKEL_C128, c->em.q_test, entry_split_for(c, PSKEL_C128), &tm, &tn);
    const bool tri = tri_for(c, PSKEL_C128);
    int b0 = 0;
    while (b0 < nb) {
        size_t dense = 0;
        int b1 = b0;
        while (b1 < nb) {
            const size_t d = (size_t)(c->gptr[c->gt[b1] + 1] - c->gptr[c->gt[b1]]) *
                             (c->gptr[c->gs[b1] + 1] - c->gptr[c->gs[b1]]);
            if (b1 > b0 && dense + d > budget) break;
            dense += d;
            ++b1;
        }
        const int nbb = b1 - b0;
        PSKEL_TRY(c->tmp.reserve(sizeof(double2) * dense + 256));
        double2 *Zb = c->tmp.as<double2>();
        std::vector<FillJob> fills(nbb);
        std::vector<GroupFillJob> gfills(nbb);
        std::vector<DenseApply> apps(nbb);
        std::vector<int> prefix(nbb + 1, 0);
        size_t zo = 0;
        int max_rows = 0;
        for (int i = 0; i < nbb; ++i) {
            const int b = b0 + i, gt = c->gt[b], gs = c->gs[b];
            const int m = c->gptr[gt + 1] - c->gptr[gt], n = c->gptr[gs + 1] - c->gptr[gs];
            const int *rows = c->d_gids.as<int>() + c->gptr[gt], *cols = c->d_gids.as<int>() + c->gptr[gs];
            double2 *Z = Zb + zo;
            zo += (size_t)m * n;
            fills[i] = FillJob{rows, cols, Z, m, n, m, 0};
            const int nt = c->gtri_ptr[gt + 1] - c->gtri_ptr[gt];
            gfills[i] = GroupFillJob{rows, c->d_gtri.as<int>() + c->gtri_ptr[gt],
                                     c->d_gadj.as<int>() + 3 * (size_t)c->gtri_ptr[gt], cols, Z, m, nt,
                                     n, m, 0, tri_cols_for(c, nt), guse_of(c, gt)};
            prefix[i + 1] = prefix[i] + (tri ? (n + gfills[i].tc - 1) / gfills[i].tc
                                             : ((m + tm - 1) / tm) * ((n + tn - 1) / tn));
            apps[i] = DenseApply{Z, rows, cols, m, n};
            max_rows = std::max(max_rows, m);
        }
        const size_t jb = std::max(sizeof(FillJob), sizeof(GroupFillJob)) * nbb;
        PSKEL_TRY(c->tmp2.reserve(jb + sizeof(int) * (nbb + 1) + sizeof(DenseApply) * nbb + 4 * 256));
        char *d = c->tmp2.as<char>();
        size_t t = 0;
        auto slot = [&](size_t bytes) { size_t x = t; t += (bytes + 255) & ~size_t(255); return d + x; };
        void *d_f = slot(jb);
        int *d_p = reinterpret_cast<int *>(slot(sizeof(int) * (nbb + 1)));
        DenseApply *d_a = reinterpret_cast<DenseApply *>(slot(sizeof(DenseApply) * nbb));
        if (tri)
            PSKEL_CUDA(cudaMemcpyAsync(d_f, gfills.data(), sizeof(GroupFillJob) * nbb,
                                       cudaMemcpyHostToDevice, c->stream));
        else
            PSKEL_CUDA(cudaMemcpyAsync(d_f, fills.data(), sizeof(FillJob) * nbb, cudaMemcpyHostToDevice,
                                       c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_p, prefix.data(), sizeof(int) * (nbb + 1), cudaMemcpyHostToDevice,
                                   c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_a, apps.data(), sizeof(DenseApply) * nbb, cudaMemcpyHostToDevice,
                                   c->stream));
        FillParams fp;
        fp.k = c->em.k;
        fp.eta = c->em.eta;
        fp.r_near = 0;
        fp.q_test = c->em.q_test;
        fp.q_src = c->em.q_src;
        fp.precision = PSKEL_C128;
        fp.split = entry_split_for(c, PSKEL_C128);
        fp.tri_cols = c->tri_cols;
            fp.max_rows = max_rows;
        if (tri)
            PSKEL_TRY(launch_tri_fill(c->mesh, fp, reinterpret_cast<GroupFillJob *>(d_f), d_p, nbb,
                                      prefix.back(), c->stream));
        else
            PSKEL_TRY(launch_fill(c->mesh, fp, reinterpret_cast<FillJob *>(d_f), d_p, nbb, prefix.back(),
                                  c->flags.as<int>(), c->stream));
        dense_apply_kernel<<<nbb, 256, 0, c->stream>>>(d_a, reinterpret_cast<const double2 *>(X), ldx,
                                                       reinterpret_cast<double2 *>(Y), ldy, nrhs);
        PSKEL_LAUNCHED(1);
        // the batch buffers are reused by the next batch
        PSKEL_CUDA(cudaStreamSynchronize(c->stream));
        b0 = b1;
    }
    return PSKEL_OK;
}

extern "C" long long pskel_kernel_launches(void) { return launches_so_far(); }

// ------------------------------------------------------------------ FMA peak microbenchmark
namespace pskel {
template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T *out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
      x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
}  // namespace pskel

template <typename T>
static int fma_peak_t(double *tflops) {
    const int blocks = sm_count() * 8, threads = 256;
    T *out = nullptr;
    PSKEL_CUDA(cudaMalloc(&out, sizeof(T) * blocks * threads));
    cudaEvent_t e0, e1;
    PSKEL_CUDA(cudaEventCreate(&e0));
    PSKEL_CUDA(cudaEventCreate(&e1));
    const int iters = sizeof(T) == 8 ? 2048 : 4096;
    fma_chain_kernel<T><<<blocks, threads>>>(out, 64, (T)0.999, (T)0.001);  // warm-up
    PSKEL_LAUNCHED(1);
    PSKEL_CUDA(cudaEventRecord(e0));
    fma_chain_kernel<T><<<blocks, threads>>>(out, iters, (T)0.999, (T)0.001);
    PSKEL_LAUNCHED(1);
    PSKEL_CUDA(cudaEventRecord(e1));
    PSKEL_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 64.0 * (double)iters * blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return PSKEL_OK;
}

extern "C" int pskel_fma_peak(double *fp32_tflops, double *fp64_tflops) {
    if (!fp32_tflops || !fp64_tflops) {
        set_error(PSKEL_ERR_ARG, "null output");
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(fma_peak_t<float>(fp32_tflops));
    PSKEL_TRY(fma_peak_t<double>(fp64_tflops));
    return PSKEL_OK;
}
