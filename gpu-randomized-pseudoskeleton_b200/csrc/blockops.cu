// Operations on the compressed blocks kept by the engine: the compressed matvec
// (y = sum over far blocks of C U R x, the reference's C(U(Rv)) of
// codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:1929-1960 for many right-hand
// sides and all blocks at once) and the recompression of every block's CUR into an SVD-truncated
// C' S R' (codes/ACA_vs_CUR/seed/svd_compress.m:19-33 with the QRs replaced by one-sided Jacobi).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine_internal.cuh"
#include "zgemm.cuh"

namespace pskel {

__device__ __forceinline__ double2 ld_c(const double2 *p, size_t i) { return p[i]; }
__device__ __forceinline__ double2 ld_c(const float2 *p, size_t i) {
    const float2 v = p[i];
    return make_double2(v.x, v.y);
}

template <typename A> struct CT;
template <> struct CT<double> { using c = double2; };
template <> struct CT<float> { using c = float2; };

template <typename A> __device__ __forceinline__ typename CT<A>::c mk(double x, double y);
template <> __device__ __forceinline__ double2 mk<double>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 mk<float>(double x, double y) { return make_float2((float)x, (float)y); }

// One block per CTA iteration: T1 = R X(cols) (r x nrhs), T2 = U T1, Y(rows) += C T2; a mirror
// block (the transpose of a stored one) uses R_p^T U_p^T C_p^T from its primary's factors.
// Arithmetic type A (float or double), storage S (float2 or double2) of C and R.
struct MatvecBlock {
    const int *rows, *cols;
    const void *C, *R;  // the stored factors: C m_c x r (ld ldc), R r x n_r (ld ldr)
    const double2 *U;
    int m, n, r, ldr;   // m, n: this block's rows and columns
    int ldc, trans;     // trans: mirror block
};

// factor element accessors: Rop(i, k) = R(i, k) (k < n), or C_p(k, i) for a mirror;
// Uop(i, k) = U(i, k) or U(k, i); Cop(i, k) = C(i, k) (i < m), or R_p(k, i)
template <typename S> __device__ __forceinline__ double2 r_op(const MatvecBlock &w, const S *R, const S *C, int i, int k) {
    return w.trans ? ld_c(C, k + (size_t)i * w.ldc) : ld_c(R, i + (size_t)k * w.ldr);
}
template <typename S> __device__ __forceinline__ double2 c_op(const MatvecBlock &w, const S *R, const S *C, int i, int k) {
    return w.trans ? ld_c(R, k + (size_t)i * w.ldr) : ld_c(C, i + (size_t)k * w.ldc);
}

template <typename A, typename S>
__global__ void __launch_bounds__(256) matvec_kernel(const MatvecBlock *__restrict__ blocks, int nb,
                                                     const typename CT<A>::c *__restrict__ X, int ldx,
                                                     A *__restrict__ Y, int ldy, int nrhs) {
    using C2 = typename CT<A>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2 *t1 = reinterpret_cast<C2 *>(smem_raw);
    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        const MatvecBlock w = blocks[b];
        C2 *t2 = t1 + w.r * nrhs;
        const S *R = reinterpret_cast<const S *>(w.R);
        const S *Cm = reinterpret_cast<const S *>(w.C);
        for (int e = threadIdx.x; e < w.r * nrhs; e += blockDim.x) {
            const int i = e % w.r, j = e / w.r;
            A sr = 0, si = 0;
            for (int k = 0; k < w.n; ++k) {
                const double2 rv = r_op(w, R, Cm, i, k);
                const C2 x = X[w.cols[k] + (size_t)j * ldx];
                sr += (A)rv.x * x.x - (A)rv.y * x.y;
                si += (A)rv.x * x.y + (A)rv.y * x.x;
            }
            t1[e] = mk<A>(sr, si);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < w.r * nrhs; e += blockDim.x) {
            const int i = e % w.r, j = e / w.r;
            A sr = 0, si = 0;
            for (int k = 0; k < w.r; ++k) {
                const double2 u = w.trans ? w.U[k + (size_t)i * w.r] : w.U[i + (size_t)k * w.r];
                const C2 t = t1[k + j * w.r];
                sr += (A)u.x * t.x - (A)u.y * t.y;
                si += (A)u.x * t.y + (A)u.y * t.x;
            }
            t2[e] = mk<A>(sr, si);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < w.m * nrhs; e += blockDim.x) {
            const int i = e % w.m, j = e / w.m;
            A sr = 0, si = 0;
            for (int k = 0; k < w.r; ++k) {
                const double2 c = c_op(w, R, Cm, i, k);
                const C2 t = t2[k + j * w.r];
                sr += (A)c.x * t.x - (A)c.y * t.y;
                si += (A)c.x * t.y + (A)c.y * t.x;
            }
            A *y = Y + 2 * (w.rows[i] + (size_t)j * ldy);
            atomicAdd(y, sr);
            atomicAdd(y + 1, si);
        }
        __syncthreads();
    }
}

// The same product organised by test group: one CTA per chunk of up to kMvChunk blocks that share
// their test group. Per block, T1 = R X(cols) has the block's X rows staged in shared memory and
// the k range split over the 8 warps (lane = row of R, JB right-hand sides in registers, broadcast
// reads of X), partial sums reduced through shared memory; T2 = U T1; the test-group accumulator
// (m x nrhs, each entry owned by one thread) gains C T2 with JB right-hand sides per thread in
// registers; it is added to Y once per chunk. Register blocking over the right-hand sides reads
// every factor entry once per JB products instead of once per product, and the chunk divides
// the global atomics by its length.
constexpr int kMvChunk = 8;
constexpr int kMvWarps = 8;

struct MatvecChunk {
    int first, count;  // blocks [first, first + count) of the group-ordered table
    const int *rows;   // the chunk's test group
    int m;
};

template <typename A, typename S, int JB>
__global__ void __launch_bounds__(256) matvec_group_kernel(const MatvecBlock *__restrict__ blocks,
                                                           const MatvecChunk *__restrict__ chunks,
                                                           const typename CT<A>::c *__restrict__ X, int ldx,
                                                           A *__restrict__ Y, int ldy, int nrhs, int max_r,
                                                           int max_n) {
    using C2 = typename CT<A>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const MatvecChunk ch = chunks[blockIdx.x];
    C2 *acc = reinterpret_cast<C2 *>(smem_raw);  // m x nrhs
    C2 *t1 = acc + (size_t)ch.m * nrhs;          // r x nrhs
    C2 *t2 = t1 + (size_t)max_r * nrhs;          // r x nrhs
    C2 *xs = t2 + (size_t)max_r * nrhs;          // n x JB
    C2 *part = xs + (size_t)max_n * JB;          // warps x 32 (JB = 1 only)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int e = threadIdx.x; e < ch.m * nrhs; e += blockDim.x) acc[e] = mk<A>(0.0, 0.0);
    for (int bi = 0; bi < ch.count; ++bi) {
        const MatvecBlock w = blocks[ch.first + bi];
        const S *R = reinterpret_cast<const S *>(w.R);
        const S *Cm = reinterpret_cast<const S *>(w.C);
        const int k0 = (w.n * wid) / kMvWarps, k1 = (w.n * (wid + 1)) / kMvWarps;
        // T1 = R X(cols)
        if (JB == 1) {
            // one right-hand side at a time: the k range split over the warps, partial sums
            // reduced through shared memory
            for (int j0 = 0; j0 < nrhs; ++j0) {
                __syncthreads();  // xs and part are free
                for (int k = threadIdx.x; k < w.n; k += blockDim.x) xs[k] = X[w.cols[k] + (size_t)j0 * ldx];
                __syncthreads();
                for (int ib = 0; ib < w.r; ib += 32) {
                    const int i = ib + lane;
                    A ar = 0, ai = 0;
                    if (i < w.r)
                        for (int k = k0; k < k1; ++k) {
                            const double2 rv = r_op(w, R, Cm, i, k);
                            const C2 x = xs[k];
                            ar += (A)rv.x * x.x - (A)rv.y * x.y;
                            ai += (A)rv.x * x.y + (A)rv.y * x.x;
                        }
                    part[wid * 32 + lane] = mk<A>(ar, ai);
                    __syncthreads();
                    if (threadIdx.x < 32 && ib + threadIdx.x < w.r) {
                        A sr = 0, si = 0;
                        for (int q = 0; q < kMvWarps; ++q) {
                            const C2 v = part[q * 32 + threadIdx.x];
                            sr += v.x;
                            si += v.y;
                        }
                        t1[(ib + threadIdx.x) + j0 * w.r] = mk<A>(sr, si);
                    }
                    __syncthreads();
                }
            }
        } else {
            // several right-hand sides: X(cols, j0 : j0 + JB) staged once (xs[k][jj]); the k range
            // split over the warps (lane = row of R, all JB right-hand sides in registers), so that
            // the CTA reads R once; the warps' partial sums are added into T1 by shared-memory
            // atomics
            for (int j0 = 0; j0 < nrhs; j0 += JB) {
                __syncthreads();  // xs is free
                for (int e = threadIdx.x; e < w.n * JB; e += blockDim.x) {
                    const int k = e / JB, jj = e - k * JB;
                    xs[e] = j0 + jj < nrhs ? X[w.cols[k] + (size_t)(j0 + jj) * ldx] : mk<A>(0.0, 0.0);
                }
                for (int e = threadIdx.x; e < w.r * JB; e += blockDim.x) {
                    const int i = e % w.r, j = j0 + e / w.r;
                    if (j < nrhs) t1[i + j * w.r] = mk<A>(0.0, 0.0);
                }
                __syncthreads();
                for (int ib = 0; ib < w.r; ib += 32) {
                    const int i = ib + lane;
                    if (i >= w.r || k0 >= k1) continue;
                    A ar[JB], ai[JB];
#pragma unroll
                    for (int q = 0; q < JB; ++q) ar[q] = ai[q] = 0;
                    for (int k = k0; k < k1; ++k) {
                        const double2 rv = r_op(w, R, Cm, i, k);
                        const A rx = (A)rv.x, ry = (A)rv.y;
                        const C2 *xk = xs + k * JB;
#pragma unroll
                        for (int q = 0; q < JB; ++q) {
                            const C2 x = xk[q];
                            ar[q] += rx * x.x - ry * x.y;
                            ai[q] += rx * x.y + ry * x.x;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < JB; ++q) {
                        const int j = j0 + q;
                        if (j < nrhs) {
                            A *t = reinterpret_cast<A *>(t1 + i + j * w.r);
                            atomicAdd(t, ar[q]);
                            atomicAdd(t + 1, ai[q]);
                        }
                    }
                }
            }
            __syncthreads();
        }
        // T2 = U T1
        for (int e = threadIdx.x; e < w.r * nrhs; e += blockDim.x) {
            const int i = e % w.r, j = e / w.r;
            A sr = 0, si = 0;
            for (int k = 0; k < w.r; ++k) {
                const double2 u = w.trans ? w.U[k + (size_t)i * w.r] : w.U[i + (size_t)k * w.r];
                const C2 t = t1[k + j * w.r];
                sr += (A)u.x * t.x - (A)u.y * t.y;
                si += (A)u.x * t.y + (A)u.y * t.x;
            }
            t2[e] = mk<A>(sr, si);
        }
        __syncthreads();
        // acc += C T2
        for (int i = threadIdx.x; i < ch.m; i += blockDim.x) {
            for (int j0 = 0; j0 < nrhs; j0 += JB) {
                A ar[JB], ai[JB];
#pragma unroll
                for (int jj = 0; jj < JB; ++jj) ar[jj] = ai[jj] = 0;
                for (int k = 0; k < w.r; ++k) {
                    const double2 cv = c_op(w, R, Cm, i, k);
                    const A cx = (A)cv.x, cy = (A)cv.y;
#pragma unroll
                    for (int jj = 0; jj < JB; ++jj) {
                        if (j0 + jj < nrhs) {
                            const C2 t = t2[k + (j0 + jj) * w.r];
                            ar[jj] += cx * t.x - cy * t.y;
                            ai[jj] += cx * t.y + cy * t.x;
                        }
                    }
                }
#pragma unroll
                for (int jj = 0; jj < JB; ++jj) {
                    if (j0 + jj < nrhs) {
                        C2 a = acc[i + (size_t)(j0 + jj) * ch.m];
                        a.x += ar[jj];
                        a.y += ai[jj];
                        acc[i + (size_t)(j0 + jj) * ch.m] = a;
                    }
                }
            }
        }
        __syncthreads();  // t1 / t2 are reused by the next block
    }
    for (int e = threadIdx.x; e < ch.m * nrhs; e += blockDim.x) {
        const int i = e % ch.m, j = e / ch.m;
        A *y = Y + 2 * (ch.rows[i] + (size_t)j * ldy);
        atomicAdd(y, acc[e].x);
        atomicAdd(y + 1, acc[e].y);
    }
}

}  // namespace pskel

using namespace pskel;

extern "C" int pskel_matvec(pskel_ctx *c, const void *X, int ldx, void *Y, int ldy, int nrhs,
                            int precision, void *stream) {
    if (!c || !X || !Y || nrhs <= 0 || nrhs > 64 || ldx < c->mesh.ne || ldy < c->mesh.ne ||
        (precision != PSKEL_C128 && precision != PSKEL_C64)) {
        set_error(PSKEL_ERR_ARG, "matvec: bad arguments (nrhs=%d ldx=%d ldy=%d)", nrhs, ldx, ldy);
        return PSKEL_ERR_ARG;
    }
    if (c->n_blocks <= 0 || (int)c->results.size() != c->n_blocks) {
        set_error(PSKEL_ERR_STATE, "matvec: no compressed blocks");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);  // NULL: legacy default stream
    const int nb = c->n_blocks;
    if (c->mv_generation != c->generation) {
        // block table in test-group order and its chunks: built once per compression
        std::vector<int> order(nb);
        for (int b = 0; b < nb; ++b) order[b] = b;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return c->gt[a] < c->gt[b]; });
        std::vector<MatvecBlock> hb(nb);
        std::vector<MatvecChunk> hc;
        int max_r = 0, max_m = 0, max_n = 0;
        for (int pos = 0; pos < nb; ++pos) {
            const int b = order[pos];
            const BlockResult &res = c->results[b];
            if (res.arena < 0) {
                set_error(PSKEL_ERR_STATE, "matvec: block %d has no retained factors", b);
                return PSKEL_ERR_STATE;
            }
            const BlockResult &pr = res.mirror >= 0 ? c->results[res.mirror] : res;
            const char *base = c->arenas[pr.arena].keep.as<char>();
            const int *rows = c->d_gids.as<int>() + c->gptr[c->gt[b]];
            hb[pos] = MatvecBlock{rows, c->d_gids.as<int>() + c->gptr[c->gs[b]], base + pr.offC,
                                  base + pr.offRx, reinterpret_cast<const double2 *>(base + pr.offU),
                                  res.m, res.n, res.r, pr.r + pr.pe, pr.m, res.mirror >= 0 ? 1 : 0};
            max_r = std::max(max_r, res.r);
            max_m = std::max(max_m, res.m);
            max_n = std::max(max_n, res.n);
            if (hc.empty() || c->gt[order[hc.back().first]] != c->gt[b] || hc.back().count == kMvChunk)
                hc.push_back(MatvecChunk{pos, 0, rows, res.m});
            ++hc.back().count;
        }
        const size_t tb = (sizeof(MatvecBlock) * nb + 255) & ~size_t(255);
        PSKEL_TRY(c->mv_table.reserve(tb + sizeof(MatvecChunk) * hc.size() + 256));
        PSKEL_CUDA(cudaStreamSynchronize(c->stream));
        PSKEL_CUDA(cudaMemcpy(c->mv_table.ptr, hb.data(), sizeof(MatvecBlock) * nb, cudaMemcpyHostToDevice));
        PSKEL_CUDA(cudaMemcpy(c->mv_table.as<char>() + tb, hc.data(), sizeof(MatvecChunk) * hc.size(),
                              cudaMemcpyHostToDevice));
        c->mv_max_r = max_r;
        c->mv_max_m = max_m;
        c->mv_max_n = max_n;
        c->mv_chunks = (int)hc.size();
        c->mv_chunk_off = tb;
        c->mv_generation = c->generation;
    }
    const size_t es = precision == PSKEL_C64 ? sizeof(float2) : sizeof(double2);
    const size_t smem = 2 * (size_t)c->mv_max_r * nrhs * es;
    if (smem > 200 * 1024) {
        set_error(PSKEL_ERR_ARG, "matvec: r x nrhs too large (%d x %d)", c->mv_max_r, nrhs);
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaMemsetAsync(Y, 0, es * (size_t)ldy * nrhs, st));
    const bool f32 = c->precision == PSKEL_C64;  // storage of the factors
    const int grid = std::min(nb, sm_count() * 8);
    const MatvecBlock *d_b = c->mv_table.as<MatvecBlock>();
    const MatvecChunk *d_c = reinterpret_cast<const MatvecChunk *>(c->mv_table.as<char>() + c->mv_chunk_off);
    // grouped version when the test group's accumulator and staging fit in shared memory; JB
    // right-hand sides per thread
    int jb = nrhs >= 16 ? 16 : (nrhs >= 8 ? 8 : 1);
    auto gsz = [&](int j) {
        return smem + es * ((size_t)c->mv_max_m * nrhs + (size_t)c->mv_max_n * j + (size_t)kMvWarps * 32);
    };
    while (jb > 1 && gsz(jb) > 200 * 1024) jb = jb == 16 ? 8 : 1;
    const size_t gsmem = gsz(jb);
    const bool grouped = gsmem <= 200 * 1024;
#define PSKEL_MV(A, S)                                                                         \
    do {                                                                                       \
        if (grouped) {                                                                         \
            auto k = jb == 16 ? matvec_group_kernel<A, S, 16>                                  \
                              : (jb == 8 ? matvec_group_kernel<A, S, 8> : matvec_group_kernel<A, S, 1>); \
            PSKEL_TRY(ensure_smem_attr(k, 200 * 1024));                                        \
            k<<<c->mv_chunks, 256, gsmem, st>>>(d_b, d_c, reinterpret_cast<const CT<A>::c *>(X), \
                                                ldx, reinterpret_cast<A *>(Y), ldy, nrhs,     \
                                                c->mv_max_r, c->mv_max_n);                     \
        } else {                                                                               \
            auto k = matvec_kernel<A, S>;                                                      \
            PSKEL_TRY(ensure_smem_attr(k, 200 * 1024));                                        \
            k<<<grid, 256, smem, st>>>(d_b, nb, reinterpret_cast<const CT<A>::c *>(X), ldx,   \
                                       reinterpret_cast<A *>(Y), ldy, nrhs);                   \
        }                                                                                      \
        PSKEL_LAUNCHED(1);                                                                     \
    } while (0)
    if (precision == PSKEL_C64) {
        if (f32) PSKEL_MV(float, float2); else PSKEL_MV(float, double2);
    } else {
        if (f32) PSKEL_MV(double, float2); else PSKEL_MV(double, double2);
    }
#undef PSKEL_MV
    return PSKEL_OK;
}

// ============================================================== recompression (FP64)
// The restatement of svd_compress.m:19-33 for every block (C m x r, U r x r, R r x n):
//   [Q_c, R_c] = qr(C),  [Q_r, R_r] = qr(R^H)           (Householder, batched)
//   M = R_c U R_r^H = u s v^H                              (QR-preconditioned Jacobi SVD)
//   keep the k values s > thresh * max s:  C' = Q_c u_k,  S = s_k,  R' = (Q_r v_k)^H
// with C' and R'^H formed by applying the reflectors to [u_k; 0] and [v_k; 0].
namespace pskel {

struct RecompBlock {
    const void *C, *R;   // stored factors (storage type of the compression)
    const double2 *U;
    double2 *Bc, *Br;    // working copies of C (m x r) and R^H (n x r): reflectors after the QR
    double2 *Rc, *Rr, *T, *M, *Vm, *Zc, *Zr, *Cp, *RpH, *Rp;
    double2 *v0c, *v0r;
    double *cc, *cr, *sm, *S;
    int *pm, *kout;
    int m, n, r, ldr;
    double thresh;
};

template <typename S>
__global__ void recomp_load_kernel(const RecompBlock *__restrict__ jobs) {
    const RecompBlock w = jobs[blockIdx.x];
    const S *C = reinterpret_cast<const S *>(w.C);
    const S *R = reinterpret_cast<const S *>(w.R);
    for (int e = threadIdx.x; e < w.m * w.r; e += blockDim.x) w.Bc[e] = ld_c(C, e);
    for (int e = threadIdx.x; e < w.n * w.r; e += blockDim.x) {
        const int i = e % w.n, j = e / w.n;  // Br(i, j) = conj(R(j, i))
        const double2 v = ld_c(R, j + (size_t)i * w.ldr);
        w.Br[e] = make_double2(v.x, -v.y);
    }
}

// u_k, v_k in the order of decreasing s: Zc(:, t) = (M V)(:, p_t) / s_{p_t}, Zr(:, t) = V(:, p_t),
// S[t] = s_{p_t}; k = #{s > thresh s_max}
__global__ void __launch_bounds__(256) recomp_factors_kernel(const RecompBlock *__restrict__ jobs) {
    const RecompBlock w = jobs[blockIdx.x];
    const double smax = w.sm[w.pm[0]];
    for (int e = threadIdx.x; e < w.r * w.r; e += blockDim.x) {
        const int i = e % w.r, t = e / w.r;
        const int c = w.pm[t];
        const double s = w.sm[c];
        const double f = s > 0 ? 1.0 / s : 0.0;
        const double2 mv = w.M[i + (size_t)c * w.r];  // M holds M V after the SVD
        w.Zc[e] = make_double2(mv.x * f, mv.y * f);
        w.Zr[e] = w.Vm[i + (size_t)c * w.r];
    }
    for (int t = threadIdx.x; t < w.r; t += blockDim.x) w.S[t] = w.sm[w.pm[t]];
    if (threadIdx.x == 0) {
        int k = 0;
        for (int t = 0; t < w.r; ++t) k += w.sm[w.pm[t]] > w.thresh * smax;
        *w.kout = k;
    }
}

// R' = (R'^H)^H : r x n (first k rows valid) from n x r
__global__ void recomp_rp_kernel(const RecompBlock *__restrict__ jobs) {
    const RecompBlock w = jobs[blockIdx.x];
    for (int e = threadIdx.x; e < w.r * w.n; e += blockDim.x) {
        const int t = e % w.r, j = e / w.r;
        const double2 v = w.RpH[j + (size_t)t * w.n];
        w.Rp[e] = make_double2(v.x, -v.y);
    }
}

}  // namespace pskel

namespace pskel {

// FP64 recompression of the primary blocks `prims` into `buf` (factors and workspace), enqueued
// on stream st (job tables in c->tmp; scratch c->tmp2, c->tmp3); fills their slots but k, which
// recompress_fp64_finish reads back.
int recompress_fp64_enqueue(pskel_ctx *c, const std::vector<int> &prims, double thresh, cudaStream_t st,
                            DevBuf &buf, Fp64Recomp &out) {
    out = Fp64Recomp();
    out.prims = prims;
    out.st = st;
    const int nb = (int)prims.size();
    if (nb == 0) return PSKEL_OK;
    const bool f32 = c->precision == PSKEL_C64;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    std::vector<size_t> off(nb + 1, 0);
    for (int pi = 0; pi < nb; ++pi) {
        const BlockResult &res = c->results[prims[pi]];
        const size_t m = res.m, n = res.n, r = res.r;
        off[pi + 1] = off[pi] + 2 * al(16 * m * r) + 3 * al(16 * n * r) + 8 * al(16 * r * r) +
                     2 * al(16 * r) + 4 * al(8 * r) + al(4 * r) + 256;
    }
    PSKEL_TRY(buf.reserve(off[nb] + 256));
    char *base = buf.as<char>();
    std::vector<RecompBlock> jobs(nb);
    std::vector<QrJob> qrs;
    qrs.reserve(2 * nb);
    std::vector<SvdJob> svds;
    svds.reserve(nb);
    std::vector<ZgemmJob> g1, g2;
    std::vector<ApplyQJob> aps;
    aps.reserve(2 * nb);
    // device job tables (the k table is referenced by the apply jobs)
    const size_t jb = sizeof(RecompBlock) * nb, s2 = sizeof(SvdJob) * nb;
    PSKEL_TRY(c->tmp.reserve(al(jb) + al(s2) + sizeof(int) * nb + 1024));
    char *d = c->tmp.as<char>();
    RecompBlock *d_jobs = reinterpret_cast<RecompBlock *>(d);
    SvdJob *d_s2 = reinterpret_cast<SvdJob *>(d + al(jb));
    int *d_k = reinterpret_cast<int *>(d + al(jb) + al(s2));
    for (int pi = 0; pi < nb; ++pi) {
        const int b = prims[pi];
        const BlockResult &res = c->results[b];
        const char *kb = c->arenas[res.arena].keep.as<char>();
        char *q = base + off[pi];
        auto take = [&](size_t bytes) { char *x = q; q += al(bytes); return x; };
        const size_t m = res.m, n = res.n, r = res.r;
        RecompBlock &w = jobs[pi];
        w.C = kb + res.offC;
        w.R = kb + res.offRx;
        w.U = reinterpret_cast<const double2 *>(kb + res.offU);
        w.Bc = reinterpret_cast<double2 *>(take(16 * m * r));
        w.Cp = reinterpret_cast<double2 *>(take(16 * m * r));
        w.Br = reinterpret_cast<double2 *>(take(16 * n * r));
        w.RpH = reinterpret_cast<double2 *>(take(16 * n * r));
        w.Rp = reinterpret_cast<double2 *>(take(16 * r * n));
        w.Rc = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Rr = reinterpret_cast<double2 *>(take(16 * r * r));
        w.T = reinterpret_cast<double2 *>(take(16 * r * r));
        w.M = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Vm = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Zc = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Zr = reinterpret_cast<double2 *>(take(16 * r * r));
        take(16 * r * r);  // spare
        w.v0c = reinterpret_cast<double2 *>(take(16 * r));
        w.v0r = reinterpret_cast<double2 *>(take(16 * r));
        w.cc = reinterpret_cast<double *>(take(8 * r));
        w.cr = reinterpret_cast<double *>(take(8 * r));
        w.sm = reinterpret_cast<double *>(take(8 * r));
        w.S = reinterpret_cast<double *>(take(8 * r));
        w.pm = reinterpret_cast<int *>(take(4 * r));
        w.kout = d_k + pi;
        w.m = res.m;
        w.n = res.n;
        w.r = res.r;
        w.ldr = res.r + res.pe;
        w.thresh = thresh;
        qrs.push_back(QrJob{w.Bc, w.Rc, w.v0c, w.cc, res.m, res.r});
        qrs.push_back(QrJob{w.Br, w.Rr, w.v0r, w.cr, res.n, res.r});
        // M = R_c (U R_r^H)
        g1.push_back(zjob(w.U, res.r, ZOP_N, w.Rr, res.r, ZOP_C, w.T, res.r, res.r, res.r, res.r));
        g2.push_back(zjob(w.Rc, res.r, ZOP_N, w.T, res.r, ZOP_N, w.M, res.r, res.r, res.r, res.r));
        svds.push_back(SvdJob{w.M, w.Vm, w.sm, w.pm, res.r, res.r, 0, 0});
        aps.push_back(ApplyQJob{w.Bc, w.v0c, w.cc, res.m, res.r, w.Zc, res.r, w.Cp, res.m, res.r, w.kout});
        aps.push_back(ApplyQJob{w.Br, w.v0r, w.cr, res.n, res.r, w.Zr, res.r, w.RpH, res.n, res.r, w.kout});
        RecompSlot &sl = c->recomp_slots[b];
        sl.Cp = w.Cp;
        sl.Rp = w.Rp;
        sl.S = w.S;
        sl.ldrp = res.r;
        sl.mirror = -1;
    }
    PSKEL_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jb, cudaMemcpyHostToDevice, st));
    PSKEL_CUDA(cudaMemcpyAsync(d_s2, svds.data(), s2, cudaMemcpyHostToDevice, st));
    if (f32) recomp_load_kernel<float2><<<nb, 256, 0, st>>>(d_jobs);
    else recomp_load_kernel<double2><<<nb, 256, 0, st>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    PSKEL_TRY(batched_qr(qrs, st, c->tmp2));
    PSKEL_TRY(launch_zgemm(g1, st, c->tmp3));
    PSKEL_TRY(launch_zgemm(g2, st, c->tmp3));
    PSKEL_TRY(batched_svd(d_s2, svds, 60, st, c->tmp2));
    recomp_factors_kernel<<<nb, 256, 0, st>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    PSKEL_TRY(batched_apply_q(aps, st, c->tmp3));
    recomp_rp_kernel<<<nb, 256, 0, st>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    out.d_s2 = d_s2;
    out.d_k = d_k;
    return PSKEL_OK;
}

// Ranks and SVD statuses of an enqueued FP64 recompression back to the host (waits for it).
int recompress_fp64_finish(pskel_ctx *c, Fp64Recomp &r) {
    const int nb = (int)r.prims.size();
    if (nb == 0) return PSKEL_OK;
    std::vector<SvdJob> h2(nb);
    std::vector<int> ks(nb);
    PSKEL_CUDA(cudaMemcpyAsync(h2.data(), r.d_s2, sizeof(SvdJob) * nb, cudaMemcpyDeviceToHost, r.st));
    PSKEL_CUDA(cudaMemcpyAsync(ks.data(), r.d_k, sizeof(int) * nb, cudaMemcpyDeviceToHost, r.st));
    PSKEL_CUDA(cudaStreamSynchronize(r.st));
    for (const SvdJob &j : h2)
        if (j.status != PSKEL_OK) {
            set_error(PSKEL_ERR_NOCONV, "recompress: Jacobi SVD of a core did not converge");
            return PSKEL_ERR_NOCONV;
        }
    for (int pi = 0; pi < nb; ++pi) c->recomp_slots[r.prims[pi]].k = ks[pi];
    return PSKEL_OK;
}

}  // namespace pskel

extern "C" int pskel_set_recompress_path(pskel_ctx *c, int path) {
    if (!c || path < 0 || path > 2) {
        set_error(PSKEL_ERR_ARG, "set_recompress_path: path must be 0 (auto), 1 (FP64) or 2 (split)");
        return PSKEL_ERR_ARG;
    }
    c->recomp_path = path;
    return PSKEL_OK;
}

extern "C" int pskel_recompress_split_blocks(pskel_ctx *c, int *split_blocks) {
    if (!c || !split_blocks) {
        set_error(PSKEL_ERR_ARG, "recompress_split_blocks: null argument");
        return PSKEL_ERR_ARG;
    }
    *split_blocks = c->recomp_split_blocks;
    return PSKEL_OK;
}

extern "C" int pskel_recompress(pskel_ctx *c, double thresh, int *ranks) {
    if (!c || !(thresh >= 0) || !(thresh < 1) || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_ARG, "recompress: bad arguments");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const int nball = c->n_blocks;
    // only blocks with their own factors are recompressed; a mirror block takes its primary's
    // recompression transposed
    std::vector<int> prims;
    for (int b = 0; b < nball; ++b) {
        if (c->results[b].arena < 0) {
            set_error(PSKEL_ERR_STATE, "recompress: block %d has no retained factors", b);
            return PSKEL_ERR_STATE;
        }
        if (c->results[b].mirror < 0) prims.push_back(b);
    }
    c->recomp_slots.assign(nball, RecompSlot{});
    // the split path (tensor cores, TF32 hi + lo operands) takes the complex-FP32 compressions
    // at thresholds of 1e-5 and above; it hands back the blocks it cannot take
    std::vector<int> split, fp64;
    for (int b : prims)
        if (recomp_split_eligible(c, b, thresh)) split.push_back(b);
        else fp64.push_back(b);
    PSKEL_CUDA(cudaEventRecord(c->ev[0], c->stream));
    // blocks whose pinv kept core values below the split products' accuracy join the FP64 set
    PSKEL_TRY(recomp_split_precheck(c, thresh, split, fp64));
    // the FP64 set (usually a few large or full-sample cores, latency-bound) runs on the second
    // stream beside the split path
    Fp64Recomp side, rest;
    cudaStream_t s2 = c->pipe_stream ? c->pipe_stream : c->stream;
    if (!fp64.empty() && s2 != c->stream) {
        PSKEL_CUDA(cudaEventRecord(c->pipe_ev[0], c->stream));
        PSKEL_CUDA(cudaStreamWaitEvent(s2, c->pipe_ev[0], 0));
    }
    PSKEL_TRY(recompress_fp64_enqueue(c, fp64, thresh, s2, c->recomp64, side));
    std::vector<int> rejected;
    PSKEL_TRY(recompress_split(c, split, thresh, rejected));
    c->recomp_split_blocks = (int)(split.size() - rejected.size());
    PSKEL_TRY(recompress_fp64_finish(c, side));
    // blocks the split path handed back (a Cholesky breakdown, an unconverged SVD)
    PSKEL_TRY(recompress_fp64_enqueue(c, rejected, thresh, c->stream, c->recomp64b, rest));
    PSKEL_TRY(recompress_fp64_finish(c, rest));
    PSKEL_CUDA(cudaEventRecord(c->ev[4], c->stream));
    PSKEL_CUDA(cudaEventSynchronize(c->ev[4]));
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[4]);
        c->timing[4] = ms;
    }
    for (int b = 0; b < nball; ++b) {
        const int mb = c->results[b].mirror;
        if (mb >= 0) {
            c->recomp_slots[b] = c->recomp_slots[mb];
            c->recomp_slots[b].mirror = mb;
        }
        if (ranks) ranks[b] = c->recomp_slots[b].k;
    }
    return PSKEL_OK;
}

extern "C" int pskel_get_recompressed(pskel_ctx *c, int b, pskel_c128 *Cp, double *S,
                                      pskel_c128 *Rp) {
    if (!c || b < 0 || b >= c->n_blocks || (int)c->recomp_slots.size() != c->n_blocks) {
        set_error(PSKEL_ERR_STATE, "get_recompressed: run pskel_recompress first");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const RecompSlot &sl = c->recomp_slots[b];
    if (sl.mirror >= 0) {  // transpose of the primary's: C' = R'_p^T, R' = C'_p^T
        const BlockResult &res = c->results[b];
        const size_t k = sl.k, mb = res.m, nb_ = res.n;
        std::vector<pskel_c128> Cpp(nb_ * k), Rpp(k * mb);
        PSKEL_TRY(pskel_get_recompressed(c, sl.mirror, Cpp.data(), S, Rpp.data()));
        if (Cp)
            for (size_t t = 0; t < k; ++t)
                for (size_t i = 0; i < mb; ++i) Cp[i + t * mb] = Rpp[t + i * k];
        if (Rp)
            for (size_t j = 0; j < nb_; ++j)
                for (size_t t = 0; t < k; ++t) Rp[t + j * k] = Cpp[j + t * nb_];
        return PSKEL_OK;
    }
    const BlockResult &res = c->results[b];
    const size_t k = sl.k;
    if (Cp) PSKEL_CUDA(cudaMemcpy(Cp, sl.Cp, 16 * (size_t)res.m * k, cudaMemcpyDeviceToHost));
    if (S) PSKEL_CUDA(cudaMemcpy(S, sl.S, 8 * k, cudaMemcpyDeviceToHost));
    if (Rp) {
        // R' is stored k x n with leading dimension ldrp >= k: copy its first k rows
        std::vector<double2> h((size_t)sl.ldrp * res.n);
        PSKEL_CUDA(cudaMemcpy(h.data(), sl.Rp, 16 * h.size(), cudaMemcpyDeviceToHost));
        for (int j = 0; j < res.n; ++j)
            for (size_t t = 0; t < k; ++t) {
                const double2 v = h[t + (size_t)j * sl.ldrp];
                Rp[t + j * k] = pskel_c128{v.x, v.y};
            }
    }
    return PSKEL_OK;
}
