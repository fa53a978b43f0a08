// Pseudo-inverse of the small cores of a compression round, one warp per core.
//
// A round's core Z(I, J) is r x r with r <= 32 for almost every block the rank predictor sizes.
// For those, gather + SVD + pinv run in one kernel with the whole matrix in the registers of one
// warp (lane l holds column l, 32 rows, zero padded), so no barrier and no shared memory is
// involved: the same QR-preconditioned one-sided Jacobi as the CTA kernel (Drmac and Veselic;
// csrc/jacobi.cu), reorganised for a warp:
//   1. the core column l from C(I, :) (promoted to FP64), and the same numbers into R(:, J) so
//      that C and R hold one set of values of Z(I, J);
//   2. Householder QR with column pivoting, A P = Q R: the pivot by a warp arg-max of the column
//      norms, the reflector of column k broadcast from lane k, every lane updating its column;
//   3. X = R^H by a butterfly transpose of the register matrix (five shuffle stages), then
//      one-sided Jacobi on X with rotations accumulated in W: in round s of a sweep lane l is
//      paired with lane l ^ s (every pair once per sweep), both lanes compute the same rotation
//      from the same three inner products and each updates its own column;
//   4. sigma_l = |X W e_l|, Q W (unit vectors) by applying the reflectors, and the pinv
//      U = P (X W) diag(1 / sigma^2) (Q W)^H over the singular values kept by the threshold,
//      computed row by row after a second transpose.
// Replaces, for these cores, Zgesvd + kernel_Sinv + Zdgmm + Zgemm of the reference round
// (codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:1873-1924).
#include <cfloat>

#include "engine_internal.cuh"

namespace pskel {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return make_double2(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src));
}
__device__ __forceinline__ double2 shfl2x(double2 v, int mask) {
    return make_double2(__shfl_xor_sync(kFull, v.x, mask), __shfl_xor_sync(kFull, v.y, mask));
}
__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 promote2(double2 v) { return v; }
__device__ __forceinline__ double2 promote2(float2 v) { return make_double2(v.x, v.y); }

// In-register transpose of a 32 x 32 matrix held one column per lane (t[i] = M(i, lane)):
// afterwards t[j] = M(lane, j).
__device__ __forceinline__ void warp_transpose(double2 (&t)[32], int lane) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        const bool up = (lane & d) != 0;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            if (i & d) continue;
            const double2 send = up ? t[i] : t[i + d];
            const double2 recv = shfl2x(send, d);
            if (up) t[i] = recv;
            else t[i + d] = recv;
        }
    }
}

}  // namespace

template <typename S>
__global__ void __launch_bounds__(kWarpCoreThreads)
    warp_core_kernel(const WarpCoreJob *__restrict__ jobs, int count, SvdJob *svd, int max_sweeps) {
    const int lane = threadIdx.x & 31;
    const int wi = blockIdx.x * (kWarpCoreThreads / 32) + (threadIdx.x >> 5);
    if (wi >= count) return;  // uniform per warp
    const WarpCoreJob job = jobs[wi];
    const int n = job.n;
    const S *C = reinterpret_cast<const S *>(job.C);
    S *Rx = reinterpret_cast<S *>(job.Rx);
    const bool col = lane < n;

    // ---- 1. core column `lane`; R(:, J) takes the same numbers
    double2 a[32];
    const int jl = col ? job.J[lane] : 0;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        double2 v = make_double2(0.0, 0.0);
        if (col && k < n) {
            const S x = C[job.I[k] + (size_t)lane * job.m];
            Rx[k + (size_t)jl * job.ldr] = x;
            v = promote2(x);
        }
        a[k] = v;
    }
    double fro = 0;
#pragma unroll
    for (int k = 0; k < 32; ++k) fro = fma(a[k].x, a[k].x, fma(a[k].y, a[k].y, fro));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(kFull, fro, o);

    // ---- 2. Householder QR with column pivoting
    int piv = lane;               // original column of the column this lane holds
    double2 my_v0 = make_double2(0.0, 0.0);
    double my_coef = 0.0;
    for (int k = 0; k < n; ++k) {
        double s2 = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i >= k) s2 = fma(a[i].x, a[i].x, fma(a[i].y, a[i].y, s2));
        double best = (lane >= k && col) ? s2 : -1.0;
        int bi = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(kFull, best, o);
            const int oi = __shfl_xor_sync(kFull, bi, o);
            if (ob > best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        const int p = bi;
        if (p != k) {
            const int src = lane == k ? p : (lane == p ? k : lane);
#pragma unroll
            for (int i = 0; i < 32; ++i) a[i] = shfl2(a[i], src);
            piv = __shfl_sync(kFull, piv, src);
        }
        // reflector H = I - coef v v^H of column k (v = x - beta e_k, H x = beta e_k)
        double2 xk = make_double2(0.0, 0.0);
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i == k) xk = a[i];
        const double2 x0 = shfl2(xk, k);
        const double xn2 = fmax(best, 0.0);
        const double ax0 = hypot(x0.x, x0.y);
        const double xn = sqrt(xn2);
        double2 beta = make_double2(0.0, 0.0), v0 = make_double2(0.0, 0.0);
        double coef = 0.0;
        if (xn > 0.0) {
            const double2 ph = ax0 > 0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
            beta = make_double2(-ph.x * xn, -ph.y * xn);
            v0 = make_double2(x0.x - beta.x, x0.y - beta.y);
            const double v2 = xn2 - ax0 * ax0 + (v0.x * v0.x + v0.y * v0.y);
            coef = v2 > 0 ? 2.0 / v2 : 0.0;
        }
        // v (rows >= k) is read from lane k twice, for v^H a_j and for the update, instead of
        // being kept in registers next to the column
        const bool upd = lane > k && col && coef != 0.0;
        double dr = 0, di = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i >= k) {
                const double2 t = shfl2(a[i], k);
                const double2 x = i == k ? v0 : t;
                dr = fma(x.x, a[i].x, fma(x.y, a[i].y, dr));
                di = fma(x.x, a[i].y, fma(-x.y, a[i].x, di));
            }
        const double fr = coef * dr, fi = coef * di;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i >= k) {
                const double2 t = shfl2(a[i], k);
                const double2 x = i == k ? v0 : t;
                if (upd) {
                    a[i].x -= fr * x.x - fi * x.y;
                    a[i].y -= fr * x.y + fi * x.x;
                }
            }
        if (lane == k) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
                if (i == k) a[i] = beta;
            my_v0 = v0;
            my_coef = coef;
        }
    }
    // reflector tails (rows below the diagonal of column `lane`) to the job's scratch; R keeps
    // the upper triangle
    if (col) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i > lane && i < n) job.refl[i + (size_t)lane * n] = a[i];
    }
#pragma unroll
    for (int i = 0; i < 32; ++i)
        if (i > lane) a[i] = make_double2(0.0, 0.0);

    // ---- 3. X = R^H (lane i: conj of row i of R), one-sided Jacobi with W accumulated
    warp_transpose(a, lane);
#pragma unroll
    for (int i = 0; i < 32; ++i) a[i].y = -a[i].y;
    double2 w[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) w[i] = make_double2(i == lane ? 1.0 : 0.0, 0.0);
    const double tol = (double)(n > 1 ? n : 1) * DBL_EPSILON;
    const double zeps = (double)n * DBL_EPSILON;
    const double zero2 = zeps * zeps * fro;
    int sweep = 0, converged = 0;
    for (; sweep < max_sweeps; ++sweep) {
        int rotated = 0;
        for (int s = 1; s < 32; ++s) {
            const bool lo = lane < (lane ^ s);  // this lane holds the pair's first column
            double al = 0, be = 0, gr = 0, gi = 0;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const double2 y = shfl2x(a[i], s);
                const double2 f = lo ? a[i] : y, g = lo ? y : a[i];
                al = fma(f.x, f.x, fma(f.y, f.y, al));
                be = fma(g.x, g.x, fma(g.y, g.y, be));
                gr = fma(f.x, g.x, fma(f.y, g.y, gr));   // Re(conj(f) g)
                gi = fma(f.x, g.y, fma(-f.y, g.x, gi));  // Im(conj(f) g)
            }
            const double ag2 = fma(gr, gr, gi * gi);
            const bool doit = ag2 > tol * tol * al * be && ag2 > 0.0 && al > zero2 && be > zero2;
            double c = 1.0, sn = 0.0;
            double2 e = make_double2(1.0, 0.0);
            if (doit) {
                const double iag = rsqrt(ag2);
                const double zeta = (be - al) * 0.5 * iag;
                double tt;
                if (fabs(zeta) > 1e150) {
                    tt = 0.5 / zeta;
                } else {
                    const double w1 = fma(zeta, zeta, 1.0);
                    tt = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + w1 * rsqrt(w1));
                }
                c = rsqrt(fma(tt, tt, 1.0));
                sn = c * tt;
                e = make_double2(gr * iag, -gi * iag);  // e^{-i phi}
            }
            if (__any_sync(kFull, doit)) {
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const double2 y = shfl2x(a[i], s);
                    const double2 z = shfl2x(w[i], s);
                    if (doit) {
                        if (lo) {  // a_i <- c a_i - s e a_j
                            const double2 ey = cmul2(e, y), ez = cmul2(e, z);
                            a[i] = make_double2(c * a[i].x - sn * ey.x, c * a[i].y - sn * ey.y);
                            w[i] = make_double2(c * w[i].x - sn * ez.x, c * w[i].y - sn * ez.y);
                        } else {   // a_j <- s a_i + c e a_j
                            const double2 ex = cmul2(e, a[i]), ew = cmul2(e, w[i]);
                            a[i] = make_double2(sn * y.x + c * ex.x, sn * y.y + c * ex.y);
                            w[i] = make_double2(sn * z.x + c * ew.x, sn * z.y + c * ew.y);
                        }
                    }
                }
                rotated |= doit ? 1 : 0;
            }
        }
        if (!__any_sync(kFull, rotated)) {
            converged = 1;
            break;
        }
    }

    // ---- 4. sigma, Q W, and the pinv
    double s2 = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) s2 = fma(a[i].x, a[i].x, fma(a[i].y, a[i].y, s2));
    const double sigma = sqrt(s2);
    double smax = sigma;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(kFull, smax, o));
    const double thr = job.relative ? job.tau * smax : job.tau;
    const bool kept = col && sigma >= thr && sigma > 0;
    const double isig2 = kept ? 1.0 / (sigma * sigma) : 0.0;
    const unsigned kmask = __ballot_sync(kFull, kept);
    // q = Q w (own column): y <- H_k y for k = n - 1 .. 0
    for (int k = n - 1; k >= 0; --k) {
        const double coef = __shfl_sync(kFull, my_coef, k);
        const double2 v0 = shfl2(my_v0, k);
        if (coef == 0.0) continue;  // uniform
        // v_k: v0 at row k, the tail below (the same address in every lane: broadcast loads)
        double dr = 0, di = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i >= k && i < n) {
                const double2 x = i == k ? v0 : job.refl[i + (size_t)k * n];
                dr = fma(x.x, w[i].x, fma(x.y, w[i].y, dr));
                di = fma(x.x, w[i].y, fma(-x.y, w[i].x, di));
            }
        const double fr = coef * dr, fi = coef * di;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i >= k && i < n) {
                const double2 x = i == k ? v0 : job.refl[i + (size_t)k * n];
                w[i].x -= fr * x.x - fi * x.y;
                w[i].y -= fr * x.y + fi * x.x;
            }
    }
    // Q W to the job's scratch (row i, column lane), read back below by every lane
    if (col) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (i < n) job.qw[i + (size_t)lane * n] = w[i];
    }
    __syncwarp();
    // row `lane` (pivoted index) of X W: t[l] = B(lane, l)
    warp_transpose(a, lane);
    // U(piv_k, b) = sum_l B(k, l) conj(QW(b, l)) / sigma_l^2 for row k = lane, in two halves of
    // 16 columns b (16 accumulators next to the row of B)
    double fl[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) fl[l] = __shfl_sync(kFull, isig2, l);
#pragma unroll 1
    for (int h = 0; h < 32; h += 16) {
        if (h >= n) break;
        double2 acc[16];
#pragma unroll
        for (int bb = 0; bb < 16; ++bb) acc[bb] = make_double2(0.0, 0.0);
#pragma unroll
        for (int l = 0; l < 32; ++l) {
            if (!((kmask >> l) & 1u)) continue;  // uniform
            const double2 bl = make_double2(a[l].x * fl[l], a[l].y * fl[l]);
            const double2 *qrow = job.qw + (size_t)l * n + h;  // the same address in every lane
#pragma unroll
            for (int bb = 0; bb < 16; ++bb) {
                if (h + bb < n) {
                    const double2 q = qrow[bb];
                    acc[bb].x = fma(bl.x, q.x, fma(bl.y, q.y, acc[bb].x));
                    acc[bb].y = fma(bl.y, q.x, fma(-bl.x, q.y, acc[bb].y));
                }
            }
        }
        if (col) {
#pragma unroll
            for (int bb = 0; bb < 16; ++bb)
                if (h + bb < n) job.U[piv + (size_t)(h + bb) * n] = acc[bb];  // row piv = P e_lane
        }
    }
    if (col) job.sigma[lane] = sigma;
    if (lane == 0) {
        *job.rank = __popc(kmask);
        svd[job.svd_index].status = converged ? PSKEL_OK : PSKEL_ERR_NOCONV;
        svd[job.svd_index].sweeps = sweep + (converged ? 1 : 0);
    }
}

int launch_warp_core(const WarpCoreJob *d_jobs, int count, SvdJob *d_svd, int max_sweeps,
                     int precision, cudaStream_t stream) {
    if (count <= 0) return PSKEL_OK;
    const int per = kWarpCoreThreads / 32;
    const int grid = (count + per - 1) / per;
    if (precision == PSKEL_C64)
        warp_core_kernel<float2><<<grid, kWarpCoreThreads, 0, stream>>>(d_jobs, count, d_svd, max_sweeps);
    else
        warp_core_kernel<double2><<<grid, kWarpCoreThreads, 0, stream>>>(d_jobs, count, d_svd, max_sweeps);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

}  // namespace pskel
