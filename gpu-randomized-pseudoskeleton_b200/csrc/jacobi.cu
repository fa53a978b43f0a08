// Batched one-sided (Hestenes) Jacobi SVD in complex FP64, and the truncated pseudo-inverse.
//
// Replaces cusolverDnZgesvd + kernel_Sinv + cublasZdgmm + cublasZgemm of the reference CUR
// round (codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:1873-1924, and the
// cur_external_cuda.cu:217-367 helpers): pinv(A) = V diag(s >= thr ? 1/s : 0) U^H.
//
// Algorithm: for every column pair (i, j) with alpha = |a_i|^2, beta = |a_j|^2,
// gamma = a_i^H a_j = |gamma| e^{i phi}, zeta = (beta - alpha) / (2 |gamma|),
// t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), c = 1/sqrt(1 + t^2), s = c t:
//     a_i <- c a_i - s e^{-i phi} a_j,   a_j <- s a_i + c e^{-i phi} a_j
// (the same unitary applied to V). Pairs are visited in the round-robin (circle) order so
// that the n/2 pairs of a round are disjoint and run in parallel, one lane team per pair with
// shuffle reductions for the three inner products. A sweep with no rotation
// (|gamma| <= n eps sqrt(alpha beta) for every pair) ends the iteration; the sweep cap turns
// into PSKEL_ERR_NOCONV in the job's status.
//
// Two kernels:
//  * resident: the whole m x n matrix and V live in shared memory of one CTA (small n, the
//    sample counts the rank predictor produces);
//  * blocked: one CTA per matrix keeps 2b columns of A and V in shared memory at a time and
//    sweeps over all block pairs, the matrix itself staying in global memory (L2-resident);
//    used for the large sample counts of the reference's doubling rule.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "pskel_internal.cuh"

namespace pskel {

static constexpr int kSvdThreads = 512;
static constexpr size_t kSmemBudget = 220 * 1024;
static constexpr int kQrRowsPerLane = 8;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// circle-method player at position pos in round rho for nn (even) players
__device__ __forceinline__ int circle_player(int pos, int rho, int nn) {
    // (pos - 1 + rho) mod (nn - 1) without a division: both terms are below nn - 1
    int v = pos - 1 + rho;
    if (v >= nn - 1) v -= nn - 1;
    return pos == 0 ? 0 : v + 1;
}

// One round-robin sweep over the w columns held in shared memory (column-major, lds rows for
// A-part and ldv rows for V-part). Returns (via *rotated) whether any rotation happened.
// All threads of the CTA must call it.
__device__ void inner_sweep(double2 *sA, int m, double2 *sV, int nv, int w, int team,
                            double tol, double zero2, int *s_rot) {
    const int tid = threadIdx.x;
    const int nteams = blockDim.x / team;
    const int t = tid / team;
    const int g = tid % team;
    const int ww = w + (w & 1);
    const int npairs = ww / 2;
    const int iters = (npairs + nteams - 1) / nteams;
    for (int rho = 0; rho < ww - 1; ++rho) {
        for (int it = 0; it < iters; ++it) {
            const int kp = t + it * nteams;
            int ci = -1, cj = -1;
            if (kp < npairs) {
                ci = circle_player(kp, rho, ww);
                cj = circle_player(ww - 1 - kp, rho, ww);
                if (ci >= w || cj >= w) ci = cj = -1;
            }
            double al = 0, be = 0, gr = 0, gi = 0;
            if (ci >= 0) {
                const double2 *ai = sA + (size_t)ci * m;
                const double2 *aj = sA + (size_t)cj * m;
                for (int r = g; r < m; r += team) {
                    const double2 x = ai[r], y = aj[r];
                    al = fma(x.x, x.x, fma(x.y, x.y, al));
                    be = fma(y.x, y.x, fma(y.y, y.y, be));
                    gr = fma(x.x, y.x, fma(x.y, y.y, gr));   // Re(conj(x) y)
                    gi = fma(x.x, y.y, fma(-x.y, y.x, gi));  // Im(conj(x) y)
                }
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                if (o < team) {
                    al += __shfl_xor_sync(0xffffffffu, al, o);
                    be += __shfl_xor_sync(0xffffffffu, be, o);
                    gr += __shfl_xor_sync(0xffffffffu, gr, o);
                    gi += __shfl_xor_sync(0xffffffffu, gi, o);
                }
            }
            if (ci >= 0) {
                const double ag2 = fma(gr, gr, gi * gi);
                // columns with squared norm <= zero2 are numerically zero: rotating them
                // against anything only moves rounding noise (and on rank-deficient cores
                // would never satisfy the relative test), so they are left alone
                if (ag2 > tol * tol * al * be && ag2 > 0.0 && al > zero2 && be > zero2) {
                    // rotation from reciprocal square roots: 1/|gamma|, sqrt(1 + zeta^2) and
                    // c = 1/sqrt(1 + t^2), plus one reciprocal for t
                    const double iag = rsqrt(ag2);
                    const double zeta = (be - al) * 0.5 * iag;
                    double tt;
                    if (fabs(zeta) > 1e150) {
                        tt = 0.5 / zeta;
                    } else {
                        const double w1 = fma(zeta, zeta, 1.0);
                        tt = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + w1 * rsqrt(w1));
                    }
                    const double c = rsqrt(fma(tt, tt, 1.0));
                    const double s = c * tt;
                    const double2 e = make_double2(gr * iag, -gi * iag);  // e^{-i phi}
                    double2 *ai = sA + (size_t)ci * m;
                    double2 *aj = sA + (size_t)cj * m;
                    for (int r = g; r < m; r += team) {
                        const double2 x = ai[r];
                        const double2 y = cmul(e, aj[r]);
                        ai[r] = make_double2(c * x.x - s * y.x, c * x.y - s * y.y);
                        aj[r] = make_double2(s * x.x + c * y.x, s * x.y + c * y.y);
                    }
                    double2 *vi = sV + (size_t)ci * nv;
                    double2 *vj = sV + (size_t)cj * nv;
                    for (int r = g; r < nv; r += team) {
                        const double2 x = vi[r];
                        const double2 y = cmul(e, vj[r]);
                        vi[r] = make_double2(c * x.x - s * y.x, c * x.y - s * y.y);
                        vj[r] = make_double2(s * x.x + c * y.x, s * x.y + c * y.y);
                    }
                    if (g == 0) *s_rot = 1;
                }
            }
        }
        __syncthreads();
    }
}

// Squared column norm below which a column counts as zero: (m eps)^2 ||A||_F^2 (the
// Frobenius norm is invariant under the rotations). All threads of the CTA must call it.
__device__ double zero_column_norm2(const double2 *A, size_t count, int m) {
    __shared__ double red[32];
    double s = 0;
    for (size_t i = threadIdx.x; i < count; i += blockDim.x) s = fma(A[i].x, A[i].x, fma(A[i].y, A[i].y, s));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    __syncthreads();
    const double e = (double)m * DBL_EPSILON;
    return e * e * t;
}

// Lanes per column pair in a Jacobi round over w columns of m rows: as many as keep at least
// two rows per lane while all w/2 pairs of a round still run at once in the CTA, at most 8 up
// to 64 columns (16 lanes per pair made the cores of 32-63 columns take 512-thread CTAs, two
// per SM; with 8 they take the 256-thread instantiation: pinv of the 30,720-RWG round 14.8 ->
// 13.3 ms) and 16 above (the few large cores of a second round, whose latency sets the round's:
// one 1024-thread CTA per core).
__device__ int jacobi_team(int m, int w, int threads) {
    const int npairs = (w + 1) / 2;
    int t = 1;
    const int cap = w > 64 ? 16 : 8;
    while (t < cap && 2 * t * 2 <= m && 2 * t * npairs <= threads) t <<= 1;
    return t;
}

__device__ int pick_team(int m) {
    int t = 1;
    while (t < 32 && 2 * t * 2 <= m) t <<= 1;  // about two rows per lane
    return t;
}

// Singular values (column norms), permutation by decreasing value, and write-back helpers.
__device__ void finish_sigma(const double2 *A, int lda, int m, int n, double *sigma, int *perm) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double s = 0;
        const double2 *a = A + (size_t)j * lda;
        for (int r = 0; r < m; ++r) s = fma(a[r].x, a[r].x, fma(a[r].y, a[r].y, s));
        sigma[j] = sqrt(s);
    }
    __syncthreads();
    if (perm) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double sj = sigma[j];
            int rank = 0;
            for (int i = 0; i < n; ++i) {
                const double si = sigma[i];
                rank += (si > sj) || (si == sj && i < j);
            }
            perm[rank] = j;
        }
    }
}

// Resident kernel, QR-preconditioned (the preconditioned one-sided Jacobi of Drmac and
// Veselic):
//   1. Householder QR with column pivoting, A P = Q R, in shared memory (the reflectors stay
//      below the diagonal);
//   2. one-sided Jacobi on X = R^H (n x n): X W = B with orthogonal columns, sigma_j = |B_j|.
//      R^H of a pivoted QR is graded, which cuts the sweeps from about 15-25 to 6-7 on the
//      far-field cores;
//   3. V = P B diag(1/sigma) (the left singular vectors of X are the right ones of A) and
//      A V = Q W diag(sigma), applying the reflectors to W diag(sigma) column by column. Each
//      column of A V then carries an error relative to its own norm (forming A V as the
//      product of A and V would carry eps |A| in every column, which the inverse of a small
//      singular value amplifies).
// Columns of B whose norm is zero give zero columns of V.
// Two instantiations: up to 1024 threads with at most 64 registers (the cores of more than 64
// columns), and up to 256 threads with at least four CTAs per SM (64 registers; the smaller
// classes launch 64-128 threads and fit more) for the classes of small cores: more resident
// cores per SM hide the latency of the rotation rounds (pinv of the 30,720-RWG round: 13.3 ms
// with a five-CTA cap of 48 registers and spills, 12.8 ms with four). Without a register cap
// the compiler takes 104 registers.
template <int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    svd_resident_kernel(SvdJob *jobs, const int *idx_map, int max_sweeps) {
    // blockDim.x is a multiple of 32 chosen by the launcher (enough lane teams for one round)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SvdJob &job = jobs[idx_map[blockIdx.x]];
    const int m = job.m, n = job.n;
    // square cores (m == n) park the reflectors in job.V during the Jacobi sweeps and let W
    // take their place, so that a CTA needs 2 n^2 complex values of shared memory, not 3 n^2
    const bool compact = m == n;
    double2 *sA = reinterpret_cast<double2 *>(smem_raw);  // m x n: R and the reflectors
    double2 *sX = sA + (size_t)m * n;                      // n x n: R^H, then B
    double2 *sW = compact ? sA : sX + (size_t)n * n;       // n x n: rotations
    double2 *sv0 = sX + (size_t)n * n + (compact ? 0 : (size_t)n * n);  // n: first entry of each reflector
    double *scoef = reinterpret_cast<double *>(sv0 + n);   // n: 2 / |v|^2
    double *snrm = scoef + n;                              // n
    int *spiv = reinterpret_cast<int *>(snrm + n);         // n
    __shared__ int s_rot, s_p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int idx = tid; idx < m * n; idx += blockDim.x) sA[idx] = job.A[idx];
    for (int j = tid; j < n; j += blockDim.x) spiv[j] = j;
    __syncthreads();
    // ---- 1. QR with column pivoting; team per column for the norms and the reflector updates
    const int qteam = pick_team(m);
    const int qteams = blockDim.x / qteam;
    const int qt = tid / qteam, qg = tid % qteam;
    for (int j0 = 0; j0 < n; j0 += qteams) {
        const int j = j0 + qt;
        double s2 = 0;
        if (j < n)
            for (int i = qg; i < m; i += qteam) {
                const double2 a = sA[i + (size_t)j * m];
                s2 = fma(a.x, a.x, fma(a.y, a.y, s2));
            }
        for (int o = 1; o < qteam; o <<= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        if (j < n && qg == 0) snrm[j] = s2;
    }
    __syncthreads();
    // truncated form (job.trunc > 0): the QR stops at the first k whose trailing block
    // R(k:, k:) has Frobenius norm <= trunc (the sum of the remaining column norms), and the
    // rest works on the leading kp rows of R
    const double trunc2 = job.trunc > 0 ? job.trunc * job.trunc : -1.0;
    int kp = n;
    for (int k = 0; k < n; ++k) {
        if (warp == 0) {
            // pivot: the remaining column of largest norm
            double best = -1.0, rest = 0.0;
            int bi = k;
            for (int j = k + lane; j < n; j += 32) {
                rest += snrm[j];
                if (snrm[j] > best) { best = snrm[j]; bi = j; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                rest += __shfl_xor_sync(0xffffffffu, rest, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (lane == 0) s_p = (k > 0 && rest <= trunc2) ? -1 : bi;
        }
        __syncthreads();
        const int p = s_p;
        if (p < 0) {  // uniform: every thread read the same s_p
            kp = k;
            break;
        }
        if (p != k) {
            for (int i = tid; i < m; i += blockDim.x) {
                const double2 t = sA[i + (size_t)k * m];
                sA[i + (size_t)k * m] = sA[i + (size_t)p * m];
                sA[i + (size_t)p * m] = t;
            }
            if (tid == 0) {
                const double t = snrm[k]; snrm[k] = snrm[p]; snrm[p] = t;
                const int ti = spiv[k]; spiv[k] = spiv[p]; spiv[p] = ti;
            }
            __syncthreads();
        }
        if (warp == 0) {
            // reflector H = I - coef v v^H with v = x - beta e_1, H x = beta e_1; v(0) goes to
            // sv0, the tail of v is x's own tail, R(k, k) = beta
            double x2 = 0;
            for (int i = k + lane; i < m; i += 32) {
                const double2 a = sA[i + (size_t)k * m];
                x2 = fma(a.x, a.x, fma(a.y, a.y, x2));
            }
            for (int o = 16; o > 0; o >>= 1) x2 += __shfl_xor_sync(0xffffffffu, x2, o);
            if (lane == 0) {
                const double2 x0 = sA[k + (size_t)k * m];
                const double ax0 = hypot(x0.x, x0.y);
                const double xn = sqrt(x2);
                if (xn == 0.0) {
                    sv0[k] = make_double2(0.0, 0.0);
                    scoef[k] = 0.0;
                } else {
                    const double2 ph = ax0 > 0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
                    const double2 beta = make_double2(-ph.x * xn, -ph.y * xn);
                    const double2 v0 = make_double2(x0.x - beta.x, x0.y - beta.y);
                    const double v2 = x2 - ax0 * ax0 + (v0.x * v0.x + v0.y * v0.y);
                    sv0[k] = v0;
                    scoef[k] = v2 > 0 ? 2.0 / v2 : 0.0;
                    sA[k + (size_t)k * m] = beta;
                }
            }
        }
        __syncthreads();
        const double coef = scoef[k];
        const double2 v0 = sv0[k];
        const double2 *v = sA + (size_t)k * m;  // v(i) = sA(i, k) for i > k
        for (int j0 = k + 1; j0 < n; j0 += qteams) {
            const int j = j0 + qt;
            double dr = 0, di = 0;
            double2 *a = sA + (size_t)j * m;
            if (j < n && coef != 0.0)
                for (int i = k + qg; i < m; i += qteam) {  // v^H a_j
                    const double2 x = i == k ? v0 : v[i], y = a[i];
                    dr = fma(x.x, y.x, fma(x.y, y.y, dr));
                    di = fma(x.x, y.y, fma(-x.y, y.x, di));
                }
            for (int o = 1; o < qteam; o <<= 1) {
                dr += __shfl_xor_sync(0xffffffffu, dr, o);
                di += __shfl_xor_sync(0xffffffffu, di, o);
            }
            double s2 = 0;
            if (j < n) {
                const double fr = coef * dr, fi = coef * di;
                for (int i = k + qg; i < m; i += qteam) {  // a_j -= f v, then |a_j(k+1:)|^2
                    const double2 x = i == k ? v0 : v[i];
                    double2 y = a[i];
                    y.x -= fr * x.x - fi * x.y;
                    y.y -= fr * x.y + fi * x.x;
                    a[i] = y;
                    if (i > k) s2 = fma(y.x, y.x, fma(y.y, y.y, s2));
                }
            }
            for (int o = 1; o < qteam; o <<= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            if (j < n && qg == 0) snrm[j] = s2;
        }
        __syncthreads();
    }
    // ---- 2. one-sided Jacobi on X = R^H, rotations accumulated in W
    for (int idx = tid; idx < n * kp; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        const double2 r = sA[j + (size_t)i * m];  // R(j, i)
        sX[idx] = j <= i ? make_double2(r.x, -r.y) : make_double2(0.0, 0.0);
    }
    const double2 *refl = sA;  // reflector k: v0 = sv0[k], tail refl[k+1 .. m-1 + k m]
    if (compact) {
        for (int idx = tid; idx < m * n; idx += blockDim.x) job.V[idx] = sA[idx];
        refl = job.V;
        __syncthreads();
    }
    for (int idx = tid; idx < kp * kp; idx += blockDim.x) {
        const int i = idx % kp, j = idx / kp;
        sW[idx] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    const int team = jacobi_team(n, kp, blockDim.x);
    const double tol = (double)(n > 1 ? n : 1) * DBL_EPSILON;
    const double zero2 = zero_column_norm2(sX, (size_t)n * kp, n);
    int sweep = 0, converged = 0;
    for (; sweep < max_sweeps; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        inner_sweep(sX, n, sW, kp, kp, team, tol, zero2, &s_rot);
        __syncthreads();
        const int rot = s_rot;
        __syncthreads();
        if (!rot) {
            converged = 1;
            break;
        }
    }
    // ---- 3. sigma, V = P B / sigma, A V = Q W sigma (columns kp.. of the truncated form: 0)
    for (int j = tid; j < n; j += blockDim.x) {
        double s2 = 0;
        if (j < kp)
            for (int i = 0; i < n; ++i) {
                const double2 b = sX[i + (size_t)j * n];
                s2 = fma(b.x, b.x, fma(b.y, b.y, s2));
            }
        snrm[j] = sqrt(s2);
    }
    __syncthreads();
    // A V column j by one team: y = [W(:, j) sigma_j; 0], then y <- H_k y for k = kp-1 .. 0;
    // the team's lanes hold rows qg, qg + qteam, ... (at most kQrRowsPerLane each)
    for (int j0 = 0; j0 < n; j0 += qteams) {
        const int j = j0 + qt;
        const bool on = j < n;
        const double sg = (on && j < kp) ? snrm[j] : 0.0;
        double2 y[kQrRowsPerLane];
#pragma unroll
        for (int e = 0; e < kQrRowsPerLane; ++e) {
            const int i = qg + e * qteam;
            const double2 w = (on && j < kp && i < kp) ? sW[i + (size_t)j * kp] : make_double2(0.0, 0.0);
            y[e] = make_double2(w.x * sg, w.y * sg);
        }
        for (int k = kp - 1; k >= 0; --k) {
            const double coef = scoef[k];
            const double2 v0 = sv0[k];
            double dr = 0, di = 0;
#pragma unroll
            for (int e = 0; e < kQrRowsPerLane; ++e) {
                const int i = qg + e * qteam;
                if (i >= k && i < m) {
                    const double2 x = i == k ? v0 : refl[i + (size_t)k * m];
                    dr = fma(x.x, y[e].x, fma(x.y, y[e].y, dr));
                    di = fma(x.x, y[e].y, fma(-x.y, y[e].x, di));
                }
            }
            for (int o = 1; o < qteam; o <<= 1) {
                dr += __shfl_xor_sync(0xffffffffu, dr, o);
                di += __shfl_xor_sync(0xffffffffu, di, o);
            }
            const double fr = coef * dr, fi = coef * di;
#pragma unroll
            for (int e = 0; e < kQrRowsPerLane; ++e) {
                const int i = qg + e * qteam;
                if (i >= k && i < m) {
                    const double2 x = i == k ? v0 : refl[i + (size_t)k * m];
                    y[e].x -= fr * x.x - fi * x.y;
                    y[e].y -= fr * x.y + fi * x.x;
                }
            }
        }
        if (on) {
#pragma unroll
            for (int e = 0; e < kQrRowsPerLane; ++e) {
                const int i = qg + e * qteam;
                if (i < m) job.A[i + (size_t)j * m] = y[e];
            }
        }
    }
    __syncthreads();  // the reflectors in job.V are read until here
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        const double sg = snrm[j];
        const double f = sg > 0 ? 1.0 / sg : 0.0;
        const double2 b = j < kp ? sX[idx] : make_double2(0.0, 0.0);
        job.V[spiv[i] + (size_t)j * n] = make_double2(b.x * f, b.y * f);
    }
    for (int j = tid; j < n; j += blockDim.x) job.sigma[j] = snrm[j];
    if (job.perm) {
        for (int j = tid; j < n; j += blockDim.x) {
            const double sj = snrm[j];
            int rank = 0;
            for (int i = 0; i < n; ++i) {
                const double si = snrm[i];
                rank += (si > sj) || (si == sj && i < j);
            }
            job.perm[rank] = j;
        }
    }
    if (tid == 0) {
        job.status = converged ? PSKEL_OK : PSKEL_ERR_NOCONV;
        job.sweeps = sweep + (converged ? 1 : 0);
    }
}

// Blocked variant: 2b columns at a time in shared memory.
__global__ void __launch_bounds__(kSvdThreads)
    svd_blocked_kernel(SvdJob *jobs, const int *idx_map, int max_sweeps, int smem_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SvdJob &job = jobs[idx_map[blockIdx.x]];
    const int m = job.m, n = job.n;
    int b = (int)(smem_bytes / (2 * (size_t)(m + n) * sizeof(double2)));
    if (b < 1) b = 1;
    if (b > n) b = n;
    int nb = (n + b - 1) / b;
    double2 *sA = reinterpret_cast<double2 *>(smem_raw);  // m x 2b
    double2 *sV = sA + (size_t)m * 2 * b;                  // n x 2b
    __shared__ int s_rot;
    __shared__ int s_any;
    // V = I
    for (size_t idx = threadIdx.x; idx < (size_t)n * n; idx += blockDim.x)
        job.V[idx] = make_double2((idx % n) == (idx / n) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    const int team = pick_team(m);
    const double tol = (double)(m > 1 ? m : 1) * DBL_EPSILON;
    const double zero2 = zero_column_norm2(job.A, (size_t)m * n, m);
    int sweep = 0, converged = 0;
    if (nb == 1) nb = 2;  // a single block still needs its own inner sweep: pair it with empty
    for (; sweep < max_sweeps; ++sweep) {
        if (threadIdx.x == 0) s_any = 0;
        for (int P = 0; P < nb; ++P) {
            for (int Q = P + 1; Q < nb; ++Q) {
                const int p0 = P * b, pw = max(0, min(b, n - p0));
                const int q0 = Q * b, qw = max(0, min(b, n - q0));
                const int w = pw + qw;
                if (w == 0) continue;
                // load columns [p0, p0+pw) and [q0, q0+qw)
                for (size_t idx = threadIdx.x; idx < (size_t)m * w; idx += blockDim.x) {
                    const int c = (int)(idx / m), r = (int)(idx % m);
                    const int gc = c < pw ? p0 + c : q0 + (c - pw);
                    sA[idx] = job.A[(size_t)gc * m + r];
                }
                for (size_t idx = threadIdx.x; idx < (size_t)n * w; idx += blockDim.x) {
                    const int c = (int)(idx / n), r = (int)(idx % n);
                    const int gc = c < pw ? p0 + c : q0 + (c - pw);
                    sV[idx] = job.V[(size_t)gc * n + r];
                }
                if (threadIdx.x == 0) s_rot = 0;
                __syncthreads();
                inner_sweep(sA, m, sV, n, w, team, tol, zero2, &s_rot);
                __syncthreads();
                if (s_rot) {
                    for (size_t idx = threadIdx.x; idx < (size_t)m * w; idx += blockDim.x) {
                        const int c = (int)(idx / m), r = (int)(idx % m);
                        const int gc = c < pw ? p0 + c : q0 + (c - pw);
                        job.A[(size_t)gc * m + r] = sA[idx];
                    }
                    for (size_t idx = threadIdx.x; idx < (size_t)n * w; idx += blockDim.x) {
                        const int c = (int)(idx / n), r = (int)(idx % n);
                        const int gc = c < pw ? p0 + c : q0 + (c - pw);
                        job.V[(size_t)gc * n + r] = sV[idx];
                    }
                    if (threadIdx.x == 0) s_any = 1;
                }
                __syncthreads();
            }
        }
        __syncthreads();
        const int any = s_any;
        __syncthreads();
        if (!any) {
            converged = 1;
            break;
        }
    }
    __syncthreads();
    finish_sigma(job.A, m, m, n, job.sigma, job.perm);
    if (threadIdx.x == 0) {
        job.status = converged ? PSKEL_OK : PSKEL_ERR_NOCONV;
        job.sweeps = sweep + (converged ? 1 : 0);
    }
}

static size_t resident_bytes(int m, int n) {
    const size_t w = m == n ? 0 : (size_t)n * n;  // square cores keep W over the QR workspace
    return sizeof(double2) * ((size_t)m * n + (size_t)n * n + w + n) +
           (2 * sizeof(double) + sizeof(int)) * (size_t)n;
}

// the resident kernel holds the m rows of one column of A V in the registers of a lane team
// (pick_team(m) lanes, at most kQrRowsPerLane rows each)
static bool resident_fits(int m, int n) {
    int t = 1;
    while (t < 32 && 2 * t * 2 <= m) t <<= 1;
    return resident_bytes(m, n) <= kSmemBudget && m <= t * kQrRowsPerLane;
}

// resident size classes: cores of n <= 16, 24, 32, 40, 48, 64, 80 columns get their own launch
// with a shared-memory size and a thread count fitted to the class, so that one large core does
// not dictate the occupancy of every CTA (seven classes instead of five: pinv of the 30,720-RWG
// round 12.8 -> 12.4 ms)
static int size_class(int n) { return n <= 16 ? 0 : n <= 24 ? 1 : n <= 32 ? 2 : n <= 40 ? 3 : n <= 48 ? 4 : n <= 64 ? 5 : 6; }

static int resident_threads_for(int n) {
    int team = 1;
    const int cap = n > 64 ? 16 : 8;
    while (team < cap && 4 * team <= n) team <<= 1;  // jacobi_team without the thread cap
    int want = team * ((n + 1) / 2);
    want = (want + 31) / 32 * 32;
    return want < 64 ? 64 : (want > 1024 ? 1024 : want);
}

int svd_plan(const std::vector<SvdJob> &h_jobs, SvdPlan &plan) {
    return svd_plan(h_jobs.data(), (int)h_jobs.size(), plan);
}

int svd_plan(const SvdJob *h_jobs, int nj, SvdPlan &plan) {
    plan.idx.clear();
    plan.idx.reserve(nj);
    plan.res.clear();
    std::vector<std::vector<int>> cls(7);
    std::vector<int> blk;
    std::vector<size_t> smem(7, 0);
    std::vector<int> maxn(7, 0);
    for (int i = 0; i < nj; ++i) {
        const SvdJob &j = h_jobs[i];
        if (j.m < j.n || j.n <= 0 || j.m <= 0) {
            set_error(PSKEL_ERR_ARG, "svd: job %d has m=%d < n=%d or is empty", i, j.m, j.n);
            return PSKEL_ERR_ARG;
        }
        if (resident_fits(j.m, j.n)) {
            const int c = size_class(j.n);
            cls[c].push_back(i);
            smem[c] = std::max(smem[c], resident_bytes(j.m, j.n));
            maxn[c] = std::max(maxn[c], j.n);
        } else {
            blk.push_back(i);
        }
    }
    for (int c = 0; c < 7; ++c) {
        if (cls[c].empty()) continue;
        plan.res.push_back(SvdPlan::Cls{(int)plan.idx.size(), (int)cls[c].size(), smem[c],
                                        resident_threads_for(maxn[c])});
        plan.idx.insert(plan.idx.end(), cls[c].begin(), cls[c].end());
    }
    plan.blk_off = (int)plan.idx.size();
    plan.blk_count = (int)blk.size();
    plan.idx.insert(plan.idx.end(), blk.begin(), blk.end());
    return PSKEL_OK;
}

int svd_resident_attr() {
    PSKEL_TRY(ensure_smem_attr(svd_resident_kernel<1024, 1>, kSmemBudget));
    PSKEL_TRY(ensure_smem_attr(svd_resident_kernel<256, 4>, kSmemBudget));
    return ensure_smem_attr(svd_blocked_kernel, kSmemBudget);
}

int svd_streams_create(SvdStreams &p) {
    if (p.ready) return PSKEL_OK;
    // high priority: in a pipelined round the SVD classes take the SM slots that retiring fill
    // CTAs free before further fill CTAs do
    int lo_pri = 0, hi_pri = 0;
    PSKEL_CUDA(cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
    for (int i = 0; i < kSvdAux; ++i) {
        PSKEL_CUDA(cudaStreamCreateWithPriority(&p.aux[i], cudaStreamNonBlocking, hi_pri));
        PSKEL_CUDA(cudaEventCreateWithFlags(&p.join[i], cudaEventDisableTiming));
    }
    PSKEL_CUDA(cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming));
    p.ready = true;
    return PSKEL_OK;
}

void svd_streams_destroy(SvdStreams &p) {
    if (!p.ready) return;
    for (int i = 0; i < kSvdAux; ++i) {
        cudaStreamDestroy(p.aux[i]);
        cudaEventDestroy(p.join[i]);
    }
    cudaEventDestroy(p.fork);
    p.ready = false;
}

int svd_launch(SvdJob *d_jobs, const int *d_idx, const SvdPlan &plan, int max_sweeps,
               cudaStream_t stream, const SvdStreams *par) {
    PSKEL_TRY(svd_resident_attr());
    const int nl = (int)plan.res.size() + (plan.blk_count > 0 ? 1 : 0);
    // launch l on the main stream (l = 0) or on side stream l - 1 (the classes are independent)
    const bool fan = par && par->ready && nl > 1;
    const int used = fan ? std::min(nl - 1, kSvdAux) : 0;
    if (fan) {
        PSKEL_CUDA(cudaEventRecord(par->fork, stream));
        for (int a = 0; a < used; ++a) PSKEL_CUDA(cudaStreamWaitEvent(par->aux[a], par->fork, 0));
    }
    auto lane = [&](int l) -> cudaStream_t { return (!fan || l == 0) ? stream : par->aux[(l - 1) % kSvdAux]; };
    int l = 0;
    // the class with the most jobs on the main stream
    std::vector<int> order(plan.res.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return plan.res[a].count > plan.res[b].count; });
    for (int ci : order) {
        const SvdPlan::Cls &c = plan.res[ci];
        cudaStream_t s = lane(l++);
        if (c.threads <= 256)
            svd_resident_kernel<256, 4><<<c.count, c.threads, c.smem, s>>>(d_jobs, d_idx + c.off, max_sweeps);
        else
            svd_resident_kernel<1024, 1><<<c.count, c.threads, c.smem, s>>>(d_jobs, d_idx + c.off, max_sweeps);
        PSKEL_LAUNCHED(1);
    }
    if (plan.blk_count > 0) {
        cudaStream_t s = lane(l++);
        svd_blocked_kernel<<<plan.blk_count, kSvdThreads, kSmemBudget, s>>>(
            d_jobs, d_idx + plan.blk_off, max_sweeps, (int)kSmemBudget);
        PSKEL_LAUNCHED(1);
    }
    for (int a = 0; a < used; ++a) {
        PSKEL_CUDA(cudaEventRecord(par->join[a], par->aux[a]));
        PSKEL_CUDA(cudaStreamWaitEvent(stream, par->join[a], 0));
    }
    return PSKEL_OK;
}

int svd_launch_single_resident(SvdJob *d_job, const int *d_idx0, int m, int n, int max_sweeps,
                               cudaStream_t stream) {
    SvdPlan plan;
    plan.res.push_back(SvdPlan::Cls{0, 1, resident_bytes(m, n), resident_threads_for(n)});
    plan.blk_off = 1;
    plan.blk_count = 0;
    return svd_launch(d_job, d_idx0, plan, max_sweeps, stream);
}

int batched_svd(SvdJob *d_jobs, const std::vector<SvdJob> &h_jobs, int max_sweeps,
                cudaStream_t stream, DevBuf &scratch) {
    if (h_jobs.empty()) return PSKEL_OK;
    SvdPlan plan;
    PSKEL_TRY(svd_plan(h_jobs, plan));
    PSKEL_TRY(scratch.reserve(sizeof(int) * plan.idx.size()));
    int *d_idx = scratch.as<int>();
    PSKEL_CUDA(cudaMemcpyAsync(d_idx, plan.idx.data(), sizeof(int) * plan.idx.size(),
                               cudaMemcpyHostToDevice, stream));
    return svd_launch(d_jobs, d_idx, plan, max_sweeps, stream);
}

// ------------------------------------------------------------------ pseudo-inverse
// P (n x m) = sum over kept j of (1/sigma_j^2) V[:, j] conj(AV[:, j])^T; one CTA per 32x32
// output tile of one job (grid.x = job, grid.y = tile), K loop over the n columns in chunks of
// 16.
__global__ void __launch_bounds__(256) pinv_kernel(const PinvJob *jobs) {
    const PinvJob job = jobs[blockIdx.x];
    const int n = job.n, m = job.m;
    const int tiles_a = (n + 31) / 32;
    const int tiles_b = (m + 31) / 32;
    if ((int)blockIdx.y >= tiles_a * tiles_b) return;
    const int a0 = (blockIdx.y % tiles_a) * 32;
    const int b0 = (blockIdx.y / tiles_a) * 32;
    __shared__ double smax;
    __shared__ double w[16];
    __shared__ double2 sVt[16][33];
    __shared__ double2 sAt[16][33];
    if (threadIdx.x == 0) {
        double mx = 0;
        for (int j = 0; j < n; ++j) mx = fmax(mx, job.sigma[j]);
        smax = mx;
    }
    __syncthreads();
    const double thr = job.relative ? job.tau * smax : job.tau;
    const int tx = threadIdx.x % 32;  // output row a0 + tx
    const int ty = threadIdx.x / 32;  // 8 groups of 4 output columns
    double2 acc[4];
    for (int c = 0; c < 4; ++c) acc[c] = make_double2(0, 0);
    for (int k0 = 0; k0 < n; k0 += 16) {
        if (threadIdx.x < 16) {
            const int j = k0 + threadIdx.x;
            double wj = 0;
            if (j < n) {
                const double s = job.sigma[j];
                if (s >= thr && s > 0) wj = 1.0 / (s * s);
            }
            w[threadIdx.x] = wj;
        }
        for (int idx = threadIdx.x; idx < 16 * 32; idx += 256) {
            const int kk = idx / 32, r = idx % 32;
            const int j = k0 + kk;
            sVt[kk][r] = (j < n && a0 + r < n) ? job.V[(size_t)j * n + a0 + r] : make_double2(0, 0);
            sAt[kk][r] = (j < n && b0 + r < m) ? job.AV[(size_t)j * m + b0 + r] : make_double2(0, 0);
        }
        __syncthreads();
        for (int kk = 0; kk < 16; ++kk) {
            const double wk = w[kk];
            if (wk == 0.0) continue;
            const double2 v = sVt[kk][tx];
            const double2 vw = make_double2(v.x * wk, v.y * wk);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double2 a = sAt[kk][ty * 4 + c];  // conj(a)
                acc[c].x = fma(vw.x, a.x, fma(vw.y, a.y, acc[c].x));
                acc[c].y = fma(vw.y, a.x, fma(-vw.x, a.y, acc[c].y));
            }
        }
        __syncthreads();
    }
    const int ra = a0 + tx;
    if (ra < n) {
        for (int c = 0; c < 4; ++c) {
            const int cb = b0 + ty * 4 + c;
            if (cb < m) job.P[ra + (size_t)cb * n] = acc[c];
        }
    }
    if (blockIdx.y == 0 && threadIdx.x == 0 && job.rank) {
        int k = 0;
        for (int j = 0; j < n; ++j) k += (job.sigma[j] >= thr && job.sigma[j] > 0);
        *job.rank = k;
    }
}

int batched_pinv(const PinvJob *d_jobs, int njobs, int max_tiles, cudaStream_t stream) {
    if (njobs <= 0) return PSKEL_OK;
    if (max_tiles > 65535) {
        set_error(PSKEL_ERR_ARG, "pinv: %d output tiles per matrix exceed the grid limit", max_tiles);
        return PSKEL_ERR_ARG;
    }
    dim3 grid(njobs, max_tiles);
    pinv_kernel<<<grid, 256, 0, stream>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

}  // namespace pskel
