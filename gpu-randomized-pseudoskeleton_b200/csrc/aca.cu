// Adaptive cross approximation of every far block at once: the comparison compressor of the
// reference's ACA-vs-CUR study, in the same batched framework as the CUR engine.
//
// The reference's ACA (ACA_julia.jl:2-112; C twin c_ACA.c:327-558 on a precomputed block; the
// method of Zhao, Vouvakis and Lee, IEEE Trans. EMC 2005) builds Z ~ U V one cross at a time,
// computing each pivot row and column of the block on demand:
//   row 1 first; per step: residual row R_i = Z(i, :) - U(i, :) V, column pivot j = argmax over
//   unused columns of |R_i|, V_k = R_i / R_i(j) (stop on a zero pivot), residual column
//   R_j = Z(:, j) - U V(:, j) = U_k, ||U V||_F^2 updated by 2 sum_t Re((U_t^H U_k)(V_k V_t^H))
//   + ||U_k||^2 ||V_k||^2, stop when ||U_k|| ||V_k|| <= tol ||U V||_F (from the second step),
//   next row = argmax over unused rows of |R_j|.
//
// Device design: one CTA (128 threads, 64 registers: 8 CTAs per SM) per block runs the whole loop; the block's row and column
// residuals, used-index marks and the pivot RWG's quadrature record live in shared memory; U
// (m x kmax, column-major) and V (kmax x n, row-major) in a per-call global buffer. Every entry
// is computed in FP64 from the 7-point quadrature records: the pivot RWG's record is staged in
// shared memory and each thread streams the other RWG's points. Pivot searches break ties toward
// the lower index (Julia's findmax). In the symmetric mode only one block of each (t, s) / (s, t)
// pair is approximated; the other is its transpose (U_b = V_p^T, V_b = U_p^T).
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine_internal.cuh"
#include "zgemm.cuh"

namespace pskel {
namespace {

constexpr int kAcaThreads = 128;
constexpr int kAcaWarps = kAcaThreads / 32;
constexpr int kAcaMaxSide = 2048;  // largest group (rows or columns) of an ACA block
constexpr int kAcaQ = 7;
constexpr int kAcaNP = 2 * kAcaQ;

struct AcaJob {
    const int *rows, *cols;  // global RWG ids (device)
    double2 *U;              // m x kmax, column-major
    double2 *V;              // kmax x n, row t at V + t n
    int *I, *J;              // pivots (local indices), kmax each
    int *out;                // k, status
    int m, n, kmax;
};

// Z(a, b) / (eta / 4 pi) from two quadrature records (fields x, y, z, ux, uy, uz, d of the 2Q
// points): sum_{p,q} (d_p d_q / k - k u_p . u_q) (sin kR + j cos kR) / R. rs: record in shared
// memory (inner loop, broadcast reads), rg: record in global memory (outer loop).
__device__ __forceinline__ double2 rec_entry(const double *__restrict__ rs,
                                             const double *__restrict__ rg, double k, double kinv) {
    double re = 0.0, im = 0.0;
#pragma unroll 1
    for (int q = 0; q < kAcaNP; ++q) {
        const double xq = rg[q], yq = rg[kAcaNP + q], zq = rg[2 * kAcaNP + q];
        const double uxq = rg[3 * kAcaNP + q], uyq = rg[4 * kAcaNP + q], uzq = rg[5 * kAcaNP + q];
        const double dq = rg[6 * kAcaNP + q] * kinv;
#pragma unroll 2
        for (int p = 0; p < kAcaNP; ++p) {
            const double dx = rs[p] - xq, dy = rs[kAcaNP + p] - yq, dz = rs[2 * kAcaNP + p] - zq;
            const double R = sqrt(dx * dx + dy * dy + dz * dz);
            const double A = rs[6 * kAcaNP + p] * dq -
                             k * (rs[3 * kAcaNP + p] * uxq + rs[4 * kAcaNP + p] * uyq + rs[5 * kAcaNP + p] * uzq);
            double s, c;
            sincos(k * R, &s, &c);
            const double f = A / R;
            re += f * s;
            im += f * c;
        }
    }
    return make_double2(re, im);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Block-wide argmax of v (>= 0; -1 marks excluded) with ties to the lower index.
__device__ int block_argmax(double v, int idx, double *sv, int *si) {
    for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        sv[w] = v;
        si[w] = idx;
    }
    __syncthreads();
    double bv = sv[0];
    int bi = si[0];
    for (int q = 1; q < kAcaWarps; ++q)
        if (sv[q] > bv || (sv[q] == bv && si[q] < bi)) {
            bv = sv[q];
            bi = si[q];
        }
    return bv < 0.0 ? -1 : bi;
}

__device__ double block_sum(double v, double *sv) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sv[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < kAcaWarps; ++q) s += sv[q];
    return s;
}

__global__ void __launch_bounds__(kAcaThreads, 8)
aca_kernel(const AcaJob *__restrict__ jobs, const double *__restrict__ rec, int stride, double k,
           double scale, double tol) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double sv[kAcaWarps];
    __shared__ int si[kAcaWarps];
    const AcaJob jb = jobs[blockIdx.x];
    const int m = jb.m, n = jb.n, kmax = jb.kmax, tid = threadIdx.x;
    double2 *Rr = reinterpret_cast<double2 *>(smem);  // row residual, then V_k (n)
    double2 *Rc = Rr + n;                              // column residual = U_k (m)
    double2 *stage = Rc + m;                           // U(i, :) or V(:, j) (kmax)
    double *prec = reinterpret_cast<double *>(stage + kmax);  // pivot record (7 NP)
    unsigned char *usedr = reinterpret_cast<unsigned char *>(prec + 7 * kAcaNP);
    unsigned char *usedc = usedr + m;
    const double kinv = 1.0 / k;
    for (int i = tid; i < m; i += kAcaThreads) usedr[i] = 0;
    for (int j = tid; j < n; j += kAcaThreads) usedc[j] = 0;
    if (tid == 0) usedr[0] = 1;
    int ic = 0, kk = 0, status = 0;
    double normz = 0.0;
    const int kcap = min(kmax, min(m, n));
    __syncthreads();
    for (;;) {
        // residual of row ic
        for (int t = tid; t < kk; t += kAcaThreads) stage[t] = jb.U[ic + (size_t)t * m];
        for (int e = tid; e < 7 * kAcaNP; e += kAcaThreads) prec[e] = rec[(size_t)jb.rows[ic] * stride + e];
        __syncthreads();
        for (int j = tid; j < n; j += kAcaThreads) {
            double2 z = rec_entry(prec, rec + (size_t)jb.cols[j] * stride, k, kinv);
            z.x *= scale;
            z.y *= scale;
            for (int t = 0; t < kk; ++t) {
                const double2 p = cmul(stage[t], jb.V[(size_t)t * n + j]);
                z.x -= p.x;
                z.y -= p.y;
            }
            Rr[j] = z;
        }
        __syncthreads();
        // column pivot: largest unused |R_i|
        double bv = -1.0;
        int bi = 0x7fffffff;
        for (int j = tid; j < n; j += kAcaThreads)
            if (!usedc[j]) {
                const double a = Rr[j].x * Rr[j].x + Rr[j].y * Rr[j].y;
                if (a > bv) {
                    bv = a;
                    bi = j;
                }
            }
        const int jc = block_argmax(bv, bi, sv, si);
        if (jc < 0) break;  // every column used (cannot happen before the rank limit)
        const double2 piv = Rr[jc];
        __syncthreads();
        if (tid == 0) usedc[jc] = 1;
        if (piv.x == 0.0 && piv.y == 0.0) {
            status = 2;
            break;
        }
        // V_k = R_i / R_i(jc)
        const double pd = 1.0 / (piv.x * piv.x + piv.y * piv.y);
        const double2 pinv = make_double2(piv.x * pd, -piv.y * pd);
        double vn = 0.0;
        for (int j = tid; j < n; j += kAcaThreads) {
            const double2 v = cmul(Rr[j], pinv);
            Rr[j] = v;
            jb.V[(size_t)kk * n + j] = v;
            vn += v.x * v.x + v.y * v.y;
        }
        for (int t = tid; t < kk; t += kAcaThreads) stage[t] = jb.V[(size_t)t * n + jc];
        for (int e = tid; e < 7 * kAcaNP; e += kAcaThreads) prec[e] = rec[(size_t)jb.cols[jc] * stride + e];
        vn = block_sum(vn, sv);  // (synchronises: Rr, stage and prec are complete)
        // residual of column jc = U_k
        double un = 0.0;
        for (int i = tid; i < m; i += kAcaThreads) {
            double2 z = rec_entry(prec, rec + (size_t)jb.rows[i] * stride, k, kinv);
            z.x *= scale;
            z.y *= scale;
            for (int t = 0; t < kk; ++t) {
                const double2 p = cmul(jb.U[i + (size_t)t * m], stage[t]);
                z.x -= p.x;
                z.y -= p.y;
            }
            Rc[i] = z;
            jb.U[i + (size_t)kk * m] = z;
            un += z.x * z.x + z.y * z.y;
        }
        un = block_sum(un, sv);
        // ||U V||_F^2 update
        if (kk == 0) {
            normz = un * vn;
        } else {
            // cross terms: sum_t Re(a_t b_t), a_t = U_t^H U_k, b_t = V_k V_t^H; one warp per t
            const int lane = tid & 31, w = tid >> 5;
            double part = 0.0;
            for (int t = w; t < kk; t += kAcaWarps) {
                double ar = 0.0, ai = 0.0, br = 0.0, bi2 = 0.0;
                for (int i = lane; i < m; i += 32) {
                    const double2 u = jb.U[i + (size_t)t * m], x = Rc[i];
                    ar += u.x * x.x + u.y * x.y;  // conj(u) x
                    ai += u.x * x.y - u.y * x.x;
                }
                for (int j = lane; j < n; j += 32) {
                    const double2 v = Rr[j], x = jb.V[(size_t)t * n + j];
                    br += v.x * x.x + v.y * x.y;  // v conj(x)
                    bi2 += v.y * x.x - v.x * x.y;
                }
                for (int o = 16; o; o >>= 1) {
                    ar += __shfl_xor_sync(0xffffffffu, ar, o);
                    ai += __shfl_xor_sync(0xffffffffu, ai, o);
                    br += __shfl_xor_sync(0xffffffffu, br, o);
                    bi2 += __shfl_xor_sync(0xffffffffu, bi2, o);
                }
                part += ar * br - ai * bi2;
            }
            if (lane != 0) part = 0.0;
            const double cross = block_sum(part, sv);
            normz += 2.0 * cross + un * vn;
        }
        if (tid == 0) {
            jb.I[kk] = ic;
            jb.J[kk] = jc;
        }
        ++kk;
        if (kk >= 2 && sqrt(un) * sqrt(vn) <= tol * sqrt(normz)) break;
        if (kk == min(m, n)) break;
        if (kk == kcap) {
            status = 1;
            break;
        }
        // next row pivot: largest unused |R_j|
        bv = -1.0;
        bi = 0x7fffffff;
        for (int i = tid; i < m; i += kAcaThreads)
            if (!usedr[i]) {
                const double a = Rc[i].x * Rc[i].x + Rc[i].y * Rc[i].y;
                if (a > bv) {
                    bv = a;
                    bi = i;
                }
            }
        ic = block_argmax(bv, bi, sv, si);
        if (ic < 0) break;
        __syncthreads();
        if (tid == 0) usedr[ic] = 1;
        __syncthreads();
    }
    if (tid == 0) {
        jb.out[0] = kk;
        jb.out[1] = status;
    }
}

__global__ void aca_norm_kernel(const double2 *const *mats, const long long *sizes, double *out) {
    __shared__ double s[256];
    const double2 *a = mats[blockIdx.x];
    const long long n = sizes[blockIdx.x];
    double acc = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) acc += a[i].x * a[i].x + a[i].y * a[i].y;
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s[0]);
}

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace pskel

using namespace pskel;

extern "C" int pskel_aca_compress(pskel_ctx *c, double tol, int kmax, int *ranks, int *status) {
    if (!c) {
        set_error(PSKEL_ERR_ARG, "aca_compress: null context");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    if (!c->have_mesh || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_STATE, "aca_compress: mesh and blocks required");
        return PSKEL_ERR_STATE;
    }
    if (!(tol > 0.0) || kmax < 1 || kmax > 1024 || c->em.q_test != kAcaQ || c->em.q_src != kAcaQ) {
        set_error(PSKEL_ERR_ARG, "aca_compress: tol > 0, 1 <= kmax <= 1024 and the 7-point rule "
                                 "(q = 7) required (tol %g kmax %d q %d)", tol, kmax, c->em.q_test);
        return PSKEL_ERR_ARG;
    }
    const int nb = c->n_blocks;
    // symmetric mode: approximate the block with the smaller index of each (t, s) / (s, t) pair
    std::vector<int> mirror(nb, -1), prims;
    for (int b = 0; b < nb; ++b) {
        const int p = c->symmetric ? c->partner[b] : -1;
        if (p >= 0 && p < b) mirror[b] = p; else prims.push_back(b);
    }
    std::vector<AcaJob> jobs(prims.size());
    std::vector<size_t> offU(nb), offV(nb), offI(nb), offJ(nb);
    size_t tot = al256(sizeof(int) * 2 * prims.size());  // k and status of every block first
    int maxm = 0, maxn = 0, maxk = 0;
    auto gsize = [&](int g) { return c->gptr[g + 1] - c->gptr[g]; };
    for (int b : prims) {
        const int m = gsize(c->gt[b]), n = gsize(c->gs[b]);
        if (m > kAcaMaxSide || n > kAcaMaxSide || m < 2 || n < 2) {
            set_error(PSKEL_ERR_ARG, "aca_compress: block %d is %d x %d (2..%d rows and columns)", b,
                      m, n, kAcaMaxSide);
            return PSKEL_ERR_ARG;
        }
        const int kb = std::min(kmax, std::min(m, n));
        offU[b] = tot; tot += al256(sizeof(double2) * (size_t)m * kb);
        offV[b] = tot; tot += al256(sizeof(double2) * (size_t)kb * n);
        offI[b] = tot; tot += al256(sizeof(int) * (size_t)kb);
        offJ[b] = tot; tot += al256(sizeof(int) * (size_t)kb);
        maxm = std::max(maxm, m);
        maxn = std::max(maxn, n);
        maxk = std::max(maxk, kb);
    }
    PSKEL_TRY(c->aca_buf.reserve(tot + 256));
    char *base = c->aca_buf.as<char>();
    const int *gids = c->d_gids.as<int>();
    for (size_t i = 0; i < prims.size(); ++i) {
        const int b = prims[i];
        const int m = gsize(c->gt[b]), n = gsize(c->gs[b]);
        jobs[i] = AcaJob{gids + c->gptr[c->gt[b]], gids + c->gptr[c->gs[b]],
                         reinterpret_cast<double2 *>(base + offU[b]), reinterpret_cast<double2 *>(base + offV[b]),
                         reinterpret_cast<int *>(base + offI[b]), reinterpret_cast<int *>(base + offJ[b]),
                         reinterpret_cast<int *>(base) + 2 * i, m, n, std::min(kmax, std::min(m, n))};
    }
    PSKEL_TRY(c->aca_tab.reserve(sizeof(AcaJob) * jobs.size() + 256));
    PSKEL_CUDA(cudaMemcpyAsync(c->aca_tab.ptr, jobs.data(), sizeof(AcaJob) * jobs.size(),
                               cudaMemcpyHostToDevice, c->stream));
    if (!c->mesh.records(kAcaQ).f64.ptr) PSKEL_TRY(build_records(c->mesh, kAcaQ, c->stream, c->flags.as<int>()));
    const size_t smem = sizeof(double2) * ((size_t)maxm + maxn + maxk) + sizeof(double) * 7 * kAcaNP +
                        (size_t)maxm + maxn + 64;
    PSKEL_TRY(ensure_smem_attr(aca_kernel, 200 * 1024));
    if (smem > 200 * 1024) {
        set_error(PSKEL_ERR_ARG, "aca_compress: shared memory %zu bytes", smem);
        return PSKEL_ERR_ARG;
    }
    const double scale = c->em.eta / (4.0 * 3.14159265358979323846);
    PSKEL_CUDA(cudaEventRecord(c->ev[0], c->stream));
    aca_kernel<<<(unsigned)jobs.size(), kAcaThreads, smem, c->stream>>>(
        c->aca_tab.as<AcaJob>(), c->mesh.records(kAcaQ).f64.as<double>(), rec_stride(kAcaQ), c->em.k,
        scale, tol);
    PSKEL_LAUNCHED(1);
    PSKEL_CUDA(cudaEventRecord(c->ev[1], c->stream));
    // per-block rank and status
    std::vector<int> ko(2 * prims.size());
    PSKEL_CUDA(cudaMemcpyAsync(ko.data(), base, sizeof(int) * ko.size(), cudaMemcpyDeviceToHost, c->stream));
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0.0f;
    PSKEL_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    c->aca_ms = ms;
    c->aca_k.assign(nb, 0);
    c->aca_status.assign(nb, 0);
    for (size_t i = 0; i < prims.size(); ++i) {
        c->aca_k[prims[i]] = ko[2 * i];
        c->aca_status[prims[i]] = ko[2 * i + 1];
    }
    for (int b = 0; b < nb; ++b)
        if (mirror[b] >= 0) {
            c->aca_k[b] = c->aca_k[mirror[b]];
            c->aca_status[b] = c->aca_status[mirror[b]];
        }
    c->aca_mirror = mirror;
    c->aca_offU = offU;
    c->aca_offV = offV;
    c->aca_offI = offI;
    c->aca_offJ = offJ;
    c->aca_kmax = kmax;
    if (ranks) std::copy(c->aca_k.begin(), c->aca_k.end(), ranks);
    if (status) std::copy(c->aca_status.begin(), c->aca_status.end(), status);
    return PSKEL_OK;
}

extern "C" int pskel_aca_get_block(pskel_ctx *c, int b, pskel_c128 *U, pskel_c128 *V, int *I, int *J) {
    if (!c || b < 0 || b >= c->n_blocks || (int)c->aca_k.size() != c->n_blocks) {
        set_error(PSKEL_ERR_STATE, "aca_get_block: run pskel_aca_compress first");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const int p = c->aca_mirror[b] >= 0 ? c->aca_mirror[b] : b;
    const int mp = c->gptr[c->gt[p] + 1] - c->gptr[c->gt[p]], np = c->gptr[c->gs[p] + 1] - c->gptr[c->gs[p]];
    const int k = c->aca_k[b];
    const char *base = c->aca_buf.as<char>();
    std::vector<double2> Up((size_t)mp * k + 1), Vp((size_t)k * np + 1);
    std::vector<int> Ip(k + 1), Jp(k + 1);
    PSKEL_CUDA(cudaMemcpy(Up.data(), base + c->aca_offU[p], sizeof(double2) * mp * k, cudaMemcpyDeviceToHost));
    PSKEL_CUDA(cudaMemcpy(Vp.data(), base + c->aca_offV[p], sizeof(double2) * k * np, cudaMemcpyDeviceToHost));
    PSKEL_CUDA(cudaMemcpy(Ip.data(), base + c->aca_offI[p], sizeof(int) * k, cudaMemcpyDeviceToHost));
    PSKEL_CUDA(cudaMemcpy(Jp.data(), base + c->aca_offJ[p], sizeof(int) * k, cudaMemcpyDeviceToHost));
    // primary: U (mp x k, column-major), V (k x np) stored row-major; mirror: U = V_p^T, V = U_p^T
    const bool mir = p != b;
    const int m = mir ? np : mp, n = mir ? mp : np;
    for (int t = 0; t < k; ++t) {
        for (int i = 0; i < m; ++i) {
            const double2 u = mir ? Vp[(size_t)t * np + i] : Up[i + (size_t)t * mp];
            if (U) U[i + (size_t)t * m] = pskel_c128{u.x, u.y};
        }
        for (int j = 0; j < n; ++j) {
            const double2 v = mir ? Up[j + (size_t)t * mp] : Vp[(size_t)t * np + j];
            if (V) V[t + (size_t)j * k] = pskel_c128{v.x, v.y};
        }
        if (I) I[t] = mir ? Jp[t] : Ip[t];
        if (J) J[t] = mir ? Ip[t] : Jp[t];
    }
    return PSKEL_OK;
}

extern "C" int pskel_aca_true_errors(pskel_ctx *c, double *err) {
    if (!c || !err || (int)c->aca_k.size() != c->n_blocks || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_STATE, "aca_true_errors: run pskel_aca_compress first");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const int nb = c->n_blocks;
    const size_t budget = (size_t)1 << 27;  // dense complex elements per batch
    const char *base = c->aca_buf.as<char>();
    auto gsize = [&](int g) { return c->gptr[g + 1] - c->gptr[g]; };
    int b0 = 0;
    while (b0 < nb) {
        size_t dense = 0;
        int b1 = b0;
        while (b1 < nb) {
            const size_t d = (size_t)gsize(c->gt[b1]) * gsize(c->gs[b1]);
            if (b1 > b0 && dense + d > budget) break;
            dense += d;
            ++b1;
        }
        const int nbb = b1 - b0;
        PSKEL_TRY(c->tmp.reserve(sizeof(double2) * dense + 256));
        double2 *Zb = c->tmp.as<double2>();
        std::vector<FillJob> fills(nbb);
        std::vector<ZgemmJob> g;
        std::vector<const double2 *> mats(nbb);
        std::vector<long long> sizes(nbb);
        std::vector<int> prefix(nbb + 1, 0);
        int tm, tn;
        fill_tile_shape(PSKEL_C128, kAcaQ, 0, &tm, &tn);
        size_t zo = 0;
        for (int i = 0; i < nbb; ++i) {
            const int b = b0 + i, m = gsize(c->gt[b]), n = gsize(c->gs[b]);
            double2 *Z = Zb + zo;
            zo += (size_t)m * n;
            fills[i] = FillJob{c->d_gids.as<int>() + c->gptr[c->gt[b]], c->d_gids.as<int>() + c->gptr[c->gs[b]],
                               Z, m, n, m, 0};
            prefix[i + 1] = prefix[i] + ((m + tm - 1) / tm) * ((n + tn - 1) / tn);
            mats[i] = Z;
            sizes[i] = (long long)m * n;
            const int p = c->aca_mirror[b] >= 0 ? c->aca_mirror[b] : b;
            const int mp = gsize(c->gt[p]), np = gsize(c->gs[p]), k = c->aca_k[b];
            if (k == 0) continue;
            const double2 *Up = reinterpret_cast<const double2 *>(base + c->aca_offU[p]);
            const double2 *Vs = reinterpret_cast<const double2 *>(base + c->aca_offV[p]);  // np x k col-major = V^T
            ZgemmJob j = p == b ? zjob(Up, mp, ZOP_N, Vs, np, ZOP_T, Z, m, m, n, k)    // Z -= U V
                                : zjob(Vs, np, ZOP_N, Up, mp, ZOP_T, Z, m, m, n, k);   // Z -= V_p^T U_p^T
            j.alpha = make_double2(-1.0, 0.0);
            j.beta = make_double2(1.0, 0.0);
            g.push_back(j);
        }
        const size_t fb = al256(sizeof(FillJob) * nbb);
        PSKEL_TRY(c->tmp2.reserve(fb + al256(sizeof(int) * (nbb + 1)) + al256(sizeof(void *) * nbb) +
                                  al256(sizeof(long long) * nbb) + 2 * al256(sizeof(double) * nbb)));
        char *d = c->tmp2.as<char>();
        FillJob *d_f = reinterpret_cast<FillJob *>(d);
        int *d_p = reinterpret_cast<int *>(d + fb);
        const double2 **d_m = reinterpret_cast<const double2 **>(d + fb + al256(sizeof(int) * (nbb + 1)));
        long long *d_s = reinterpret_cast<long long *>(reinterpret_cast<char *>(d_m) + al256(sizeof(void *) * nbb));
        double *d_nz = reinterpret_cast<double *>(reinterpret_cast<char *>(d_s) + al256(sizeof(long long) * nbb));
        double *d_ne = reinterpret_cast<double *>(reinterpret_cast<char *>(d_nz) + al256(sizeof(double) * nbb));
        PSKEL_CUDA(cudaMemcpyAsync(d_f, fills.data(), sizeof(FillJob) * nbb, cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_p, prefix.data(), sizeof(int) * (nbb + 1), cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_m, mats.data(), sizeof(void *) * nbb, cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_s, sizes.data(), sizeof(long long) * nbb, cudaMemcpyHostToDevice, c->stream));
        FillParams fp;
        fp.k = c->em.k;
        fp.eta = c->em.eta;
        fp.r_near = 0;
        fp.q_test = fp.q_src = kAcaQ;
        fp.precision = PSKEL_C128;
        fp.split = 0;
        PSKEL_TRY(launch_fill(c->mesh, fp, d_f, d_p, nbb, prefix.back(), c->flags.as<int>(), c->stream));
        aca_norm_kernel<<<nbb, 256, 0, c->stream>>>(d_m, d_s, d_nz);
        PSKEL_LAUNCHED(1);
        if (!g.empty()) PSKEL_TRY(launch_zgemm(g, c->stream, c->tmp3));
        aca_norm_kernel<<<nbb, 256, 0, c->stream>>>(d_m, d_s, d_ne);
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
