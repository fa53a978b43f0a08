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

// One block per CTA iteration: T1 = R X(cols) (r x nrhs), T2 = U T1, Y(rows) += C T2.
// Arithmetic type A (float or double), storage S (float2 or double2) of C and R.
struct MatvecBlock {
    const int *rows, *cols;
    const void *C, *R;
    const double2 *U;
    int m, n, r, ldr;
};

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
                const double2 rv = ld_c(R, i + (size_t)k * w.ldr);
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
                const double2 u = w.U[i + (size_t)k * w.r];
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
                const double2 c = ld_c(Cm, i + (size_t)k * w.m);
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
        // block table: built once per compression, uploaded synchronously
        std::vector<MatvecBlock> hb(nb);
        int max_r = 0;
        for (int b = 0; b < nb; ++b) {
            const BlockResult &res = c->results[b];
            if (res.arena < 0) {
                set_error(PSKEL_ERR_STATE, "matvec: block %d has no retained factors", b);
                return PSKEL_ERR_STATE;
            }
            const char *base = c->arenas[res.arena].keep.as<char>();
            hb[b] = MatvecBlock{c->d_gids.as<int>() + c->gptr[c->gt[b]],
                                c->d_gids.as<int>() + c->gptr[c->gs[b]], base + res.offC,
                                base + res.offRx, reinterpret_cast<const double2 *>(base + res.offU),
                                res.m, res.n, res.r, res.r + res.pe};
            max_r = std::max(max_r, res.r);
        }
        PSKEL_TRY(c->mv_table.reserve(sizeof(MatvecBlock) * nb + 256));
        PSKEL_CUDA(cudaStreamSynchronize(c->stream));
        PSKEL_CUDA(cudaMemcpy(c->mv_table.ptr, hb.data(), sizeof(MatvecBlock) * nb,
                              cudaMemcpyHostToDevice));
        c->mv_max_r = max_r;
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
#define PSKEL_MV(A, S)                                                                         \
    do {                                                                                       \
        auto k = matvec_kernel<A, S>;                                                          \
        PSKEL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                        200 * 1024));                                          \
        k<<<grid, 256, smem, st>>>(d_b, nb, reinterpret_cast<const CT<A>::c *>(X), ldx, \
                                          reinterpret_cast<A *>(Y), ldy, nrhs);               \
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
// For each block (C m x r, U r x r, R r x n):
//   one-sided Jacobi  C V_c = B_c,  R^H V_r = B_r   (B orthogonal columns, sigma = column norms)
//   core              M = diag(s_c) V_c^H U V_r diag(s_r)          (singular values of C U R)
//   Jacobi            M V_m = B_m,  s_m = column norms, u_m = B_m / s_m
//   C' = B_c diag(1/s_c) u_m,  R'^H = B_r diag(1/s_r) V_m,  S = s_m   (sorted, k kept where
//   s_m > thresh * max s_m, the rule of svd_compress.m:25-28)
// Columns of B_c, B_r below 1e-14 of their largest are dropped (they carry no part of C U R).
namespace pskel {

struct RecompBlock {
    const void *C, *R;   // stored factors (storage type of the compression)
    const double2 *U;
    double2 *Bc, *Vc, *Br, *Vr, *T, *M, *Vm, *Tc, *Tr, *Cp, *RpH, *Rp;
    double *sc, *sr, *sm, *S;
    int *pc, *pr, *pm, *k;
    int *kout;  // the kept rank, in a table of all blocks
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

__device__ double block_max(const double *v, int n, double *red) {
    double mx = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, v[i]);
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// M <- diag(s_c) M diag(s_r) with the small singular values of C and R dropped
__global__ void __launch_bounds__(256) recomp_scale_kernel(const RecompBlock *__restrict__ jobs) {
    __shared__ double red[256];
    const RecompBlock w = jobs[blockIdx.x];
    const double mc = block_max(w.sc, w.r, red), mr = block_max(w.sr, w.r, red);
    for (int e = threadIdx.x; e < w.r * w.r; e += blockDim.x) {
        const int i = e % w.r, j = e / w.r;
        const double a = w.sc[i] > 1e-14 * mc ? w.sc[i] : 0.0;
        const double b = w.sr[j] > 1e-14 * mr ? w.sr[j] : 0.0;
        const double2 v = w.M[e];
        w.M[e] = make_double2(v.x * a * b, v.y * a * b);
    }
}

// Tc(:, t) = diag(1/s_c) B_m(:, pm[t]) / s_m[pm[t]],  Tr(:, t) = diag(1/s_r) V_m(:, pm[t]),
// S[t] = s_m[pm[t]], k = #{s_m > thresh s_m,max}
__global__ void __launch_bounds__(256) recomp_factors_kernel(const RecompBlock *__restrict__ jobs) {
    __shared__ double red[256];
    const RecompBlock w = jobs[blockIdx.x];
    const double mc = block_max(w.sc, w.r, red), mr = block_max(w.sr, w.r, red);
    const double smax = w.sm[w.pm[0]];
    for (int e = threadIdx.x; e < w.r * w.r; e += blockDim.x) {
        const int i = e % w.r, t = e / w.r;
        const int c = w.pm[t];
        const double s = w.sm[c];
        const double ic = w.sc[i] > 1e-14 * mc ? 1.0 / w.sc[i] : 0.0;
        const double ir = w.sr[i] > 1e-14 * mr ? 1.0 / w.sr[i] : 0.0;
        const double f = s > 0 ? ic / s : 0.0;
        const double2 bm = w.M[i + (size_t)c * w.r];  // M holds B_m after the SVD
        const double2 vm = w.Vm[i + (size_t)c * w.r];
        w.Tc[e] = make_double2(bm.x * f, bm.y * f);
        w.Tr[e] = make_double2(vm.x * ir, vm.y * ir);
    }
    for (int t = threadIdx.x; t < w.r; t += blockDim.x) w.S[t] = w.sm[w.pm[t]];
    if (threadIdx.x == 0) {
        int k = 0;
        for (int t = 0; t < w.r; ++t) k += w.sm[w.pm[t]] > w.thresh * smax;
        *w.k = k;
        *w.kout = k;
    }
}

// R' = (R'^H)^H : r x n from n x r
__global__ void recomp_rp_kernel(const RecompBlock *__restrict__ jobs) {
    const RecompBlock w = jobs[blockIdx.x];
    for (int e = threadIdx.x; e < w.r * w.n; e += blockDim.x) {
        const int t = e % w.r, j = e / w.r;
        const double2 v = w.RpH[j + (size_t)t * w.n];
        w.Rp[e] = make_double2(v.x, -v.y);
    }
}

}  // namespace pskel

extern "C" int pskel_recompress(pskel_ctx *c, double thresh, int *ranks) {
    if (!c || !(thresh >= 0) || c->n_blocks <= 0) {
        set_error(PSKEL_ERR_ARG, "recompress: bad arguments");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const int nb = c->n_blocks;
    const bool f32 = c->precision == PSKEL_C64;
    // workspace (all FP64 complex): Bc m r, Br n r, Vc Vr T M Vm Tc Tr r r each, Cp m r, RpH n r,
    // Rp r n, plus real vectors
    std::vector<size_t> off(nb + 1, 0);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    for (int b = 0; b < nb; ++b) {
        const BlockResult &res = c->results[b];
        if (res.arena < 0) {
            set_error(PSKEL_ERR_STATE, "recompress: block %d has no retained factors", b);
            return PSKEL_ERR_STATE;
        }
        const size_t m = res.m, n = res.n, r = res.r;
        size_t s = al(16 * m * r) * 2 + al(16 * n * r) * 2 + al(16 * r * n) + 7 * al(16 * r * r) +
                   4 * al(8 * r) + 4 * al(4 * r) + 256;
        off[b + 1] = off[b] + s;
    }
    PSKEL_TRY(c->recomp.reserve(off[nb] + 256));
    char *base = c->recomp.as<char>();
    std::vector<RecompBlock> jobs(nb);
    std::vector<SvdJob> svd1, svd2;
    svd1.reserve(2 * nb);
    svd2.reserve(nb);
    std::vector<ZgemmJob> g1, g2, g3;
    c->recomp_slots.assign(nb, {});
    for (int b = 0; b < nb; ++b) {
        const BlockResult &res = c->results[b];
        const char *kb = c->arenas[res.arena].keep.as<char>();
        char *q = base + off[b];
        auto take = [&](size_t bytes) { char *x = q; q += al(bytes); return x; };
        const size_t m = res.m, n = res.n, r = res.r;
        RecompBlock &w = jobs[b];
        w.C = kb + res.offC;
        w.R = kb + res.offRx;
        w.U = reinterpret_cast<const double2 *>(kb + res.offU);
        w.Bc = reinterpret_cast<double2 *>(take(16 * m * r));
        w.Cp = reinterpret_cast<double2 *>(take(16 * m * r));
        w.Br = reinterpret_cast<double2 *>(take(16 * n * r));
        w.RpH = reinterpret_cast<double2 *>(take(16 * n * r));
        w.Rp = reinterpret_cast<double2 *>(take(16 * r * n));
        w.Vc = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Vr = reinterpret_cast<double2 *>(take(16 * r * r));
        w.T = reinterpret_cast<double2 *>(take(16 * r * r));
        w.M = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Vm = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Tc = reinterpret_cast<double2 *>(take(16 * r * r));
        w.Tr = reinterpret_cast<double2 *>(take(16 * r * r));
        w.sc = reinterpret_cast<double *>(take(8 * r));
        w.sr = reinterpret_cast<double *>(take(8 * r));
        w.sm = reinterpret_cast<double *>(take(8 * r));
        w.S = reinterpret_cast<double *>(take(8 * r));
        w.pc = reinterpret_cast<int *>(take(4 * r));
        w.pr = reinterpret_cast<int *>(take(4 * r));
        w.pm = reinterpret_cast<int *>(take(4 * r));
        w.k = reinterpret_cast<int *>(take(4 * r));
        w.m = res.m;
        w.n = res.n;
        w.r = res.r;
        w.ldr = res.r + res.pe;
        w.thresh = thresh;
        svd1.push_back(SvdJob{w.Bc, w.Vc, w.sc, w.pc, res.m, res.r, 0, 0});
        svd1.push_back(SvdJob{w.Br, w.Vr, w.sr, w.pr, res.n, res.r, 0, 0});
        svd2.push_back(SvdJob{w.M, w.Vm, w.sm, w.pm, res.r, res.r, 0, 0});
        g1.push_back(zjob(w.U, res.r, ZOP_N, w.Vr, res.r, ZOP_N, w.T, res.r, res.r, res.r, res.r));
        g2.push_back(zjob(w.Vc, res.r, ZOP_C, w.T, res.r, ZOP_N, w.M, res.r, res.r, res.r, res.r));
        g3.push_back(zjob(w.Bc, res.m, ZOP_N, w.Tc, res.r, ZOP_N, w.Cp, res.m, res.m, res.r, res.r));
        g3.push_back(zjob(w.Br, res.n, ZOP_N, w.Tr, res.r, ZOP_N, w.RpH, res.n, res.n, res.r, res.r));
        c->recomp_slots[b] = RecompSlot{(size_t)((char *)w.Cp - base), (size_t)((char *)w.Rp - base),
                                        (size_t)((char *)w.S - base), 0};
    }
    // device job tables
    const size_t jb = sizeof(RecompBlock) * nb, s1 = sizeof(SvdJob) * svd1.size(),
                 s2 = sizeof(SvdJob) * svd2.size();
    PSKEL_TRY(c->tmp.reserve(jb + s1 + s2 + sizeof(int) * nb + 1024));
    char *d = c->tmp.as<char>();
    RecompBlock *d_jobs = reinterpret_cast<RecompBlock *>(d);
    SvdJob *d_s1 = reinterpret_cast<SvdJob *>(d + ((jb + 255) & ~size_t(255)));
    SvdJob *d_s2 = reinterpret_cast<SvdJob *>(reinterpret_cast<char *>(d_s1) + ((s1 + 255) & ~size_t(255)));
    int *d_k = reinterpret_cast<int *>(reinterpret_cast<char *>(d_s2) + ((s2 + 255) & ~size_t(255)));
    for (int b = 0; b < nb; ++b) jobs[b].kout = d_k + b;
    PSKEL_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jb, cudaMemcpyHostToDevice, c->stream));
    PSKEL_CUDA(cudaMemcpyAsync(d_s1, svd1.data(), s1, cudaMemcpyHostToDevice, c->stream));
    PSKEL_CUDA(cudaMemcpyAsync(d_s2, svd2.data(), s2, cudaMemcpyHostToDevice, c->stream));
    if (f32) recomp_load_kernel<float2><<<nb, 256, 0, c->stream>>>(d_jobs);
    else recomp_load_kernel<double2><<<nb, 256, 0, c->stream>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    PSKEL_TRY(batched_svd(d_s1, svd1, 60, c->stream, c->tmp2));
    PSKEL_TRY(launch_zgemm(g1, c->stream, c->tmp3));
    PSKEL_TRY(launch_zgemm(g2, c->stream, c->tmp3));
    recomp_scale_kernel<<<nb, 256, 0, c->stream>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    PSKEL_TRY(batched_svd(d_s2, svd2, 60, c->stream, c->tmp2));
    recomp_factors_kernel<<<nb, 256, 0, c->stream>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    PSKEL_TRY(launch_zgemm(g3, c->stream, c->tmp3));
    recomp_rp_kernel<<<nb, 256, 0, c->stream>>>(d_jobs);
    PSKEL_LAUNCHED(1);
    // ranks and SVD statuses back to the host
    std::vector<SvdJob> h1(svd1.size()), h2(svd2.size());
    PSKEL_CUDA(cudaMemcpyAsync(h1.data(), d_s1, s1, cudaMemcpyDeviceToHost, c->stream));
    PSKEL_CUDA(cudaMemcpyAsync(h2.data(), d_s2, s2, cudaMemcpyDeviceToHost, c->stream));
    std::vector<int> ks(nb);
    PSKEL_CUDA(cudaMemcpyAsync(ks.data(), d_k, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->stream));
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    for (const SvdJob &j : h1)
        if (j.status != PSKEL_OK) {
            set_error(PSKEL_ERR_NOCONV, "recompress: Jacobi SVD of a factor did not converge");
            return PSKEL_ERR_NOCONV;
        }
    for (const SvdJob &j : h2)
        if (j.status != PSKEL_OK) {
            set_error(PSKEL_ERR_NOCONV, "recompress: Jacobi SVD of a core did not converge");
            return PSKEL_ERR_NOCONV;
        }
    for (int b = 0; b < nb; ++b) {
        c->recomp_slots[b].k = ks[b];
        if (ranks) ranks[b] = ks[b];
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
    const BlockResult &res = c->results[b];
    const char *base = c->recomp.as<char>();
    const size_t k = sl.k;
    if (Cp) PSKEL_CUDA(cudaMemcpy(Cp, base + sl.offCp, 16 * (size_t)res.m * k, cudaMemcpyDeviceToHost));
    if (S) PSKEL_CUDA(cudaMemcpy(S, base + sl.offS, 8 * k, cudaMemcpyDeviceToHost));
    if (Rp) {
        // R' is stored r x n (ld r): copy its first k rows
        std::vector<double2> h((size_t)res.r * res.n);
        PSKEL_CUDA(cudaMemcpy(h.data(), base + sl.offRp, 16 * h.size(), cudaMemcpyDeviceToHost));
        for (int j = 0; j < res.n; ++j)
            for (size_t t = 0; t < k; ++t) {
                const double2 v = h[t + (size_t)j * res.r];
                Rp[t + j * k] = pskel_c128{v.x, v.y};
            }
    }
    return PSKEL_OK;
}
