/*
 * pskel.h - C ABI of the B200 pseudoskeleton (CUR) library (libpskel_b200.so).
 *
 * Two groups of entry points:
 *
 *  1. Reference-named symbols, drop-ins for the ones the reference's Julia drivers ccall from
 *     "./functionsExternal_cuda.so" and "./functions_cur_external_cuda.so". Argument lists and
 *     return types are the reference's, in the same order; each declaration cites the
 *     definition it replaces (paths relative to codes/GPU_implementation/seed/). As in the
 *     reference, every pointer is a HOST pointer, every matrix is column-major, and the
 *     r1/r2/row_samples/col_samples arrays hold 1-based RWG ids stored as doubles even though
 *     the C prototype says int* (the Julia callers pass Vector{Cdouble}; the reference copies
 *     n*sizeof(double) bytes, user_impedance_for_julia_cuda.cu:1100-1101,1735-1736).
 *     Launch-geometry arguments (blocks_*, threads_*, limx, limy) are accepted and ignored:
 *     the library picks its own launch shapes. Errors: functions returning double return NaN,
 *     functions returning int return 0 (the reference returns 1 on success and has no error
 *     path); pskel_last_error() gives the reason.
 *
 *  2. pskel_* handle API: the mesh, group lists and compressed blocks stay resident on the
 *     device; calls return PSKEL_OK (0) or a negative status.
 *
 * Mesh arrays (column-major Float64, 1-based ids, as passed by the Julia wrappers, e.g.
 * compres_single_block_spheres_for_sweep2.jl:380-388): vertex 3 x Nv, topol 3 x Nt,
 * trian 3 x Nt, edges 4 x Ne (T+, T-, opposite vertex in T+, opposite vertex in T-),
 * un 3 x Nt, ds 1 x Nt, ln Ne, cent 3 x Nt. Only vertex, topol, edges, ln and cent are read.
 */
#ifndef PSKEL_H
#define PSKEL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* complex128 laid out like Julia ComplexF64 / cuDoubleComplex */
typedef struct { double re, im; } pskel_c128;
/* complex64 laid out like Julia ComplexF32 / cuFloatComplex */
typedef struct { float re, im; } pskel_c64;

/* ---------------------------------------------------------------- status codes */
#define PSKEL_OK 0
#define PSKEL_ERR_ARG (-1)        /* bad size, pointer or option */
#define PSKEL_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define PSKEL_ERR_NOCONV (-3)     /* Jacobi SVD hit its sweep limit */
#define PSKEL_ERR_NEAR (-4)       /* unused: near pairs are filled by the near-field rule */
#define PSKEL_ERR_OOM (-5)        /* device allocation failed */
#define PSKEL_ERR_RANGE (-6)      /* an RWG id is out of range */
#define PSKEL_ERR_UNSUPPORTED (-7) /* field != 1 (only EFIE is implemented) */
#define PSKEL_ERR_STATE (-8)      /* call order (e.g. no mesh uploaded) */

/* Last error of the calling thread: status code and a short message. */
int pskel_last_error(const char **message);

/* ======================================================= 1. reference-named entry points */

/* Dense fill of Z(r1, r2) into Ztotal (n_r1 x n_r2 complex128). Returns the fill kernel time
   in ms. Replaces impedance_matrix_cuda_elbyel4, user_impedance_for_julia_cuda.cu:1022-1064
   (Julia caller compres_single_block_spheres_for_sweep2.jl:433-478). */
double impedance_matrix_cuda_elbyel4(pskel_c128 *Ztotal, int field, double k, double eta,
    double Rinteg_s, double Ranal_s, double Rinteg_f, int cor_solid, int flag, int *r1, int *r2,
    double *vertex, double *topol, double *trian, double *edges, double *un, double *ds,
    double *ln, double *cent, int N, int n_r1, int n_r2, int rows_vertex, int cols_vertex,
    int rows_topol, int cols_topol, int rows_trian, int cols_trian, int rows_edges,
    int cols_edges, int rows_un, int cols_un, int rows_ds, int cols_ds, int n_ln,
    int rows_cent, int cols_cent, int blocks_x, int blocks_y, int threads_x, int threads_y,
    int limx, int limy);

/* Same fill, returns 1. Replaces impedance_matrix_cuda_elbyel3,
   user_impedance_for_julia_cuda.cu:770-812 (caller compres_single_block_spheres.jl:1708). */
int impedance_matrix_cuda_elbyel3(pskel_c128 *Ztotal, int field, double k, double eta,
    double Rinteg_s, double Ranal_s, double Rinteg_f, int cor_solid, int flag, int *r1, int *r2,
    double *vertex, double *topol, double *trian, double *edges, double *un, double *ds,
    double *ln, double *cent, int N, int n_r1, int n_r2, int rows_vertex, int cols_vertex,
    int rows_topol, int cols_topol, int rows_trian, int cols_trian, int rows_edges,
    int cols_edges, int rows_un, int cols_un, int rows_ds, int cols_ds, int n_ln,
    int rows_cent, int cols_cent, int blocks_x, int blocks_y, int threads_x, int threads_y,
    int limx, int limy);

/* Same fill into split real/imaginary arrays, returns 1. Replaces
   impedance_matrix_cuda_elbyel2, user_impedance_for_julia_cuda.cu:602-645
   (caller compres_single_block_spheres.jl:1578). */
int impedance_matrix_cuda_elbyel2(double *Zr, double *Zi, int field, double k, double eta,
    double Rinteg_s, double Ranal_s, double Rinteg_f, int cor_solid, int flag, int *r1, int *r2,
    double *vertex, double *topol, double *trian, double *edges, double *un, double *ds,
    double *ln, double *cent, int N, int n_r1, int n_r2, int rows_vertex, int cols_vertex,
    int rows_topol, int cols_topol, int rows_trian, int cols_trian, int rows_edges,
    int cols_edges, int rows_un, int cols_un, int rows_ds, int cols_ds, int n_ln,
    int rows_cent, int cols_cent, int blocks_x, int blocks_y, int threads_x, int threads_y,
    int limx, int limy);

/* Split-array fill of Z(r1, r2) into Zr/Zi; the C/U/R outputs are left untouched and
   tol_compress is ignored, exactly as in the reference. Returns 1. Replaces cuda_cur_pure,
   user_impedance_for_julia_cuda.cu:1273-1432 (caller compres_single_block_spheres.jl:2035). */
int cuda_cur_pure(double *Zr, double *Zi, int field, double k, double eta, double Rinteg_s,
    double Ranal_s, double Rinteg_f, int cor_solid, int flag, int *r1, int *r2, double *vertex,
    double *topol, double *trian, double *edges, double *un, double *ds, double *ln,
    double *cent, double *Cmat_r, double *Cmat_i, double *Umat_r, double *Umat_i,
    double *Rmat_r, double *Rmat_i, int N, int n_r1, int n_r2, int rows_vertex,
    int cols_vertex, int rows_topol, int cols_topol, int rows_trian, int cols_trian,
    int rows_edges, int cols_edges, int rows_un, int cols_un, int rows_ds, int cols_ds,
    int n_ln, int rows_cent, int cols_cent, int blocks_x, int blocks_y, int threads_x,
    int threads_y, int limx, int limy, double tol_compress);

/* One CUR round with caller-supplied samples: C = Z(r1, col_samples) (n_r1 x cur_order),
   U = pinv(Z(row_samples, col_samples)) with singular values below the ABSOLUTE threshold
   pinv_tol dropped, R = Z(row_samples, r2) (cur_order x n_r2), Avtest_new = C (U (R vtest)).
   Returns ||Avtest_old - Avtest_new|| / ||Avtest_new||; vec_time_cuda[0] = device time of
   the round in ms (the reference reports alloc + compute ms and excludes the mesh upload and
   result download, user_impedance_for_julia_cuda.cu:1706-1711,1965-1975; here the device
   buffers are pooled, so the figure is compute only). Ztotal is unused. Replaces
   cuda_complete_compression, user_impedance_for_julia_cuda.cu:1564-1629
   (caller compres_single_block_spheres_for_sweep2.jl:591-660). */
double cuda_complete_compression(pskel_c128 *Ccompressed, pskel_c128 *Ucompressed,
    pskel_c128 *Rcompressed, int cur_order, double *vec_time_cuda, double pinv_tol,
    pskel_c128 *Avtest_old, pskel_c128 *Avtest_new, pskel_c128 *vtest, int *col_samples,
    int *row_samples, int C_blocks_x, int C_blocks_y, int C_threads_x, int C_threads_y,
    int U_blocks_x, int U_blocks_y, int U_threads_x, int U_threads_y, int R_blocks_x,
    int R_blocks_y, int R_threads_x, int R_threads_y, pskel_c128 *Ztotal, int field, double k,
    double eta, double Rinteg_s, double Ranal_s, double Rinteg_f, int cor_solid, int flag,
    int *r1, int *r2, double *vertex, double *topol, double *trian, double *edges, double *un,
    double *ds, double *ln, double *cent, int N, int n_r1, int n_r2, int rows_vertex,
    int cols_vertex, int rows_topol, int cols_topol, int rows_trian, int cols_trian,
    int rows_edges, int cols_edges, int rows_un, int cols_un, int rows_ds, int cols_ds,
    int n_ln, int rows_cent, int cols_cent, int blocks_x, int blocks_y, int threads_x,
    int threads_y, int limx, int limy);

/* Avtest_new = C (U (R vtest)) with C M1 x N1, U N1 x N1, R N1 x M2; returns
   ||Avtest_old - Avtest_new|| / ||Avtest_new||. Replaces compute_error_compression,
   user_impedance_for_julia_cuda.cu:1449-1556 and cur_external_cuda.cu:612-725
   (caller compres_single_block_spheres_for_sweep2.jl:992-995). */
double compute_error_compression(pskel_c128 *C, pskel_c128 *U, pskel_c128 *R,
    pskel_c128 *Avtest_old, pskel_c128 *Avtest_new, pskel_c128 *vtest, int M1, int N1, int M2);

/* CUR of a dense host matrix A (M x N) at given 1-based samples: C = A(:, col_samples),
   R = A(row_samples, :), U = pinv(A(row_samples, col_samples)) with absolute threshold
   tolerance. Returns 1. The sample arrays are Int64, as the Julia caller passes them
   (compres_single_block_spheres_for_sweep2.jl:777-789 declares Ptr{Int64}; the reference's C
   prototype says int*). Replaces aux_pinv_compression, cur_external_cuda.cu:572-610. */
int aux_pinv_compression(pskel_c128 *C, pskel_c128 *U, pskel_c128 *R, pskel_c128 *A,
    int64_t *row_samples, int64_t *col_samples, int ns, int M, int N, double tolerance);

/* pinvA (N x M) = V diag(s >= treshold ? 1/s : 0) U^H of A (M x N); also returns the thin
   left singular vectors U (M x min(M,N)), S (min(M,N)) and, as the reference does,
   diag(1/s) V^H in Vt (N x N, rows beyond min(M,N) zero). Returns 1. Replaces cuda_pinv,
   cur_external_cuda.cu:217-367. */
int cuda_pinv(pskel_c128 *pinvA, pskel_c128 *U, double *S, pskel_c128 *Vt, pskel_c128 *A,
    int M, int N, double treshold);

/* Thin SVD A = U diag(S) Vt of A (M x N): U M x min(M,N), S min(M,N) descending, Vt N x N
   (rows beyond min(M,N) zero). Returns 1. Replaces cuda_svd (cur_external_cuda.cu:400-517)
   and cuda_svd2 (cur_external_cuda.cu:86-201), which compute the same outputs. */
int cuda_svd(pskel_c128 *U, double *S, pskel_c128 *Vt, pskel_c128 *A, int M, int N);
int cuda_svd2(pskel_c128 *U, double *S, pskel_c128 *Vt, pskel_c128 *A, int M, int N);

/* In place V[i] = V[i] < treshold ? 0 : 1/V[i]. Returns 1. Replaces cuda_filter,
   cur_external_cuda.cu:372-398. */
int cuda_filter(double *V, double treshold, int N);

/* =========================================================== 2. pskel_* handle API */

typedef struct pskel_ctx pskel_ctx;

/* Precision of the sampled fills and of the stored C/R factors. */
#define PSKEL_C128 0
#define PSKEL_C64 1

/* Where each block's first sample count comes from. */
#define PSKEL_START_REFERENCE 0 /* min(m,n)/10, as the reference's drivers */
#define PSKEL_START_GIVEN 1     /* the per-block r0 array (e.g. the rank predictor) */

typedef struct {
    double k, eta;       /* wavenumber and impedance */
    int q_test, q_src;   /* quadrature points per triangle: 1 (centroid) or 7 */
} pskel_em_t;

typedef struct {
    double tol;          /* target relative Frobenius error of each block */
    double tau;          /* pinv threshold */
    int tau_relative;    /* 1: keep s >= tau*s_max, 0: keep s >= tau (reference rule) */
    int precision;       /* PSKEL_C128 or PSKEL_C64 */
    int start;           /* PSKEL_START_* */
    int oversample;      /* p added to a given r0 */
    int extra_rows;      /* unsampled rows of the randomized error estimate (<= 32) */
    int extra_cols;      /* unsampled columns of the randomized error estimate (<= 32) */
    int max_rounds;      /* adaptive rounds before giving up (the block keeps its last CUR) */
    int recompress;      /* 1: run the recompression after the last round */
    uint64_t seed;       /* Philox seed of the index sets */
    double recompress_tol; /* relative singular-value threshold of the recompression */
    double est_safety;   /* a block is accepted when est <= tol / est_safety (>= 1) */
    int use_graph;       /* 1: replay the first round from a CUDA graph captured on a repeat call */
    int per_block;       /* 1: drive the blocks one at a time (each block's rounds synchronise
                            with the host), the way the reference's drivers call its GPU CUR per
                            block; the kernels, samples and results per block are those of the
                            batched mode, but only the stats are kept (factors of the last block
                            only) */
    double est_verify;   /* > 1: a block that passes with est in (tol / (est_safety * est_verify),
                            tol / est_safety] is re-checked on a second, independent set of extra
                            rows and columns (drawn outside all of its samples, Philox streams 4
                            and 5 of its round) and passes only if the estimate pooled over both
                            sets does; <= 1: no re-check. */
    double full_tau;     /* > 0: relative pinv threshold of a block sampled on its whole smaller
                            side (r = min(m, n)), where more samples cannot help: the smaller of
                            tau and full_tau (e.g. 1e-10, so that C U R reproduces the block);
                            0: tau there too */
} pskel_opts_t;

/* Per-block outcome, filled by pskel_compress_blocks. */
typedef struct {
    int m, n;            /* block rows (test RWG) and columns (source RWG) */
    int r;               /* final sample count */
    int rank;            /* singular values kept by the pinv */
    int rank_recompressed; /* rank after recompression (0 if not run) */
    int rounds;          /* sampling rounds used (1 = first guess accepted) */
    int status;          /* PSKEL_OK or a negative status */
    double est;          /* randomized error estimate of the final round: the larger of the
                            relative errors on the extra rows and on the extra columns (pooled
                            over both sample sets for a re-checked block) */
} pskel_block_stat_t;

int pskel_create(pskel_ctx **ctx, int device);
int pskel_destroy(pskel_ctx *ctx);

/* Upload a mesh (reference layout, host arrays) and build the device quadrature records. */
int pskel_upload_mesh(pskel_ctx *ctx, const double *vertex, int nv, const double *topol,
                      int nt, const double *edges, int ne, const double *ln,
                      const double *cent, const pskel_em_t *em);

/* Fill Z(rows, cols) into a DEVICE buffer (column-major, leading dimension ld) with 0-based
   int32 RWG ids in DEVICE memory; precision PSKEL_C128 (pskel_c128*) or PSKEL_C64
   (pskel_c64*). Asynchronous on the context's stream. */
int pskel_fill_device(pskel_ctx *ctx, const int *rows_dev, int nr, const int *cols_dev,
                      int nc, void *Z_dev, int ld, int precision);

/* Fill Z(rows, cols) (complex FP64, DEVICE buffers as in pskel_fill_device) with the near-field
   rule of the reference's element routine (functionsExternal.so::impedance_matrix, the radii
   of compres_single_block_spheres.jl:800-840): per triangle pair with centroid distance dc, the
   4-point rule on the test side if dc < rinteg_f and on the source side if dc < rinteg_s (else
   the rule q_far: 1 = centroid as the reference, 7 = the 7-point rule), the static 1/R of the
   source triangle integrated exactly if dc < ranal_s, and the same-triangle term as a converged
   double integral (the reference's own is an approximation a few per cent off). One thread
   per entry. Asynchronous on the context's stream. */
int pskel_fill_near_device(pskel_ctx *ctx, const int *rows_dev, int nr, const int *cols_dev,
                           int nc, pskel_c128 *Z_dev, int ld, double rinteg_s, double ranal_s,
                           double rinteg_f, int q_far);

/* Groups (CSR over 0-based RWG ids) and the block list: block b = (test group gt[b],
   source group gs[b]). Host arrays; copied to the device. */
int pskel_set_blocks(pskel_ctx *ctx, const int *group_ptr, const int *group_ids,
                     int n_groups, const int *gt, const int *gs, int n_blocks);

/* Compress every block. r0 (host, n_blocks) is read when opts->start == PSKEL_START_GIVEN.
   stats (host, n_blocks) receives the per-block outcome. The factors stay on the device. */
int pskel_compress_blocks(pskel_ctx *ctx, const pskel_opts_t *opts, const int *r0,
                          pskel_block_stat_t *stats);

/* Timing and work counters of the last pskel_compress_blocks call: out[0..5] = device ms of
   the phases sample, fill, pinv, estimate (re-checks included), recompress (set by the last
   pskel_recompress after the compression) and the whole call (a round replayed from a CUDA
   graph is booked under fill as a whole); out[6] = entries filled, out[7] =
   point pairs evaluated, out[8] = fill launches, out[9] = rounds, out[10] = mean and out[11] =
   maximum Jacobi sweeps of the core SVDs. n = length of out (<= 12). */
int pskel_last_timing(pskel_ctx *ctx, double *out, int n);

/* Pipelining of a compression round of at least 2048 blocks: the blocks split into `chunks`
   (1 .. 8; default 2; 1 = off) of decreasing fill work; the fill of chunk k + 1 (one CTA per
   tile) overlaps the core SVD, pinv and estimate of chunk k, which run on a high-priority
   stream. The results are those of the unpipelined round. In a pipelined round the timing's
   fill phase covers all fills with the earlier chunks' pinv and estimate beside them, and the
   pinv phase the last chunk's pinv and estimate. */
int pskel_set_pipeline(pskel_ctx *ctx, int chunks);

/* Sample count of a block's next round: max(r + 1, ceil(factor * r)), capped by the block's
   smaller side (1 < factor <= 4; default 2, the reference's doubling,
   compres_single_block_spheres_for_sweep2.jl:878-973). */
int pskel_set_round_growth(pskel_ctx *ctx, double factor);

/* Copy block b's factors to host buffers (complex128): C m x r, U r x r, R r x n, 0-based
   local samples I (r) and J (r). Any pointer may be NULL. */
int pskel_get_block(pskel_ctx *ctx, int b, pskel_c128 *C, pskel_c128 *U, pskel_c128 *R,
                    int *I, int *J);

/* Fill-kernel variant used by this context for the complex128 and complex64 fills:
   8 = triangle-moment kernel (default; used when every group has at most 512 RWG, else 0),
   0 = per-entry kernel with two matrix rows per thread, 1, 2 or 4 = per-entry kernel with that
   many lanes per entry and a warp-shuffle reduction over the quadrature points, -1 = keep the
   current choice. Set by the autotuner. */
int pskel_set_fill_split(pskel_ctx *ctx, int split_c128, int split_c64);

/* Columns per CTA tile of the triangle-moment fill: 4, 8 (default) or 16, or 0 for a width per
   job (in [4, 16], the one whose triangle x column item count best fills a CTA's 256 threads).
   Chosen per GPU and workload by the autotuner (pskel/autotune.py), which times the variants
   on the block list. */
int pskel_set_tri_cols(pskel_ctx *ctx, int cols);

/* Pair geometry of the complex-FP32 triangle-moment fill: 0 = differences, distance and phase
   in FP64 (default); 1 = FP64 only per (triangle, column) item (the distance from the column's
   first point to the triangle centroid and its phase), FP32 per point pair from the two small
   offsets (phase error ~1e-7 turn). Selected by the autotuner. */
int pskel_set_fill_geometry(pskel_ctx *ctx, int fp32_offsets);

/* Symmetric mode (on = 1): of every pair of blocks (t, s) and (s, t) in the block list, only the
   one with the smaller index is compressed; the other is its transpose (the Galerkin EFIE matrix
   is symmetric, Z = Z^T, for equal test and source rules): C = R_p^T, U = U_p^T, R = C_p^T with
   the sample sets swapped, which is exactly the CUR that the other block's own round would form
   from those samples, with the same error. pskel_get_block, pskel_true_errors, pskel_matvec,
   pskel_recompress and the store treat such blocks as transposes. The per-block driving mode
   ignores it. No counterpart in the reference, which compresses single blocks. */
int pskel_set_symmetric(pskel_ctx *ctx, int on);

/* Single-level octree partition of the uploaded mesh's RWG basis functions and its far-field
   block list, built on the device. The reference has no partitioner: its multi-block driver
   (compres_single_block_spheres.jl:1109-1347) reads MATLAB-made block lists; this builds the
   partition its far-field workloads are defined on. Each RWG goes to the cube of side `leaf`
   (aligned at `origin`, 3 doubles; NULL = centre of the bounding box of the basis centres)
   holding its basis centre (user_get_OG_basis_center.m:36-39); groups are the non-empty cubes
   in Morton order; groups below `min_group` are folded, smallest first, into the nearest group
   (size-weighted centre); far pairs are (i, j), i != j (i < j if `symmetric`), with centres at
   least admissibility * sqrt(3) * leaf apart, in row-major order. Outputs the group and block
   counts; pskel_octree_get copies the result out. Exactly the host restatement's partition
   (every step IEEE-rounded in the same order). */
int pskel_octree_build(pskel_ctx *ctx, double leaf, const double *origin, double admissibility,
                       int min_group, int symmetric, int *n_groups, long long *n_blocks);

/* Write the recompressed far field (after pskel_recompress) to a file: the partition, per block
   its sizes, kept rank k and mirror link, the factors C' (m x k), S (k), R' (k x n) of every
   block that is not a transpose, and an FNV-1a hash (layout in csrc/storefile.cu). thresh is
   recorded as the recompression threshold used. No counterpart in the reference, which keeps
   its compressed blocks in Julia session files. */
int pskel_store_save(pskel_ctx *ctx, const char *path, double thresh);

/* Load such a file into a context whose mesh (same RWG count) is uploaded: installs its groups
   and blocks (as pskel_set_blocks) and its recompressed factors, after which
   pskel_get_recompressed, pskel_store_build and pskel_store_matvec run as after a
   pskel_recompress (pskel_matvec, the CUR form, needs the CUR factors and is refused). Rejects a
   wrong magic, version, RWG count, inconsistent records or a hash mismatch. n_blocks receives
   the block count. */
int pskel_store_load(pskel_ctx *ctx, const char *path, int *n_blocks);

/* Adaptive cross approximation of every far block of the block list (the comparison method of
   the reference's ACA-vs-CUR study: ACA_julia.jl:2-112, c_ACA.c:327-558), one CTA per block on
   the device, entries computed on demand in complex FP64 with the 7-point rule (the mesh must be
   uploaded with q = 7). Same steps as the reference: first row first, column pivot = largest
   unused entry of the row residual, row pivot = largest unused entry of the column residual,
   stop when ||U_k|| ||V_k|| <= tol ||U V||_F (from the second step), on a zero pivot or at full
   rank; kmax caps the rank (status 1 when it stops a block). In the symmetric mode one block of
   each (t, s) / (s, t) pair is approximated and the other is its transpose. ranks / status
   (host, n_blocks, may be NULL): rank k and 0 (converged or full rank), 1 (kmax reached) or 2
   (zero pivot). */
int pskel_aca_compress(pskel_ctx *ctx, double tol, int kmax, int *ranks, int *status);

/* Factors of block b after pskel_aca_compress: U (m x k, column-major), V (k x n, column-major),
   Z(rows, cols) ~ U V, and the pivot rows I / columns J (k each, 0-based within the block);
   any may be NULL. */
int pskel_aca_get_block(pskel_ctx *ctx, int b, pskel_c128 *U, pskel_c128 *V, int *I, int *J);

/* Relative Frobenius error of every ACA block against its dense complex-FP64 fill; err (host,
   n_blocks). */
int pskel_aca_true_errors(pskel_ctx *ctx, double *err);

/* Near-field blocks for the H-matrix product: the n_near group pairs (nt[b], ns[b]) of the
   groups set by pskel_set_blocks (normally every pair that is not far, diagonal included) are
   filled densely (complex FP64) with the near-field rule of pskel_fill_near_device and kept on
   the device; bytes receives their size. The reference assembles whole matrices from block lists
   (compres_single_block_spheres.jl:1404-1505) and solves them densely or by CBF
   (compres_single_block_spheres.jl:983-1017). */
int pskel_near_build(pskel_ctx *ctx, const int *nt, const int *ns, int n_near, double rinteg_s,
                     double ranal_s, double rinteg_f, int q_far, long long *bytes);

/* Y (+)= sum over near blocks of Z_b X(cols_b) scattered to rows_b (DEVICE complex-FP64 arrays,
   N x nrhs, nrhs <= 16; accumulate = 0 overwrites Y). With pskel_matvec (which overwrites Y with
   the far product) this is the whole H-matrix product. stream NULL = legacy default stream. */
int pskel_near_matvec(pskel_ctx *ctx, const pskel_c128 *X, int ldx, pskel_c128 *Y, int ldy,
                      int nrhs, int accumulate, void *stream);

/* Plane-wave excitation E (DEVICE, N complex FP64) of the uploaded mesh, as the reference's
   test_fields (compres_single_block_spheres_for_sweep2.jl:60-85): incidence theta_deg, phi_deg,
   polarisation rot_deg, the edge-weighted tangential field at the two triangle centroids. Like
   the reference, phi is divided by 180 without the factor pi. */
int pskel_plane_wave(pskel_ctx *ctx, double theta_deg, double phi_deg, double rot_deg,
                     pskel_c128 *E, void *stream);

/* Copy the last octree partition to host arrays (any may be NULL): group_ptr (G + 1 CSR
   offsets), group_ids (N 0-based RWG ids, ascending within each group), centres (G x 3
   row-major), extents (G diameters of the groups' bounding spheres about their mean centre),
   gt / gs (n_blocks test and source groups). The arrays feed pskel_set_blocks directly. */
int pskel_octree_get(pskel_ctx *ctx, int *group_ptr, int *group_ids, double *centres,
                     double *extents, int *gt, int *gs);

/* Relative Frobenius error of every block against a dense FP64 fill (device-side, block by
   block); err (host, n_blocks). */
int pskel_true_errors(pskel_ctx *ctx, double *err);
/* The same for the n blocks listed in blocks (host, 0-based): err[i] is block blocks[i]'s error
   (for a sample of a workload whose full dense fill would take long). */
int pskel_true_errors_blocks(pskel_ctx *ctx, const int *blocks, int n, double *err);

/* Dense reference of the far-field product: Y = sum over far blocks of Z_b X(cols_b) with every
   block filled densely in complex FP64 (the same rule as the compression), for checking a
   compressed product. X, Y: DEVICE pskel_c128 arrays (RWG count x nrhs, column-major, ldx and
   ldy >= RWG count); Y is overwritten. Runs on the context's stream and waits for it. */
int pskel_dense_far_matvec(pskel_ctx *ctx, const void *X, int ldx, void *Y, int ldy, int nrhs);

/* Compressed far-field matvec over every block of the last compression:
   Y(:, j) = sum_b P_t(b) C_b U_b R_b P_s(b)^T X(:, j), j < nrhs <= 64, with P_t, P_s the
   scatter/gather of the blocks' test and source groups (the near field is not included).
   Replaces, for all blocks and many right-hand sides at once, the per-block C(U(R v)) of
   codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:1929-1960 (cuda_complete_
   compression's error check). X (ldx >= RWG count) and Y (ldy >= RWG count) are DEVICE
   arrays, column-major, interleaved complex of the arithmetic precision (PSKEL_C128: double,
   PSKEL_C64: float); Y is overwritten. Enqueued on stream (NULL: the legacy default stream),
   returns without waiting; the first call after a compression also uploads the block table
   (synchronously). */
int pskel_matvec(pskel_ctx *ctx, const void *X, int ldx, void *Y, int ldy, int nrhs,
                 int precision, void *stream);

/* Recompression of every block's C U R into an SVD-truncated C' diag(S) R' (k terms kept,
   S > thresh * S_max, 0 <= thresh < 1): codes/ACA_vs_CUR/seed/svd_compress.m:19-33. Two paths:
   - FP64: Householder QR of C and R^H (in place of the unshipped qr_cbd), the QR-preconditioned
     Jacobi SVD of the r x r core R_c U R_r^H, the reflectors applied to the kept vectors;
   - split (complex-FP32 compressions, cores of rank <= 64): with the core's SVD from the
     compression, C U R = X S Yh^H where X = C V S^-1 and Yh = R^H W S^-1 are well conditioned;
     X, Yh and the rebuild C' = X Zx, R'^H = Yh Zy are tensor-core products of TF32 hi + lo
     operands with FP32 accumulation (~1e-6 relative), their Gram matrices, Cholesky factors,
     the core M = Lx^H S Ly and its Jacobi SVD are FP64; trailing terms of total weight below
     1e-2 thresh S_max are left out before the SVD. C' and R'^H are orthonormal to ~1e-6.
   The path is chosen per block (pskel_set_recompress_path): by default the split path for
   complex-FP32 compressions at thresh >= 1e-5, FP64 otherwise and for the blocks the split path
   hands back (rank above 64, a Cholesky breakdown, an unconverged SVD). ranks (host, n_blocks,
   may be NULL) receives k per block. The factors stay on the device until the next
   compression; the device time is reported as the "recompress" phase of pskel_last_timing. */
int pskel_recompress(pskel_ctx *ctx, double thresh, int *ranks);

/* Recompression path: 0 automatic (as above), 1 FP64 for every block, 2 the split path for
   every complex-FP32 block of rank <= 64 at any threshold. */
int pskel_set_recompress_path(pskel_ctx *ctx, int path);

/* Blocks of the last pskel_recompress that took the split path (the others, mirrors aside,
   took FP64). */
int pskel_recompress_split_blocks(pskel_ctx *ctx, int *split_blocks);

/* Copy block b's recompressed factors to host buffers: C' m x k, S (k, descending),
   R' k x n (complex128, column-major). Any pointer may be NULL. */
int pskel_get_recompressed(pskel_ctx *ctx, int b, pskel_c128 *Cp, double *S, pskel_c128 *Rp);

/* Compressed store of the recompressed blocks for the tensor-core matvec: diag(S) R' of the
   blocks stacked per source group and C' stacked per test group, in 128-row tiles laid out for
   the tensor cores, each real value in the operand format `mode`:
     PSKEL_STORE_BF16X3  bf16 hi + lo planes, three bf16 products per step (about 1e-5);
     PSKEL_STORE_TF32    one TF32 plane, one TF32 product (about 5e-4; the same bytes);
     PSKEL_STORE_TF32X3  TF32 hi + lo planes, three TF32 products (about 1e-6; twice the bytes).
   Requires pskel_recompress after the last compression. bytes (may be NULL) receives the size
   of the planes. No reference counterpart (the reference keeps each block's C, U, R apart). */
#define PSKEL_STORE_BF16X3 0
#define PSKEL_STORE_TF32 1
#define PSKEL_STORE_TF32X3 2
int pskel_store_build_mode(pskel_ctx *ctx, int mode, long long *bytes);
/* pskel_store_build_mode with PSKEL_STORE_BF16X3. */
int pskel_store_build(pskel_ctx *ctx, long long *bytes);

/* Y = sum over far blocks of C' diag(S) R' X for nrhs <= 16 right-hand sides, as two grouped
   GEMMs on the tensor cores (tcgen05 in the store's operand format, FP32 accumulation). X (ldx >= RWG count) and Y (ldy >= RWG count) are DEVICE arrays of pskel_c64,
   column-major; Y is overwritten. Enqueued on stream (NULL: the legacy default stream);
   returns without waiting. Replaces, for the recompressed blocks, the per-block C(U(R v)) of
   user_impedance_for_julia_cuda.cu:1929-1960. */
int pskel_store_matvec(pskel_ctx *ctx, const void *X, int ldx, void *Y, int ldy, int nrhs,
                       void *stream);
/* pskel_store_matvec with general strides, in pskel_c64 elements: X(i, j) at
   X[i x_row_stride + j x_col_stride], Y(i, j) at Y[i y_row_stride + j y_col_stride]; Y is
   column-major (y_row_stride 1, y_col_stride >= RWG count) or row-major (y_col_stride 1,
   y_row_stride >= nrhs). A row-major (RWG count, nrhs) tensor is passed without a transposed
   copy. No reference counterpart (the reference's matvec takes one vector). */
int pskel_store_matvec_strided(pskel_ctx *ctx, const void *X, long long x_row_stride,
                               long long x_col_stride, void *Y, long long y_row_stride,
                               long long y_col_stride, int nrhs, void *stream);

/* Error word of the last pskel_store_matvec (0: every pipeline wait completed; 1: a bounded
   wait ran out and the affected tiles were skipped). Waits for the device. */
int pskel_store_status(pskel_ctx *ctx, int *error_word);

/* ================================================= 3. rank / sample-count predictor (MLP) */
/* 8 -> 64 -> 64 -> 1 MLP with GELU in FP32 (parameter layout W1[64x8] b1[64] W2[64x64] b2[64]
   W3[1x64] b3[1], row-major, contiguous). All pointers are DEVICE pointers; stream may be
   NULL (legacy default stream). No counterpart in the reference, which grows the sample
   count adaptively only (compres_single_block_spheres_for_sweep2.jl:878-973). */
int pskel_mlp_num_params(void);
/* y[s] = MLP(x[s, 0:8]) for s < n (x row-major n x 8, standardised features). */
int pskel_mlp_forward(const float *params, const float *x, int n, float *y, void *stream);
/* grad = d/dparams of mean((MLP(x) - t)^2) over the batch; loss[0] = summed squared error. */
int pskel_mlp_grad(const float *params, const float *x, const float *t, int n, float *grad,
                   float *loss, void *stream);
/* One Adam step (t >= 1) on params with moment buffers m, v. */
int pskel_mlp_adam(float *params, const float *grad, float *m, float *v, int t, float lr,
                   float beta1, float beta2, float eps, void *stream);

/* Truncated pseudo-inverse P (N x M) of one complex128 matrix A (M x N), M, N <= 64, that
   allocates no device memory: for callers that cannot call cudaMalloc (a host framework that
   owns device memory through its own pool, or a latency-critical loop where an allocation
   could block or synchronise the device). No counterpart in the reference, whose pinv
   helpers allocate on every call. A and P (and the optional sigma, min(M, N) values sorted
   descending, and rank) are DEVICE buffers; singular values below tau (relative = 0) or
   tau * s_max (relative = 1) are dropped. The scratch is one fixed 256 KiB device array per
   GPU, shared by all calls: calls that overlap on the GPU race. The first call on a device
   looks up that array's address; make it before any stream capture. Returns after its stream
   has finished, with PSKEL_ERR_ARG for sizes above 64, PSKEL_ERR_NOCONV if the Jacobi
   sweeps did not converge and PSKEL_ERR_STATE, without doing anything, when the stream is
   being captured (the call waits for its stream). */
int pskel_pinv_noalloc(const pskel_c128 *A, int M, int N, double tau, int relative,
                       pskel_c128 *P, double *sigma, int *rank, void *stream);

/* Diagnostics: for n phases t (DEVICE array, in wavelengths) writes 8 values per phase to
   out: the fill kernels' own sin(2 pi t), cos(2 pi t) in FP64, the same in FP32, CUDA's
   sincospi(2 t) for comparison, then the half-turn FP32 form of the complex-FP32 fill with FP32
   pair geometry. Runs on the legacy default stream. No reference counterpart. */
int pskel_diag_sincos(const double *t, int n, double *out);

/* Device kernels launched by this library since load (graph replays count their kernel
   nodes); used to report how many of the library's kernels ran in a timed region. */
long long pskel_kernel_launches(void);

/* Measured FMA throughput of this GPU's FP32 and FP64 pipes (TFLOP/s, 2 flops per FMA), from
   a dependent-chain microbenchmark of about a hundred milliseconds. */
int pskel_fma_peak(double *fp32_tflops, double *fp64_tflops);

#ifdef __cplusplus
}
#endif
#endif /* PSKEL_H */
