// Internal state of the pskel_* handle API (engine.cu, blockops.cu).
#pragma once

#include <vector>

#include "pskel_internal.cuh"

namespace pskel {

constexpr int kMaxGroup = 8192;  // largest m or n the sampler accepts
constexpr int kMaxExtra = 32;

struct BlockWork {
    const int *rows_g;  // global RWG ids of the test group (m)
    const int *cols_g;  // global RWG ids of the source group (n)
    int m, n, r, pe, pc;
    int block_id, round;
    int *I, *J, *Ix, *Jx;  // local indices (sorted)
    int *Ig;            // global ids of rows I then Ix (r + pe)
    int *Jg;            // global ids of columns J then Jx (r + pc)
    void *C;            // m x (r + pc): C = Z(:, J), then the extra columns Z(:, Jx)
    void *Rx;           // (r + pe) x n, ld = r + pe: R = Z(I, :), then the extra rows Z(Ix, :)
    double2 *AV, *V, *U;
    double2 *T;         // estimator scratch: C(Ix, :) U (pe x r), then U R(:, Jx) (r x pc)
    double *sigma;
    int *perm, *rank;
    double *est;
};

// Single-level octree partition of the uploaded mesh's RWG basis centres and its far-pair list,
// built on the device (csrc/octree.cu). Group ids, extents and the far list stay in device
// memory; offsets and centres are kept on the host as well.
struct OctreeState {
    DevBuf hdr, c, idx, ka, kb, va, vb, cnt, start, bc, map, fkey, fkey2, gids, gptr, fc, ext;
    DevBuf rowcnt, rowoff, gt, gs, tmp;
    int n = 0, n_groups = 0;
    long long n_blocks = 0;
    std::vector<int> h_gptr;
    std::vector<double> h_centres;  // (G, 3) row-major
    bool valid = false;
};
void octree_release(OctreeState &o);

}  // namespace pskel

using pskel::BlockWork;
using pskel::DevBuf;
using pskel::DevMesh;

struct BlockResult {
    int m = 0, n = 0, r = 0, pe = 0, pc = 0, round = -1, rank = 0, status = 0;
    double est = 0;
    int arena = -1;
    size_t offC = 0, offRx = 0, offU = 0, offI = 0, offJ = 0;
    // the core's SVD from the pinv (offsets in the round arena): A V (work, r x r), V (work,
    // r x r), sigma and its decreasing order (keep); `rank` columns were kept by the pinv
    size_t offAV = 0, offV = 0, offSig = 0, offPerm = 0;
    // >= 0: this block is the transpose of block `mirror` (Galerkin symmetry Z = Z^T), whose
    // factors it shares: C = R_p^T, U = U_p^T, R = C_p^T, I = J_p, J = I_p. m and n are this
    // block's own sizes; the other fields describe the primary's storage.
    int mirror = -1;
};

struct RoundArena {
    DevBuf keep;     // C, Rx, U, samples, sigma, est ... of the blocks of the round
    DevBuf work;     // AV, V of the round and the storage of its re-checks (scratch, but owned
                     // per round so that a captured round keeps valid pointers while later
                     // rounds grow their own)
    DevBuf tables;   // device copies of the job tables
    DevBuf outs;     // RoundOut per block of the round, then its re-checks' sums and gates
};

struct RecompSlot {
    double2 *Cp = nullptr;  // m x k, ld m
    double2 *Rp = nullptr;  // k x n, ld ldrp (>= k)
    double *S = nullptr;    // k, decreasing
    int k = 0;
    int mirror = -1;  // >= 0: the transpose of that block's recompression (pointers are its)
    int ldrp = 0;
};

// Compressed store of the recompressed blocks (csrc/store.cu): host copy of its layout.
struct StoreTile {
    long long a_off, b_off;  // A and B offsets (bf16 elements) within the phase's region
    int kc, rows, out0;      // K chunks, valid rows, first T row (phase 1) or first row of the
                             // test group's 2m-row stack (phase 2)
    int phase;
    int ids0 = 0, m = 0;     // phase 2: the test group's first id and its rows
};
struct StoreGroup {
    long long b_base;  // B offset within the phase's region
    int kc, K;         // chunks, real K
    int ids0;          // offset of the group's ids in the group id list
};
struct StoreLayout {
    std::vector<StoreTile> tiles1, tiles2;
    std::vector<StoreGroup> groups1;  // source groups (phase-1 B operands, built per matvec)
    long long a1 = 0, a2 = 0, b1 = 0, b2 = 0;
    int trows = 0;
    int n_items1 = 0, n_items2 = 0;  // GEMM work items per phase
    int n_bitems1 = 0;  // phase-1 B-builder work items (8-chunk blocks)
    void *d_t1 = nullptr, *d_t2 = nullptr, *d_g1 = nullptr, *d_bi1 = nullptr;
    bool ready = false;
    long long generation = -1;
    int mode = PSKEL_STORE_BF16X3;  // operand format of the planes
};

struct pskel_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6] = {};
    pskel::SvdStreams svd_par;  // side streams of the concurrent SVD size classes
    // pipelined round: the blocks split into chunks; the pinv and estimate of chunk k run on a
    // high-priority stream while the fill of chunk k + 1 runs on the context's stream
    static constexpr int kMaxChunks = 8;
    cudaStream_t pipe_stream = nullptr;
    cudaEvent_t pipe_ev[kMaxChunks + 1] = {};
    cudaEvent_t chunk_ev[kMaxChunks] = {};  // a chunk's outcome collected (its re-check may start)
    int pipe_chunks = 2;        // chunks of a round with at least kPipeMinBlocks blocks (1: off)
    double growth = 2.0;        // sample count factor from one round to the next (2: doubling)
    DevMesh mesh;
    pskel_em_t em{};
    bool have_mesh = false;
    DevBuf flags;
    int n_groups = 0, n_blocks = 0;
    std::vector<int> gptr, gids, gt, gs;
    DevBuf d_gids;
    // triangle structure of the groups for the triangle-moment fill
    std::vector<int> h_edges;            // T+, T-, v+, v- per RWG (0-based), host copy
    std::vector<int> gtri_ptr;           // CSR offsets into gtri / (3x) gadj
    DevBuf d_gtri, d_gadj;
    DevBuf d_guse;                       // per (group triangle, slot): free vertex - centroid, s l
    std::vector<double> h_vertex, h_ln, h_cent;  // host copies of the mesh arrays it is built from
    bool use_tri = false;
    std::vector<RoundArena> arenas;
    std::vector<BlockResult> graph_results;  // round-0 result slots of the captured graph
    std::vector<BlockResult> results;
    int precision = PSKEL_C128;
    int split[2] = {8, 8};  // fill variant: 8 triangle moments, 0 two rows per thread, 1/2/4 lanes per entry
    int tri_cols = pskel::kTriFillColsDefault;  // columns per CTA of the triangle-moment fill
    int geom32 = 0;  // complex-FP32 fill: 1 = FP32 pair geometry from per-item offsets
    int symmetric = 0;        // compress one block of each (t, s) / (s, t) pair, mirror the other
    std::vector<int> partner; // per block: index of the block with swapped groups, or -1
    double timing[13] = {};  // [0..11] as reported by pskel_last_timing, [12] core SVD count
    // CUDA graph of the first round
    cudaGraphExec_t graph = nullptr;
    long long graph_kernels = 0;  // kernel nodes of the captured graph
    std::vector<int> graph_key;
    std::vector<int> last_key;  // round-0 key of the previous call (capture on a repeat)
    DevBuf tmp, tmp2, tmp3;
    DevBuf recomp;                          // recompressed factors (split path, loaded store)
    DevBuf recomp64, recomp64b;             // FP64 path: recompressed factors and workspace
    DevBuf rc_work, rc_tab, rc_idx;         // split path: workspace, job tables, SVD order
    pskel::PinnedBuf rc_host;               // split path: host copy of the job tables
    pskel::PinnedBuf plan_host;             // a compression round's job tables, staged for upload
    std::vector<pskel::SvdJob> rc_hs;       // split path: host SVD jobs (kept: no per-call allocation)
    int recomp_path = 0;                    // 0 auto, 1 FP64 only, 2 split whenever eligible
    int recomp_split_blocks = 0;            // blocks of the last recompression on the split path
    std::vector<RecompSlot> recomp_slots;   // per block: C', R', S and the rank k
    long long generation = 0;               // incremented by every compression
    DevBuf mv_table;                        // matvec block table (built once per compression)
    long long mv_generation = -1;
    int mv_max_r = 0, mv_max_m = 0, mv_max_n = 0, mv_chunks = 0;  // largest rank / groups, chunks
    size_t mv_chunk_off = 0;                        // byte offset of the chunk table in mv_table
    StoreLayout store;                      // compressed store (bf16 hi/lo planes, tiled)
    DevBuf st_ah, st_al, st_bh, st_bl, st_t, st_tab, st_tiles, st_err;  // st_t: phase-1 row places
    pskel::OctreeState octree;              // device octree partition (pskel_octree_build)
    DevBuf near_jobs, near_mom;             // near-field fill: job table, same-triangle moments
    DevBuf near_data, near_tab;             // near blocks (dense complex FP64) and their table
    int n_near = -1, near_max_n = 0;        // -1: no near blocks built
    // adaptive cross approximation of the far blocks (csrc/aca.cu)
    DevBuf aca_buf, aca_tab;
    std::vector<int> aca_k, aca_status, aca_mirror;
    std::vector<size_t> aca_offU, aca_offV, aca_offI, aca_offJ;
    int aca_kmax = 0;
    float aca_ms = 0.0f;
};

namespace pskel {
// Recompression (csrc/blockops.cu, csrc/recomp_tc.cu) of primary blocks: the FP64 path, and the
// split-precision tensor-core path with the blocks it hands back to the FP64 one.
struct Fp64Recomp {  // one enqueued FP64 recompression
    std::vector<int> prims;
    SvdJob *d_s2 = nullptr;
    int *d_k = nullptr;
    cudaStream_t st = nullptr;
};
int recompress_fp64_enqueue(pskel_ctx *c, const std::vector<int> &prims, double thresh, cudaStream_t st,
                            DevBuf &buf, Fp64Recomp &out);
int recompress_fp64_finish(pskel_ctx *c, Fp64Recomp &r);
bool recomp_split_eligible(const pskel_ctx *c, int b, double thresh);
// moves the split-eligible blocks whose pinv kept core values below the split products'
// accuracy (see recomp_tc.cu) from `split` to `fp64` (one device check and read-back)
int recomp_split_precheck(pskel_ctx *c, double thresh, std::vector<int> &split, std::vector<int> &fp64);
int recompress_split(pskel_ctx *c, const std::vector<int> &blocks, double thresh, std::vector<int> &rejected);
}  // namespace pskel
