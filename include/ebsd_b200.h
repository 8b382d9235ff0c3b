/*
 * ebsd_b200 — C-ABI of the B200 (sm_100a) dictionary-indexing kernels.
 *
 * The reference (ebsdtorch, pure Python/PyTorch) has no native interface; its
 * dictionary-indexing path is a chain of PyTorch calls inside
 *   ebsdtorch/ebsd/indexing.py:14-211   dictionary_index_orientations
 *   ebsdtorch/ebsd/indexing.py:214-476  pca_dictionary_index_orientations
 * Each entry point below replaces one link of that chain; the comment on it
 * names the reference code it stands in for. The Python package
 * ebsdtorch_b200 binds these symbols with ctypes and mirrors the reference's
 * Python API on top of them.
 *
 * Conventions
 *  - All pointers are device pointers unless stated otherwise; buffers are
 *    allocated by the caller. The library makes no device allocation of its
 *    own; its only device memory is the 32 MiB scratch array of
 *    ebsd_match_topk_noalloc, part of the module image, which every GPU
 *    that loads the library holds until the process exits.
 *  - Work is enqueued on `stream` (a cudaStream_t passed as void*); calls are
 *    asynchronous unless stated otherwise.
 *  - Return value: 0 success, > 0 argument error (nothing launched),
 *    < 0 negated cudaError_t. ebsd_last_error() returns the message.
 *  - Kernels that spin-wait take `int* d_status` (device int, zero before
 *    the call); a wait that exceeds its limit stores EBSD_DEVICE_TIMEOUT there
 *    and the kernel returns early instead of hanging.
 *  - Low-precision row layouts ("lp rows"): row-major, `ld` elements per row,
 *    ld a multiple of 64 (bf16) or 128 (e4m3), padding zero-filled.
 */
#ifndef EBSD_B200_H
#define EBSD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EBSD_OK 0
#define EBSD_ERR_ARG 1
#define EBSD_ERR_UNSUPPORTED 2
#define EBSD_DEVICE_TIMEOUT 0x7001

/* element types of low-precision rows */
#define EBSD_DT_F32 0
#define EBSD_DT_BF16 1
#define EBSD_DT_E4M3 2

/* ---- library ---------------------------------------------------------- */

/* Library version (major*10000 + minor*100 + patch). */
int ebsd_version(void);

/* Debug checks: in the library built with -DEBSD_CHECK, kernels test their
 * computed shared-memory, TMEM and global offsets; a failed check records
 * its source line and skips the access. Returns the first recorded line (0
 * when none; the file name goes to `file`) and clears the records; -1 when
 * the library was built without checks. */
int ebsd_debug_check_line(char* file, size_t n);

/* Copy the last error message of this host thread into buf (NUL-terminated).
 * Returns the full message length. */
int ebsd_last_error(char* buf, size_t n);

/* 0 if `device` is an sm_100 GPU this library can run on. */
int ebsd_device_check(int device);

/* ---- A1/A2: SO(3) cubochoric grid restricted to a Laue fundamental zone ---
 * Replaces ebsdtorch/s2_and_so3/laue_fz_ori.py:516-557
 * (sample_ori_fz_laue_angle: so3_cubochoric_grid sampling.py:179-205,
 *  cu2qu orientations.py:1136, ori_in_fz_laue laue_fz_ori.py:144-239).
 * Computed in FP64. The random permutation of the reference (torch.randperm on
 * the global CPU generator) is applied by the caller with ebsd_gather_rows. */

/* Bytes of workspace needed for an edge^3 grid. */
size_t ebsd_grid_workspace_bytes(int edge_length);

/* Pass 1: FZ membership of all edge^3 grid points; writes the number of FZ
 * points to *d_count (device int64). */
int ebsd_grid_fz_count(int laue_id, int edge_length, void* workspace, size_t workspace_bytes,
                       int64_t* d_count, void* stream);

/* Pass 2 (after pass 1 on the same workspace): the FZ quaternions (w,x,y,z),
 * w >= 0, in the reference's grid order, to out_f32 (n x 4) and, if not NULL,
 * out_f64 (n x 4) and out_cells (n, the linear grid index (i*e + j)*e + k of
 * each point). */
int ebsd_grid_fz_write(int laue_id, int edge_length, const void* workspace, size_t workspace_bytes,
                       float* out_f32, double* out_f64, int32_t* out_cells, void* stream);

/* out[i, :] = in[index[i], :] for rows of `width` floats.
 * Replaces the `so3_samples_fz[torch.randperm(n)]` gather
 * (laue_fz_ori.py:554-555) and `ori_tensor[matches]` (indexing.py:205). */
int ebsd_gather_rows(const float* in, int64_t n_in, int width, const int64_t* index, int64_t n_out,
                     float* out, void* stream);

/* ---- A4-A7: dictionary projector ----------------------------------------
 * Replaces, per dictionary chunk, indexing.py:117-143 — qu_apply
 * (quaternions.py:186-213), MasterPattern.interpolate (master_pattern.py:
 * 141-209: rosca_lambert_side_by_side sphere.py:145-185 then bilinear
 * grid_sample, align_corners=False, padding_mode="border"), the signal mask
 * column select and the row mean subtraction.
 *
 * master_pattern: (mp_h, mp_w2) fp32, north | south hemispheres side by side.
 * rays_soa:       3 x n_pix fp32 unit rays (x row, y row, z row), already
 *                 masked.
 * quats:          (n_rows, 4) fp32 orientations.
 * Outputs (each may be NULL):
 *   out_f32 (n_rows x ld_f32): zero-mean rows (or raw rows if !subtract_mean)
 *   out_lp  (n_rows x ld_lp) : those rows scaled to unit L2 norm, in lp_dtype;
 *                              e4m3 rows are further scaled by 1/out_lp_scale
 *   out_norm (n_rows)        : L2 norm of the zero-mean row
 *   out_lp_scale (n_rows)    : e4m3 dequantisation scale (absmax/448) */
int ebsd_project_dictionary(const float* master_pattern, int mp_h, int mp_w2, const float* rays_soa,
                            int n_pix, const float* quats, int64_t n_rows, int subtract_mean,
                            float* out_f32, int64_t ld_f32, void* out_lp, int lp_dtype, int64_t ld_lp,
                            float* out_norm, float* out_lp_scale, void* stream);

/* ---- A8: pattern preparation ----------------------------------------------
 * Replaces ExperimentPatterns.get_patterns (experiment_pats.py:318-346:
 * avg_pool2d binning) and indexing.py:175-187 (mask select, row mean
 * subtraction). patterns: n_rows images of (height, width) fp32, image i at
 * patterns + i * pattern_stride. pix_index (n_pix int32 indices into the
 * binned image, row-major) may be NULL for all binned pixels. Outputs as for
 * ebsd_project_dictionary. Also used with height = 1 to normalise generic
 * fp32 rows (PCA-projected rows). */
int ebsd_prep_patterns(const float* patterns, int64_t n_rows, int height, int width,
                       int64_t pattern_stride, int binning, const int32_t* pix_index, int n_pix,
                       int subtract_mean, float* out_f32, int64_t ld_f32, void* out_lp, int lp_dtype,
                       int64_t ld_lp, float* out_norm, float* out_lp_scale, void* stream);
/* Same, for patterns stored as detector counts or half floats:
 * pattern_dtype EBSD_PAT_F32 (float), EBSD_PAT_U16 (uint16), EBSD_PAT_U8
 * (uint8) or EBSD_PAT_F16 (IEEE half); values are converted to FP32 before
 * binning. pattern_stride is in elements. (The reference keeps its
 * ExperimentPatterns in float; integer counts halve or quarter the bytes read
 * and copied.) */
#define EBSD_PAT_F32 0
#define EBSD_PAT_U16 1
#define EBSD_PAT_U8 2
#define EBSD_PAT_F16 3
int ebsd_prep_patterns_typed(const void* patterns, int pattern_dtype, int64_t n_rows, int height, int width,
                             int64_t pattern_stride, int binning, const int32_t* pix_index, int n_pix,
                             int subtract_mean, float* out_f32, int64_t ld_f32, void* out_lp, int lp_dtype,
                             int64_t ld_lp, float* out_norm, float* out_lp_scale, void* stream);

/* Bilinear sample of the side-by-side master pattern at n points on the
 * sphere (xyz, n x 3 fp32; normalised first when `normalize`), grid_sample
 * semantics align_corners=False, padding_mode="border".
 * Replaces MasterPattern.interpolate (master_pattern.py:141-209). */
int ebsd_sample_master_pattern(const float* master_pattern, int mp_h, int mp_w2, const float* xyz,
                               int64_t n, int normalize, float* out, void* stream);

/* b x b average pooling of n images (MasterPattern.bin, master_pattern.py:
 * 94-113). out: n x (height/b) x (width/b). */
int ebsd_avg_pool(const float* in, int64_t n, int height, int width, int binning, float* out,
                  void* stream);

/* ---- A9/A10: pattern x dictionary contraction with streaming top-k ------
 * Replaces knn_batch (ebsdtorch/utils/knn.py:80-103, `query @ data.t()` then
 * torch.topk) and the ChunkedKNN running merge (knn.py:219-266). One tcgen05
 * kernel: TMA-fed smem tiles, FP32 accumulators in TMEM, and an epilogue that
 * keeps each query's best `n_cand` candidates in registers, so the
 * similarity matrix never reaches HBM.
 *
 * queries_lp: (n_queries_pad x k_pad) lp rows, n_queries_pad % 128 == 0.
 * dict_lp:    (n_dict_pad x k_pad) lp rows,    n_dict_pad % 256 == 0.
 * score(q, d) = dot(queries_lp[q], dict_lp[d]) * col_scale[d]
 *               (col_scale NULL means 1); columns d >= n_dict_valid ignored.
 * n_cand in {1, 2, 4, 8, 16, 32, 64}. splits: number of dictionary ranges
 * (0 = automatic, see ebsd_match_auto_splits). Each (query tile, range) writes
 * its best n_cand (score, index + index_base) per query, sorted descending, to
 *   part_val/part_idx[(q * part_slots + slot_base + range) * n_cand + j].
 * part_slots >= slot_base + splits. */
int ebsd_match_auto_splits(int64_t n_queries_pad, int64_t n_dict_pad);
/* The automatic number of dictionary ranges for rows of lp_dtype (the launch
 * variant, and so the plan, may depend on the element type: see
 * ebsd_set_match_dual); ebsd_match_auto_splits plans for bf16 rows. */
int ebsd_match_auto_splits_typed(int64_t n_queries_pad, int64_t n_dict_pad, int lp_dtype);

/* No counterpart in the reference (which has no device-side waits): sets the
 * limit, in nanoseconds, of every bounded wait inside the tensor-core kernels
 * launched after the call (ebsd_match_topk*, ebsd_gemm_nt, ebsd_cnn_conv_fwd
 * and the allocation-free match); ns <= 0 restores the default of 4 s.
 * Returns the previous limit. A wait that runs out stores
 * EBSD_DEVICE_TIMEOUT in the call's status word, and the kernel returns
 * after its own copies and MMAs have completed, leaving the context usable.
 * Meant for tests and for callers that want a tighter watchdog. */
int64_t ebsd_set_wait_limit_ns(int64_t ns);

/* No counterpart in the reference: on != 0 runs the top-k matches launched
 * after the call as CTA pairs where they can (256-row dictionary tiles, the
 * angular ranking, an even number of 128-row query tiles and no persistent
 * launch): the two CTAs of a cluster share one tcgen05.mma.cta_group::2 of
 * M = 256 query rows, and each stages half of every dictionary tile. Results
 * and the partial-result layout are the same as the one-CTA kernel's.
 * Returns the previous setting (0 by default); on < 0 only returns it. */
int ebsd_set_match_pairs(int on);
/* No counterpart in the reference: which eligible top-k matches that follow
 * (as for ebsd_set_match_pairs) take TWO query tiles per CTA: two M = 128
 * MMAs per K step share one staged 256-row dictionary tile, a third less
 * operand traffic from L2 per FLOP. mode 0: none; 1: all; 2 (default): those
 * of e4m3 rows. ebsd_match_auto_splits_typed then plans twice the dictionary
 * ranges. Results and the partial-result layout are the same as the one-tile
 * kernel's. CTA pairs, when on, take precedence. Returns the previous mode;
 * mode < 0 only returns it. */
int ebsd_set_match_dual(int mode);
/* Clusters of the pair kernel that fit on the current device at once (one
 * wave), or a negative CUDA error. */
int ebsd_match_pair_max_clusters(void);


int ebsd_match_topk(const void* queries_lp, int64_t n_queries_pad, const void* dict_lp,
                    int64_t n_dict_pad, int64_t n_dict_valid, int64_t k_pad, int lp_dtype,
                    const float* col_scale, int n_cand, int splits, float* part_val,
                    int32_t* part_idx, int part_slots, int slot_base, int32_t index_base,
                    int* d_status, void* stream);
/* The same match with the launch shape chosen by the caller (the batch
 * planner's autotuner): tile_n 128 or 256 dictionary rows per CTA tile (0 =
 * 256; n_dict_pad must be a multiple of it), and max_ctas > 0 for a
 * persistent launch of min(units, max_ctas) CTAs that each loop over work
 * units u, u + grid, ... (0 = one CTA per unit). Splits larger than the
 * number of dictionary tiles are reduced to it. col_bias / row_scale (both
 * or neither; 16-byte aligned; row_scale has n_queries_pad entries) add
 * col_bias[d] * row_scale[q] to every score: with col_scale = 2 |d|,
 * col_bias = -|d|^2 and row_scale = 1 / |q| on unit rows the scores rank
 * by the smallest squared euclidean distance (knn.py:85-91). */
int ebsd_match_topk_tiled(const void* queries_lp, int64_t n_queries_pad, const void* dict_lp,
                          int64_t n_dict_pad, int64_t n_dict_valid, int64_t k_pad, int lp_dtype,
                          const float* col_scale, const float* col_bias, const float* row_scale,
                          int n_cand, int splits, float* part_val, int32_t* part_idx,
                          int part_slots, int slot_base, int32_t index_base, int tile_n, int max_ctas,
                          int* d_status, void* stream);

/* ---- A10 (final) + FP32 re-score ------------------------------------------
 * Replaces ChunkedKNN.retrieve_topk (knn.py:268-287). Per query: merge the
 * part_slots x n_cand candidate lists, take the best n_rescore by the
 * approximate score, recompute their exact FP32 scores, optionally merge
 * with a running result (run_val/run_idx, k_out per query, may be NULL; its
 * indices must not overlap the new candidates'), and write the best k_out
 * sorted descending (ties: lower index first; missing entries -inf / -1).
 *   similarity EBSD_SIM_DOT:    exact = q_f32[q] . d_f32[idx - d_index_base]
 *                               (n_pix terms), the reference metric (knn.py:96-97)
 *   similarity EBSD_SIM_COSINE: exact = that dot / (q_norm[q] d_norm[idx - d_index_base])
 *   similarity EBSD_SIM_EUCLIDEAN: the squared distance
 *                               q_norm[q]^2 + d_norm[.]^2 - 2 dot (knn.py:85-91); the
 *                               best k_out are the smallest, sorted ascending, and
 *                               missing entries are +inf / -1; run_val holds distances
 *   similarity EBSD_SIM_MANHATTAN: candidates scored -L1 (ebsd_manhattan_topk), no
 *                               re-score (d_f32 NULL); distances out, as for euclidean
 * (candidate indices are global; d_f32/d_norm hold rows d_index_base ..
 * d_index_base + d_rows - 1; a candidate outside that range is dropped)
 * With d_f32 == NULL nothing is re-scored and the score is
 *   s = approx * (q_lp_scale ? q_lp_scale[q] : 1) * (DOT or EUCLIDEAN ? q_norm[q] : 1),
 * and the euclidean distance q_norm[q]^2 - s. */
#define EBSD_SIM_DOT 0
#define EBSD_SIM_COSINE 1
#define EBSD_SIM_EUCLIDEAN 2
#define EBSD_SIM_MANHATTAN 3
int ebsd_merge_rescore(const float* part_val, const int32_t* part_idx, int64_t n_queries,
                       int part_slots, int n_cand, const float* q_f32, int64_t ld_q,
                       const float* d_f32, int64_t ld_d, int64_t d_index_base, int64_t d_rows,
                       int n_pix,
                       const float* q_norm, const float* d_norm, const float* q_lp_scale,
                       int similarity, int n_rescore,
                       int k_out, const float* run_val, const int64_t* run_idx, float* out_val,
                       int64_t* out_idx, void* stream);

/* ---- distance_metric="manhattan" -------------------------------------------
 * Replaces knn_batch's manhattan branch (knn.py:92-93: the L1 distance of the
 * zero-mean rows, smallest first), which is not a contraction: FP32 rows on
 * the CUDA cores. q_f32 (n_queries x n_pix, row stride ld_q; n_queries_pad a
 * multiple of 64), d_f32 (n_dict x n_pix, stride ld_d). The dictionary is cut
 * into `splits` ranges (1 <= splits <= ceil(n_dict / 64)); each (64-query
 * tile, range) writes its best n_cand (score = -L1, index + index_base),
 * sorted best first, in ebsd_match_topk's candidate layout (rows up to
 * n_queries_pad). ebsd_merge_rescore(_gated) with EBSD_SIM_MANHATTAN and no
 * re-score turns them into distances. */
int ebsd_manhattan_topk(const float* q_f32, int64_t ld_q, int64_t n_queries, int64_t n_queries_pad,
                        const float* d_f32, int64_t ld_d, int64_t n_dict, int n_pix, int n_cand, int splits,
                        float* part_val, int32_t* part_idx, int part_slots, int slot_base, int32_t index_base,
                        void* stream);

/* As ebsd_merge_rescore, with a margin gate on the FP32 re-score (no
 * counterpart in the reference, which scores every candidate in its match
 * dtype). gate_rel > 0 must bound |s' - s| / w for every candidate, where s'
 * is the low-precision score per unit query norm, s the exact one, and w the
 * dictionary row norm (dot metric) or 1 (cosine). Only candidates whose upper
 * bound s' + gate_rel * w reaches the k_out-th largest lower bound among the
 * n_rescore best are re-scored; the others cannot be in the exact top k_out,
 * so the result equals ebsd_merge_rescore's. gate_rel = 0 re-scores all
 * n_rescore. n_rescored (may be NULL) accumulates the number of rows
 * re-scored. */
int ebsd_merge_rescore_gated(const float* part_val, const int32_t* part_idx, int64_t n_queries,
                             int part_slots, int n_cand, const float* q_f32, int64_t ld_q,
                             const float* d_f32, int64_t ld_d, int64_t d_index_base, int64_t d_rows,
                             int n_pix, const float* q_norm, const float* d_norm,
                             const float* q_lp_scale, int similarity, int n_rescore, int k_out,
                             const float* run_val, const int64_t* run_idx, float* out_val,
                             int64_t* out_idx, float gate_rel, unsigned long long* n_rescored,
                             void* stream);

/* ---- allocation-free match ------------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot call cudaMalloc where they index patterns -- e.g. a detector
 * acquisition callback that must never block (cudaMalloc / cudaFree can
 * synchronise the device), or a host application that owns all device memory
 * and forbids its plugins to allocate. Same result as ebsd_match_topk followed
 * by ebsd_merge_rescore without re-scoring: per query the best k_out
 * (1..64) candidates by dot(queries_lp[q], dict_lp[d]) * col_scale[d] *
 * (q_scale ? q_scale[q] : 1), sorted descending, into out_val / out_idx
 * (n_queries x k_out); if out_status is not NULL the device status word
 * (0 or EBSD_DEVICE_TIMEOUT) is copied there.
 * The candidate-list scratch is a fixed 32 MiB device array inside the library
 * (held by every GPU that loads it until the process exits), so
 * n_queries_pad * next_pow2(k_out) * 8 bytes must not exceed 32 MiB - 256 B;
 * larger calls are rejected with EBSD_ERR_ARG. No cudaMalloc, cudaFree or
 * allocating library routine is called. The first call on each device looks
 * up the array's device address (cudaGetSymbolAddress, with that device
 * current); make that first call before any stream capture. Under CUDA's
 * lazy module loading (the default) that first lookup also loads the module,
 * which allocates the array and can block or fail for lack of memory: make
 * one warm-up call at set-up time, not from the callback that must not
 * block. The address is cached per device ordinal for the runtime's primary
 * context: other driver contexts and use after cudaDeviceReset are not
 * supported. All calls share the array and it keeps the last call's
 * contents: calls that overlap on the GPU race and must be serialised by the
 * caller. */
int ebsd_match_topk_noalloc(const void* queries_lp, int64_t n_queries, int64_t n_queries_pad,
                            const void* dict_lp, int64_t n_dict_pad, int64_t n_dict_valid,
                            int64_t k_pad, int lp_dtype, const float* col_scale,
                            const float* q_scale, int k_out, float* out_val, int64_t* out_idx,
                            int* out_status, void* stream);

/* ---- A11/A12: PCA -------------------------------------------------------------
 * C (m_valid x n_valid, row stride ldc) = alpha * A B^T (+ C if accumulate),
 * A (m_pad x k_pad), B (n_pad x k_pad) lp rows, m_pad % 128 == 0,
 * n_pad % 256 == 0. tcgen05 kernel with a store epilogue.
 * splits <= 0 gives one 256-row B tile per work unit; splits > 0 makes each
 * (A tile, B range) unit stream n_pad / 256 / splits B tiles. Used for the
 * covariance (pca_covmat.py:53-91 einsum), the PCA projections
 * (indexing.py:401, 421, 452 torch.matmul) and the CNN gradient GEMMs. */
int ebsd_gemm_nt(const void* A, int64_t m_pad, const void* B, int64_t n_pad, int64_t k_pad,
                 int lp_dtype, float alpha, int accumulate, float* C, int64_t ldc, int64_t m_valid,
                 int64_t n_valid, int splits, int* d_status, void* stream);

/* C (m x n, row stride ldc) = alpha * A B^T (+ C if accumulate) from FP32
 * rows A (m x k, stride lda) and B (n x k, stride ldb), read as TF32
 * (rounded on the copy) by the same tcgen05 kernel (kind::tf32); no padding
 * needed (lda, ldb multiples of 4, 16-byte aligned operands). The PCA
 * projections (indexing.py:401, 421, 452). splits as for ebsd_gemm_nt. */
int ebsd_gemm_f32(const float* A, int64_t lda, int64_t m, const float* B, int64_t ldb, int64_t n, int64_t k,
                  float alpha, int accumulate, float* C, int64_t ldc, int splits, int* d_status, void* stream);

/* Column means of an (n_rows x n_cols) fp32 matrix (row stride ld). */
int ebsd_col_mean(const float* X, int64_t n_rows, int n_cols, int64_t ld, float* mean, void* stream);

/* Three-term bf16 split of fp32 data so that one bf16 GEMM over a tripled K
 * reproduces an FP32-accurate product: x = hi + lo, and
 *   pattern 0 writes [hi | hi | lo], pattern 1 writes [hi | lo | hi]
 * (segments of seg_len elements, zero padded). transpose = 0: row r of X
 * (minus shift, if not NULL, per column) becomes row r of out (n_rows x ld_out,
 * ld_out >= 3 * seg_len, seg_len >= n_cols). transpose = 1: column c becomes
 * row c of out (n_cols x ld_out, seg_len >= n_rows). */
int ebsd_split3_bf16(const float* X, int64_t n_rows, int n_cols, int64_t ld, const float* shift,
                     int transpose, int pattern, void* out, int64_t ld_out, int64_t seg_len,
                     void* stream);

/* ---- A14: disorientation angle (measurement) --------------------------------
 * Replaces disori_angle_laue (laue_fz_misori.py:148-203) for one Laue group:
 * out[i] = min over Laue operators of the rotation angle of q1[i] q2[i]^-1
 * (radians). */
int ebsd_disori_angle(const float* q1, const float* q2, int64_t n, int laue_id, float* out,
                      void* stream);

/* ---- orientation grid refinement (the step after DI) ------------------------
 * Replaces orientation_grid_refinement's per-batch loop (refining.py:71-244)
 * for one phase: for each pattern i, n_iter times, the n_grid (odd) local
 * cubochoric offsets grid_cu (get_local_orientation_grid, refining.py:13-68)
 * times the pattern's current scale become rotations cu2qu(.) composed with
 * the current orientation, moved to the FZ (fz_left 0: the reference's
 * ori_to_fz_laue, q g; 1: g q, which keeps the pattern), simulated with
 * grid_sample(align_corners=True) on the master pattern (mp_h x mp_w2, binned
 * already when binning), mean-subtracted and dotted with exp_rows[i] (zero-
 * mean FP32, row stride ld_e); the best becomes current and, when it is the
 * grid centre, the scale is multiplied by shrink. coords_soa (3 x n_pix): unit
 * rays, or un-normalised detector coordinates when offsets (n x 2, the scan
 * positions, average_pattern_center=False) is given. Writes q_out (n x 4,
 * may alias q_in) and dots (n x n_iter) = the best score of each iteration. */
int ebsd_refine_grid(const float* master_pattern, int mp_h, int mp_w2, const float* coords_soa, int n_pix,
                     const float* offsets, const float* exp_rows, int64_t ld_e, const float* q_in, int64_t n,
                     const float* grid_cu, int n_grid, int laue_id, int fz_left, int n_iter, float shrink,
                     float* q_out, float* dots, void* stream);

/* ---- experimental-pattern preprocessing --------------------------------------
 * FP32 patterns as n rows of n_pix pixels (row stride ld). */

/* mean[c] = mean over the n rows of column c (FP64 sums: partial holds
 * n_splits x n_pix doubles). With ebsd_subtract_pattern this replaces
 * ExperimentPatterns.subtract_overall_background (experiment_pats.py:223-232). */
int ebsd_pattern_mean(const float* patterns, int64_t n, int n_pix, int64_t ld, double* partial, int n_splits,
                      float* mean, void* stream);
/* patterns[r, c] -= v[c] in place. */
int ebsd_subtract_pattern(float* patterns, int64_t n, int n_pix, int64_t ld, const float* v, void* stream);
/* ExperimentPatterns.normalize_per_pattern (experiment_pats.py:255-285), in
 * place: mode 0 "minmax" (x - min) / (1e-4 + max - min), 1 "zeromean", 2
 * "standard" (zero mean, divided by the unbiased standard deviation). */
int ebsd_normalize_patterns(float* patterns, int64_t n, int n_pix, int64_t ld, int mode, void* stream);
/* clahe_grayscale (preprocessing/clahe.py:17-130) on n images of height x
 * width (row stride ld, written to out with stride ld_out; in place allowed
 * when ld == ld_out): clip_limit, n_bins and the grid_h x grid_w tile grid as
 * the reference takes them. Fused extras for standard_clean
 * (experiment_pats.py:287-297): subtract (n_pix, or NULL) is subtracted and
 * minmax_in applies the min-max normalisation before the equalisation,
 * minmax_out after it. grid_h * grid_w * n_bins * 8 bytes of tables must fit
 * in 220 KiB of shared memory; images that fit beside them are staged there
 * (one read, one write per pixel). */
int ebsd_clahe(const float* images, int64_t n, int height, int width, int64_t ld, const float* subtract,
               int minmax_in, float clip_limit, int n_bins, int grid_h, int grid_w, int minmax_out, float* out,
               int64_t ld_out, void* stream);
/* NLPAR window passes (nlpar.py:94-121 and 185-191) over a scan_h x scan_w
 * scan of patterns (row (y * scan_w + x), stride ld; zero outside the scan).
 * offsets (n_off_total x 2 int32, device) are the window offsets (di, dj),
 * |di|, |dj| <= k_rad <= 7, in the reference's order; one call covers offsets
 * o0 .. o0 + n_off - 1 (n_off <= 128). ebsd_nlpar_dists writes
 * dists[pt, o] = sum_p (x[pt + off_o, p] - x[pt, p])^2 (scan_h * scan_w x
 * n_off_total); ebsd_nlpar_average writes (accumulate 0) or adds
 * (accumulate 1) out[pt, p] = sum_o weights[pt, o] x[pt + off_o, p]. An
 * offset outside the window yields NaN; each offset may appear at most once
 * per call (the window's offsets, as the reference's window is). */
int ebsd_nlpar_dists(const float* data, int scan_h, int scan_w, int n_pix, int64_t ld, int k_rad,
                     const int* offsets, int o0, int n_off, int n_off_total, float* dists, void* stream);
int ebsd_nlpar_average(const float* data, int scan_h, int scan_w, int n_pix, int64_t ld, int k_rad,
                       const int* offsets, int o0, int n_off, int n_off_total, const float* weights, int accumulate,
                       float* out, int64_t ld_out, void* stream);
/* The NLPAR weights between the two passes (nlpar.py:122-183), in place over
 * dists (scan_h * scan_w x n_off, offsets as above, n_off >= 9): noise
 * estimate sigma = sqrt(min(dists[:, 1..8]) / (2 n_pix)), normalised
 * distances (dists - n_pix s2) / (sqrt(2 n_pix) s2) with s2 = sigma^2 +
 * sigma_neighbour^2 (1 outside the scan), clamped and negated; 10 Newton
 * iterations (stopping once |obj| < coeff_fit_tol) fitting the coefficient g
 * so that the mean softmax weight of offset 0 over offsets 0..8 equals coeff;
 * then softmax over the window of w / g^2 (+ center_logit_bias at offset 0 when
 * > 0; neighbours outside the scan get weight 0). workspace: device memory of
 * ebsd_nlpar_workspace_bytes(scan_h, scan_w) bytes, 16-byte aligned. Launches
 * 14 kernels; nothing synchronises with the host. */
size_t ebsd_nlpar_workspace_bytes(int scan_h, int scan_w);
int ebsd_nlpar_weights(float* dists, int scan_h, int scan_w, int n_pix, const int* offsets, int n_off, float coeff,
                       float coeff_fit_tol, float center_logit_bias, void* workspace, size_t workspace_bytes,
                       void* stream);

/* ---- pattern-centre fitting (spatial FFT search) -----------------------------
 * The kernels around the FFT cross-correlation of spatial_fft_pc_fitter
 * (fitting.py:359-540); the dictionary on the enlarged detector comes from
 * ebsd_project_dictionary (subtract_mean 0) and the FFTs from the caller.
 * ebsd_pcfit_prep: n binned patterns (height x width, contiguous) ->
 * (x - min) / max(x - min), minus the mean when zero_mean, written into
 * out (n x padded_h x padded_w, zero elsewhere) at (pad_top, pad_left)
 * (fitting.py:387-412). ebsd_pcfit_reduce: corr (n x n_patterns x padded_h x
 * padded_w) holds the circular cross-correlations of n dictionary entries;
 * for every (pattern, shift) the maximum over the n entries, read through
 * fftshift, updates best = max(best, max) and, where the maximum equals the
 * new best, best_index = index_base + its entry (fitting.py:498-507). */
int ebsd_pcfit_prep(const float* patterns, int n, int height, int width, int padded_h, int padded_w, int pad_top,
                    int pad_left, int zero_mean, float* out, void* stream);
int ebsd_pcfit_reduce(const float* corr, int n, int n_patterns, int padded_h, int padded_w, int64_t index_base,
                      float* best, int64_t* best_index, void* stream);

/* The cross-correlation itself without an FFT library (replaces
 * fitting.py:413 rfft2 and fitting.py:484-485 irfft2(sim_fft * pattern_fft)
 * plus the max over the batch, fitting.py:493-507), for enlarged detectors
 * of 2..127 rows and columns; larger ones return EBSD_ERR_ARG (and
 * ebsd_pcfit_xcorr_table_bytes returns 0).
 * Spectra hold 4 * (padded_h / 2 + 1) * (padded_w / 2 + 1) floats per image:
 * [trig][part][ky][kx] with Cc = sum_y T cos(2 pi ky y / H), Ss = sum_y T sin(.)
 * of the row transform T (S[ky] = Cc - i Ss, S[H - ky] = Cc + i Ss).
 * ebsd_pcfit_xcorr_tables: DFT matrices (hi / lo bf16 halves, in the
 *   shared-memory layout the kernels copy) into `tables` (16-byte aligned,
 *   ebsd_pcfit_xcorr_table_bytes bytes), once per detector size.
 * ebsd_pcfit_spectra: spectra of n images (rows of padded_h x padded_w
 *   floats, `ld` floats apart).
 * ebsd_pcfit_pattern_terms: the terms of the experimental patterns' conjugate
 *   spectra that the correlation uses, from their spectra (same layout).
 * ebsd_pcfit_xcorr_max: for every (pattern, shift), the maximum over the
 *   n_sims simulated patterns (their spectra) of the circular
 *   cross-correlation, read through fftshift, and its index (index_base +
 *   entry; the first maximum wins), merged into keys (n_patterns x padded_h
 *   x padded_w uint64, zero before a batch) by atomicMax. Tensor-core DFTs
 *   in a 3-term bf16 split (about 3e-5 of the maps' RMS). Bounded waits:
 *   EBSD_DEVICE_TIMEOUT in *status.
 * ebsd_pcfit_fold: folds a batch's keys into the running best of one pc_z
 *   (best = max(best, batch max); best_index replaced where they are equal)
 *   and clears the keys. */
int64_t ebsd_pcfit_xcorr_table_bytes(int padded_h, int padded_w);
int ebsd_pcfit_xcorr_tables(int padded_h, int padded_w, void* tables, int64_t bytes, void* stream);
int ebsd_pcfit_spectra(const float* images, int64_t ld, int64_t n, int padded_h, int padded_w, const void* tables,
                       float* spectra, int* status, void* stream);
int ebsd_pcfit_pattern_terms(const float* spectra, int64_t n, int padded_h, int padded_w, float* terms,
                             void* stream);
int ebsd_pcfit_xcorr_max(const float* sim_spectra, int64_t n_sims, const float* pattern_terms, int n_patterns,
                         int padded_h, int padded_w, const void* tables, unsigned long long* keys,
                         int64_t index_base, int* status, void* stream);
int ebsd_pcfit_fold(unsigned long long* keys, int64_t n, float* best, int64_t* best_index, void* stream);

/* ---- local dictionary search around orientation proposals --------------------
 * No counterpart in the reference (search step of the learned-proposal path).
 * cell_to_row (edge^3 int32): dictionary row of each cubochoric grid cell or
 * -1, built by ebsd_cell_to_row from the cells of ebsd_grid_fz_write and the
 * dictionary permutation (row j holds FZ point perm[j]; perm NULL = identity).
 * ebsd_local_search: per query, the dictionary orientations within
 * max_angle_rad of a symmetric copy of proposals[q] that lie in the grid cells
 * within radius_cells of that copy are scored by the exact FP32 dot of
 * q_f32[q] with d_f32[row]; the best row and score are written (ties: lower
 * row; -1 / -inf when no candidate), and the candidate count if out_ncand.
 * With d_lp (unit-norm bf16 / e4m3 rows as the projector writes them, row
 * stride ld_lp, zero padding) candidates are first ranked by
 * d_norm * d_lp_scale * (q . lp) and only the best n_rescore (<= 8) are
 * re-scored in FP32; n_rescore 0 returns the low-precision estimate of the
 * best candidate (for intermediate coarse-to-fine stages). */
int ebsd_cell_to_row(const int32_t* cells, const int64_t* perm, int64_t n, int64_t n_cells, int32_t* cell_to_row,
                     void* stream);
int ebsd_local_search(const float* q_f32, int64_t ld_q, int64_t n_queries, const float* proposals, int laue_id,
                      int edge_length, const int32_t* cell_to_row, const float* dict_quats, const float* d_f32,
                      int64_t ld_d, const void* d_lp, int lp_dtype, int64_t ld_lp, const float* d_norm,
                      const float* d_lp_scale, int n_rescore, int64_t n_dict, int n_pix, int radius_cells,
                      float max_angle_rad, int max_candidates, int64_t* out_idx, float* out_score,
                      int32_t* out_ncand, void* stream);

/* ---- A15: 6-D rotation representation and the learned proposal ------------
 * 6-D (Zhou et al.) -> quaternion (orientations.py:986-1005 zh2qu: Gram-Schmidt
 * rows b1, b2, b3 then om2qu), optional rotation matrices (n x 9). */
int ebsd_zh_to_qu(const float* zh, int64_t n, float* out_qu, float* out_om, void* stream);
/* quaternion -> 6-D, the first two matrix rows (orientations.py:1008-1020). */
int ebsd_qu_to_zh(const float* qu, int64_t n, float* out_zh, void* stream);
/* Training objective of the orientation-proposal network (no counterpart in
 * the reference): loss[i] = min over the Laue operators g of
 * ||zh2om(zh[i]) - om(g q_true[i])||_F^2 (crystal symmetry acts on the left)
 * and grad = grad_scale * dloss/dzh. */
int ebsd_rot6d_sym_loss(const float* zh, const float* q_true, int64_t n, int laue_id, float grad_scale,
                        float* out_loss, float* out_grad, void* stream);

/* CNN building blocks (3x3 / stride 2 / pad 1 convolutions on NHWC bf16
 * activations as im2col + tcgen05 GEMM; FP32 dense head; Adam).
 * im2col: cols (m_pad x ld bf16, ld % 8 == 0, 16-byte aligned) gets the
 * patches of x (B x H x W x C), zero rows/columns as padding. */
int ebsd_cnn_im2col(const void* x, int B, int H, int W, int C, int64_t m_pad, int ld, void* cols, void* stream);
/* First-layer (single input channel) convolution computed directly:
 * out16 / out32 ((B Ho Wo) x cout, 16-byte aligned; out32 may be null) =
 * act(conv(x, w16[:, :9]) + bias), cout in {16, 32, 64}, w16 row stride ldw. */
int ebsd_cnn_conv_c1(const void* x, int B, int H, int W, const void* w16, int ldw, const float* bias, int cout,
                     int relu, void* out16, float* out32, void* stream);
int ebsd_cnn_col2im(const float* dcols, int64_t ld, int B, int H, int W, int C, float* dx, void* stream);
/* Convolution forward as one tcgen05 GEMM with a fused epilogue:
 * out[r, c] = act(sum_k cols[r, k] w16[c, k] + bias[c]) for rows r < n_rows
 * and channels c < cout, stored bf16 (row stride ld_out) and, when out32 is
 * not null, FP32 with the same layout. w16 (cout_pad x k_pad, cout_pad % 128
 * == 0) and cols (rows_pad x k_pad, rows_pad % 256 == 0) are bf16, k_pad %
 * 64 == 0; act is ReLU when relu != 0. splits as for ebsd_gemm_nt. */
int ebsd_cnn_conv_fwd(const void* w16, int64_t cout_pad, const void* cols, int64_t rows_pad, int64_t k_pad,
                      const float* bias, int cout, int64_t n_rows, int relu, void* out16, int64_t ld_out,
                      float* out32, int splits, int* d_status, void* stream);
int ebsd_cnn_bias_act(const float* y, int64_t ldy, const float* bias, int64_t M, int C, int relu, void* out,
                      int64_t ld_out, float* out32, void* stream);
int ebsd_cnn_relu_grad(const float* dy, int64_t ldy, const void* act, int64_t lda, int64_t M, int C, float* g32,
                       void* g16, int64_t ld_out, void* stream);
int ebsd_cnn_col_sum(const float* g, int64_t M, int C, float* db, void* stream);
int ebsd_cnn_transpose(const void* in, int in_is_f32, int64_t rows, int64_t cols, int64_t ld_in, void* out,
                       int64_t out_rows, int64_t ld_out, void* stream);
int ebsd_cnn_scale_cast(const float* x, int64_t n, float scale, void* out, void* stream);
int ebsd_cnn_dense_fwd(const float* x, int64_t ldx, const float* w, const float* b, int M, int N, int K, int relu,
                       float* y, void* y16, void* stream);
int ebsd_cnn_dense_bwd(const float* dy, const float* x, int64_t ldx, const float* w, int M, int N, int K,
                       float* dw, float* db, float* dx, void* stream);
int ebsd_cnn_adam(float* w, float* m, float* v, const float* g, int64_t rows, int cols, float lr, float b1,
                  float b2, float eps, int step, float weight_decay, void* w16, int64_t ld16, void* w16t,
                  int64_t ld16t, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EBSD_B200_H */
