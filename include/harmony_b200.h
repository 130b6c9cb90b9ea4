/* harmony_b200.h -- C ABI of the B200 Harmony integration engine (sm_100a).
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*) and returns an int status.  On failure hb_last_error()
 * returns a message for the calling thread.  The library never allocates
 * device memory: callers pass a workspace of hb_plan_workspace_bytes() bytes,
 * mirroring the caller-allocated workspaces of the reference
 * (src/rapids_singlecell/preprocessing/_harmony/__init__.py:356-384,593-599,648-656).
 *
 * Reference interfaces replaced (paths inside the rapids_singlecell tree):
 *   hb_harmonize          -> harmonize() driving _harmony_clustering_cuda.clustering_loop and
 *                            _harmony_correction_batched_cuda.correction_batched
 *                            (preprocessing/_harmony/__init__.py:41-289;
 *                             _cuda/harmony/clustering/clustering.cu:397-469;
 *                             _cuda/harmony/correction/correction_batched.cu:134-164)
 *   hb_l2_normalize       -> _harmony_normalize_cuda.l2_row_normalize
 *                            (_cuda/harmony/normalize/kernels_normalize.cuh:7-54)
 *   hb_block_lists        -> pcg_hash_kernel + iota + cub::DeviceRadixSort::SortPairs
 *                            (_cuda/harmony/clustering/clustering.cu:292-305)
 *   hb_penalty            -> _harmony_pen_cuda.penalty (_cuda/harmony/pen/kernels_pen.cuh:8-21)
 *   hb_ridge_inverse      -> _harmony_correction_cuda.compute_inv_mat
 *                            (_cuda/harmony/correction/kernels_correction_fast.cuh:24-123)
 *   hb_lambda_kb          -> _compute_lambda_kb (preprocessing/_harmony/__init__.py:454-480)
 *   hb_kmeans_init        -> the cuML KMeans fit in _initialize_centroids (__init__.py:290-323)
 *   hb_similarity         -> the similarity GEMM of clustering_loop_impl
 *                            (_cuda/harmony/clustering/clustering.cu:284-289)
 */
#ifndef HARMONY_B200_H
#define HARMONY_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HB_API __attribute__((visibility("default")))
#else
#define HB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define HB_OK 0
#define HB_ERR_INVALID 1      /* bad argument (shape, parameter range)            */
#define HB_ERR_WORKSPACE 2    /* workspace smaller than hb_plan_workspace_bytes()  */
#define HB_ERR_TIMEOUT 3      /* a bounded device-side wait gave up               */
#define HB_ERR_CUDA 4         /* CUDA runtime error                                */
#define HB_ERR_INTERNAL 5     /* device-side consistency check failed             */
#define HB_ERR_UNSUPPORTED 6  /* size outside the engine's supported range        */

/* arithmetic of the soft k-means (storage of Z_norm and R) */
#define HB_FP32 0  /* plain float32, the drop-in for harmony_integrate(dtype=np.float32) */
#define HB_FP64 1  /* plain float64, the drop-in for the reference default dtype         */
#define HB_BF16 2  /* bf16 Z_norm / R, tensor-core similarity + centroids, fp32 accumulate */
#define HB_FP16 3  /* fp16 Z_norm / R, tensor-core similarity + centroids, fp32 accumulate */

typedef struct hb_params {
  int64_t n_cells;
  int32_t n_pcs;
  int32_t n_clusters;
  int32_t n_batches;
  int32_t precision;            /* HB_FP32 ... HB_FP16 */
  int64_t block_size;           /* int(n_cells * block_proportion), >= 1 */
  int32_t max_iter_harmony;
  int32_t max_iter_clustering;
  double tol_harmony;
  double tol_clustering;
  double sigma;
  double ridge_lambda;
  double alpha;
  double batch_prune_threshold; /* used when prune != 0 */
  int32_t prune;                /* batch_prune_threshold is not None */
  int32_t stabilized_penalty;   /* harmony2 penalty */
  int32_t dynamic_lambda;       /* harmony2 lambda = alpha * E */
  int32_t max_sweep_ctas;       /* 0: the persistent sweep may use every SM; otherwise at most this
                                   many CTAs (SMs).  Problems that run at the same time on one GPU
                                   must together stay within the SM count, or their grid barriers
                                   can wait on each other */
  uint64_t random_state;
  int64_t sweep_wait_ns;        /* bound of each grid-barrier wait of the persistent sweep (16-bit path):
                                   after this long the wait gives up and the run returns HB_ERR_TIMEOUT;
                                   0 means 2 s */
  int32_t test_unmet_arrivals;  /* test hook, 0 in normal use: the sweep's grid barrier waits for this many
                                   arrivals more than its CTAs make, so every wait runs out (bounded by
                                   sweep_wait_ns) and the run must return HB_ERR_TIMEOUT */
  int32_t sweep_form;           /* layout of the persistent sweep (16-bit path): 0 the engine's choice;
                                   HB_SWEEP_2x2_2BUF ... HB_SWEEP_1x4_1BUF force one (HB_ERR_UNSUPPORTED
                                   at the run when it does not fit the shared memory); set by the
                                   autotuner (rapids_singlecell_b200.autotune) */
} hb_params;

/* Layouts of the persistent sweep: thread groups x threads per row, A tiles per group */
#define HB_SWEEP_AUTO 0
#define HB_SWEEP_2x2_2BUF 1  /* two 256-thread tile streams, two threads per row, two A tiles each */
#define HB_SWEEP_2x2_1BUF 2
#define HB_SWEEP_1x4_2BUF 3  /* one 512-thread tile stream, four threads per row */
#define HB_SWEEP_1x4_1BUF 4

typedef struct hb_plan hb_plan;

/* Optional device-time profile of one run (CUDA events around the timed launches). */
typedef struct hb_profile {
  int64_t kernel_launches;    /* kernels launched by the run */
  int64_t block_launches;     /* fused block-update launches */
  double block_ms;            /* summed device time of those launches */
  double block_bytes;         /* algorithmic HBM bytes they move (unpadded rows) */
  int64_t centroid_launches;  /* centroid-sum launch pairs (partials + reduce) */
  double centroid_ms;
  double centroid_bytes;
} hb_profile;

/* Outputs of one run (host memory owned by the caller). */
typedef struct hb_outputs {
  double* objectives;         /* [1 + max_iter_harmony]: initial + one per outer iteration */
  int32_t* n_objectives;
  double* kmeans_objectives;  /* optional [max_iter_harmony * max_iter_clustering] */
  int32_t* kmeans_iters;      /* optional [max_iter_harmony]: k-means iterations run per outer */
  int32_t* converged;         /* 1 if the outer loop met tol_harmony */
  hb_profile* profile;        /* optional: filled when not NULL */
} hb_outputs;

/* Validates the parameters and builds a plan (no device memory).  HB_ERR_UNSUPPORTED for shapes
 * the engine does not run: n_clusters > 256, n_pcs > 256 (> 128 on the 16-bit paths), and on the
 * 16-bit paths a (n_pcs, n_clusters, n_batches) whose sweep tables and tiles do not fit one CTA's
 * shared memory (asked of the sweep's layouts when a device is present, else at the launch). */
HB_API int hb_plan_create(const hb_params* params, hb_plan** plan);
HB_API void hb_plan_destroy(hb_plan* plan);
HB_API size_t hb_plan_workspace_bytes(const hb_plan* plan);

/* Full Harmony integration of one problem.
 *   X             device [n_cells, n_pcs] row-major; float64 for HB_FP64, else float32
 *   cats          device int32 [n_cells] batch code per cell (0 .. n_batches-1)
 *   cell_index    device int32 [n_cells] cells sorted by batch (stable), or NULL: the
 *                 engine then builds it in the workspace (needs n_batches <= 4096)
 *   batch_offsets host int64 [n_batches + 1] CSR offsets into cell_index
 *   theta         host float64 [n_batches] (tau discount already applied)
 *   Y0            device [n_clusters, n_pcs] initial centroids, same dtype as X
 *   Z_hat         device [n_cells, n_pcs] output, same dtype as X
 * Limits: n_pcs <= 256 (<= 128 on the 16-bit path), n_clusters <= 256.
 * The call enqueues the loop on `stream` without reading results back: the k-means stop, the
 * outer convergence test and the error flags are evaluated on the device, and the launches after
 * the point where the loop ends return at once.  The host stays at most two outer iterations
 * ahead of the device (it sleeps on the end event of iteration o - 2 before enqueuing iteration
 * o, while iteration o - 1 is still queued, so the device never waits for the host), stops
 * enqueuing once an ended run shows in those events, and synchronises the stream once, at the
 * end, to read the objectives and the status.
 */
HB_API int hb_harmonize(hb_plan* plan, const void* X, const int32_t* cats, const int32_t* cell_index,
                 const int64_t* batch_offsets, const double* theta, const void* Y0,
                 void* workspace, size_t workspace_bytes, void* Z_hat, hb_outputs* out,
                 void* stream);

/* ---- kernel-level entry points (the reference's per-kernel bindings) ---- */

/* dst[r, :cols] = src[r, :cols] * min(rsqrt(sum src^2), 1e12); dtype HB_FP32 / HB_FP64 */
HB_API int hb_l2_normalize(const void* src, void* dst, int64_t rows, int32_t cols, int32_t dtype,
                    void* stream);

/* Cell lists of every block of `n_iters` k-means iterations (seeds given on the host):
 * idx[c*n + j*block_size + r] is the r-th cell of block j for seed c.  Block j holds the
 * cells whose shuffle keys rank in [j*block_size, (j+1)*block_size); inside a block cells
 * are ordered by (cats[i], i), or by i when cats is NULL. */
HB_API size_t hb_block_lists_workspace_bytes(int64_t n, int64_t block_size, int32_t n_batches);
HB_API int hb_block_lists(int64_t n, int64_t block_size, const uint32_t* seeds, int32_t n_iters,
                   const int32_t* cats, int32_t n_batches, int32_t* idx, void* workspace,
                   size_t workspace_bytes, void* stream);

/* hb_block_lists without a workspace: the scratch is a fixed device array of the library,
 * HB_BLOCK_LISTS_STATIC_MAX_BYTES per device, and the call allocates nothing.  No counterpart in
 * the reference (its clustering loop allocates its workspace with CuPy).  For callers that cannot
 * allocate device memory at the call: a serving loop that must not call cudaMalloc (it
 * synchronises the device and can fail under memory pressure), or a C host with no allocator.
 * Returns HB_ERR_WORKSPACE when hb_block_lists_workspace_bytes() exceeds the limit.  The first
 * call on a device looks up the array (cudaGetSymbolAddress) and should come before any stream
 * capture; the looked-up address is kept for the life of the process, so the entry point must not
 * be called again on a device after cudaDeviceReset().  Calls that overlap in time race on the
 * array; it keeps the last call's contents.  n_iters == 0 returns HB_OK without device work. */
#define HB_BLOCK_LISTS_STATIC_MAX_BYTES ((size_t)16 << 20)
HB_API int hb_block_lists_static(int64_t n, int64_t block_size, const uint32_t* seeds, int32_t n_iters,
                                 const int32_t* cats, int32_t n_batches, int32_t* idx, void* stream);

/* penalty[b,k] = ((E+1)/(O[+E]+1)) ** theta[b]; float64 arrays [B,K], theta [B] */
HB_API int hb_penalty(const double* E, const double* O, const double* theta, double* penalty,
               int32_t n_batches, int32_t n_clusters, int32_t stabilized, void* stream);

/* lambda[b,k] per _compute_lambda_kb; float64 [B,K], N_b [B] */
HB_API int hb_lambda_kb(const double* E, const double* O, const double* N_b, double* lambda_kb,
                 int32_t n_batches, int32_t n_clusters, double alpha, double threshold,
                 int32_t prune, double ridge_lambda, int32_t dynamic_lambda, void* stream);

/* inv[k] = closed-form inverse of [[N_k, O_k^T],[O_k, diag(O_k + lambda_k)]], float64,
 * inv is [n_clusters, n_batches+1, n_batches+1] */
HB_API int hb_ridge_inverse(const double* O, const double* lambda_kb, double* inv, int32_t n_batches,
                     int32_t n_clusters, void* stream);

/* Similarity rows on the tensor core: S[q, k] = Zn[idx[q], :] . Yn[k, :] for q < n, k < n_clusters.
 * Zn [*, ldz] and Yn [n_clusters, ldy] are 16-bit (dtype HB_FP16 / HB_BF16), zero-padded past
 * n_pcs (<= 128); ldz, ldy multiples of 8.  S is float32 [n, n_clusters].  *err (device int32)
 * is set non-zero if a bounded tensor-core wait gave up.  Replaces the similarity GEMM of
 * the reference (_cuda/harmony/clustering/clustering.cu:284-289). */
HB_API int hb_similarity(const void* Zn, int32_t ldz, const void* Yn, int32_t ldy, const int32_t* idx,
                  int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t dtype, float* S,
                  int32_t* err, void* stream);

/* ---- kernel-level entry points of the 16-bit path (the launchers hb_harmonize drives, run alone).
 * 16-bit arrays (dtype HB_BF16 / HB_FP16) of cells have rows = 128 ceil(n / 128) + 8 rows, the
 * rows past n zero (the tiles of 128 cells are read whole); row strides are multiples of 8. ---- */

/* Centroid pass in cell order (TMA tiles, tcgen05): Yn[k] = l2normalise(sum_i R[i][k] Zn[i]) (16-bit
 * [n_clusters][ldy], zero past n_pcs; inverse norm capped at 1e12) and Osum[key][k] = sum over the
 * cells i with ckey[i] == key of R[i][k] (float64 [n_keys][n_clusters]), ckey int32 [n] in
 * [0, n_keys).  With the key (block, batch) the second output is the per-block "remove old"
 * sums of the sweep.  Replaces the centroid GEMM and normalisation (clustering.cu:272-281) and the
 * per-block R column sums (clustering.cu:321-332).  n_pcs <= 128, n_clusters <= 256, n_keys <= 256
 * within the kernel's shared memory (HB_ERR_UNSUPPORTED otherwise).  *err (device int32, cleared
 * by the call) is set non-zero if a bounded wait gave up. */
HB_API size_t hb_tc_centroids_workspace_bytes(int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t n_keys);
HB_API int hb_tc_centroids(const void* Zn, int32_t ldz, const void* R, int32_t ldr, int64_t n, int32_t n_pcs,
                           int32_t n_clusters, const int32_t* ckey, int32_t n_keys, int32_t dtype, void* Yn,
                           int32_t ldy, double* Osum, void* workspace, size_t workspace_bytes, int32_t* err,
                           void* stream);

/* Ridge moments on the tensor core: M[k][b+1][c] = sum over the cells i of batch b of R[i][k] X[i][c]
 * and M[k][0][c] = the sum over all batches (float64 [n_clusters][n_batches+1][n_pcs]).  X float32
 * [n][n_pcs] enters as bf16 hi + lo parts; cell_index int32 [n] lists the cells sorted by batch and
 * batch_offsets (host int64 [n_batches+1]) are its offsets.  Replaces the moment GEMMs of
 * correction_batched_impl (correction_batched.cu:55-100).  n_pcs <= 256, n_clusters <= 256. */
HB_API size_t hb_tc_moments_workspace_bytes(int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t n_batches);
HB_API int hb_tc_moments(const float* X, const void* R, int32_t ldr, const int32_t* cell_index,
                         const int64_t* batch_offsets, int64_t n, int32_t n_pcs, int32_t n_clusters,
                         int32_t n_batches, int32_t dtype, double* M, void* workspace, size_t workspace_bytes,
                         int32_t* err, void* stream);

/* Correction apply on the tensor core: Z_hat[i] = X[i] - sum_k R[i][k] W[b_i][k] (float32 [n][n_pcs])
 * and Zn[i] = l2normalise(Z_hat[i]) (16-bit [rows][ldz], zero past n_pcs), W float32
 * [n_batches][n_clusters][n_pcs], b_i the batch of cell i (from cell_index and batch_offsets as for
 * hb_tc_moments).  X and W enter as bf16 hi + lo parts.  Replaces the apply of
 * correction_batched_impl (kernels_outer.cuh:41-65) fused with the renormalisation of
 * _harmony/__init__.py:276.  *err = 7 flags |X| or |W| outside the fp16 range (HB_FP16).
 * n_pcs <= 128, n_clusters <= 256. */
HB_API size_t hb_tc_apply_workspace_bytes(int64_t n, int32_t n_batches);
HB_API int hb_tc_apply(const float* X, const void* R, int32_t ldr, const float* W, const int32_t* cell_index,
                       const int64_t* batch_offsets, int64_t n, int32_t n_pcs, int32_t n_clusters,
                       int32_t n_batches, int32_t dtype, float* Z_hat, void* Zn, int32_t ldz, void* workspace,
                       size_t workspace_bytes, int32_t* err, void* stream);

/* Initial centroids by a seeded k-means on the L2-normalised rows of X (float32 [n, n_pcs],
 * row-major): k-means++ seeding over a sample of min(n, 64 n_clusters, 16384) cells drawn
 * from `seed`, then up to max_iter Lloyd iterations over all cells with tensor-core (bf16)
 * assignment, stopping when |Y_new - Y_old|_F <= tol |Y_new|_F.  Y_out (float32
 * [n_clusters, n_pcs], device) receives the centres (not normalised); *n_iter_out the Lloyd
 * iterations run.  n_pcs <= 128 with n_clusters <= 256, or n_pcs <= 256 with n_clusters <= 128;
 * n_clusters <= n.  Synchronises the stream once
 * per iteration.  Replaces the cuML KMeans(init="k-means||", max_iter=25) fit of the
 * reference's _initialize_centroids (preprocessing/_harmony/__init__.py:290-323); cuML's
 * random streams are not reproduced. */
HB_API size_t hb_kmeans_workspace_bytes(int64_t n, int32_t n_pcs, int32_t n_clusters);
HB_API int hb_kmeans_init(const float* X, int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t max_iter,
                          double tol, uint64_t seed, float* Y_out, int32_t* n_iter_out, void* workspace,
                          size_t workspace_bytes, void* stream);

/* ---- PCA by the covariance eigendecomposition (preprocessing/_pca.py:339-353 ->
 * preprocessing/_sparse_pca/_sparse_pca.py:26-127): Gram matrix and column sums on the tensor
 * core, covariance, and the projection onto the leading components.  The eigendecomposition of
 * the n_genes x n_genes covariance is left to the caller (the reference calls cp.linalg.eigh,
 * _sparse_pca.py:47). ---- */

/* gram[i][j] = sum_r X[r][i] X[r][j] (float64 [n_genes][n_genes], both triangles) and
 * col_sums[i] = sum_r X[r][i] (float64 [n_genes]) of a dense float32 X [n][ldx] (device).  Each
 * float32 value enters the bf16 tensor-core products as hi + lo parts (about 16 significant
 * bits), accumulated in float32 per 128-row tile run and summed in float64.  Replaces the Gram
 * build of _create_gram_matrix (_sparse_pca.py:202-248; gram_csr_upper_kernel,
 * _cuda/spca/kernels_spca.cuh:5-28) and the column means of _get_mean_var
 * (preprocessing/_utils.py:88-105).  n_genes <= 32768.  Synchronises the stream once. */
HB_API size_t hb_pca_gram_workspace_bytes(int64_t n, int32_t n_genes);
HB_API int hb_pca_gram(const float* X, int64_t n, int32_t n_genes, int64_t ldx, double* gram, double* col_sums,
                       void* workspace, size_t workspace_bytes, void* stream);

/* cov = gram / n - mean mean^T with mean = col_sums / n (zero_center != 0), or cov = gram
 * (zero_center == 0, the reference's uncentred path); float64 [n_genes][n_genes]; mean
 * (optional, float64 [n_genes]) receives the column means.  Replaces _compute_cov and
 * cov_from_gram_kernel (_sparse_pca/_helper.py:21-32; _cuda/spca/kernels_spca.cuh:48-62). */
HB_API int hb_pca_covariance(const double* gram, const double* col_sums, int64_t n, int32_t n_genes,
                             int32_t zero_center, double* cov, double* mean, void* stream);

/* X_pca[r][c] = sum_g X[r][g] components[c][g] - (mean ? sum_g mean[g] components[c][g] : 0),
 * float32 [n][n_comps]; components float32 [n_comps][n_genes] (device), mean float64 [n_genes]
 * or NULL.  X and the components enter the bf16 tensor-core products as hi + lo parts.
 * n_comps <= 256.  Replaces PCA_sparse._transform_cupy (_sparse_pca.py:84-95).  Synchronises the
 * stream once. */
HB_API size_t hb_pca_project_workspace_bytes(int32_t n_genes, int32_t n_comps);
HB_API int hb_pca_project(const float* X, int64_t n, int32_t n_genes, int64_t ldx, const float* components,
                          int32_t n_comps, const double* mean, float* X_pca, void* workspace,
                          size_t workspace_bytes, void* stream);

/* Dense float32 copy out[r][c] (row stride ldo, zero where no entry is stored) of a CSR matrix
 * (indptr int64 [n_rows + 1], indices int32, data float32; device).  *err (device int32, set
 * to zero by the call) flags a column index outside [0, n_cols) -> HB_ERR_INVALID.  The sparse
 * input of the reference's covariance PCA (csr_matrix, _sparse_pca.py:202-214) enters the
 * dense Gram and projection kernels through this copy. */
HB_API int hb_csr_to_dense(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n_rows,
                           int32_t n_cols, float* out, int64_t ldo, int32_t* err, void* stream);

/* ---- exact k nearest neighbours (the brute-force search of pp.neighbors,
 * preprocessing/_neighbors/_algorithms/_brute.py:14-37, a cuML NearestNeighbors(algorithm="brute")
 * call in the reference) ---- */
#define HB_KNN_SQEUCLIDEAN 0
#define HB_KNN_EUCLIDEAN 1     /* also "l2" */
#define HB_KNN_COSINE 2        /* 1 - cosine similarity */
#define HB_KNN_INNER_PRODUCT 3 /* similarity, largest first */

/* For each of n_queries float32 rows (device, [n_queries][n_dims]) the k nearest of n_data rows
 * (device, [n_data][n_dims]); indices int64 [n_queries][k] and distances float32 [n_queries][k]
 * (device), ascending by distance then index.  Dot products run on the tensor core as bf16 hi + lo
 * parts; each query's best candidates are re-ranked with exact float32 distances (difference form
 * for the euclidean metrics).  Pass the same pointer and count for queries and data for a kNN
 * graph (the call of pp.neighbors, _neighbors/__init__.py:223-230).  n_dims <= 128, k <= 56
 * (k <= 24 above 64 dims).  Synchronises the stream once. */
HB_API size_t hb_knn_workspace_bytes(int64_t n_queries, int64_t n_data, int32_t n_dims, int32_t same,
                                     int32_t metric);
HB_API int hb_knn(const float* queries, int64_t n_queries, const float* data, int64_t n_data, int32_t n_dims,
                  int32_t k, int32_t metric, int64_t* indices, float* distances, void* workspace,
                  size_t workspace_bytes, void* stream);

HB_API const char* hb_last_error(void);
HB_API const char* hb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HARMONY_B200_H */
