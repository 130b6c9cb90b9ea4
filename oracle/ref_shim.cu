// TEST INFRASTRUCTURE ONLY -- the reference's own Harmony kernels behind a C ABI.
//
// This file is compiled by oracle/Makefile together with rapids_singlecell's
// kernel headers, read in place from the reference source tree
// (src/rapids_singlecell/_cuda/harmony/*/kernels_*.cuh, _cuda/spca/kernels_spca.cuh,
// _cuda/mean_var/kernels_mv.cuh and _cuda/cublas_helpers.cuh), into
// oracle/_ref/libharmony_ref.so.
// The reference's nanobind modules (*.cu) cannot be built here (nanobind is not
// installed), so this shim replays their launch sequences -- grid and block
// shapes, GEMM calls and kernel order -- around the unmodified kernels.  The
// tests use it to pin the NumPy oracle and to check the engine against the
// reference itself on a GPU.  Nothing under rapids_singlecell_b200/ links or
// loads this library; the product path never reaches it.
//
// Launch sequences restated (paths inside the rapids_singlecell tree):
//   ref_clustering_loop     _cuda/harmony/clustering/clustering.cu:241-393
//   ref_compute_objective   _cuda/harmony/clustering/clustering.cu:188-237
//   ref_correction_batched  _cuda/harmony/correction/correction_batched.cu:17-130
//   ref_l2_row_normalize    _cuda/harmony/normalize/normalize.cu:23-31
//   ref_l1_normalize        _cuda/harmony/normalize/normalize.cu:11-20
//   ref_scatter_add         preprocessing/_harmony/_helper.py:63-145 with
//                           _cuda/harmony/scatter/scatter.cu:14-53
//   ref_colsum              preprocessing/_harmony/_helper.py:310-361 with
//                           _cuda/harmony/colsum/colsum.cu:14-55
//   ref_outer               _cuda/harmony/outer/outer.cu:10-19
//   ref_pca_cov_csr         preprocessing/_sparse_pca/_sparse_pca.py:138-199 (_cov_sparse) with
//                           _cuda/spca/spca.cu:12-44, _cuda/mean_var/mean_var.cu:24-31 and
//                           preprocessing/_utils.py:88-105 (the column means)
//
// Every entry point returns 0 on success or a CUDA / cuBLAS error code (negated
// for cuBLAS); ref_last_error() gives the message.
#include <cub/device/device_radix_sort.cuh>
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "cublas_helpers.cuh"
#include "harmony/clustering/kernels_clustering.cuh"
#include "harmony/colsum/kernels_colsum.cuh"
#include "harmony/correction/kernels_correction_fast.cuh"
#include "harmony/kmeans/kernels_kmeans.cuh"
#include "harmony/normalize/kernels_normalize.cuh"
#include "harmony/outer/kernels_outer.cuh"
#include "harmony/pen/kernels_pen.cuh"
#include "harmony/scatter/kernels_scatter.cuh"
#include "mean_var/kernels_mv.cuh"
#include "spca/kernels_spca.cuh"

namespace {

thread_local std::string g_err;

struct Fail : std::runtime_error {
  int code;
  Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Fail((int)e, std::string(what) + ": " + cudaGetErrorString(e));
}
void launched(const char* what) { cuda_ok(cudaGetLastError(), what); }
void blas_ok(cublasStatus_t s, const char* what) {
  if (s != CUBLAS_STATUS_SUCCESS) throw Fail(-(int)s, std::string(what) + ": cuBLAS status " + std::to_string((int)s));
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const Fail& e) {
    g_err = e.what();
    return e.code == 0 ? 1 : e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

int n_sm() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 1;
}

// One cuBLAS handle per thread (the reference takes CuPy's per-device handle).
cublasHandle_t handle() {
  thread_local cublasHandle_t h = nullptr;
  if (!h) blas_ok(cublasCreate(&h), "cublasCreate");
  return h;
}

// Device scratch that lives for one call.
struct Scratch {
  std::vector<void*> ptrs;
  template <typename T>
  T* get(size_t count) {
    void* p = nullptr;
    cuda_ok(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
    ptrs.push_back(p);
    return (T*)p;
  }
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
};

// strided_grid of the reference's nb_types.h: one block per block_size items, capped by gridDim.x.
unsigned strided_grid(long long nwork, int block_size) {
  long long ideal = (nwork + block_size - 1) / block_size;
  long long capped = std::min<long long>(ideal, INT_MAX);
  return (unsigned)(capped < 1 ? 1 : capped);
}

constexpr unsigned kWarp = 32;
constexpr unsigned kMaxBlockDim = 256;
constexpr int kBlock1D = 256;
constexpr int kMaxBlock1D = 1024;
constexpr int kBlocksPerSm = 8;
constexpr int kScatterSharedBlocksPerSm = 4;
constexpr int kScatterSharedCellsPerBlock = 64;

// clustering.cu:33-45
int grid_1d(long long n, int sms) {
  long long blocks = (n + kBlock1D - 1) / kBlock1D;
  return std::max(1, std::min(sms * kBlocksPerSm, (int)std::min<long long>(blocks, INT_MAX)));
}
unsigned warp_aligned_bdim(unsigned n) { return std::min(kMaxBlockDim, std::max(kWarp, (n + kWarp - 1u) / kWarp * kWarp)); }

// clustering.cu:63-107 (0 = columns, 1 = atomics, 2 = gemm)
template <typename T>
void colsum_dispatch(int algo, const T* A, T* out, const T* ones, int rows, int cols, int sms, cudaStream_t st) {
  T one = T(1), zero = T(0);
  switch (algo) {
    case 0: {
      int threads = std::min(kMaxBlock1D, std::max((int)kWarp, (rows + (int)kWarp - 1) / (int)kWarp * (int)kWarp));
      colsum_kernel<T><<<std::min(cols, sms * kBlocksPerSm), threads, 0, st>>>(A, out, rows, cols);
      launched("colsum_kernel");
      break;
    }
    case 1: {
      cuda_ok(cudaMemsetAsync(out, 0, cols * sizeof(T), st), "memset");
      int col_tiles = (cols + (int)kWarp - 1) / (int)kWarp;
      int target_row_tiles = std::max(1, sms * kScatterSharedBlocksPerSm / std::max(1, col_tiles));
      int rows_per_tile = std::max((int)kWarp, (rows + target_row_tiles - 1) / target_row_tiles);
      int row_tiles = (rows + rows_per_tile - 1) / rows_per_tile;
      colsum_atomic_kernel<T><<<dim3(col_tiles, row_tiles), dim3(kWarp, kWarp), 0, st>>>(A, out, rows, cols,
                                                                                        rows_per_tile);
      launched("colsum_atomic_kernel");
      break;
    }
    default:
      blas_ok(cublas_gemv<T>(handle(), CUBLAS_OP_N, cols, rows, &one, A, cols, ones, 1, &zero, out, 1),
              "cublas_gemv(colsum)");
      break;
  }
}

// clustering.cu:111-135
template <typename T>
void scatter_add_to_O(const T* R_buf, const int* cats_in, int bs, int K, int B, int switcher, T* O,
                      bool use_shared, size_t shared_bytes, int sms, cudaStream_t st) {
  if (use_shared) {
    int max_blocks = std::max(1, (bs + kScatterSharedCellsPerBlock - 1) / kScatterSharedCellsPerBlock);
    int blocks = std::min(sms * kScatterSharedBlocksPerSm, max_blocks);
    scatter_add_shared_kernel<T><<<blocks, kBlock1D, shared_bytes, st>>>(R_buf, cats_in, bs, K, B, switcher, O);
    launched("scatter_add_shared_kernel");
  } else {
    size_t N = (size_t)bs * K;
    scatter_add_kernel<T><<<grid_1d((long long)N, sms), kBlock1D, 0, st>>>(R_buf, cats_in, (size_t)bs, (size_t)K,
                                                                          (size_t)switcher, O);
    launched("scatter_add_kernel");
  }
}

// compute_objective_impl (clustering.cu:188-237)
template <typename T>
T objective(const T* R, const T* S, const T* O, const T* E, const T* theta, T sigma, T* obj_scalar, int n, int K,
            int B, bool stabilized, cudaStream_t st) {
  const int sms = n_sm();
  cuda_ok(cudaMemsetAsync(obj_scalar, 0, sizeof(T), st), "memset");
  {
    size_t N = (size_t)n * K;
    kmeans_err_kernel<T><<<grid_1d((long long)N, sms), kBlock1D, 0, st>>>(R, S, N, obj_scalar);
    launched("kmeans_err_kernel");
  }
  entropy_kernel<T><<<n, warp_aligned_bdim(K), 0, st>>>(R, sigma, n, K, obj_scalar);
  launched("entropy_kernel");
  {
    int ob_total = B * K;
    int threads = (int)warp_aligned_bdim(ob_total);
    int blocks = std::max(1, std::min(sms, (ob_total + threads - 1) / threads));
    if (stabilized)
      diversity_kernel<T, true><<<blocks, threads, 0, st>>>(O, E, theta, sigma, B, K, obj_scalar);
    else
      diversity_kernel<T, false><<<blocks, threads, 0, st>>>(O, E, theta, sigma, B, K, obj_scalar);
    launched("diversity_kernel");
  }
  T host_obj;
  cuda_ok(cudaMemcpyAsync(&host_obj, obj_scalar, sizeof(T), cudaMemcpyDeviceToHost, st), "D2H");
  cuda_ok(cudaStreamSynchronize(st), "sync");
  return host_obj;
}

// clustering_loop_impl (clustering.cu:241-393).  The workspace that the
// reference's Python side allocates (__init__.py:356-384) is allocated here.
// objectives: host [max_iter]; *n_iter: iterations run.
template <typename T>
void clustering_loop(const T* Z_norm, T* R, T* E, T* O, const T* Pr_b, const int* cats, const T* theta, int n,
                     int d, int K, int B, int block_size, int colsum_algo, double sigma_d, double tol_d, int max_iter,
                     unsigned seed, bool stabilized, T* objectives_out, int* n_iter, cudaStream_t st) {
  Scratch ws;
  T* Y = ws.get<T>((size_t)K * d);
  T* Y_norm = ws.get<T>((size_t)K * d);
  T* sim = ws.get<T>((size_t)n * K);
  int* idx_list = ws.get<int>(n);
  int* idx_alt = ws.get<int>(n);
  unsigned* keys = ws.get<unsigned>(n);
  unsigned* keys_alt = ws.get<unsigned>(n);
  size_t cub_bytes = 0;
  cuda_ok(cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, keys, keys_alt, idx_list, idx_alt, n, 0, 32),
          "cub temp query");
  uint8_t* cub_temp = ws.get<uint8_t>(cub_bytes);
  T* R_out = ws.get<T>((size_t)std::max(block_size, 1) * K);
  int* cats_in = ws.get<int>(std::max(block_size, 1));
  T* R_in_sum = ws.get<T>(K);
  T* R_out_sum = ws.get<T>(K);
  T* pen = ws.get<T>((size_t)B * K);
  T* obj_scalar = ws.get<T>(1);
  T* ones = ws.get<T>(std::max(block_size, 1));
  {
    std::vector<T> h(std::max(block_size, 1), T(1));
    cuda_ok(cudaMemcpyAsync(ones, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st), "H2D");
    cuda_ok(cudaStreamSynchronize(st), "sync");
  }
  const T sigma = (T)sigma_d, tol = (T)tol_d;
  cublasHandle_t h = handle();
  blas_ok(cublasSetStream(h, st), "cublasSetStream");
  T term = T(-2) / sigma;
  T one = T(1), zero = T(0);
  int ob_total = B * K;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cuda_ok(cudaGetDeviceProperties(&prop, dev), "props");
  const int sms = prop.multiProcessorCount;
  size_t shared_bytes = (size_t)B * K * sizeof(T);
  bool use_shared = shared_bytes <= (size_t)prop.sharedMemPerBlock;
  std::vector<T> objs;
  constexpr int kWindow = 3;
  for (int iter = 0; iter < max_iter; iter++) {
    blas_ok(cublas_gemm<T>(h, CUBLAS_OP_N, CUBLAS_OP_T, d, K, n, &one, Z_norm, d, R, K, &zero, Y, d),
            "cublas_gemm(centroids)");
    l2_row_normalize_kernel<T><<<K, warp_aligned_bdim(d), 0, st>>>(Y, Y_norm, K, d);
    launched("l2_row_normalize_kernel");
    blas_ok(cublas_gemm<T>(h, CUBLAS_OP_T, CUBLAS_OP_N, K, n, d, &one, Y_norm, d, Z_norm, d, &zero, sim, K),
            "cublas_gemm(similarities)");
    pcg_hash_kernel<<<grid_1d(n, sms), kBlock1D, 0, st>>>(keys, n, seed + iter);
    launched("pcg_hash_kernel");
    iota_kernel<<<grid_1d(n, sms), kBlock1D, 0, st>>>(idx_list, n);
    launched("iota_kernel");
    cuda_ok(cub::DeviceRadixSort::SortPairs(cub_temp, cub_bytes, keys, keys_alt, idx_list, idx_alt, n, 0, 32, st),
            "cub radix sort");
    for (int pos = 0; pos < n; pos += block_size) {
      int bs = std::min(block_size, n - pos);
      const int* block_idx = idx_alt + pos;
      gather_rows_kernel<T><<<grid_1d((long long)bs * K, sms), kBlock1D, 0, st>>>(R, block_idx, R_out, bs, K);
      launched("gather_rows_kernel");
      gather_int_kernel<<<grid_1d(bs, sms), kBlock1D, 0, st>>>(cats, block_idx, cats_in, bs);
      launched("gather_int_kernel");
      colsum_dispatch<T>(colsum_algo, R_out, R_in_sum, ones, bs, K, sms, st);
      scatter_add_to_O<T>(R_out, cats_in, bs, K, B, 0, O, use_shared, shared_bytes, sms, st);
      outer_kernel<T><<<(ob_total + kBlock1D - 1) / kBlock1D, kBlock1D, 0, st>>>(E, Pr_b, R_in_sum, (long long)B,
                                                                                 (long long)K, 0LL);
      launched("outer_kernel");
      if (stabilized)
        penalty_kernel<T, true><<<(ob_total + kBlock1D - 1) / kBlock1D, kBlock1D, 0, st>>>(E, O, theta, pen, B, K);
      else
        penalty_kernel<T, false><<<(ob_total + kBlock1D - 1) / kBlock1D, kBlock1D, 0, st>>>(E, O, theta, pen, B, K);
      launched("penalty_kernel");
      fused_pen_norm_kernel<T, int><<<bs, warp_aligned_bdim(K), 0, st>>>(sim, pen, cats_in, block_idx, R_out, term,
                                                                         bs, K);
      launched("fused_pen_norm_kernel");
      scatter_rows_kernel<T><<<grid_1d((long long)bs * K, sms), kBlock1D, 0, st>>>(R_out, block_idx, R, bs, K);
      launched("scatter_rows_kernel");
      colsum_dispatch<T>(colsum_algo, R_out, R_out_sum, ones, bs, K, sms, st);
      scatter_add_to_O<T>(R_out, cats_in, bs, K, B, 1, O, use_shared, shared_bytes, sms, st);
      outer_kernel<T><<<(ob_total + kBlock1D - 1) / kBlock1D, kBlock1D, 0, st>>>(E, Pr_b, R_out_sum, (long long)B,
                                                                                 (long long)K, 1LL);
      launched("outer_kernel");
    }
    T host_obj = objective<T>(R, sim, O, E, theta, sigma, obj_scalar, n, K, B, stabilized, st);
    objs.push_back(host_obj);
    if ((int)objs.size() >= kWindow + 1) {
      T obj_old = T(0), obj_new = T(0);
      for (int i = 0; i < kWindow; i++) {
        obj_old += objs[objs.size() - 2 - i];
        obj_new += objs[objs.size() - 1 - i];
      }
      if ((obj_old - obj_new) < tol * std::abs(obj_old)) break;
    }
  }
  for (size_t i = 0; i < objs.size(); ++i) objectives_out[i] = objs[i];
  *n_iter = (int)objs.size();
  cuda_ok(cudaStreamSynchronize(st), "sync");
}

// correction_batched_impl (correction_batched.cu:17-130); Z receives the corrected embedding.
template <typename T>
void correction_batched(const T* X, const T* R, const T* O, const int* cats, const int* cat_offsets,
                        const int* cell_indices, const T* lambda_kb, int n, int d, int K, int B, T* Z,
                        cudaStream_t st) {
  Scratch ws;
  const int nb1 = B + 1;
  T* inv_mats = ws.get<T>((size_t)K * nb1 * nb1);
  T* P = ws.get<T>((size_t)K * nb1 * d);
  T* W_all = ws.get<T>((size_t)K * nb1 * d);
  T* g_factor = ws.get<T>((size_t)K * B);
  T* g_P_row0 = ws.get<T>((size_t)K * B);
  T* X_sorted = ws.get<T>((size_t)n * d);
  T* R_sorted = ws.get<T>((size_t)n * K);
  cuda_ok(cudaMemcpyAsync(Z, X, (size_t)n * d * sizeof(T), cudaMemcpyDeviceToDevice, st), "copy");
  int bdim = std::min((int)kMaxBlockDim, std::max((int)kWarp, (B + (int)kWarp - 1) / (int)kWarp * (int)kWarp));
  compute_inv_mats_kernel<T><<<K, bdim, 0, st>>>(O, lambda_kb, inv_mats, g_factor, g_P_row0, B, K, -1);
  launched("compute_inv_mats_kernel");
  cublasHandle_t h = handle();
  blas_ok(cublasSetStream(h, st), "cublasSetStream");
  T one = T(1), zero = T(0);
  cuda_ok(cudaMemsetAsync(P, 0, (size_t)K * nb1 * d * sizeof(T), st), "memset");
  blas_ok(cublas_gemm<T>(h, CUBLAS_OP_N, CUBLAS_OP_T, d, K, n, &one, X, d, R, K, &zero, P, nb1 * d),
          "cublas_gemm(correction_batched row0)");
  gather_rows_kernel<T><<<strided_grid((long long)n * d, kBlock1D), kBlock1D, 0, st>>>(X, cell_indices, X_sorted, n, d);
  launched("gather_rows_kernel");
  gather_rows_kernel<T><<<strided_grid((long long)n * K, kBlock1D), kBlock1D, 0, st>>>(R, cell_indices, R_sorted, n, K);
  launched("gather_rows_kernel");
  std::vector<int> off(B + 1);
  cuda_ok(cudaMemcpyAsync(off.data(), cat_offsets, (size_t)(B + 1) * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  cuda_ok(cudaStreamSynchronize(st), "sync");
  for (int b = 0; b < B; b++) {
    int nbc = off[b + 1] - off[b];
    if (nbc == 0) continue;
    blas_ok(cublas_gemm<T>(h, CUBLAS_OP_N, CUBLAS_OP_T, d, K, nbc, &one, X_sorted + (size_t)off[b] * d, d,
                           R_sorted + (size_t)off[b] * K, K, &zero, P + (b + 1) * d, nb1 * d),
            "cublas_gemm(correction_batched per-batch)");
  }
  blas_ok(cublas_gemm_strided_batched<T>(h, CUBLAS_OP_N, CUBLAS_OP_N, d, nb1, nb1, &one, P, d, (long long)nb1 * d,
                                         inv_mats, nb1, (long long)nb1 * nb1, &zero, W_all, d, (long long)nb1 * d, K),
          "cublas_gemm_strided_batched(correction_batched W_all)");
  cuda_ok(cudaMemset2DAsync(W_all, (size_t)nb1 * d * sizeof(T), 0, d * sizeof(T), K, st), "memset2d");
  batched_correction_kernel<T><<<strided_grid((long long)n * d, kBlock1D), kBlock1D, 0, st>>>(Z, W_all, cats, R, n,
                                                                                              d, K, nb1);
  launched("batched_correction_kernel");
  cuda_ok(cudaStreamSynchronize(st), "sync");
}

// _scatter_add_cp (_helper.py:63-145): shared-memory kernel or plain kernel by the same rule.
template <typename T>
void scatter_add(const T* X, T* out, const int* cats, int n, int cols, int switcher, int B, cudaStream_t st) {
  constexpr int kMinCellsForShared = 50000, kMinCellsPerBatch = 10000, kMinCellsPerBlock = 64;
  constexpr size_t kMaxShared = 48 * 1024;
  bool use_shared = false;
  if (B > 0 && n >= kMinCellsForShared) {
    const int cells_per_batch = n / B;
    if ((size_t)B * cols * sizeof(T) <= kMaxShared && cells_per_batch >= kMinCellsPerBatch) use_shared = true;
  }
  if (use_shared) {
    int n_blocks = std::min(n_sm() * 4, std::max(1, (n + kMinCellsPerBlock - 1) / kMinCellsPerBlock));
    scatter_add_shared_kernel<T><<<n_blocks, kBlock1D, (size_t)B * cols * sizeof(T), st>>>(X, cats, n, cols, B,
                                                                                          switcher, out);
    launched("scatter_add_shared_kernel");
  } else {
    size_t N = (size_t)n * cols;
    scatter_add_kernel<T><<<strided_grid((long long)N, kBlock1D), kBlock1D, 0, st>>>(X, cats, (size_t)n, (size_t)cols,
                                                                                     (size_t)switcher, out);
    launched("scatter_add_kernel");
  }
}

// _column_sum / _column_sum_atomic / _gemm_colsum (_helper.py:310-361; colsum.cu:14-55)
template <typename T>
void colsum(const T* A, T* out, int rows, int cols, int algo, cudaStream_t st) {
  const int sms = n_sm();
  if (algo == 0) {
    int threads = std::min(kMaxBlock1D, std::max((int)kWarp, (rows + (int)kWarp - 1) / (int)kWarp * (int)kWarp));
    colsum_kernel<T><<<std::min(cols, sms * kBlocksPerSm), threads, 0, st>>>(A, out, rows, cols);
    launched("colsum_kernel");
  } else if (algo == 1) {
    cuda_ok(cudaMemsetAsync(out, 0, cols * sizeof(T), st), "memset");
    int col_tiles = (cols + (int)kWarp - 1) / (int)kWarp;
    int target_row_tiles = std::max(1, sms * 4 / std::max(1, col_tiles));
    size_t rows_per_tile = std::max((size_t)kWarp, (size_t)(rows + target_row_tiles - 1) / target_row_tiles);
    int row_tiles = (int)((rows + rows_per_tile - 1) / rows_per_tile);
    colsum_atomic_kernel<T><<<dim3(col_tiles, row_tiles), dim3(kWarp, kWarp), 0, st>>>(A, out, rows, cols,
                                                                                      rows_per_tile);
    launched("colsum_atomic_kernel");
  } else {
    Scratch ws;
    T* ones = ws.get<T>(rows);
    std::vector<T> h(rows, T(1));
    cuda_ok(cudaMemcpyAsync(ones, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st), "H2D");
    T one = T(1), zero = T(0);
    blas_ok(cublasSetStream(handle(), st), "cublasSetStream");
    blas_ok(cublas_gemv<T>(handle(), CUBLAS_OP_N, cols, rows, &one, A, cols, ones, 1, &zero, out, 1), "gemv");
    cuda_ok(cudaStreamSynchronize(st), "sync");
  }
}

// _cov_sparse (_sparse_pca.py:138-199) of a float32 CSR matrix with int32 indices:
// gram_csr_upper -> copy_upper_to_lower; the column means in float64 by mean_var_minor
// (_utils.py:88-105) cast to float32; gram *= 1 / n; cov_from_gram.  return_gram: the raw
// Gram (not scaled, no mean).  cov: float32 [ncols][ncols]; mean: float32 [ncols].
void pca_cov_csr(const int* indptr, const int* indices, const float* data, int nrows, int ncols, long long nnz,
                 int return_gram, float* cov, float* mean, cudaStream_t st) {
  cuda_ok(cudaMemsetAsync(cov, 0, sizeof(float) * (size_t)ncols * ncols, st), "memset");
  gram_csr_upper_kernel<float, int><<<strided_grid(nrows, 1), 128, 0, st>>>(indptr, indices, data, nrows, ncols, cov);
  launched("gram_csr_upper_kernel");
  const dim3 mb(32, 32), mg(strided_grid(ncols, 32), strided_grid(ncols, 32));
  copy_upper_to_lower_kernel<float><<<mg, mb, 0, st>>>(cov, ncols);
  launched("copy_upper_to_lower_kernel");
  if (return_gram) {
    cuda_ok(cudaStreamSynchronize(st), "sync");
    return;
  }
  Scratch ws;
  double* m64 = ws.get<double>(ncols);
  double* v64 = ws.get<double>(ncols);
  cuda_ok(cudaMemsetAsync(m64, 0, sizeof(double) * ncols, st), "memset");
  cuda_ok(cudaMemsetAsync(v64, 0, sizeof(double) * ncols, st), "memset");
  if (nnz > 0) {
    mean_var_minor_kernel<float, int><<<strided_grid(nnz, 256), 256, 0, st>>>(indices, data, m64, v64, nnz);
    launched("mean_var_minor_kernel");
  }
  std::vector<double> h(ncols);
  cuda_ok(cudaMemcpyAsync(h.data(), m64, sizeof(double) * ncols, cudaMemcpyDeviceToHost, st), "D2H");
  cuda_ok(cudaStreamSynchronize(st), "sync");
  std::vector<float> hm(ncols);
  for (int i = 0; i < ncols; ++i) hm[i] = (float)(h[i] / nrows);  // mean /= major; .astype(x.dtype)
  cuda_ok(cudaMemcpyAsync(mean, hm.data(), sizeof(float) * ncols, cudaMemcpyHostToDevice, st), "H2D");
  // gram_matrix *= 1 / x.shape[0] (float32 array times a Python float)
  std::vector<float> g((size_t)ncols * ncols);
  cuda_ok(cudaMemcpyAsync(g.data(), cov, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, st), "D2H");
  cuda_ok(cudaStreamSynchronize(st), "sync");
  const float inv = (float)(1.0 / (double)nrows);
  for (float& x : g) x *= inv;
  cuda_ok(cudaMemcpyAsync(cov, g.data(), sizeof(float) * g.size(), cudaMemcpyHostToDevice, st), "H2D");
  cov_from_gram_kernel<float><<<mg, mb, 0, st>>>(cov, cov, mean, mean, ncols);
  launched("cov_from_gram_kernel");
  cuda_ok(cudaStreamSynchronize(st), "sync");
}

}  // namespace

extern "C" int ref_pca_cov_csr_f32(const int* indptr, const int* indices, const float* data, int nrows, int ncols,
                                   long long nnz, int return_gram, float* cov, float* mean, void* stream) {
  return guarded([&] { pca_cov_csr(indptr, indices, data, nrows, ncols, nnz, return_gram, cov, mean,
                                   (cudaStream_t)stream); });
}

#define REF_BOTH(NAME, ARGS_T, CALL)                                                      \
  extern "C" int NAME##_f32 ARGS_T(float) { return guarded([&] { CALL(float); }); }       \
  extern "C" int NAME##_f64 ARGS_T(double) { return guarded([&] { CALL(double); }); }

extern "C" const char* ref_last_error(void) { return g_err.c_str(); }

#define CL_ARGS(T)                                                                                          \
  (const T* Z_norm, T* R, T* E, T* O, const T* Pr_b, const int* cats, const T* theta, int n, int d, int K,    \
   int B, int block_size, int colsum_algo, double sigma, double tol, int max_iter, unsigned seed,             \
   int stabilized, T* objectives, int* n_iter, void* stream)
#define CL_CALL(T)                                                                                          \
  clustering_loop<T>(Z_norm, R, E, O, Pr_b, cats, theta, n, d, K, B, block_size, colsum_algo, sigma, tol,     \
                     max_iter, seed, stabilized != 0, objectives, n_iter, (cudaStream_t)stream)
REF_BOTH(ref_clustering_loop, CL_ARGS, CL_CALL)

#define OBJ_ARGS(T)                                                                                         \
  (const T* R, const T* S, const T* O, const T* E, const T* theta, double sigma, int n, int K, int B,        \
   int stabilized, T* out, void* stream)
#define OBJ_CALL(T)                                                                                         \
  {                                                                                                         \
    Scratch ws;                                                                                             \
    *out = objective<T>(R, S, O, E, theta, (T)sigma, ws.get<T>(1), n, K, B, stabilized != 0,                \
                        (cudaStream_t)stream);                                                              \
  }
REF_BOTH(ref_compute_objective, OBJ_ARGS, OBJ_CALL)

#define CB_ARGS(T)                                                                                          \
  (const T* X, const T* R, const T* O, const int* cats, const int* cat_offsets, const int* cell_indices,     \
   const T* lambda_kb, int n, int d, int K, int B, T* Z, void* stream)
#define CB_CALL(T) \
  correction_batched<T>(X, R, O, cats, cat_offsets, cell_indices, lambda_kb, n, d, K, B, Z, (cudaStream_t)stream)
REF_BOTH(ref_correction_batched, CB_ARGS, CB_CALL)

#define L2_ARGS(T) (const T* src, T* dst, int rows, int cols, void* stream)
#define L2_CALL(T)                                                                                          \
  {                                                                                                         \
    l2_row_normalize_kernel<T><<<rows, warp_aligned_bdim(cols), 0, (cudaStream_t)stream>>>(src, dst, rows,  \
                                                                                          cols);           \
    launched("l2_row_normalize_kernel");                                                                    \
  }
REF_BOTH(ref_l2_row_normalize, L2_ARGS, L2_CALL)

#define L1_ARGS(T) (T* X, long long rows, long long cols, void* stream)
#define L1_CALL(T)                                                                                          \
  {                                                                                                         \
    normalize_kernel<T><<<(unsigned)rows, warp_aligned_bdim((unsigned)cols), 0, (cudaStream_t)stream>>>(X, rows, \
                                                                                                      cols); \
    launched("normalize_kernel");                                                                           \
  }
REF_BOTH(ref_l1_normalize, L1_ARGS, L1_CALL)

#define SA_ARGS(T) (const T* X, T* out, const int* cats, int n, int cols, int switcher, int B, void* stream)
#define SA_CALL(T) scatter_add<T>(X, out, cats, n, cols, switcher, B, (cudaStream_t)stream)
REF_BOTH(ref_scatter_add, SA_ARGS, SA_CALL)

#define CS_ARGS(T) (const T* A, T* out, int rows, int cols, int algo, void* stream)
#define CS_CALL(T) colsum<T>(A, out, rows, cols, algo, (cudaStream_t)stream)
REF_BOTH(ref_colsum, CS_ARGS, CS_CALL)

#define OU_ARGS(T) (T* E, const T* Pr_b, const T* R_sum, long long n_cats, long long cols, long long switcher, void* stream)
#define OU_CALL(T)                                                                                          \
  {                                                                                                         \
    outer_kernel<T><<<strided_grid(n_cats * cols, 256), 256, 0, (cudaStream_t)stream>>>(E, Pr_b, R_sum, n_cats, \
                                                                                       cols, switcher);     \
    launched("outer_kernel");                                                                               \
  }
REF_BOTH(ref_outer, OU_ARGS, OU_CALL)
