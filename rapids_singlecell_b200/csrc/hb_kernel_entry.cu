// Kernel-level entry points of the 16-bit path: the cell-order centroid pass, the ridge
// moments and the correction apply, each run alone on caller buffers (the reference binds its
// clustering and correction steps one by one as well, _cuda/harmony/clustering/clustering.cu:
// 397-504, _cuda/harmony/correction/correction_batched.cu:135-172).  hb_harmonize drives the
// same launchers; these entry points let a caller (and the kernel-level tests) check them
// against a plain computation on the same 16-bit inputs.
#include "hb_internal.h"

using namespace hb;

namespace {

int sixteen_bit(int32_t dtype, const char* who) {
  if (dtype == HB_BF16 || dtype == HB_FP16) return HB_OK;
  set_error("%s: dtype must be HB_BF16 or HB_FP16", who);
  return HB_ERR_INVALID;
}

// split-n chunks of the moments and 128-cell tiles of the apply over the batch-sorted list,
// as the plan builds them
int64_t moment_chunk_len(int64_t n, int d, int K) {
  const int cen_tiles = div_up(K, 128) * div_up(d, 64);
  const int64_t target = std::max(1, 2 * num_sms() / cen_tiles);
  return std::max<int64_t>(256, (n + target - 1) / target);
}

bool offsets_ok(const int64_t* off, int B, int64_t n) {
  if (!off || off[0] != 0 || off[B] != n) return false;
  for (int b = 0; b < B; ++b)
    if (off[b + 1] < off[b]) return false;
  return true;
}

}  // namespace

extern "C" {

HB_API size_t hb_tc_centroids_workspace_bytes(int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t n_keys) {
  if (n < 1 || n_pcs < 1 || n_clusters < 1 || n_keys < 1) return 0;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tc_centroid_grid(n_clusters), (n + 511) / 512));
  Carver cv(nullptr, 0);
  cv.take<float>((size_t)grid * n_clusters * n_pcs);
  cv.take<float>((size_t)grid * n_keys * n_clusters);
  return cv.off + 256;
}

HB_API int hb_tc_centroids(const void* Zn, int32_t ldz, const void* R, int32_t ldr, int64_t n, int32_t n_pcs,
                           int32_t n_clusters, const int32_t* ckey, int32_t n_keys, int32_t dtype, void* Yn,
                           int32_t ldy, double* Osum, void* workspace, size_t workspace_bytes, int32_t* err,
                           void* stream) {
  HB_TRY(sixteen_bit(dtype, "hb_tc_centroids"));
  if (!Zn || !R || !ckey || !Yn || !Osum || !err || n < 1 || n > 2147483647LL || n_pcs < 1 || n_clusters < 1 ||
      n_keys < 1 || ldz < n_pcs || ldz % 8 || ldr < n_clusters || ldr % 8 || ldy < n_pcs || ldy % 8) {
    set_error("hb_tc_centroids: bad argument");
    return HB_ERR_INVALID;
  }
  if (!cs_supported(n_pcs, n_clusters, n_keys, ldz)) {
    set_error("hb_tc_centroids: shape outside the cell-order pass (n_pcs=%d n_clusters=%d n_keys=%d)", n_pcs,
              n_clusters, n_keys);
    return HB_ERR_UNSUPPORTED;
  }
  const size_t need = hb_tc_centroids_workspace_bytes(n, n_pcs, n_clusters, n_keys);
  if (!workspace || workspace_bytes < need) {
    set_error("hb_tc_centroids: workspace too small: %zu < %zu", workspace_bytes, need);
    return HB_ERR_WORKSPACE;
  }
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tc_centroid_grid(n_clusters), (n + 511) / 512));
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  float* P = cv.take<float>((size_t)grid * n_clusters * n_pcs);
  float* Opart = cv.take<float>((size_t)grid * n_keys * n_clusters);
  const int64_t rows_alloc = (n + 127) / 128 * 128 + 8;
  cudaStream_t st = (cudaStream_t)stream;
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
  CenStreamArgs ca{n, (int)((rows_alloc - 8) / 128), ckey, n_pcs, n_clusters, n_keys, P, Opart, err, Yn, ldy,
                   nullptr, 0};
  if (dtype == HB_BF16)
    return launch_tc_centroid_stream<__nv_bfloat16>(ca, Zn, ldz, R, ldr, rows_alloc, grid, Osum, st);
  return launch_tc_centroid_stream<__half>(ca, Zn, ldz, R, ldr, rows_alloc, grid, Osum, st);
}

HB_API size_t hb_tc_moments_workspace_bytes(int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t n_batches) {
  if (n < 1 || n_pcs < 1 || n_clusters < 1 || n_batches < 1) return 0;
  const int64_t len = moment_chunk_len(n, n_pcs, n_clusters);
  const int64_t chunks = (n + len - 1) / len + n_batches;
  Carver cv(nullptr, 0);
  cv.take<float>((size_t)chunks * n_clusters * n_pcs);
  cv.take<AccumChunk>((size_t)chunks);
  cv.take<int32_t>((size_t)n_batches + 1);
  return cv.off + 256;
}

HB_API int hb_tc_moments(const float* X, const void* R, int32_t ldr, const int32_t* cell_index,
                         const int64_t* batch_offsets, int64_t n, int32_t n_pcs, int32_t n_clusters,
                         int32_t n_batches, int32_t dtype, double* M, void* workspace, size_t workspace_bytes,
                         int32_t* err, void* stream) {
  HB_TRY(sixteen_bit(dtype, "hb_tc_moments"));
  if (!X || !R || !cell_index || !M || !err || n < 1 || n > 2147483647LL || n_pcs < 1 || n_pcs > 256 ||
      n_clusters < 1 || n_clusters > 256 || n_batches < 1 || ldr < n_clusters || ldr % 8 ||
      !offsets_ok(batch_offsets, n_batches, n)) {
    set_error("hb_tc_moments: bad argument");
    return HB_ERR_INVALID;
  }
  const size_t need = hb_tc_moments_workspace_bytes(n, n_pcs, n_clusters, n_batches);
  if (!workspace || workspace_bytes < need) {
    set_error("hb_tc_moments: workspace too small: %zu < %zu", workspace_bytes, need);
    return HB_ERR_WORKSPACE;
  }
  const int64_t len = moment_chunk_len(n, n_pcs, n_clusters);
  std::vector<AccumChunk> mch;
  std::vector<int32_t> bco(n_batches + 1, 0);
  for (int b = 0; b < n_batches; ++b) {
    bco[b] = (int32_t)mch.size();
    for (int64_t s = batch_offsets[b]; s < batch_offsets[b + 1]; s += len)
      mch.push_back(AccumChunk{s, (int32_t)std::min<int64_t>(len, batch_offsets[b + 1] - s), b});
  }
  bco[n_batches] = (int32_t)mch.size();
  const int64_t max_chunks = (n + len - 1) / len + n_batches;
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  float* Mpart = cv.take<float>((size_t)max_chunks * n_clusters * n_pcs);
  AccumChunk* d_chunks = cv.take<AccumChunk>((size_t)max_chunks);
  int32_t* d_bco = cv.take<int32_t>((size_t)n_batches + 1);
  cudaStream_t st = (cudaStream_t)stream;
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
  // pageable sources: the copies complete (staged) before the calls return
  HB_CUDA(cudaMemcpyAsync(d_chunks, mch.data(), sizeof(AccumChunk) * mch.size(), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(d_bco, bco.data(), sizeof(int32_t) * bco.size(), cudaMemcpyHostToDevice, st));
  if (dtype == HB_BF16)
    HB_TRY(launch_tc_moments<__nv_bfloat16>((const __nv_bfloat16*)R, ldr, X, n_pcs, cell_index, d_chunks,
                                            (int)mch.size(), n_clusters, n_pcs, Mpart, err, st));
  else
    HB_TRY(launch_tc_moments<__half>((const __half*)R, ldr, X, n_pcs, cell_index, d_chunks, (int)mch.size(),
                                     n_clusters, n_pcs, Mpart, err, st));
  return launch_m_reduce<float>(Mpart, mch.data(), (int)mch.size(), d_bco, n_clusters, n_batches, n_pcs, M, st);
}

HB_API size_t hb_tc_apply_workspace_bytes(int64_t n, int32_t n_batches) {
  if (n < 1 || n_batches < 1) return 0;
  Carver cv(nullptr, 0);
  cv.take<ApplyTile>((size_t)((n + 127) / 128 + n_batches));
  return cv.off + 256;
}

HB_API int hb_tc_apply(const float* X, const void* R, int32_t ldr, const float* W, const int32_t* cell_index,
                       const int64_t* batch_offsets, int64_t n, int32_t n_pcs, int32_t n_clusters,
                       int32_t n_batches, int32_t dtype, float* Z_hat, void* Zn, int32_t ldz, void* workspace,
                       size_t workspace_bytes, int32_t* err, void* stream) {
  HB_TRY(sixteen_bit(dtype, "hb_tc_apply"));
  if (!X || !R || !W || !cell_index || !Z_hat || !Zn || !err || n < 1 || n > 2147483647LL || n_pcs < 1 ||
      n_pcs > 128 || n_clusters < 1 || n_clusters > 256 || n_batches < 1 || ldr < n_clusters || ldr % 8 ||
      ldz < n_pcs || ldz % 8 || !offsets_ok(batch_offsets, n_batches, n)) {
    set_error("hb_tc_apply: bad argument");
    return HB_ERR_INVALID;
  }
  const size_t need = hb_tc_apply_workspace_bytes(n, n_batches);
  if (!workspace || workspace_bytes < need) {
    set_error("hb_tc_apply: workspace too small: %zu < %zu", workspace_bytes, need);
    return HB_ERR_WORKSPACE;
  }
  std::vector<ApplyTile> tiles;
  for (int b = 0; b < n_batches; ++b)
    for (int64_t s = batch_offsets[b]; s < batch_offsets[b + 1]; s += 128)
      tiles.push_back(ApplyTile{s, (int32_t)std::min<int64_t>(128, batch_offsets[b + 1] - s), b});
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  ApplyTile* d_tiles = cv.take<ApplyTile>((size_t)((n + 127) / 128 + n_batches));
  cudaStream_t st = (cudaStream_t)stream;
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
  if (tiles.empty()) return HB_OK;
  HB_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), sizeof(ApplyTile) * tiles.size(), cudaMemcpyHostToDevice, st));
  if (dtype == HB_BF16)
    return launch_tc_apply<__nv_bfloat16>(X, n_pcs, (const __nv_bfloat16*)R, ldr, W, cell_index, d_tiles,
                                          (int)tiles.size(), n_clusters, n_pcs, Z_hat, n_pcs, (__nv_bfloat16*)Zn,
                                          ldz, err, st);
  return launch_tc_apply<__half>(X, n_pcs, (const __half*)R, ldr, W, cell_index, d_tiles, (int)tiles.size(),
                                 n_clusters, n_pcs, Z_hat, n_pcs, (__half*)Zn, ldz, err, st);
}

}  // extern "C"
