// Plan, workspace layout and the Harmony iteration driver behind the C ABI.
//
// The loop structure follows harmonize() (preprocessing/_harmony/__init__.py:
// 41-289) and clustering_loop_impl (_cuda/harmony/clustering/clustering.cu:
// 241-393); the kernels it launches are this engine's own (hb_simt.cu,
// hb_membership.cu).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>
#include <cudaTypedefs.h>
#include "hb_internal.h"

namespace hb {

static thread_local char g_err[1024] = "";
thread_local int64_t g_launches = 0;

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int make_row_gather_map(CUtensorMap* tm, const void* base, int64_t rows, int ld, bool bf16) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&encode, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !encode) {
      encode = nullptr;
      set_error("cuTensorMapEncodeTiled is not available from the driver");
      return HB_ERR_CUDA;
    }
  }
  if (((uintptr_t)base & 15) || (ld * 2) % 16) {
    set_error("row gather map: base must be 16-byte aligned and rows a multiple of 16 bytes");
    return HB_ERR_INVALID;
  }
  cuuint64_t gdim[2] = {(cuuint64_t)ld, (cuuint64_t)rows};
  cuuint64_t gstride[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {64, 1};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(tm, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                            const_cast<void*>(base), gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d) for rows=%lld ld=%d", (int)r, (long long)rows, ld);
    return HB_ERR_CUDA;
  }
  return HB_OK;
}

int allow_max_dyn_smem(const void* fn) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return HB_OK;
  cudaFuncAttributes fa;
  HB_CUDA(cudaFuncGetAttributes(&fa, fn));
  int optin = 0;
  HB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  HB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
  done.insert({fn, dev});
  return HB_OK;
}

int num_sms() {
  int dev = 0, v = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 148;
}

}  // namespace hb

using namespace hb;

struct hb_plan {
  hb_params p;
  int esz;        // bytes of the input / output type (4 or 8)
  int ssz;        // bytes of the Z_norm / R storage type (2, 4 or 8)
  int asz;        // bytes of the split-n partial sums (4 or 8)
  int ldz, ldr, ldy;
  MembershipLayout ml;
  MembershipLayout ml1;  // one block ordered by batch: the cell_index when the caller passes none
  int cen_chunks; // split-n chunks of the centroid sum
  int cen_tiles;  // output tiles per chunk
  int max_m_chunks, max_apply_tiles;
  int64_t m_chunk_len;
  int64_t rows_alloc;  // rows of Z_norm and R: whole 128-cell tiles + 8, the padding rows zero
  bool cen_stream;     // 16-bit path: centroid pass in cell order (hb_centroid_stream.cu)
  int nkeys;           // (block, batch) keys: blocks * (batches + 1)
  size_t ws_bytes;
  std::vector<cudaEvent_t> events;       // profiling pool (created on first profiled run)
  std::vector<cudaEvent_t> flag_events;  // one per outer iteration: its end flags have arrived
  ~hb_plan() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    for (cudaEvent_t e : flag_events) cudaEventDestroy(e);
  }
};

namespace {

struct Work {
  void* Zn;
  void* R;
  void* Yn;
  void* Ypart;
  void* Mpart;
  void* W;
  double* O[3];
  double* Pr;
  double* theta;
  double* Nb;
  double* obj_acc;
  double* obj_out;
  double* M;
  double* Omin;  // [nblk][B+1][K] old contribution of each block of the current iteration
  unsigned* barrier;  // grid-barrier counter of the persistent sweep
  int32_t* idx;
  int32_t* lcat;
  int32_t* ckey;    // cell-order (block, batch) keys of the chunk's iterations (streaming centroid pass)
  float* Opart;     // per-CTA per-key sums of the streaming centroid pass
  int32_t* cell_index;  // cells sorted by batch (stable), built when the caller passes none
  int* err;
  RunCtl* ctl;      // device-side run control (k-means stop, run end, convergence)
  int* stop;        // &ctl->stop
  double* objs;     // [max_iter_harmony + 1] objective after each outer iteration
  double* kobj;     // [max_iter_harmony][max_iter_clustering] k-means objectives
  int32_t* kiters;  // [max_iter_harmony] k-means iterations run
  AccumChunk* cen_chunks;
  AccumChunk* m_chunks;
  int32_t* batch_chunk_off;
  ApplyTile* apply_tiles;
  void* pen_g;      // plain paths: [B][K] penalty table in global memory (many batches)
  MembershipBufs mb;
  MembershipBufs mb1;
};

void carve(const hb_plan& P, Carver& cv, Work& w) {
  const hb_params& p = P.p;
  const int64_t n = p.n_cells;
  const int K = p.n_clusters, B = p.n_batches, d = p.n_pcs;
  w.Zn = cv.take<char>((size_t)P.rows_alloc * P.ldz * P.ssz);
  w.R = cv.take<char>((size_t)P.rows_alloc * P.ldr * P.ssz);
  w.Yn = cv.take<char>((size_t)K * P.ldy * P.ssz);
  w.Ypart = cv.take<char>((size_t)P.cen_chunks * K * d * P.asz);
  w.Mpart = cv.take<char>((size_t)P.max_m_chunks * K * d * P.asz);
  w.W = cv.take<char>((size_t)B * K * d * P.esz);
  // observed counts: [B][K] plus a column-sum row (kept by the 16-bit sweep)
  for (int i = 0; i < 3; ++i) w.O[i] = cv.take<double>((size_t)(B + 1) * K);
  w.Pr = cv.take<double>(B);
  w.theta = cv.take<double>(B);
  w.Nb = cv.take<double>(B);
  w.obj_acc = cv.take<double>(1);
  w.obj_out = cv.take<double>(std::max(p.max_iter_clustering, 1) + 1);
  w.M = cv.take<double>((size_t)K * (B + 1) * d);
  w.Omin = cv.take<double>((size_t)P.ml.nblk * (B + 1) * K);
  w.barrier = cv.take<unsigned>(4);
  w.idx = cv.take<int32_t>((size_t)kMaxIterChunk * n);
  w.lcat = cv.take<int32_t>((size_t)kMaxIterChunk * n);
  w.ckey = P.cen_stream ? cv.take<int32_t>((size_t)kMaxIterChunk * n) : nullptr;
  w.Opart = P.cen_stream ? cv.take<float>((size_t)P.cen_chunks * P.nkeys * K) : nullptr;
  w.err = cv.take<int>(4);
  w.ctl = cv.take<RunCtl>(1);
  w.stop = w.ctl ? &w.ctl->stop : nullptr;
  w.objs = cv.take<double>((size_t)p.max_iter_harmony + 1);
  w.kobj = cv.take<double>((size_t)p.max_iter_harmony * std::max(p.max_iter_clustering, 1));
  w.kiters = cv.take<int32_t>(p.max_iter_harmony);
  w.cen_chunks = cv.take<AccumChunk>(P.cen_chunks);
  w.m_chunks = cv.take<AccumChunk>(P.max_m_chunks);
  w.batch_chunk_off = cv.take<int32_t>(B + 1);
  w.apply_tiles = cv.take<ApplyTile>(P.max_apply_tiles);
  w.pen_g = P.ssz == 2 ? nullptr : (void*)cv.take<char>((size_t)B * K * P.ssz);
  membership_carve(cv, P.ml, w.mb);
  w.cell_index = cv.take<int32_t>((size_t)n);
  membership_carve(cv, P.ml1, w.mb1);
}

int validate(const hb_params& p) {
  if (p.n_cells < 1 || p.n_cells > 2147483647LL) { set_error("n_cells must be in [1, 2^31)"); return HB_ERR_INVALID; }
  if (p.n_pcs < 1) { set_error("n_pcs must be >= 1"); return HB_ERR_INVALID; }
  if (p.n_clusters < 1) { set_error("n_clusters must be >= 1"); return HB_ERR_INVALID; }
  if (p.n_batches < 1) { set_error("n_batches must be >= 1"); return HB_ERR_INVALID; }
  if (p.block_size < 1) { set_error("block_size = int(n_cells * block_proportion) must be >= 1"); return HB_ERR_INVALID; }
  if (p.max_iter_harmony < 1) { set_error("max_iter_harmony must be >= 1"); return HB_ERR_INVALID; }
  if (p.max_iter_clustering < 0) { set_error("max_iter_clustering must be >= 0"); return HB_ERR_INVALID; }
  if (!(p.sigma > 0)) { set_error("sigma must be > 0"); return HB_ERR_INVALID; }
  if (p.sweep_wait_ns < 0 || p.sweep_wait_ns > 60000000000LL) {
    set_error("sweep_wait_ns must be in [0, 60 s]");
    return HB_ERR_INVALID;
  }
  if (p.test_unmet_arrivals < 0 || p.test_unmet_arrivals > 1) {
    set_error("test_unmet_arrivals must be 0 or 1");
    return HB_ERR_INVALID;
  }
  if (p.sweep_form < HB_SWEEP_AUTO || p.sweep_form > HB_SWEEP_1x4_1BUF) {
    set_error("sweep_form must be in [0, 4]");
    return HB_ERR_INVALID;
  }
  const int64_t nblk = (p.n_cells + p.block_size - 1) / p.block_size;
  if (nblk > kMaxBlocks) {
    set_error("block_proportion too small: %lld blocks per iteration (max %d)", (long long)nblk, kMaxBlocks);
    return HB_ERR_UNSUPPORTED;
  }
  if (p.n_clusters > 256) { set_error("n_clusters=%d exceeds the supported maximum of 256", p.n_clusters); return HB_ERR_UNSUPPORTED; }
  if (p.n_pcs > 256) { set_error("n_pcs=%d exceeds the supported maximum of 256", p.n_pcs); return HB_ERR_UNSUPPORTED; }
  if (p.precision < HB_FP32 || p.precision > HB_FP16) {
    set_error("unknown precision %d", p.precision);
    return HB_ERR_INVALID;
  }
  if ((p.precision == HB_BF16 || p.precision == HB_FP16) && p.n_pcs > 128) {
    set_error("n_pcs=%d exceeds 128 for the tensor-core path", p.n_pcs);
    return HB_ERR_UNSUPPORTED;
  }
  // the 16-bit sweep keeps its penalty and delta tables in shared memory; the plain paths
  // switch to global tables (k_pen_table, direct atomics) when theirs do not fit
  const size_t smem = (size_t)4 * 2 * p.n_batches * p.n_clusters;
  if ((p.precision == HB_BF16 || p.precision == HB_FP16) && smem > 160 * 1024) {
    set_error("n_batches * n_clusters = %d too large for the tensor-core sweep's shared-memory tables; "
              "use precision fp32 or fp64", p.n_batches * p.n_clusters);
    return HB_ERR_UNSUPPORTED;
  }
  if (p.precision == HB_BF16 || p.precision == HB_FP16) {
    // the sweep's shared memory also holds the tile buffers, the centroid tile and the staged
    // R rows beside those tables: ask the layouts themselves (as the launch will)
    bool fits = true;
    if (tc_sweep_fits_any((int)p.n_pcs, (int)p.n_clusters, (int)p.n_batches, fits) != HB_OK) {
      (void)cudaGetLastError();  // no device to ask here: the launch makes the same test
      set_error("%s", "");
      fits = true;
    }
    if (!fits) {
      set_error("n_batches=%d with n_clusters=%d and n_pcs=%d does not fit the tensor-core sweep's shared "
                "memory; use precision fp32 or fp64", p.n_batches, p.n_clusters, p.n_pcs);
      return HB_ERR_UNSUPPORTED;
    }
  }
  if ((size_t)16 * p.n_batches > 200 * 1024) {
    set_error("n_batches=%d exceeds 12800 (ridge solve tables)", p.n_batches);
    return HB_ERR_UNSUPPORTED;
  }
  if (MembershipLayout ml = membership_layout(p.n_cells, p.block_size, 1); ml.cap > 16384) {
    set_error("n_cells=%lld too large for the block splitter select", (long long)p.n_cells);
    return HB_ERR_UNSUPPORTED;
  }
  return HB_OK;
}

}  // namespace

extern "C" {

const char* hb_last_error(void) { return g_err; }
const char* hb_version(void) { return "harmony_b200 0.1 (sm_100a)"; }

int hb_plan_create(const hb_params* params, hb_plan** plan) {
  if (!params || !plan) { set_error("null argument"); return HB_ERR_INVALID; }
  HB_TRY(validate(*params));
  hb_plan* P = new hb_plan();
  P->p = *params;
  const hb_params& p = P->p;
  P->esz = p.precision == HB_FP64 ? 8 : 4;
  P->ssz = (p.precision == HB_BF16 || p.precision == HB_FP16) ? 2 : P->esz;
  P->asz = P->esz;
  const int vec = 16 / P->ssz;
  P->ldz = (int)align_up(p.n_pcs, vec);
  P->ldr = (int)align_up(p.n_clusters, vec);
  P->ldy = P->ldz;
  P->ml = membership_layout(p.n_cells, p.block_size, p.n_batches);
  P->ml1 = membership_layout(p.n_cells, p.n_cells, p.n_batches);
  const int sms = num_sms();
  P->cen_tiles = div_up(p.n_clusters, 128) * div_up(p.n_pcs, 64);
  const int64_t target = std::max(1, 2 * sms / P->cen_tiles);
  P->cen_chunks = (int)std::max<int64_t>(1, std::min<int64_t>(target, (p.n_cells + 255) / 256));
  // 16-bit path: one partial per CTA, at most one CTA per SM and per 128-cell tile (four
  // tiles per CTA at least, so that small problems leave SMs to concurrent ones)
  if (P->ssz == 2)
    P->cen_chunks = (int)std::max<int64_t>(1, std::min<int64_t>(tc_centroid_grid(p.n_clusters),
                                                                (p.n_cells + 511) / 512));
  P->m_chunk_len = std::max<int64_t>(256, (p.n_cells + target - 1) / target);
  P->max_m_chunks = (int)((p.n_cells + P->m_chunk_len - 1) / P->m_chunk_len) + p.n_batches;
  P->max_apply_tiles = (int)((p.n_cells + 31) / 32) + p.n_batches;
  P->rows_alloc = (p.n_cells + 127) / 128 * 128 + 8;
  P->nkeys = P->ml.nblk * (p.n_batches + 1);
  P->cen_stream = false;
  if (P->ssz == 2 && cs_supported((int)p.n_pcs, (int)p.n_clusters, P->nkeys, P->ldz)) {
    // the 4-D tile maps must encode for these row strides (no memory is touched)
    CUtensorMap probe;
    const bool bf = p.precision == HB_BF16;
    P->cen_stream = make_tile_map4(&probe, (const void*)(uintptr_t)4096, P->rows_alloc, P->ldz, (P->ldz + 63) / 64, bf) ==
                        HB_OK &&
                    make_tile_map4(&probe, (const void*)(uintptr_t)4096, P->rows_alloc, P->ldr,
                                   2 * (((int)p.n_clusters + 127) / 128), bf) == HB_OK;
  }
  Carver cv(nullptr, 0);
  Work w;
  carve(*P, cv, w);
  P->ws_bytes = cv.off + 256;
  *plan = P;
  return HB_OK;
}

void hb_plan_destroy(hb_plan* plan) { delete plan; }

size_t hb_plan_workspace_bytes(const hb_plan* plan) { return plan ? plan->ws_bytes : 0; }

int hb_similarity(const void* Zn, int32_t ldz, const void* Yn, int32_t ldy, const int32_t* idx, int64_t n,
                  int32_t n_pcs, int32_t n_clusters, int32_t dtype, float* S, int32_t* err, void* stream) {
  if (n < 1 || n_pcs < 1 || n_pcs > 128 || n_clusters < 1 || n_clusters > 256 || ldz % 8 || ldy % 8 ||
      ldz < n_pcs || ldy < n_pcs || !Zn || !Yn || !idx || !S || !err) {
    set_error("hb_similarity: bad argument");
    return HB_ERR_INVALID;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == HB_FP16)
    return launch_tc_similarity<__half>((const __half*)Zn, ldz, (const __half*)Yn, ldy, idx, nullptr, n, n_pcs,
                                        n_clusters, S, err, st);
  if (dtype == HB_BF16)
    return launch_tc_similarity<__nv_bfloat16>((const __nv_bfloat16*)Zn, ldz, (const __nv_bfloat16*)Yn, ldy,
                                               idx, nullptr, n, n_pcs, n_clusters, S, err, st);
  set_error("hb_similarity: dtype must be HB_FP16 or HB_BF16");
  return HB_ERR_INVALID;
}

}  // extern "C"

namespace {

// block update of the plain paths (the 16-bit path runs the persistent sweep instead)
template <typename S>
int block_update(const BlockArgs& a, const double* in, double* out, double* zero, cudaStream_t st) {
  static_assert(std::is_same<S, double>::value || std::is_same<S, float>::value, "plain paths only");
  if constexpr (std::is_same<S, double>::value) return launch_block_update_f64(a, in, out, zero, st);
  else return launch_block_update_f32(a, in, out, zero, st);
}

struct ORing {
  double* buf[3];
  int cur = 0;
  // launch a block update that reads the current state and produces the next
  template <typename S>
  int step(const BlockArgs& a, cudaStream_t st) {
    const int out = (cur + 1) % 3, zero = (cur + 2) % 3;
    HB_TRY(block_update<S>(a, buf[cur], buf[out], buf[zero], st));
    cur = out;
    return HB_OK;
  }
  double* state() const { return buf[cur]; }
};

// T: type of X / Y0 / Z_hat (float or double); S: storage of Z_norm and R
// (T itself on the plain paths, half / bfloat16 on the tensor-core path).
template <typename T, typename S>
int run_impl(hb_plan* P, const T* X, const int32_t* cats, const int32_t* cell_index,
             const int64_t* batch_offsets, const double* theta, const T* Y0, void* ws,
             size_t ws_bytes, T* Zhat, hb_outputs* out, cudaStream_t st) {
  using TA = T;  // split-n partial sums
  const int64_t launches0 = g_launches;
  const hb_params& p = P->p;
  const int64_t n = p.n_cells;
  const int K = p.n_clusters, B = p.n_batches, d = p.n_pcs;
  if (ws_bytes < P->ws_bytes || !ws) {
    set_error("workspace too small: %zu < %zu", ws_bytes, P->ws_bytes);
    return HB_ERR_WORKSPACE;
  }
  Carver cv((void*)align_up((size_t)ws, 256), ws_bytes - 256);
  Work w;
  carve(*P, cv, w);

  // ---- host-side tables ----------------------------------------------------
  std::vector<double> Nb(B), Pr(B), th(theta, theta + B);
  for (int b = 0; b < B; ++b) {
    Nb[b] = (double)(batch_offsets[b + 1] - batch_offsets[b]);
    Pr[b] = Nb[b] / (double)n;
  }
  if (batch_offsets[0] != 0 || batch_offsets[B] != n) {
    set_error("batch_offsets must start at 0 and end at n_cells");
    return HB_ERR_INVALID;
  }
  if (!cell_index) {
    // counting sort of the cells by batch: the partition with a single block
    if (B > 1 && P->ml1.nsub != B) {
      set_error("cell_index must be given when n_batches > %d", kMaxBuckets);
      return HB_ERR_INVALID;
    }
    HB_TRY(membership_build_dev(P->ml1, w.mb1, nullptr, 0, 1, cats, w.cell_index, st));
    cell_index = w.cell_index;
  }
  std::vector<AccumChunk> cen(P->cen_chunks);
  {
    const int64_t len = (n + P->cen_chunks - 1) / P->cen_chunks;
    for (int c = 0; c < P->cen_chunks; ++c) {
      int64_t s = c * len, e = std::min<int64_t>(n, s + len);
      cen[c] = AccumChunk{s, (int32_t)std::max<int64_t>(0, e - s), 0};
    }
  }
  constexpr bool tc_corr = !std::is_same<S, float>::value && !std::is_same<S, double>::value;
  const int64_t apply_rows = tc_corr ? 128 : 32;  // cells per apply tile (tensor-core tiles are 128 rows)
  std::vector<AccumChunk> mch;
  std::vector<int32_t> bco(B + 1, 0);
  std::vector<ApplyTile> tiles;
  for (int b = 0; b < B; ++b) {
    bco[b] = (int32_t)mch.size();
    for (int64_t s = batch_offsets[b]; s < batch_offsets[b + 1]; s += P->m_chunk_len)
      mch.push_back(AccumChunk{s, (int32_t)std::min<int64_t>(P->m_chunk_len, batch_offsets[b + 1] - s), b});
    for (int64_t s = batch_offsets[b]; s < batch_offsets[b + 1]; s += apply_rows)
      tiles.push_back(ApplyTile{s, (int32_t)std::min<int64_t>(apply_rows, batch_offsets[b + 1] - s), b});
  }
  bco[B] = (int32_t)mch.size();
  HB_CUDA(cudaMemcpyAsync(w.Nb, Nb.data(), sizeof(double) * B, cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(w.Pr, Pr.data(), sizeof(double) * B, cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(w.theta, th.data(), sizeof(double) * B, cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(w.cen_chunks, cen.data(), sizeof(AccumChunk) * cen.size(), cudaMemcpyHostToDevice, st));
  if (!mch.empty())
    HB_CUDA(cudaMemcpyAsync(w.m_chunks, mch.data(), sizeof(AccumChunk) * mch.size(), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(w.batch_chunk_off, bco.data(), sizeof(int32_t) * (B + 1), cudaMemcpyHostToDevice, st));
  if (!tiles.empty())
    HB_CUDA(cudaMemcpyAsync(w.apply_tiles, tiles.data(), sizeof(ApplyTile) * tiles.size(), cudaMemcpyHostToDevice, st));
  for (int i = 0; i < 3; ++i) HB_CUDA(cudaMemsetAsync(w.O[i], 0, sizeof(double) * (B + 1) * K, st));
  HB_CUDA(cudaMemsetAsync(w.obj_acc, 0, sizeof(double), st));
  HB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
  HB_CUDA(cudaMemsetAsync(w.ctl, 0, sizeof(RunCtl), st));
  // the sweep's grid-barrier counts (each sweep launch leaves them zero for the next)
  HB_CUDA(cudaMemsetAsync(w.barrier, 0, 4 * sizeof(unsigned), st));
  // the splitter's overflow flag ends the run on the device (k_outer_end) and is read at the
  // end: cleared once per run
  HB_TRY(membership_clear_err(w.mb, st));

  S* Zn = (S*)w.Zn;
  S* R = (S*)w.R;
  S* Yn = (S*)w.Yn;
  ORing ring{{w.O[0], w.O[1], w.O[2]}, 0};

  BlockArgs base{};
  base.Zn = Zn; base.ldz = P->ldz; base.R = R; base.ldr = P->ldr; base.cats = cats;
  base.Yn = Yn; base.ldy = P->ldy; base.Pr = w.Pr; base.theta = w.theta; base.obj_acc = w.obj_acc;
  base.sigma = p.sigma; base.d = d; base.K = K; base.B = B; base.stabilized = p.stabilized_penalty;
  base.pen_g = w.pen_g;

  // ---- initial state (_harmony/__init__.py:292-353) ------------------------
  // padding rows of Z_norm and R (read by the tile loads of the streaming centroid pass) are zero
  HB_CUDA(cudaMemsetAsync((char*)Zn + (size_t)n * P->ldz * P->ssz, 0, (size_t)(P->rows_alloc - n) * P->ldz * P->ssz, st));
  HB_CUDA(cudaMemsetAsync((char*)R + (size_t)n * P->ldr * P->ssz, 0, (size_t)(P->rows_alloc - n) * P->ldr * P->ssz, st));
  HB_TRY(launch_l2_normalize<T, S>(X, n, d, d, Zn, P->ldz, st));
  HB_TRY(launch_l2_normalize<T, S>(Y0, K, d, d, Yn, P->ldy, st));
  double* obj_init = w.objs;  // objs[0]: the objective of the initial state
  constexpr bool tc_path = !std::is_same<S, float>::value && !std::is_same<S, double>::value;
  // one persistent sweep (16-bit path) over `nblk` blocks of `idx`, objective into obj_dst
  int* sweep_stop = nullptr;  // device-side k-means stop passed to the next sweep launch, with sweep_it
  int sweep_it = 0;
  auto sweep = [&](const int32_t* idx, const int32_t* lcat, int64_t bs, int nb, const double* Omin, int init,
                   double* obj_dst) -> int {
    if constexpr (tc_path) {
      SweepArgs sa{};
      sa.Zn = Zn; sa.ldz = P->ldz; sa.R = R; sa.ldr = P->ldr; sa.cats = cats; sa.Yn = Yn; sa.ldy = P->ldy;
      sa.idx = idx; sa.lcat = lcat; sa.n = n; sa.bs = bs; sa.nblk = nb;
      sa.Obuf[0] = w.O[0]; sa.Obuf[1] = w.O[1]; sa.Obuf[2] = w.O[2]; sa.b0 = ring.cur;
      sa.Omin = Omin; sa.Pr = w.Pr; sa.theta = w.theta; sa.obj_acc = w.obj_acc; sa.obj_out = obj_dst;
      sa.sigma = p.sigma; sa.d = d; sa.K = K; sa.B = B; sa.stabilized = p.stabilized_penalty;
      sa.init_mode = init; sa.batch_sorted = P->ml.nsub > 1 || B <= 1;
      sa.max_ctas = p.max_sweep_ctas; sa.barrier = w.barrier; sa.err = w.err;
      sa.wait_ns = p.sweep_wait_ns > 0 ? (uint64_t)p.sweep_wait_ns : 2000000000ull;
      sa.unmet = (unsigned)p.test_unmet_arrivals;
      sa.form = p.sweep_form;
      sa.stop = sweep_stop; sa.it = sweep_it; sa.tol = p.tol_clustering;
      HB_TRY(launch_tc_sweep<S>(sa, st));
      ring.cur = (ring.cur + nb) % 3;
      return HB_OK;
    } else {
      (void)idx; (void)lcat; (void)bs; (void)nb; (void)Omin; (void)init; (void)obj_dst;
      set_error("internal: sweep on the plain path");
      return HB_ERR_INTERNAL;
    }
  };
  if constexpr (tc_path) {
    HB_TRY(sweep(nullptr, cats, n, 1, nullptr, 1, obj_init));
  } else {
    BlockArgs a = base;
    a.idx_new = nullptr; a.new_start = 0; a.n_new = n; a.Om_cur = nullptr; a.Om_next = nullptr;
    a.init_mode = 1;
    HB_TRY(ring.step<S>(a, st));
    HB_TRY(launch_objective_finalize(ring.state(), w.Pr, w.theta, p.sigma, B, K, p.stabilized_penalty,
                                     w.obj_acc, obj_init, st));
  }
  const MembershipLayout& ml = P->ml;
  const int nblk = ml.nblk;
  const int mc = p.max_iter_clustering, mh = p.max_iter_harmony;
  const size_t kstride = (size_t)std::max(mc, 1);
  // pinned read-back: the (ostop, conv) flags of each outer iteration, then the one final read
  // (run control, objectives, k-means iteration counts and objectives, error flags)
  const size_t flag_bytes = align_up(sizeof(int) * 2 * mh, 8);
  const size_t fin_doubles = (size_t)mh + 1 + (size_t)mh * kstride;
  PinnedLease host(flag_bytes + sizeof(double) * fin_doubles + sizeof(int32_t) * mh + sizeof(RunCtl) +
                   2 * sizeof(int));
  if (!host.ptr) {
    set_error("pinned host buffer for the read-backs: cudaMallocHost failed");
    return HB_ERR_CUDA;
  }
  int* h_flag = (int*)host.ptr;
  double* h_objs = (double*)((char*)host.ptr + flag_bytes);
  double* h_kobj = h_objs + mh + 1;
  int32_t* h_kiters = (int32_t*)(h_kobj + (size_t)mh * kstride);
  RunCtl* h_ctl = (RunCtl*)(h_kiters + mh);
  int* h_err = (int*)(h_ctl + 1);
  while ((int)P->flag_events.size() < mh) {
    cudaEvent_t e;
    HB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming | cudaEventBlockingSync));
    P->flag_events.push_back(e);
  }

  // optional device-time profile: event pairs around block-update and centroid launches
  hb_profile* prof = out ? out->profile : nullptr;
  struct Span { int cat; int e0, e1; double bytes; int outer, it; };
  std::vector<Span> spans;
  size_t next_ev = 0;
  auto ev = [&]() -> cudaEvent_t {
    if (next_ev == P->events.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      P->events.push_back(e);
    }
    return P->events[next_ev++];
  };
  auto span_begin = [&](int cat, double bytes, int outer, int it) -> int {
    if (!prof) return -1;
    spans.push_back(Span{cat, (int)next_ev, -1, bytes, outer, it});
    cudaEventRecord(ev(), st);
    return (int)spans.size() - 1;
  };
  auto span_end = [&](int i) {
    if (i < 0) return;
    spans[i].e1 = (int)next_ev;
    cudaEventRecord(ev(), st);
  };
  const double zb = (double)d * P->ssz, rb = (double)K * P->ssz;
  // every k-means launch is gated on the device-side stop, and every correction launch on the
  // end of the run (RunCtl); with tol_clustering = -inf the window-3 test never passes
  // A run with both tolerances at -inf cannot stop early: its launches carry no gate (an error
  // flag raised on the way is reported at the end of the run).
  const bool can_stop = !(std::isinf(p.tol_clustering) && p.tol_clustering < 0) ||
                        !(std::isinf(p.tol_harmony) && p.tol_harmony < 0);
  int* const dstop = can_stop ? w.stop : nullptr;
  const int* const ogate = can_stop ? &w.ctl->ostop : nullptr;

  int checked = 0;  // outer iterations whose end flags the host has seen
  bool host_stop = false;
  for (int outer = 0; outer < mh && !host_stop; ++outer) {
    const uint32_t seed = (uint32_t)((p.random_state + (uint64_t)outer * 1000003ull) & 0xffffffffull);
    // the host stays at most two outer iterations ahead of the device: it sleeps on the end event
    // of iteration outer - 2 while the device still has iteration outer - 1 queued
    if (outer >= 2) {
      HB_CUDA(cudaEventSynchronize(P->flag_events[outer - 2]));
      for (; checked <= outer - 2 && !host_stop; ++checked)
        host_stop = h_flag[2 * checked] || h_flag[2 * checked + 1];
      if (host_stop) break;
    }
    HB_TRY(launch_outer_begin(w.ctl, st));
    const int ring0 = ring.cur;
    for (int it0 = 0; it0 < mc; it0 += kMaxIterChunk) {
      const int C = std::min(kMaxIterChunk, mc - it0);
      HB_TRY(membership_build_dev(ml, w.mb, nullptr, seed + (uint32_t)it0, C, cats, w.idx, st, w.lcat,
                                  w.ckey, B, dstop));
      for (int c = 0; c < C; ++c) {
        const int it = it0 + c;
        const int32_t* idx = w.idx + (size_t)c * n;
        const int32_t* lcat = w.lcat + (size_t)c * n;
        // centroids Y = R^T Z_norm, L2-normalised (clustering.cu:272-281).  The pass walks
        // the block-ordered cell list, so it also sums every block's current rows per
        // batch: the "remove old contribution" terms of the sweep (clustering.cu:321-332).
        const size_t omsz = (size_t)(B + 1) * K;
        // the other passes add into Omin; the cell-order pass writes every entry
        bool writes_omin = false;
        if constexpr (tc_path) writes_omin = P->cen_stream;
        if (!writes_omin) HB_CUDA(cudaMemsetAsync(w.Omin, 0, sizeof(double) * nblk * omsz, st));
        int sp = span_begin(1, (double)n * (zb + rb + 8), outer, it);
        if constexpr (tc_path) {
          if (P->cen_stream) {
            CenStreamArgs ca{n, (int)((P->rows_alloc - 8) / 128), w.ckey + (size_t)c * n, d, K, P->nkeys,
                             (float*)w.Ypart, w.Opart, w.err, Yn, P->ldy, dstop, B + 1};
            HB_TRY(launch_tc_centroid_stream<S>(ca, Zn, P->ldz, R, P->ldr, P->rows_alloc, P->cen_chunks, w.Omin, st));
          } else {
            CenArgs ca{Zn, P->ldz, R, P->ldr, cats, idx, lcat, n, ml.bs, d, K, B, (float*)w.Ypart, w.Omin, w.err,
                       dstop};
            HB_TRY(launch_tc_centroid<S>(ca, P->cen_chunks, st));
          }
        } else {
          HB_TRY(launch_accum<S, S, TA>(R, P->ldr, Zn, P->ldz, idx, w.cen_chunks, P->cen_chunks, K, d,
                                        (TA*)w.Ypart, st, OminArgs{w.Omin, cats, ml.bs, B}, dstop));
        }
        bool reduced = false;  // the cell-order pass reduces its partials itself
        if constexpr (tc_path) reduced = P->cen_stream;
        if (!reduced)
          HB_TRY(launch_centroid_reduce<TA, S>((TA*)w.Ypart, P->cen_chunks, K, d, Yn, P->ldy, st, dstop));
        span_end(sp);
        // sweep the blocks (clustering.cu:308-372)
        if constexpr (tc_path) {
          sp = span_begin(0, (double)n * (zb + rb + 8), outer, it);
          sweep_stop = dstop;
          sweep_it = it;
          HB_TRY(sweep(idx, lcat, ml.bs, nblk, w.Omin, 0, w.obj_out + it));
          sweep_stop = nullptr;
          span_end(sp);
        } else {
          for (int j = 0; j < nblk; ++j) {
            BlockArgs a = base;
            const int64_t s0 = (int64_t)j * ml.bs;
            a.idx_new = idx + s0;
            a.n_new = std::min<int64_t>(ml.bs, n - s0);
            a.Om_cur = j == 0 ? w.Omin : nullptr;
            a.Om_next = j + 1 < nblk ? w.Omin + (size_t)(j + 1) * omsz : nullptr;
            a.stop = dstop;
            sp = span_begin(0, (double)a.n_new * (zb + rb + 8), outer, it);
            HB_TRY(ring.step<S>(a, st));
            span_end(sp);
          }
          HB_TRY(launch_objective_finalize(ring.state(), w.Pr, w.theta, p.sigma, B, K, p.stabilized_penalty,
                                           w.obj_acc, w.obj_out + it, st, dstop, it, p.tol_clustering));
        }
      }
    }
    // objectives, ring position, outer convergence test, error flags (on the device)
    OuterEndArgs oe{w.ctl, w.obj_out, w.objs, w.kobj, w.kiters, {w.O[0], w.O[1], w.O[2]}, outer, mc,
                    ring0, nblk, (size_t)(B + 1) * K, p.tol_harmony, w.err, w.mb.err};
    HB_TRY(launch_outer_end(oe, st));

    // ---- ridge correction (correction_batched.cu:17-130) -------------------
    if constexpr (tc_path) {
      HB_TRY(launch_tc_moments<S>(R, P->ldr, X, d, cell_index, w.m_chunks, (int)mch.size(), K, d,
                                  (float*)w.Mpart, w.err, st, ogate));
    } else {
      HB_TRY(launch_accum<S, T, TA>(R, P->ldr, X, d, cell_index, w.m_chunks, (int)mch.size(), K, d,
                                    (TA*)w.Mpart, st, OminArgs{nullptr, nullptr, 1, 1}, ogate));
    }
    HB_TRY(launch_m_reduce<TA>((TA*)w.Mpart, mch.data(), (int)mch.size(), w.batch_chunk_off, K, B, d,
                               w.M, st, ogate));
    CorrArgs ca{w.M, ring.state(), w.Pr, w.Nb, p.alpha, p.ridge_lambda, p.batch_prune_threshold,
                p.prune, p.dynamic_lambda, K, B, d};
    HB_TRY(launch_ridge_solve<T>(ca, (T*)w.W, st, ogate));
    if constexpr (tc_path) {
      HB_TRY(launch_tc_apply<S>(X, d, R, P->ldr, (const float*)w.W, cell_index, w.apply_tiles, (int)tiles.size(),
                                K, d, Zhat, d, Zn, P->ldz, w.err, st, ogate));
    } else {
      HB_TRY(launch_apply_t<T, S, S>(X, d, R, P->ldr, (T*)w.W, cell_index, w.apply_tiles,
                                     (int)tiles.size(), K, d, Zhat, d, Zn, P->ldz, st, ogate));
    }
    // the host stops enqueuing once it sees, without waiting, that an outer iteration ended the
    // run; the iterations it enqueued before that return at once on the device
    HB_CUDA(cudaMemcpyAsync(h_flag + 2 * outer, &w.ctl->ostop, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    HB_CUDA(cudaEventRecord(P->flag_events[outer], st));
    while (checked <= outer) {
      const cudaError_t q = cudaEventQuery(P->flag_events[checked]);
      if (q == cudaErrorNotReady) {
        if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
        break;
      }
      HB_CUDA(q);
      if (h_flag[2 * checked] || h_flag[2 * checked + 1]) {
        host_stop = true;
        break;
      }
      ++checked;
    }
  }
  // ---- the one read of the run ------------------------------------------------
  HB_CUDA(cudaMemcpyAsync(h_ctl, w.ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaMemcpyAsync(h_objs, w.objs, sizeof(double) * (mh + 1), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaMemcpyAsync(h_kiters, w.kiters, sizeof(int32_t) * mh, cudaMemcpyDeviceToHost, st));
  if (out && out->kmeans_objectives && mc > 0)
    HB_CUDA(cudaMemcpyAsync(h_kobj, w.kobj, sizeof(double) * mh * kstride, cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaMemcpyAsync(&h_err[0], w.mb.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaMemcpyAsync(&h_err[1], w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (h_err[0]) { set_error("block splitter candidate buffer overflow"); return HB_ERR_INTERNAL; }
  if (h_err[1] == 7) { set_error("fp16 correction: |X| or |W| reaches 65504, outside the fp16 range; use bf16"); return HB_ERR_UNSUPPORTED; }
  if (h_err[1]) { set_error("tensor-core wait timed out (code %d)", h_err[1]); return HB_ERR_TIMEOUT; }
  const int n_outer = std::min(h_ctl->n_outer, mh);
  const int converged = h_ctl->conv;
  if (prof) {
    *prof = hb_profile{};
    for (const Span& sp : spans) {
      float ms = 0.f;
      if (sp.e1 < 0) continue;
      // launches after the device-side stop returned at once: not counted
      if (sp.outer >= n_outer || sp.it >= h_kiters[sp.outer]) continue;
      HB_CUDA(cudaEventElapsedTime(&ms, P->events[sp.e0], P->events[sp.e1]));
      if (sp.cat == 0) { prof->block_launches++; prof->block_ms += ms; prof->block_bytes += sp.bytes; }
      else { prof->centroid_launches++; prof->centroid_ms += ms; prof->centroid_bytes += sp.bytes; }
    }
    prof->kernel_launches = g_launches - launches0;
  }
  if (out) {
    if (out->objectives)
      for (int i = 0; i <= n_outer; ++i) out->objectives[i] = h_objs[i];
    if (out->n_objectives) *out->n_objectives = (int32_t)(n_outer + 1);
    if (out->converged) *out->converged = converged;
    for (int o = 0; o < n_outer; ++o) {
      if (out->kmeans_iters) out->kmeans_iters[o] = h_kiters[o];
      if (out->kmeans_objectives)
        for (int i = 0; i < h_kiters[o]; ++i)
          out->kmeans_objectives[(size_t)o * mc + i] = h_kobj[(size_t)o * kstride + i];
    }
  }
  return HB_OK;
}

}  // namespace

extern "C" {

int hb_harmonize(hb_plan* plan, const void* X, const int32_t* cats, const int32_t* cell_index,
                 const int64_t* batch_offsets, const double* theta, const void* Y0, void* workspace,
                 size_t workspace_bytes, void* Z_hat, hb_outputs* out, void* stream) {
  if (!plan || !X || !cats || !batch_offsets || !theta || !Y0 || !Z_hat) {
    set_error("hb_harmonize: null argument");
    return HB_ERR_INVALID;
  }
  cudaStream_t st = (cudaStream_t)stream;
  switch (plan->p.precision) {
    case HB_FP64:
      return run_impl<double, double>(plan, (const double*)X, cats, cell_index, batch_offsets, theta,
                                      (const double*)Y0, workspace, workspace_bytes, (double*)Z_hat, out, st);
    case HB_FP16:
      return run_impl<float, __half>(plan, (const float*)X, cats, cell_index, batch_offsets, theta,
                                     (const float*)Y0, workspace, workspace_bytes, (float*)Z_hat, out, st);
    case HB_BF16:
      return run_impl<float, __nv_bfloat16>(plan, (const float*)X, cats, cell_index, batch_offsets, theta,
                                            (const float*)Y0, workspace, workspace_bytes, (float*)Z_hat, out,
                                            st);
    default:
      return run_impl<float, float>(plan, (const float*)X, cats, cell_index, batch_offsets, theta,
                                    (const float*)Y0, workspace, workspace_bytes, (float*)Z_hat, out, st);
  }
}

int hb_l2_normalize(const void* src, void* dst, int64_t rows, int32_t cols, int32_t dtype, void* stream) {
  if (rows < 0 || cols < 1) { set_error("bad shape"); return HB_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == HB_FP64) return launch_l2_normalize<double, double>((const double*)src, rows, cols, cols, (double*)dst, cols, st);
  if (dtype == HB_FP32) return launch_l2_normalize<float, float>((const float*)src, rows, cols, cols, (float*)dst, cols, st);
  set_error("hb_l2_normalize: dtype must be HB_FP32 or HB_FP64");
  return HB_ERR_INVALID;
}

size_t hb_block_lists_workspace_bytes(int64_t n, int64_t block_size, int32_t n_batches) {
  if (n < 1 || block_size < 1) return 0;
  MembershipLayout L = membership_layout(n, block_size, n_batches);
  Carver cv(nullptr, 0);
  MembershipBufs B;
  membership_carve(cv, L, B);
  return cv.off + 256;
}

int hb_block_lists(int64_t n, int64_t block_size, const uint32_t* seeds, int32_t n_iters,
                   const int32_t* cats, int32_t n_batches, int32_t* idx, void* workspace,
                   size_t workspace_bytes, void* stream) {
  if (n < 1 || block_size < 1 || !seeds || !idx || n_iters < 0) {
    set_error("hb_block_lists: bad argument");
    return HB_ERR_INVALID;
  }
  if (n_iters == 0) return HB_OK;
  MembershipLayout L = membership_layout(n, block_size, cats ? n_batches : 1);
  if (L.nblk > kMaxBlocks) { set_error("too many blocks"); return HB_ERR_UNSUPPORTED; }
  if (L.cap > 16384) { set_error("n too large"); return HB_ERR_UNSUPPORTED; }
  if (workspace_bytes < hb_block_lists_workspace_bytes(n, block_size, cats ? n_batches : 1)) {
    set_error("workspace too small");
    return HB_ERR_WORKSPACE;
  }
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  MembershipBufs B;
  membership_carve(cv, L, B);
  cudaStream_t st = (cudaStream_t)stream;
  HB_TRY(membership_clear_err(B, st));
  for (int c0 = 0; c0 < n_iters; c0 += kMaxIterChunk) {
    const int C = std::min(kMaxIterChunk, n_iters - c0);
    HB_TRY(membership_build(L, B, seeds + c0, C, cats, idx + (size_t)c0 * n, st));
  }
  int err = 0;
  HB_CUDA(cudaMemcpyAsync(&err, B.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (err) { set_error("candidate overflow"); return HB_ERR_INTERNAL; }
  return HB_OK;
}

}  // extern "C"
