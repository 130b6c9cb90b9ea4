// Exact brute-force k nearest neighbours on the tensor core: the neighbour search
// of pp.neighbors(algorithm="brute") (preprocessing/_neighbors/_algorithms/_brute.py:14,
// a cuML NearestNeighbors(algorithm="brute") call in the reference).
//
//   k_knn_prep    per row: (for cosine) L2 normalisation, the squared norm in float32,
//                 and bf16 hi + lo parts of the row (x = hi + lo to ~16 significant bits)
//   k_knn_search  one CTA per 128-query tile: for every 128-row tile of the data,
//                 D = Q . X^T on tcgen05 as hi.hi + hi.lo + lo.hi with the float32
//                 accumulator in TMEM; the epilogue turns the dot products into distances
//                 (|q|^2 + |x|^2 - 2 q.x, or -q.x for cosine / inner product) and keeps each
//                 thread's KC best candidates (half of a query's columns per thread) in a
//                 sorted list in shared memory.  The next data tile is loaded while the
//                 epilogue runs.  At the end each query's 2 KC candidates are re-ranked
//                 with exact float32 distances computed from the original rows (the
//                 difference form for euclidean, so a point's distance to itself is 0).
#include "hb_tc_tile.cuh"
#include "../../include/harmony_b200.h"

namespace hb {
namespace {

constexpr int kKnnEuclid = HB_KNN_EUCLIDEAN, kKnnCosine = HB_KNN_COSINE, kKnnInner = HB_KNN_INNER_PRODUCT;

// row of X (float32) -> normalised copy (cosine), squared norm, bf16 hi / lo (zero padded)
__global__ void k_knn_prep(const float* __restrict__ X, int64_t n, int d, int dpad, int cosine,
                           __nv_bfloat16* __restrict__ Xh, __nv_bfloat16* __restrict__ Xl, float* __restrict__ nrm,
                           float* __restrict__ Xn, int64_t npad) {
  const int lane = threadIdx.x & 31;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < npad;
       row += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    float ss = 0.f;
    if (row < n)
      for (int c = lane; c < d; c += 32) {
        const float x = X[row * d + c];
        ss = fmaf(x, x, ss);
      }
    ss = warp_sum(ss);
    const float scale = (cosine && row < n) ? 1.f / fmaxf(sqrtf(ss), 1e-30f) : 1.f;
    for (int c = lane; c < dpad; c += 32) {
      const float x = (row < n && c < d) ? X[row * d + c] * scale : 0.f;
      if (cosine && row < n && c < d) Xn[row * d + c] = x;
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      Xh[row * dpad + c] = h;
      Xl[row * dpad + c] = __float2bfloat16_rn(x - __bfloat162float(h));
    }
    if (lane == 0) nrm[row] = row < n ? (cosine ? 1.f : ss) : 0.f;
  }
}

struct KnnArgs {
  const float* Q;        // queries (float32 [nq][d]; the normalised copy for cosine)
  const float* X;        // data
  const __nv_bfloat16 *Qh, *Ql, *Xh, *Xl;
  const float *qn, *xn;  // squared norms
  int64_t nq, nx;
  int d, dpad, k, metric;
  int64_t* idx_out;      // [nq][k]
  float* dist_out;       // [nq][k]
  int* err;
};

// insert (dist, id) into a list sorted ascending, list entry i of this thread at [i * 256]
template <int KC>
__device__ __forceinline__ void list_insert(float* ld, int* li, float dist, int id, float& thr) {
  int p = KC - 1;
  while (p > 0 && ld[(p - 1) * 256] > dist) {
    ld[p * 256] = ld[(p - 1) * 256];
    li[p * 256] = li[(p - 1) * 256];
    --p;
  }
  ld[p * 256] = dist;
  li[p * 256] = id;
  thr = ld[(KC - 1) * 256];
}

// NB = 2: two data-tile buffers and two TMEM accumulators, so the MMA of data tile t+1 runs
// while the epilogue of tile t reads its dot products (and tile t+2 loads); NB = 1 when shared
// memory holds one data tile only (128 dimensions, or the 64-entry candidate lists).
template <int KC, int NB>
__global__ void __launch_bounds__(256, 1) k_knn_search(KnnArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kblk = a.dpad / 64;
  const uint32_t atile = (uint32_t)kblk * 16384u;   // 128 rows x dpad bf16
  const uint32_t oAh = 0, oAl = atile, oB = 2 * atile;  // data buffer b: hi at oB + 2 b atile, lo after
  const uint32_t oNrm = oB + 2u * NB * atile;        // [4][128] data-tile norms (tile t in slot t & 3)
  const uint32_t oLd = oNrm + 2048, oLi = oLd + (uint32_t)KC * 256u * 4u;
  const uint32_t oSt = oLi + (uint32_t)KC * 256u * 4u;  // [8][256] staged distances, then ids
  const uint32_t oMisc = oSt + 8u * 256u * 8u;
  float* nrm_s = (float*)(sm + oNrm);
  float* ld = (float*)(sm + oLd) + tid;
  int* li = (int*)(sm + oLi) + tid;
  float* sd = (float*)(sm + oSt) + tid;
  int* si = (int*)(sm + oSt + 8u * 256u * 4u) + tid;
  uint64_t* mbar = (uint64_t*)(sm + oMisc);          // [NB]
  uint32_t* tmem_slot = (uint32_t*)(sm + oMisc + 16);
  const uint32_t sm32 = tc::smem_u32(sm);
  const int64_t q0 = (int64_t)blockIdx.x * 128;
  const int64_t ntiles = (a.nx + 127) / 128;
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, 128u * NB);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    for (int b = 0; b < NB; ++b) tc::mbar_init(mbar + b, 1);
    tc::fence_mbar_init();
  }
  // rows of dpad bf16, K-major, 128B swizzle; rows are padded to whole tiles
  const int nch = a.dpad / 8;
  auto load_rows = [&](uint32_t dst_h, uint32_t dst_l, const __nv_bfloat16* Sh, const __nv_bfloat16* Sl,
                       int64_t r0) {
    for (int e = tid; e < 128 * nch; e += 256) {
      const int r = e / nch, ch = e % nch;
      const uint32_t off = (uint32_t)(ch >> 3) * 16384u + tc::sw128_off((uint32_t)r, (uint32_t)(ch & 7));
      const size_t src = (size_t)(r0 + r) * a.dpad + ch * 8;
      tc::cp_async16(sm32 + dst_h + off, Sh + src, 16u);
      tc::cp_async16(sm32 + dst_l + off, Sl + src, 16u);
    }
  };
  auto load_tile = [&](int64_t tt) {  // data tile tt into buffer tt % NB, its norms into slot tt & 3
    const uint32_t bh = oB + 2u * (uint32_t)(tt % NB) * atile;
    load_rows(bh, bh + atile, a.Xh, a.Xl, tt * 128);
    if (tid < 128) nrm_s[(tt & 3) * 128 + tid] = a.xn[tt * 128 + tid];
  };
  load_rows(oAh, oAl, a.Qh, a.Ql, q0);
  load_tile(0);
  if (NB == 2 && ntiles > 1) load_tile(1);
  for (int i = 0; i < KC; ++i) {
    ld[i * 256] = INFINITY;
    li[i * 256] = -1;
  }
  float thr = INFINITY;
  tc::cp_async_wait_all();
  tc::fence_proxy_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc::idesc_f16(128, 128, true, false, false);
  auto issue = [&](int64_t tt) {  // thread 0: D[b] = Q . X_tile^T, three hi / lo products
    const int b = (int)(tt % NB);
    const uint32_t bh = sm32 + oB + 2u * (uint32_t)b * atile;
    const int nks = a.dpad / 16;
    for (int s = 0; s < nks; ++s) {
      const uint32_t o = (uint32_t)(s >> 2) * 16384u + (uint32_t)(s & 3) * 32u;
      const uint64_t ah = tc::sdesc_sw128(sm32 + oAh + o, 16, 1024), al = tc::sdesc_sw128(sm32 + oAl + o, 16, 1024);
      const uint64_t xh = tc::sdesc_sw128(bh + o, 16, 1024), xl = tc::sdesc_sw128(bh + atile + o, 16, 1024);
      const uint32_t d = tmem + (uint32_t)(b * 128);
      tc::mma_f16(d, ah, xh, idesc, s > 0 ? 1u : 0u);
      tc::mma_f16(d, ah, xl, idesc, 1u);
      tc::mma_f16(d, al, xh, idesc, 1u);
    }
    tc::mma_commit(mbar + b);
  };
  auto join = [&]() {  // loads landed, the epilogue's TMEM reads done, then the next MMA may run
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  };
  const int row = (warp & 3) * 32 + lane, half = warp >> 2;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(half * 64);
  const int64_t q = q0 + row;
  const bool live = q < a.nq;
  const float qnorm = live ? a.qn[q] : 0.f;
  const bool dot_metric = a.metric == kKnnCosine || a.metric == kKnnInner;
  if (tid == 0) issue(0);
  for (int64_t t = 0; t < ntiles; ++t) {
    const int b = (int)(t % NB);
    if (!tc::mbar_wait(mbar + b, (uint32_t)((t / NB) & 1), kMaxPolls)) atomicExch(a.err, 8);
    tc::fence_after_sync();
    if (NB == 2) {
      if (t + 1 < ntiles) {  // its operands loaded during the previous epilogue: start its MMA
        join();
        if (tid == 0) issue(t + 1);
      }
      if (t + 2 < ntiles) load_tile(t + 2);  // into the buffer tile t has finished with
    } else if (t + 1 < ntiles) {
      load_tile(t + 1);
    }
    // epilogue: the thread's 64 columns in one wait (tcgen05.ld is warp-collective: every lane
    // loads, lanes past the last query skip the lists)
    float v[8][8];
#pragma unroll
    for (int c = 0; c < 8; ++c) tc::tmem_ld8(tl + (uint32_t)(b * 128 + 8 * c), v[c]);
    tc::tmem_ld_wait();
    // fast pass, eight candidates at a time: the ones below the thread's threshold are staged
    // (no branch); the sorted lists are only touched when some lane of the warp staged one
    {
      const float* nr = nrm_s + (t & 3) * 128 + half * 64;
      const int base = (int)(t * 128) + half * 64;
      const int nvalid = (int)min((int64_t)64, a.nx - (int64_t)base);  // candidates of this half
      // dist < thr  <=>  key < thr - |q|^2 with key = |x|^2 - 2 q.x (euclidean), -q.x (dot)
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float4 n0 = *(const float4*)(nr + 8 * c), n1 = *(const float4*)(nr + 8 * c + 4);
        const float nn[8] = {n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, n1.z, n1.w};
        const float lim = dot_metric ? thr : thr - qnorm;
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float key = dot_metric ? -v[c][i] : fmaf(-2.f, v[c][i], nn[i]);
          const bool take = live && key < lim && 8 * c + i < nvalid;
          if (take) {
            sd[cnt * 256] = dot_metric ? key : key + qnorm;
            si[cnt * 256] = base + 8 * c + i;
          }
          cnt += take ? 1 : 0;
        }
        if (__any_sync(0xffffffffu, cnt > 0))
          for (int e = 0; e < cnt; ++e) {
            const float dd = sd[e * 256];
            if (dd < thr) list_insert<KC>(ld, li, dd, si[e * 256], thr);
          }
      }
    }
    tc::fence_before_sync();
    if (NB == 1 && t + 1 < ntiles) {
      join();
      if (tid == 0) issue(t + 1);
    }
  }
  __syncthreads();
  // exact re-rank: thread `row` (half 0) takes both halves' candidates of its query
  if (half == 0 && live) {
    float bd[64];
    int bi[64];
    const int kk = a.k;
    for (int i = 0; i < kk; ++i) {
      bd[i] = INFINITY;
      bi[i] = -1;
    }
    const float* qrow = a.Q + q * a.d;
    for (int h = 0; h < 2; ++h) {
      const int* ci = (const int*)(sm + oLi) + h * 128 + row;
      for (int i = 0; i < KC; ++i) {
        const int id = ci[i * 256];
        if (id < 0) continue;
        const float* xr = a.X + (int64_t)id * a.d;
        float acc = 0.f;
        if (dot_metric) {
          for (int c = 0; c < a.d; ++c) acc = fmaf(qrow[c], xr[c], acc);
          acc = a.metric == kKnnCosine ? 1.f - acc : -acc;
        } else {
          for (int c = 0; c < a.d; ++c) {
            const float df = qrow[c] - xr[c];
            acc = fmaf(df, df, acc);
          }
        }
        // insert by (distance, index) ascending into the k best
        if (acc < bd[kk - 1] || (acc == bd[kk - 1] && id < bi[kk - 1])) {
          int p = kk - 1;
          while (p > 0 && (bd[p - 1] > acc || (bd[p - 1] == acc && bi[p - 1] > id))) {
            bd[p] = bd[p - 1];
            bi[p] = bi[p - 1];
            --p;
          }
          bd[p] = acc;
          bi[p] = id;
        }
      }
    }
    for (int i = 0; i < kk; ++i) {
      float out = bd[i];
      if (a.metric == kKnnEuclid) out = sqrtf(fmaxf(out, 0.f));
      else if (a.metric == kKnnInner) out = -out;
      a.idx_out[q * kk + i] = bi[i];
      a.dist_out[q * kk + i] = out;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 128u * NB);
  }
}

struct KnnPlan {
  int dpad;
  int64_t nqpad, nxpad;
  size_t bytes;
};

KnnPlan knn_plan(int64_t nq, int64_t nx, int d, bool same, bool cosine) {
  KnnPlan P{};
  P.dpad = d <= 64 ? 64 : 128;
  P.nqpad = (nq + 127) / 128 * 128;
  P.nxpad = (nx + 127) / 128 * 128;
  size_t b = 0;
  auto add = [&](size_t x) { b += align_up(x, 256); };
  add((size_t)P.nxpad * P.dpad * 2);  // Xh
  add((size_t)P.nxpad * P.dpad * 2);  // Xl
  add((size_t)P.nxpad * 4);           // norms
  if (cosine) add((size_t)nx * d * 4);  // normalised data
  if (!same) {
    add((size_t)P.nqpad * P.dpad * 2);
    add((size_t)P.nqpad * P.dpad * 2);
    add((size_t)P.nqpad * 4);
    if (cosine) add((size_t)nq * d * 4);
  }
  add(16);  // error flag
  P.bytes = b + 256;
  return P;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

HB_API size_t hb_knn_workspace_bytes(int64_t n_queries, int64_t n_data, int32_t n_dims, int32_t same, int32_t metric) {
  if (n_queries < 1 || n_data < 1 || n_dims < 1) return 0;
  return knn_plan(n_queries, n_data, n_dims, same != 0, metric == HB_KNN_COSINE).bytes;
}

HB_API int hb_knn(const float* queries, int64_t n_queries, const float* data, int64_t n_data, int32_t n_dims,
                  int32_t k, int32_t metric, int64_t* indices, float* distances, void* workspace,
                  size_t workspace_bytes, void* stream) {
  if (!queries || !data || !indices || !distances || n_queries < 1 || n_data < 1 || n_dims < 1 || k < 1 ||
      metric < HB_KNN_SQEUCLIDEAN || metric > HB_KNN_INNER_PRODUCT) {
    set_error("hb_knn: bad argument");
    return HB_ERR_INVALID;
  }
  if (k > n_data) {
    set_error("hb_knn: k=%d exceeds the %lld data points", k, (long long)n_data);
    return HB_ERR_INVALID;
  }
  if (n_dims > 128 || k > 56 || n_data > 2147483647LL || (k > 24 && n_dims > 64)) {
    set_error("hb_knn: unsupported shape (n_dims <= 128, k <= 56 and k <= 24 above 64 dims)");
    return HB_ERR_UNSUPPORTED;
  }
  const bool same = queries == data && n_queries == n_data;
  const bool cosine = metric == HB_KNN_COSINE;
  const KnnPlan P = knn_plan(n_queries, n_data, n_dims, same, cosine);
  if (!workspace || workspace_bytes < P.bytes) {
    set_error("hb_knn: workspace too small (%zu < %zu)", workspace_bytes, P.bytes);
    return HB_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  __nv_bfloat16* Xh = cv.take<__nv_bfloat16>((size_t)P.nxpad * P.dpad);
  __nv_bfloat16* Xl = cv.take<__nv_bfloat16>((size_t)P.nxpad * P.dpad);
  float* xn = cv.take<float>((size_t)P.nxpad);
  float* Xc = cosine ? cv.take<float>((size_t)n_data * n_dims) : nullptr;
  __nv_bfloat16 *Qh = Xh, *Ql = Xl;
  float *qn = xn, *Qc = Xc;
  if (!same) {
    Qh = cv.take<__nv_bfloat16>((size_t)P.nqpad * P.dpad);
    Ql = cv.take<__nv_bfloat16>((size_t)P.nqpad * P.dpad);
    qn = cv.take<float>((size_t)P.nqpad);
    Qc = cosine ? cv.take<float>((size_t)n_queries * n_dims) : nullptr;
  }
  int* err = cv.take<int>(4);
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  const int sms = num_sms();
  k_knn_prep<<<(unsigned)std::min<int64_t>((P.nxpad * 32 + 255) / 256, 16 * sms), 256, 0, st>>>(
      data, n_data, n_dims, P.dpad, cosine, Xh, Xl, xn, Xc, P.nxpad);
  HB_LAUNCH_CHECK();
  if (!same) {
    k_knn_prep<<<(unsigned)std::min<int64_t>((P.nqpad * 32 + 255) / 256, 16 * sms), 256, 0, st>>>(
        queries, n_queries, n_dims, P.dpad, cosine, Qh, Ql, qn, Qc, P.nqpad);
    HB_LAUNCH_CHECK();
  }
  KnnArgs a{cosine ? Qc : queries, cosine ? Xc : data, Qh, Ql, Xh, Xl, qn, xn, n_queries, n_data, n_dims,
            P.dpad, k, metric, indices, distances, err};
  const int KC = k <= 24 ? 32 : 64;
  const int NB = (KC == 32 && P.dpad == 64) ? 2 : 1;  // two data tiles fit beside the 32-entry lists
  const uint32_t atile = (uint32_t)(P.dpad / 64) * 16384u;
  const size_t smem = (2 + 2 * (size_t)NB) * atile + 2048 + 2 * (size_t)KC * 256 * 4 + 8 * 256 * 8 + 64 + 1024;
  const unsigned grid = (unsigned)((n_queries + 127) / 128);
  const void* fn = KC == 64 ? (const void*)k_knn_search<64, 1>
                            : (NB == 2 ? (const void*)k_knn_search<32, 2> : (const void*)k_knn_search<32, 1>);
  HB_TRY(allow_max_dyn_smem(fn));
  if (KC == 64) k_knn_search<64, 1><<<grid, 256, smem, st>>>(a);
  else if (NB == 2) k_knn_search<32, 2><<<grid, 256, smem, st>>>(a);
  else k_knn_search<32, 1><<<grid, 256, smem, st>>>(a);
  HB_LAUNCH_CHECK();
  int h_err = 0;
  HB_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (h_err) {
    set_error("hb_knn: tensor-core wait timed out (code %d)", h_err);
    return HB_ERR_TIMEOUT;
  }
  return HB_OK;
}

}  // extern "C"
