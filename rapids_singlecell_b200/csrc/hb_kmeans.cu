// Seeded k-means initialisation of the Harmony centroids on the GPU.
//
// The reference starts Harmony from cuML's KMeans (init="k-means||", n_init=1,
// max_iter=25, random_state) fitted on the L2-normalised embedding, and then
// L2-normalises the centres (preprocessing/_harmony/__init__.py:290-323).  cuML
// is a third-party library whose random streams cannot be reproduced here; this
// is the engine's own seeded k-means in the same role, with the same iteration
// budget:
//   seeding  k-means++ (Arthur & Vassilvitskii, 2007: each new centre is drawn
//            with probability proportional to the squared distance to the
//            nearest centre chosen so far) over a sample of m cells (all cells
//            when n <= m, else m draws with replacement), in float64 with
//            explicitly rounded operations in a fixed order (one thread per sample
//            for the distances, one CTA for each draw); the draws come from
//            splitmix64 (Steele, Lea & Flood, 2014) of (seed, counter), so a seed
//            fixes the result bit for bit;
//   Lloyd    up to max_iter iterations over all cells: the assignment is the
//            tensor-core similarity of a 128-cell tile of bf16 Z_norm against the
//            bf16 centres (fp32 in TMEM), argmax_k (z.y_k - |y_k|^2 / 2), which is
//            the nearest centre for unit rows; the tile's rows are added to their
//            centre's sum by a second MMA (Z_tile^T times the one-hot of the labels,
//            accumulated in TMEM); the per-CTA sums are reduced per centre in float64,
//            and a centre that lost all its cells keeps its position.
//            Stops when |Y_new - Y_old|_F <= tol |Y_new|_F.
#include "hb_tc_tile.cuh"

namespace hb {

// ---- counter-based draws ------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// draw `ctr` of stream `seed`
__host__ __device__ __forceinline__ uint64_t km_draw(uint64_t seed, uint64_t ctr) {
  return splitmix64(splitmix64(seed) ^ ctr);
}
// uniform in [0, 1) from the top 53 bits
__host__ __device__ __forceinline__ double km_u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

// counters: draw 0 picks the first centre, draw 1 + r the centre of round r, draw
// kSampleBase + j the j-th sampled cell
constexpr uint64_t kSampleBase = 1ull << 40;
constexpr int kSeedThreads = 1024;

// k-means++ over the sample, in three kernels with the sample rows column-major in S
// [d][m] (float64), so that the per-sample loops of a warp read consecutive addresses.
// The arithmetic is fixed for reproducibility: sums over columns in column order, the
// 1024 chunks of ceil(m / 1024) consecutive samples each summed in order, then the chunk
// sums in order.

// S[:, j] = the L2-normalised row of sampled cell j (inverse norm capped at 1e12,
// kernels_normalize.cuh:7-54); every cell in order when m == n.
__global__ void __launch_bounds__(256) k_km_sample(const float* __restrict__ X, int64_t n, int d, int m,
                                                  uint64_t seed, double* __restrict__ S) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int64_t cell = (int64_t)m == n ? j : (int64_t)(km_draw(seed, kSampleBase + (uint64_t)j) % (uint64_t)n);
  const float* x = X + cell * d;
  double ss = 0.0;
  for (int c = 0; c < d; ++c) ss = __dadd_rn(ss, __dmul_rn((double)x[c], (double)x[c]));
  double inv = __ddiv_rn(1.0, __dsqrt_rn(ss));
  if (!(inv <= 1e12)) inv = 1e12;
  for (int c = 0; c < d; ++c) S[(size_t)c * m + j] = __dmul_rn((double)x[c], inv);
}

// D2[j] = squared distance of sample j to the last chosen centre (sample *pick), or the
// smaller of that and D2[j] after the first centre.
__global__ void __launch_bounds__(256) k_km_dist(const double* __restrict__ S, int m, int d,
                                                const int* __restrict__ pick, int first, double* __restrict__ D2) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int p = *pick;
  double acc = 0.0;
  for (int c = 0; c < d; ++c) {
    const double df = __dsub_rn(S[(size_t)c * m + j], S[(size_t)c * m + p]);
    acc = __dadd_rn(acc, __dmul_rn(df, df));
  }
  D2[j] = first ? acc : fmin(D2[j], acc);
}

// Centre r: sample draw(seed, 0) % m for r = 0, else the sample at which the running sum
// of D2 first exceeds u * total (u from draw(seed, 1 + r)); a uniform draw when every
// sample sits on a chosen centre.  Writes *pick and Y[r] (float32).
__global__ void __launch_bounds__(kSeedThreads) k_km_pick(const double* __restrict__ S, const double* __restrict__ D2,
                                                         int m, int d, int r, uint64_t seed, int* __restrict__ pick,
                                                         float* __restrict__ Y) {
  __shared__ double part[kSeedThreads];  // chunk sums, then their exclusive prefix
  __shared__ double total;
  __shared__ int sel;
  const int t = threadIdx.x;
  if (r == 0) {
    if (t == 0) sel = (int)(km_draw(seed, 0) % (uint64_t)m);
  } else {
    const int ch = (m + kSeedThreads - 1) / kSeedThreads;
    const int j0 = min(m, t * ch), j1 = min(m, (t + 1) * ch);
    double local = 0.0;
    for (int j = j0; j < j1; ++j) local = __dadd_rn(local, D2[j]);
    part[t] = local;
    __syncthreads();
    if (t == 0) {  // exclusive prefix over the chunks, in order
      double run = 0.0;
      for (int q = 0; q < kSeedThreads; ++q) {
        const double v = part[q];
        part[q] = run;
        run = __dadd_rn(run, v);
      }
      total = run;
      sel = -1;
    }
    __syncthreads();
    const uint64_t h = km_draw(seed, 1 + (uint64_t)r);
    if (!(total > 0.0)) {  // every sample sits on a chosen centre: a uniform pick
      if (t == 0) sel = (int)(h % (uint64_t)m);
    } else {
      const double target = __dmul_rn(km_u01(h), total);
      const double lo = part[t], hi = t + 1 < kSeedThreads ? part[t + 1] : total;
      if (lo <= target && target < hi) {
        double acc = lo;
        int got = -1, last = -1;
        for (int j = j0; j < j1; ++j) {
          if (D2[j] > 0.0) last = j;
          acc = __dadd_rn(acc, D2[j]);
          if (target < acc) {
            got = j;
            break;
          }
        }
        sel = got >= 0 ? got : last;  // rounding left the target past the chunk's last sum
      }
    }
    __syncthreads();
    if (t == 0 && sel < 0) {  // the product rounded up to the total: the last sample with weight
      for (int j = m - 1; j >= 0 && sel < 0; --j)
        if (D2[j] > 0.0) sel = j;
      if (sel < 0) sel = 0;
    }
  }
  __syncthreads();
  const int p = sel;
  for (int c = t; c < d; c += kSeedThreads) Y[(size_t)r * d + c] = (float)S[(size_t)c * m + p];
  if (t == 0) *pick = p;
}

// ---- Lloyd iterations ------------------------------------------------------------------
// Shared memory of the assignment kernel: two 128-cell bf16 tiles (the next tile's rows
// are gathered while the current one is assigned), the resident centres, the one-hot
// operand of the tile's labels, the half squared norms, per-row choices and counts.
// TMEM: the similarity tile (L.tcols columns) and the CTA's centre sums (npad columns).
struct KmLayout {
  TcLayout t;     // similarity tile geometry (dpad, kblk, npad, tcols)
  int nbK;        // 64-cluster blocks of the one-hot operand
  int nM;         // 128-PC row blocks of the centre sums (M = 128 per MMA): 2 above 128 PCs
  int nbufA;      // tile buffers: 2, or 1 above 128 PCs (the 64 KB tiles)
  int tcols_all;  // TMEM columns allocated
  uint32_t offA, offB, offH, offHn, offCnt, offBest, offRows, offMisc, bytes;
};

inline KmLayout km_layout(int d, int K) {
  KmLayout L{};
  L.t.dpad = d <= 64 ? 64 : (d <= 128 ? 128 : 256);
  L.t.kblk = L.t.dpad / 64;
  L.t.npad = (K + 15) / 16 * 16;
  L.t.tcols = L.t.npad <= 128 ? 128 : 256;
  L.nbK = (L.t.npad + 63) / 64;
  L.nM = L.t.dpad > 128 ? 2 : 1;
  L.nbufA = L.t.dpad > 128 ? 1 : 2;
  int t = 32;
  while (t < (1 + L.nM) * L.t.tcols) t <<= 1;
  L.tcols_all = t;
  auto al = [](uint32_t x, uint32_t a) { return (x + a - 1) / a * a; };
  uint32_t o = 0;
  L.offA = o; o += (uint32_t)L.nbufA * (uint32_t)L.t.kblk * 16384u;
  L.offB = o; o += (uint32_t)L.t.kblk * (uint32_t)L.t.npad * 128u;
  L.offH = al(o, 1024); o = L.offH + (uint32_t)L.nbK * 16384u;
  L.offHn = al(o, 16); o = L.offHn + (uint32_t)L.t.npad * 4u;
  L.offCnt = al(o, 16); o = L.offCnt + (uint32_t)L.t.npad * 4u;
  L.offBest = o; o += 2u * 128u * 8u;  // value and index per (half, row)
  L.offRows = o; o += 4u * 128u * 4u;  // cell id and (unused) batch per row, per tile buffer
  L.offMisc = al(o, 16); o = L.offMisc + 64u;
  L.bytes = o + 1024u;  // slack for the 1024-byte alignment of the base
  return L;
}

// One Lloyd assignment pass over the CTA's tiles: label = argmax_k (z . y_k - hn_k) of every
// cell (lowest k on ties); the CTA's sums P[cta][k][:] of its cells' bf16 rows and counts
// C[cta][k].  The sums are a second MMA per tile, D[c][k] += sum_r Z[r][c] H[r][k] with H
// the one-hot of the tile's labels, accumulated in TMEM: A = Z_tile^T is the gathered tile
// read MN-major (64-value blocks 16 KB apart, 8-cell groups 1 KB apart); M = 128 always
// (with 64 PCs the upper rows read the next buffer and are discarded).
template <typename H>
__global__ void __launch_bounds__(256, 1) k_km_assign(const H* __restrict__ Zh, int ldz, const H* __restrict__ Yh,
                                                      int ldy, const float* __restrict__ hn, int64_t n, int K, int d,
                                                      KmLayout KL, float* __restrict__ P, float* __restrict__ C,
                                                      int* err) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const TcLayout& L = KL.t;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* hns = (float*)(sm + KL.offHn);
  int* cnt = (int*)(sm + KL.offCnt);
  float* bestv = (float*)(sm + KL.offBest);  // [2][128]
  int* besti = (int*)(bestv + 256);          // [2][128]
  int* cid = (int*)(sm + KL.offRows);        // [2][128]
  int* ccat = cid + 256;                     // [2][128]
  uint64_t* mbar = (uint64_t*)(sm + KL.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + KL.offMisc + 8);
  unsigned char* oh = sm + KL.offH;
  const uint32_t atile = (uint32_t)L.kblk * 16384u;
  const uint32_t sA0 = tc::smem_u32(sm + KL.offA), sB = tc::smem_u32(sm + KL.offB), sH = tc::smem_u32(oh);
  const int nbK = KL.nbK;
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)KL.tcols_all);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  load_centroids_swizzled(Yh, ldy, K, sB, L);
  for (int k = tid; k < L.npad; k += 256) {
    hns[k] = k < K ? hn[k] : 0.f;
    cnt[k] = 0;
  }
  for (uint32_t e = (uint32_t)tid * 16u; e < (uint32_t)nbK * 16384u; e += 256u * 16u)
    *(uint4*)(oh + e) = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  // centre sums: lane = PC (128-PC block mb at tacc + mb * tcols), column = cluster
  const uint32_t tacc = tmem + (uint32_t)L.tcols;
  const int64_t ntiles = (n + 127) / 128;
  const uint32_t idesc1 = tc::idesc_f16(128, L.npad, is_bf16<H>::value, false, false);
  const uint32_t idesc2 = tc::idesc_f16(128, L.npad, is_bf16<H>::value, true, true);
  const int half = warp >> 2, row = (warp & 3) * 32 + lane;
  const int nh = (L.npad / 2 + 7) / 8 * 8;
  const int c_lo = half * nh, c_hi = min(L.npad, c_lo + nh);
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  // one-hot element (cell r, cluster k): MN-major [8-cell group][64-cluster block][8 x 128 B]
  auto oh_off = [&](int r, int k) -> uint32_t {
    return (uint32_t)(r >> 3) * (uint32_t)nbK * 1024u + (uint32_t)(k >> 6) * 1024u + (uint32_t)(r & 7) * 128u +
           ((((uint32_t)(k & 63) >> 3) ^ (uint32_t)(r & 7)) << 4) + (uint32_t)(k & 7) * 2u;
  };
  const H one = from_f<H>(1.f), zero = from_f<H>(0.f);
  int old_lab = -1;  // the one-hot entry this thread's row set (threads < 128)
  uint32_t phase = 0;
  if ((int64_t)blockIdx.x < ntiles) gather_rows_swizzled(Zh, ldz, nullptr, 0, n, blockIdx.x, sA0, L, cid, ccat, nullptr);
  int buf = 0, it = 0;
  const int bstep = KL.nbufA == 2 ? 1 : 0;  // with one tile buffer the next tile waits for this one's sums
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, buf ^= bstep, ++it) {
    tc::cp_async_wait_all();  // this tile's rows have landed
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) issue_similarity_mma(tmem, sA0 + (uint32_t)buf * atile, sB, L, idesc1, mbar);
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(err, 9);
    phase ^= 1u;
    tc::fence_after_sync();
    // the commit also covers the previous tile's sum MMA: its tile buffer and the one-hot
    // are free; the next tile's rows land while this one is assigned
    const int64_t nxt = tile + gridDim.x;
    if (KL.nbufA == 2 && nxt < ntiles)
      gather_rows_swizzled(Zh, ldz, nullptr, 0, n, nxt, sA0 + (uint32_t)(buf ^ 1) * atile, L, cid + (buf ^ 1) * 128,
                           ccat + (buf ^ 1) * 128, nullptr);
    float best = -INFINITY;
    int bi = 0;
    for (int c = c_lo; c < c_hi; c += 8) {
      float v[8];
      tc::tmem_ld8(tl + (uint32_t)c, v);
      tc::tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = c + i;
        if (k < K) {
          const float s = v[i] - hns[k];
          if (s > best) {
            best = s;
            bi = k;
          }
        }
      }
    }
    bestv[half * 128 + row] = best;
    besti[half * 128 + row] = bi;
    tc::fence_before_sync();
    __syncthreads();
    const int nvalid = (int)(n - tile * 128 < 128 ? n - tile * 128 : 128);
    if (tid < 128) {  // this row's one-hot entry and count
      if (old_lab >= 0) *(H*)(oh + oh_off(tid, old_lab)) = zero;
      old_lab = -1;
      if (tid < nvalid) {
        const int l = bestv[128 + tid] > bestv[tid] ? besti[128 + tid] : besti[tid];
        *(H*)(oh + oh_off(tid, l)) = one;
        atomicAdd(&cnt[l], 1);
        old_lab = l;
      }
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t sA = sA0 + (uint32_t)buf * atile;
      for (int mb = 0; mb < KL.nM; ++mb) {  // 128 PCs (two 64-value blocks) per MMA row block
        for (int k = 0; k < 8; ++k) {  // 8 steps of 16 cells
          const uint64_t ad = tc::sdesc_sw128(sA + (uint32_t)mb * 32768u + (uint32_t)k * 2048u, 16384u, 1024u);
          const uint64_t bd =
              tc::sdesc_sw128(sH + (uint32_t)k * 2u * (uint32_t)nbK * 1024u, 1024u, (uint32_t)nbK * 1024u);
          tc::mma_f16(tacc + (uint32_t)(mb * L.tcols), ad, bd, idesc2, (it > 0 || k > 0) ? 1u : 0u);
        }
      }
      if (KL.nbufA == 1) tc::mma_commit(mbar);
    }
    if (KL.nbufA == 1) {
      // one tile buffer: the next tile's rows are gathered once this tile's sums have read it
      if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(err, 9);
      phase ^= 1u;
      tc::fence_after_sync();
      if (tile + gridDim.x < ntiles)
        gather_rows_swizzled(Zh, ldz, nullptr, 0, n, tile + gridDim.x, sA0, L, cid, ccat, nullptr);
    }
  }
  // the sums out of TMEM: warp w reads PCs 128 mb + 32 (w % 4) .. + 31, its half of the clusters
  if (it > 0) {
    if (tid == 0) tc::mma_commit(mbar);
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(err, 9);
    tc::fence_after_sync();
  }
  for (int mb = 0; mb < KL.nM; ++mb) {
    const int c = mb * 128 + (warp & 3) * 32 + lane;
    const uint32_t ta = tacc + (uint32_t)(mb * L.tcols) + ((uint32_t)((warp & 3) * 32) << 16);
    float* out = P + (size_t)blockIdx.x * K * d;
    for (int k0 = c_lo; k0 < c_hi; k0 += 8) {
      float v[8];
      tc::tmem_ld8(ta + (uint32_t)k0, v);
      tc::tmem_ld_wait();
      if (c < d)
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (k0 + i < K) out[(size_t)(k0 + i) * d + c] = it > 0 ? v[i] : 0.f;
    }
  }
  for (int k = tid; k < K; k += 256) C[(size_t)blockIdx.x * K + k] = (float)cnt[k];
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)KL.tcols_all);
  }
}

// New centre k = blockIdx.x: the mean of its cells over the G CTA partials (float64),
// or the old centre when it has none; writes the float32 centre, its bf16 copy (zero
// padded to ldy), hn_k = |bf16 centre|^2 / 2, and adds |shift|^2 and |new|^2 to shift[0..1].
// With G = 0 it only derives the bf16 copy and hn from the current centres.
template <typename H>
__global__ void __launch_bounds__(256) k_km_update(const float* __restrict__ P, const float* __restrict__ C, int G,
                                                   int K, int d, float* __restrict__ Yf, H* __restrict__ Yh, int ldy,
                                                   float* __restrict__ hn, double* __restrict__ shift) {
  __shared__ double part[8][256];
  __shared__ double cpart[8];
  __shared__ double red[32];
  const int lane = threadIdx.x, y = threadIdx.y, t = y * 32 + lane;
  const int k = blockIdx.x;
  for (int c = lane; c < d; c += 32) {  // d <= 256
    double s = 0.0;
#pragma unroll 8
    for (int g = y; g < G; g += 8) s += (double)__ldg(P + ((size_t)g * K + k) * d + c);
    part[y][c] = s;
  }
  if (lane == 0) {
    double cn = 0.0;
    for (int g = y; g < G; g += 8) cn += (double)__ldg(C + (size_t)g * K + k);
    cpart[y] = cn;
  }
  __syncthreads();
  double count = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) count += cpart[q];
  double dsh = 0.0, nrm = 0.0, hsq = 0.0;
  if (t < d) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += part[q][t];
    const double yold = (double)Yf[(size_t)k * d + t];
    const float yf = count > 0.0 ? (float)(s / count) : (float)yold;
    const H yh = from_f<H>(yf);
    dsh = ((double)yf - yold) * ((double)yf - yold);
    nrm = (double)yf * (double)yf;
    hsq = (double)h2f(yh) * (double)h2f(yh);
    Yf[(size_t)k * d + t] = yf;
    Yh[(size_t)k * ldy + t] = yh;
  } else if (t < ldy) {
    Yh[(size_t)k * ldy + t] = from_f<H>(0.f);
  }
  dsh = block_sum(dsh, red);
  nrm = block_sum(nrm, red);
  hsq = block_sum(hsq, red);
  if (t == 0) {
    hn[k] = (float)(0.5 * hsq);
    atomicAdd(&shift[0], dsh);
    atomicAdd(&shift[1], nrm);
  }
}

}  // namespace hb

namespace hb {
namespace {

using Bf = __nv_bfloat16;

// sample of the k-means++ seeding: every cell up to 64 K cells, at most 16384
int64_t km_sample_size(int64_t n, int K) { return std::min<int64_t>(n, std::min<int64_t>(64LL * K, 16384)); }

struct KmWork {
  Bf* Zh;        // [n][ldz] bf16 L2-normalised rows
  double* S;     // [m][d] seeding sample
  double* D2;    // [m]
  float* Yf;     // [K][d] centres
  Bf* Yh;        // [K][ldy] bf16 centres
  float* hn;     // [K] half squared norms of the bf16 centres
  float* P;      // [G][K][d] per-CTA centre sums
  float* C;      // [G][K] per-CTA counts
  double* shift; // [2] |Y_new - Y_old|^2, |Y_new|^2
  int* err;
  int* pick;     // sample index of the last chosen seed
};

size_t km_carve(Carver& cv, int64_t n, int d, int K, int G, KmWork& w) {
  const int ld = (int)align_up((size_t)d, 8);
  const int64_t m = km_sample_size(n, K);
  w.Zh = cv.take<Bf>((size_t)n * ld);
  w.S = cv.take<double>((size_t)m * d);
  w.D2 = cv.take<double>((size_t)m);
  w.Yf = cv.take<float>((size_t)K * d);
  w.Yh = cv.take<Bf>((size_t)K * ld);
  w.hn = cv.take<float>((size_t)K);
  w.P = cv.take<float>((size_t)G * K * d);
  w.C = cv.take<float>((size_t)G * K);
  w.shift = cv.take<double>(2);
  w.err = cv.take<int>(1);
  w.pick = cv.take<int>(1);
  return cv.off + 256;  // room to align the caller's base
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

HB_API size_t hb_kmeans_workspace_bytes(int64_t n, int32_t n_pcs, int32_t n_clusters) {
  if (n < 1 || n_pcs < 1 || n_clusters < 1) return 0;
  Carver cv(nullptr, 0);
  KmWork w;
  return km_carve(cv, n, n_pcs, n_clusters, num_sms(), w);
}

HB_API int hb_kmeans_init(const float* X, int64_t n, int32_t n_pcs, int32_t n_clusters, int32_t max_iter,
                          double tol, uint64_t seed, float* Y_out, int32_t* n_iter_out, void* workspace,
                          size_t workspace_bytes, void* stream) {
  const int d = n_pcs, K = n_clusters;
  if (!X || !Y_out || !workspace || n < 1 || d < 1 || K < 1 || K > n || max_iter < 0 || !(tol >= 0.0)) {
    set_error("hb_kmeans_init: bad argument");
    return HB_ERR_INVALID;
  }
  if (d > 256 || K > 256 || (d > 128 && K > 128)) {
    set_error("hb_kmeans_init: n_pcs=%d, n_clusters=%d out of range (n_pcs <= 128 with n_clusters <= 256, "
              "or n_pcs <= 256 with n_clusters <= 128)", d, K);
    return HB_ERR_UNSUPPORTED;
  }
  const int G = num_sms();
  if (workspace_bytes < hb_kmeans_workspace_bytes(n, d, K)) {
    set_error("hb_kmeans_init: workspace too small");
    return HB_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  KmWork w;
  km_carve(cv, n, d, K, G, w);
  const int ld = (int)align_up((size_t)d, 8);
  const int m = (int)km_sample_size(n, K);
  const KmLayout KL = km_layout(d, K);
  PinnedLease host(4 * sizeof(double));
  if (!host.ptr) {
    set_error("hb_kmeans_init: cudaMallocHost failed");
    return HB_ERR_CUDA;
  }
  double* h_shift = (double*)host.ptr;
  int* h_err = (int*)(h_shift + 2);

  HB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
  HB_TRY(launch_l2_normalize<float, Bf>(X, n, d, d, w.Zh, ld, st));
  const unsigned sgrid = (unsigned)((m + 255) / 256);
  k_km_sample<<<sgrid, 256, 0, st>>>(X, n, d, m, seed, w.S);
  HB_LAUNCH_CHECK();
  for (int r = 0; r < K; ++r) {
    if (r > 0) {
      k_km_dist<<<sgrid, 256, 0, st>>>(w.S, m, d, w.pick, r == 1, w.D2);
      HB_LAUNCH_CHECK();
    }
    k_km_pick<<<1, kSeedThreads, 0, st>>>(w.S, w.D2, m, d, r, seed, w.pick, w.Yf);
    HB_LAUNCH_CHECK();
  }
  HB_CUDA(cudaMemsetAsync(w.shift, 0, 2 * sizeof(double), st));
  k_km_update<Bf><<<K, dim3(32, 8), 0, st>>>(w.P, w.C, 0, K, d, w.Yf, w.Yh, ld, w.hn, w.shift);
  HB_LAUNCH_CHECK();
  const void* fn = (const void*)k_km_assign<Bf>;
  HB_TRY(allow_max_dyn_smem(fn));
  int iters = 0;
  for (int it = 0; it < max_iter; ++it) {
    HB_CUDA(cudaMemsetAsync(w.shift, 0, 2 * sizeof(double), st));
    k_km_assign<Bf><<<G, 256, KL.bytes, st>>>(w.Zh, ld, w.Yh, ld, w.hn, n, K, d, KL, w.P, w.C, w.err);
    HB_LAUNCH_CHECK();
    k_km_update<Bf><<<K, dim3(32, 8), 0, st>>>(w.P, w.C, G, K, d, w.Yf, w.Yh, ld, w.hn, w.shift);
    HB_LAUNCH_CHECK();
    HB_CUDA(cudaMemcpyAsync(h_shift, w.shift, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    HB_CUDA(cudaStreamSynchronize(st));
    ++iters;
    if (h_shift[0] <= tol * tol * h_shift[1]) break;
  }
  HB_CUDA(cudaMemcpyAsync(Y_out, w.Yf, sizeof(float) * (size_t)K * d, cudaMemcpyDeviceToDevice, st));
  HB_CUDA(cudaMemcpyAsync(h_err, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (*h_err) {
    set_error("hb_kmeans_init: tensor-core wait timed out (code %d)", *h_err);
    return HB_ERR_TIMEOUT;
  }
  if (n_iter_out) *n_iter_out = iters;
  return HB_OK;
}

}  // extern "C"
