// PCA by the covariance eigendecomposition, the reference's covariance path
// (preprocessing/_pca.py:339-353 -> _sparse_pca/_sparse_pca.py:26-127): the Gram
// matrix X^T X and the column means, cov = X^T X / n - mean mean^T (or the plain
// Gram for zero_center=False), eigh (cuSOLVER, called by the host), and the
// projection X_pca = X C^T - mean C^T.  The reference builds the Gram with one
// float atomic per pair of nonzeros of a row (kernels_spca.cuh:5-28) and projects
// with a sparse-dense product; here both run on the tensor core:
//
//   k_pca_gram     one CTA per (128-gene block I, 128-gene block J >= I, row split):
//                  128-row tiles of X read once, split into bf16 hi + lo parts
//                  (x = hi + lo to ~16 significant bits) and staged MN-major;
//                  D[i][j] += hi_i hi_j + hi_i lo_j + lo_i hi_j on tcgen05 with the
//                  float32 accumulator in TMEM, drained into the CTA's float64 partial
//                  every kDrainTiles row tiles: the tensor core's float32 accumulation
//                  rounds with a bias, so its error grows with the length of the chain
//                  (one chain over 100,000 rows measured 9e-4 relative; 2,048 rows keep it
//                  near the hi/lo split's 1e-5); diagonal blocks also sum their columns in
//                  float64 (the means).
//   k_pca_reduce   float64 sum of the row-split partials into the full symmetric
//                  Gram matrix and the column sums.
//   k_pca_cov      cov = G / n - mean mean^T in float64.
//   k_pca_project  per 128-row tile: D[row][comp] = sum over 64-gene chunks of
//                  X (hi/lo) . C (hi/lo) on tcgen05, minus the mean impact.
//   k_csr_densify  CSR rows scattered into a dense float32 matrix (sparse input).
#include "hb_tc_tile.cuh"
#include "../../include/harmony_b200.h"

namespace hb {
namespace {

constexpr int kGB = 128;          // genes per Gram block (M = N = 128)
constexpr int kDrainTiles = 16;   // 128-row tiles per float32 accumulation chain in TMEM

// byte offset of 16-byte chunk c8 of 64-element block nb in row r of an MN-major,
// 128-byte-swizzled tile with `nblocks` 64-element blocks per 8-row group
__device__ __forceinline__ uint32_t mn_off(uint32_t r, uint32_t nb, uint32_t c8, uint32_t nblocks) {
  return (r >> 3) * (nblocks * 1024u) + nb * 1024u + (r & 7u) * 128u + ((c8 ^ (r & 7u)) << 4);
}

__device__ __forceinline__ void split8(const float (&x)[8], __nv_bfloat16 (&hi)[8], __nv_bfloat16 (&lo)[8]) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    hi[i] = __float2bfloat16_rn(x[i]);
    lo[i] = __float2bfloat16_rn(x[i] - __bfloat162float(hi[i]));
  }
}

// x[0..8) = X[row][col .. col + 8), zero past n_genes or for a row outside the split
__device__ __forceinline__ void load8(const float* __restrict__ X, int64_t ldx, int64_t row, bool ok, int col,
                                      int g, bool vec, float (&x)[8]) {
  if (ok && vec && col + 8 <= g) {
    const float4 u = __ldg((const float4*)(X + row * ldx + col));
    const float4 w = __ldg((const float4*)(X + row * ldx + col + 4));
    x[0] = u.x; x[1] = u.y; x[2] = u.z; x[3] = u.w;
    x[4] = w.x; x[5] = w.y; x[6] = w.z; x[7] = w.w;
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (ok && col + i < g) ? __ldg(X + row * ldx + col + i) : 0.f;
  }
}

struct GramArgs {
  const float* X;
  int64_t n, ldx;
  int g, nI, T, S;
  int vec;          // rows 16-byte aligned: float4 loads
  double* Gpart;    // [S][T][128][128] float64 partials
  double* Cpart;    // [S][nI][128] column sums (written by the diagonal blocks)
  int* err;
};

// upper-triangle block pair of tile t: row-major over I, J = I .. nI-1
__device__ __forceinline__ void tile_ij(int t, int nI, int& I, int& J) {
  int i = 0;
  while (t >= nI - i) {
    t -= nI - i;
    ++i;
  }
  I = i;
  J = i + t;
}
__host__ __device__ __forceinline__ int tile_of(int I, int J, int nI) { return I * nI - I * (I - 1) / 2 + (J - I); }

constexpr uint32_t kGramAh = 0, kGramAl = 32768, kGramBh = 65536, kGramBl = 98304, kGramMisc = 131072;
constexpr uint32_t kGramRed = kGramMisc + 64;                   // [16][128] float64 column-sum partials
constexpr uint32_t kGramSmem = kGramRed + 16 * 128 * 8 + 1024;  // + 1024-byte alignment slack

__global__ void __launch_bounds__(256, 1) k_pca_gram(GramArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = blockIdx.x % a.T, s = blockIdx.x / a.T;
  int I, J;
  tile_ij(t, a.nI, I, J);
  const bool diag = I == J;
  uint64_t* mbar = (uint64_t*)(sm + kGramMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + kGramMisc + 8);
  const uint32_t sm32 = tc::smem_u32(sm);
  const int64_t r0 = a.n * s / a.S, r1 = a.n * (s + 1) / a.S;
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, 128u);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc::idesc_f16(128, 128, true, true, true);
  // thread -> (8-gene chunk c of the block, rows rr + 16 p): 16 threads cover one row of
  // a block with coalesced 32-byte loads
  const int c = tid & 15, rr = tid >> 4;
  const int gI = I * kGB + 8 * c, gJ = J * kGB + 8 * c;
  double cs[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) cs[i] = 0.0;
  // D[i][j] -> Gpart[s][t][i][j] (float64): warps 0-3 columns 0..63, warps 4-7 columns 64..127
  const int dm = (warp & 3) * 32 + lane, dc_lo = (warp >> 2) * 64;
  const uint32_t dtl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  double* dout = a.Gpart + ((size_t)s * a.T + t) * (kGB * kGB) + (size_t)dm * kGB;
  auto drain = [&](bool add) {
    for (int c0 = dc_lo; c0 < dc_lo + 64; c0 += 8) {
      float v[8];
      tc::tmem_ld8(dtl + (uint32_t)c0, v);
      tc::tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 8; ++i) dout[c0 + i] = add ? dout[c0 + i] + (double)v[i] : (double)v[i];
    }
  };
  auto zero_partial = [&]() {
    for (int c0 = dc_lo; c0 < dc_lo + 64; ++c0) dout[c0] = 0.0;
  };
  int it = 0;
  for (int64_t base = r0; base < r1; base += 128, ++it) {
#pragma unroll 2
    for (int p = 0; p < 8; ++p) {
      const int r = rr + 16 * p;
      const int64_t row = base + r;
      const bool ok = row < r1;
      const uint32_t off = mn_off((uint32_t)r, (uint32_t)(c >> 3), (uint32_t)(c & 7), 2u);
      float x[8];
      __align__(16) __nv_bfloat16 hi[8], lo[8];
      load8(a.X, a.ldx, row, ok, gI, a.g, a.vec != 0, x);
      if (diag)
#pragma unroll
        for (int i = 0; i < 8; ++i) cs[i] += (double)x[i];
      split8(x, hi, lo);
      *(uint4*)(sm + kGramAh + off) = *(const uint4*)hi;
      *(uint4*)(sm + kGramAl + off) = *(const uint4*)lo;
      if (!diag) {
        load8(a.X, a.ldx, row, ok, gJ, a.g, a.vec != 0, x);
        split8(x, hi, lo);
        *(uint4*)(sm + kGramBh + off) = *(const uint4*)hi;
        *(uint4*)(sm + kGramBl + off) = *(const uint4*)lo;
      }
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t ah0 = sm32 + kGramAh, al0 = sm32 + kGramAl;
      const uint32_t bh0 = diag ? ah0 : sm32 + kGramBh, bl0 = diag ? al0 : sm32 + kGramBl;
      for (int ks = 0; ks < 8; ++ks) {  // 8 steps of 16 rows
        const uint32_t o = (uint32_t)ks * 2u * 2u * 1024u;
        const uint64_t ah = tc::sdesc_sw128(ah0 + o, 1024, 2048), al = tc::sdesc_sw128(al0 + o, 1024, 2048);
        const uint64_t bh = tc::sdesc_sw128(bh0 + o, 1024, 2048), bl = tc::sdesc_sw128(bl0 + o, 1024, 2048);
        tc::mma_f16(tmem, ah, bh, idesc, (it % kDrainTiles > 0 || ks > 0) ? 1u : 0u);
        tc::mma_f16(tmem, ah, bl, idesc, 1u);
        tc::mma_f16(tmem, al, bh, idesc, 1u);
      }
      tc::mma_commit(mbar);
    }
    // the operands are rewritten by the next row tile: wait for the MMAs
    if (!tc::mbar_wait(mbar, (uint32_t)(it & 1), kMaxPolls)) atomicExch(a.err, 8);
    tc::fence_after_sync();
    // end of a chain (or of the rows): D is added into the float64 partial and the next
    // tile's first MMA starts a new chain (the loop-top barrier orders these loads before it)
    if (it % kDrainTiles == kDrainTiles - 1 || base + 128 >= r1) drain(it >= kDrainTiles);
  }
  if (it == 0) zero_partial();
  if (diag) {  // column sums of block I: 16 threads per 8-gene chunk
    double* red = (double*)(sm + kGramRed);
#pragma unroll
    for (int i = 0; i < 8; ++i) red[rr * 128 + 8 * c + i] = cs[i];
    __syncthreads();
    if (tid < 128) {
      double v = 0.0;
      for (int q = 0; q < 16; ++q) v += red[q * 128 + tid];
      a.Cpart[((size_t)s * a.nI + I) * kGB + tid] = v;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 128u);
  }
}

// G[i][j] = G[j][i] = sum over splits of the partial of the upper block pair (float64)
__global__ void k_pca_reduce(const double* __restrict__ Gpart, const double* __restrict__ Cpart, int g, int nI,
                             int T, int S, double* __restrict__ G, double* __restrict__ csum) {
  const int64_t ne = (int64_t)g * g;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(e / g), j = (int)(e % g);
    if (i > j) continue;  // the lower triangle is written as the mirror
    const int I = i / kGB, J = j / kGB;
    const size_t at = (size_t)tile_of(I, J, nI) * kGB * kGB + (size_t)(i % kGB) * kGB + (j % kGB);
    double v = 0.0;
    for (int q = 0; q < S; ++q) v += Gpart[(size_t)q * T * kGB * kGB + at];
    G[(size_t)i * g + j] = v;
    G[(size_t)j * g + i] = v;
  }
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g; e += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int q = 0; q < S; ++q) v += Cpart[(size_t)q * nI * kGB + e];
    csum[e] = v;
  }
}

// cov = G / n - mean mean^T (zero_center) or cov = G; mean = column sums / n
__global__ void k_pca_cov(const double* __restrict__ G, const double* __restrict__ csum, int64_t n, int g,
                          int zero_center, double* __restrict__ cov, double* __restrict__ mean) {
  const int64_t ne = (int64_t)g * g;
  const double inv_n = 1.0 / (double)n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / g), j = (int)(e % g);
    cov[e] = zero_center ? G[e] * inv_n - (csum[i] * inv_n) * (csum[j] * inv_n) : G[e];
    if (mean && j == 0) mean[i] = csum[i] * inv_n;
  }
}

// hi / lo bf16 copies of the components [kpad][gpad] (zero padded) and the mean impact
// mp[k] = sum_g mean[g] C[k][g] (float64); one CTA per component row
__global__ void k_pca_prep(const float* __restrict__ C, int k, int g, int kpad, int gpad,
                           const double* __restrict__ mean, __nv_bfloat16* __restrict__ Ch,
                           __nv_bfloat16* __restrict__ Cl, double* __restrict__ mp) {
  __shared__ double red[32];
  const int row = blockIdx.x;
  double acc = 0.0;
  for (int j = threadIdx.x; j < gpad; j += blockDim.x) {
    const float x = (row < k && j < g) ? C[(size_t)row * g + j] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    Ch[(size_t)row * gpad + j] = h;
    Cl[(size_t)row * gpad + j] = __float2bfloat16_rn(x - __bfloat162float(h));
    if (mean && j < g) acc += mean[j] * (double)x;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0 && row < k) mp[row] = mean ? acc : 0.0;
}

struct ProjArgs {
  const float* X;
  int64_t n, ldx;
  int g, k, kpad, gpad, vec;
  const __nv_bfloat16* Ch;
  const __nv_bfloat16* Cl;
  const double* mp;
  float* out;  // [n][k]
  int* err;
};

// X_pca rows of 128-row tiles: D[row][comp] = sum over 64-gene chunks of (Xh + Xl).(Ch + Cl)
// without the lo.lo term; A (X rows) and B (components) are K-major 128B-swizzled tiles.
__global__ void __launch_bounds__(256) k_pca_project(ProjArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bbytes = (uint32_t)a.kpad * 128u;
  const uint32_t oAh = 0, oAl = 16384, oBh = 32768, oBl = 32768 + bbytes, oMisc = 32768 + 2 * bbytes;
  uint64_t* mbar = (uint64_t*)(sm + oMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + oMisc + 8);
  const uint32_t sm32 = tc::smem_u32(sm);
  uint32_t tcols = 32;
  while (tcols < (uint32_t)a.kpad) tcols <<= 1;
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc::idesc_f16(128, a.kpad, true, false, false);
  const int64_t ntiles = (a.n + 127) / 128;
  const int nq = a.gpad / 64;
  uint32_t ph = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t base = tile * 128;
    for (int q = 0; q < nq; ++q) {
      // A: 128 rows x 64 genes: thread -> (row tid / 8 + 32 p, chunk tid % 8)
      const int ch = tid & 7;
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int r = (tid >> 3) + 32 * p;
        const int64_t row = base + r;
        float x[8];
        __align__(16) __nv_bfloat16 hi[8], lo[8];
        load8(a.X, a.ldx, row, row < a.n, q * 64 + ch * 8, a.g, a.vec != 0, x);
        split8(x, hi, lo);
        const uint32_t off = tc::sw128_off((uint32_t)r, (uint32_t)ch);
        *(uint4*)(sm + oAh + off) = *(const uint4*)hi;
        *(uint4*)(sm + oAl + off) = *(const uint4*)lo;
      }
      // B: kpad components x 64 genes of the chunk
      for (int e = tid; e < a.kpad * 8; e += 256) {
        const int kr = e >> 3, c8 = e & 7;
        const size_t src = (size_t)kr * a.gpad + (size_t)q * 64 + c8 * 8;
        const uint32_t off = tc::sw128_off((uint32_t)kr, (uint32_t)c8);
        tc::cp_async16(sm32 + oBh + off, a.Ch + src, 16u);
        tc::cp_async16(sm32 + oBl + off, a.Cl + src, 16u);
      }
      tc::cp_async_wait_all();
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (tid == 0) {
        for (int ks = 0; ks < 4; ++ks) {
          const uint64_t ah = tc::sdesc_sw128(sm32 + oAh + ks * 32u, 16, 1024);
          const uint64_t al = tc::sdesc_sw128(sm32 + oAl + ks * 32u, 16, 1024);
          const uint64_t bh = tc::sdesc_sw128(sm32 + oBh + ks * 32u, 16, 1024);
          const uint64_t bl = tc::sdesc_sw128(sm32 + oBl + ks * 32u, 16, 1024);
          tc::mma_f16(tmem, ah, bh, idesc, (q > 0 || ks > 0) ? 1u : 0u);
          tc::mma_f16(tmem, ah, bl, idesc, 1u);
          tc::mma_f16(tmem, al, bh, idesc, 1u);
        }
        tc::mma_commit(mbar);
      }
      if (!tc::mbar_wait(mbar, ph, kMaxPolls)) atomicExch(a.err, 8);
      ph ^= 1u;
      tc::fence_after_sync();
    }
    // epilogue: row (warp & 3) * 32 + lane, columns split between warps 0-3 and 4-7
    {
      const int r = (warp & 3) * 32 + lane;
      const int64_t row = base + r;
      const int half = (a.kpad / 2 + 7) / 8 * 8;
      const int c_lo = (warp >> 2) * half, c_hi = min(a.kpad, c_lo + half);
      const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
      for (int c0 = c_lo; c0 < c_hi; c0 += 8) {
        float v[8];
        tc::tmem_ld8(tl + (uint32_t)c0, v);
        tc::tmem_ld_wait();
        if (row < a.n)
#pragma unroll
          for (int i = 0; i < 8; ++i)
            if (c0 + i < a.k) a.out[row * a.k + c0 + i] = (float)((double)v[i] - a.mp[c0 + i]);
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, tcols);
  }
}

// one warp per row: out[row][indices[p]] = data[p] for p in [indptr[row], indptr[row + 1])
__global__ void k_csr_densify(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                              const float* __restrict__ data, int64_t n_rows, int n_cols, float* __restrict__ out,
                              int64_t ldo, int* err) {
  const int lane = threadIdx.x & 31;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows;
       row += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t p0 = indptr[row], p1 = indptr[row + 1];
    for (int64_t p = p0 + lane; p < p1; p += 32) {
      const int col = indices[p];
      if (col < 0 || col >= n_cols) {
        atomicExch(err, 9);
        continue;
      }
      out[row * ldo + col] = data[p];
    }
  }
}

struct GramPlan {
  int nI, T, S;
  size_t part_bytes, cpart_bytes, err_off, bytes;
};

GramPlan gram_plan(int64_t n, int g) {
  GramPlan P{};
  P.nI = (g + kGB - 1) / kGB;
  P.T = P.nI * (P.nI + 1) / 2;
  // row splits: about four CTAs per SM in all, at least 512 rows per CTA, partials <= 2 GiB
  const int sms = num_sms();
  int64_t S = std::max<int64_t>(1, (4 * sms + P.T - 1) / P.T);
  S = std::min<int64_t>(S, std::max<int64_t>(1, n / 512));
  while (S > 1 && (size_t)S * P.T * kGB * kGB * 8 > ((size_t)2 << 30)) --S;
  P.S = (int)S;
  P.part_bytes = align_up((size_t)P.S * P.T * kGB * kGB * 8, 256);
  P.cpart_bytes = align_up((size_t)P.S * P.nI * kGB * 8, 256);
  P.err_off = P.part_bytes + P.cpart_bytes;
  P.bytes = P.err_off + 256;
  return P;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

HB_API size_t hb_pca_gram_workspace_bytes(int64_t n, int32_t n_genes) {
  if (n < 1 || n_genes < 1) return 0;
  return gram_plan(n, n_genes).bytes + 256;
}

HB_API int hb_pca_gram(const float* X, int64_t n, int32_t n_genes, int64_t ldx, double* gram, double* col_sums,
                       void* workspace, size_t workspace_bytes, void* stream) {
  if (!X || !gram || !col_sums || n < 1 || n_genes < 1 || ldx < n_genes) {
    set_error("hb_pca_gram: bad argument");
    return HB_ERR_INVALID;
  }
  if (n_genes > 32768) {
    set_error("hb_pca_gram: n_genes=%d exceeds 32768", n_genes);
    return HB_ERR_UNSUPPORTED;
  }
  const GramPlan P = gram_plan(n, n_genes);
  if (!workspace || workspace_bytes < P.bytes + 256) {
    set_error("hb_pca_gram: workspace too small (%zu < %zu)", workspace_bytes, P.bytes + 256);
    return HB_ERR_WORKSPACE;
  }
  char* ws = (char*)align_up((size_t)workspace, 256);
  cudaStream_t st = (cudaStream_t)stream;
  int* err = (int*)(ws + P.err_off);
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  GramArgs a{X, n, ldx, n_genes, P.nI, P.T, P.S, ((uintptr_t)X % 16 == 0 && ldx % 4 == 0) ? 1 : 0,
             (double*)ws, (double*)(ws + P.part_bytes), err};
  HB_TRY(allow_max_dyn_smem((const void*)k_pca_gram));
  k_pca_gram<<<P.T * P.S, 256, kGramSmem, st>>>(a);
  HB_LAUNCH_CHECK();
  const int64_t ne = (int64_t)n_genes * n_genes;
  k_pca_reduce<<<(unsigned)std::min<int64_t>((ne + 255) / 256, 8 * num_sms()), 256, 0, st>>>(
      a.Gpart, a.Cpart, n_genes, P.nI, P.T, P.S, gram, col_sums);
  HB_LAUNCH_CHECK();
  int h_err = 0;
  HB_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (h_err) {
    set_error("hb_pca_gram: tensor-core wait timed out (code %d)", h_err);
    return HB_ERR_TIMEOUT;
  }
  return HB_OK;
}

HB_API int hb_pca_covariance(const double* gram, const double* col_sums, int64_t n, int32_t n_genes,
                             int32_t zero_center, double* cov, double* mean, void* stream) {
  if (!gram || !col_sums || !cov || n < 1 || n_genes < 1) {
    set_error("hb_pca_covariance: bad argument");
    return HB_ERR_INVALID;
  }
  const int64_t ne = (int64_t)n_genes * n_genes;
  k_pca_cov<<<(unsigned)std::min<int64_t>((ne + 255) / 256, 8 * num_sms()), 256, 0, (cudaStream_t)stream>>>(
      gram, col_sums, n, n_genes, zero_center, cov, mean);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

HB_API size_t hb_pca_project_workspace_bytes(int32_t n_genes, int32_t n_comps) {
  if (n_genes < 1 || n_comps < 1) return 0;
  const size_t kpad = (size_t)(n_comps + 15) / 16 * 16, gpad = (size_t)(n_genes + 63) / 64 * 64;
  return align_up(kpad * gpad * 2, 256) * 2 + align_up(kpad * 8, 256) + 256 + 256;
}

HB_API int hb_pca_project(const float* X, int64_t n, int32_t n_genes, int64_t ldx, const float* components,
                          int32_t n_comps, const double* mean, float* X_pca, void* workspace, size_t workspace_bytes,
                          void* stream) {
  if (!X || !components || !X_pca || n < 1 || n_genes < 1 || ldx < n_genes || n_comps < 1) {
    set_error("hb_pca_project: bad argument");
    return HB_ERR_INVALID;
  }
  if (n_comps > 256) {
    set_error("hb_pca_project: n_comps=%d exceeds 256", n_comps);
    return HB_ERR_UNSUPPORTED;
  }
  const size_t need = hb_pca_project_workspace_bytes(n_genes, n_comps);
  if (!workspace || workspace_bytes < need) {
    set_error("hb_pca_project: workspace too small (%zu < %zu)", workspace_bytes, need);
    return HB_ERR_WORKSPACE;
  }
  const int kpad = (n_comps + 15) / 16 * 16, gpad = (n_genes + 63) / 64 * 64;
  Carver cv((void*)align_up((size_t)workspace, 256), workspace_bytes - 256);
  __nv_bfloat16* Ch = cv.take<__nv_bfloat16>((size_t)kpad * gpad);
  __nv_bfloat16* Cl = cv.take<__nv_bfloat16>((size_t)kpad * gpad);
  double* mp = cv.take<double>((size_t)kpad);
  int* err = cv.take<int>(4);
  cudaStream_t st = (cudaStream_t)stream;
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  HB_CUDA(cudaMemsetAsync(mp, 0, sizeof(double) * kpad, st));
  k_pca_prep<<<kpad, 256, 0, st>>>(components, n_comps, n_genes, kpad, gpad, mean, Ch, Cl, mp);
  HB_LAUNCH_CHECK();
  const size_t smem = 32768 + 2 * (size_t)kpad * 128 + 64 + 1024;
  HB_TRY(allow_max_dyn_smem((const void*)k_pca_project));
  const int64_t ntiles = (n + 127) / 128;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, 2 * num_sms()));
  ProjArgs pa{X, n, ldx, n_genes, n_comps, kpad, gpad, ((uintptr_t)X % 16 == 0 && ldx % 4 == 0) ? 1 : 0,
              Ch, Cl, mp, X_pca, err};
  k_pca_project<<<grid, 256, smem, st>>>(pa);
  HB_LAUNCH_CHECK();
  int h_err = 0;
  HB_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (h_err) {
    set_error("hb_pca_project: tensor-core wait timed out (code %d)", h_err);
    return HB_ERR_TIMEOUT;
  }
  return HB_OK;
}

HB_API int hb_csr_to_dense(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n_rows,
                           int32_t n_cols, float* out, int64_t ldo, int32_t* err, void* stream) {
  if (!indptr || !out || !err || n_rows < 0 || n_cols < 1 || ldo < n_cols) {
    set_error("hb_csr_to_dense: bad argument");
    return HB_ERR_INVALID;
  }
  if (n_rows == 0) return HB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  HB_CUDA(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)n_rows * ldo, st));
  HB_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
  k_csr_densify<<<(unsigned)std::min<int64_t>((n_rows * 32 + 255) / 256, 16 * num_sms()), 256, 0, st>>>(
      indptr, indices, data, n_rows, n_cols, out, ldo, err);
  HB_LAUNCH_CHECK();
  int h_err = 0;
  HB_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (h_err) {
    set_error("hb_csr_to_dense: column index outside [0, n_cols)");
    return HB_ERR_INVALID;
  }
  return HB_OK;
}

}  // extern "C"
