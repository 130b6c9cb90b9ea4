// Tensor-core centroid pass of the 16-bit path, streaming in cell order.
//
// The same sums as k_tc_centroid (hb_centroid_tc.cu): P[cluster][pc] = sum over
// cells of R[cell][cluster] Z_norm[cell][pc] (the centroid GEMM of the reference,
// _cuda/harmony/clustering/clustering.cu:272-276) and, per (block, batch) key of
// the coming sweep, the sum of the cells' R rows (the "remove old contribution"
// terms, clustering.cu:321-332), and per block their sum over the batches (key
// (block, B), the column sums).  Here the cells are read in storage order, so
// each 128-cell tile of Z_norm and of R is one TMA tile load instead of a row
// gather, and the per-key sums become a second MMA against a one-hot operand:
//   D1[cluster][pc]  += R_tile^T Z_tile
//   D2[cluster][key] += R_tile^T H_tile,  H[cell][key] = 1 for the cell's key
// both accumulated in TMEM over the CTA's tiles (A = R_tile^T is shared).  The
// one-hot tile stays resident: per tile only the previous tile's ones are
// cleared and the new ones set.  D1 and D2 are written once per CTA and summed
// over the CTAs by k_cs_reduce (one launch for both).
//
// Tensor maps: Z_norm and R viewed as 4-D {64 values, 8 rows, 64-value blocks,
// 8-row groups}, box {64, 8, blocks, 16}, so one load lands a tile in the
// MN-major layout [group][block][8 rows x 128 B] (128B swizzle).  The blocks of
// a row reach past its stored columns into the next row; those values only feed
// D rows / columns that are discarded.  The row count is padded to whole tiles
// (+8 rows) and the padding rows are zero, so they add nothing.
#include <cudaTypedefs.h>
#include "hb_tc_tile.cuh"

namespace hb {

struct CsLayout {
  int nbZ, nbB, nbK, nM2, ncolsZ, nkpad, tcols, stages;
  int noh;  // one-hot operands (2: the one-hot of tile i+1 is written while tile i's MMAs run)
  uint32_t stZ, stB, offZ, offB, offOH, ohBytes, offBar, bytes;
};

inline CsLayout cs_layout(int d, int K, int nkeys, int ldz) {
  CsLayout L{};
  L.nbZ = (ldz + 63) / 64;
  L.ncolsZ = 64 * L.nbZ;
  L.nM2 = (K + 127) / 128;
  L.nbB = 2 * L.nM2;            // 64-cluster blocks in pairs (M = 128 per MMA)
  L.nkpad = (nkeys + 15) / 16 * 16;
  L.nbK = (L.nkpad + 63) / 64;
  int t = 32;
  while (t < L.nM2 * (L.ncolsZ + L.nkpad)) t <<= 1;
  L.tcols = t;
  L.stZ = (uint32_t)L.nbZ * 16384u;
  L.stB = (uint32_t)L.nbB * 16384u;
  L.ohBytes = (uint32_t)L.nbK * 16384u;
  // two one-hot operands when they fit beside three tile stages (without the second one the
  // per-tile period is MMA -> one-hot rewrite -> MMA in series; with two stages the loads
  // fall behind, which costs more: 500k cells, 180 keys measured 73 vs 68 us per pass)
  for (int noh = 2; noh >= 1; --noh) {
    bool fits = false;
    for (int st = 4; st >= (noh == 2 ? 3 : 2) && !fits; --st) {
      uint32_t o = 0;
      L.offZ = o; o += (uint32_t)st * L.stZ;
      L.offB = o; o += (uint32_t)st * L.stB;
      L.offOH = o; o += (uint32_t)noh * L.ohBytes;
      L.offBar = o; o += 16u * 8u + 16u;
      L.bytes = o + 1024u;
      L.stages = st;
      L.noh = noh;
      fits = L.bytes <= 220u * 1024u;
    }
    if (fits) break;
  }
  (void)d;
  return L;
}

// The streaming pass applies when its accumulators fit in TMEM and its tiles in shared memory.
bool cs_supported(int d, int K, int nkeys, int ldz) {
  const CsLayout L = cs_layout(d, K, nkeys, ldz);
  return d <= 128 && K <= 256 && L.nkpad <= 256 && L.nM2 * (L.ncolsZ + L.nkpad) <= 512 &&
         L.bytes <= 220u * 1024u;
}

__device__ __forceinline__ void mbar_arrive_cta(uint64_t* m) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(m)) : "memory");
}

template <typename H>
__global__ void __launch_bounds__(256, 1) k_tc_centroid_stream(CenStreamArgs a, CsLayout L,
                                                               const __grid_constant__ CUtensorMap tmZ,
                                                               const __grid_constant__ CUtensorMap tmR) {
  if (a.stop && *(volatile const int*)a.stop) return;  // the k-means loop has stopped on the device
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int K = a.K, S = L.stages;
  const int NOH = L.noh;
  uint64_t* full = (uint64_t*)(sm + L.offBar);  // [S] tile landed
  uint64_t* mma_done = full + 4;                // [NOH] MMAs of a tile on one-hot b completed (phase per such tile)
  uint64_t* oh_ready = full + 6;                // [NOH] one-hot b holds its next tile (phase per such tile)
  uint64_t* empty = full + 8;                   // [S] MMAs of the stage's last tile completed
  uint64_t* acc_bar = full + 12;                // all MMAs of the CTA completed (one phase)
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offBar + 128);
  const uint32_t sm32 = tc::smem_u32(sm);
  const int t0 = (int)((int64_t)a.ntiles * blockIdx.x / gridDim.x);
  const int nt = (int)((int64_t)a.ntiles * (blockIdx.x + 1) / gridDim.x) - t0;
  const uint32_t tile_bytes = (uint32_t)(L.nbZ + L.nbB) * 16384u;

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) tc::mbar_init(full + s, 1);
    for (int b = 0; b < NOH; ++b) {
      tc::mbar_init(mma_done + b, 1);
      tc::mbar_init(oh_ready + b, 4);
    }
    for (int s = 0; s < S; ++s) tc::mbar_init(empty + s, 1);
    tc::mbar_init(acc_bar, 1);
    tc::fence_mbar_init();
  }
  for (uint32_t e = tid * 16u; e < (uint32_t)NOH * L.ohBytes; e += 256u * 16u)
    *(uint4*)(sm + L.offOH + e) = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  if (tid == 0) {
    for (int j = 0; j < S && j < nt; ++j) {
      tc::mbar_arrive_expect_tx(full + j, tile_bytes);
      tc::tma_load4d(sm32 + L.offZ + j * L.stZ, &tmZ, 0, 0, 0, (t0 + j) * 16, full + j);
      tc::tma_load4d(sm32 + L.offB + j * L.stB, &tmR, 0, 0, 0, (t0 + j) * 16, full + j);
    }
  }
  const uint32_t idesc1 = tc::idesc_f16(128, L.ncolsZ, is_bf16<H>::value, true, true);
  const uint32_t idesc2 = tc::idesc_f16(128, L.nkpad, is_bf16<H>::value, true, true);
  // Roles (no CTA-wide barrier inside the loop):
  //   thread 0      MMA issuer: waits for the tile (full[s]) and its one-hot (oh_ready[b],
  //                 b = i % NOH), commits to mma_done[b];
  //   thread 32     TMA producer: loads tile j into its stage once the MMAs of the
  //                 stage's previous tile completed (empty[s]);
  //   warps 4-7     one-hot writers (row = thread - 128): once the MMAs of tile i - NOH
  //                 (the last user of one-hot b) completed, clear its ones and set tile
  //                 i's; one arrival per warp on oh_ready[b].
  // One barrier pair per one-hot operand: a waiter of either never falls two phases behind.
  if (tid == 0) {
    for (int i = 0; i < nt; ++i) {
      const int s = i % S;
      if (!tc::mbar_wait(full + s, (uint32_t)((i / S) & 1), kMaxPolls)) atomicExch(a.err, 6);
      const int b = i % NOH;
      if (!tc::mbar_wait(oh_ready + b, (uint32_t)((i / NOH) & 1), kMaxPolls)) atomicExch(a.err, 6);
      tc::fence_after_sync();
      const uint32_t sZ = sm32 + L.offZ + s * L.stZ, sB = sm32 + L.offB + s * L.stB;
      const uint32_t sH = sm32 + L.offOH + (uint32_t)b * L.ohBytes;
      for (int m = 0; m < L.nM2; ++m) {
        const uint32_t d1 = tmem + (uint32_t)(m * L.ncolsZ);
        const uint32_t d2 = tmem + (uint32_t)(L.nM2 * L.ncolsZ + m * L.nkpad);
        for (int k = 0; k < 8; ++k) {  // 8 steps of 16 cells
          const uint64_t ad = tc::sdesc_sw128(sB + (uint32_t)(2 * m) * 1024u + (uint32_t)k * 2u * (uint32_t)L.nbB * 1024u,
                                              1024, (uint32_t)L.nbB * 1024u);
          const uint64_t bz = tc::sdesc_sw128(sZ + (uint32_t)k * 2u * (uint32_t)L.nbZ * 1024u, 1024,
                                              (uint32_t)L.nbZ * 1024u);
          const uint64_t bh = tc::sdesc_sw128(sH + (uint32_t)k * 2u * (uint32_t)L.nbK * 1024u, 1024,
                                              (uint32_t)L.nbK * 1024u);
          const uint32_t acc = (i > 0 || k > 0) ? 1u : 0u;
          tc::mma_f16(d1, ad, bz, idesc1, acc);
          tc::mma_f16(d2, ad, bh, idesc2, acc);
        }
      }
      tc::mma_commit(empty + s);
      tc::mma_commit(mma_done + b);
    }
    if (nt > 0) tc::mma_commit(acc_bar);
  } else if (tid == 32) {
    for (int j = S; j < nt; ++j) {  // tile j reuses the stage of tile j - S
      const int sj = j % S;
      if (!tc::mbar_wait(empty + sj, (uint32_t)(((j / S) + 1) & 1), kMaxPolls)) atomicExch(a.err, 5);
      tc::mbar_arrive_expect_tx(full + sj, tile_bytes);
      tc::tma_load4d(sm32 + L.offZ + sj * L.stZ, &tmZ, 0, 0, 0, (t0 + j) * 16, full + sj);
      tc::tma_load4d(sm32 + L.offB + sj * L.stB, &tmR, 0, 0, 0, (t0 + j) * 16, full + sj);
    }
  } else if (warp >= 4) {
    const int row = tid - 128;
    auto key_of = [&](int i) -> int {  // key of row `row` of the CTA's tile i (-1 past the cells)
      const int64_t cell = (int64_t)(t0 + i) * 128 + row;
      return (i < nt && cell < a.n) ? __ldg(a.ckey + cell) : -1;
    };
    // one-hot element (row r, key k): MN-major [group][nbK][8 rows x 128 B]
    auto oh_off = [&](int r, int k) -> uint32_t {
      return (uint32_t)(r >> 3) * (uint32_t)L.nbK * 1024u + (uint32_t)(k >> 6) * 1024u + (uint32_t)(r & 7) * 128u +
             ((((uint32_t)(k & 63) >> 3) ^ (uint32_t)(r & 7)) << 4) + (uint32_t)(k & 7) * 2u;
    };
    const H one = from_f<H>(1.f), zero = from_f<H>(0.f);
    int kq[4];  // keys of tiles i .. i+3
#pragma unroll
    for (int q = 0; q < 4; ++q) kq[q] = key_of(q);
    int key_old[2] = {-1, -1};  // the key set in each one-hot operand
    for (int i = 0; i < nt; ++i) {
      const int b = i % NOH;
      if (i >= NOH && !tc::mbar_wait(mma_done + b, (uint32_t)(((i - NOH) / NOH) & 1), kMaxPolls))
        atomicExch(a.err, 5);
      unsigned char* oh = sm + L.offOH + (uint32_t)b * L.ohBytes;
      const int key = kq[0], ko = key_old[b];
      // a cell's ones: its key and, with kpb, the column-sum key (block, B) of its block
      if (ko >= 0) {
        *(H*)(oh + oh_off(row, ko)) = zero;
        if (a.kpb) *(H*)(oh + oh_off(row, ko - ko % a.kpb + a.kpb - 1)) = zero;
      }
      if (key >= 0) {
        *(H*)(oh + oh_off(row, key)) = one;
        if (a.kpb) *(H*)(oh + oh_off(row, key - key % a.kpb + a.kpb - 1)) = one;
      }
      key_old[b] = key;
      kq[0] = kq[1];
      kq[1] = kq[2];
      kq[2] = kq[3];
      kq[3] = key_of(i + 4);
      tc::fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive_cta(oh_ready + b);
    }
  }
  // Threads without a role wait here in the hardware barrier: spinning on an mbarrier in the
  // warps of the issuer and the producer would take their issue slots for the whole loop.
  // Then the single-phase acc_bar (the warps without a role never tracked mma_done's phases).
  __syncthreads();
  if (nt > 0 && !tc::mbar_wait(acc_bar, 0, kMaxPolls)) atomicExch(a.err, 4);
  tc::fence_after_sync();
  // ---- epilogue: D1 -> P[cta][cluster][pc], D2 -> Opart[cta][key][cluster] -------------
  {
    const int half = warp >> 2, q = warp & 3;
    for (int m = 0; m < L.nM2; ++m) {
      const int k = m * 128 + q * 32 + lane;
      const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16);
      float* outP = a.P + (size_t)blockIdx.x * K * a.d;
      const int h1 = L.ncolsZ / 2;
      for (int c0 = half * h1; c0 < (half + 1) * h1; c0 += 8) {
        float v[8];
        tc::tmem_ld8(tl + (uint32_t)(m * L.ncolsZ + c0), v);
        tc::tmem_ld_wait();
        if (k < K)
#pragma unroll
          for (int i = 0; i < 8; ++i)
            if (c0 + i < a.d) outP[(size_t)k * a.d + c0 + i] = nt > 0 ? v[i] : 0.f;
      }
      float* outO = a.Opart + (size_t)blockIdx.x * a.nkeys * K;
      const int h2 = (L.nkpad / 2 + 7) / 8 * 8;
      for (int c0 = half * h2; c0 < min(L.nkpad, (half + 1) * h2); c0 += 8) {
        float v[8];
        tc::tmem_ld8(tl + (uint32_t)(L.nM2 * L.ncolsZ + m * L.nkpad + c0), v);
        tc::tmem_ld_wait();
        if (k < K)
#pragma unroll
          for (int i = 0; i < 8; ++i)
            if (c0 + i < a.nkeys) outO[(size_t)(c0 + i) * K + k] = nt > 0 ? v[i] : 0.f;
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)L.tcols);
  }
}

// Both reductions of the per-CTA partials in one launch (one wave), 32 x kRedY threads per
// CTA; threadIdx.y takes every kRedY-th CTA partial and the float64 sums are combined in
// shared memory:
//   CTAs 0 .. K-1: centroid row k = blockIdx.x, Y[k] = sum_g P[g][k][:], written L2-normalised
//                  as 16-bit Y_norm (inverse norm capped at 1e12, kernels_normalize.cuh:7-54);
//   the others:    32 consecutive (key, cluster) entries e, Omin[e] = sum_g Opart[g][e].
constexpr int kRedY = 16;
template <typename H>
__global__ void __launch_bounds__(32 * kRedY) k_cs_reduce(const float* __restrict__ P, const float* __restrict__ Opart, int G,
                                                   int K, int d, int nkeys, H* __restrict__ Yn, int ldy,
                                                   double* __restrict__ Omin, const int* stop) {
  if (stop && *(volatile const int*)stop) return;  // the k-means loop has stopped on the device
  __shared__ double part[kRedY][128];
  __shared__ double red[32];
  const int lane = threadIdx.x, y = threadIdx.y, t = y * 32 + lane;
  if ((int)blockIdx.x < K) {
    const int k = blockIdx.x;
    for (int c0 = 0; c0 < d; c0 += 128) {  // d <= 128 on this path: one round
      for (int c = c0 + lane; c < min(d, c0 + 128); c += 32) {
        double s = 0.0;
#pragma unroll 8
        for (int g = y; g < G; g += kRedY) s += (double)__ldg(P + ((size_t)g * K + k) * d + c);
        part[y][c - c0] = s;
      }
    }
    __syncthreads();
    double v = 0.0, ss = 0.0;
    if (t < d) {
#pragma unroll
      for (int q = 0; q < kRedY; ++q) v += part[q][t];
      ss = v * v;
    }
    ss = block_sum(ss, red);
    double inv = rsqrt(ss);
    if (inv > 1e12) inv = 1e12;
    for (int c = t; c < ldy; c += 32 * kRedY) Yn[(size_t)k * ldy + c] = from_f<H>(c < d ? (float)(v * inv) : 0.f);
    return;
  }
  const int64_t ne = (int64_t)nkeys * K;
  const int64_t e = (int64_t)(blockIdx.x - K) * 32 + lane;
  double s = 0.0;
  if (e < ne) {
#pragma unroll 8
    for (int g = y; g < G; g += kRedY) s += (double)__ldg(Opart + (size_t)g * ne + e);
  }
  part[y][lane] = s;
  __syncthreads();
  if (y == 0 && e < ne) {
    double tot = 0.0;
#pragma unroll
    for (int q = 0; q < kRedY; ++q) tot += part[q][lane];
    Omin[e] = tot;
  }
}

// 4-D view {64 values, 8 rows, blocks, 8-row groups} of a [rows][ld] 16-bit array, box {64, 8, blocks, 16}.
int make_tile_map4(CUtensorMap* tm, const void* base, int64_t rows, int ld, int blocks, bool bf16) {
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
  if (((uintptr_t)base & 15) || (ld * 2) % 16 || rows % 8) {
    set_error("tile map: base must be 16-byte aligned, rows a multiple of 16 bytes and of 8");
    return HB_ERR_INVALID;
  }
  cuuint64_t gdim[4] = {64, 8, (cuuint64_t)blocks, (cuuint64_t)(rows / 8)};
  cuuint64_t gstride[3] = {(cuuint64_t)ld * 2, 128, (cuuint64_t)ld * 16};
  cuuint32_t box[4] = {64, 8, (cuuint32_t)blocks, 16};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = encode(tm, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4,
                            const_cast<void*>(base), gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (4-D tile map) failed (%d) for rows=%lld ld=%d", (int)r, (long long)rows, ld);
    return HB_ERR_CUDA;
  }
  return HB_OK;
}

template <typename H>
int launch_tc_centroid_stream(const CenStreamArgs& a, const void* Zn, int ldz, const void* R, int ldr,
                              int64_t rows_alloc, int grid, double* Omin, cudaStream_t st) {
  const CsLayout L = cs_layout(a.d, a.K, a.nkeys, ldz);
  CUtensorMap tmZ, tmR;
  HB_TRY(make_tile_map4(&tmZ, Zn, rows_alloc, ldz, L.nbZ, is_bf16<H>::value));
  HB_TRY(make_tile_map4(&tmR, R, rows_alloc, ldr, L.nbB, is_bf16<H>::value));
  const void* fn = (const void*)k_tc_centroid_stream<H>;
  // one CTA per SM: the request is padded so that a second CTA never fits (TMEM)
  const size_t smem = std::max<size_t>(L.bytes, 116u * 1024u);
  HB_TRY(allow_max_dyn_smem(fn));
  k_tc_centroid_stream<H><<<grid, 256, smem, st>>>(a, L, tmZ, tmR);
  HB_LAUNCH_CHECK();
  const int64_t ne = (int64_t)a.nkeys * a.K;
  k_cs_reduce<H><<<(unsigned)(a.K + (ne + 31) / 32), dim3(32, kRedY), 0, st>>>(a.P, a.Opart, grid, a.K, a.d, a.nkeys,
                                                                        (H*)a.Yn, a.ldy, Omin, a.stop);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_centroid_stream<__half>(const CenStreamArgs&, const void*, int, const void*, int, int64_t,
                                               int, double*, cudaStream_t);
template int launch_tc_centroid_stream<__nv_bfloat16>(const CenStreamArgs&, const void*, int, const void*, int,
                                                      int64_t, int, double*, cudaStream_t);

}  // namespace hb
