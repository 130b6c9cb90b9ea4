// Tensor-core ridge correction of the 16-bit path (correction_batched.cu:17-130).
//
// Moments: M[b][k][:] = sum over the cells of batch b of R[cell][k] X[cell][:],
// one CTA per run of cells of one batch (the split-n chunks of the batch-sorted
// cell list), D[k][pc] = R_tile^T X_tile accumulated in TMEM over the chunk's
// 128-cell tiles; the chunk partials are summed per batch by k_m_reduce.
// Apply: Z_hat = X - R W[batch] for 128-cell tiles of one batch, D[cell][pc] =
// R_tile W_b on the tensor core, then Z_hat and its L2-normalised 16-bit copy
// (the next iteration's Z_norm) in the epilogue.
//
// X and W are float32.  The tensor core takes both operands in the 16-bit type
// of R, so each float32 operand is split into hi + lo 16-bit parts (hi = x
// rounded, lo = x - hi rounded) and multiplied twice; with R exact in 16 bits
// the products keep ~16 significant bits of X and W, accumulated in float32.
// In fp16 the split needs |x| < 65504: larger values set error code 7.
#include "hb_tc_tile.cuh"

namespace hb {
namespace {

// byte offset of chunk (64-element block nb, 16-byte chunk c8) of row r in an
// MN-major tile with `nblocks` blocks per 8-row group
__device__ __forceinline__ uint32_t mn_off(uint32_t r, uint32_t nb, uint32_t c8, uint32_t nblocks) {
  return (r >> 3) * (nblocks * 1024u) + nb * 1024u + (r & 7u) * 128u + ((c8 ^ (r & 7u)) << 4);
}

// hi / lo 16-bit parts of 8 float32 values; flags values outside the fp16 range
template <typename H>
__device__ __forceinline__ void split8(const float (&x)[8], H (&hi)[8], H (&lo)[8], bool& bad) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (!is_bf16<H>::value && fabsf(x[i]) >= 65504.f) bad = true;
    hi[i] = from_f<H>(x[i]);
    lo[i] = from_f<H>(x[i] - h2f(hi[i]));
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Moments
struct MomLayout {
  int nM, nbR, nbX, ncols, tcols;
  uint32_t offR, offXh, offXl, offId, offMisc, bytes;
};

inline MomLayout mom_layout(int K, int d) {
  MomLayout L{};
  L.nM = (K + 127) / 128;
  L.nbR = 2 * L.nM;              // 64-cluster blocks, in pairs (M = 128 per MMA)
  L.nbX = (d + 63) / 64;         // 64-PC blocks (N = 64 nbX)
  L.ncols = 64 * L.nbX;
  int t = 32;
  while (t < L.nM * L.ncols) t <<= 1;
  L.tcols = t;
  uint32_t o = 0;
  L.offR = o; o += (uint32_t)L.nbR * 16384u;
  L.offXh = o; o += (uint32_t)L.nbX * 16384u;
  L.offXl = o; o += (uint32_t)L.nbX * 16384u;
  L.offId = o; o += 128u * 4u;
  L.offMisc = o; o += 16u;
  L.bytes = o + 1024u;
  return L;
}

template <typename H>
__global__ void __launch_bounds__(256) k_tc_moments(const H* __restrict__ R, int ldr, const float* __restrict__ X,
                                                    int ldx, const int32_t* __restrict__ cell_index,
                                                    const AccumChunk* __restrict__ chunks, int K, int d,
                                                    float* __restrict__ Mpart, MomLayout L, int* err,
                                                    const int* gate) {
  if (gated(gate)) return;  // before the TMEM allocation: every thread of the CTA returns
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int* ids = (int*)(sm + L.offId);
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  const uint32_t sm32 = tc::smem_u32(sm);
  const AccumChunk ch = chunks[blockIdx.x];
  const int ntiles = (ch.len + 127) / 128;
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
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
  const uint32_t idesc = tc::idesc_f16(128, L.ncols, is_bf16<H>::value, true, true);
  const int rch = ldr / 8, xch = L.nbX * 8;
  bool bad = false;
  for (int t = 0; t < ntiles; ++t) {
    const int nr = min(128, ch.len - t * 128);
    if (tid < 128) ids[tid] = tid < nr ? cell_index[ch.start + (int64_t)t * 128 + tid] : -1;
    __syncthreads();
    // R rows (MN-major: clusters contiguous), zero rows past the chunk
    for (int e = tid; e < 128 * rch; e += 256) {
      const int r = e / rch, c = e % rch;
      const int cell = ids[r];
      tc::cp_async16(sm32 + L.offR + mn_off((uint32_t)r, (uint32_t)(c >> 3), (uint32_t)(c & 7), (uint32_t)L.nbR),
                     cell >= 0 ? (const void*)(R + (int64_t)cell * ldr + c * 8) : (const void*)R,
                     cell >= 0 ? 16u : 0u);
    }
    // X rows split into hi / lo parts (MN-major: PCs contiguous), zero past d
    for (int e = tid; e < 128 * xch; e += 256) {
      const int r = e / xch, c = e % xch;
      const int cell = ids[r];
      float x[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int col = c * 8 + i;
        x[i] = (cell >= 0 && col < d) ? __ldg(X + (int64_t)cell * ldx + col) : 0.f;
      }
      __align__(16) H hi[8], lo[8];
      split8<H>(x, hi, lo, bad);
      const uint32_t off = mn_off((uint32_t)r, (uint32_t)(c >> 3), (uint32_t)(c & 7), (uint32_t)L.nbX);
      *(uint4*)(sm + L.offXh + off) = *(const uint4*)hi;
      *(uint4*)(sm + L.offXl + off) = *(const uint4*)lo;
    }
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      for (int ks = 0; ks < 8; ++ks) {  // 8 steps of 16 cells
        const uint64_t bh = tc::sdesc_sw128(sm32 + L.offXh + (uint32_t)ks * 2u * L.nbX * 1024u, 1024,
                                            (uint32_t)L.nbX * 1024u);
        const uint64_t bl = tc::sdesc_sw128(sm32 + L.offXl + (uint32_t)ks * 2u * L.nbX * 1024u, 1024,
                                            (uint32_t)L.nbX * 1024u);
        for (int m = 0; m < L.nM; ++m) {
          const uint64_t ad = tc::sdesc_sw128(sm32 + L.offR + (uint32_t)(2 * m) * 1024u + (uint32_t)ks * 2u * L.nbR * 1024u,
                                              1024, (uint32_t)L.nbR * 1024u);
          const uint32_t dcol = tmem + (uint32_t)(m * L.ncols);
          tc::mma_f16(dcol, ad, bh, idesc, (t > 0 || ks > 0) ? 1u : 0u);
          tc::mma_f16(dcol, ad, bl, idesc, 1u);
        }
      }
      tc::mma_commit(mbar);
    }
    // the tile's buffers are rewritten by the next tile: wait for its MMAs
    if (!tc::mbar_wait(mbar, (uint32_t)(t & 1), kMaxPolls)) atomicExch(err, 8);
    tc::fence_after_sync();
  }
  if (bad) atomicExch(err, 7);
  // D[k][pc] -> Mpart[chunk][k][pc]; warps 4-7 take the second 128 clusters, or the
  // second half of the PC columns when there is one cluster block
  {
    const int m = L.nM == 2 ? (warp >> 2) : 0;
    const int k = m * 128 + (warp & 3) * 32 + lane;
    const int c_lo = L.nM == 2 ? 0 : (warp >> 2) * (L.ncols / 2);
    const int c_hi = L.nM == 2 ? L.ncols : c_lo + L.ncols / 2;
    const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(m * L.ncols);
    float* out = Mpart + (size_t)blockIdx.x * K * d;
    for (int c0 = c_lo; c0 < c_hi; c0 += 8) {
      float v[8];
      tc::tmem_ld8(tl + (uint32_t)c0, v);
      tc::tmem_ld_wait();
      if (k < K)
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (c0 + i < d) out[(size_t)k * d + c0 + i] = ntiles > 0 ? v[i] : 0.f;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)L.tcols);
  }
}

template <typename H>
int launch_tc_moments(const H* R, int ldr, const float* X, int ldx, const int32_t* cell_index,
                      const AccumChunk* chunks, int n_chunks, int K, int d, float* Mpart, int* err,
                      cudaStream_t st, const int* gate) {
  if (n_chunks == 0) return HB_OK;
  if (K > 256 || d > 256) {
    set_error("tensor-core correction: unsupported shape (K=%d d=%d)", K, d);
    return HB_ERR_UNSUPPORTED;
  }
  const MomLayout L = mom_layout(K, d);
  const void* fn = (const void*)k_tc_moments<H>;
  HB_TRY(allow_max_dyn_smem(fn));
  k_tc_moments<H><<<n_chunks, 256, L.bytes, st>>>(R, ldr, X, ldx, cell_index, chunks, K, d, Mpart, L, err,
                                                                gate);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_moments<__half>(const __half*, int, const float*, int, const int32_t*, const AccumChunk*,
                                       int, int, int, float*, int*, cudaStream_t, const int*);
template int launch_tc_moments<__nv_bfloat16>(const __nv_bfloat16*, int, const float*, int, const int32_t*,
                                              const AccumChunk*, int, int, int, float*, int*, cudaStream_t,
                                              const int*);

// ---------------------------------------------------------------------------
// Apply
struct ApLayout {
  int npad, kblk, nbX, ncols, tcols, ldxs;
  uint32_t offA, offWh, offWl, offX, offId, offSs, offMisc, bytes;
};

inline ApLayout ap_layout(int K, int d) {
  ApLayout L{};
  L.npad = (K + 15) / 16 * 16;   // MMA K extent (clusters)
  L.kblk = (L.npad + 63) / 64;   // 64-cluster blocks of the K-major R tile
  L.nbX = (d + 63) / 64;
  L.ncols = 64 * L.nbX;
  int t = 32;
  while (t < L.ncols) t <<= 1;
  L.tcols = t;
  uint32_t o = 0;
  L.offA = o; o += (uint32_t)L.kblk * 16384u;
  const uint32_t wt = (uint32_t)(L.npad / 8) * L.nbX * 1024u;  // npad rows of W_b, MN-major
  L.offWh = o; o += wt;
  L.offWl = o; o += wt;
  L.ldxs = d + 1;  // odd row stride: a warp reading one column of 32 rows hits 32 banks
  L.offX = o; o += 128u * (uint32_t)L.ldxs * 4u;
  L.offId = o; o += 128u * 4u;
  L.offSs = o; o += 3u * 128u * 4u;
  L.offMisc = o; o += 16u;
  L.bytes = o + 1024u;
  return L;
}

template <typename H>
__global__ void __launch_bounds__(256, 2) k_tc_apply(const float* __restrict__ X, int ldx, const H* __restrict__ R,
                                                  int ldr, const float* __restrict__ W,
                                                  const int32_t* __restrict__ cell_index,
                                                  const ApplyTile* __restrict__ tiles, int n_tiles, int K, int d,
                                                  float* __restrict__ Zhat, int ldzh, H* __restrict__ Zn, int ldz,
                                                  ApLayout L, int* err, const int* gate) {
  if (gated(gate)) return;  // before the TMEM allocation: every thread of the CTA returns
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int* ids = (int*)(sm + L.offId);
  float* ssp = (float*)(sm + L.offSs);  // [2][128] row sums of squares of the column halves
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  const uint32_t sm32 = tc::smem_u32(sm);
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
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
  const uint32_t idesc = tc::idesc_f16(128, L.ncols, is_bf16<H>::value, false, true);
  const int t0 = (int)((int64_t)n_tiles * blockIdx.x / gridDim.x);
  const int t1 = (int)((int64_t)n_tiles * (blockIdx.x + 1) / gridDim.x);
  const int xch = L.nbX * 8, rch = L.npad / 8;
  const int half = warp >> 2, row = (warp & 3) * 32 + lane;
  const int hc = L.ncols / 2;  // columns per half
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  int cur_b = -1;
  bool bad = false;
  uint32_t phase = 0;
  // the tile descriptor and row ids of the next tile are loaded a tile ahead (registers)
  ApplyTile nxt = t0 < t1 ? tiles[t0] : ApplyTile{0, 0, 0};
  int nid = (t0 < t1 && tid < nxt.len) ? cell_index[nxt.start + tid] : -1;
  for (int t = t0; t < t1; ++t) {
    const ApplyTile tile = nxt;
    if (tile.batch != cur_b) {
      // W_b (clusters x PCs) split into hi / lo parts; MN-major B operand, rows past K zero
      cur_b = tile.batch;
      const float* Wb = W + (size_t)cur_b * K * d;
      constexpr int kWB = 4;  // (cluster, 8-PC chunk) items whose loads are in flight together
      for (int e0 = tid; e0 < L.npad * xch; e0 += 256 * kWB) {
        float x[kWB][8];
#pragma unroll
        for (int u = 0; u < kWB; ++u) {
          const int e = e0 + u * 256;
          const int k = e / xch, c = e % xch;
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int col = c * 8 + i;
            x[u][i] = (e < L.npad * xch && k < K && col < d) ? __ldg(Wb + (size_t)k * d + col) : 0.f;
          }
        }
#pragma unroll
        for (int u = 0; u < kWB; ++u) {
          const int e = e0 + u * 256;
          if (e < L.npad * xch) {
            const int k = e / xch, c = e % xch;
            __align__(16) H hi[8], lo[8];
            split8<H>(x[u], hi, lo, bad);
            const uint32_t off = mn_off((uint32_t)k, (uint32_t)(c >> 3), (uint32_t)(c & 7), (uint32_t)L.nbX);
            *(uint4*)(sm + L.offWh + off) = *(const uint4*)hi;
            *(uint4*)(sm + L.offWl + off) = *(const uint4*)lo;
          }
        }
      }
    }
    if (tid < 128) ids[tid] = nid;
    __syncthreads();
    // R rows, K-major A tile (zero past ldr and for missing rows)
    for (int e = tid; e < 128 * rch; e += 256) {
      const int r = e / rch, c = e % rch;
      const int cell = ids[r];
      const bool ok = cell >= 0 && c * 8 < ldr;
      tc::cp_async16(sm32 + L.offA + (uint32_t)(c >> 3) * 16384u + tc::sw128_off((uint32_t)r, (uint32_t)(c & 7)),
                     ok ? (const void*)(R + (int64_t)cell * ldr + c * 8) : (const void*)R, ok ? 16u : 0u);
    }
    // X rows of the tile (consecutive threads on consecutive columns of a row), all copies in
    // flight at once with the R rows (zero for missing rows)
    {
      const uint32_t sX32 = sm32 + L.offX;
      const int dr = 256 / d, dc = 256 % d;
      int r = tid / d, c = tid % d;
      for (; r < 128;) {
        const int cell = ids[r];
        tc::cp_async4(sX32 + (uint32_t)(r * L.ldxs + c) * 4u,
                      cell >= 0 ? (const void*)(X + (int64_t)cell * ldx + c) : (const void*)X, cell >= 0 ? 4u : 0u);
        r += dr;
        c += dc;
        if (c >= d) { c -= d; ++r; }
      }
    }
    if (t + 1 < t1) {  // the next tile's descriptor and ids, in flight with this tile's copies
      nxt = tiles[t + 1];
      nid = tid < nxt.len ? cell_index[nxt.start + tid] : -1;
    }
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      for (int ks = 0; ks < L.npad / 16; ++ks) {  // 16 clusters per step
        const uint64_t ad = tc::sdesc_sw128(sm32 + L.offA + (uint32_t)(ks >> 2) * 16384u + (uint32_t)(ks & 3) * 32u,
                                            16, 1024);
        const uint64_t bh = tc::sdesc_sw128(sm32 + L.offWh + (uint32_t)ks * 2u * L.nbX * 1024u, 1024,
                                            (uint32_t)L.nbX * 1024u);
        const uint64_t bl = tc::sdesc_sw128(sm32 + L.offWl + (uint32_t)ks * 2u * L.nbX * 1024u, 1024,
                                            (uint32_t)L.nbX * 1024u);
        tc::mma_f16(tmem, ad, bh, idesc, ks > 0 ? 1u : 0u);
        tc::mma_f16(tmem, ad, bl, idesc, 1u);
      }
      tc::mma_commit(mbar);
    }
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(err, 8);
    phase ^= 1u;
    tc::fence_after_sync();
    // epilogue: z = X - D in shared memory, the row's L2 norm over both column halves, then
    // Z_hat and Z_norm with coalesced stores (consecutive threads on consecutive columns)
    float* sX = (float*)(sm + L.offX);
    float* sinv = ssp + 256;
    {
      float ss = 0.f;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (q * 8 < hc) {
          const int c0 = half * hc + q * 8;
          float v[8];
          tc::tmem_ld8(tl + (uint32_t)c0, v);
          tc::tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int c = c0 + i;
            if (c < d) {
              const float zz = sX[row * L.ldxs + c] - v[i];
              sX[row * L.ldxs + c] = zz;
              ss = fmaf(zz, zz, ss);
            }
          }
        }
      }
      ssp[half * 128 + row] = ss;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 128) {
      float inv = rsqrtf(ssp[tid] + ssp[128 + tid]);
      sinv[tid] = inv > 1e12f ? 1e12f : inv;
    }
    __syncthreads();
    {
      const int dr = 256 / d, dc = 256 % d;
      int r = tid / d, c = tid % d;
      for (; r < tile.len;) {
        Zhat[(int64_t)ids[r] * ldzh + c] = sX[r * L.ldxs + c];
        r += dr;
        c += dc;
        if (c >= d) { c -= d; ++r; }
      }
      const int nch = ldz / 8;
      for (int e = tid; e < tile.len * nch; e += 256) {
        const int rr = e / nch, ch = e - rr * nch;
        const float inv = sinv[rr];
        __align__(16) H h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int cc = ch * 8 + i;
          h[i] = from_f<H>(cc < d ? sX[rr * L.ldxs + cc] * inv : 0.f);
        }
        *(uint4*)(Zn + (int64_t)ids[rr] * ldz + ch * 8) = *(const uint4*)h;
      }
    }
    __syncthreads();  // ids, sX and the TMEM accumulator are reused by the next tile
  }
  if (bad) atomicExch(err, 7);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)L.tcols);
  }
}

template <typename H>
int launch_tc_apply(const float* X, int ldx, const H* R, int ldr, const float* W, const int32_t* cell_index,
                    const ApplyTile* tiles, int n_tiles, int K, int d, float* Zhat, int ldzh, H* Zn, int ldz,
                    int* err, cudaStream_t st, const int* gate) {
  if (n_tiles == 0) return HB_OK;
  if (K > 256 || d > 128) {
    set_error("tensor-core correction: unsupported shape (K=%d d=%d)", K, d);
    return HB_ERR_UNSUPPORTED;
  }
  const ApLayout L = ap_layout(K, d);
  const void* fn = (const void*)k_tc_apply<H>;
  HB_TRY(allow_max_dyn_smem(fn));
  // CTAs per SM by shared memory (the occupancy query counts one per SM for a TMEM-allocating
  // kernel); at most 512 / tcols so that the TMEM allocations always fit
  const int per_sm = std::max(1, std::min<int>(512 / L.tcols, (int)(233472u / (L.bytes + 2048u))));
  const int grid = std::max(1, std::min(n_tiles, num_sms() * per_sm));
  k_tc_apply<H><<<grid, 256, L.bytes, st>>>(X, ldx, R, ldr, W, cell_index, tiles, n_tiles, K, d, Zhat, ldzh, Zn,
                                             ldz, L, err, gate);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_apply<__half>(const float*, int, const __half*, int, const float*, const int32_t*,
                                     const ApplyTile*, int, int, int, float*, int, __half*, int, int*, cudaStream_t,
                                     const int*);
template int launch_tc_apply<__nv_bfloat16>(const float*, int, const __nv_bfloat16*, int, const float*,
                                            const int32_t*, const ApplyTile*, int, int, int, float*, int,
                                            __nv_bfloat16*, int, int*, cudaStream_t, const int*);

}  // namespace hb
