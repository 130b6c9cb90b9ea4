// Tensor-core centroid pass of the 16-bit path.
//
// Y^T (PCs x clusters) = Z_norm^T . R summed over all cells (the reference runs
// a cuBLAS GEMM, _cuda/harmony/clustering/clustering.cu:272-276).  Each CTA
// walks an even slice of the iteration's block-ordered cell list in tiles of
// 128 cells, gathers the 16-bit Z_norm and R rows into swizzled shared tiles
// (both operands MN-major: the cell index is the reduction dimension), and
// accumulates D[pc][cluster] in TMEM across its whole slice.  The partial D is
// written once per CTA and reduced by k_centroid_reduce.  From the staged R
// tile the CTA also sums the rows per (block, batch): the "remove old
// contribution" terms of the next sweep (clustering.cu:321-332), as Omin.
//
// Shared layout of one operand tile: 16 groups of 8 cells; a group holds the
// operand's 64-element blocks (1024 bytes each, 128B-swizzled rows of 8
// cells) side by side.  Descriptor: leading byte offset = 1024 (next 64-element
// block), stride byte offset = blocks * 1024 (next 8-cell group).
#include "hb_tc_tile.cuh"

namespace hb {

struct CenLayout {
  int npad, nbB, tcols, stages;
  uint32_t offA[3], offB[3], offCid, offCat, offMisc, bytes;
};

inline CenLayout cen_layout(int K) {
  CenLayout L{};
  L.npad = (K + 15) / 16 * 16;
  L.nbB = (L.npad + 63) / 64;
  L.tcols = L.npad <= 128 ? 128 : 256;
  for (int st = 3; st >= 2; --st) {  // as many stages as fit: st-1 gathers in flight
    uint32_t o = 0;
    for (int s = 0; s < 3; ++s) { L.offA[s] = o; if (s < st) o += 2u * 16384u; }
    for (int s = 0; s < 3; ++s) { L.offB[s] = o; if (s < st) o += (uint32_t)L.nbB * 16384u; }
    L.offCid = o; o += 4u * 128u * 4u;   // id ring: stages + 1 slots
    L.offCat = o; o += 4u * 128u * 4u;
    L.offMisc = o; o += 16u;
    // 8 KB of slack: reads stay inside the allocation under either reading of the
    // descriptor's leading / stride offsets (see the layout note above)
    L.bytes = o + 8192u + 1024u;
    L.stages = st;
    if (L.bytes <= 227u * 1024u) break;
  }
  return L;
}

// byte offset of chunk (block nb, 16B chunk c8) of cell r in a tile with `nblocks` blocks per group
__device__ __forceinline__ uint32_t mn_off(uint32_t r, uint32_t nb, uint32_t c8, uint32_t nblocks) {
  return (r >> 3) * (nblocks * 1024u) + nb * 1024u + (r & 7u) * 128u + ((c8 ^ (r & 7u)) << 4);
}

// Producer (warp 0): gather tile `t` into stage `s`.  Lane q takes rows 4q..4q+3:
// it reads their cell ids and batches, records the (block, batch) key of each row,
// and issues one TMA gather of 4 rows per 64-element block of Z_norm and of R.
// Rows past the slice use row index n (out of range: zero fill).
__device__ __forceinline__ void cen_produce(const CenArgs& a, const CenLayout& L, const CUtensorMap* tmZ,
                                            const CUtensorMap* tmR, int64_t pos, int nr, uint32_t sA,
                                            uint32_t sB, uint64_t* full, int* key, int* runs) {
  const int lane = threadIdx.x & 31;
  const uint32_t bytes = 32u * (uint32_t)(2 + L.nbB) * 512u;
  int rows[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = lane * 4 + i;
    int cell = (int)a.n;  // out of range -> zeros
    int k = -1;
    if (r < nr) {
      cell = __ldg(a.idx + pos + r);
      k = (int)((pos + r) / a.bs) * (a.B + 1) + __ldg(a.lcat + pos + r);
    }
    rows[i] = cell;
    key[r] = k;
  }
  // run starts (rows whose key differs from the previous row's), compacted in
  // ascending row order: round i looks at rows 32 i + lane.
  // runs[0] = count, runs[1..count] = starts, runs[count+1] = nr
  __syncwarp();
  int cnt = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = i * 32 + lane;
    const bool start = r < nr && (r == 0 || key[r] != key[r - 1]);
    const unsigned m = __ballot_sync(0xffffffffu, start);
    if (start) runs[1 + cnt + __popc(m & ((1u << lane) - 1u))] = r;
    cnt += __popc(m);
  }
  if (lane == 0) {
    runs[0] = cnt;
    runs[1 + cnt] = nr;
  }
  // keys and runs are published by the arrive (release) that follows them
  __syncwarp();
  if (lane == 0) tc::mbar_arrive_expect_tx(full, bytes);
  __syncwarp();
  tc::fence_proxy_async_smem();
  const uint32_t g = (uint32_t)(lane >> 1), ro = (uint32_t)(lane & 1) * 512u;  // 8-row group, half
#pragma unroll
  for (int nb = 0; nb < 2; ++nb)
    tc::tma_gather4(sA + g * 2048u + (uint32_t)nb * 1024u + ro, tmZ, nb * 64, rows[0], rows[1], rows[2],
                    rows[3], full);
  for (int nb = 0; nb < L.nbB; ++nb)
    tc::tma_gather4(sB + g * (uint32_t)L.nbB * 1024u + (uint32_t)nb * 1024u + ro, tmR, nb * 64, rows[0],
                    rows[1], rows[2], rows[3], full);
}

// Warp roles: warp 0 produces (ids, keys, TMA gathers), lane 0 of warp 1 issues the
// MMAs, warps 2-7 (192 threads) consume the staged R rows for the per-(block,
// batch) sums.  Stages pass between roles through mbarriers only:
//   full[s]  : producer arrive + TMA bytes          -> MMA issuer, consumers
//   empty[s] : 6 consumer-warp arrivals + MMA commit -> producer (stage reuse)
//   acc      : final MMA commit                      -> epilogue (TMEM read)
constexpr int CEN_CONSUMER_WARPS = 6;

// One consumer column: sums of R[.., kcol] over runs of equal (block, batch) key.
struct CenColumn {
  int kcol;
  int key;
  double tot;
  const unsigned char* base;  // shared-memory base of the column
  uint32_t c8;
  __device__ __forceinline__ void init(unsigned char* sm, const CenLayout& L, int k) {
    kcol = k;
    key = -1;
    tot = 0.0;
    base = sm + (k >> 6) * 1024 + (k & 7) * 2;
    c8 = (uint32_t)((k & 63) >> 3);
  }
  __device__ __forceinline__ void flush(const CenArgs& a) {
    if (key < 0) return;
    atomicAdd(&a.Omin[(size_t)key * a.K + kcol], tot);  // the sweep keeps no column-sum row
  }
  template <typename H>
  __device__ __forceinline__ void tile(const CenArgs& a, const CenLayout& L, int s, const int* kr,
                                       const int* rl) {
    const unsigned char* tb = base + L.offB[0] + (uint32_t)s * (uint32_t)L.nbB * 16384u;
    const uint32_t gstride = (uint32_t)L.nbB * 1024u;
    const int nrun = rl[0];
    for (int u = 0; u < nrun; ++u) {
      const int r0 = rl[1 + u], r1 = rl[2 + u];
      const int kk = kr[r0];
      if (kk != key) {
        flush(a);
        key = kk;
        tot = 0.0;
      }
      float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
      int r = r0;
#define HB_CEN_VAL(rw)                                                                  \
  h2f(*(const H*)(tb + ((uint32_t)(rw) >> 3) * gstride + ((uint32_t)(rw) & 7u) * 128u + \
                  ((c8 ^ ((uint32_t)(rw) & 7u)) << 4)))
      for (; r + 4 <= r1; r += 4) {
        s0 += HB_CEN_VAL(r);
        s1 += HB_CEN_VAL(r + 1);
        s2 += HB_CEN_VAL(r + 2);
        s3 += HB_CEN_VAL(r + 3);
      }
      for (; r < r1; ++r) s0 += HB_CEN_VAL(r);
#undef HB_CEN_VAL
      tot += (double)((s0 + s1) + (s2 + s3));
    }
  }
};

template <typename H>
__global__ void __launch_bounds__(256, 1) k_tc_centroid(CenArgs a, CenLayout L,
                                                        const __grid_constant__ CUtensorMap tmZ,
                                                        const __grid_constant__ CUtensorMap tmR) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int K = a.K;
  int* keys = (int*)(sm + L.offCat);            // [S][128] (block, batch) key per row
  uint64_t* bars = (uint64_t*)(sm + L.offCid);  // full[3], empty[3], acc
  uint64_t* full = bars;
  uint64_t* empty = bars + 3;
  uint64_t* acc_bar = bars + 6;
  int* runs = (int*)(sm + L.offCid + 64);         // [3][130] per-stage run lists
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  // stage s: A tile at offA[0] + s * 32 KB, B tile at offB[0] + s * nbB * 16 KB
  const uint32_t sm32 = tc::smem_u32(sm);
  const uint32_t aStride = 2u * 16384u, bStride = (uint32_t)L.nbB * 16384u;
  const int S = L.stages;
  const int64_t lo = a.n * blockIdx.x / gridDim.x, hi = a.n * (blockIdx.x + 1) / gridDim.x;
  const int ntiles = (int)((hi - lo + 127) / 128);
  auto tile_rows = [&](int t) { const int64_t p = lo + (int64_t)t * 128; return (int)(hi - p < 128 ? hi - p : 128); };

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      tc::mbar_init(full + s, 1);
      tc::mbar_init(empty + s, CEN_CONSUMER_WARPS + 1);
    }
    tc::mbar_init(acc_bar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---- producer ----------------------------------------------------------------
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % S;
      if (t >= S && !tc::mbar_wait(empty + s, (uint32_t)((t / S - 1) & 1), kMaxPolls)) atomicExch(a.err, 6);
      cen_produce(a, L, &tmZ, &tmR, lo + (int64_t)t * 128, tile_rows(t), sm32 + L.offA[0] + s * aStride,
                  sm32 + L.offB[0] + s * bStride, full + s, keys + s * 128, runs + s * 130);
    }
  } else if (warp == 1) {
    // ---- MMA issuer ------------------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, true, true);
      for (int t = 0; t < ntiles; ++t) {
        const int s = t % S;
        if (!tc::mbar_wait(full + s, (uint32_t)((t / S) & 1), kMaxPolls)) atomicExch(a.err, 5);
        tc::fence_after_sync();
        for (int k = 0; k < 8; ++k) {  // 8 steps of 16 cells
          const uint64_t ad = tc::sdesc_sw128(sm32 + L.offA[0] + s * aStride + (uint32_t)k * 2u * 2048u, 1024, 2048);
          const uint64_t bd = tc::sdesc_sw128(sm32 + L.offB[0] + s * bStride + (uint32_t)k * 2u * (uint32_t)L.nbB * 1024u,
                                              1024, (uint32_t)L.nbB * 1024u);
          tc::mma_f16(tmem, ad, bd, idesc, (t > 0 || k > 0) ? 1u : 0u);
        }
        tc::mma_commit(empty + s);
      }
      if (ntiles > 0) tc::mma_commit(acc_bar);
    }
  } else {
    // ---- consumers: per-(block, batch) row sums of R ------------------------------
    const int c = tid - 64;
    CenColumn colA, colB;  // columns c and c + 192
    colA.init(sm, L, c);
    colB.init(sm, L, c + 192);
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % S;
      if (!tc::mbar_wait(full + s, (uint32_t)((t / S) & 1), kMaxPolls)) atomicExch(a.err, 5);
      const int* kr = keys + s * 128;
      const int* rl = runs + s * 130;
      if (colA.kcol < K) colA.tile<H>(a, L, s, kr, rl);
      if (colB.kcol < K) colB.tile<H>(a, L, s, kr, rl);
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(empty + s)) : "memory");
    }
    if (colA.kcol < K) colA.flush(a);
    if (colB.kcol < K) colB.flush(a);
  }
  // ---- epilogue: partial D[pc][cluster] -> P[cta][cluster][pc] -------------------------
  if (ntiles > 0 && !tc::mbar_wait(acc_bar, 0, kMaxPolls)) atomicExch(a.err, 4);
  tc::fence_after_sync();
  {
    const int half = warp >> 2, c = (warp & 3) * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const int nh = (L.npad / 2 + 7) / 8 * 8;
    const int k_lo = half * nh, k_hi = min(L.npad, k_lo + nh);
    float* out = a.P + (size_t)blockIdx.x * K * a.d;
    for (int k0 = k_lo; k0 < k_hi; k0 += 8) {
      float v[8];
      tc::tmem_ld8(tl + (uint32_t)k0, v);
      tc::tmem_ld_wait();
      if (c < a.d)
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (k0 + i < K) out[(size_t)(k0 + i) * a.d + c] = ntiles > 0 ? v[i] : 0.f;
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
int launch_tc_centroid(const CenArgs& a, int grid, cudaStream_t st) {
  const CenLayout L = cen_layout(a.K);
  if (a.d > 128 || a.K > 256 || L.bytes > 227u * 1024u) {
    set_error("tensor-core centroid pass: unsupported shape (d=%d K=%d)", a.d, a.K);
    return HB_ERR_UNSUPPORTED;
  }
  const void* fn = (const void*)k_tc_centroid<H>;
  const int occ_tmem = std::max(1, 512 / L.tcols);
  size_t smem = L.bytes;
  if ((228u * 1024u) / (smem + 1024) > (size_t)occ_tmem)
    smem = std::min<size_t>(227u * 1024u, 228u * 1024u / occ_tmem - 2048);
  HB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CUtensorMap tmZ, tmR;
  HB_TRY(make_row_gather_map(&tmZ, a.Zn, a.n, a.ldz, is_bf16<H>::value));
  HB_TRY(make_row_gather_map(&tmR, a.R, a.n, a.ldr, is_bf16<H>::value));
  k_tc_centroid<H><<<grid, 256, smem, st>>>(a, L, tmZ, tmR);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_centroid<__half>(const CenArgs&, int, cudaStream_t);
template int launch_tc_centroid<__nv_bfloat16>(const CenArgs&, int, cudaStream_t);

int tc_centroid_grid(int K) {
  const CenLayout L = cen_layout(K);
  const int per_sm = std::max(1, std::min(512 / L.tcols, (int)((228u * 1024u) / (L.bytes + 1024))));
  return num_sms() * per_sm;
}

}  // namespace hb
