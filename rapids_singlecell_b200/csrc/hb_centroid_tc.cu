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
// Pipeline (all 256 threads, one barrier per tile): while tile i is multiplied,
// the row gathers of tiles i+1 .. i+S-1 are in flight (16-byte cp.async copies,
// consecutive threads on consecutive chunks of a row), and the cell ids of the
// tiles after them are loaded one and two tiles ahead.  The (block, batch) sums
// are a second MMA per tile: R_tile^T . I, with I[row][run] = 1 when the row is
// in the run (rows are ordered by key, so a tile holds few runs); the run sums
// are read from TMEM one tile later and added to Omin when the key changes.
//
// Shared layout of one operand tile: 16 groups of 8 cells; a group holds the
// operand's 64-element blocks (1024 bytes each, 128B-swizzled rows of 8
// cells) side by side.  Descriptor: leading byte offset = 1024 (next 64-element
// block), stride byte offset = blocks * 1024 (next 8-cell group).  Only the
// stored columns of a row are copied: the columns past them feed D rows / columns
// that are discarded, and rows past the slice are zero-filled in both operands.
#include "hb_tc_tile.cuh"

namespace hb {

constexpr int kCenRuns = 32;  // runs per tile summed on the tensor core (more: SIMT path)

struct CenLayout {
  int npad, nbA, nbB, tcolsP, nM2, tcols, stages;
  int zch, rch;  // 16-byte chunks stored per Z_norm / R row
  uint32_t stA, stB, offA, offB, offInd, offId, offKey, offMisc, bytes;
};

inline CenLayout cen_layout(int K, int ldz, int ldr) {
  CenLayout L{};
  L.npad = (K + 15) / 16 * 16;
  L.nbB = (L.npad + 127) / 128 * 2;  // the run-sum MMAs (M = 128) read 64-cluster blocks in pairs
  L.tcolsP = L.npad <= 128 ? 128 : 256;
  L.nM2 = (K + 127) / 128;                  // M = 128 MMAs of the run sums
  L.tcols = L.tcolsP + 2 * 64 * L.nM2;      // P, then two run-sum accumulators of 64 columns per MMA
  L.zch = ldz / 8;
  L.rch = ldr / 8;
  // two 64-PC blocks (M = 128) even when the PCs fit in one: a one-block tile whose
  // second block aliases the next 8-cell group produced wrong sums on B200
  L.nbA = 2;
  L.stA = (uint32_t)L.nbA * 16384u;
  L.stB = (uint32_t)L.nbB * 16384u;
  for (int st = 4; st >= 2; --st) {
    uint32_t o = 0;
    L.offA = o; o += (uint32_t)st * L.stA;
    L.offB = o; o += (uint32_t)st * L.stB;
    L.offInd = o; o += 2u * 2u * (uint32_t)kCenRuns * 128u;  // two run-indicator tiles [2 K-blocks][32 runs][128 B]
    L.offId = o; o += (uint32_t)(st + 1) * 128u * 4u;   // id and key rings: stages + 1 slots
    L.offKey = o; o += (uint32_t)(st + 1) * 128u * 4u;
    L.offMisc = o; o += 8u * 8u + 16u;
    L.bytes = o + 1024u;  // slack for 1024-byte alignment of the base
    L.stages = st;
    if (L.bytes <= 227u * 1024u) break;
  }
  return L;
}

// byte offset of chunk (block nb, 16B chunk c8) of cell r in a tile with `nblocks` blocks per group
__device__ __forceinline__ uint32_t mn_off(uint32_t r, uint32_t nb, uint32_t c8, uint32_t nblocks) {
  return (r >> 3) * (nblocks * 1024u) + nb * 1024u + (r & 7u) * 128u + ((c8 ^ (r & 7u)) << 4);
}

// Copies of the Z_norm and R rows of one tile (cell ids in `cid`, -1 = zero row).
// Items are (row, chunk) pairs, consecutive threads on consecutive chunks.
template <typename H>
__device__ __forceinline__ void cen_gather(const CenArgs& a, const CenLayout& L, const int* cid,
                                           uint32_t sA, uint32_t sB) {
  const H* Zn = (const H*)a.Zn;
  const H* R = (const H*)a.R;
  {
    const int C = L.zch, dr = 256 / C, dc = 256 % C;
    int r = threadIdx.x / C, ch = threadIdx.x % C;
    for (; r < 128;) {
      const int cell = cid[r];
      const bool ok = cell >= 0;
      tc::cp_async16(sA + mn_off((uint32_t)r, (uint32_t)(ch >> 3), (uint32_t)(ch & 7), 2u),
                     ok ? (const void*)(Zn + (int64_t)cell * a.ldz + ch * 8) : (const void*)Zn, ok ? 16u : 0u);
      r += dr;
      ch += dc;
      if (ch >= C) { ch -= C; ++r; }
    }
  }
  {
    const int C = L.rch, dr = 256 / C, dc = 256 % C;
    int r = threadIdx.x / C, ch = threadIdx.x % C;
    for (; r < 128;) {
      const int cell = cid[r];
      const bool ok = cell >= 0;
      tc::cp_async16(sB + mn_off((uint32_t)r, (uint32_t)(ch >> 3), (uint32_t)(ch & 7), (uint32_t)L.nbB),
                     ok ? (const void*)(R + (int64_t)cell * a.ldr + ch * 8) : (const void*)R, ok ? 16u : 0u);
      r += dr;
      ch += dc;
      if (ch >= C) { ch -= C; ++r; }
    }
  }
}

// Runs of equal (block, batch) key in one tile: starts (ascending, terminated by
// the row count), their keys, their number; simt = more than kCenRuns runs.
struct TileRuns {
  int start[kCenRuns + 1];
  int key[kCenRuns];
  int n, simt;
};

// Warp 0: runs of a tile from its row keys, and the indicator operand
// I[row][run] (K-major, 128B-swizzled: two 64-row blocks of kCenRuns run rows).
template <typename H>
__device__ __forceinline__ void cen_runs(const int* kr, TileRuns& tr, unsigned char* ind) {
  const int lane = threadIdx.x & 31;
  int cnt = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = i * 32 + lane;
    const int k = kr[r];
    const bool start = k >= 0 && (r == 0 || kr[r - 1] != k);
    const unsigned m = __ballot_sync(0xffffffffu, start);
    const int at = cnt + __popc(m & lanemask_lt());
    if (start && at < kCenRuns) {
      tr.start[at] = r;
      tr.key[at] = k;
    }
    cnt += __popc(m);
  }
  int nr = 0;  // valid rows (keys of rows past the slice are -1, at the end)
#pragma unroll
  for (int i = 0; i < 4; ++i) nr += __popc(__ballot_sync(0xffffffffu, kr[i * 32 + lane] >= 0));
  const int n = min(cnt, kCenRuns);
  if (lane == 0) {
    tr.start[n] = nr;
    tr.n = n;
    tr.simt = cnt > kCenRuns;
  }
  __syncwarp();
  if (cnt > kCenRuns) return;
  const int n16 = (n + 15) / 16 * 16;
  const H one = from_f<H>(1.f), zero = from_f<H>(0.f);
  for (int e = lane; e < n16 * 16; e += 32) {
    const int q = e >> 4, kb = (e >> 3) & 1, c = e & 7;
    const int r0 = kb * 64 + c * 8;
    const int s = q < n ? tr.start[q] : 0, t = q < n ? tr.start[q + 1] : 0;
    __align__(16) H v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (r0 + i >= s && r0 + i < t) ? one : zero;
    *(uint4*)(ind + kb * (kCenRuns * 128) + tc::sw128_off((uint32_t)q, (uint32_t)c)) = *(const uint4*)v;
  }
  tc::fence_proxy_async_smem();
}

// Running (key, sum) of one cluster over the runs it sees, and the running sum of the
// key's block (key (block, B): the block's column sums); each flushed to Omin with a
// float64 atomic when its key changes.
struct RunAcc {
  int key = -1, bkey = -1;
  double acc = 0.0, bacc = 0.0;
  __device__ __forceinline__ void add(const CenArgs& a, int kc, int k, double v) {
    if (k != key) {
      if (key >= 0 && acc != 0.0) atomicAdd(&a.Omin[(size_t)key * a.K + kc], acc);
      key = k;
      acc = 0.0;
      const int bk = k - k % (a.B + 1) + a.B;
      if (bk != bkey) {
        if (bkey >= 0 && bacc != 0.0) atomicAdd(&a.Omin[(size_t)bkey * a.K + kc], bacc);
        bkey = bk;
        bacc = 0.0;
      }
    }
    acc += v;
    bacc += v;
  }
  __device__ __forceinline__ void flush(const CenArgs& a, int kc) {
    if (key >= 0 && acc != 0.0) atomicAdd(&a.Omin[(size_t)key * a.K + kc], acc);
    if (bkey >= 0 && bacc != 0.0) atomicAdd(&a.Omin[(size_t)bkey * a.K + kc], bacc);
    key = bkey = -1;
    acc = bacc = 0.0;
  }
};

template <typename H>
__global__ void __launch_bounds__(256, 1) k_tc_centroid(CenArgs a, CenLayout L) {
  if (a.stop && *(volatile const int*)a.stop) return;  // the k-means loop has stopped on the device
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int K = a.K, S = L.stages, NS = L.stages + 1;
  int* ids = (int*)(sm + L.offId);     // [NS][128] cell id per row
  int* keys = (int*)(sm + L.offKey);   // [NS][128] (block, batch) key per row
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);  // [S] MMAs of the stage's tile completed
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 64);
  __shared__ TileRuns truns[3];
  const uint32_t sm32 = tc::smem_u32(sm);
  const int64_t lo = a.n * blockIdx.x / gridDim.x, hi = a.n * (blockIdx.x + 1) / gridDim.x;
  const int ntiles = (int)((hi - lo + 127) / 128);
  // id and key of row r of tile t (-1 past the slice)
  auto load_row = [&](int t, int r, int& cell, int& key) {
    cell = -1;
    key = -1;
    const int64_t p = lo + (int64_t)t * 128 + r;
    if (t < ntiles && p < hi) {
      cell = __ldg(a.idx + p);
      key = (int)(p / a.bs) * (a.B + 1) + __ldg(a.lcat + p);
    }
  };
  auto mma_done = [&](int t) {  // wait for the MMAs of tile t
    if (!tc::mbar_wait(mbar + t % S, (uint32_t)((t / S) & 1), kMaxPolls)) atomicExch(a.err, 5);
  };

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) tc::mbar_init(mbar + s, 1);
    tc::fence_mbar_init();
  }
  int pcell = -1, pkey = -1;  // prefetched row of a later tile (threads < 128)
  if (tid < 128) {
    for (int t = 0; t < S; ++t) {
      int c, k;
      load_row(t, tid, c, k);
      ids[t * 128 + tid] = c;
      keys[t * 128 + tid] = k;
    }
    load_row(S, tid, pcell, pkey);
  }
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  for (int t = 0; t < S - 1; ++t) {
    if (t < ntiles) cen_gather<H>(a, L, ids + t * 128, sm32 + L.offA + t * L.stA, sm32 + L.offB + t * L.stB);
    tc::cp_async_commit();
  }
  if (warp == 0 && ntiles > 0) cen_runs<H>(keys, truns[0], sm + L.offInd);
  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, true, true);
  // run-sum readers: warp w reads TMEM lanes 32 (w % 4) of MMA w / 4 (clusters 128 (w/4) + lane row)
  const int rd_m = warp >> 2, rd_c = rd_m * 128 + (warp & 3) * 32 + lane;
  const bool reader = rd_m < L.nM2;
  RunAcc racc;
  // SIMT path of tiles with many runs: thread (part, kc) owns column kc for a row range
  const int np = K < 256 ? 256 / K : 1;
  const int part = tid / K, kc = tid % K;
  const int sr0 = part * 128 / np, sr1 = (part + 1) * 128 / np;
  RunAcc sacc;

  auto read_runs = [&](int t) {  // add the run sums of tile t (its MMAs completed)
    const TileRuns& tr = truns[t % 3];
    if (tr.simt || !reader) return;
    const uint32_t col = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)L.tcolsP +
                         (uint32_t)((t & 1) * 64 * L.nM2 + rd_m * 64);
    for (int q0 = 0; q0 < tr.n; q0 += 8) {
      float v[8];
      tc::tmem_ld8(col + (uint32_t)q0, v);
      tc::tmem_ld_wait();
      if (rd_c < K)
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (q0 + i < tr.n) racc.add(a, rd_c, tr.key[q0 + i], (double)v[i]);
    }
  };

  for (int i = 0; i < ntiles; ++i) {
    const int s = i % S;
    // tile i has landed (the later S-2 tiles may still be in flight)
    if (S >= 4) tc::cp_async_wait_group<2>();
    else if (S == 3) tc::cp_async_wait_group<1>();
    else tc::cp_async_wait_group<0>();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t sBs = sm32 + L.offB + s * L.stB;
    if (tid == 0) {
      for (int k = 0; k < 8; ++k) {  // P += Z_tile^T R_tile, 8 steps of 16 cells
        const uint64_t ad = tc::sdesc_sw128(sm32 + L.offA + s * L.stA + (uint32_t)k * 2u * (uint32_t)L.nbA * 1024u,
                                            1024, (uint32_t)L.nbA * 1024u);
        const uint64_t bd = tc::sdesc_sw128(sBs + (uint32_t)k * 2u * (uint32_t)L.nbB * 1024u, 1024,
                                            (uint32_t)L.nbB * 1024u);
        tc::mma_f16(tmem, ad, bd, idesc, (i > 0 || k > 0) ? 1u : 0u);
      }
      const TileRuns& tr = truns[i % 3];
      if (!tr.simt && tr.n > 0) {  // run sums: D2[cluster][run] = R_tile^T I
        const int n16 = (tr.n + 15) / 16 * 16;
        const uint32_t idesc2 = tc::idesc_f16(128, n16, is_bf16<H>::value, true, false);
        const uint32_t sI = sm32 + L.offInd + (uint32_t)(i & 1) * 2u * kCenRuns * 128u;
        for (int m = 0; m < L.nM2; ++m) {
          const uint32_t d2 = tmem + (uint32_t)L.tcolsP + (uint32_t)((i & 1) * 64 * L.nM2 + m * 64);
          for (int k = 0; k < 8; ++k) {
            const uint64_t ad = tc::sdesc_sw128(sBs + (uint32_t)(2 * m) * 1024u + (uint32_t)k * 2u * (uint32_t)L.nbB * 1024u,
                                                1024, (uint32_t)L.nbB * 1024u);
            const uint64_t bd = tc::sdesc_sw128(sI + (uint32_t)(k >> 2) * (kCenRuns * 128u) + (uint32_t)(k & 3) * 32u, 16,
                                                1024);
            tc::mma_f16(d2, ad, bd, idesc2, k > 0 ? 1u : 0u);
          }
        }
      }
      tc::mma_commit(mbar + s);
    }
    // the MMAs of tile i-1 are done: its stage, run sums and indicator tile are free
    if (i >= 1) {
      mma_done(i - 1);
      tc::fence_after_sync();
      read_runs(i - 1);
    }
    // gathers of tile i+S-1 into the stage of tile i-1
    const int tn = i + S - 1;
    if (tn < ntiles) cen_gather<H>(a, L, ids + (tn % NS) * 128, sm32 + L.offA + (tn % S) * L.stA,
                                   sm32 + L.offB + (tn % S) * L.stB);
    tc::cp_async_commit();
    // ids of tile i+S into its slot (that of tile i-1); prefetch those of tile i+S+1
    if (tid < 128) {
      ids[((i + S) % NS) * 128 + tid] = pcell;
      keys[((i + S) % NS) * 128 + tid] = pkey;
      load_row(i + S + 1, tid, pcell, pkey);
    }
    // runs and indicator tile of tile i+1 (its keys were stored before this tile's barrier)
    if (warp == 0 && i + 1 < ntiles)
      cen_runs<H>(keys + ((i + 1) % NS) * 128, truns[(i + 1) % 3], sm + L.offInd + ((i + 1) & 1) * 2 * kCenRuns * 128);
    // tiles with many runs: per-row sums by column owners
    if (truns[i % 3].simt && part < np && kc < K) {
      const int* kr = keys + (i % NS) * 128;
      const unsigned char* tb = sm + L.offB + s * L.stB + (kc >> 6) * 1024;
      const uint32_t c8 = (uint32_t)((kc & 63) >> 3);
      for (int r = sr0; r < sr1; ++r) {
        const int k = kr[r];
        if (k < 0) break;
        const float v = h2f(*(const H*)(tb + (r >> 3) * L.nbB * 1024 + (r & 7) * 128 + ((c8 ^ (uint32_t)(r & 7)) << 4) +
                                        (kc & 7) * 2));
        sacc.add(a, kc, k, (double)v);
      }
    }
  }
  if (ntiles > 0) {
    mma_done(ntiles - 1);
    tc::fence_after_sync();
    read_runs(ntiles - 1);
  }
  if (reader && rd_c < K) racc.flush(a, rd_c);
  if (part < np && kc < K) sacc.flush(a, kc);
  // ---- epilogue: partial D[pc][cluster] -> P[cta][cluster][pc] -------------------------
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
  const CenLayout L = cen_layout(a.K, a.ldz, a.ldr);
  if (a.d > 128 || a.K > 256 || L.bytes > 227u * 1024u) {
    set_error("tensor-core centroid pass: unsupported shape (d=%d K=%d)", a.d, a.K);
    return HB_ERR_UNSUPPORTED;
  }
  const void* fn = (const void*)k_tc_centroid<H>;
  // one CTA per SM: the request is padded so that a second CTA never fits (TMEM)
  const size_t smem = std::max<size_t>(L.bytes, 116u * 1024u);
  HB_TRY(allow_max_dyn_smem(fn));
  k_tc_centroid<H><<<grid, 256, smem, st>>>(a, L);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_centroid<__half>(const CenArgs&, int, cudaStream_t);
template int launch_tc_centroid<__nv_bfloat16>(const CenArgs&, int, cudaStream_t);

int tc_centroid_grid(int K) {
  (void)K;
  return num_sms();
}

}  // namespace hb
