// Block membership of the soft k-means sweep.
//
// The reference shuffles cells once per k-means iteration by sorting
// (pcg_key(i ^ seed), i) with a full CUB radix sort and then walks the sorted
// order in blocks of `block_size` cells (_cuda/harmony/clustering/clustering.cu:
// 292-310).  Only the SET of cells in each block matters to the result, so this
// engine never sorts: keys are recomputed from the cell index on the fly, the
// (nblk-1) block-boundary keys are found by a two-level radix select (a 12-bit
// histogram, then an exact sort of the few candidates that share a boundary
// bin), and a stable partition writes each block's cells in ascending cell
// order.  Everything is batched over up to kMaxIterChunk iterations per launch
// (grid.y = iteration), because keys do not depend on the data.
#include "hb_common.cuh"
#include "hb_internal.h"

namespace hb {

// seed of iteration c of the chunk: an explicit list, or consecutive from seed0
__device__ __forceinline__ uint32_t seed_of(const uint32_t* seeds, uint32_t seed0, int c) {
  return seeds ? seeds[c] : seed0 + (uint32_t)c;
}

// ---------------------------------------------------------------------------
// 1) 12-bit key histogram, one per iteration.
__global__ void k_key_hist(int64_t n, const uint32_t* __restrict__ seeds,
                           uint32_t seed0, uint32_t* __restrict__ hist, const int* gate) {
  if (gated(gate)) return;
  __shared__ uint32_t sh[kNumBins];
  const int c = blockIdx.y;
  const uint32_t seed = seed_of(seeds, seed0, c);
  for (int b = threadIdx.x; b < kNumBins; b += blockDim.x) sh[b] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    atomicAdd(&sh[pcg_key((uint32_t)i, seed) >> kBinShift], 1u);
  }
  __syncthreads();
  uint32_t* h = hist + (size_t)c * kNumBins;
  for (int b = threadIdx.x; b < kNumBins; b += blockDim.x)
    if (sh[b]) atomicAdd(&h[b], sh[b]);
}

// 2) Locate each boundary rank r_j = j*bs in the histogram: bin p_j and the
//    residual rank q_j inside it.  Distinct boundary bins become "slots".
__global__ void k_boundary_bins(int64_t bs, int nb, const uint32_t* __restrict__ hist,
                                int* __restrict__ bnd_slot, uint32_t* __restrict__ bnd_q,
                                int* __restrict__ slot_bin, int* __restrict__ nslots,
                                int16_t* __restrict__ lut, uint32_t* __restrict__ cand_cnt,
                                int max_slots, const int* gate) {
  if (gated(gate)) return;
  __shared__ uint32_t cum[kNumBins];
  __shared__ uint32_t wsum[32];
  __shared__ int pbin[kMaxBlocks];
  const int c = blockIdx.x;
  const uint32_t* h = hist + (size_t)c * kNumBins;
  // exclusive scan of 4096 bins with blockDim == 1024 (4 bins per thread)
  const int t = threadIdx.x;
  uint32_t v[4], s = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) { v[q] = h[t * 4 + q]; s += v[q]; }
  uint32_t incl = s;
  const int lane = t & 31, w = t >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t x = wsum[lane];
    uint32_t xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += y;
    }
    wsum[lane] = xi - x;
  }
  __syncthreads();
  uint32_t run = wsum[w] + incl - s;
#pragma unroll
  for (int q = 0; q < 4; ++q) { cum[t * 4 + q] = run; run += v[q]; }
  int16_t* L = lut + (size_t)c * kNumBins;
  for (int b = t; b < kNumBins; b += blockDim.x) L[b] = -1;
  __syncthreads();
  for (int j = t; j < nb; j += blockDim.x) {
    const uint32_t r = (uint32_t)((int64_t)(j + 1) * bs);
    int lo = 0, hi = kNumBins - 1;  // largest p with cum[p] <= r
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (cum[mid] <= r) lo = mid; else hi = mid - 1;
    }
    pbin[j] = lo;
    bnd_q[(size_t)c * kMaxBlocks + j] = r - cum[lo];
  }
  __syncthreads();
  if (t == 0) {
    int ns = 0;
    for (int j = 0; j < nb; ++j) {
      if (j == 0 || pbin[j] != pbin[j - 1]) {
        slot_bin[(size_t)c * max_slots + ns] = pbin[j];
        L[pbin[j]] = (int16_t)ns;
        cand_cnt[(size_t)c * max_slots + ns] = 0;
        ++ns;
      }
      bnd_slot[(size_t)c * kMaxBlocks + j] = ns - 1;
    }
    nslots[c] = ns;
  }
}

// 3) Collect the keys that fall in a boundary bin.
__global__ void k_collect_candidates(int64_t n, const uint32_t* __restrict__ seeds, uint32_t seed0,
                                     const int16_t* __restrict__ lut,
                                     uint32_t* __restrict__ cand_cnt,
                                     uint32_t* __restrict__ cand, int max_slots, int cap,
                                     int* __restrict__ err, const int* gate) {
  if (gated(gate)) return;
  __shared__ int16_t sl[kNumBins];
  const int c = blockIdx.y;
  const uint32_t seed = seed_of(seeds, seed0, c);
  for (int b = threadIdx.x; b < kNumBins; b += blockDim.x) sl[b] = lut[(size_t)c * kNumBins + b];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t key = pcg_key((uint32_t)i, seed);
    const int s = sl[key >> kBinShift];
    if (s >= 0) {
      uint32_t pos = atomicAdd(&cand_cnt[(size_t)c * max_slots + s], 1u);
      if (pos < (uint32_t)cap)
        cand[((size_t)c * max_slots + s) * cap + pos] = key;
      else
        atomicExch(err, 1);
    }
  }
}

// 4) Sort each slot's candidates (bitonic, in shared memory) and read off the
//    exact boundary keys.
__global__ void k_select_splitters(int nb, int cap_pow2, const int* __restrict__ nslots,
                                   const uint32_t* __restrict__ cand_cnt,
                                   const uint32_t* __restrict__ cand,
                                   const int* __restrict__ bnd_slot,
                                   const uint32_t* __restrict__ bnd_q,
                                   uint32_t* __restrict__ split, int max_slots, int cap, const int* gate) {
  if (gated(gate)) return;
  extern __shared__ uint32_t keys[];
  const int c = blockIdx.y, s = blockIdx.x;
  if (s >= nslots[c]) return;
  const uint32_t m = min(cand_cnt[(size_t)c * max_slots + s], (uint32_t)cap);
  const uint32_t* src = cand + ((size_t)c * max_slots + s) * cap;
  int P = 1;
  while (P < (int)m) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) keys[i] = (i < (int)m) ? src[i] : 0xffffffffu;
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          uint32_t a = keys[i], b = keys[ixj];
          bool up = ((i & k) == 0);
          if ((a > b) == up) { keys[i] = b; keys[ixj] = a; }
        }
      }
      __syncthreads();
    }
  }
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    if (bnd_slot[(size_t)c * kMaxBlocks + j] == s) {
      uint32_t q = bnd_q[(size_t)c * kMaxBlocks + j];
      split[(size_t)c * kMaxBlocks + j] = keys[min(q, (uint32_t)(P - 1))];
    }
  }
}

__device__ __forceinline__ int block_of(uint32_t key, const uint32_t* sp, int nb) {
  // number of boundary keys <= key  (sp ascending)
  int lo = 0, hi = nb;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (sp[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// 5) Per-tile bucket counts.  A bucket is (block, batch): within a block the
//    cells are ordered by batch code, then by cell index, so every tile of a
//    block holds long runs of one batch (used by the O accumulation).
__global__ void k_part_count(int64_t n, int nblk, int nsub, const int32_t* __restrict__ cats,
                             const uint32_t* __restrict__ seeds, uint32_t seed0,
                             const uint32_t* __restrict__ split, uint32_t* __restrict__ counts, int ntiles,
                             const int* gate) {
  if (gated(gate)) return;
  extern __shared__ uint32_t cnt[];   // [nblk * nsub]
  __shared__ uint32_t sp[kMaxBlocks];
  const int c = blockIdx.y, tile = blockIdx.x;
  const uint32_t seed = seed_of(seeds, seed0, c);
  const int nb = nblk - 1, nbk = nblk * nsub;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) sp[j] = split[(size_t)c * kMaxBlocks + j];
  for (int j = threadIdx.x; j < nbk; j += blockDim.x) cnt[j] = 0;
  __syncthreads();
  const int64_t base = (int64_t)tile * kPartTile;
  for (int q = threadIdx.x; q < kPartTile; q += blockDim.x) {
    int64_t i = base + q;
    if (i < n) {
      const int bucket = block_of(pcg_key((uint32_t)i, seed), sp, nb) * nsub + (nsub > 1 ? cats[i] : 0);
      atomicAdd(&cnt[bucket], 1u);
    }
  }
  __syncthreads();
  uint32_t* out = counts + ((size_t)c * ntiles + tile) * nbk;
  for (int j = threadIdx.x; j < nbk; j += blockDim.x) out[j] = cnt[j];
}

// 6) Column scan over tiles: offsets[tile][bucket] = sum_{t'<tile} counts[t'][bucket];
//    totals[bucket] = the column total.
__global__ void k_part_scan(int nbk, int ntiles, const uint32_t* __restrict__ counts,
                            uint32_t* __restrict__ offsets, uint32_t* __restrict__ totals, const int* gate) {
  if (gated(gate)) return;
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry_s;
  const int bk = blockIdx.x, c = blockIdx.y;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) carry_s = 0;
  __syncthreads();
  for (int t0 = 0; t0 < ntiles; t0 += blockDim.x) {
    const int tile = t0 + t;
    const size_t at = ((size_t)c * ntiles + tile) * nbk + bk;
    uint32_t v = (tile < ntiles) ? counts[at] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      const int nw = blockDim.x >> 5;
      uint32_t x = (lane < nw) ? wsum[lane] : 0u, xi = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
        if (lane >= o) xi += y;
      }
      if (lane < nw) wsum[lane] = xi - x;
    }
    __syncthreads();
    const uint32_t carry = carry_s;
    if (tile < ntiles) offsets[at] = carry + wsum[w] + incl - v;
    __syncthreads();
    if (t == blockDim.x - 1) carry_s = carry + wsum[w] + incl;
    __syncthreads();
  }
  if (t == 0) totals[(size_t)c * nbk + bk] = carry_s;
}

// 7) Stable scatter: cell i lands at base(bucket) + offsets[tile][bucket] + (rank
//    of i among the tile's cells of the same bucket, ascending), where base =
//    blk*bs + cells of lower batches in the same block.
__global__ void __launch_bounds__(256) k_part_scatter(int64_t n, int64_t bs, int nblk, int nsub,
                                                      const int32_t* __restrict__ cats,
                                                      const uint32_t* __restrict__ seeds, uint32_t seed0,
                                                      const uint32_t* __restrict__ split,
                                                      const uint32_t* __restrict__ offsets,
                                                      const uint32_t* __restrict__ totals,
                                                      int ntiles, int32_t* __restrict__ idx,
                                                      int32_t* __restrict__ lcat, int32_t* __restrict__ ckey,
                                                      int B, const int* gate) {
  if (gated(gate)) return;
  extern __shared__ uint32_t dyn[];
  const int nbk = nblk * nsub;
  uint32_t* base = dyn;               // [nbk]
  uint32_t* wc = dyn + nbk;           // [8][nbk]
  __shared__ uint32_t sp[kMaxBlocks];
  const int c = blockIdx.y, tile = blockIdx.x;
  const uint32_t seed = seed_of(seeds, seed0, c);
  const int nb = nblk - 1;
  const int t = threadIdx.x, w = t >> 5;
  for (int j = t; j < nb; j += 256) sp[j] = split[(size_t)c * kMaxBlocks + j];
  const uint32_t* off = offsets + ((size_t)c * ntiles + tile) * nbk;
  const uint32_t* tot = totals + (size_t)c * nbk;
  for (int blk = t; blk < nblk; blk += 256) {
    uint32_t run = (uint32_t)((int64_t)blk * bs);
    for (int q = 0; q < nsub; ++q) {
      const int bk = blk * nsub + q;
      base[bk] = run + off[bk];
      run += tot[bk];
    }
  }
  for (int j = t; j < 8 * nbk; j += 256) wc[j] = 0;
  __syncthreads();
  int32_t* out = idx + (size_t)c * n;
  const int64_t tbase = (int64_t)tile * kPartTile;
  for (int r = 0; r < kPartTile / 256; ++r) {
    const int64_t i = tbase + r * 256 + t;
    const bool valid = i < n;
    const int bk = valid ? block_of(pcg_key((uint32_t)i, seed), sp, nb) * nsub + (nsub > 1 ? cats[i] : 0)
                         : nbk;
    const unsigned peers = __match_any_sync(0xffffffffu, bk);
    const unsigned lrank = __popc(peers & lanemask_lt());
    if (valid && lrank == 0) wc[w * nbk + bk] = __popc(peers);
    __syncthreads();
    for (int j = t; j < nbk; j += 256) {
      uint32_t run = base[j];
#pragma unroll
      for (int q = 0; q < 8; ++q) { uint32_t x = wc[q * nbk + j]; wc[q * nbk + j] = run; run += x; }
      base[j] = run;
    }
    __syncthreads();
    if (valid) {
      const uint32_t at = wc[w * nbk + bk] + lrank;
      out[at] = (int32_t)i;
      const int cat = cats ? cats[i] : 0;
      if (lcat) lcat[(size_t)c * n + at] = cat;
      if (ckey) ckey[(size_t)c * n + i] = (int)((int64_t)at / bs) * (B + 1) + cat;
    }
    __syncthreads();
    for (int j = t; j < nbk; j += 256) {
#pragma unroll
      for (int q = 0; q < 8; ++q) wc[q * nbk + j] = 0;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------

MembershipLayout membership_layout(int64_t n, int64_t bs, int nsub) {
  MembershipLayout L{};
  L.n = n;
  L.bs = bs;
  L.nsub = nsub < 1 ? 1 : nsub;
  L.nblk = (int)((n + bs - 1) / bs);
  L.ntiles = div_up(n, kPartTile);
  const double mu = (double)n / kNumBins;
  int cap = (int)(mu + 8.0 * sqrt(mu) + 64.0);
  int p = 1;
  while (p < cap) p <<= 1;
  L.cap = p;
  L.max_slots = L.nblk > 1 ? L.nblk - 1 : 1;
  if ((int64_t)L.nblk * L.nsub > kMaxBuckets) L.nsub = 1;  // too many (block, batch) buckets
  return L;
}

void membership_carve(Carver& cv, const MembershipLayout& L, MembershipBufs& B) {
  const int C = kMaxIterChunk;
  B.seeds = cv.take<uint32_t>(C);
  B.hist = cv.take<uint32_t>((size_t)C * kNumBins);
  B.bnd_slot = cv.take<int>((size_t)C * kMaxBlocks);
  B.bnd_q = cv.take<uint32_t>((size_t)C * kMaxBlocks);
  B.slot_bin = cv.take<int>((size_t)C * L.max_slots);
  B.nslots = cv.take<int>(C);
  B.lut = cv.take<int16_t>((size_t)C * kNumBins);
  B.cand_cnt = cv.take<uint32_t>((size_t)C * L.max_slots);
  B.cand = cv.take<uint32_t>((size_t)C * L.max_slots * L.cap);
  B.split = cv.take<uint32_t>((size_t)C * kMaxBlocks);
  B.counts = cv.take<uint32_t>((size_t)C * L.ntiles * L.nblk * L.nsub);
  B.offsets = cv.take<uint32_t>((size_t)C * L.ntiles * L.nblk * L.nsub);
  B.totals = cv.take<uint32_t>((size_t)C * L.nblk * L.nsub);
  B.err = cv.take<int>(4);
}

// Writes, for each of `n_iters` (<= kMaxIterChunk) seeds, the cell list of every
// block: idx[c*n + j*bs + r] is the r-th cell (ascending) of block j.
int membership_build(const MembershipLayout& L, const MembershipBufs& B, const uint32_t* h_seeds,
                     int n_iters, const int32_t* cats, int32_t* idx, cudaStream_t st, int32_t* lcat,
                     int32_t* ckey, int n_batches) {
  if (n_iters < 1 || n_iters > kMaxIterChunk) {
    set_error("membership_build: n_iters out of range");
    return HB_ERR_INVALID;
  }
  HB_CUDA(cudaMemcpyAsync(B.seeds, h_seeds, sizeof(uint32_t) * n_iters, cudaMemcpyHostToDevice, st));
  return membership_build_dev(L, B, B.seeds, 0, n_iters, cats, idx, st, lcat, ckey, n_batches);
}

// Clears the candidate-overflow flag.  The build functions only ever set it, so a caller
// clears it once before its first chunk and reads it once after the last one.
int membership_clear_err(const MembershipBufs& B, cudaStream_t st) {
  HB_CUDA(cudaMemsetAsync(B.err, 0, sizeof(int), st));
  return HB_OK;
}

// Block lists for the consecutive seeds seed0 .. seed0+n_iters-1 (no host copy),
// or for the device list `seeds` when it is not null.  Sets B.err on a candidate
// overflow and never clears it (membership_clear_err).
int membership_build_dev(const MembershipLayout& L, const MembershipBufs& B, const uint32_t* seeds,
                         uint32_t seed0, int n_iters, const int32_t* cats, int32_t* idx,
                         cudaStream_t st, int32_t* lcat, int32_t* ckey, int n_batches, const int* gate) {
  const int nb = L.nblk - 1;
  const int sms = num_sms();
  const int nsub = cats ? L.nsub : 1;
  const int nbk = L.nblk * nsub;
  HB_CUDA(cudaMemsetAsync(B.hist, 0, sizeof(uint32_t) * (size_t)n_iters * kNumBins, st));
  int g = std::min(div_up(L.n, 256 * 8), 2 * sms);
  if (g < 1) g = 1;
  if (nb > 0) {
  k_key_hist<<<dim3(g, n_iters), 256, 0, st>>>(L.n, seeds, seed0, B.hist, gate);
  HB_LAUNCH_CHECK();
  k_boundary_bins<<<n_iters, 1024, 0, st>>>(L.bs, nb, B.hist, B.bnd_slot, B.bnd_q, B.slot_bin,
                                            B.nslots, B.lut, B.cand_cnt, L.max_slots, gate);
  HB_LAUNCH_CHECK();
  k_collect_candidates<<<dim3(g, n_iters), 256, 0, st>>>(L.n, seeds, seed0, B.lut, B.cand_cnt, B.cand,
                                                         L.max_slots, L.cap, B.err, gate);
  HB_LAUNCH_CHECK();
  const size_t smem = sizeof(uint32_t) * (size_t)L.cap;
  if (smem > 48 * 1024)
    HB_TRY(allow_max_dyn_smem((const void*)k_select_splitters));
  k_select_splitters<<<dim3(L.max_slots, n_iters), 512, smem, st>>>(
      nb, L.cap, B.nslots, B.cand_cnt, B.cand, B.bnd_slot, B.bnd_q, B.split, L.max_slots, L.cap, gate);
  HB_LAUNCH_CHECK();
  }
  if (sizeof(uint32_t) * nbk > 48 * 1024)
    HB_TRY(allow_max_dyn_smem((const void*)k_part_count));
  k_part_count<<<dim3(L.ntiles, n_iters), 256, sizeof(uint32_t) * nbk, st>>>(
      L.n, L.nblk, nsub, cats, seeds, seed0, B.split, B.counts, L.ntiles, gate);
  HB_LAUNCH_CHECK();
  k_part_scan<<<dim3(nbk, n_iters), 1024, 0, st>>>(nbk, L.ntiles, B.counts, B.offsets, B.totals, gate);
  HB_LAUNCH_CHECK();
  const size_t ssm = sizeof(uint32_t) * 9 * (size_t)nbk;
  if (ssm > 48 * 1024)
    HB_TRY(allow_max_dyn_smem((const void*)k_part_scatter));
  k_part_scatter<<<dim3(L.ntiles, n_iters), 256, ssm, st>>>(L.n, L.bs, L.nblk, nsub, cats, seeds, seed0,
                                                           B.split, B.offsets, B.totals, L.ntiles, idx, lcat, ckey,
                                                           n_batches, gate);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

}  // namespace hb
