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

// Cell ids and (block, batch) keys of one tile: one coalesced list read.
__device__ __forceinline__ void cen_load_ids(const CenArgs& a, int64_t pos, int nr, int* cid, int* key) {
  const int r = threadIdx.x;
  if (r < 128) {
    const int64_t cell = r < nr ? (int64_t)__ldg(a.idx + pos + r) : -1;
    cid[r] = (int)cell;
    key[r] = cell >= 0 ? (int)((pos + r) / a.bs) * (a.B + 1) + __ldg(a.cats + cell) : -1;
  }
}

// Copies of one tile from ids already in shared memory; consecutive lanes copy
// consecutive 16-byte chunks of the same rows.
template <typename H>
__device__ __forceinline__ void cen_copy(const CenArgs& a, const CenLayout& L, uint32_t sA, uint32_t sB,
                                         const int* cid) {
  const H* Zn = (const H*)a.Zn;
  const H* R = (const H*)a.R;
  const int zch = 16;             // 128 PCs (zero-padded) = 16 chunks, 2 blocks
  const int nch = zch + L.nbB * 8;
  for (int e = threadIdx.x; e < 128 * nch; e += blockDim.x) {
    const int r = e / nch, ch = e % nch;
    const int64_t cell = cid[r];
    if (ch < zch) {
      const bool ok = cell >= 0 && ch * 8 < a.ldz;
      tc::cp_async16(sA + mn_off(r, ch >> 3, ch & 7, 2),
                     ok ? (const void*)(Zn + cell * a.ldz + ch * 8) : (const void*)Zn, ok ? 16u : 0u);
    } else {
      const int c = ch - zch;
      const bool ok = cell >= 0 && c * 8 < a.ldr;
      tc::cp_async16(sB + mn_off(r, c >> 3, c & 7, L.nbB),
                     ok ? (const void*)(R + cell * a.ldr + c * 8) : (const void*)R, ok ? 16u : 0u);
    }
  }
}

template <typename H>
__global__ void __launch_bounds__(256, 1) k_tc_centroid(CenArgs a, CenLayout L) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int K = a.K;
  int* cid = (int*)(sm + L.offCid);
  int* ccat = (int*)(sm + L.offCat);
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  const uint32_t sA[3] = {tc::smem_u32(sm + L.offA[0]), tc::smem_u32(sm + L.offA[1]),
                          tc::smem_u32(sm + L.offA[2])};
  const uint32_t sB[3] = {tc::smem_u32(sm + L.offB[0]), tc::smem_u32(sm + L.offB[1]),
                          tc::smem_u32(sm + L.offB[2])};
  const int S = L.stages;
  const int64_t lo = a.n * blockIdx.x / gridDim.x, hi = a.n * (blockIdx.x + 1) / gridDim.x;
  const int ntiles = (int)((hi - lo + 127) / 128);

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  const int SI = S + 1;  // id ring slots
  auto tile_rows = [&](int t) { const int64_t p = lo + (int64_t)t * 128; return (int)(hi - p < 128 ? hi - p : 128); };
  // prologue: ids of the first S tiles, copies of the first S-1 (one cp.async group each)
  for (int t = 0; t < S; ++t)
    if (t < ntiles) cen_load_ids(a, lo + (int64_t)t * 128, tile_rows(t), cid + t * 128, ccat + t * 128);
  __syncthreads();
  for (int t = 0; t < S - 1; ++t) {
    if (t < ntiles) cen_copy<H>(a, L, sA[t], sB[t], cid + t * 128);
    tc::cp_async_commit();
  }
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, true, true);

  // O_minus column owners: (column k, row half h); K <= 128 uses both halves
  const int ncol = K > 128 ? 256 : 128;
  const int kcol = tid % ncol, rhalf = tid / ncol;
  const int nhalves = 256 / ncol;
  const bool owner = kcol < K;
  float om_acc = 0.f;   // current run, this 8-row group
  double om_tot = 0.0;  // current run, earlier groups (float64 keeps long runs exact enough)
  int om_key = -1;
  uint32_t phase = 0;

  for (int t = 0; t < ntiles; ++t) {
    const int buf = t % S;
    const int64_t pos = lo + (int64_t)t * 128;
    const int nr = (int)(hi - pos < 128 ? hi - pos : 128);
    if (S == 3) tc::cp_async_wait_group<1>(); else tc::cp_async_wait_group<0>();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      for (int s = 0; s < 8; ++s) {  // 8 steps of 16 cells
        const uint64_t ad = tc::sdesc_sw128(sA[buf] + (uint32_t)s * 2u * 2048u, 1024, 2048);
        const uint64_t bd = tc::sdesc_sw128(sB[buf] + (uint32_t)s * 2u * (uint32_t)L.nbB * 1024u, 1024,
                                            (uint32_t)L.nbB * 1024u);
        tc::mma_f16(tmem, ad, bd, idesc, (t > 0 || s > 0) ? 1u : 0u);
      }
      tc::mma_commit(mbar);
    }
    {
      const int tn = t + S - 1, bn = tn % S;  // refill the stage freed by tile t-1
      if (tn < ntiles) cen_copy<H>(a, L, sA[bn], sB[bn], cid + (tn % SI) * 128);
      tc::cp_async_commit();
      const int ti = t + S;  // ids two steps ahead, into the slot tile t-1 used
      if (ti < ntiles) cen_load_ids(a, lo + (int64_t)ti * 128, tile_rows(ti), cid + (ti % SI) * 128,
                                    ccat + (ti % SI) * 128);
    }
    // per-(block, batch) row sums of R from the staged tile; the row keys were
    // stored by the gather, swizzle offsets of the 8 rows of a group are fixed
    if (owner) {
      const int* keys = ccat + (t % SI) * 128;
      const unsigned char* tb = sm + L.offB[buf] + (kcol >> 6) * 1024 + (kcol & 7) * 2;
      const uint32_t gstride = (uint32_t)L.nbB * 1024u;
      const int c8 = (kcol & 63) >> 3;
      uint32_t tab[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) tab[i] = (uint32_t)i * 128u + ((uint32_t)(c8 ^ i) << 4);
      const int rows_per = 128 / nhalves;
      const int r0 = rhalf * rows_per, r1 = min(nr, r0 + rows_per);
      for (int g = r0; g < r1; g += 8) {
        const unsigned char* gb = tb + (uint32_t)(g >> 3) * gstride;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int r = g + i;
          if (r < r1) {
            const int key = keys[r];
            if (key != om_key) {
              if (om_key >= 0) {
                const double v = om_tot + (double)om_acc;
                atomicAdd(&a.Omin[(size_t)om_key * K + kcol], v);
                atomicAdd(&a.Omin[(size_t)(om_key - om_key % (a.B + 1) + a.B) * K + kcol], v);
              }
              om_key = key;
              om_acc = 0.f;
              om_tot = 0.0;
            }
            om_acc += h2f(*(const H*)(gb + tab[i]));
          }
        }
        om_tot += (double)om_acc;
        om_acc = 0.f;
      }
    }
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(a.err, 4);
    phase ^= 1u;
  }
  if (owner && om_key >= 0) {
    const double v = om_tot + (double)om_acc;
    atomicAdd(&a.Omin[(size_t)om_key * K + kcol], v);
    atomicAdd(&a.Omin[(size_t)(om_key - om_key % (a.B + 1) + a.B) * K + kcol], v);
  }
  tc::fence_after_sync();
  // partial D[pc][cluster] -> P[cta][cluster][pc]; lane = PC, warps 0-3 / 4-7 split the columns
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
  k_tc_centroid<H><<<grid, 256, smem, st>>>(a, L);
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
