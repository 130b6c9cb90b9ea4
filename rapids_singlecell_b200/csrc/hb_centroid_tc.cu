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
  int npad, nbB, tcols;
  uint32_t offA[2], offB[2], offCid, offCat, offMisc, bytes;
};

inline CenLayout cen_layout(int K) {
  CenLayout L{};
  L.npad = (K + 15) / 16 * 16;
  L.nbB = (L.npad + 63) / 64;
  L.tcols = L.npad <= 128 ? 128 : 256;
  uint32_t o = 0;
  for (int s = 0; s < 2; ++s) { L.offA[s] = o; o += 2u * 16384u; }
  for (int s = 0; s < 2; ++s) { L.offB[s] = o; o += (uint32_t)L.nbB * 16384u; }
  L.offCid = o; o += 2u * 128u * 4u;
  L.offCat = o; o += 2u * 128u * 4u;
  L.offMisc = o; o += 16u;
  // 8 KB of slack: reads stay inside the allocation under either reading of the
  // descriptor's leading / stride offsets (see the layout note above)
  L.bytes = o + 8192u + 1024u;
  return L;
}

// byte offset of chunk (block nb, 16B chunk c8) of cell r in a tile with `nblocks` blocks per group
__device__ __forceinline__ uint32_t mn_off(uint32_t r, uint32_t nb, uint32_t c8, uint32_t nblocks) {
  return (r >> 3) * (nblocks * 1024u) + nb * 1024u + (r & 7u) * 128u + ((c8 ^ (r & 7u)) << 4);
}

template <typename H>
__device__ __forceinline__ void cen_gather(const CenArgs& a, const CenLayout& L, int64_t pos, int nr,
                                           uint32_t sA, uint32_t sB, int* cid, int* ccat) {
  // thread t owns row t % 128 and every other chunk of it (one cell-id load per thread)
  const H* Zn = (const H*)a.Zn;
  const H* R = (const H*)a.R;
  const int zch = 16;             // 128 PCs (zero-padded) = 16 chunks, 2 blocks
  const int rch = L.nbB * 8;      // cluster chunks
  const int r = threadIdx.x & 127, part = threadIdx.x >> 7, nparts = blockDim.x >> 7;
  const int64_t cell = r < nr ? (int64_t)__ldg(a.idx + pos + r) : -1;
  if (part == 0) {
    cid[r] = (int)cell;
    ccat[r] = cell >= 0 ? __ldg(a.cats + cell) : 0;
  }
  const H* zs = cell >= 0 ? Zn + cell * a.ldz : Zn;
  const H* rs = cell >= 0 ? R + cell * a.ldr : R;
  for (int ch = part; ch < zch + rch; ch += nparts) {
    if (ch < zch) {
      const bool ok = cell >= 0 && ch * 8 < a.ldz;
      tc::cp_async16(sA + mn_off(r, ch >> 3, ch & 7, 2), ok ? (const void*)(zs + ch * 8) : (const void*)Zn,
                     ok ? 16u : 0u);
    } else {
      const int c = ch - zch;
      const bool ok = cell >= 0 && c * 8 < a.ldr;
      tc::cp_async16(sB + mn_off(r, c >> 3, c & 7, L.nbB), ok ? (const void*)(rs + c * 8) : (const void*)R,
                     ok ? 16u : 0u);
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
  const uint32_t sA[2] = {tc::smem_u32(sm + L.offA[0]), tc::smem_u32(sm + L.offA[1])};
  const uint32_t sB[2] = {tc::smem_u32(sm + L.offB[0]), tc::smem_u32(sm + L.offB[1])};
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
  if (ntiles > 0) cen_gather<H>(a, L, lo, (int)(hi - lo < 128 ? hi - lo : 128), sA[0], sB[0], cid, ccat);
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, true, true);

  // O_minus column owners: (column k, row half h); K <= 128 uses both halves
  const int ncol = K > 128 ? 256 : 128;
  const int kcol = tid % ncol, rhalf = tid / ncol;
  const int nhalves = 256 / ncol;
  const bool owner = kcol < K;
  double om_acc = 0.0;
  int om_key = -1;
  uint32_t phase = 0;

  for (int t = 0; t < ntiles; ++t) {
    const int buf = t & 1;
    const int64_t pos = lo + (int64_t)t * 128;
    const int nr = (int)(hi - pos < 128 ? hi - pos : 128);
    tc::cp_async_wait_all();
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
    if (t + 1 < ntiles)
      cen_gather<H>(a, L, pos + 128, (int)(hi - pos - 128 < 128 ? hi - pos - 128 : 128), sA[buf ^ 1], sB[buf ^ 1],
                    cid + (buf ^ 1) * 128, ccat + (buf ^ 1) * 128);
    // per-(block, batch) row sums of R from the staged tile (the block changes at
    // most where the list position crosses a multiple of bs)
    if (owner) {
      const unsigned char* tb = sm + L.offB[buf];
      const int nb = kcol >> 6, c8 = (kcol & 63) >> 3, w8 = kcol & 7;
      const int r0 = rhalf * (128 / nhalves), r1 = min(nr, r0 + 128 / nhalves);
      if (r0 < r1) {
        int blk = (int)((pos + r0) / a.bs);
        int64_t next_edge = (int64_t)(blk + 1) * a.bs;
        for (int r = r0; r < r1; ++r) {
          if (pos + r >= next_edge) {
            ++blk;
            next_edge += a.bs;
          }
          const int key = blk * (a.B + 1) + ccat[buf * 128 + r];
          if (key != om_key) {
            if (om_key >= 0) {
              atomicAdd(&a.Omin[(size_t)om_key * K + kcol], om_acc);
              atomicAdd(&a.Omin[(size_t)(om_key - om_key % (a.B + 1) + a.B) * K + kcol], om_acc);
            }
            om_key = key;
            om_acc = 0.0;
          }
          const H* p = (const H*)(tb + mn_off(r, nb, c8, L.nbB)) + w8;
          om_acc += (double)h2f(*p);
        }
      }
    }
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(a.err, 4);
    phase ^= 1u;
  }
  if (owner && om_key >= 0) {
    atomicAdd(&a.Omin[(size_t)om_key * K + kcol], om_acc);
    atomicAdd(&a.Omin[(size_t)(om_key - om_key % (a.B + 1) + a.B) * K + kcol], om_acc);
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
