// Similarity rows on the tensor core (tcgen05), the kernel-level entry point
// hb_similarity.  It uses the sweep's own pieces (hb_tc_tile.cuh): the centroid
// tile staged by load_centroids_swizzled, the 128-byte-swizzled K-major A tile
// and issue_similarity_mma, so a test of it checks the sweep's MMA operand
// layout and descriptors against a plain fp32 product.
#include "hb_tc_tile.cuh"

namespace hb {

// Similarity rows S[q][k] = Z_norm[idx[q]] . Y_norm[k] on the tensor core (the
// reference materialises the same matrix with a cuBLAS GEMM, clustering.cu:284-289).
template <typename H>
__global__ void __launch_bounds__(256, 1) k_tc_similarity(const H* __restrict__ Zn, int ldz,
                                                          const H* __restrict__ Yn, int ldy,
                                                          const int32_t* __restrict__ idx,
                                                          const int32_t* __restrict__ cats, int64_t n,
                                                          int K, float* __restrict__ S, TcLayout L,
                                                          int* err) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int* cid = (int*)(sm + L.offCid);
  int* ccat = (int*)(sm + L.offCat);
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  const uint32_t sA = tc::smem_u32(sm + L.offA0), sB = tc::smem_u32(sm + L.offB);
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  load_centroids_swizzled(Yn, ldy, K, sB, L);
  const int64_t ntiles = (n + 127) / 128;
  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, false, false);
  const int half = warp >> 2, row = (warp & 3) * 32 + lane;
  const int nh = (L.npad / 2 + 7) / 8 * 8;
  const int c_lo = half * nh, c_hi = min(L.npad, c_lo + nh);
  uint32_t phase = 0;
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    __syncthreads();
    gather_rows_swizzled(Zn, ldz, idx, 0, n, tile, sA, L, cid, ccat, cats);
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) issue_similarity_mma(tmem, sA, sB, L, idesc, mbar);
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(err, 2);
    phase ^= 1u;
    tc::fence_after_sync();
    const int64_t q = tile * 128 + row;
    for (int c = c_lo; c < c_hi; c += 8) {
      float v[8];
      tc::tmem_ld8(tl + (uint32_t)c, v);
      tc::tmem_ld_wait();
      if (q < n)
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (c + i < K) S[q * K + c + i] = v[i];
    }
    tc::fence_before_sync();
  }
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)L.tcols);
  }
}

template <typename H>
static int prepare(const void* fn, const TcLayout& L, int* occ_out) {
  if (L.bytes > 227u * 1024u) {
    set_error("tensor-core similarity: shared-memory tables too large");
    return HB_ERR_UNSUPPORTED;
  }
  HB_TRY(allow_max_dyn_smem(fn));
  int occ = 1;
  HB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, L.bytes));
  // at most 512 TMEM columns per SM are shared by the resident CTAs
  occ = std::max(1, std::min(occ, 512 / L.tcols));
  *occ_out = occ;
  return HB_OK;
}

template <typename H>
int launch_tc_similarity(const H* Zn, int ldz, const H* Yn, int ldy, const int32_t* idx,
                         const int32_t* cats, int64_t n, int d, int K, float* S, int* err,
                         cudaStream_t st) {
  const TcLayout L = tc_layout(d, K, 1, (K + 7) / 8 * 8, 4);
  int occ = 1;
  HB_TRY(prepare<H>((const void*)k_tc_similarity<H>, L, &occ));
  const int64_t tiles = (n + 127) / 128;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)num_sms() * occ));
  size_t smem = L.bytes;
  const size_t per_sm = 228u * 1024u;
  if (per_sm / (smem + 1024) > (size_t)occ) smem = std::min<size_t>(227u * 1024u, per_sm / occ - 2048);
  if (smem != L.bytes)
    HB_TRY(allow_max_dyn_smem((const void*)k_tc_similarity<H>));
  k_tc_similarity<H><<<grid, 256, smem, st>>>(Zn, ldz, Yn, ldy, idx, cats, n, K, S, L, err);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_similarity<__half>(const __half*, int, const __half*, int, const int32_t*,
                                          const int32_t*, int64_t, int, int, float*, int*, cudaStream_t);
template int launch_tc_similarity<__nv_bfloat16>(const __nv_bfloat16*, int, const __nv_bfloat16*, int,
                                                 const int32_t*, const int32_t*, int64_t, int, int, float*,
                                                 int*, cudaStream_t);

}  // namespace hb
