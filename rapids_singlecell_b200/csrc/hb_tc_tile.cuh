// Shared pieces of the tensor-core tile kernels: shared-memory layout, operand
// staging into 128-byte-swizzled tiles, and the similarity MMA issue.
#pragma once
#include "hb_internal.h"
#include "hb_tc.cuh"

namespace hb {

constexpr uint32_t kMaxPolls = 1u << 24;  // bounded mbarrier wait (seconds), then error flag

struct TcLayout {
  int dpad;     // MMA K extent: 64 or 128 (zero-padded PCs)
  int kblk;     // dpad / 64 swizzle atoms along K
  int npad;     // MMA N: clusters rounded up to 16
  int tcols;    // TMEM columns allocated (power of two >= npad)
  int ldst;     // staging row stride (elements)
  int nbufA;    // A tiles (2 = gather of tile i+1 overlaps tile i)
  int ldr_chunks;
  uint32_t offA0, offA1, offB, offRst, offPen, offOsm, offCid, offCat, offRs, offMisc, bytes;
};

inline TcLayout tc_layout(int d, int K, int B, int ldr, int elem_bytes_pen) {
  TcLayout L{};
  L.dpad = d <= 64 ? 64 : 128;
  L.kblk = L.dpad / 64;
  L.npad = (K + 15) / 16 * 16;
  L.tcols = L.npad <= 128 ? 128 : 256;
  L.ldst = (K + 7) / 8 * 8 + 8;
  if (L.ldst < L.npad) L.ldst = L.npad;
  L.ldr_chunks = ldr / 8;
  const uint32_t atile = (uint32_t)L.kblk * 16384u;
  auto al = [](uint32_t x, uint32_t a) { return (x + a - 1) / a * a; };
  for (int nb = 2; nb >= 1; --nb) {
    uint32_t o = 0;
    L.offA0 = o; o += atile;
    L.offA1 = nb == 2 ? o : L.offA0; if (nb == 2) o += atile;
    L.offB = o; o += (uint32_t)L.kblk * L.npad * 128u;
    L.offRst = al(o, 16); o = L.offRst + 128u * L.ldst * 2u;
    L.offPen = al(o, 16); o = L.offPen + (uint32_t)B * K * elem_bytes_pen;
    L.offOsm = al(o, 16); o = L.offOsm + (uint32_t)B * K * 4u;
    L.offCid = al(o, 16); o = L.offCid + 2u * 128u * 4u;
    L.offCat = o; o += 2u * 128u * 4u;
    L.offRs = o; o += 2u * 128u * 4u;
    L.offMisc = al(o, 16); o = L.offMisc + 16u + 32u * 8u;
    L.bytes = o + 1024u;  // slack for 1024-byte alignment of the base
    L.nbufA = nb;
    if (L.bytes <= 227u * 1024u) break;
  }
  return L;
}

template <typename H> struct is_bf16 { static constexpr bool value = false; };
template <> struct is_bf16<__nv_bfloat16> { static constexpr bool value = true; };

__device__ __forceinline__ float h2f(__half x) { return __half2float(x); }
__device__ __forceinline__ float h2f(__nv_bfloat16 x) { return __bfloat162float(x); }

template <typename H>
__device__ __forceinline__ void load_centroids_swizzled(const H* __restrict__ Yn, int ldy, int K,
                                                        uint32_t sB, const TcLayout& L) {
  const int nch = L.dpad / 8;
  for (int e = threadIdx.x; e < L.npad * nch; e += blockDim.x) {
    const int k = e / nch, ch = e % nch;
    const bool ok = k < K && ch * 8 < ldy;
    const uint32_t dst = sB + (uint32_t)(ch >> 3) * (uint32_t)(L.npad * 128) + tc::sw128_off(k, ch & 7);
    tc::cp_async16(dst, ok ? (const void*)(Yn + (size_t)k * ldy + ch * 8) : (const void*)Yn, ok ? 16u : 0u);
  }
}

// Gather the embedding rows of one 128-cell tile into a swizzled K-major A tile.
// Thread t owns row t % 128 and every (blockDim/128)-th chunk of it: one cell-id
// load per thread, then its copies are issued back to back.
template <typename H>
__device__ __forceinline__ void gather_rows_swizzled(const H* __restrict__ Zn, int ldz,
                                                     const int32_t* __restrict__ idx, int64_t start,
                                                     int64_t n, int64_t tile, uint32_t sA,
                                                     const TcLayout& L, int* cid, int* ccat,
                                                     const int32_t* __restrict__ cats) {
  const int nch = L.dpad / 8;
  const int r = threadIdx.x & 127, part = threadIdx.x >> 7, nparts = blockDim.x >> 7;
  const int64_t q = tile * 128 + r;
  const int64_t cell = q < n ? (idx ? (int64_t)__ldg(idx + q) : start + q) : -1;
  if (part == 0) {
    cid[r] = (int)cell;
    ccat[r] = (cell >= 0 && cats) ? __ldg(cats + cell) : 0;
  }
  const H* src = cell >= 0 ? Zn + cell * ldz : Zn;
  for (int ch = part; ch < nch; ch += nparts) {
    const bool ok = cell >= 0 && ch * 8 < ldz;
    const uint32_t dst = sA + (uint32_t)(ch >> 3) * 16384u + tc::sw128_off(r, ch & 7);
    tc::cp_async16(dst, ok ? (const void*)(src + ch * 8) : (const void*)Zn, ok ? 16u : 0u);
  }
}

// S = A_tile . B^T on the tensor core; one thread issues, commit arrives on mbar.
__device__ __forceinline__ void issue_similarity_mma(uint32_t tmem, uint32_t sA, uint32_t sB,
                                                     const TcLayout& L, uint32_t idesc, uint64_t* mbar) {
  tc::fence_after_sync();
  const int nks = L.dpad / 16;
  for (int s = 0; s < nks; ++s) {
    const uint64_t ad = tc::sdesc_sw128(sA + (uint32_t)(s >> 2) * 16384u + (uint32_t)(s & 3) * 32u, 16, 1024);
    const uint64_t bd = tc::sdesc_sw128(sB + (uint32_t)(s >> 2) * (uint32_t)(L.npad * 128) + (uint32_t)(s & 3) * 32u,
                                        16, 1024);
    tc::mma_f16(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
  }
  tc::mma_commit(mbar);
}

}  // namespace hb
