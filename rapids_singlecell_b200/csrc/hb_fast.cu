// Tensor-core (tcgen05) kernels of the 16-bit Harmony path.
//
// k_tc_block_update is the fused soft-k-means block update: for a tile of 128
// cells of the current block it gathers their normalised embeddings (16-bit)
// into a 128-byte-swizzled shared-memory tile, multiplies by the resident
// normalised centroids on the tensor core (fp32 accumulator in TMEM), and in
// the epilogue applies exp(-2/sigma (1-s)), the diversity penalty, the row
// L1 normalisation, writes the new 16-bit assignment row, and accumulates the
// observed-count delta and the objective terms.  The similarity matrix never
// leaves the SM (the reference materialises it in HBM, clustering.cu:284-289,
// and runs ~12 kernels per block, clustering.cu:308-372).
#include "hb_tc_tile.cuh"

namespace hb {

template <typename H>
__global__ void __launch_bounds__(256, 1) k_tc_block_update(TcArgs p, TcLayout L) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const BlockArgs& a = p.a;
  const int K = a.K, B = a.B;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* pen = (float*)(sm + L.offPen);
  float* osm = (float*)(sm + L.offOsm);
  H* Rst = (H*)(sm + L.offRst);
  int* cid = (int*)(sm + L.offCid);
  int* ccat = (int*)(sm + L.offCat);
  float* rsp = (float*)(sm + L.offRs);
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  double* red = (double*)(sm + L.offMisc + 16);
  const H* Zn = (const H*)a.Zn;
  const H* Yn = (const H*)a.Yn;
  H* R = (H*)a.R;
  const uint32_t sA[2] = {tc::smem_u32(sm + L.offA0), tc::smem_u32(sm + L.offA1)};
  const uint32_t sB = tc::smem_u32(sm + L.offB);
  const int64_t ntiles = (a.n_new + 127) / 128;

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  if (p.O_zero)
    for (int e = blockIdx.x * 256 + tid; e < B * K; e += gridDim.x * 256) p.O_zero[e] = 0.0;

  // operands of the first tile and the resident centroids (async) ...
  if (ntiles > 0) {
    load_centroids_swizzled(Yn, a.ldy, K, sB, L);
    if (blockIdx.x < ntiles)
      gather_rows_swizzled(Zn, a.ldz, a.idx_new, a.new_start, a.n_new, blockIdx.x, sA[0], L, cid, ccat,
                           a.cats);
  }
  // ... while the penalty table is computed from the current O (kernels_pen.cuh:8-21)
  if (a.n_new > 0 && !a.init_mode) {
    for (int k = tid; k < K; k += 256) {
      double col = 0;
      for (int b = 0; b < B; ++b) {
        const size_t e = (size_t)b * K + k;
        col += p.O_in[e] - (a.Om_cur ? a.Om_cur[e] : 0.0);
      }
      for (int b = 0; b < B; ++b) {
        const size_t e = (size_t)b * K + k;
        const float o = (float)(p.O_in[e] - (a.Om_cur ? a.Om_cur[e] : 0.0));
        const float E = (float)(a.Pr[b] * col);
        const float denom = a.stabilized ? (o + E + 1.f) : (o + 1.f);
        pen[b * K + k] = powf((E + 1.f) / denom, (float)a.theta[b]);
      }
    }
  }
  for (int e = tid; e < B * K; e += 256) osm[e] = 0.f;
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, false, false);
  const float c2 = (float)(-2.0 / a.sigma * 1.4426950408889634);  // exp(x) = exp2(x log2 e)
  const float sig = (float)a.sigma;
  const int half = warp >> 2;
  const int row = (warp & 3) * 32 + lane;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const int nh = (L.npad / 2 + 7) / 8 * 8;
  const int c_lo = half * nh, c_hi = min(L.npad, c_lo + nh);
  double obj_local = 0.0;
  uint32_t phase = 0;
  int it = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int buf = (L.nbufA == 2) ? (it & 1) : 0;
    if (L.nbufA == 1 && it > 0) {
      __syncthreads();
      gather_rows_swizzled(Zn, a.ldz, a.idx_new, a.new_start, a.n_new, tile, sA[0], L, cid, ccat, a.cats);
    }
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) issue_similarity_mma(tmem, sA[buf], sB, L, idesc, mbar);
    const int64_t nxt = tile + gridDim.x;
    if (L.nbufA == 2 && nxt < ntiles)
      gather_rows_swizzled(Zn, a.ldz, a.idx_new, a.new_start, a.n_new, nxt, sA[buf ^ 1], L,
                           cid + (buf ^ 1) * 128, ccat + (buf ^ 1) * 128, a.cats);
    if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(p.err, 2);
    phase ^= 1u;
    tc::fence_after_sync();

    const int cell = cid[buf * 128 + row];
    const int cat = ccat[buf * 128 + row];
    const float* prow = pen + cat * K;
    // pass 1: v = exp(-2/sigma (1-s)) * pen, row partial sums; v overwrites s in TMEM
    float rs = 0.f, km = 0.f;
    for (int c = c_lo; c < c_hi; c += 8) {
      float v[8];
      tc::tmem_ld8(tl + (uint32_t)c, v);
      tc::tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = c + i;
        float val = 0.f;
        if (k < K) {
          val = exp2f(c2 * (1.f - v[i]));
          if (!a.init_mode) val *= prow[k];
          km += val * 2.f * (1.f - v[i]);
        }
        rs += val;
        v[i] = val;
      }
      tc::tmem_st8(tl + (uint32_t)c, v);
    }
    tc::tmem_st_wait();
    rsp[half * 128 + row] = rs;
    __syncthreads();
    const float rsum = rsp[row] + rsp[128 + row];
    const float inv = a.init_mode ? 1.f / fmaxf(rsum, 1e-12f) : 1.f / rsum;
    // pass 2: normalise, round to 16 bits, stage the row, entropy term
    float ent = 0.f;
    for (int c = c_lo; c < c_hi; c += 8) {
      float v[8];
      tc::tmem_ld8(tl + (uint32_t)c, v);
      tc::tmem_ld_wait();
      __align__(16) H hv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float r = v[i] * inv;
        hv[i] = from_f<H>(r);
        if (c + i < K) ent += r * logf(r + 1e-12f);
      }
      *(uint4*)(Rst + row * L.ldst + c) = *(const uint4*)hv;
    }
    tc::fence_before_sync();
    if (cell >= 0) obj_local += (double)(inv * km) + (double)(sig * ent);
    __syncthreads();
    const int nvalid = (int)(a.n_new - tile * 128 < 128 ? a.n_new - tile * 128 : 128);
    // observed-count delta: one thread per cluster column, runs of equal batch
    if (tid < K) {
      const int* cc = ccat + buf * 128;
      float acc = 0.f;
      int cur = cc[0];
      for (int r = 0; r < nvalid; ++r) {
        const int c = cc[r];
        if (c != cur) {
          osm[cur * K + tid] += acc;
          acc = 0.f;
          cur = c;
        }
        acc += h2f(Rst[r * L.ldst + tid]);
      }
      osm[cur * K + tid] += acc;
    }
    // write the new assignment rows
    for (int e = tid; e < nvalid * L.ldr_chunks; e += 256) {
      const int r = e / L.ldr_chunks, ch = e % L.ldr_chunks;
      const int64_t cl = cid[buf * 128 + r];
      *(uint4*)(R + cl * a.ldr + ch * 8) = *(const uint4*)(Rst + r * L.ldst + ch * 8);
    }
  }

  __syncthreads();
  for (int e = tid; e < B * K; e += 256) {
    double v = (double)osm[e];
    if (blockIdx.x == 0) {
      if (p.O_in) v += p.O_in[e];
      if (a.Om_cur) v -= a.Om_cur[e];
      if (a.Om_next) v -= a.Om_next[e];
    }
    if (v != 0.0) atomicAdd(&p.O_out[e], v);
  }
  const double tot = block_sum(obj_local, red);
  if (tid == 0 && tot != 0.0) atomicAdd(a.obj_acc, tot);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)L.tcols);
  }
}

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
    set_error("tensor-core block update: shared-memory tables too large");
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
int launch_tc_block_update(const BlockArgs& a, const double* O_in, double* O_out, double* O_zero,
                           int* err, cudaStream_t st) {
  const TcLayout L = tc_layout(a.d, a.K, a.B, a.ldr, 4);
  int occ = 1;
  HB_TRY(prepare<H>((const void*)k_tc_block_update<H>, L, &occ));
  const int64_t tiles = (a.n_new + 127) / 128;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)num_sms() * occ));
  // keep residency at `occ` CTAs per SM (TMEM budget) by padding the shared-memory request
  size_t smem = L.bytes;
  const size_t per_sm = 228u * 1024u;
  if (per_sm / (smem + 1024) > (size_t)occ) smem = std::min<size_t>(227u * 1024u, per_sm / occ - 2048);
  if (smem != L.bytes)
    HB_TRY(allow_max_dyn_smem((const void*)k_tc_block_update<H>));
  k_tc_block_update<H><<<grid, 256, smem, st>>>(TcArgs{a, O_in, O_out, O_zero, err}, L);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_tc_block_update<__half>(const BlockArgs&, const double*, double*, double*, int*, cudaStream_t);
template int launch_tc_block_update<__nv_bfloat16>(const BlockArgs&, const double*, double*, double*, int*,
                                                   cudaStream_t);

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
