// Persistent soft-k-means sweep of the 16-bit path (one launch per k-means
// iteration).
//
// The reference updates R block by block with ~12 launches per block, the
// similarity matrix round-tripping through HBM (_cuda/harmony/clustering/
// clustering.cu:308-372).  Here one cooperative launch walks all blocks of an
// iteration.  For block j every CTA takes an even, contiguous slice of the
// block's cell list (ordered by batch, then cell), and for each tile of <= 128
// cells: gathers the 16-bit normalised embeddings into a swizzled shared tile,
// runs S = Z_tile . Y_norm^T on the tensor core (fp32 in TMEM), and in the
// epilogue forms R = normalise_L1(exp(-2/sigma (1-s)) * pen[batch]), writes it,
// and adds it to a per-CTA observed-count delta.  The deltas are flushed with
// float64 atomics and a bounded grid barrier separates the blocks, because the
// penalty of block j+1 depends on the counts after block j.  The "remove old
// contribution" step of every block comes precomputed from the centroid pass
// (Omin), so no R row is read in the sweep.
//
// O state: three rotating buffers of (B+1) x K float64 (row B holds the column
// sums, i.e. E / Pr_b).  Block j reads buffer (b0+j)%3, accumulates into
// (b0+j+1)%3 (already zero) and zeroes (b0+j+2)%3 for block j+1.
#include "hb_tc_tile.cuh"

namespace hb {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for a cooperative launch.  Every wait is bounded: after
// ~2^26 polls the CTA records error 3 and proceeds (the host reports a timeout).
__device__ __forceinline__ void grid_barrier(unsigned* ctr, unsigned target, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    unsigned spins = 0;
    while (ld_acquire_u32(ctr) < target) {
      if (++spins > (1u << 26)) {
        atomicExch(err, 3);
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
}

// The slice of block j processed by CTA c of G: list positions [lo, hi).
__device__ __forceinline__ void slice_of(const SweepArgs& a, int j, int c, int G, int64_t& lo, int64_t& hi) {
  const int64_t s = (int64_t)j * a.bs;
  const int64_t nj = min(a.bs, a.n - s);
  lo = s + nj * c / G;
  hi = s + nj * (c + 1) / G;
}

// Work cursor over (block, tile start) for this CTA; tile = up to 128 positions.
struct Cursor {
  int j;
  int64_t pos, hi;
};

__device__ __forceinline__ bool cursor_first(const SweepArgs& a, int j, Cursor& cu) {
  for (; j < a.nblk; ++j) {
    int64_t lo, hi;
    slice_of(a, j, blockIdx.x, gridDim.x, lo, hi);
    if (lo < hi) {
      cu.j = j;
      cu.pos = lo;
      cu.hi = hi;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ bool cursor_next(const SweepArgs& a, const Cursor& cu, Cursor& nx) {
  if (cu.pos + 128 < cu.hi) {
    nx = cu;
    nx.pos = cu.pos + 128;
    return true;
  }
  return cursor_first(a, cu.j + 1, nx);
}

template <typename H>
__device__ __forceinline__ void gather_item(const SweepArgs& a, const Cursor& cu, uint32_t sA,
                                            const TcLayout& L, int* cid, int* ccat) {
  const int64_t nr = cu.hi - cu.pos < 128 ? cu.hi - cu.pos : 128;
  gather_rows_swizzled((const H*)a.Zn, a.ldz, a.idx ? a.idx + cu.pos : nullptr, cu.pos, nr, 0, sA, L,
                       cid, ccat, a.cats);
}

// NT = 256: warps 0-3 and 4-7 take the two column halves of the same 128 rows
// (one CTA per SM).  NT = 128: each thread owns a full row; used when two CTAs
// fit on an SM so that one CTA's latency chain overlaps the other's.
template <typename H, int NT>
__global__ void __launch_bounds__(NT, 1) k_tc_sweep(SweepArgs a, TcLayout L) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const int K = a.K, B = a.B;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* pen = (float*)(sm + L.offPen);   // [B][K]
  float* osm = (float*)(sm + L.offOsm);   // [B][K] observed-count delta of this CTA
  H* Rst = (H*)(sm + L.offRst);
  int* cid = (int*)(sm + L.offCid);       // [2][128]
  int* ccat = (int*)(sm + L.offCat);      // [2][128]
  float* rsp = (float*)(sm + L.offRs);    // [2][128]
  uint64_t* mbar = (uint64_t*)(sm + L.offMisc);
  uint32_t* tmem_slot = (uint32_t*)(sm + L.offMisc + 8);
  double* red = (double*)(sm + L.offMisc + 16);
  __shared__ float dsum[256];             // column sums of the delta (row B)
  __shared__ double ocol[256];            // column sums of the state
  __shared__ int2 crange[kMaxBlocks];    // batch range of this CTA's slice, per block
  __shared__ int runs[130];               // tile run starts (batch changes), terminated by nrows
  __shared__ int nruns;
  H* R = (H*)a.R;
  const uint32_t sA[2] = {tc::smem_u32(sm + L.offA0), tc::smem_u32(sm + L.offA1)};
  const uint32_t sB = tc::smem_u32(sm + L.offB);
  const size_t ldo = (size_t)(B + 1) * K;

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)L.tcols);
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  load_centroids_swizzled((const H*)a.Yn, a.ldy, K, sB, L);
  Cursor cu;
  bool have = cursor_first(a, 0, cu);
  if (have) gather_item<H>(a, cu, sA[0], L, cid, ccat);
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, false, false);
  const float c2 = (float)(-2.0 / a.sigma * 1.4426950408889634);  // exp(x) = exp2(x log2 e)
  const float sig = (float)a.sigma;
  const int half = NT == 256 ? warp >> 2 : 0;
  const int row = (warp & 3) * 32 + lane;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const int nh = NT == 256 ? (L.npad / 2 + 7) / 8 * 8 : L.npad;
  const int c_lo = half * nh, c_hi = min(L.npad, c_lo + nh);
  double obj_local = 0.0;
  uint32_t phase = 0;
  int buf = 0;
  bool pre_issued = false;  // the MMA of the current tile was issued before the last barrier
  // batch range of every block's slice (the list is ordered by batch within a block)
  for (int j = tid; j < a.nblk; j += NT) {
    int64_t lo, hi;
    slice_of(a, j, blockIdx.x, gridDim.x, lo, hi);
    int cmin = 0, cmax = B - 1;
    if (a.idx && a.batch_sorted && lo < hi) {
      cmin = __ldg(a.lcat + lo);
      cmax = __ldg(a.lcat + hi - 1);
    }
    crange[j] = make_int2(cmin, lo < hi ? cmax : cmin - 1);
  }

  for (int j = 0; j < a.nblk; ++j) {
    const double* Oin = a.Obuf[(a.b0 + j) % 3];
    double* Oout = a.Obuf[(a.b0 + j + 1) % 3];
    double* Ozero = a.Obuf[(a.b0 + j + 2) % 3];
    const double* Omc = (a.Omin && j == 0) ? a.Omin : nullptr;                       // this block
    const double* Omn = (a.Omin && j + 1 < a.nblk) ? a.Omin + (size_t)(j + 1) * ldo : nullptr;  // next
    int64_t lo, hi;
    slice_of(a, j, blockIdx.x, gridDim.x, lo, hi);
    for (size_t e = (size_t)blockIdx.x * NT + tid; e < ldo; e += (size_t)gridDim.x * NT) Ozero[e] = 0.0;
    for (int k = tid; k < K; k += NT) {
      double s = Oin[(size_t)B * K + k];
      if (Omc) s -= Omc[(size_t)B * K + k];
      ocol[k] = s;
      dsum[k] = 0.f;
    }
    __syncthreads();
    const int cmin = crange[j].x, cmax = crange[j].y;
    // log2 of the penalty rows of the batches present (kernels_pen.cuh:8-21):
    // log2 pen = theta_b * log2((E+1)/(O[+E]+1)); zero the delta rows
    for (int e = tid; e < (cmax - cmin + 1) * K; e += NT) {
      const int b = cmin + e / K, k = e % K;
      const size_t o_at = (size_t)b * K + k;
      osm[o_at] = 0.f;
      float lp = 0.f;
      if (!a.init_mode) {
        const float o = (float)(Oin[o_at] - (Omc ? Omc[o_at] : 0.0));
        const float E = (float)(a.Pr[b] * ocol[k]);
        const float denom = a.stabilized ? (o + E + 1.f) : (o + 1.f);
        lp = (float)a.theta[b] * log2f((E + 1.f) / denom);
      }
      pen[o_at] = lp;
    }
    // ---- tiles of this block ------------------------------------------------
    while (have && cu.j == j) {
      if (!pre_issued) {
        tc::cp_async_wait_all();
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) issue_similarity_mma(tmem, sA[buf], sB, L, idesc, mbar);
      } else {
        __syncthreads();  // penalty rows of this block are complete
      }
      pre_issued = false;
      Cursor nx;
      const bool have_nx = cursor_next(a, cu, nx);
      if (have_nx) gather_item<H>(a, nx, sA[buf ^ 1], L, cid + (buf ^ 1) * 128, ccat + (buf ^ 1) * 128);
      if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(a.err, 2);
      phase ^= 1u;
      tc::fence_after_sync();
      const int nvalid = (int)(cu.hi - cu.pos < 128 ? cu.hi - cu.pos : 128);
      const int cell = cid[buf * 128 + row];
      const int cat = ccat[buf * 128 + row];
      const float* prow = pen + cat * K;  // log2 of the penalty row
      // pass 1: v = exp(-2/sigma (1-s)) * pen = exp2(c2 (1-s) + log2 pen) (one SFU op),
      // row partial sums of v, v (1-s) (kmeans error) and v * exponent (entropy);
      // v overwrites s in TMEM.  Two 8-column loads are in flight per wait.
      float rs = 0.f, km = 0.f, vx = 0.f;
      for (int c = c_lo; c < c_hi; c += 16) {
        const bool two = c + 8 < c_hi;
        float v[8], w2[8];
        tc::tmem_ld8(tl + (uint32_t)c, v);
        if (two) tc::tmem_ld8(tl + (uint32_t)(c + 8), w2);
        tc::tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          if (i >= 8 && !two) break;
          float& x = i < 8 ? v[i] : w2[i - 8];
          const int k = c + i;
          float val = 0.f;
          if (k < K) {
            const float om = 1.f - x;
            const float ex = fmaf(c2, om, prow[k]);
            val = tc::ex2_approx(ex);
            km = fmaf(val, om, km);
            vx = fmaf(val, ex, vx);
          }
          rs += val;
          x = val;
        }
        tc::tmem_st8(tl + (uint32_t)c, v);
        if (two) tc::tmem_st8(tl + (uint32_t)(c + 8), w2);
      }
      km *= 2.f;
      tc::tmem_st_wait();
      if (NT == 256) rsp[half * 128 + row] = rs;
      // run starts of equal batch inside the tile (rows are ordered by batch)
      if (warp == 0) {
        int cnt = 0;
        for (int r0 = 0; r0 < nvalid; r0 += 32) {
          const int r = r0 + lane;
          const bool start = r < nvalid && (r == 0 || ccat[buf * 128 + r] != ccat[buf * 128 + r - 1]);
          const unsigned m = __ballot_sync(0xffffffffu, start);
          if (start) runs[cnt + __popc(m & lanemask_lt())] = r;
          cnt += __popc(m);
        }
        if (lane == 0) {
          runs[cnt] = nvalid;
          nruns = cnt;
        }
      }
      __syncthreads();
      const float rsum = NT == 256 ? rsp[row] + rsp[128 + row] : rs;
      const float inv = a.init_mode ? 1.f / fmaxf(rsum, 1e-12f) : 1.f / rsum;
      // pass 2: normalise, round to 16 bits, stage the row
      for (int c = c_lo; c < c_hi; c += 16) {
        const bool two = c + 8 < c_hi;
        float v[8], w2[8];
        tc::tmem_ld8(tl + (uint32_t)c, v);
        if (two) tc::tmem_ld8(tl + (uint32_t)(c + 8), w2);
        tc::tmem_ld_wait();
        __align__(16) H hv[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          if (i >= 8 && !two) break;
          hv[i] = from_f<H>((i < 8 ? v[i] : w2[i - 8]) * inv);
        }
        *(uint4*)(Rst + row * L.ldst + c) = *(const uint4*)hv;
        if (two) *(uint4*)(Rst + row * L.ldst + c + 8) = *(const uint4*)(hv + 8);
      }
      tc::fence_before_sync();
      // objective terms of the row (kernels_kmeans.cuh:30-96, kernels_clustering.cuh:8-62):
      // kmeans error sum r (2 (1-s)); entropy sum r ln r = (ln 2 / rs) sum v x - ln rs
      // (r = v / rs, ln v = x ln 2); each half adds its partial sums, half 0 the -ln rs.
      if (cell >= 0) {
        double e = (double)(inv * km) + (double)(sig * 0.6931471805599453f * inv * vx);
        if (half == 0) e -= (double)sig * log((double)(a.init_mode ? fmaxf(rsum, 1e-12f) : rsum));
        obj_local += e;
      }
      __syncthreads();
      // observed-count delta: one thread per cluster column, summed per batch run
      for (int kc = tid; kc < K; kc += NT) {
        float tot = 0.f;
        for (int q = 0; q < nruns; ++q) {
          const int r0 = runs[q], r1 = runs[q + 1];
          float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
          int r = r0;
          for (; r + 4 <= r1; r += 4) {
            s0 += h2f(Rst[(r + 0) * L.ldst + kc]);
            s1 += h2f(Rst[(r + 1) * L.ldst + kc]);
            s2 += h2f(Rst[(r + 2) * L.ldst + kc]);
            s3 += h2f(Rst[(r + 3) * L.ldst + kc]);
          }
          for (; r < r1; ++r) s0 += h2f(Rst[r * L.ldst + kc]);
          const float srun = (s0 + s1) + (s2 + s3);
          osm[ccat[buf * 128 + r0] * K + kc] += srun;
          tot += srun;
        }
        dsum[kc] += tot;
      }
      // write the new assignment rows
      for (int e = tid; e < nvalid * L.ldr_chunks; e += NT) {
        const int r = e / L.ldr_chunks, ch = e % L.ldr_chunks;
        const int64_t cl = cid[buf * 128 + r];
        *(uint4*)(R + cl * a.ldr + ch * 8) = *(const uint4*)(Rst + r * L.ldst + ch * 8);
      }
      buf ^= 1;
      have = have_nx;
      cu = nx;
    }
    // ---- flush this CTA's delta and carry the state (CTA 0) ----------------------
    __syncthreads();
    for (int e = tid; e < (cmax - cmin + 1) * K; e += NT) {
      const size_t o_at = (size_t)cmin * K + e;
      const double v = (double)osm[o_at];
      if (v != 0.0) atomicAdd(&Oout[o_at], v);
    }
    for (int k = tid; k < K; k += NT)
      if (dsum[k] != 0.f) atomicAdd(&Oout[(size_t)B * K + k], (double)dsum[k]);
    // carry the state forward (O_in - old(this block) - old(next block)), spread over the CTAs
    for (size_t e = ldo * blockIdx.x / gridDim.x + tid; e < ldo * (blockIdx.x + 1) / gridDim.x; e += NT) {
      double v = Oin[e];
      if (Omc) v -= Omc[e];
      if (Omn) v -= Omn[e];
      if (v != 0.0) atomicAdd(&Oout[e], v);
    }
    // the similarity of the next block's first tile does not depend on the counts:
    // start it before the barrier
    if (have && cu.j == j + 1) {
      tc::cp_async_wait_all();
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0) issue_similarity_mma(tmem, sA[buf], sB, L, idesc, mbar);
      pre_issued = true;
    }
    if (j == a.nblk - 1) {
      const double tot = block_sum(obj_local, red);
      if (tid == 0 && tot != 0.0) atomicAdd(a.obj_acc, tot);
    }
    grid_barrier(a.barrier, (unsigned)(j + 1) * gridDim.x, a.err);
  }

  // ---- objective: diversity term from the final state (kernels_clustering.cuh:68-103)
  if (blockIdx.x == 0) {
    const double* Of = a.Obuf[(a.b0 + a.nblk) % 3];
    double acc = 0.0;
    for (int e = tid; e < B * K; e += NT) {
      const int b = e / K, k = e % K;
      const double o = Of[e];
      const double E = a.Pr[b] * Of[(size_t)B * K + k];
      const double num_ = a.stabilized ? (o + E + 1.0) : (o + 1.0);
      acc += a.theta[b] * o * log(num_ / (E + 1.0));
    }
    acc = block_sum(acc, red);
    if (tid == 0) {
      *a.obj_out = *a.obj_acc + a.sigma * acc;
      *a.obj_acc = 0.0;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, (uint32_t)L.tcols);
  }
}

template <typename H, int NT>
static int launch_sweep_nt(const SweepArgs& a, const TcLayout& L, int occ_target, cudaStream_t st) {
  const void* fn = (const void*)k_tc_sweep<H, NT>;
  cudaFuncAttributes fa;
  HB_CUDA(cudaFuncGetAttributes(&fa, fn));
  const size_t stat = fa.sharedSizeBytes;  // static shared memory of the kernel
  size_t smem = L.bytes;
  const size_t per_sm = 228u * 1024u;
  // pad the request so that no more than occ_target CTAs share an SM (TMEM budget)
  if (per_sm / (smem + stat + 1024) > (size_t)occ_target)
    smem = std::min<size_t>(227u * 1024u - stat, per_sm / occ_target - stat - 2048);
  if (smem < L.bytes) smem = L.bytes;
  HB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, smem));
  occ = std::min(occ, occ_target);
  if (occ < 1) {
    set_error("tensor-core sweep: kernel does not fit on an SM");
    return HB_ERR_UNSUPPORTED;
  }
  const int64_t tiles = std::max<int64_t>(1, (std::min<int64_t>(a.bs, a.n) + 127) / 128);
  const int grid = (int)std::min<int64_t>((int64_t)num_sms() * occ, tiles);
  SweepArgs args = a;
  TcLayout lay = L;
  void* kargs[] = {(void*)&args, (void*)&lay};
  HB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(NT), kargs, smem, st));
  ++g_launches;
  return HB_OK;
}

template <typename H>
int launch_tc_sweep(const SweepArgs& a, cudaStream_t st) {
  const TcLayout L = tc_layout(a.d, a.K, a.B, a.ldr, 4);
  if (L.bytes > 227u * 1024u) {
    set_error("tensor-core sweep: shared-memory tables too large (B=%d K=%d d=%d)", a.B, a.K, a.d);
    return HB_ERR_UNSUPPORTED;
  }
  return launch_sweep_nt<H, 256>(a, L, std::max(1, 512 / L.tcols), st);
}
template int launch_tc_sweep<__half>(const SweepArgs&, cudaStream_t);
template int launch_tc_sweep<__nv_bfloat16>(const SweepArgs&, cudaStream_t);

}  // namespace hb
