// Persistent soft-k-means sweep of the 16-bit path (one launch per k-means
// iteration).
//
// The reference updates R block by block with ~12 launches per block, the
// similarity matrix round-tripping through HBM (_cuda/harmony/clustering/
// clustering.cu:308-372).  Here one cooperative launch walks all blocks of an
// iteration.  For block j every CTA takes an even, contiguous slice of the
// block's cell list (ordered by batch, then cell) and splits it between its NG
// thread groups of 256 threads; each group, for each tile of <= 128 cells:
// gathers the 16-bit normalised embeddings into a swizzled shared tile, runs
// S = Z_tile . Y_norm^T on the tensor core (fp32 in its own TMEM columns), and in
// the epilogue forms R = normalise_L1(exp(-2/sigma (1-s)) * pen[batch]), writes
// it, and adds it to its observed-count delta.  The deltas are flushed with
// float64 atomics and a bounded grid barrier separates the blocks, because the
// penalty of block j+1 depends on the counts after block j.  The "remove old
// contribution" step of every block comes precomputed from the centroid pass
// (Omin), so no R row is read in the sweep.
//
// Two groups per CTA instead of two CTAs per SM: the runtime admits one
// TMEM-allocating CTA per SM into a cooperative launch, and the groups share
// the penalty table and the centroid tile.
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

// Grid-wide barrier of a cooperative launch, split in two: arrive once this
// CTA's writes of the block are issued, wait before the next block's counts are
// read; work that does not depend on the other CTAs goes in between.  The wait
// is bounded: after `limit_ns` (2 s unless the plan says otherwise), or once any
// CTA has given up, the CTA records error 3 and proceeds (the host reports a
// timeout).
// The arrival is a release reduction: the CTA's writes of the block (ordered before it by the
// CTA barrier) are visible to every CTA whose acquire load sees the count.
__device__ __forceinline__ void grid_arrive(unsigned* ctr) {
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(ctr) : "memory");
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void grid_wait(unsigned* ctr, unsigned target, int* err, uint64_t limit_ns) {
  if (threadIdx.x == 0) {
    const uint64_t t0 = globaltimer_ns();
    unsigned spins = 0;
    while (ld_acquire_u32(ctr) < target) {
      // give up after limit_ns, or at once when another CTA has already given up
      if ((++spins & 255u) == 0 &&
          (globaltimer_ns() - t0 > limit_ns || *(volatile int*)err != 0)) {
        atomicExch(err, 3);
        break;
      }
    }
  }
  // the acquire load above and this CTA barrier order the block's loads after every
  // arrival's release (no further fence; polls back to back, each is an L2 round trip)
  __syncthreads();
}

// Profiling build only (-DHB_SWEEP_TRACE): per-phase timestamps of thread 0 of every CTA for
// every block of the last sweep launch, %globaltimer (ns, comparable across SMs) and clock64
// (cycles, this SM), read back with hb_debug_sweep_trace().  Compiled out otherwise.
#ifdef HB_SWEEP_TRACE
constexpr int kTraceCtas = 160, kTraceBlocks = 64, kTracePts = 12;
__device__ uint64_t g_sweep_trace_ns[kTraceCtas * kTraceBlocks * kTracePts];
__device__ uint64_t g_sweep_trace_clk[kTraceCtas * kTraceBlocks * kTracePts];
#define HB_TRACE(j, pt)                                                                              \
  do {                                                                                               \
    if (threadIdx.x == 0 && blockIdx.x < kTraceCtas && (j) < kTraceBlocks) {                         \
      const size_t at_ = ((size_t)blockIdx.x * kTraceBlocks + (j)) * kTracePts + (pt);               \
      g_sweep_trace_ns[at_] = globaltimer_ns();                                                      \
      g_sweep_trace_clk[at_] = (uint64_t)clock64();                                                  \
    }                                                                                                \
  } while (0)
#else
#define HB_TRACE(j, pt) \
  do {                  \
  } while (0)
#endif

// barrier of the `nthreads` threads of thread group g (named barrier 1 + g)
__device__ __forceinline__ void group_sync(int g, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(nthreads) : "memory");
}

// Shared memory of the sweep: NG groups, each with one or two A tiles, a staging
// tile, its delta table and row tables; one centroid tile and one penalty table.
// With one A tile the next tile's rows are gathered into it once the current
// tile's MMA has completed (which is where they are gathered with two as well);
// two let the gather of a block's first tile overlap the previous block's end.
struct SweepLayout {
  TcLayout t;        // tile geometry (dpad, npad, tcols per group, ldst)
  int ng;
  int nbuf;          // A tiles per group (2, or 1 when two do not fit)
  uint32_t atile;    // bytes of one A tile
  uint32_t offA, offB, offRst, rstBytes, offPen, offOsm, osmBytes, offRows, offMisc, offBt, bytes;
};

inline SweepLayout sweep_layout(int d, int K, int B, int ldr, int ng, int nbuf) {
  SweepLayout S{};
  S.t = tc_layout(d, K, B, ldr, 4);
  S.ng = ng;
  S.nbuf = nbuf;
  auto al = [](uint32_t x, uint32_t a) { return (x + a - 1) / a * a; };
  S.atile = (uint32_t)S.t.kblk * 16384u;
  uint32_t o = 0;
  S.offA = o; o += (uint32_t)(ng * nbuf) * S.atile;
  S.offB = o; o += (uint32_t)S.t.kblk * S.t.npad * 128u;
  S.rstBytes = al(128u * S.t.ldst * 2u, 16);
  S.offRst = al(o, 16); o = S.offRst + (uint32_t)ng * S.rstBytes;
  S.offPen = al(o, 16); o = S.offPen + (uint32_t)B * S.t.npad * 4u;  // rows padded to npad
  S.osmBytes = al((uint32_t)B * K * 4u, 16);
  S.offOsm = al(o, 16); o = S.offOsm + (uint32_t)ng * S.osmBytes;
  S.offRows = al(o, 16); o = S.offRows + (uint32_t)ng * 4096u;  // cid, ccat [2][128]; rsp [<= 4][128]
  S.offMisc = al(o, 16); o = S.offMisc + 64u + 32u * 8u;
  S.offBt = al(o, 16); o = S.offBt + (uint32_t)B * 8u;  // Pr_b and theta_b (float32)
  S.bytes = o + 1024u;  // slack for 1024-byte alignment of the base
  return S;
}

// The slice of block j processed by (virtual) worker c of G: list positions [lo, hi).
__device__ __forceinline__ void slice_of(const SweepArgs& a, int j, int c, int G, int64_t& lo, int64_t& hi) {
  const int64_t s = (int64_t)j * a.bs;
  const int64_t nj = min(a.bs, a.n - s);
  lo = s + nj * c / G;
  hi = s + nj * (c + 1) / G;
}

// Work cursor over (block, tile start) of one thread group; tile = up to 128 positions.
struct Cursor {
  int j;
  int64_t pos, hi;
};

// sl[j] = the group's slice of block j (list positions [x, y)), precomputed per kernel
__device__ __forceinline__ bool cursor_first(const SweepArgs& a, int j, const int2* sl, Cursor& cu) {
  for (; j < a.nblk; ++j) {
    const int2 r = sl[j];
    if (r.x < r.y) {
      cu.j = j;
      cu.pos = r.x;
      cu.hi = r.y;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ bool cursor_next(const SweepArgs& a, const Cursor& cu, const int2* sl, Cursor& nx) {
  if (cu.pos + 128 < cu.hi) {
    nx = cu;
    nx.pos = cu.pos + 128;
    return true;
  }
  return cursor_first(a, cu.j + 1, sl, nx);
}

__device__ __forceinline__ int tile_rows(const Cursor& cu) {
  return (int)(cu.hi - cu.pos < 128 ? cu.hi - cu.pos : 128);
}

// Cell id and batch of row r of the tile at list position pos.  Issued early;
// the registers are consumed by stage_tile once the loads have landed.
struct TileIds {
  int cell, cat;
};
__device__ __forceinline__ TileIds load_tile_ids(const SweepArgs& a, int64_t pos, int nr, int r) {
  TileIds t{-1, 0};
  if (r < nr) {
    t.cell = a.idx ? __ldg(a.idx + pos + r) : (int)(pos + r);
    t.cat = __ldg(a.lcat + pos + r);
  }
  return t;
}

// Copies of the tile's normalised embedding rows into the 128B-swizzled K-major
// A tile (zero fill past the PCs and for missing rows).  gt = thread index in the
// group of 128 nparts threads: it owns row gt % 128 and every nparts-th 16-byte chunk of it.
template <typename H>
__device__ __forceinline__ void stage_tile(const SweepArgs& a, TileIds t, int gt, uint32_t sA, int dpad,
                                           int* cid, int* ccat, int nparts) {
  const int r = gt & 127, part = gt >> 7;
  if (part == 0) {
    cid[r] = t.cell;
    ccat[r] = t.cat;
  }
  const H* Zn = (const H*)a.Zn;
  const H* src = t.cell >= 0 ? Zn + (int64_t)t.cell * a.ldz : Zn;
  const int nch = dpad / 8;
  for (int ch = part; ch < nch; ch += nparts) {
    const bool ok = t.cell >= 0 && ch * 8 < a.ldz;
    const uint32_t dst = sA + (uint32_t)(ch >> 3) * 16384u + tc::sw128_off(r, ch & 7);
    tc::cp_async16(dst, ok ? (const void*)(src + ch * 8) : (const void*)Zn, ok ? 16u : 0u);
  }
}

// Starts of the runs of equal batch in a tile (rows are ordered by batch inside
// a block), ascending, terminated by nvalid.  Executed by one full warp.
__device__ __forceinline__ void tile_runs(const int* cc, int nvalid, int* runs, int* nruns) {
  const int lane = threadIdx.x & 31;
  int cnt = 0;
  for (int r0 = 0; r0 < nvalid; r0 += 32) {
    const int r = r0 + lane;
    const bool start = r < nvalid && (r == 0 || cc[r] != cc[r - 1]);
    const unsigned m = __ballot_sync(0xffffffffu, start);
    if (start) runs[cnt + __popc(m & lanemask_lt())] = r;
    cnt += __popc(m);
  }
  if (lane == 0) {
    runs[cnt] = nvalid;
    *nruns = cnt;
  }
}

// NG thread groups of 128 QS threads per CTA; each row of a tile is split over QS threads
// (column ranges), warps w, w + 4, ... of a group reading the same TMEM lanes.
template <typename H, int NG, int QS>
__global__ void __launch_bounds__(128 * QS * NG, 1) k_tc_sweep(SweepArgs a, SweepLayout SL) {
  // the k-means loop has stopped on the device (set by an earlier launch: every CTA sees it)
  if (a.stop && *(volatile const int*)a.stop) return;
  constexpr int GS = 128 * QS;  // threads of a group
  constexpr int NT = GS * NG;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const TcLayout& L = SL.t;
  const int K = a.K, B = a.B;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = tid / GS, gt = tid % GS, gw = gt >> 5;   // thread group, index and warp in it
  const int nvw = gridDim.x * NG;  // workers (thread groups) of the launch
  float* pen = (float*)(sm + SL.offPen);                     // [B][npad] exponent offsets
  float* osm = (float*)(sm + SL.offOsm + g * SL.osmBytes);   // [B][K] observed-count delta
  H* Rst = (H*)(sm + SL.offRst + g * SL.rstBytes);           // [128][ldst] staged rows
  int* cid = (int*)(sm + SL.offRows + g * 4096);             // [2][128] cell per row
  int* ccat = cid + 256;                                     // [2][128] batch per row
  float* rsp = (float*)(ccat + 256);                         // [QS][128] row sums of the column ranges
  uint64_t* mbar = (uint64_t*)(sm + SL.offMisc) + g;
  uint32_t* tmem_slot = (uint32_t*)(sm + SL.offMisc + 32);
  double* red = (double*)(sm + SL.offMisc + 64);
  float* prb = (float*)(sm + SL.offBt);  // [B] Pr_b, then [B] theta_b: read every block, so kept here
  float* thb = prb + B;
  __shared__ float ocol_s[2][256];         // column sums of the state (E / Pr_b), by block parity
  __shared__ int2 crange[kMaxBlocks];      // batch range of this CTA's slice, per block
  __shared__ int2 gslice[NG][kMaxBlocks];  // each group's slice of every block (list positions)
  __shared__ int runs_s[NG][2][130];       // run starts of the two tile buffers
  __shared__ int nruns_s[NG][2];
  __shared__ double carry_s[NT];           // the thread's first state-carry entry of the block
  int(*runs)[130] = runs_s[g];
  int* nruns = nruns_s[g];
  H* R = (H*)a.R;
  const uint32_t sA[2] = {tc::smem_u32(sm + SL.offA + (uint32_t)(SL.nbuf * g) * SL.atile),
                          tc::smem_u32(sm + SL.offA + (uint32_t)(SL.nbuf * g + SL.nbuf - 1) * SL.atile)};
  const uint32_t sB = tc::smem_u32(sm + SL.offB);
  const size_t ldo = (size_t)(B + 1) * K;
  // this CTA's share of the state carry: the batch rows and the column-sum row B, which the
  // flush keeps equal to the sum of the batch rows
  const int carry0 = (int)((int64_t)(B + 1) * K * blockIdx.x / gridDim.x);
  const int carry1 = (int)((int64_t)(B + 1) * K * (blockIdx.x + 1) / gridDim.x);

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, (uint32_t)(NG * L.tcols));
    tc::tmem_relinquish();
    tc::fence_before_sync();
  }
  if (gt == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  load_centroids_swizzled((const H*)a.Yn, a.ldy, K, sB, L);
  for (int b = tid; b < B; b += NT) {
    prb[b] = (float)a.Pr[b];
    thb[b] = (float)a.theta[b];
  }
  for (int e = tid; e < NG * a.nblk; e += NT) {
    const int gg = e / a.nblk, jj = e % a.nblk;
    int64_t lo, hi;
    slice_of(a, jj, blockIdx.x * NG + gg, nvw, lo, hi);
    gslice[gg][jj] = make_int2((int)lo, (int)hi);
  }
  __syncthreads();
  const int2* gsl = gslice[g];
  Cursor cu;
  bool have = cursor_first(a, 0, gsl, cu);
  if (have) stage_tile<H>(a, load_tile_ids(a, cu.pos, tile_rows(cu), gt & 127), gt, sA[0], L.dpad, cid, ccat, QS);
  __syncthreads();
  if (have && gw == 0) tile_runs(ccat, tile_rows(cu), runs[0], &nruns[0]);
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot + (uint32_t)(g * L.tcols);

  const uint32_t idesc = tc::idesc_f16(128, L.npad, is_bf16<H>::value, false, false);
  const float c2 = (float)(-2.0 / a.sigma * 1.4426950408889634);  // exp(x) = exp2(x log2 e)
  const int ldp = L.npad;
  const float sig = (float)a.sigma;
  const int half = gw >> 2;  // warps 4 half .. 4 half + 3 of the group: column range `half` of QS
  const int row = (gw & 3) * 32 + lane;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const int nh = (L.npad / QS + 7) / 8 * 8;  // columns per range (a multiple of 8)
  const int c_lo = half * nh, c_hi = min(L.npad, c_lo + nh);
  double obj_local = 0.0;
  uint32_t phase = 0;
  int buf = 0;
  bool pre_issued = false;  // the MMA of the group's current tile was issued before the last barrier
  int pend_rows = 0, pend_buf = 0;  // rows of the block's last tile whose R store is deferred
  // batch range of every block's CTA slice (the list is ordered by batch within a block);
  // the CTA slice is the union of its groups' slices
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

  __syncthreads();
  for (int j = 0; j < a.nblk; ++j) {
    HB_TRACE(j, 0);
    const double* Oin = a.Obuf[(a.b0 + j) % 3];
    double* Oout = a.Obuf[(a.b0 + j + 1) % 3];
    double* Ozero = a.Obuf[(a.b0 + j + 2) % 3];
    const double* Omc = (a.Omin && j == 0) ? a.Omin : nullptr;                       // this block
    const double* Omn = (a.Omin && j + 1 < a.nblk) ? a.Omin + (size_t)(j + 1) * ldo : nullptr;  // next
    for (size_t e = (size_t)blockIdx.x * NT + tid; e < ldo; e += (size_t)gridDim.x * NT) Ozero[e] = 0.0;
    // one round of loads: this CTA's share of the state carry (O_in - old(this block) -
    // old(next block); the first NT entries, parked in shared memory below so that the flush
    // before the grid arrival does not wait for L2), the column sums (row B of the state) and
    // the state entries of the first penalty rows
    const bool carry_mine = carry0 + tid < carry1;
    double c_in = 0.0, c_mc = 0.0, c_mn = 0.0;
    if (carry_mine) {
      c_in = Oin[carry0 + tid];
      if (Omc) c_mc = Omc[carry0 + tid];
      if (Omn) c_mn = Omn[carry0 + tid];
    }
    float* ocol = ocol_s[j & 1];
    const int cmin = crange[j].x, cmax = crange[j].y;
    const int npen = (cmax - cmin + 1) * ldp;
    constexpr int kPre = 2;
    float opre[kPre];
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
      const int e = tid + q * NT, k = e % ldp;
      opre[q] = 0.f;
      if (!a.init_mode && e < npen && k < K) {
        const size_t o_at = (size_t)(cmin + e / ldp) * K + k;
        opre[q] = (float)(Oin[o_at] - (Omc ? Omc[o_at] : 0.0));
      }
    }
    if (!a.init_mode)
      for (int k = tid; k < K; k += NT) {
        const size_t o_at = (size_t)B * K + k;
        ocol[k] = (float)(Oin[o_at] - (Omc ? Omc[o_at] : 0.0));
      }
    if (carry_mine) carry_s[tid] = c_in - c_mc - c_mn;  // read back by this thread at the flush
    __syncthreads();
    HB_TRACE(j, 1);
    // exponent offsets of the batches present: v = exp2(c2 (1 - s) + log2 pen)
    // = exp2(pc - c2 s) with pc = c2 + theta_b log2((E+1)/(O[+E]+1)) (kernels_pen.cuh:8-21);
    // padding columns get a large negative offset (v = 0).  Zero the delta rows.
    for (int e = tid, q = 0; e < npen; e += NT, ++q) {
      const int b = cmin + e / ldp, k = e % ldp;
      float pc = -1e30f;
      if (k < K) {
        const size_t o_at = (size_t)b * K + k;
#pragma unroll
        for (int gq = 0; gq < NG; ++gq) ((float*)(sm + SL.offOsm + gq * SL.osmBytes))[o_at] = 0.f;
        float lp = 0.f;
        if (!a.init_mode) {
          float o = 0.f;
#pragma unroll
          for (int i = 0; i < kPre; ++i)
            if (q == i) o = opre[i];
          if (q >= kPre) o = (float)(Oin[o_at] - (Omc ? Omc[o_at] : 0.0));
          const float E = prb[b] * ocol[k];
          const float denom = a.stabilized ? (o + E + 1.f) : (o + 1.f);
          lp = thb[b] * (tc::lg2_approx(E + 1.f) - tc::lg2_approx(denom));
        }
        pc = c2 + lp;
      }
      pen[(size_t)b * ldp + k] = pc;
    }
    __syncthreads();
    HB_TRACE(j, 2);
    // ---- this group's tiles of the block ------------------------------------------
    while (have && cu.j == j) {
      if (!pre_issued) {
        tc::cp_async_wait_all();
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        group_sync(g, GS);
        if (gt == 0) issue_similarity_mma(tmem, sA[buf], sB, L, idesc, mbar);
      }
      pre_issued = false;
      Cursor nx;
      const bool have_nx = cursor_next(a, cu, gsl, nx);
      TileIds tn{-1, 0};
      if (have_nx) tn = load_tile_ids(a, nx.pos, tile_rows(nx), gt & 127);
      if (!tc::mbar_wait(mbar, phase, kMaxPolls)) atomicExch(a.err, 2);
      phase ^= 1u;
      tc::fence_after_sync();
      HB_TRACE(j, 3);
      const int nvalid = tile_rows(cu);
      const int cell = cid[buf * 128 + row];
      const int cat = ccat[buf * 128 + row];
      const float* prow = pen + cat * ldp;  // exponent offsets of the row's batch
      // pass 1: v = exp(-2/sigma (1-s)) * pen = exp2(pc - c2 s) (one SFU op), row
      // partial sums of v, v s (kmeans error) and v * exponent (entropy); v
      // overwrites s in TMEM.  Two 8-column loads are in flight per wait.
      // warps whose 32 rows all lie past the tile's cells skip both passes (warp-uniform)
      const bool rows_live = (gw & 3) * 32 < nvalid;
      float rs = 0.f, kx = 0.f, vx = 0.f;
      if (rows_live) for (int c = c_lo; c < c_hi; c += 16) {
        const bool two = c + 8 < c_hi;
        float v[8], w2[8], pc[16];
        tc::tmem_ld8(tl + (uint32_t)c, v);
        if (two) tc::tmem_ld8(tl + (uint32_t)(c + 8), w2);
        *(float4*)(pc + 0) = *(const float4*)(prow + c);
        *(float4*)(pc + 4) = *(const float4*)(prow + c + 4);
        if (two) {
          *(float4*)(pc + 8) = *(const float4*)(prow + c + 8);
          *(float4*)(pc + 12) = *(const float4*)(prow + c + 12);
        }
        tc::tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          if (i >= 8 && !two) break;
          float& x = i < 8 ? v[i] : w2[i - 8];
          const float ex = fmaf(-c2, x, pc[i]);
          const float val = tc::ex2_approx(ex);
          kx = fmaf(val, x, kx);
          vx = fmaf(val, ex, vx);
          rs += val;
          x = val;
        }
        tc::tmem_st8(tl + (uint32_t)c, v);
        if (two) tc::tmem_st8(tl + (uint32_t)(c + 8), w2);
      }
      const float km = 2.f * (rs - kx);  // sum v (2 (1 - s))
      tc::tmem_st_wait();
      rsp[half * 128 + row] = rs;
      group_sync(g, GS);
      HB_TRACE(j, 4);
      float rsum = 0.f;
#pragma unroll
      for (int q = 0; q < QS; ++q) rsum += rsp[q * 128 + row];
      const float rsafe = a.init_mode ? fmaxf(rsum, 1e-12f) : rsum;
      const float inv = 1.f / rsafe;
      // pass 2: normalise, round to 16 bits, stage the row (for the counts and the R store)
      if (rows_live) for (int c = c_lo; c < c_hi; c += 16) {
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
      tc::fence_proxy_async_smem();  // the staged rows are the source of bulk stores
      tc::fence_before_sync();
      // objective terms of the row (kernels_kmeans.cuh:30-96, kernels_clustering.cuh:8-62):
      // kmeans error sum r (2 (1-s)); entropy sum r ln r = (ln 2 / rs) sum v x - ln rs
      // (r = v / rs, ln v = x ln 2); each half adds its partial sums, half 0 the -ln rs.
      if (cell >= 0) {
        constexpr float kLn2 = 0.6931471805599453f;
        float e = inv * fmaf(sig * kLn2, vx, km);
        if (half == 0) e -= sig * kLn2 * tc::lg2_approx(rsafe);
        obj_local += (double)e;
      }
      // copies of the next tile (its ids have landed by now)
      if (have_nx) stage_tile<H>(a, tn, gt, sA[buf ^ 1], L.dpad, cid + (buf ^ 1) * 128, ccat + (buf ^ 1) * 128, QS);
      group_sync(g, GS);
      HB_TRACE(j, 5);
      // the new assignment rows: one bulk store per row (ldr 16-bit values).  The last
      // tile of the block stores its rows after the grid arrival, while the other CTAs
      // finish the block (nothing reads R during the sweep).
      const bool last_of_block = !(have_nx && nx.j == j);
      if (!last_of_block) {
        if (gt < nvalid) tc::bulk_store(R + (int64_t)cid[buf * 128 + gt] * a.ldr, tc::smem_u32(Rst + gt * L.ldst),
                                        (uint32_t)a.ldr * 2u);
        tc::bulk_commit();
      } else {
        pend_rows = nvalid;
        pend_buf = buf;
      }
      if (have_nx && gw == 0) tile_runs(ccat + (buf ^ 1) * 128, tile_rows(nx), runs[buf ^ 1], &nruns[buf ^ 1]);
      // observed-count delta: one thread per cluster column (warp 0 last), summed per batch run
      const int* rn = runs[buf];
      const int nrn = nruns[buf];
      for (int kc = (gt + GS - 32) % GS; kc < K; kc += GS) {
        for (int q = 0; q < nrn; ++q) {
          const int r0 = rn[q], r1 = rn[q + 1];
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
        }
      }
      if (!last_of_block) tc::bulk_wait_read_all();  // Rst is rewritten by the next tile (after a barrier)
      buf ^= 1;
      have = have_nx;
      cu = nx;
    }
    // ---- flush the CTA's deltas and carry the state ------------------------------
    HB_TRACE(j, 6);
    __syncthreads();
    // one thread per cluster column: the CTA's batch rows, then their sum into row B
    for (int k = tid; k < K; k += NT) {
      float colv = 0.f;
      for (int b = cmin; b <= cmax; ++b) {
        const size_t o_at = (size_t)b * K + k;
        float v = 0.f;
#pragma unroll
        for (int q = 0; q < NG; ++q) v += ((const float*)(sm + SL.offOsm + q * SL.osmBytes))[o_at];
        if (v != 0.f) atomicAdd(&Oout[o_at], (double)v);
        colv += v;
      }
      if (colv != 0.f) atomicAdd(&Oout[(size_t)B * K + k], (double)colv);
    }
    // carry the state forward (O_in - old(this block) - old(next block)), spread over the CTAs
    if (carry_mine && carry_s[tid] != 0.0) atomicAdd(&Oout[carry0 + tid], carry_s[tid]);
    for (int e = carry0 + tid + NT; e < carry1; e += NT) {
      double v = Oin[e];
      if (Omc) v -= Omc[e];
      if (Omn) v -= Omn[e];
      if (v != 0.0) atomicAdd(&Oout[e], v);
    }
    if (j == a.nblk - 1) {
      const double tot = block_sum(obj_local, red);
      if (tid == 0 && tot != 0.0) atomicAdd(a.obj_acc, tot);
    }
    HB_TRACE(j, 7);
    grid_arrive(a.barrier);
    HB_TRACE(j, 8);
    if (pend_rows > 0) {  // coalesced 16-byte stores: consecutive threads on consecutive chunks of a row
      const int nch = a.ldr / 8;
      for (int e = gt; e < pend_rows * nch; e += GS) {
        const int r = e / nch, c = e - r * nch;
        *(uint4*)(R + (int64_t)cid[pend_buf * 128 + r] * a.ldr + c * 8) = *(const uint4*)(Rst + r * L.ldst + c * 8);
      }
      pend_rows = 0;
    }
    // the similarity of the group's next tile (next block) does not depend on the
    // counts: start it while the other CTAs finish this block
    if (have && cu.j == j + 1) {
      tc::cp_async_wait_all();
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      group_sync(g, GS);
      if (gt == 0) issue_similarity_mma(tmem, sA[buf], sB, L, idesc, mbar);
      pre_issued = true;
    }
    HB_TRACE(j, 9);
    grid_wait(a.barrier, (unsigned)(j + 1) * (gridDim.x + a.unmet), a.err, a.wait_ns);
    HB_TRACE(j, 10);
  }

  // ---- objective: diversity term from the final state (kernels_clustering.cuh:68-103)
  if (blockIdx.x == 0) {
    const double* Of = a.Obuf[(a.b0 + a.nblk) % 3];
    float* ocol = ocol_s[0];
    for (int k = tid; k < K; k += NT) ocol[k] = (float)Of[(size_t)B * K + k];
    __syncthreads();
    double acc = 0.0;
    for (int e = tid; e < B * K; e += NT) {
      const int b = e / K, k = e % K;
      const double o = Of[e];
      const double E = a.Pr[b] * (double)ocol[k];
      const double num_ = a.stabilized ? (o + E + 1.0) : (o + 1.0);
      acc += a.theta[b] * o * log(num_ / (E + 1.0));
    }
    acc = block_sum(acc, red);
    if (tid == 0) {
      const double obj = *a.obj_acc + a.sigma * acc;
      *a.obj_out = obj;
      *a.obj_acc = 0.0;
      // window-3 convergence over this outer iteration's objectives (clustering.cu:380-387),
      // the same expressions as the host test
      if (a.stop && a.it >= 3) {
        const double* h = a.obj_out - a.it;
        const double o = h[a.it - 1] + h[a.it - 2] + h[a.it - 3];
        const double nw = obj + h[a.it - 1] + h[a.it - 2];
        if ((o - nw) < a.tol * fabs(o)) *a.stop = a.it + 1;
      }
    }
  }
  tc::bulk_wait_all();
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(*tmem_slot, (uint32_t)(NG * L.tcols));
  }
  // the grid barrier resets itself for the next launch: the last CTA out (every other CTA has
  // passed its final wait) zeroes the arrival and exit counts
  if (tid == 0 && atomicAdd(a.barrier + 1, 1u) == gridDim.x - 1) {
    a.barrier[0] = 0u;
    a.barrier[1] = 0u;
  }
}

template <typename H, int NG, int QS>
static int launch_sweep_ng(const SweepArgs& a, const SweepLayout& SL, cudaStream_t st) {
  const void* fn = (const void*)k_tc_sweep<H, NG, QS>;
  const size_t smem = SL.bytes;
  HB_TRY(allow_max_dyn_smem(fn));
  int occ = 0;
  HB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128 * QS * NG, smem));
  if (occ < 1) {
    set_error("tensor-core sweep: kernel does not fit on an SM");
    return HB_ERR_UNSUPPORTED;
  }
  // one CTA per SM: the TMEM of an SM is shared out between the CTA's groups
  const int64_t tiles = std::max<int64_t>(1, (std::min<int64_t>(a.bs, a.n) + 127) / 128);
  int64_t cap = num_sms();
  if (a.max_ctas > 0) cap = std::min<int64_t>(cap, a.max_ctas);
  const int grid = (int)std::min<int64_t>(cap, tiles);
  SweepArgs args = a;
  SweepLayout lay = SL;
  void* kargs[] = {(void*)&args, (void*)&lay};
  HB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(128 * QS * NG), kargs, smem, st));
  ++g_launches;
  return HB_OK;
}

// Dynamic plus static shared memory of k_tc_sweep<H, NG, QS> fits in one CTA.
template <typename H, int NG, int QS>
static int sweep_fits(const SweepLayout& SL, bool& fits) {
  cudaFuncAttributes fa;
  HB_CUDA(cudaFuncGetAttributes(&fa, (const void*)k_tc_sweep<H, NG, QS>));
  int dev = 0, optin = 0;
  HB_CUDA(cudaGetDevice(&dev));
  HB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  fits = (size_t)SL.bytes + fa.sharedSizeBytes <= (size_t)optin && NG * SL.t.tcols <= 512;
  return HB_OK;
}

// Layout preference: two thread groups (two threads per row) before one group (four threads
// per row, so the CTA still runs 512 threads), two A tiles per group before one.
template <typename H>
int launch_tc_sweep(const SweepArgs& a, cudaStream_t st) {
  bool fits = false;
  if (a.form != HB_SWEEP_AUTO) {  // a forced layout (the autotuner's choice)
    const int ng = a.form <= HB_SWEEP_2x2_1BUF ? 2 : 1;
    const int nbuf = (a.form == HB_SWEEP_2x2_2BUF || a.form == HB_SWEEP_1x4_2BUF) ? 2 : 1;
    const SweepLayout SF = sweep_layout(a.d, a.K, a.B, a.ldr, ng, nbuf);
    if (ng == 2) {
      HB_TRY((sweep_fits<H, 2, 2>(SF, fits)));
      if (fits) return launch_sweep_ng<H, 2, 2>(a, SF, st);
    } else {
      HB_TRY((sweep_fits<H, 1, 4>(SF, fits)));
      if (fits) return launch_sweep_ng<H, 1, 4>(a, SF, st);
    }
    set_error("tensor-core sweep: layout %d does not fit in shared memory (B=%d K=%d d=%d)", a.form, a.B, a.K, a.d);
    return HB_ERR_UNSUPPORTED;
  }
  // Blocks of at most one 128-cell tile per CTA run one 512-thread stream per CTA (four threads
  // a row: each tile's row pass is shorter); larger blocks two 256-thread streams (more tiles in
  // flight per SM).  B200, C2 shapes, bf16, us per sweep: 59 tiles a block 162 (one stream) vs
  // 174 (two), 118 tiles 170 vs 182, 196 tiles 249 vs 202, 392 tiles 358 vs 308.
  int64_t cap = num_sms();
  if (a.max_ctas > 0) cap = std::min<int64_t>(cap, a.max_ctas);
  const bool one_stream_first = (std::min<int64_t>(a.bs, a.n) + 127) / 128 <= cap;
  for (int pass = 0; pass < 2; ++pass) {
    if ((pass == 0) != one_stream_first) {
      for (int nbuf = 2; nbuf >= 1; --nbuf) {
        const SweepLayout S2 = sweep_layout(a.d, a.K, a.B, a.ldr, 2, nbuf);
        HB_TRY((sweep_fits<H, 2, 2>(S2, fits)));
        if (fits) return launch_sweep_ng<H, 2, 2>(a, S2, st);
      }
    } else {
      for (int nbuf = 2; nbuf >= 1; --nbuf) {
        const SweepLayout S1 = sweep_layout(a.d, a.K, a.B, a.ldr, 1, nbuf);
        HB_TRY((sweep_fits<H, 1, 4>(S1, fits)));
        if (fits) return launch_sweep_ng<H, 1, 4>(a, S1, st);
      }
    }
  }
  set_error("tensor-core sweep: shared-memory tables too large (B=%d K=%d d=%d)", a.B, a.K, a.d);
  return HB_ERR_UNSUPPORTED;
}
template int launch_tc_sweep<__half>(const SweepArgs&, cudaStream_t);
template int launch_tc_sweep<__nv_bfloat16>(const SweepArgs&, cudaStream_t);

int tc_sweep_fits_any(int d, int K, int B, bool& fits) {
  const int ldr = (K + 7) / 8 * 8;
  fits = false;
  for (int ng = 2; ng >= 1 && !fits; --ng)
    for (int nbuf = 2; nbuf >= 1 && !fits; --nbuf) {
      const SweepLayout S = sweep_layout(d, K, B, ldr, ng, nbuf);
      if (ng == 2) {
        HB_TRY((sweep_fits<__nv_bfloat16, 2, 2>(S, fits)));
      } else {
        HB_TRY((sweep_fits<__nv_bfloat16, 1, 4>(S, fits)));
      }
    }
  return HB_OK;
}

}  // namespace hb

#ifdef HB_SWEEP_TRACE
// [kTraceCtas][kTraceBlocks][kTracePts] timestamps of the last sweep (profiling build only)
extern "C" __attribute__((visibility("default"))) int hb_debug_sweep_trace(uint64_t* ns, uint64_t* clk,
                                                                           size_t count) {
  const size_t n = std::min(count, (size_t)hb::kTraceCtas * hb::kTraceBlocks * hb::kTracePts);
  if (cudaMemcpyFromSymbol(ns, hb::g_sweep_trace_ns, n * sizeof(uint64_t)) != cudaSuccess) return 4;
  if (cudaMemcpyFromSymbol(clk, hb::g_sweep_trace_clk, n * sizeof(uint64_t)) != cudaSuccess) return 4;
  return 0;
}
#endif
