// SIMT kernels of the plain (fp32 / fp64) Harmony path, plus the pieces shared
// with the 16-bit path (normalisation, ridge solve, correction apply).
#include <type_traits>
#include "hb_internal.h"

namespace hb {

template <typename T>
using compute_t = typename std::conditional<std::is_same<T, double>::value, double, float>::type;

// ---------------------------------------------------------------------------
// Row L2 normalise (kernels_normalize.cuh:7-54 semantics), one warp per row.
// Columns [cols, ld_dst) of the destination are zero-filled (padding).
template <typename TI, typename TO>
__global__ void k_l2_normalize(const TI* __restrict__ src, int64_t rows, int cols, int lds,
                               TO* __restrict__ dst, int ldd) {
  using TC = compute_t<TI>;
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    const TI* s = src + r * lds;
    TC ss = 0;
    for (int c = lane; c < cols; c += 32) {
      TC v = (TC)to_f(s[c]);
      ss += v * v;
    }
    ss = warp_sum(ss);
    TC inv = num<TC>::rsqrt_(ss);
    if (inv > TC(1e12)) inv = TC(1e12);
    TO* o = dst + r * ldd;
    for (int c = lane; c < ldd; c += 32)
      o[c] = (c < cols) ? from_f<TO>((TC)to_f(s[c]) * inv) : from_f<TO>(TC(0));
  }
}

template <typename TI, typename TO>
int launch_l2_normalize(const TI* src, int64_t rows, int cols, int ld_src, TO* dst, int ld_dst,
                        cudaStream_t st) {
  if (rows == 0) return HB_OK;
  int blocks = (int)std::min<int64_t>((rows + 7) / 8, (int64_t)num_sms() * 16);
  k_l2_normalize<TI, TO><<<blocks, 256, 0, st>>>(src, rows, cols, ld_src, dst, ld_dst);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_l2_normalize<float, float>(const float*, int64_t, int, int, float*, int, cudaStream_t);
template int launch_l2_normalize<double, double>(const double*, int64_t, int, int, double*, int, cudaStream_t);
template int launch_l2_normalize<float, __half>(const float*, int64_t, int, int, __half*, int, cudaStream_t);
template int launch_l2_normalize<float, __nv_bfloat16>(const float*, int64_t, int, int, __nv_bfloat16*, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Split-n weighted outer-product accumulation:
//   P[chunk][k][c] = sum_{i in chunk} W[i][k] * V[i][c]
// A CTA owns a 128 (k) x 64 (c) output tile of one chunk; 256 threads, 8 x 4
// accumulators each.  Used for the centroid sum R^T Z_norm (identity cell
// list, clustering.cu:272-276) and for the per-batch ridge moments R_b^T X_b
// (batch-sorted cell list, correction_batched.cu:55-100).
constexpr int ACC_BK = 128, ACC_BD = 64;

template <typename TS, typename TV, typename TA>
__global__ void __launch_bounds__(256) k_accum(const TS* __restrict__ W, int ldw,
                                               const TV* __restrict__ V, int ldv,
                                               const int32_t* __restrict__ cell_index,
                                               const AccumChunk* __restrict__ chunks, int K,
                                               int d, int ktiles, TA* __restrict__ P, OminArgs om,
                                               const int* gate) {
  if (gated(gate)) return;
  constexpr int ROWS = sizeof(TA) == 8 ? 16 : 32;
  constexpr int NW = ROWS * ACC_BK / 256;  // W elements per thread per step
  constexpr int NV = ROWS * ACC_BD / 256;  // V elements per thread per step
  __shared__ TA ws[ROWS][ACC_BK];
  __shared__ TA vs[ROWS][ACC_BD];
  __shared__ int rkey_s[ROWS];
  const AccumChunk ch = chunks[blockIdx.x];
  const int kt = blockIdx.y % ktiles, dt = blockIdx.y / ktiles;
  const int k0 = kt * ACC_BK, d0 = dt * ACC_BD;
  const int tid = threadIdx.x, tk = tid & 15, td = tid >> 4;
  TA acc[8][4];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = TA(0);

  TA rw[NW], rv[NV];
  int rkey = -1;
  // per-(block, batch) sums of the W rows (the "old contribution" of each block),
  // only by the CTAs of the first PC tile; rows arrive ordered by (block, batch)
  const bool do_om = om.Omin != nullptr && dt == 0;
  double om_acc = 0.0;
  int om_key = -1;
  auto load = [&](int pos) {
    if (do_om && tid < ROWS) {
      rkey = -1;
      if (pos + tid < ch.len) {
        const int64_t qq = ch.start + pos + tid;
        const int64_t cell = cell_index ? (int64_t)__ldg(cell_index + qq) : qq;
        rkey = (int)(qq / om.bs) * (om.B + 1) + __ldg(om.cats + cell);
      }
    }
#pragma unroll
    for (int q = 0; q < NW; ++q) {
      const int e = tid + q * 256, r = e / ACC_BK, kk = e % ACC_BK;
      TA v = TA(0);
      if (pos + r < ch.len && k0 + kk < K) {
        const int64_t qq = ch.start + pos + r;
        const int64_t cell = cell_index ? (int64_t)__ldg(cell_index + qq) : qq;
        v = (TA)to_f(W[cell * ldw + k0 + kk]);
      }
      rw[q] = v;
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const int e = tid + q * 256, r = e / ACC_BD, cc = e % ACC_BD;
      TA v = TA(0);
      if (pos + r < ch.len && d0 + cc < d) {
        const int64_t qq = ch.start + pos + r;
        const int64_t cell = cell_index ? (int64_t)__ldg(cell_index + qq) : qq;
        v = (TA)to_f(V[cell * ldv + d0 + cc]);
      }
      rv[q] = v;
    }
  };
  load(0);
  for (int pos = 0; pos < ch.len; pos += ROWS) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NW; ++q) { const int e = tid + q * 256; ws[e / ACC_BK][e % ACC_BK] = rw[q]; }
#pragma unroll
    for (int q = 0; q < NV; ++q) { const int e = tid + q * 256; vs[e / ACC_BD][e % ACC_BD] = rv[q]; }
    if (do_om && tid < ROWS) rkey_s[tid] = rkey;
    __syncthreads();
    if (pos + ROWS < ch.len) load(pos + ROWS);  // next step's loads overlap this step's math
    if (do_om && tid < ACC_BK && k0 + tid < K) {
      const int nrow = min(ROWS, ch.len - pos);
      for (int r = 0; r < nrow; ++r) {
        const int key = rkey_s[r];
        if (key != om_key) {
          if (om_key >= 0) {
            atomicAdd(&om.Omin[(size_t)om_key * K + k0 + tid], om_acc);
            const int sum_row = om_key - om_key % (om.B + 1) + om.B;
            atomicAdd(&om.Omin[(size_t)sum_row * K + k0 + tid], om_acc);
          }
          om_key = key;
          om_acc = 0.0;
        }
        om_acc += (double)ws[r][tid];
      }
    }
#pragma unroll 4
    for (int r = 0; r < ROWS; ++r) {
      TA wv[8], vv[4];
      // cluster tk + 16 a: the 16 threads of a half-warp read 16 consecutive values (no bank
      // conflicts; with tk * 8 + a they were 8 (fp64) or 4 (fp32) ways)
#pragma unroll
      for (int a = 0; a < 8; ++a) wv[a] = ws[r][tk + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) vv[b] = vs[r][td * 4 + b];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += wv[a] * vv[b];
    }
  }
  if (do_om && om_key >= 0 && tid < ACC_BK && k0 + tid < K) {
    atomicAdd(&om.Omin[(size_t)om_key * K + k0 + tid], om_acc);
    const int sum_row = om_key - om_key % (om.B + 1) + om.B;
    atomicAdd(&om.Omin[(size_t)sum_row * K + k0 + tid], om_acc);
  }
  TA* out = P + (size_t)blockIdx.x * K * d;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int k = k0 + tk + 16 * a;
    if (k >= K) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int c = d0 + td * 4 + b;
      if (c < d) out[(size_t)k * d + c] = acc[a][b];
    }
  }
}

template <typename TS, typename TV, typename TA>
int launch_accum(const TS* W, int ldw, const TV* V, int ldv, const int32_t* cell_index,
                 const AccumChunk* chunks, int n_chunks, int K, int d, TA* P, cudaStream_t st,
                 OminArgs om, const int* gate) {
  if (n_chunks == 0) return HB_OK;
  const int ktiles = div_up(K, ACC_BK), dtiles = div_up(d, ACC_BD);
  k_accum<TS, TV, TA><<<dim3(n_chunks, ktiles * dtiles), 256, 0, st>>>(W, ldw, V, ldv, cell_index,
                                                                       chunks, K, d, ktiles, P, om, gate);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
#define HB_ACCUM_INST(TS, TV, TA)                                                                  \
  template int launch_accum<TS, TV, TA>(const TS*, int, const TV*, int, const int32_t*, const AccumChunk*, \
                                        int, int, int, TA*, cudaStream_t, OminArgs, const int*);
HB_ACCUM_INST(float, float, float)
HB_ACCUM_INST(double, double, double)
HB_ACCUM_INST(__half, float, float)
HB_ACCUM_INST(__nv_bfloat16, float, float)
HB_ACCUM_INST(__half, __half, float)
HB_ACCUM_INST(__nv_bfloat16, __nv_bfloat16, float)
#undef HB_ACCUM_INST

// Y_norm[k] = l2normalise(sum over chunks of P[chunk][k]) -- fixed summation
// order (deterministic), float64 accumulation.  One CTA per centroid row; 8
// warps split the chunks, lanes split the PCs.
constexpr int RED_Y = 8;

template <typename TA>
__device__ __forceinline__ void reduce_rows_into(const TA* __restrict__ P, int q0, int q1,
                                                 size_t stride, size_t off, int d,
                                                 double* __restrict__ part, double* __restrict__ out) {
  // part: [RED_Y][d] scratch, out: [d]
  for (int c = threadIdx.x; c < d; c += 32) {
    double s = 0;
#pragma unroll 8
    for (int q = q0 + (int)threadIdx.y; q < q1; q += RED_Y) s += (double)__ldg(P + (size_t)q * stride + off + c);
    part[threadIdx.y * d + c] = s;
  }
  __syncthreads();
  const int t = threadIdx.y * 32 + threadIdx.x;
  for (int c = t; c < d; c += 32 * RED_Y) {
    double s = 0;
#pragma unroll
    for (int y = 0; y < RED_Y; ++y) s += part[y * d + c];
    out[c] = s;
  }
  __syncthreads();
}

template <typename TA, typename TY>
__global__ void k_centroid_reduce(const TA* __restrict__ P, int n_chunks, int K, int d,
                                  TY* __restrict__ Yn, int ldy, const int* stop) {
  if (stop && *(volatile const int*)stop) return;  // the k-means loop has stopped on the device
  extern __shared__ double sm[];
  double* part = sm;              // [RED_Y][d]
  double* ys = sm + RED_Y * d;    // [d]
  __shared__ double red[32];
  const int k = blockIdx.x;
  reduce_rows_into(P, 0, n_chunks, (size_t)K * d, (size_t)k * d, d, part, ys);
  const int t = threadIdx.y * 32 + threadIdx.x;
  double ss = 0;
  for (int c = t; c < d; c += 32 * RED_Y) ss += ys[c] * ys[c];
  ss = block_sum(ss, red);
  double inv = rsqrt(ss);
  if (inv > 1e12) inv = 1e12;
  for (int c = t; c < ldy; c += 32 * RED_Y)
    Yn[(size_t)k * ldy + c] = (c < d) ? from_f<TY>((compute_t<TY>)(ys[c] * inv)) : from_f<TY>(compute_t<TY>(0));
}

template <typename TA, typename TY>
int launch_centroid_reduce(const TA* P, int n_chunks, int K, int d, TY* Yn, int ldy, cudaStream_t st,
                           const int* stop) {
  k_centroid_reduce<TA, TY><<<K, dim3(32, RED_Y), sizeof(double) * (RED_Y + 1) * d, st>>>(P, n_chunks, K, d, Yn,
                                                                                        ldy, stop);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_centroid_reduce<float, float>(const float*, int, int, int, float*, int, cudaStream_t, const int*);
template int launch_centroid_reduce<double, double>(const double*, int, int, int, double*, int, cudaStream_t, const int*);
template int launch_centroid_reduce<float, __half>(const float*, int, int, int, __half*, int, cudaStream_t, const int*);
template int launch_centroid_reduce<float, __nv_bfloat16>(const float*, int, int, int, __nv_bfloat16*, int, cudaStream_t, const int*);

// ---------------------------------------------------------------------------
// Fused block update (plain path).
//
// For the cells of block j (list idx_new) the CTA computes the similarity row
// s = Z_norm[i] . Y_norm^T, the new assignment row
//   R[i] = normalise_L1( exp(-2/sigma (1-s)) * pen[cat_i] )
// (kernels_pen.cuh:27-82), writes it, and accumulates its contribution to the
// observed counts O[cat_i] plus the kmeans-error and entropy terms of the
// objective (kernels_kmeans.cuh:30-96, kernels_clustering.cuh:8-62).  For the
// cells of block j+1 (list idx_old) it subtracts their current R rows from O,
// which is the "remove old contribution" step the reference runs at the start
// of the next block (clustering.cu:312-332).  E is never stored: E[b][k] =
// Pr_b * sum_b' O[b'][k], the quantity the reference maintains incrementally
// (clustering.cu:328-331,367-370).
//
// O is triple-buffered: the kernel reads the state O_in, accumulates
// O_in + delta into O_out (zeroed beforehand), and zeroes O_zero (the buffer
// the previous launch read), so no CTA ever reads a buffer another CTA of the
// same launch is writing.
constexpr int BU_THREADS = 256;
template <typename T> constexpr int bu_dc() { return sizeof(T) == 8 ? 16 : 32; }

struct BlockArgsDev {
  BlockArgs a;
  const double* O_in;
  double* O_out;
  double* O_zero;
};

// Penalty table in global memory for the many-batch form of the block update: one CTA per
// cluster column k sums the state's column (E / Pr_b) in float64, then writes pen[b][k] for
// every batch (kernels_pen.cuh:8-21), as the in-kernel table below does.
template <typename T>
__global__ void k_pen_table(BlockArgsDev p, T* __restrict__ pen) {
  __shared__ double red[32];
  const BlockArgs& a = p.a;
  if (gated(a.stop)) return;
  const int K = a.K, B = a.B, k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const size_t e = (size_t)b * K + k;
    s += p.O_in[e] - (a.Om_cur ? a.Om_cur[e] : 0.0);
  }
  const double col = block_sum(s, red);
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const size_t e = (size_t)b * K + k;
    const T o = (T)(p.O_in[e] - (a.Om_cur ? a.Om_cur[e] : 0.0));
    const T E = (T)(a.Pr[b] * col);
    const T denom = a.stabilized ? (o + E + T(1)) : (o + T(1));
    pen[e] = num<T>::pow_((E + T(1)) / denom, (T)a.theta[b]);
  }
}

// GT (global tables): the penalty table comes from k_pen_table and the observed-count deltas
// go straight to O_out with float64 atomics, so shared memory holds no B x K table and any
// number of batches fits.
// Two CTAs per SM up to 128 clusters (at most 128 registers; in float64 the compiler otherwise
// took 142, and one CTA of 8 warps per SM left the kernel latency-bound).
// RPT rows per thread: tiles of TM = 16 RPT cells, each thread RPT rows x KPT clusters.
template <typename T, int KPT, bool GT, int RPT>
__global__ void __launch_bounds__(BU_THREADS, KPT <= 8 ? 2 : 1) k_block_update(BlockArgsDev p) {
  constexpr int DC = bu_dc<T>();
  constexpr int K16 = 16 * KPT;
  constexpr int BU_TM = 16 * RPT;
  constexpr int NZ = BU_TM * DC / BU_THREADS;   // Z elements per thread per chunk
  constexpr int NY = K16 * DC / BU_THREADS;     // Y elements per thread per chunk
  const BlockArgs& a = p.a;
  const int K = a.K, B = a.B, d = a.d;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const size_t tab = GT ? 0 : (size_t)B * K;
  T* pen = GT ? (T*)a.pen_g : (T*)smem_raw;    // [B][K]
  T* osm = (T*)smem_raw + tab;                 // [B][K] (shared-table form)
  T* zt = (T*)smem_raw + 2 * tab;              // [TM][DC+1]
  T* yt = zt + BU_TM * (DC + 1);               // [K16][DC+1]
  int64_t* cid = (int64_t*)(yt + (size_t)K16 * (DC + 1));  // [TM]
  int* ccat = (int*)(cid + BU_TM);             // [TM]
  __shared__ double red[32];

  const int tid = threadIdx.x, cg = tid >> 4, kg = tid & 15;
  const T* Zn = (const T*)a.Zn;
  const T* Yn = (const T*)a.Yn;
  T* R = (T*)a.R;
  if (gated(a.stop)) return;

  // zero the buffer the previous launch read
  if (p.O_zero)
    for (int e = blockIdx.x * BU_THREADS + tid; e < B * K; e += gridDim.x * BU_THREADS) p.O_zero[e] = 0.0;

  // penalty table from the current state (kernels_pen.cuh:8-21)
  if (!GT && a.n_new > 0 && !a.init_mode) {
    double* ocol = (double*)zt;  // scratch: K doubles fit in zt + yt
    for (int k = tid; k < K; k += BU_THREADS) {
      double s = 0;
      for (int b = 0; b < B; ++b) {
        const size_t e = (size_t)b * K + k;
        s += p.O_in[e] - (a.Om_cur ? a.Om_cur[e] : 0.0);
      }
      ocol[k] = s;
    }
    __syncthreads();
    for (int e = tid; e < B * K; e += BU_THREADS) {
      const int b = e / K, k = e % K;
      const T o = (T)(p.O_in[e] - (a.Om_cur ? a.Om_cur[e] : 0.0));
      const T E = (T)(a.Pr[b] * ocol[k]);
      const T denom = a.stabilized ? (o + E + T(1)) : (o + T(1));
      pen[e] = num<T>::pow_((E + T(1)) / denom, (T)a.theta[b]);
    }
  }
  if (!GT)
    for (int e = tid; e < B * K; e += BU_THREADS) osm[e] = T(0);
  __syncthreads();

  const T term = T(-2) / (T)a.sigma;
  const T sig = (T)a.sigma;
  double obj_local = 0.0;
  const int nchunk = (d + DC - 1) / DC;
  const int64_t ntiles_new = (a.n_new + BU_TM - 1) / BU_TM;
  T rz[NZ], ry[NY];
  auto load_chunk = [&](int d0) {
#pragma unroll
    for (int q = 0; q < NZ; ++q) {
      const int e = tid + q * BU_THREADS, r = e / DC, c = e % DC;
      const int64_t cell = cid[r];
      rz[q] = (cell >= 0 && d0 + c < d) ? Zn[cell * a.ldz + d0 + c] : T(0);
    }
#pragma unroll
    for (int q = 0; q < NY; ++q) {
      const int e = tid + q * BU_THREADS, k = e / DC, c = e % DC;
      ry[q] = (k < K && d0 + c < d) ? Yn[(size_t)k * a.ldy + d0 + c] : T(0);
    }
  };
  for (int64_t tile = blockIdx.x; tile < ntiles_new; tile += gridDim.x) {
    const int64_t r0 = tile * BU_TM;
    __syncthreads();
    if (tid < BU_TM) {
      const int64_t q = r0 + tid;
      int64_t cell = -1;
      if (q < a.n_new) cell = a.idx_new ? (int64_t)a.idx_new[q] : a.new_start + q;
      cid[tid] = cell;
      ccat[tid] = cell >= 0 ? a.cats[cell] : 0;
    }
    __syncthreads();
    load_chunk(0);
    T s[RPT][KPT];
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
      for (int j = 0; j < KPT; ++j) s[i][j] = T(0);
    for (int ck = 0; ck < nchunk; ++ck) {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NZ; ++q) { const int e = tid + q * BU_THREADS; zt[(e / DC) * (DC + 1) + e % DC] = rz[q]; }
#pragma unroll
      for (int q = 0; q < NY; ++q) { const int e = tid + q * BU_THREADS; yt[(e / DC) * (DC + 1) + e % DC] = ry[q]; }
      __syncthreads();
      if (ck + 1 < nchunk) load_chunk((ck + 1) * DC);
#pragma unroll 4
      for (int c = 0; c < DC; ++c) {
        T z[RPT], y[KPT];
#pragma unroll
        for (int i = 0; i < RPT; ++i) z[i] = zt[(cg * RPT + i) * (DC + 1) + c];
#pragma unroll
        for (int j = 0; j < KPT; ++j) y[j] = yt[(kg + 16 * j) * (DC + 1) + c];
#pragma unroll
        for (int i = 0; i < RPT; ++i)
#pragma unroll
          for (int j = 0; j < KPT; ++j) s[i][j] += z[i] * y[j];
      }
    }
    // epilogue: exp * penalty, L1 normalise, write, O delta, objective terms
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int row = cg * RPT + i;
      const int64_t cell = cid[row];
      const int cat = ccat[row];
      T v[KPT];
      T rs = T(0), km = T(0);
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        const int k = kg + 16 * j;
        T val = T(0);
        if (k < K) {
          val = num<T>::exp_(term * (T(1) - s[i][j]));
          if (!a.init_mode) val *= pen[cat * K + k];
          km += val * T(2) * (T(1) - s[i][j]);
        }
        v[j] = val;
        rs += val;
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        rs += __shfl_xor_sync(0xffffffffu, rs, o);
        km += __shfl_xor_sync(0xffffffffu, km, o);
      }
      T inv;
      if (a.init_mode) {
        T nrm = rs < T(1e-12) ? T(1e-12) : rs;
        inv = T(1) / nrm;
      } else {
        inv = T(1) / rs;
      }
      T rs2 = T(0);
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        v[j] *= inv;
        rs2 += v[j];
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) rs2 += __shfl_xor_sync(0xffffffffu, rs2, o);
      const T inv2 = T(1) / rs2;
      T ent = T(0);
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        const int k = kg + 16 * j;
        if (k < K) {
          const T x = v[j] * inv2;
          ent += x * num<T>::log_(x + T(1e-12));
        }
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) ent += __shfl_xor_sync(0xffffffffu, ent, o);
      if (cell >= 0) {
        T* Rrow = R + cell * a.ldr;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
          const int k = kg + 16 * j;
          if (k < K) {
            Rrow[k] = v[j];
            if (GT) atomicAdd(&p.O_out[(size_t)cat * K + k], (double)v[j]);
            else atomicAdd(&osm[cat * K + k], v[j]);
          } else if (k < a.ldr) {
            Rrow[k] = T(0);
          }
        }
        if (kg == 0) obj_local += (double)(km * inv) + (double)(sig * ent);
      }
    }
  }

  __syncthreads();
  for (int e = tid; e < B * K; e += BU_THREADS) {
    if (GT && blockIdx.x != 0) break;  // the deltas are in O_out already; CTA 0 carries the state
    double v = GT ? 0.0 : (double)osm[e];
    if (blockIdx.x == 0) {
      // this CTA also carries the state forward: O_in - old(this block) - old(next block)
      if (p.O_in) v += p.O_in[e];
      if (a.Om_cur) v -= a.Om_cur[e];
      if (a.Om_next) v -= a.Om_next[e];
    }
    if (v != 0.0) atomicAdd(&p.O_out[e], v);
  }
  const double tot = block_sum(obj_local, red);
  if (tid == 0 && tot != 0.0) atomicAdd(a.obj_acc, tot);
}

// Sets the form's function attributes and returns its CTAs per SM for `smem` bytes.
template <typename T, int KPT, bool GT, int RPT>
static int block_form_occ(size_t smem, int& occ) {
  const void* fn = (const void*)k_block_update<T, KPT, GT, RPT>;
  HB_TRY(allow_max_dyn_smem(fn));
  // float64: the largest shared-memory carveout, so that two CTAs fit on an SM (563 -> 500 ms
  // per C2 step with the 128-register bound); the float32 forms keep the default, which leaves
  // them more L1 (with the largest carveout they measured 285 -> 334 ms)
  if (sizeof(T) == 8) HB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  occ = 1;
  HB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_block_update<T, KPT, GT, RPT>, BU_THREADS, smem));
  if (occ < 1) occ = 1;
  return HB_OK;
}

template <typename T, int KPT, bool GT, int RPT>
static int launch_block_form(const BlockArgsDev& p, size_t smem, int occ, cudaStream_t st) {
  const BlockArgs& a = p.a;
  const int64_t tiles = (a.n_new + 16 * RPT - 1) / (16 * RPT);
  int grid = (int)std::min<int64_t>(std::max<int64_t>(tiles, 1), (int64_t)num_sms() * occ);
  if (GT && a.n_new > 0 && !a.init_mode) {
    k_pen_table<T><<<a.K, 256, 0, st>>>(p, (T*)a.pen_g);
    HB_LAUNCH_CHECK();
  }
  k_block_update<T, KPT, GT, RPT><<<grid, BU_THREADS, smem, st>>>(p);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

// Rows per thread: 4 (64-cell tiles), or 3 (48-cell tiles) when that takes fewer row rounds per
// CTA slot.  The tiles of a block are spread over all CTA slots, so a block of 391 tiles of 64
// cells on 296 slots (C2, 25,000 cells) runs two rounds of 4 rows, as 521 tiles of 48 cells run
// two rounds of 3.
template <typename T, int KPT, bool GT>
static int launch_block_rows(const BlockArgsDev& p, size_t tables, cudaStream_t st) {
  constexpr int DC = bu_dc<T>();
  auto smem_of = [&](int tm) {
    return sizeof(T) * (tm * (DC + 1) + (size_t)16 * KPT * (DC + 1)) + tm * (sizeof(int64_t) + sizeof(int)) +
           64 + tables;
  };
  int occ4 = 1, occ3 = 1;
  HB_TRY((block_form_occ<T, KPT, GT, 4>(smem_of(64), occ4)));
  HB_TRY((block_form_occ<T, KPT, GT, 3>(smem_of(48), occ3)));
  const int64_t n = std::max<int64_t>(p.a.n_new, 1), sms = num_sms();
  const int64_t rounds4 = ((n + 63) / 64 + sms * occ4 - 1) / (sms * occ4);
  const int64_t rounds3 = ((n + 47) / 48 + sms * occ3 - 1) / (sms * occ3);
  if (3 * rounds3 < 4 * rounds4) return launch_block_form<T, KPT, GT, 3>(p, smem_of(48), occ3, st);
  return launch_block_form<T, KPT, GT, 4>(p, smem_of(64), occ4, st);
}

// Shared-memory tables while they fit (the O deltas of a CTA summed on chip); global tables
// and direct float64 atomics for more batches.
template <typename T, int KPT>
static int launch_block_kpt(const BlockArgsDev& p, cudaStream_t st) {
  const BlockArgs& a = p.a;
  constexpr int DC = bu_dc<T>();
  const size_t base = sizeof(T) * (64 * (DC + 1) + (size_t)16 * KPT * (DC + 1)) +
                      64 * (sizeof(int64_t) + sizeof(int)) + 64;
  const size_t tables = sizeof(T) * (size_t)2 * a.B * a.K;
  if (base + tables <= 160 * 1024) return launch_block_rows<T, KPT, false>(p, tables, st);
  if (!a.pen_g) {
    set_error("block update: no global penalty table for B=%d K=%d", a.B, a.K);
    return HB_ERR_INTERNAL;
  }
  return launch_block_rows<T, KPT, true>(p, 0, st);
}

template <typename T>
int launch_block_update_dev(const BlockArgsDev& p, cudaStream_t st) {
  const int K = p.a.K;
  if (K <= 64) return launch_block_kpt<T, 4>(p, st);
  if (K <= 128) return launch_block_kpt<T, 8>(p, st);
  if (K <= 208) return launch_block_kpt<T, 13>(p, st);
  if (K <= 256) return launch_block_kpt<T, 16>(p, st);
  set_error("n_clusters=%d exceeds the supported maximum of 256", K);
  return HB_ERR_UNSUPPORTED;
}

int launch_block_update_f32(const BlockArgs& a, const double* O_in, double* O_out, double* O_zero,
                            cudaStream_t st) {
  return launch_block_update_dev<float>(BlockArgsDev{a, O_in, O_out, O_zero}, st);
}
int launch_block_update_f64(const BlockArgs& a, const double* O_in, double* O_out, double* O_zero,
                            cudaStream_t st) {
  return launch_block_update_dev<double>(BlockArgsDev{a, O_in, O_out, O_zero}, st);
}

// ---------------------------------------------------------------------------
// Objective tail: diversity term from O (kernels_clustering.cuh:68-103) added to
// the accumulated kmeans-error + entropy terms, all in float64.
__global__ void k_objective_finalize(const double* __restrict__ O, const double* __restrict__ Pr,
                                     const double* __restrict__ theta, double sigma, int B, int K,
                                     int stabilized, double* __restrict__ obj_acc,
                                     double* __restrict__ obj_out, int* stop, int it, double tol) {
  __shared__ double red[32];
  if (gated(stop)) return;
  double acc = 0;
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double col = 0;
    for (int b = 0; b < B; ++b) col += O[(size_t)b * K + k];
    for (int b = 0; b < B; ++b) {
      const double o = O[(size_t)b * K + k];
      const double E = Pr[b] * col;
      const double num_ = stabilized ? (o + E + 1.0) : (o + 1.0);
      acc += theta[b] * o * log(num_ / (E + 1.0));
    }
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) {
    const double obj = *obj_acc + sigma * acc;
    *obj_out = obj;
    *obj_acc = 0.0;
    // window-3 convergence of the k-means loop (clustering.cu:380-387) on this and the three
    // previous objectives of the loop
    if (stop && it >= 3) {
      const double o = obj_out[-1] + obj_out[-2] + obj_out[-3];
      const double nw = obj + obj_out[-1] + obj_out[-2];
      if ((o - nw) < tol * fabs(o)) *stop = it + 1;
    }
  }
}

int launch_objective_finalize(const double* O, const double* Pr, const double* theta, double sigma,
                              int B, int K, int stabilized, double* obj_acc, double* obj_out,
                              cudaStream_t st, int* stop, int it, double tol) {
  k_objective_finalize<<<1, 256, 0, st>>>(O, Pr, theta, sigma, B, K, stabilized, obj_acc, obj_out, stop,
                                          it, tol);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

// ---------------------------------------------------------------------------
// Run control (one thread / one CTA; the flags are read by the gates of later launches)
__global__ void k_outer_begin(RunCtl* c) {
  if (c->conv) c->ostop = 1;
  c->stop = c->ostop;
}

int launch_outer_begin(RunCtl* ctl, cudaStream_t st) {
  k_outer_begin<<<1, 1, 0, st>>>(ctl);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

__global__ void __launch_bounds__(256) k_outer_end(OuterEndArgs a) {
  RunCtl* c = a.ctl;
  if (gated(&c->ostop)) return;
  const int st = *(volatile const int*)&c->stop;
  const int done = st > 0 ? min(st, a.max_iter) : a.max_iter;
  for (int i = threadIdx.x; i < done; i += blockDim.x) a.kobj[(size_t)a.outer * a.max_iter + i] = a.obj_out[i];
  // the launches after the stop left the state where the last iteration put it; the host
  // enqueued the rest of the loop against the ring position of a loop that ran to the end
  const int s = (int)((a.ring0 + (int64_t)done * a.nblk) % 3);
  const int e = (int)((a.ring0 + (int64_t)a.max_iter * a.nblk) % 3);
  if (s != e) {
    for (size_t i = threadIdx.x; i < a.o_elems; i += blockDim.x) a.Obuf[e][i] = a.Obuf[s][i];
    __syncthreads();
    // the buffer after the state is the next accumulation target: zero on entry
    double* z = a.Obuf[(e + 1) % 3];
    for (size_t i = threadIdx.x; i < a.o_elems; i += blockDim.x) z[i] = 0.0;
  }
  if (threadIdx.x == 0) {
    a.kiters[a.outer] = done;
    const double prev = a.objs[a.outer];
    const double cur = done > 0 ? a.obj_out[done - 1] : 0.0;
    a.objs[a.outer + 1] = cur;
    c->n_outer = a.outer + 1;
    if (*a.err || *a.mb_err) c->ostop = 1;
    else if ((prev - cur) < a.tol_harmony * fabs(prev)) c->conv = 1;
  }
}

int launch_outer_end(const OuterEndArgs& a, cudaStream_t st) {
  k_outer_end<<<1, 256, 0, st>>>(a);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

// ---------------------------------------------------------------------------
// Ridge moments: M[k][b+1][c] = sum over batch-b chunks of P, M[k][0] = sum_b.
template <typename TA>
__global__ void k_m_reduce(const TA* __restrict__ P, const int32_t* __restrict__ batch_chunk_off,
                           int K, int B, int d, double* __restrict__ M, const int* gate) {
  if (gated(gate)) return;
  extern __shared__ double sm[];
  double* part = sm;              // [RED_Y][d]
  double* row = sm + RED_Y * d;   // [d]
  double* row0 = row + d;         // [d]
  const int k = blockIdx.x;
  const int t = threadIdx.y * 32 + threadIdx.x;
  for (int c = t; c < d; c += 32 * RED_Y) row0[c] = 0;
  for (int b = 0; b < B; ++b) {
    reduce_rows_into(P, batch_chunk_off[b], batch_chunk_off[b + 1], (size_t)K * d, (size_t)k * d, d,
                     part, row);
    for (int c = t; c < d; c += 32 * RED_Y) {
      M[((size_t)k * (B + 1) + b + 1) * d + c] = row[c];
      row0[c] += row[c];
    }
    __syncthreads();
  }
  for (int c = t; c < d; c += 32 * RED_Y) M[((size_t)k * (B + 1)) * d + c] = row0[c];
}

template <typename TA>
int launch_m_reduce(const TA* P, const AccumChunk*, int, const int32_t* d_batch_chunk_off, int K,
                    int B, int d, double* M, cudaStream_t st, const int* gate) {
  k_m_reduce<TA><<<K, dim3(32, RED_Y), sizeof(double) * (RED_Y + 2) * d, st>>>(P, d_batch_chunk_off,
                                                                              K, B, d, M, gate);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_m_reduce<float>(const float*, const AccumChunk*, int, const int32_t*, int, int, int, double*,
                                    cudaStream_t, const int*);
template int launch_m_reduce<double>(const double*, const AccumChunk*, int, const int32_t*, int, int, int, double*,
                                     cudaStream_t, const int*);

// ---------------------------------------------------------------------------
// Ridge lambda (_harmony/__init__.py:454-480), closed-form arrowhead inverse
// (kernels_correction_fast.cuh:24-123) and W = inv * M with W[0] = 0
// (correction_batched.cu:102-120), one CTA per cluster, float64.  Because the
// inverse is an arrowhead, row b+1 of inv*M is p_b u + f_b M[b+1] with
// u = (M[0] + sum_j p_j M[j+1]) / c, so W costs O(B d) per cluster.
// W is written as [B][K][d] so that each batch's K x d slice is contiguous.
template <typename TW>
__global__ void k_ridge_solve(CorrArgs a, TW* __restrict__ W, const int* gate) {
  if (gated(gate)) return;
  extern __shared__ double sh[];
  double* f = sh;          // [B]
  double* p = sh + a.B;    // [B]
  __shared__ double red[32];
  const int k = blockIdx.x, B = a.B, K = a.K, d = a.d;
  double col = 0;
  for (int b = 0; b < B; ++b) col += a.O[(size_t)b * K + k];  // N_k
  double cneg = 0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const double o = a.O[(size_t)b * K + k];
    double lam;
    if (!a.dynamic_lambda) {
      lam = a.ridge_lambda;
    } else {
      lam = a.alpha * (a.Pr[b] * col);
      if (a.prune) {
        const double nb = a.Nb[b];
        const double safe = nb > 0 ? nb : 1.0;
        if (o / safe < a.threshold || nb == 0) lam = 1e30;
      }
    }
    if (o + lam == 0.0) lam = 1e30;
    const double fb = 1.0 / (o + lam);
    f[b] = fb;
    p[b] = -fb * o;
    cneg += fb * o * o;
  }
  cneg = block_sum(cneg, red);
  const double cinv = 1.0 / (col - cneg);
  const double* Mk = a.M + (size_t)k * (B + 1) * d;
  for (int c = threadIdx.x; c < d; c += blockDim.x) {
    double u = Mk[c];
    for (int b = 0; b < B; ++b) u += p[b] * Mk[(size_t)(b + 1) * d + c];
    u *= cinv;
    for (int b = 0; b < B; ++b)
      W[((size_t)b * K + k) * d + c] = (TW)(p[b] * u + f[b] * Mk[(size_t)(b + 1) * d + c]);
  }
}

template <typename TW>
int launch_ridge_solve(const CorrArgs& a, TW* W, cudaStream_t st, const int* gate) {
  const size_t smem = sizeof(double) * 2 * a.B;
  if (smem > 48 * 1024) HB_TRY(allow_max_dyn_smem((const void*)k_ridge_solve<TW>));
  k_ridge_solve<TW><<<a.K, 128, smem, st>>>(a, W, gate);
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_ridge_solve<float>(const CorrArgs&, float*, cudaStream_t, const int*);
template int launch_ridge_solve<double>(const CorrArgs&, double*, cudaStream_t, const int*);

// ---------------------------------------------------------------------------
// Correction apply (kernels_outer.cuh:41-65) fused with the L2 renormalisation
// of the corrected embedding (_harmony/__init__.py:276):
//   Z_hat[i] = X[i] - R[i] . W[cat_i],   Z_norm[i] = l2normalise(Z_hat[i])
// A CTA takes a tile of <= 32 cells of one batch (batch-sorted cell list), so
// the batch's W slice is shared; 8 warps x 4 cells, lanes over PCs.
constexpr int AP_TM = 32, AP_KC = 32;

template <typename T, typename TS, typename TZ, int DQ>
__global__ void __launch_bounds__(256) k_apply(const T* __restrict__ X, int ldx,
                                               const TS* __restrict__ R, int ldr,
                                               const T* __restrict__ W,
                                               const int32_t* __restrict__ cell_index,
                                               const ApplyTile* __restrict__ tiles, int K, int d,
                                               T* __restrict__ Zhat, int ldzh, TZ* __restrict__ Zn,
                                               int ldz, const int* gate) {
  using TC = compute_t<T>;
  // clusters per staged W slice: 16 for float64 above 128 PCs, so the slice stays within the
  // 48 KB of static shared memory
  constexpr int KC = (sizeof(TC) == 8 && DQ > 4) ? 16 : AP_KC;
  __shared__ TC rt[AP_TM][KC + 1];
  __shared__ TC wt[KC][32 * DQ];
  __shared__ int64_t cid[AP_TM];
  if (gated(gate)) return;
  const ApplyTile tl = tiles[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid < AP_TM) cid[tid] = tid < tl.len ? (int64_t)cell_index[tl.start + tid] : -1;
  TC acc[4][DQ];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < DQ; ++q) acc[i][q] = TC(0);
  const T* Wb = W + (size_t)tl.batch * K * d;
  for (int k0 = 0; k0 < K; k0 += KC) {
    __syncthreads();
    for (int e = tid; e < AP_TM * KC; e += 256) {
      const int r = e / KC, kk = e % KC;
      const int64_t cell = cid[r];
      rt[r][kk] = (cell >= 0 && k0 + kk < K) ? (TC)to_f(R[cell * ldr + k0 + kk]) : TC(0);
    }
    for (int e = tid; e < KC * 32 * DQ; e += 256) {
      const int kk = e / (32 * DQ), c = e % (32 * DQ);
      wt[kk][c] = (k0 + kk < K && c < d) ? (TC)Wb[(size_t)(k0 + kk) * d + c] : TC(0);
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < KC; ++kk) {
      TC r[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = rt[w * 4 + i][kk];
#pragma unroll
      for (int q = 0; q < DQ; ++q) {
        const TC wv = wt[kk][lane + 32 * q];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i][q] += r[i] * wv;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t cell = cid[w * 4 + i];
    TC zh[DQ];
    TC ss = 0;
#pragma unroll
    for (int q = 0; q < DQ; ++q) {
      const int c = lane + 32 * q;
      zh[q] = (cell >= 0 && c < d) ? (TC)X[cell * ldx + c] - acc[i][q] : TC(0);
      ss += zh[q] * zh[q];
    }
    ss = warp_sum(ss);
    TC inv = num<TC>::rsqrt_(ss);
    if (inv > TC(1e12)) inv = TC(1e12);
    if (cell >= 0) {
#pragma unroll
      for (int q = 0; q < DQ; ++q) {
        const int c = lane + 32 * q;
        if (c < d) Zhat[cell * ldzh + c] = (T)zh[q];
        if (c < ldz) Zn[cell * ldz + c] = from_f<TZ>(c < d ? zh[q] * inv : TC(0));
      }
    }
  }
}

template <typename T, typename TS, typename TZ>
int launch_apply_t(const T* X, int ldx, const TS* R, int ldr, const T* W, const int32_t* cell_index,
                   const ApplyTile* tiles, int n_tiles, int K, int d, T* Zhat, int ldzh, TZ* Zn,
                   int ldz, cudaStream_t st, const int* gate) {
  if (n_tiles == 0) return HB_OK;
  const int dq = div_up(std::max(d, ldz), 32);
#define HB_AP(DQv)                                                                                 \
  k_apply<T, TS, TZ, DQv><<<n_tiles, 256, 0, st>>>(X, ldx, R, ldr, W, cell_index, tiles, K, d, Zhat, \
                                                   ldzh, Zn, ldz, gate)
  if (dq <= 1) HB_AP(1);
  else if (dq <= 2) HB_AP(2);
  else if (dq <= 4) HB_AP(4);
  else if (dq <= 8) HB_AP(8);
  else {
    set_error("n_pcs=%d exceeds the supported maximum of 256", d);
    return HB_ERR_UNSUPPORTED;
  }
#undef HB_AP
  HB_LAUNCH_CHECK();
  return HB_OK;
}
template int launch_apply_t<float, float, float>(const float*, int, const float*, int, const float*,
                                                 const int32_t*, const ApplyTile*, int, int, int,
                                                 float*, int, float*, int, cudaStream_t, const int*);
template int launch_apply_t<double, double, double>(const double*, int, const double*, int,
                                                    const double*, const int32_t*, const ApplyTile*,
                                                    int, int, int, double*, int, double*, int,
                                                    cudaStream_t, const int*);
template int launch_apply_t<float, __half, __half>(const float*, int, const __half*, int, const float*,
                                                   const int32_t*, const ApplyTile*, int, int, int,
                                                   float*, int, __half*, int, cudaStream_t, const int*);
template int launch_apply_t<float, __nv_bfloat16, __nv_bfloat16>(
    const float*, int, const __nv_bfloat16*, int, const float*, const int32_t*, const ApplyTile*, int,
    int, int, float*, int, __nv_bfloat16*, int, cudaStream_t, const int*);

}  // namespace hb
