// Internal interfaces between the engine's translation units.
#pragma once

#include <algorithm>
#include <cmath>
#include <mutex>
#include <utility>
#include <vector>
#include <cuda.h>
#include "hb_common.cuh"

namespace hb {

// ---- block membership -------------------------------------------------------
struct MembershipLayout {
  int64_t n, bs;
  int nblk, ntiles, cap, max_slots;
  int nsub;  // batch codes per block bucket (1 = order by cell index only)
};
struct MembershipBufs {
  uint32_t* seeds;
  uint32_t* hist;
  int* bnd_slot;
  uint32_t* bnd_q;
  int* slot_bin;
  int* nslots;
  int16_t* lut;
  uint32_t* cand_cnt;
  uint32_t* cand;
  uint32_t* split;
  uint32_t* counts;
  uint32_t* offsets;
  uint32_t* totals;
  int* err;
};
MembershipLayout membership_layout(int64_t n, int64_t bs, int nsub);
void membership_carve(Carver& cv, const MembershipLayout& L, MembershipBufs& B);
// lcat (optional): lcat[c*n + p] = cats[idx[c*n + p]], the batch of each list position;
// ckey (optional): ckey[c*n + i] = block(i) * (n_batches + 1) + cats[i], the (block, batch)
// key of each cell
int membership_build(const MembershipLayout& L, const MembershipBufs& B, const uint32_t* h_seeds,
                     int n_iters, const int32_t* cats, int32_t* idx, cudaStream_t st,
                     int32_t* lcat = nullptr, int32_t* ckey = nullptr, int n_batches = 0);
// B.err (candidate overflow) is set by the builds and cleared only by membership_clear_err
int membership_clear_err(const MembershipBufs& B, cudaStream_t st);
// gate (optional): every launch of the build returns at once while *gate is non-zero
int membership_build_dev(const MembershipLayout& L, const MembershipBufs& B, const uint32_t* seeds,
                         uint32_t seed0, int n_iters, const int32_t* cats, int32_t* idx,
                         cudaStream_t st, int32_t* lcat = nullptr, int32_t* ckey = nullptr,
                         int n_batches = 0, const int* gate = nullptr);

// ---- SIMT kernels of the plain (fp32 / fp64) path ----------------------------
// Row L2 normalisation, inverse norm clamped to 1e12 (reference semantics).
template <typename TI, typename TO>
int launch_l2_normalize(const TI* src, int64_t rows, int cols, int ld_src, TO* dst, int ld_dst,
                        cudaStream_t st);

struct AccumChunk {  // a run of cells that all belong to batch `batch`
  int64_t start;     // position in the cell list (identity or batch-sorted index)
  int32_t len;
  int32_t batch;
};

// Optional by-product of the centroid pass over a block-ordered cell list:
// Omin[pos / bs][cats[cell]][k] += W[cell][k] and Omin[pos / bs][B][k] += W[cell][k]
// (layout [nblk][B+1][K], float64, zeroed by the caller)
struct OminArgs {
  double* Omin;
  const int32_t* cats;
  int64_t bs;
  int B;
};

// P[chunk][k][c] = sum over the chunk's cells i of W[i][k] * V[i][c]
// (gate, here and below: nullptr, or a device flag; the launch returns at once while it is set)
template <typename TS, typename TV, typename TA>
int launch_accum(const TS* W, int ldw, const TV* V, int ldv, const int32_t* cell_index,
                 const AccumChunk* chunks, int n_chunks, int K, int d, TA* P, cudaStream_t st,
                 OminArgs om = OminArgs{nullptr, nullptr, 1, 1}, const int* gate = nullptr);

// Y_norm[k] = l2norm(sum_chunks P[chunk][k]); optional 16-bit copy.
template <typename TA, typename TY>
int launch_centroid_reduce(const TA* P, int n_chunks, int K, int d, TY* Yn, int ldy,
                           cudaStream_t st, const int* stop = nullptr);

struct BlockArgs {
  const void* Zn;
  int ldz;
  void* R;
  int ldr;
  const int32_t* cats;
  const void* Yn;
  int ldy;
  double* O;            // [B][K] observed counts (float64)
  const double* Pr;     // [B] batch proportions
  const double* theta;  // [B]
  const int32_t* idx_new;  // nullptr -> identity (start at new_start)
  int64_t new_start;
  int64_t n_new;
  const double* Om_cur;   // [B][K] old contribution of this block (nullptr = none)
  const double* Om_next;  // [B][K] old contribution of the next block (nullptr = none)
  double* obj_acc;      // kmeans error + entropy of the new rows
  double sigma;
  int d, K, B;
  int stabilized;
  int init_mode;        // no penalty, L1 clamp 1e-12 (initial R)
  void* pen_g;          // [B][K] of the storage type: the penalty table in global memory, used when
                        // the B x K tables do not fit in shared memory (many batches)
  const int* stop;      // nullptr, or the device-side k-means stop: return at once when set
};
int launch_block_update_f32(const BlockArgs& a, const double* O_in, double* O_out, double* O_zero,
                            cudaStream_t st);
int launch_block_update_f64(const BlockArgs& a, const double* O_in, double* O_out, double* O_zero,
                            cudaStream_t st);

// stop (optional): the device-side k-means stop; the launch returns at once when it is set,
// otherwise it applies the window-3 test to obj_out[-it .. 0] and sets *stop = it + 1
// (clustering.cu:380-387)
int launch_objective_finalize(const double* O, const double* Pr, const double* theta, double sigma,
                              int B, int K, int stabilized, double* obj_acc, double* obj_out,
                              cudaStream_t st, int* stop = nullptr, int it = 0, double tol = 0.0);

// ---- device-side run control ----------------------------------------------------
// A run enqueues its whole loop without a host sync: the k-means stop (window-3 test), the
// outer convergence test and the error flags are evaluated on the device, and every launch
// after the point where the loop would have ended returns at once (its gate is set).
struct RunCtl {
  int stop;     // k-means stop of the current outer iteration: 0 while running, else set
  int ostop;    // the run has ended (converged, or an error flag was raised)
  int conv;     // the last outer iteration passed the convergence test
  int n_outer;  // outer iterations whose k-means loop ran
};
struct OuterEndArgs {
  RunCtl* ctl;
  const double* obj_out;  // k-means objectives of this outer iteration
  double* objs;           // [max_iter_harmony + 1]: [0] initial, [o + 1] after outer iteration o
  double* kobj;           // [max_iter_harmony][max_iter_clustering]
  int32_t* kiters;        // [max_iter_harmony] k-means iterations run
  double* Obuf[3];        // the state ring of the block updates
  int outer, max_iter;    // this outer iteration; k-means launches enqueued per outer iteration
  int ring0, nblk;        // ring position at the start of the loop; block updates per iteration
  size_t o_elems;         // doubles per state buffer
  double tol_harmony;
  const int* err;         // tensor-core error flag
  const int* mb_err;      // block splitter overflow flag
};
// outer iteration start: a converged run ends; the k-means gate opens unless the run has ended
int launch_outer_begin(RunCtl* ctl, cudaStream_t st);
// end of the k-means loop of one outer iteration: records the objectives, moves the state to
// the ring position the host enqueued against (when the loop stopped early), applies the outer
// convergence test (_harmony/__init__.py:722-734) and ends the run on an error flag
int launch_outer_end(const OuterEndArgs& a, cudaStream_t st);

// ---- tensor-core kernels of the 16-bit path ------------------------------------
// 2-D tensor map over a row-major 16-bit matrix [rows][ld] for row gathers:
// box = 64 elements x 1 row, 128-byte swizzle, zero fill out of bounds.
int make_row_gather_map(CUtensorMap* tm, const void* base, int64_t rows, int ld, bool bf16);
template <typename H>
int launch_tc_similarity(const H* Zn, int ldz, const H* Yn, int ldy, const int32_t* idx,
                         const int32_t* cats, int64_t n, int d, int K, float* S, int* err,
                         cudaStream_t st);

struct SweepArgs {
  const void* Zn;
  int ldz;
  void* R;
  int ldr;
  const int32_t* cats;
  const void* Yn;
  int ldy;
  const int32_t* idx;      // block-ordered cell list (nullptr: identity, one block)
  const int32_t* lcat;     // batch of each list position (cats itself for the identity list)
  int64_t n, bs;
  int nblk;
  double* Obuf[3];
  int b0;
  const double* Omin;      // [nblk][B+1][K] old contribution per block (nullptr: none)
  const double* Pr;
  const double* theta;
  double* obj_acc;         // running kmeans-error + entropy (zero on entry, zero on exit)
  double* obj_out;         // objective of this iteration (written by CTA 0)
  double sigma;
  int d, K, B;
  int stabilized;
  int init_mode;
  int batch_sorted;        // the list is ordered by batch within each block
  int max_ctas;            // 0: one CTA per SM; otherwise at most this many CTAs
  unsigned* barrier;       // [2] arrival and exit counts: zero on entry, zeroed again by the launch
  uint64_t wait_ns;        // bound of each grid-barrier wait
  unsigned unmet;          // arrivals the barrier waits for beyond the grid's (test hook; 0)
  int form;                // HB_SWEEP_*: 0 the launcher's choice, else a forced layout
  int* err;
  // device-side k-means stop (nullptr: none): the launch returns at once when *stop is set;
  // otherwise CTA 0 applies the window-3 test to obj_out[-it .. 0] and sets *stop = it + 1
  int* stop;
  int it;
  double tol;
};

// Whether one of the sweep's layouts fits a (d, K, B) shape in one CTA (the layouts and the
// test launch_tc_sweep uses); an error status when the kernel's attributes cannot be read.
int tc_sweep_fits_any(int d, int K, int B, bool& fits);
template <typename H>
int launch_tc_sweep(const SweepArgs& a, cudaStream_t st);

struct CenArgs {
  const void* Zn;
  int ldz;
  const void* R;
  int ldr;
  const int32_t* cats;
  const int32_t* idx;   // block-ordered cell list
  const int32_t* lcat;  // batch of each list position
  int64_t n, bs;
  int d, K, B;
  float* P;             // [G][K][d] partial sums
  double* Omin;         // [nblk][B+1][K]
  int* err;
  const int* stop;      // nullptr, or the device-side k-means stop: return at once when set
};

template <typename H>
int launch_tc_centroid(const CenArgs& a, int grid, cudaStream_t st);
int tc_centroid_grid(int K);

// centroid pass in cell order (hb_centroid_stream.cu)
struct CenStreamArgs {
  int64_t n;
  int ntiles;            // 128-cell tiles over the padded rows
  const int32_t* ckey;   // [n] (block, batch) key of each cell for the coming sweep
  int d, K, nkeys;
  float* P;              // [G][K][d] partial sums
  float* Opart;          // [G][nkeys][K] partial per-key sums
  int* err;
  void* Yn;              // [K][ldy] 16-bit normalised centroids (written by the reduction)
  int ldy;
  const int* stop;       // nullptr, or the device-side k-means stop: return at once when set
  int kpb;               // keys per block (B + 1): every cell also counts toward key (block, B), the
                         // block's column sums; 0: keys are independent
};
bool cs_supported(int d, int K, int nkeys, int ldz);
int make_tile_map4(CUtensorMap* tm, const void* base, int64_t rows, int ld, int blocks, bool bf16);
template <typename H>
int launch_tc_centroid_stream(const CenStreamArgs& a, const void* Zn, int ldz, const void* R, int ldr,
                              int64_t rows_alloc, int grid, double* Omin, cudaStream_t st);

struct CorrArgs {
  const double* M;      // [K][B+1][d]
  const double* O;      // [B][K]
  const double* Pr;     // [B]
  const double* Nb;     // [B]
  double alpha, ridge_lambda, threshold;
  int prune, dynamic_lambda;
  int K, B, d;
};
template <typename TW>
int launch_ridge_solve(const CorrArgs& a, TW* W, cudaStream_t st, const int* gate = nullptr);

template <typename TA>
int launch_m_reduce(const TA* P, const AccumChunk* h_chunks, int n_chunks,
                    const int32_t* d_batch_chunk_off, int K, int B, int d, double* M, cudaStream_t st,
                    const int* gate = nullptr);

struct ApplyTile {
  int64_t start;   // position in the batch-sorted cell list
  int32_t len;
  int32_t batch;
};
template <typename T, typename TS, typename TZ>
int launch_apply_t(const T* X, int ldx, const TS* R, int ldr, const T* W, const int32_t* cell_index,
                   const ApplyTile* tiles, int n_tiles, int K, int d, T* Zhat, int ldzh, TZ* Zn,
                   int ldz, cudaStream_t st, const int* gate = nullptr);

// tensor-core correction of the 16-bit path (X, W float32; R, Z_norm 16-bit)
template <typename H>
int launch_tc_moments(const H* R, int ldr, const float* X, int ldx, const int32_t* cell_index,
                      const AccumChunk* chunks, int n_chunks, int K, int d, float* Mpart, int* err,
                      cudaStream_t st, const int* gate = nullptr);
template <typename H>
int launch_tc_apply(const float* X, int ldx, const H* R, int ldr, const float* W, const int32_t* cell_index,
                    const ApplyTile* tiles, int n_tiles, int K, int d, float* Zhat, int ldzh, H* Zn, int ldz,
                    int* err, cudaStream_t st, const int* gate = nullptr);

// ---- host helpers -------------------------------------------------------------
// Pinned host buffers for read-backs, reused across runs and never freed.  Copies into
// pageable memory are staged by the driver and serialised plans running at the same time
// on other streams; cudaFreeHost would synchronise the device.
class PinnedLease {
 public:
  explicit PinnedLease(size_t bytes) {
    std::lock_guard<std::mutex> lock(mu());
    auto& pool = free_list();
    for (size_t i = 0; i < pool.size(); ++i)
      if (pool[i].second >= bytes) {
        ptr = pool[i].first;
        size = pool[i].second;
        pool.erase(pool.begin() + (long)i);
        return;
      }
    size = std::max<size_t>(bytes, 4096);
    if (cudaMallocHost(&ptr, size) != cudaSuccess) {
      cudaGetLastError();
      ptr = nullptr;
    }
  }
  ~PinnedLease() {
    if (!ptr) return;
    std::lock_guard<std::mutex> lock(mu());
    free_list().emplace_back(ptr, size);
  }
  PinnedLease(const PinnedLease&) = delete;
  PinnedLease& operator=(const PinnedLease&) = delete;
  void* ptr = nullptr;
  size_t size = 0;

 private:
  static std::mutex& mu() {
    static std::mutex m;
    return m;
  }
  static std::vector<std::pair<void*, size_t>>& free_list() {
    static std::vector<std::pair<void*, size_t>> v;
    return v;
  }
};

}  // namespace hb
