// Block lists without any allocation: hb_block_lists with its scratch in a
// fixed device array of this translation unit instead of a caller workspace.
//
// For callers that cannot allocate device memory at the point of the call: a
// serving loop that must not call cudaMalloc (it synchronises the device and
// can fail under memory pressure in the middle of a request), or a plain C host
// that has no allocator or memory pool to carve a workspace from.  Such a
// caller passes only its inputs and outputs; nothing here calls cudaMalloc,
// cudaFree or an allocating library routine.
//
// Limits and behaviour:
//   * the scratch is HB_BLOCK_LISTS_STATIC_MAX_BYTES (16 MiB) per device; a call
//     whose hb_block_lists_workspace_bytes() exceeds it is rejected with
//     HB_ERR_WORKSPACE and a message naming both sizes;
//   * the first call on a device (with that device current) looks up the
//     array's device address with cudaGetSymbolAddress, which may load this
//     module; make that first call before any stream capture.  The address is
//     cached per device for the life of the process: after cudaDeviceReset()
//     it is stale, so do not call this entry point again after a reset;
//   * the array is shared by every call on the device: calls that overlap in
//     time (other streams or host threads) race on it, and it keeps the last
//     call's contents.  The parts that must start at zero (the key histogram
//     and the overflow flag) are cleared on the stream by every call that
//     writes lists; n_iters == 0 returns at once without touching the device.
#include <mutex>

#include "hb_internal.h"
#include "../../include/harmony_b200.h"

namespace hb {
namespace {

constexpr size_t kStaticScratchBytes = HB_BLOCK_LISTS_STATIC_MAX_BYTES;
__device__ __align__(256) unsigned char g_block_lists_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
int static_scratch(void** out) {
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("hb_block_lists_static: device ordinal %d out of range", dev);
    return HB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_block_lists_scratch);
    if (e != cudaSuccess || !p) {
      set_error("hb_block_lists_static: cudaGetSymbolAddress failed on device %d: %s", dev,
                cudaGetErrorString(e));
      return HB_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return HB_OK;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

HB_API int hb_block_lists_static(int64_t n, int64_t block_size, const uint32_t* seeds, int32_t n_iters,
                                 const int32_t* cats, int32_t n_batches, int32_t* idx, void* stream) {
  if (n < 1 || block_size < 1 || !seeds || !idx || n_iters < 0) {
    set_error("hb_block_lists_static: bad argument");
    return HB_ERR_INVALID;
  }
  if (n_iters == 0) return HB_OK;  // no lists to write: the device is not touched
  const MembershipLayout L = membership_layout(n, block_size, cats ? n_batches : 1);
  if (L.nblk > kMaxBlocks) { set_error("hb_block_lists_static: too many blocks"); return HB_ERR_UNSUPPORTED; }
  if (L.cap > 16384) { set_error("hb_block_lists_static: n too large"); return HB_ERR_UNSUPPORTED; }
  const size_t need = hb_block_lists_workspace_bytes(n, block_size, cats ? n_batches : 1);
  if (need > kStaticScratchBytes) {
    set_error("hb_block_lists_static: needs %zu bytes of scratch, the static scratch holds %zu "
              "(use hb_block_lists with a workspace)",
              need, kStaticScratchBytes);
    return HB_ERR_WORKSPACE;
  }
  void* scratch = nullptr;
  HB_TRY(static_scratch(&scratch));
  Carver cv((void*)align_up((size_t)scratch, 256), kStaticScratchBytes - 256);
  MembershipBufs B;
  membership_carve(cv, L, B);
  cudaStream_t st = (cudaStream_t)stream;
  HB_TRY(membership_clear_err(B, st));  // the flag covers every chunk of this call
  for (int c0 = 0; c0 < n_iters; c0 += kMaxIterChunk) {
    const int C = std::min(kMaxIterChunk, n_iters - c0);
    HB_TRY(membership_build(L, B, seeds + c0, C, cats, idx + (size_t)c0 * n, st));
  }
  int err = 0;
  HB_CUDA(cudaMemcpyAsync(&err, B.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));
  if (err) { set_error("hb_block_lists_static: candidate overflow"); return HB_ERR_INTERNAL; }
  return HB_OK;
}

}  // extern "C"
