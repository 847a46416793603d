// nfx_spread_noalloc: spreading for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc or hand the library a workspace: code
// running inside another framework's operator that is given only its operand
// and result buffers (an XLA/JAX FFI handler, for example), or code held to a
// fixed device-memory budget.  This entry point spreads with no allocation at
// all: the bin-sort scratch (keys, permutation, bin counts, subproblem tables)
// lives in the file-scope array below, which every GPU that loads the library
// holds until the process exits.
//
// * Limit: kNoAllocScratchBytes (64 MiB) of scratch, enough for about 1.8
//   million 2D complex64 points (the sort keeps 36-40 bytes per float point:
//   keys, permutation, radix ping-pong buffers and two copies of the folded
//   coordinates); a request needing more is rejected with NFX_ERR_UNSUPPORTED
//   before any device work.
// * Set-up: the first call on a device, with that device current, looks up the
//   array's device address with cudaGetSymbolAddress (host code cannot use the
//   array's name as a device pointer); make that first call before any stream
//   capture.  The address is kept for the life of the process: it does not
//   survive a cudaDeviceReset, after which this entry point must not be called.
// * Sharing: every call on a device uses the same array and leaves its
//   contents behind.  Nothing in it needs to start at zero: the sort writes every
//   entry it later reads.  Calls that overlap on the GPU (different streams,
//   different host threads) race on the array; serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "nfx.h"
#include "nfx_internal.h"

namespace nfx {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};
}  // namespace

}  // namespace nfx

using namespace nfx;

extern "C" {

size_t nfx_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int nfx_spread_noalloc(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* c,
                       int n_trans, void* fw, void* stream) {
  size_t need = 0;
  int st = nfx_sort_workspace_bytes(opts, M, &need);
  if (st != NFX_OK) return st;
  if (need > kNoAllocScratchBytes) {
    set_error("nfx_spread_noalloc: this request needs " + std::to_string(need) +
              " bytes of scratch but the library's fixed scratch holds " + std::to_string(kNoAllocScratchBytes) +
              " bytes; use nfx_spread with a workspace");
    return NFX_ERR_UNSUPPORTED;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("nfx_spread_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return NFX_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) {
    set_error("nfx_spread_noalloc: device index " + std::to_string(dev) +
              " is beyond the 64 devices whose scratch address the library keeps");
    return NFX_ERR_UNSUPPORTED;
  }
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) {
        set_error(std::string("nfx_spread_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return NFX_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = p;
    }
    scratch = g_noalloc_ptr[dev];
  }
  return nfx_spread(opts, x, y, z, M, c, n_trans, fw, scratch, kNoAllocScratchBytes, stream);
}

}  // extern "C"
