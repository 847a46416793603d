// cuFFT glue: a mutex-guarded, size-limited (least recently used out) cache of
// batched in-place C2C/Z2Z plans keyed by (device, precision, dims, batch).  Plans
// own no work area: each (device, stream) has one, grown stream-ordered to the
// largest plan run on it and attached to the plan just before its launch, so the
// same plan can run concurrently on several streams (a plan's own work area would
// be shared by them) and cached plans hold no device memory.  Replaces the jnp.fft calls of
// nufftax/transforms/nufft1.py:81,154,232-235 and nufft2.py:317,383,454-457:
// sign = +1 is the unnormalised inverse transform (nufftax's ifftn(.) * prod(nf)),
// sign = -1 the forward transform.
#include <cufft.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "nfx.h"
#include "nfx_internal.h"

namespace nfx {

namespace {
using PlanKey = std::tuple<int, int, int, int, int, int, int>;  // dev, prec, dim, nf1, nf2, nf3, batch
std::mutex g_plan_mu;
struct PlanEntry {
  cufftHandle plan;
  size_t work_bytes;
  uint64_t last_use;
};
std::map<PlanKey, PlanEntry>& plans() {
  static std::map<PlanKey, PlanEntry> m;
  return m;
}
struct WorkArea {
  void* ptr = nullptr;
  size_t bytes = 0;
};
std::map<std::pair<int, cudaStream_t>, WorkArea>& work_areas() {
  static std::map<std::pair<int, cudaStream_t>, WorkArea> m;
  return m;
}
uint64_t g_tick = 0;
size_t g_plan_limit = 1024;

// Keep at most g_plan_limit plans; the least recently used one is destroyed
// after the device is idle (an in-flight transform may still use the plan).
// Only calls on a stream that is not capturing evict (the synchronisation would
// end a capture): nfx_fft_work_bytes and captured nfx_fft_ws calls let the cache
// run over its limit until the next such call.
void evict_if_full() {
  while (plans().size() >= g_plan_limit && !plans().empty()) {
    auto victim = plans().begin();
    for (auto it = plans().begin(); it != plans().end(); ++it)
      if (it->second.last_use < victim->second.last_use) victim = it;
    cudaDeviceSynchronize();
    cufftDestroy(victim->second.plan);
    plans().erase(victim);
  }
}

int cufft_fail(cufftResult r, const char* where) {
  set_error(std::string(where) + ": cuFFT error " + std::to_string((int)r));
  return NFX_ERR_CUFFT;
}

// The work area of (dev, stream), at least `bytes` long.  A smaller one is freed
// in stream order (its last user was a launch on the same stream).
int stream_work_area(int dev, cudaStream_t s, size_t bytes, void** out) {
  WorkArea& w = work_areas()[{dev, s}];
  if (w.bytes < bytes) {
    if (w.ptr != nullptr) cudaFreeAsync(w.ptr, s);
    w.ptr = nullptr;
    w.bytes = 0;
    cudaError_t e = cudaMallocAsync(&w.ptr, bytes, s);
    if (e != cudaSuccess) {
      w.ptr = nullptr;
      set_error(std::string("cuFFT work area: ") + cudaGetErrorString(e));
      return NFX_ERR_CUDA;
    }
    w.bytes = bytes;
  }
  *out = w.ptr;
  return NFX_OK;
}

// The cached plan of (current device, precision, nf, n_trans) and its work-area size.
// Call with g_plan_mu held.
int get_plan(int precision, int dim, const int nf[3], int n_trans, bool may_evict, cufftHandle* plan,
             size_t* work_bytes) {
  if ((precision != NFX_F32 && precision != NFX_F64) || dim < 1 || dim > 3 || nf == nullptr || n_trans < 1) {
    set_error("invalid nfx_fft arguments");
    return NFX_ERR_INVALID;
  }
  int n[3];
  long long dist = 1;
  for (int d = 0; d < dim; ++d) {
    if (nf[d] < 1) {
      set_error("nf < 1");
      return NFX_ERR_INVALID;
    }
    n[d] = nf[dim - 1 - d];  // slowest axis first for cuFFT
    dist *= nf[d];
  }
  int dev = 0;
  cudaGetDevice(&dev);
  PlanKey key(dev, precision, dim, nf[0], dim > 1 ? nf[1] : 1, dim > 2 ? nf[2] : 1, n_trans);
  auto it = plans().find(key);
  if (it != plans().end()) {
    *plan = it->second.plan;
    *work_bytes = it->second.work_bytes;
    it->second.last_use = ++g_tick;
    return NFX_OK;
  }
  if (may_evict) evict_if_full();
  cufftResult r = cufftCreate(plan);
  if (r != CUFFT_SUCCESS) return cufft_fail(r, "cufftCreate");
  r = cufftSetAutoAllocation(*plan, 0);
  if (r == CUFFT_SUCCESS)
    r = cufftMakePlanMany(*plan, dim, n, nullptr, 1, (int)dist, nullptr, 1, (int)dist,
                          precision == NFX_F32 ? CUFFT_C2C : CUFFT_Z2Z, n_trans, work_bytes);
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(*plan);
    return cufft_fail(r, "cufftMakePlanMany");
  }
  plans()[key] = PlanEntry{*plan, *work_bytes, ++g_tick};
  return NFX_OK;
}

int exec_plan(cufftHandle plan, int precision, void* data, int sign, void* work, cudaStream_t stream) {
  cufftResult r = cufftSetStream(plan, stream);
  if (r != CUFFT_SUCCESS) return cufft_fail(r, "cufftSetStream");
  if (work != nullptr) {
    r = cufftSetWorkArea(plan, work);
    if (r != CUFFT_SUCCESS) return cufft_fail(r, "cufftSetWorkArea");
  }
  const int dir = sign > 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
  if (precision == NFX_F32)
    r = cufftExecC2C(plan, (cufftComplex*)data, (cufftComplex*)data, dir);
  else
    r = cufftExecZ2Z(plan, (cufftDoubleComplex*)data, (cufftDoubleComplex*)data, dir);
  if (r != CUFFT_SUCCESS) return cufft_fail(r, "cufftExec");
  return NFX_OK;
}

int check_exec_args(void* data, int sign) {
  if (data == nullptr || (sign != 1 && sign != -1)) {
    set_error("invalid nfx_fft arguments");
    return NFX_ERR_INVALID;
  }
  return NFX_OK;
}
}  // namespace
}  // namespace nfx

using namespace nfx;

extern "C" {

int nfx_fft(int precision, int dim, const int nf[3], int n_trans, void* data, int sign, void* stream) {
  int st = check_exec_args(data, sign);
  if (st != NFX_OK) return st;
  // A captured launch would keep the stream's work area, which later calls on the
  // same stream handle reuse or replace: captures pass their own (nfx_fft_ws).
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing((cudaStream_t)stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    set_error("nfx_fft: stream is capturing; use nfx_fft_ws with a work area owned by the graph");
    return NFX_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_plan_mu);
  cufftHandle plan;
  size_t work_bytes = 0;
  st = get_plan(precision, dim, nf, n_trans, true, &plan, &work_bytes);
  if (st != NFX_OK) return st;
  void* work = nullptr;
  if (work_bytes > 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    st = stream_work_area(dev, (cudaStream_t)stream, work_bytes, &work);
    if (st != NFX_OK) return st;
  }
  return exec_plan(plan, precision, data, sign, work, (cudaStream_t)stream);
}

int nfx_fft_work_bytes(int precision, int dim, const int nf[3], int n_trans, size_t* bytes) {
  if (bytes == nullptr) {
    set_error("nfx_fft_work_bytes: bytes is NULL");
    return NFX_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_plan_mu);
  cufftHandle plan;
  return get_plan(precision, dim, nf, n_trans, false, &plan, bytes);
}

int nfx_fft_ws(int precision, int dim, const int nf[3], int n_trans, void* data, int sign, void* work,
               size_t work_bytes, void* stream) {
  int st = check_exec_args(data, sign);
  if (st != NFX_OK) return st;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  const bool capturing =
      cudaStreamIsCapturing((cudaStream_t)stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone;
  std::lock_guard<std::mutex> lk(g_plan_mu);
  cufftHandle plan;
  size_t need = 0;
  st = get_plan(precision, dim, nf, n_trans, !capturing, &plan, &need);
  if (st != NFX_OK) return st;
  if (need > 0 && (work == nullptr || work_bytes < need)) {
    set_error("nfx_fft_ws: work area of " + std::to_string(work_bytes) + " bytes, plan needs " +
              std::to_string(need));
    return NFX_ERR_WORKSPACE;
  }
  return exec_plan(plan, precision, data, sign, need > 0 ? work : nullptr, (cudaStream_t)stream);
}

int nfx_fft_cache_clear(void) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  if (!plans().empty() || !work_areas().empty()) cudaDeviceSynchronize();
  for (auto& kv : plans()) cufftDestroy(kv.second.plan);
  plans().clear();
  int cur = 0;
  cudaGetDevice(&cur);
  for (auto& kv : work_areas()) {
    if (kv.second.ptr == nullptr) continue;
    cudaSetDevice(kv.first.first);
    cudaDeviceSynchronize();
    cudaFree(kv.second.ptr);
  }
  cudaSetDevice(cur);
  work_areas().clear();
  return NFX_OK;
}

int nfx_fft_cache_limit(int max_plans) {
  if (max_plans < 1) {
    set_error("nfx_fft_cache_limit: need at least one plan");
    return NFX_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plan_limit = (size_t)max_plans;
  return NFX_OK;
}

}  // extern "C"
