// Instantiates the 1D spread / interp / gradient kernels for float (one
// translation unit per precision and dimension so they compile in parallel).
#include "nfx_spreadinterp.cuh"

namespace nfx {
template cudaError_t dispatch_spread<float, 1>(int, const PointArgs<float>&, const void*, void*, cudaStream_t);
template cudaError_t dispatch_interp<float, 1>(int, const PointArgs<float>&, const void*, void*, cudaStream_t);
template cudaError_t dispatch_grad<float, 1>(int, const PointArgs<float>&, const void*, const void*, void*, void*,
                                               void*, void*, cudaStream_t);
template cudaError_t dispatch_batch<float, 1>(int, bool, const void*, int, const int*, int64_t, size_t,
                                             cudaStream_t);
}  // namespace nfx
