// Instantiates the 3D spread / interp / gradient kernels for double (one
// translation unit per precision and dimension so they compile in parallel).
#include "nfx_spreadinterp.cuh"

namespace nfx {
template cudaError_t dispatch_spread<double, 3>(int, const PointArgs<double>&, const void*, void*, cudaStream_t);
template cudaError_t dispatch_interp<double, 3>(int, const PointArgs<double>&, const void*, void*, cudaStream_t);
template cudaError_t dispatch_grad<double, 3>(int, const PointArgs<double>&, const void*, const void*, void*, void*,
                                               void*, void*, cudaStream_t);
template cudaError_t dispatch_batch<double, 3>(int, bool, const void*, int, const int*, int64_t, size_t,
                                             cudaStream_t);
}  // namespace nfx
