// Pack step of the slab exchange between ranks: the values a peer needs are gathered by index from this rank's
// state array into a contiguous send buffer (the pick of utils/face_connector.go:143-187), which the host then
// sends; the receiver's halo is the place step, read by the stage through its gather map.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "dgk.h"
#include "runner.hpp"

namespace dgk {
namespace {

template <typename T>
__global__ void gather_values_kernel(const T *__restrict__ src, int64_t src_count, const int64_t *__restrict__ idx,
                                     int64_t n, T *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = idx[i];
    dst[i] = (j >= 0 && j < src_count) ? src[j] : T(0);
  }
}

}  // namespace
}  // namespace dgk

extern "C" int dgk_gather_values(const void *src, int32_t dtype, int64_t src_count, const int64_t *idx, int64_t n,
                                 void *dst, void *cuda_stream) {
  try {
    if (n < 0 || (n > 0 && (!src || !idx || !dst))) throw dgk::Error(DGK_ERR_INVALID, "gather: null pointer or n < 0");
    if (n == 0) return DGK_OK;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((n + threads - 1) / threads, 148 * 16);
    if (dtype == DGK_FLOAT64)
      dgk::gather_values_kernel<double><<<blocks, threads, 0, st>>>(static_cast<const double *>(src), src_count, idx, n,
                                                                    static_cast<double *>(dst));
    else if (dtype == DGK_FLOAT32)
      dgk::gather_values_kernel<float><<<blocks, threads, 0, st>>>(static_cast<const float *>(src), src_count, idx, n,
                                                                   static_cast<float *>(dst));
    else
      throw dgk::Error(DGK_ERR_UNSUPPORTED, "gather: dtype must be float32 or float64");
    dgk::cuda_check(cudaGetLastError(), "gather_values_kernel launch");
    return DGK_OK;
  } catch (const dgk::Error &e) {
    dgk::set_global_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    dgk::set_global_error(e.what());
    return DGK_ERR_INVALID;
  }
}
