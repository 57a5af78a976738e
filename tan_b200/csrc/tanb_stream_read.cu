// tanb_stream_read: a plain streaming read of a device buffer, the floor that
// one bandwidth-bound launch of a given size reaches on this GPU. The bench
// times it over the same byte count as the partition MAC it reports, so that
// the MAC's launch can be compared with the best a launch of that size does
// (at tens of MB a single launch is bounded by its fixed start and drain cost,
// not by the HBM rate).
//
// Every thread sums four independent 16-byte loads per iteration (streaming
// hint: the data is read once), the CTA reduces in shared memory and adds its
// sum to *out with one atomic, so the loads cannot be optimised away.
#include <cuda_runtime.h>

#include "../../include/tanb.h"
#include "tanb_internal.h"

namespace {

__global__ void __launch_bounds__(1024) stream_read_kernel(const float4* __restrict__ p, size_t n4,
                                                           float* __restrict__ out) {
  __shared__ float red[32];
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float acc = 0.f;
  for (; i + 3 * stride < n4; i += 4 * stride) {
    const float4 a = __ldcs(p + i), b = __ldcs(p + i + stride), c = __ldcs(p + i + 2 * stride),
                 d = __ldcs(p + i + 3 * stride);
    acc += (a.x + a.y + a.z + a.w) + (b.x + b.y + b.z + b.w) + (c.x + c.y + c.z + c.w) + (d.x + d.y + d.z + d.w);
  }
  for (; i < n4; i += stride) {
    const float4 a = __ldcs(p + i);
    acc += a.x + a.y + a.z + a.w;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) atomicAdd(out, acc);
  }
}

}  // namespace

extern "C" int32_t tanb_stream_read(const void* src, size_t bytes, float* out, uint32_t ctas_per_sm,
                                    uint32_t threads, void* stream) {
  if (!src || !out) {
    tanb::set_last_error("tanb_stream_read: null pointer");
    return TANB_INVALID_POINTER;
  }
  if ((reinterpret_cast<uintptr_t>(src) & 15) || bytes % 16 || ctas_per_sm == 0 || ctas_per_sm > 32 ||
      threads < 32 || threads > 1024 || threads % 32) {
    tanb::set_last_error("tanb_stream_read: src and bytes must be 16-byte multiples, ctas_per_sm in [1, 32], "
                         "threads a multiple of 32 in [32, 1024]");
    return TANB_INVALID_ARG;
  }
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) {
    stream_read_kernel<<<(unsigned)sms * ctas_per_sm, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const float4*>(src), bytes / 16, out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    tanb::set_last_error(cudaGetErrorString(e));
    return TANB_FAIL;
  }
  return TANB_OK;
}
