// TANConverter and TANMixer on the GPU (the entry points tanb_converter_* and
// tanb_mixer_* of include/tanb.h).
//
// Host-pointer overloads reproduce the reference's CPU code bit for bit:
//   short -> float  out = in * (gain / 32767)            ConverterImpl.cpp:217-246
//   float -> short  while >= 8 samples remain: round half to even (cvtps2dq:
//                   NaN and |x| >= 2^31 give INT_MIN) and saturate, no clip
//                   report; the last n mod 8: truncate (cvttss2si), clamp,
//                   report clipping                      ConverterImpl.cpp:287-408
//   mix             out = in[0], out += in[c] in order   MixerImpl.cpp:226-250
// Device-pointer overloads reproduce the reference's OpenCL kernels:
//   float -> short  clamp to [-32768, 32767] reporting clipping, then truncate
//                   (NaN converts to 0)                  Converter.cl:97-120
//   mix             sum = 0, sum += in[c] in order       Mixer.cl:26-41
// Products and sums use explicit round-to-nearest intrinsics so that no
// multiply-add contraction changes a result. Host rows are staged in pinned
// memory that the kernels read and write in place (mapped host memory).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/tanb.h"
#include "tanb_host_pool.h"
#include "tanb_internal.h"

namespace tanb {
namespace {

constexpr int kMaxRows = 64;  // buffers per launch (pointers travel as kernel parameters)

struct RowTable {
  const void* in[kMaxRows];
  void* out[kMaxRows];
};

// cvtps2dq / cvttss2si: out-of-range and NaN convert to INT_MIN.
__device__ __forceinline__ int x86_cvt_rne(float f) {
  return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rn(f) : INT_MIN;
}
__device__ __forceinline__ int x86_cvt_trunc(float f) {
  return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : INT_MIN;
}

__global__ void s16_to_f32_kernel(RowTable t, size_t in_step, size_t out_step, size_t n, float scale) {
  const int16_t* in = static_cast<const int16_t*>(t.in[blockIdx.y]);
  float* out = static_cast<float*>(t.out[blockIdx.y]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i * out_step] = __fmul_rn((float)in[i * in_step], scale);
}

// mode 0: the CPU overload's positional rule; mode 1: the OpenCL kernel's rule.
__global__ void f32_to_s16_kernel(RowTable t, size_t in_step, size_t out_step, size_t n, float scale, int mode,
                                  int* clip) {
  const float* in = static_cast<const float*>(t.in[blockIdx.y]);
  int16_t* out = static_cast<int16_t*>(t.out[blockIdx.y]);
  const size_t n8 = n & ~size_t(7);
  bool c = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float f = __fmul_rn(in[i * in_step], scale);
    int v;
    if (mode == 0) {
      if (i < n8) {
        v = min(max(x86_cvt_rne(f), -32768), 32767);
      } else {
        v = x86_cvt_trunc(f);
        if (v > 32767) { v = 32767; c = true; }
        if (v < -32768) { v = -32768; c = true; }
      }
    } else {
      if (f > 32767.f) { f = 32767.f; c = true; }
      if (f < -32768.f) { f = -32768.f; c = true; }
      v = (f != f) ? 0 : __float2int_rz(f);
    }
    out[i * out_step] = (int16_t)v;
  }
  if (c) atomicOr(clip, 1);
}

template <class T>
__global__ void copy_kernel(RowTable t, size_t in_step, size_t out_step, size_t n) {
  const T* in = static_cast<const T*>(t.in[blockIdx.y]);
  T* out = static_cast<T*>(t.out[blockIdx.y]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i * out_step] = in[i * in_step];
}

// Adds rows t.in[0..rows) into out in order. first: out starts as row 0 (CPU
// rule) or as 0 (OpenCL rule) when this is the first chunk; otherwise out holds
// the running sum of the previous chunks.
__global__ void mix_kernel(RowTable t, int rows, float* out, size_t n, int first, int cpu_rule) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float s;
    int r0 = 0;
    if (!first) {
      s = out[i];
    } else if (cpu_rule) {
      s = static_cast<const float*>(t.in[0])[i];
      r0 = 1;
    } else {
      s = 0.f;
    }
    for (int r = r0; r < rows; ++r) s = __fadd_rn(s, static_cast<const float*>(t.in[r])[i]);
    out[i] = s;
  }
}

__global__ void mix_strided_kernel(const float* in, size_t stride, int channels, float* out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < channels; ++c) s = __fadd_rn(s, in[(size_t)c * stride + i]);
    out[i] = s;
  }
}

dim3 grid_for(size_t n, int rows) {
  const size_t blocks = std::min<size_t>((n + 255) / 256, 1184);
  return dim3((unsigned)std::max<size_t>(1, blocks), (unsigned)rows);
}

int32_t cfail(int32_t code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}

#define CV_CUDA(expr)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return tanb::cfail(e_ == cudaErrorMemoryAllocation ? TANB_OUT_OF_MEMORY : TANB_FAIL, \
                   "%s failed: %s", #expr, cudaGetErrorString(e_));                    \
  } while (0)

// Grow-only pinned buffer.
struct Pinned {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t reserve(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
};

}  // namespace
}  // namespace tanb

struct tanb_converter {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  cudaStream_t stream = nullptr;
  int* clip = nullptr;  // mapped pinned flag
  tanb::Pinned stage_in, stage_out;
};

struct tanb_mixer {
  tanb_context* ctx = nullptr;
  std::mutex mu;
  cudaStream_t stream = nullptr;
  size_t n = 0;
  int channels = 0;
  tanb::Pinned stage_in, stage_out;
};

namespace {

using tanb::RowTable;
using tanb::kMaxRows;

// Host overload of a conversion: stage spans of every row in pinned memory,
// convert with the kernel in place, scatter the compact outputs.
template <class Tin, class Tout, class Launch>
int32_t host_convert(tanb_converter* cv, const Tin* const* in, size_t in_step, size_t n, Tout* const* out,
                     size_t out_step, int count, Launch&& launch) {
  const size_t span = (n - 1) * in_step + 1;
  CV_CUDA(cv->stage_in.reserve((size_t)count * span * sizeof(Tin)));
  CV_CUDA(cv->stage_out.reserve((size_t)count * n * sizeof(Tout)));
  Tin* sin = static_cast<Tin*>(cv->stage_in.p);
  Tout* sout = static_cast<Tout*>(cv->stage_out.p);
  for (int r = 0; r < count; ++r) tanb::copy_for_device(sin + (size_t)r * span, in[r], span * sizeof(Tin));
  for (int r0 = 0; r0 < count; r0 += kMaxRows) {
    const int rows = std::min(kMaxRows, count - r0);
    RowTable t{};
    for (int r = 0; r < rows; ++r) {
      t.in[r] = sin + (size_t)(r0 + r) * span;
      t.out[r] = sout + (size_t)(r0 + r) * n;
    }
    CV_CUDA(launch(t, rows, in_step, (size_t)1));
  }
  CV_CUDA(cudaStreamSynchronize(cv->stream));
  for (int r = 0; r < count; ++r)
    for (size_t i = 0; i < n; ++i) out[r][i * out_step] = sout[(size_t)r * n + i];
  return TANB_OK;
}

int32_t check_conv_args(const void* in, const void* out, size_t n, float gain) {
  if (!in) return tanb::cfail(TANB_INVALID_ARG, "inputBuffer == NULL");
  if (!out) return tanb::cfail(TANB_INVALID_ARG, "outputBuffer == NULL");
  if (n == 0) return tanb::cfail(TANB_INVALID_ARG, "numOfSamplesToProcess <= 0");
  if (!(gain > 0)) return tanb::cfail(TANB_INVALID_ARG, "conversionGain <= 0");
  return TANB_OK;
}

int32_t s16_to_f32_host(tanb_converter* cv, const int16_t* const* in, size_t in_step, size_t n, float* const* out,
                        size_t out_step, float gain, int count) {
  const float scale = gain / 32767;  // rounded once, as the reference
  return host_convert(cv, in, in_step, n, out, out_step, count,
                      [&](const RowTable& t, int rows, size_t is, size_t os) {
                        tanb::s16_to_f32_kernel<<<tanb::grid_for(n, rows), 256, 0, cv->stream>>>(t, is, os, n,
                                                                                                  scale);
                        return cudaGetLastError();
                      });
}

int32_t f32_to_s16_host(tanb_converter* cv, const float* const* in, size_t in_step, size_t n, int16_t* const* out,
                        size_t out_step, float gain, int count, int32_t* clipped) {
  const float scale = 32767 * gain;
  *cv->clip = 0;
  int32_t r = host_convert(cv, in, in_step, n, out, out_step, count,
                           [&](const RowTable& t, int rows, size_t is, size_t os) {
                             tanb::f32_to_s16_kernel<<<tanb::grid_for(n, rows), 256, 0, cv->stream>>>(
                                 t, is, os, n, scale, 0, cv->clip);
                             return cudaGetLastError();
                           });
  if (r == TANB_OK && clipped) *clipped = *cv->clip ? 1 : 0;
  return r;
}

}  // namespace

extern "C" {

int32_t tanb_converter_create(tanb_context* ctx, tanb_converter** out) {
  if (!ctx || !out) return tanb::cfail(TANB_INVALID_POINTER, "null argument");
  *out = nullptr;
  tanb_converter* cv = new tanb_converter();
  cv->ctx = ctx;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cv->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&cv->clip), sizeof(int), cudaHostAllocMapped);
  if (e != cudaSuccess) {
    if (cv->stream) cudaStreamDestroy(cv->stream);
    delete cv;
    cudaGetLastError();
    return tanb::cfail(TANB_FAIL, "converter setup: %s", cudaGetErrorString(e));
  }
  *cv->clip = 0;
  *out = cv;
  return TANB_OK;
}

int32_t tanb_converter_release(tanb_converter* cv) {
  if (!cv) return TANB_OK;
  {
    std::lock_guard<std::mutex> lock(cv->mu);
    cudaSetDevice(cv->ctx->device);
    cudaStreamSynchronize(cv->stream);
    cv->stage_in.release();
    cv->stage_out.release();
    cudaFreeHost(cv->clip);
    cudaStreamDestroy(cv->stream);
  }
  delete cv;
  return TANB_OK;
}

int32_t tanb_converter_short_to_float(tanb_converter* cv, const int16_t* in, size_t in_step, size_t n, float* out,
                                      size_t out_step, float gain) {
  if (!cv) return tanb::cfail(TANB_INVALID_POINTER, "null converter");
  int32_t r = check_conv_args(in, out, n, gain);
  if (r != TANB_OK) return r;
  std::lock_guard<std::mutex> lock(cv->mu);
  CV_CUDA(cudaSetDevice(cv->ctx->device));
  return s16_to_f32_host(cv, &in, in_step, n, &out, out_step, gain, 1);
}

int32_t tanb_converter_float_to_short(tanb_converter* cv, const float* in, size_t in_step, size_t n, int16_t* out,
                                      size_t out_step, float gain, int32_t* clipped) {
  if (!cv) return tanb::cfail(TANB_INVALID_POINTER, "null converter");
  int32_t r = check_conv_args(in, out, n, gain);
  if (r != TANB_OK) return r;
  std::lock_guard<std::mutex> lock(cv->mu);
  CV_CUDA(cudaSetDevice(cv->ctx->device));
  return f32_to_s16_host(cv, &in, in_step, n, &out, out_step, gain, 1, clipped);
}

int32_t tanb_converter_short_to_float_batch(tanb_converter* cv, const int16_t* const* in, size_t in_step, size_t n,
                                            float* const* out, size_t out_step, float gain, int32_t count) {
  if (!cv) return tanb::cfail(TANB_INVALID_POINTER, "null converter");
  int32_t r = check_conv_args(in, out, n, gain);
  if (r != TANB_OK) return r;
  if (count <= 0) return TANB_OK;  // the reference's loop runs zero times
  for (int i = 0; i < count; ++i)
    if (!in[i] || !out[i]) return tanb::cfail(TANB_INVALID_ARG, "buffer %d == NULL", i);
  std::lock_guard<std::mutex> lock(cv->mu);
  CV_CUDA(cudaSetDevice(cv->ctx->device));
  return s16_to_f32_host(cv, in, in_step, n, out, out_step, gain, count);
}

int32_t tanb_converter_float_to_short_batch(tanb_converter* cv, const float* const* in, size_t in_step, size_t n,
                                            int16_t* const* out, size_t out_step, float gain, int32_t count,
                                            int32_t* clipped) {
  if (!cv) return tanb::cfail(TANB_INVALID_POINTER, "null converter");
  int32_t r = check_conv_args(in, out, n, gain);
  if (r != TANB_OK) return r;
  if (clipped) *clipped = 0;
  if (count <= 0) return TANB_OK;
  for (int i = 0; i < count; ++i)
    if (!in[i] || !out[i]) return tanb::cfail(TANB_INVALID_ARG, "buffer %d == NULL", i);
  std::lock_guard<std::mutex> lock(cv->mu);
  CV_CUDA(cudaSetDevice(cv->ctx->device));
  return f32_to_s16_host(cv, in, in_step, n, out, out_step, gain, count, clipped);
}

int32_t tanb_converter_convert_device(tanb_converter* cv, const void* const* in, size_t in_step,
                                      const size_t* in_offsets, int32_t in_type, void* const* out, size_t out_step,
                                      const size_t* out_offsets, int32_t out_type, size_t n, float gain,
                                      int32_t count, int32_t* clipped) {
  if (!cv) return tanb::cfail(TANB_INVALID_POINTER, "null converter");
  int32_t r = check_conv_args(in, out, n, gain);
  if (r != TANB_OK) return r;
  if (count <= 0) return tanb::cfail(TANB_INVALID_ARG, "count of conversions <= 0");
  if ((in_type != TANB_SAMPLE_TYPE_FLOAT && in_type != TANB_SAMPLE_TYPE_SHORT) ||
      (out_type != TANB_SAMPLE_TYPE_FLOAT && out_type != TANB_SAMPLE_TYPE_SHORT))
    return tanb::cfail(TANB_NOT_IMPLEMENTED, "Argument types not supported for conversion");
  for (int i = 0; i < count; ++i)
    if (!in[i] || !out[i]) return tanb::cfail(TANB_INVALID_ARG, "buffer %d == NULL", i);
  std::lock_guard<std::mutex> lock(cv->mu);
  CV_CUDA(cudaSetDevice(cv->ctx->device));
  const size_t isz = in_type == TANB_SAMPLE_TYPE_FLOAT ? 4 : 2, osz = out_type == TANB_SAMPLE_TYPE_FLOAT ? 4 : 2;
  const bool to_short = in_type == TANB_SAMPLE_TYPE_FLOAT && out_type == TANB_SAMPLE_TYPE_SHORT;
  if (to_short && clipped) {
    CV_CUDA(cudaStreamSynchronize(cv->stream));  // the flag of an earlier call may still be written
    *cv->clip = 0;
  }
  for (int r0 = 0; r0 < count; r0 += kMaxRows) {
    const int rows = std::min(kMaxRows, count - r0);
    RowTable t{};
    for (int j = 0; j < rows; ++j) {
      t.in[j] = static_cast<const char*>(in[r0 + j]) + (in_offsets ? in_offsets[r0 + j] : 0) * isz;
      t.out[j] = static_cast<char*>(out[r0 + j]) + (out_offsets ? out_offsets[r0 + j] : 0) * osz;
    }
    const dim3 g = tanb::grid_for(n, rows);
    if (to_short) {
      tanb::f32_to_s16_kernel<<<g, 256, 0, cv->stream>>>(t, in_step, out_step, n, 32767 * gain, 1, cv->clip);
    } else if (in_type == TANB_SAMPLE_TYPE_SHORT && out_type == TANB_SAMPLE_TYPE_FLOAT) {
      tanb::s16_to_f32_kernel<<<g, 256, 0, cv->stream>>>(t, in_step, out_step, n, gain / 32767);
    } else if (in_type == TANB_SAMPLE_TYPE_FLOAT) {
      tanb::copy_kernel<float><<<g, 256, 0, cv->stream>>>(t, in_step, out_step, n);
    } else {
      tanb::copy_kernel<int16_t><<<g, 256, 0, cv->stream>>>(t, in_step, out_step, n);
    }
    CV_CUDA(cudaGetLastError());
  }
  // the reference reads the overflow flag back (blocking) only when asked for it
  if (to_short && clipped) {
    CV_CUDA(cudaStreamSynchronize(cv->stream));
    *clipped = *cv->clip ? 1 : 0;
  }
  return TANB_OK;
}

int32_t tanb_converter_synchronize(tanb_converter* cv) {
  if (!cv) return tanb::cfail(TANB_INVALID_POINTER, "null converter");
  std::lock_guard<std::mutex> lock(cv->mu);
  CV_CUDA(cudaSetDevice(cv->ctx->device));
  CV_CUDA(cudaStreamSynchronize(cv->stream));
  return TANB_OK;
}

void* tanb_converter_stream(tanb_converter* cv) { return cv ? (void*)cv->stream : nullptr; }

int32_t tanb_mixer_create(tanb_context* ctx, size_t buffer_size, int32_t channels, tanb_mixer** out) {
  if (!ctx || !out) return tanb::cfail(TANB_INVALID_POINTER, "null argument");
  *out = nullptr;
  if (buffer_size == 0 || channels <= 0) return tanb::cfail(TANB_INVALID_ARG, "buffer_size and channels must be > 0");
  tanb_mixer* m = new tanb_mixer();
  m->ctx = ctx;
  m->n = buffer_size;
  m->channels = channels;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete m;
    cudaGetLastError();
    return tanb::cfail(TANB_FAIL, "mixer setup: %s", cudaGetErrorString(e));
  }
  *out = m;
  return TANB_OK;
}

int32_t tanb_mixer_release(tanb_mixer* m) {
  if (!m) return TANB_OK;
  {
    std::lock_guard<std::mutex> lock(m->mu);
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->stream);
    m->stage_in.release();
    m->stage_out.release();
    cudaStreamDestroy(m->stream);
  }
  delete m;
  return TANB_OK;
}

namespace {

cudaError_t mix_rows(tanb_mixer* m, const float* const* rows, float* out, int cpu_rule) {
  for (int r0 = 0; r0 < m->channels; r0 += kMaxRows) {
    const int k = std::min(kMaxRows, m->channels - r0);
    RowTable t{};
    for (int j = 0; j < k; ++j) t.in[j] = rows[r0 + j];
    tanb::mix_kernel<<<tanb::grid_for(m->n, 1), 256, 0, m->stream>>>(t, k, out, m->n, r0 == 0, cpu_rule);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

int32_t tanb_mixer_mix(tanb_mixer* m, const float* const* in, float* out) {
  if (!m) return tanb::cfail(TANB_INVALID_POINTER, "null mixer");
  if (!in || !out) return tanb::cfail(TANB_INVALID_ARG, "null buffer");
  for (int c = 0; c < m->channels; ++c)
    if (!in[c]) return tanb::cfail(TANB_INVALID_ARG, "ppBufferInput[%d] == NULL", c);
  std::lock_guard<std::mutex> lock(m->mu);
  CV_CUDA(cudaSetDevice(m->ctx->device));
  const size_t n = m->n, C = (size_t)m->channels;
  CV_CUDA(m->stage_in.reserve(C * n * sizeof(float)));
  CV_CUDA(m->stage_out.reserve(n * sizeof(float)));
  float* sin = static_cast<float*>(m->stage_in.p);
  float* sout = static_cast<float*>(m->stage_out.p);
  std::vector<const float*> rows(C);
  for (size_t c = 0; c < C; ++c) {
    tanb::copy_for_device(sin + c * n, in[c], n * sizeof(float));
    rows[c] = sin + c * n;
  }
  CV_CUDA(mix_rows(m, rows.data(), sout, 1));
  CV_CUDA(cudaStreamSynchronize(m->stream));
  std::memcpy(out, sout, n * sizeof(float));
  return TANB_OK;
}

int32_t tanb_mixer_mix_device(tanb_mixer* m, const float* const* in, float* out) {
  if (!m) return tanb::cfail(TANB_INVALID_POINTER, "null mixer");
  if (!in || !out) return tanb::cfail(TANB_INVALID_ARG, "null buffer");
  for (int c = 0; c < m->channels; ++c)
    if (!in[c]) return tanb::cfail(TANB_INVALID_ARG, "pBufferInput[%d] == NULL", c);
  std::lock_guard<std::mutex> lock(m->mu);
  CV_CUDA(cudaSetDevice(m->ctx->device));
  CV_CUDA(mix_rows(m, in, out, 0));
  return TANB_OK;
}

int32_t tanb_mixer_mix_device_strided(tanb_mixer* m, const float* in, float* out, size_t input_stride) {
  if (!m) return tanb::cfail(TANB_INVALID_POINTER, "null mixer");
  if (!in || !out) return tanb::cfail(TANB_INVALID_ARG, "null buffer");
  std::lock_guard<std::mutex> lock(m->mu);
  CV_CUDA(cudaSetDevice(m->ctx->device));
  tanb::mix_strided_kernel<<<tanb::grid_for(m->n, 1), 256, 0, m->stream>>>(in, input_stride, m->channels, out, m->n);
  CV_CUDA(cudaGetLastError());
  return TANB_OK;
}

int32_t tanb_mixer_synchronize(tanb_mixer* m) {
  if (!m) return tanb::cfail(TANB_INVALID_POINTER, "null mixer");
  std::lock_guard<std::mutex> lock(m->mu);
  CV_CUDA(cudaSetDevice(m->ctx->device));
  CV_CUDA(cudaStreamSynchronize(m->stream));
  return TANB_OK;
}

void* tanb_mixer_stream(tanb_mixer* m) { return m ? (void*)m->stream : nullptr; }

}  // extern "C"
